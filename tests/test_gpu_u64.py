"""The 64-bit word variant (include/ntt_b200_u64.h) on the GPU, bit-exact
against the 64-bit oracle (the reference's CPU butterfly loops restated with
128-bit products, itself checked against the O(N^2) definition on CPU).
Needs a B200."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rand64(T, seed, polys=1):
    rng = np.random.default_rng(seed)
    return np.stack([np.stack([rng.integers(0, int(q), 1 << T.logN, dtype=np.uint64) for q in T.q])
                     for _ in range(polys)])


def dev64(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def host64(t):
    return t.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("logN,limbs,polys,start", [
    (1, 2, 1, 1 << 59), (5, 3, 2, 1 << 60), (12, 4, 3, (1 << 61) + 7),
    (13, 2, 2, 1 << 59), (16, 3, 2, 1 << 61), (17, 2, 1, 3 << 60)] + [
    # every other compiled launch shape (whole limbs up to 2^12, then the
    # column and row launches of 2^13..2^17), one limb near 2^61
    (n, 1, 2, (1 << 61) + 3 * n) for n in (2, 3, 4, 6, 7, 8, 9, 10, 11, 14, 15)])
def test_u64_bit_exact(torch_cuda, logN, limbs, polys, start):
    torch = torch_cuda
    import ntt_b200 as nb
    mods = [tuple(m) for m in nb.find_moduli64(logN, limbs, start)]
    T = O.LimbTables64(logN, mods)
    x = rand64(T, logN * 11 + limbs, polys)
    x[0, 0, :2] = [T.q[0] - 1, 0]  # the largest canonical word and zero
    d = dev64(torch, x)
    with nb.Plan64(logN, mods) as p:
        p.forward_many(d, polys)
        torch.cuda.synchronize()
        got = host64(d).reshape(x.shape)
        for k in range(polys):
            assert np.array_equal(got[k], T.to_mont(T.forward(x[k]))), (logN, k)
        p.inverse_many(d, polys)
        torch.cuda.synchronize()
        assert np.array_equal(host64(d).reshape(x.shape), x)


def test_u64_strided_batch(torch_cuda):
    """Polynomials poly_stride words apart: the gap is left untouched."""
    torch = torch_cuda
    import ntt_b200 as nb
    logN, limbs, polys = 14, 2, 3
    mods = [tuple(m) for m in nb.find_moduli64(logN, limbs, 1 << 60)]
    T = O.LimbTables64(logN, mods)
    N = 1 << logN
    stride = limbs * N + 64
    x = rand64(T, 5, polys)
    buf = np.full(polys * stride, 0x5A5A5A5A5A5A5A5A, dtype=np.uint64)
    for k in range(polys):
        buf[k * stride:k * stride + limbs * N] = x[k].reshape(-1)
    d = dev64(torch, buf)
    with nb.Plan64(logN, mods) as p:
        p.forward_many(d, polys, stride)
        torch.cuda.synchronize()
        got = host64(d)
        for k in range(polys):
            assert np.array_equal(got[k * stride:k * stride + limbs * N].reshape(limbs, N),
                                  T.to_mont(T.forward(x[k])))
            assert (got[k * stride + limbs * N:(k + 1) * stride] == 0x5A5A5A5A5A5A5A5A).all()
        p.inverse_many(d, polys, stride)
        torch.cuda.synchronize()
        assert np.array_equal(host64(d), buf)


def test_u64_errors(torch_cuda):
    torch = torch_cuda
    import ntt_b200 as nb
    mods = [tuple(m) for m in nb.find_moduli64(12, 1, 1 << 60)]
    with nb.Plan64(12, mods) as p:
        x = torch.zeros(2 * (1 << 12) + 2, dtype=torch.int64, device="cuda")
        with pytest.raises(nb.NttError) as e:
            p.forward_many(x[1:], 1)  # 8-byte, not 16-byte, aligned
        assert e.value.name == "NTT_ERR_MISALIGNED"
        with pytest.raises(nb.NttError) as e:
            p.forward_many(x, 2, 100)  # stride below limbs * N
        assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"
