"""Plans with compressed twiddle tables (NTT_PLAN_COMPRESSED_TWIDDLES; needs a
B200).

The reference's Cheddar handler can take the twiddles of its last stage as a
product of an MSB and an LSB table (OF-Twiddle, src/NTT_cheddar.cu:42-43,
80-84, 1283-1289).  Here the last four stages keep one base entry per run of
consecutive entries plus 16 unit-step factors (3N/16 + 16 pairs per limb
instead of N).  Checks: the device tables equal the layout rebuilt from the
oracle's tables (tests/twiddle_ref.py), and every transform a compressed plan
runs is bit-exact against the oracle (and so against a full-table plan).
"""
import numpy as np
import pytest

from oracle import oracle as O
from twiddle_ref import compressed_tables

pytestmark = pytest.mark.gpu


def plan_moduli(logN, limbs, bits):
    start = {"baseline": 974258177, 30: int(2 ** 29.5), 31: int(2 ** 30.5)}[bits]
    return O.ascending_primes(logN, limbs, start)


def to_dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda().reshape(-1)


def to_host(t, shape):
    return t.cpu().numpy().view(np.uint32).reshape(shape)


def read_device(torch, ptr, words):
    import ctypes
    torch.cuda.synchronize()
    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    out = np.empty(words, dtype=np.uint32)
    assert rt.cudaMemcpy(out.ctypes.data, ptr, words * 4, 2) == 0
    return out


@pytest.mark.parametrize("logN", [15, 16, 17])
def test_compressed_device_tables(torch_cuda, logN):
    torch = torch_cuda
    import ntt_b200 as nb
    mods = plan_moduli(logN, 2, 30) + plan_moduli(logN, 2, 31)
    T = O.LimbTables(logN, mods)
    ef, ei = compressed_tables(T)
    E = 3 * (1 << logN) // 16 + 16
    with nb.Plan(logN, mods, compressed_twiddles=True) as p:
        info = p.info
        assert info.twiddle_entries == E
        with nb.Plan(logN, mods) as full:
            assert full.info.twiddle_entries == 1 << logN
            assert info.device_bytes < full.info.device_bytes / 5
        f, i, _ = p.tables()
        assert np.array_equal(read_device(torch, f, 4 * E * 2).reshape(4, E, 2), ef)
        assert np.array_equal(read_device(torch, i, 4 * E * 2).reshape(4, E, 2), ei)


@pytest.mark.parametrize("logN,limbs,bits,polys", [
    (16, 16, "baseline", 3), (16, 5, 31, 2), (15, 4, 30, 3), (15, 3, 31, 1),
    (17, 3, 30, 2), (17, 2, 31, 1)])
def test_compressed_transforms_match_oracle(torch_cuda, logN, limbs, bits, polys):
    torch = torch_cuda
    import ntt_b200 as nb
    mods = plan_moduli(logN, limbs, bits)
    T = O.LimbTables(logN, mods)
    N = 1 << logN
    stride = limbs * N + 8  # a gap between polynomials, left untouched
    xs = [O.uniform_limbs(logN, T.q, 40 + p) for p in range(polys)]
    xs[0][0, :3] = [0, T.q[0] - 1, 0xFFFFFFFF]
    buf = np.full(polys * stride, 0xA5A5A5A5, dtype=np.uint32)
    for p in range(polys):
        buf[p * stride:p * stride + limbs * N] = xs[p].reshape(-1)
    with nb.Plan(logN, mods, compressed_twiddles=True) as plan:
        d = to_dev(torch, buf)
        plan.forward_many(d, polys, stride)
        torch.cuda.synchronize()
        got = to_host(d, buf.shape)
        for p in range(polys):
            seg = got[p * stride:p * stride + limbs * N].reshape(limbs, N)
            assert np.array_equal(seg, T.forward_mont(xs[p])), p
            assert (got[p * stride + limbs * N:(p + 1) * stride] == 0xA5A5A5A5).all()
        plan.inverse_many(d, polys, stride)
        torch.cuda.synchronize()
        got = to_host(d, buf.shape)
        want = buf.copy()
        want[2] = 0xFFFFFFFF % T.q[0]
        assert np.array_equal(got, want)
        # single-polynomial calls run the single-polynomial configuration
        d1 = to_dev(torch, xs[-1])
        plan.forward(d1)
        torch.cuda.synchronize()
        assert np.array_equal(to_host(d1, xs[-1].shape), T.forward_mont(xs[-1]))
        plan.inverse(d1)
        torch.cuda.synchronize()
        want1 = xs[-1] % T.q[:, None]  # the planted 0xFFFFFFFF (polys == 1) comes back reduced
        assert np.array_equal(to_host(d1, xs[-1].shape), want1)


def test_compressed_scaled_skip_and_range(torch_cuda):
    torch = torch_cuda
    import ntt_b200 as nb
    logN, limbs = 16, 6
    mods = plan_moduli(logN, limbs, 31)
    T = O.LimbTables(logN, mods)
    rng = np.random.default_rng(8)
    c = np.array([int(rng.integers(1, q)) for q in T.q], dtype=np.uint32)
    q64 = T.q.astype(np.uint64)[:, None]
    x = O.uniform_limbs(logN, T.q, 77)
    cx = ((x.astype(np.uint64) * c.astype(np.uint64)[:, None]) % q64).astype(np.uint32)
    with nb.Plan(logN, mods, compressed_twiddles=True) as plan:
        d = to_dev(torch, x)
        plan.forward_scaled(d, to_dev(torch, c))
        torch.cuda.synchronize()
        F = T.forward_mont(cx)
        assert np.array_equal(to_host(d, x.shape), F)
        # scaled inverse on limbs [2, 5): c_k * INTT on those, the rest stays
        plan.inverse_scaled_range(d, 2, 5, to_dev(torch, c[2:5]))
        torch.cuda.synchronize()
        want = F.copy()
        want[2:5] = ((cx[2:5].astype(np.uint64) * c[2:5].astype(np.uint64)[:, None])
                     % q64[2:5]).astype(np.uint32)
        assert np.array_equal(to_host(d, x.shape), want)
        d = to_dev(torch, x)
        plan.forward_skip(d, 1, 3)
        torch.cuda.synchronize()
        want = T.forward_mont(x)
        want[1:3] = x[1:3]
        assert np.array_equal(to_host(d, x.shape), want)


def test_compressed_refusals(torch_cuda):
    torch = torch_cuda
    import ntt_b200 as nb
    with pytest.raises(nb.NttError) as e:
        nb.Plan(14, plan_moduli(14, 2, 30), compressed_twiddles=True)
    assert e.value.name == "NTT_ERR_UNSUPPORTED"
    logN, limbs = 16, 2
    mods = plan_moduli(logN, limbs, 30)
    with nb.Plan(logN, mods, compressed_twiddles=True) as plan:
        a = torch.zeros(limbs << logN, dtype=torch.int32, device="cuda")
        b = torch.zeros(limbs << logN, dtype=torch.int32, device="cuda")
        with pytest.raises(nb.NttError) as e:
            plan.multiply_many(a, b, 1)
        assert e.value.name == "NTT_ERR_UNSUPPORTED"
        with pytest.raises(nb.NttError) as e:
            plan.forward_sub_scale(a, b, 0, 1)
        assert e.value.name == "NTT_ERR_UNSUPPORTED"
        # a cluster configuration cannot be pinned on a compressed plan
        cluster = [i for i, c in enumerate(nb.kernel_configs())
                   if c.logN == logN and c.exchange == 0]
        with pytest.raises(nb.NttError) as e:
            plan.force_config(cluster[0], cluster[0])
        assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"
