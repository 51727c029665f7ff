"""The warp-per-limb kernel of logN 6..9 (warp.cu: the limb in registers, the
last five stages pairing lanes through shfl.xor) against the oracle and
against the shared-memory kernel it replaces (small.cu), with the scale, the
limb map and the subtract-and-scale output.  Needs a B200.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def to_dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda().reshape(-1)


def to_host(t, shape):
    return t.cpu().numpy().view(np.uint32).reshape(shape)


@pytest.mark.parametrize("logN", [6, 7, 8, 9])
@pytest.mark.parametrize("bits", [30, 31])
def test_warp_kernel_matches_oracle_and_shared(torch_cuda, logN, bits):
    torch = torch_cuda
    import ntt_b200 as nb
    limbs, polys = 5, 3
    mods = O.ascending_primes(logN, limbs, int(2 ** 29.5) if bits == 30 else int(2 ** 30.5))
    T = O.LimbTables(logN, mods)
    xs = np.stack([O.uniform_limbs(logN, T.q, 9 * p + logN) for p in range(polys)])
    xs[0, 1, :3] = [0, T.q[1] - 1, 0xFFFFFFFF]
    F = np.stack([T.forward_mont(x) for x in xs])
    with nb.Plan(logN, mods) as warp, nb.Plan(logN, mods) as shared:
        shared.set_small_kernel(nb.SMALL_SHARED)
        outs = []
        for p in (warp, shared):
            d = to_dev(torch, xs)
            p.forward_many(d, polys)
            torch.cuda.synchronize()
            got = to_host(d, xs.shape)
            assert np.array_equal(got, F)
            p.inverse_many(d, polys)
            torch.cuda.synchronize()
            outs.append(to_host(d, xs.shape))
        want = xs.copy()
        want[0, 1, 2] = 0xFFFFFFFF % T.q[1]
        assert np.array_equal(outs[0], want) and np.array_equal(outs[1], want)
        # scaled forward, limb map and the subtract-and-scale output agree too
        rng = np.random.default_rng(logN)
        c = np.array([int(rng.integers(0, q)) for q in T.q], dtype=np.uint32)
        sub = np.stack([O.uniform_limbs(logN, T.q[1:4], 70 + p) for p in range(polys)])
        res = []
        for p in (warp, shared):
            a = to_dev(torch, xs)
            p.forward_sub_scale(a, to_dev(torch, sub), 1, 4, to_dev(torch, c), None, polys)
            b = to_dev(torch, xs)
            p.forward_skip(b, 2, 4, polys)
            torch.cuda.synchronize()
            res.append((to_host(a, xs.shape), to_host(b, xs.shape)))
        assert np.array_equal(res[0][0], res[1][0])
        assert np.array_equal(res[0][1], res[1][1])
        skip_want = F.copy()
        skip_want[:, 2:4] = xs[:, 2:4]
        assert np.array_equal(res[0][1], skip_want)


def test_small_kernel_knob(torch_cuda):
    import ntt_b200 as nb
    with nb.Plan(8, O.ascending_primes(8, 1, int(2 ** 29.5))) as p:
        with pytest.raises(nb.NttError) as e:
            p.set_small_kernel(7)
        assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"
