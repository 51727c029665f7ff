"""Transforms with a per-limb constant folded into stage 0 (needs a B200).

ntt_forward_scaled computes NTT(c_l * x) and ntt_inverse_scaled c_l * INTT(x)
per limb l, as Cheddar's NTTHandler does inside its kernels (the NTTPhase1
pre-multiply, src/NTT_cheddar.cu:286-293; INTTAndMultConst,
src/NTT_cheddar.cu:743-813).  Oracle: the CPU transforms of the reference
(cpu_ntt_butterfly / cpu_intt_butterfly) with the product by c_l mod q_l
taken on the CPU.  Bit-exact.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def scale_mod(x, c, q):
    return ((x.astype(np.uint64) * c.astype(np.uint64)[:, None]) % q.astype(np.uint64)[:, None]
            ).astype(np.uint32)


@pytest.mark.parametrize("logN,limbs,bits,polys", [(16, 16, "baseline", 3), (12, 5, 31, 2),
                                                  (17, 3, 30, 1), (8, 4, 30, 2), (14, 2, 31, 1)])
def test_scaled_transforms_match_oracle(torch_cuda, logN, limbs, bits, polys):
    torch = torch_cuda
    import ntt_b200 as nb
    start = {"baseline": 974258177, 30: int(2 ** 29.5), 31: int(2 ** 30.5)}[bits]
    mods = O.ascending_primes(logN, limbs, start)
    T = O.LimbTables(logN, mods)
    rng = np.random.default_rng(logN * 7 + limbs)
    c = np.array([int(rng.integers(0, q)) for q in T.q], dtype=np.uint32)
    c[0] = 0 if limbs > 2 else c[0]  # zero is a constant too
    xs = [O.uniform_limbs(logN, T.q, 100 + p) for p in range(polys)]
    with nb.Plan(logN, mods) as plan:
        d = torch.from_numpy(np.stack(xs).view(np.int32)).cuda().reshape(-1)
        s = torch.from_numpy(c.view(np.int32)).cuda()
        plan.forward_scaled(d, s, polys)
        torch.cuda.synchronize()
        got = d.cpu().numpy().view(np.uint32).reshape(polys, limbs, -1)
        for p in range(polys):
            assert np.array_equal(got[p], T.forward_mont(scale_mod(xs[p], c, T.q))), p
        # inverse of the spectra, scaled: c * INTT(NTT(c x)) = c^2 x
        plan.inverse_scaled(d, s, polys)
        torch.cuda.synchronize()
        got = d.cpu().numpy().view(np.uint32).reshape(polys, limbs, -1)
        for p in range(polys):
            assert np.array_equal(got[p], scale_mod(scale_mod(xs[p], c, T.q), c, T.q)), p
        # the unscaled entry points on the same plan are unaffected
        x = xs[0]
        d1 = torch.from_numpy(x.view(np.int32)).cuda()
        plan.forward(d1)
        plan.inverse(d1)
        torch.cuda.synchronize()
        assert np.array_equal(d1.cpu().numpy().view(np.uint32), x)


def test_scaled_inverse_of_plain_forward(torch_cuda):
    torch = torch_cuda
    import ntt_b200 as nb
    mods = O.ascending_primes(16, 4, int(2 ** 29.5))
    T = O.LimbTables(16, mods)
    x = O.uniform_limbs(16, T.q, 9)
    c = np.array([3, 1, int(T.q[2]) - 1, 123456789 % int(T.q[3])], dtype=np.uint32)
    with nb.Plan(16, mods) as plan:
        d = torch.from_numpy(x.view(np.int32)).cuda()
        s = torch.from_numpy(c.view(np.int32)).cuda()
        plan.forward(d)
        plan.inverse_scaled(d, s)
        torch.cuda.synchronize()
        assert np.array_equal(d.cpu().numpy().view(np.uint32), scale_mod(x, c, T.q))


def test_scaled_needs_a_scale_array(torch_cuda):
    import ntt_b200 as nb
    mods = O.ascending_primes(12, 1, int(2 ** 29.5))
    with nb.Plan(12, mods) as plan:
        r = nb._lib.ntt_forward_scaled(plan._h, None, 1, 0, None, None)
        assert nb.STATUS_NAMES[r] == "NTT_ERR_INVALID_ARGUMENT"
