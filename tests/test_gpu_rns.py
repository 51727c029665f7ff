"""The NTT steps of RNS basis conversion (needs a B200): ModUp's forward over
all limbs but a skipped range, ModDown's forward with the subtract-and-scale
output, and the scaled inverse on a limb range.

References: Cheddar's NTTForModUp (src/NTT_cheddar.cu:886-955),
NTTForModDown with NTTPhase2ForModDown (src/NTT_cheddar.cu:456-601,
957-1027) and INTTForModDown (src/NTT_cheddar.cu:1029-1128).  Oracle: the
reference's CPU transforms (cpu_ntt_butterfly / cpu_intt_butterfly, in
Montgomery form where the GPU forward's output is), with the subtraction and
the constant products taken mod q on the CPU.  Bit-exact.  Sizes cover the
three kernel families: logN 8 (single-CTA kernel), 12 (cluster kernel) and
16 (split kernel, the default at logN 15..17).
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = [(8, 5, 30, 2), (12, 6, 31, 3), (16, 6, "baseline", 2), (16, 4, 31, 1),
         (14, 3, 30, 2), (17, 3, 31, 1)]


def plan_moduli(logN, limbs, bits):
    start = {"baseline": 974258177, 30: int(2 ** 29.5), 31: int(2 ** 30.5)}[bits]
    return O.ascending_primes(logN, limbs, start)


def u64(x):
    return np.asarray(x).astype(np.uint64)


def sub_scale_expect(F, s, c, d, q):
    """(F - d s) c mod q per limb; F, s: [limbs, N]; c, d, q: [limbs]."""
    q = u64(q)[:, None]
    ds = (u64(s) * u64(d)[:, None]) % q
    t = (u64(F) + q - ds) % q
    return ((t * u64(c)[:, None]) % q).astype(np.uint32)


def to_dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda().reshape(-1)


def to_host(t, shape):
    return t.cpu().numpy().view(np.uint32).reshape(shape)


@pytest.mark.parametrize("logN,limbs,bits,polys", CASES)
def test_forward_skip(torch_cuda, logN, limbs, bits, polys):
    torch = torch_cuda
    import ntt_b200 as nb
    mods = plan_moduli(logN, limbs, bits)
    T = O.LimbTables(logN, mods)
    xs = np.stack([O.uniform_limbs(logN, T.q, 7 * p + logN) for p in range(polys)])
    with nb.Plan(logN, mods) as plan:
        for lo, hi in ((1, 3), (0, 1), (limbs - 2, limbs), (2, 2), (0, limbs)):
            d = to_dev(torch, xs)
            plan.forward_skip(d, lo, hi, polys)
            torch.cuda.synchronize()
            got = to_host(d, xs.shape)
            for p in range(polys):
                want = T.forward_mont(xs[p])
                want[lo:hi] = xs[p][lo:hi]  # skipped limbs untouched
                assert np.array_equal(got[p], want), (lo, hi, p)


@pytest.mark.parametrize("logN,limbs,bits,polys", CASES)
def test_forward_sub_scale(torch_cuda, logN, limbs, bits, polys):
    torch = torch_cuda
    import ntt_b200 as nb
    mods = plan_moduli(logN, limbs, bits)
    T = O.LimbTables(logN, mods)
    rng = np.random.default_rng(logN + 3 * limbs)
    xs = np.stack([O.uniform_limbs(logN, T.q, 11 * p + 1) for p in range(polys)])
    F = np.stack([T.forward_mont(x) for x in xs])
    c = np.array([int(rng.integers(0, q)) for q in T.q], dtype=np.uint32)
    lo, hi = 1, limbs - 1
    qs = np.asarray(T.q[lo:hi])
    d = np.array([int(rng.integers(0, q)) for q in qs], dtype=np.uint32)
    N = 1 << logN
    # the subtrahend: (hi - lo) limbs per polynomial, a gap of 4 words
    # between polynomials (sub_stride), Montgomery-domain words in [0, q)
    sub_stride = (hi - lo) * N + 4
    sub = np.zeros(polys * sub_stride, dtype=np.uint32)
    subs = []
    for p in range(polys):
        sp = O.uniform_limbs(logN, qs, 50 + p)
        sub[p * sub_stride:p * sub_stride + (hi - lo) * N] = sp.reshape(-1)
        subs.append(sp)
    ones = np.ones(limbs, dtype=np.uint32)
    with nb.Plan(logN, mods) as plan:
        for use_c, use_d in ((True, True), (False, True), (True, False), (False, False)):
            da = to_dev(torch, xs)
            ds = to_dev(torch, sub)
            dc = to_dev(torch, c) if use_c else None
            dd = to_dev(torch, d) if use_d else None
            plan.forward_sub_scale(da, ds, lo, hi, dc, dd, polys, sub_stride=sub_stride)
            torch.cuda.synchronize()
            got = to_host(da, xs.shape)
            cc = c if use_c else ones
            for p in range(polys):
                s_full = np.zeros_like(xs[p])
                s_full[lo:hi] = subs[p]
                d_full = np.ones(limbs, dtype=np.uint32)
                d_full[lo:hi] = d if use_d else 1
                want = sub_scale_expect(F[p], s_full, cc, d_full, T.q)
                assert np.array_equal(got[p], want), (use_c, use_d, p)
            # the subtrahend is only read
            assert np.array_equal(to_host(ds, sub.shape), sub)


@pytest.mark.parametrize("logN,limbs,bits,polys", CASES)
def test_inverse_scaled_range(torch_cuda, logN, limbs, bits, polys):
    torch = torch_cuda
    import ntt_b200 as nb
    mods = plan_moduli(logN, limbs, bits)
    T = O.LimbTables(logN, mods)
    rng = np.random.default_rng(5 * logN + limbs)
    xs = np.stack([O.uniform_limbs(logN, T.q, 3 * p + 2) for p in range(polys)])
    F = np.stack([T.forward_mont(x) for x in xs])
    with nb.Plan(logN, mods) as plan:
        for lo, hi in ((1, limbs), (0, 2), (limbs - 1, limbs), (0, limbs)):
            c = np.array([int(rng.integers(0, q)) for q in T.q[lo:hi]], dtype=np.uint32)
            d = to_dev(torch, F)
            plan.inverse_scaled_range(d, lo, hi, to_dev(torch, c), polys)
            torch.cuda.synchronize()
            got = to_host(d, xs.shape)
            q = u64(T.q[lo:hi])[:, None]
            for p in range(polys):
                want = F[p].copy()
                want[lo:hi] = ((u64(xs[p][lo:hi]) * u64(c)[:, None]) % q).astype(np.uint32)
                assert np.array_equal(got[p], want), (lo, hi, p)
        # no constant: the plain inverse of the range
        d = to_dev(torch, F)
        plan.inverse_scaled_range(d, 1, limbs, None, polys)
        torch.cuda.synchronize()
        got = to_host(d, xs.shape)
        for p in range(polys):
            assert np.array_equal(got[p][1:], xs[p][1:])
            assert np.array_equal(got[p][0], F[p][0])


def test_moddown_pipeline_identity(torch_cuda):
    """Full size, no oracle: when the subtrahend is the spectrum of the very
    polynomial being transformed, (NTT(x) - NTT(x)) * c vanishes on every
    limb whatever the constants."""
    torch = torch_cuda
    import ntt_b200 as nb
    logN, limbs = 16, 8
    mods = plan_moduli(logN, limbs, "baseline")
    T = O.LimbTables(logN, mods)
    x = O.uniform_limbs(logN, T.q, 99)
    with nb.Plan(logN, mods) as plan:
        spec = to_dev(torch, x)
        plan.forward(spec)  # the original limbs, NTT domain
        coef = to_dev(torch, x)
        pinv = np.array([pow(97, int(q) - 2, int(q)) for q in T.q], dtype=np.uint32)
        plan.forward_sub_scale(coef, spec.clone(), 0, limbs, to_dev(torch, pinv), None, 1)
        torch.cuda.synchronize()
        assert not to_host(coef, x.shape).any()


def test_rns_errors(torch_cuda):
    torch = torch_cuda
    import ntt_b200 as nb
    logN, limbs = 12, 4
    mods = plan_moduli(logN, limbs, 30)
    N = 1 << logN
    with nb.Plan(logN, mods) as plan:
        a = torch.zeros(limbs * N + 8, dtype=torch.int32, device="cuda")
        s = torch.zeros(limbs * N + 8, dtype=torch.int32, device="cuda")
        for call in (lambda: plan.forward_skip(a, 2, 1),
                     lambda: plan.forward_skip(a, 0, limbs + 1),
                     lambda: plan.inverse_scaled_range(a, -1, 2),
                     lambda: plan.forward_sub_scale(a, s, 1, limbs + 1),
                     lambda: plan.forward_sub_scale(a, None, 0, 2),
                     # overlapping subtrahend
                     lambda: plan.forward_sub_scale(a, a[N:], 0, 2)):
            with pytest.raises(nb.NttError) as e:
                call()
            assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"
        with pytest.raises(nb.NttError) as e:
            plan.forward_sub_scale(a, s[1:], 0, 2)  # 4-byte, not 16-byte, aligned
        assert e.value.name == "NTT_ERR_MISALIGNED"
        # an empty subtrahend range is the scaled forward
        plan.forward_sub_scale(a, None, 2, 2)
        torch.cuda.synchronize()


def test_rns_steps_at_full_size(torch_cuda):
    """2^17 x 64 limbs (the largest plan), no oracle: ModUp's forward equals
    the plain forward on every limb outside the skipped range and leaves that
    range alone; ModDown's forward against the plain forward's own spectrum is
    zero; the scaled inverse of a limb range undoes the forward there; the
    product with a resident spectrum equals the unfused calls."""
    torch = torch_cuda
    import ntt_b200 as nb
    logN, limbs = 17, 64
    mods = plan_moduli(logN, limbs, 31)
    q = np.array([m[0] for m in mods], dtype=np.uint64)
    N = 1 << logN
    x = O.uniform_limbs(logN, q, 2024)
    with nb.Plan(logN, mods) as plan:
        plain = to_dev(torch, x)
        plan.forward(plain)
        skip = to_dev(torch, x)
        plan.forward_skip(skip, 20, 44)
        sub = to_dev(torch, x)
        plan.forward_sub_scale(sub, plain.clone(), 0, limbs, None, None)
        torch.cuda.synchronize()
        P, S = to_host(plain, x.shape), to_host(skip, x.shape)
        assert np.array_equal(S[:20], P[:20]) and np.array_equal(S[44:], P[44:])
        assert np.array_equal(S[20:44], x[20:44])
        assert not to_host(sub, x.shape).any()
        back = plain.clone()
        plan.inverse_scaled_range(back, 8, 40, None)
        torch.cuda.synchronize()
        B = to_host(back, x.shape)
        assert np.array_equal(B[8:40], x[8:40])
        assert np.array_equal(B[:8], P[:8]) and np.array_equal(B[40:], P[40:])
        # product with a resident spectrum vs forward, pointwise, inverse
        y = O.uniform_limbs(logN, q, 2025)
        b1, b2 = to_dev(torch, y), to_dev(torch, y)
        plan.multiply_spectrum_many(plain, b1, 1)
        plan.forward(b2)
        plan.pointwise_mul(b2, plain, b2)
        plan.inverse(b2)
        torch.cuda.synchronize()
        assert torch.equal(b1, b2)
        assert N * limbs == b1.numel()
