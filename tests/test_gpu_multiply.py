"""Plan-level negacyclic product (ntt_multiply_many: NTT(b), NTT(a) with the
pointwise Montgomery product folded into its store, INTT(b)) against the
unfused plain calls (forward, forward, ntt_pointwise_mul, inverse) and the
schoolbook product mod q.  Needs a B200.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb(torch_cuda):
    import ntt_b200
    return ntt_b200


@pytest.fixture(scope="module")
def mixes(nb):
    from ntt_b200 import mixes
    return mixes


def host(t):
    return t.cpu().numpy().view(np.uint32)


def pair_inputs(torch, mixes, nb, logN, mods, pairs, seed):
    job = mixes.MixJob(nb.OP_MULTIPLY, logN, mods)
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    a = torch.stack([mixes.uniform_device(torch, job, g) for _ in range(pairs)])
    b = torch.stack([mixes.uniform_device(torch, job, g) for _ in range(pairs)])
    return a, b


def unfused(p, a, b, pairs):
    ta, tb = a.clone(), b.clone()
    p.forward_many(ta, pairs)
    p.forward_many(tb, pairs)
    p.pointwise_mul(tb, ta, tb, pairs)
    p.inverse_many(tb, pairs)
    return tb


@pytest.mark.parametrize("logN,bits", [(10, 30), (12, 31), (13, 30), (14, 31), (15, 30),
                                       (16, 31), (17, 30)])
def test_multiply_many_matches_unfused(torch_cuda, nb, mixes, logN, bits):
    torch = torch_cuda
    pairs, limbs = 3, 5
    mods = list(mixes.prime_pool(logN, bits, limbs))
    a, b = pair_inputs(torch, mixes, nb, logN, mods, pairs, 70 + logN)
    a_h = host(a).copy()
    p = nb.Plan(logN, mods)
    expect = unfused(p, a, b, pairs)
    p.multiply_many(a, b, pairs)
    torch.cuda.synchronize()
    assert torch.equal(b, expect)
    assert np.array_equal(host(a), a_h)  # the factor a is read only
    assert p.check() == 0
    p.close()


def test_multiply_many_every_logn16_config(torch_cuda, nb, mixes):
    """Every compiled logN-16 configuration (one and two polynomials per job),
    an odd number of pairs (the last two-polynomial job repeats a pair)."""
    torch = torch_cuda
    pairs, limbs = 5, 3
    mods = list(mixes.prime_pool(16, 30, limbs))
    a, b = pair_inputs(torch, mixes, nb, 16, mods, pairs, 5)
    ref = nb.Plan(16, mods)
    expect = unfused(ref, a, b, pairs)
    for idx, c in enumerate(nb.kernel_configs()):
        if c.logN != 16:
            continue
        p = nb.Plan(16, mods)
        p.force_config(idx, idx)
        x = b.clone()
        p.multiply_many(a, x, pairs)
        torch.cuda.synchronize()
        assert torch.equal(x, expect), f"config {idx}"
        p.close()
    ref.close()


def test_multiply_many_schoolbook_sample(torch_cuda, nb, mixes):
    """The fused multiply configuration's shape (2^16, 24 limbs of 30-bit
    primes): 64 sampled (pair, limb, coefficient) triples against the O(N)
    schoolbook negacyclic coefficient mod q."""
    torch = torch_cuda
    logN, pairs, limbs = 16, 2, 24
    mods = list(mixes.prime_pool(logN, 30, limbs))
    a, b = pair_inputs(torch, mixes, nb, logN, mods, pairs, 9)
    a_h, b_h = host(a).copy(), host(b).copy()
    p = nb.Plan(logN, mods)
    p.multiply_many(a, b, pairs)
    torch.cuda.synchronize()
    c = host(b)
    rng = np.random.default_rng(16)
    for _ in range(64):
        i, l, k = int(rng.integers(pairs)), int(rng.integers(limbs)), int(rng.integers(1 << logN))
        assert int(c[i, l, k]) == O.negacyclic_coeff(a_h[i, l], b_h[i, l], logN, mods[l][0], k)
    p.close()


def test_multiply_many_errors(torch_cuda, nb, mixes):
    torch = torch_cuda
    mods = list(mixes.prime_pool(12, 30, 2))
    p = nb.Plan(12, mods)
    x = torch.zeros(4, 2 << 12, dtype=torch.int32, device="cuda")
    with pytest.raises(nb.NttError) as e:  # b overlaps a
        p.multiply_many(x[0], x[0], 1)
    assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"
    with pytest.raises(nb.NttError) as e:
        p.multiply_many(x[0].data_ptr() + 4, x[2], 1)
    assert e.value.name == "NTT_ERR_MISALIGNED"
    p.close()
    small = nb.Plan(8, list(mixes.prime_pool(8, 30, 1)))
    y = torch.zeros(2, 1 << 8, dtype=torch.int32, device="cuda")
    with pytest.raises(nb.NttError) as e:
        small.multiply_many(y[0], y[1], 1)
    assert e.value.name == "NTT_ERR_UNSUPPORTED"
    small.close()


@pytest.mark.parametrize("logN,bits,compressed", [(8, 30, False), (12, 31, False),
                                                  (15, 30, False), (16, 31, False),
                                                  (16, 30, True), (17, 30, False)])
def test_multiply_spectrum_many(torch_cuda, nb, mixes, logN, bits, compressed):
    """b <- INTT(NTT(b) (.) NTT(a)) with NTT(a) resident: equal to the unfused
    calls on every kernel family (the split forward's spectrum-product
    store at logN 15..17, forward + pointwise + inverse elsewhere and on
    compressed plans); the spectrum is only read."""
    torch = torch_cuda
    pairs, limbs = 3, 4
    mods = list(mixes.prime_pool(logN, bits, limbs))
    a, b = pair_inputs(torch, mixes, nb, logN, mods, pairs, 40 + logN)
    p = nb.Plan(logN, mods, compressed_twiddles=compressed)
    expect = unfused(p, a, b, pairs)
    spec = a.clone()
    p.forward_many(spec, pairs)
    spec_h = host(spec).copy()
    p.multiply_spectrum_many(spec, b, pairs)
    torch.cuda.synchronize()
    assert torch.equal(b, expect)
    assert np.array_equal(host(spec), spec_h)
    p.close()


def test_multiply_spectrum_schoolbook_and_errors(torch_cuda, nb, mixes):
    torch = torch_cuda
    logN, pairs, limbs = 16, 2, 6
    mods = list(mixes.prime_pool(logN, 30, limbs))
    a, b = pair_inputs(torch, mixes, nb, logN, mods, pairs, 21)
    a_h, b_h = host(a).copy(), host(b).copy()
    p = nb.Plan(logN, mods)
    spec = a.clone()
    p.forward_many(spec, pairs)
    p.multiply_spectrum_many(spec, b, pairs)
    torch.cuda.synchronize()
    c = host(b)
    rng = np.random.default_rng(61)
    for _ in range(32):
        i, l, k = int(rng.integers(pairs)), int(rng.integers(limbs)), int(rng.integers(1 << logN))
        assert int(c[i, l, k]) == O.negacyclic_coeff(a_h[i, l], b_h[i, l], logN, mods[l][0], k)
    with pytest.raises(nb.NttError) as e:  # the spectrum overlaps b
        p.multiply_spectrum_many(b, b, 1)
    assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"
    with pytest.raises(nb.NttError) as e:
        p.multiply_spectrum_many(spec.data_ptr() + 4, b, 1)
    assert e.value.name == "NTT_ERR_MISALIGNED"
    p.close()


@pytest.mark.parametrize("logN", [15, 16, 17])
def test_multiply_forms_on_split_plans(torch_cuda, nb, mixes, logN):
    """Both forms of ntt_multiply_many on split plans (one launch; split
    forward, cluster forward with the product, split inverse) equal the
    unfused calls, and the factor a is only read."""
    torch = torch_cuda
    pairs, limbs = 3, 4
    mods = list(mixes.prime_pool(logN, 30, limbs))
    a, b = pair_inputs(torch, mixes, nb, logN, mods, pairs, 90 + logN)
    a_h = host(a).copy()
    ref = nb.Plan(logN, mods)
    expect = unfused(ref, a, b, pairs)
    for form in (nb.MULTIPLY_ONE_LAUNCH, nb.MULTIPLY_THREE_LAUNCHES):
        p = nb.Plan(logN, mods)
        p.set_multiply_form(form)
        x = b.clone()
        p.multiply_many(a, x, pairs)
        torch.cuda.synchronize()
        assert torch.equal(x, expect), form
        assert np.array_equal(host(a), a_h)
        p.close()
    with pytest.raises(nb.NttError) as e:
        ref.set_multiply_form(5)
    assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"
    ref.close()
