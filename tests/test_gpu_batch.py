"""Ragged batches (one persistent launch over many polynomials of different
logN, limb counts, modulus chains and operations) against the plain
per-call path and the CPU oracle.  Needs a B200.

Every tile must be bit-identical to ntt_forward / ntt_inverse of a plan with
the same modulus (itself pinned to the oracle in test_gpu_parity.py); a
sample of (job, limb) pairs is also checked against the oracle directly, and
multiplies against the schoolbook negacyclic product.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
R32 = 1 << 32


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


def make_inputs(torch, mixes, jobs, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    data = [mixes.uniform_device(torch, j, g) for j in jobs]
    ops = [mixes.uniform_device(torch, j, g) if j.op == 2 else None for j in jobs]
    return data, ops


def mont_pointwise(x, y, mods):
    """x * y * 2^-32 mod q per limb (numpy, exact)."""
    out = np.empty_like(x)
    for l, (q, _) in enumerate(mods):
        rinv = pow(R32, q - 2, q)
        xy = (x[l].astype(np.uint64) * y[l].astype(np.uint64)) % np.uint64(q)
        out[l] = ((xy * np.uint64(rinv)) % np.uint64(q)).astype(np.uint32)
    return out


def plain_expected(torch, nb, job, x, a=None):
    """The plain per-call path on copies."""
    p = nb.Plan(job.logN, job.moduli)
    d = x.clone()
    if job.op == nb.OP_FORWARD:
        p.forward(d)
    elif job.op == nb.OP_INVERSE:
        p.inverse(d)
    else:
        fa = a.clone()
        p.forward(fa)
        p.forward(d)
        torch.cuda.synchronize()
        prod = mont_pointwise(host(fa), host(d), job.moduli)
        d = torch.from_numpy(prod.view(np.int32)).cuda()
        p.inverse(d)
    torch.cuda.synchronize()
    p.close()
    return host(d)


def run_batch_and_compare(torch, nb, mixes, jobs, seed, **opts):
    data, ops = make_inputs(torch, mixes, jobs, seed)
    expect = [plain_expected(torch, nb, j, x, a) for j, x, a in zip(jobs, data, ops)]
    with nb.Batch([(j.op, j.logN, j.moduli, x, a) for j, x, a in zip(jobs, data, ops)],
                  **opts) as b:
        info = b.info
        b.run()
        torch.cuda.synchronize()
    for i, (j, x) in enumerate(zip(jobs, data)):
        got = host(x)
        assert np.array_equal(got, expect[i]), f"job {i} (op {j.op}, logN {j.logN}, limbs {j.limbs})"
    return info, data


def test_ragged_forward_inverse_cluster16(torch_cuda, nb, mixes):
    jobs = mixes.ragged_mix(seed=11, count=48, logn=range(12, 18), limbs=(1, 6), bits=(30, 31),
                            ops=((nb.OP_FORWARD, 1), (nb.OP_INVERSE, 1)))
    info, _ = run_batch_and_compare(torch_cuda, nb, mixes, jobs, 1)
    assert info.cluster_ctas == 16 and info.tiles == sum(j.limbs for j in jobs)


def test_ragged_cluster8(torch_cuda, nb, mixes):
    jobs = mixes.ragged_mix(seed=12, count=40, logn=range(12, 17), limbs=(1, 9), bits=(30, 31),
                            ops=((nb.OP_FORWARD, 1), (nb.OP_INVERSE, 1)))
    info, _ = run_batch_and_compare(torch_cuda, nb, mixes, jobs, 2, cluster_ctas=8)
    assert info.cluster_ctas == 8


def test_ragged_cluster16_without_logn17(torch_cuda, nb, mixes):
    jobs = mixes.ragged_mix(seed=13, count=30, logn=range(12, 17), limbs=(1, 5),
                            ops=((nb.OP_FORWARD, 1), (nb.OP_INVERSE, 1)))
    run_batch_and_compare(torch_cuda, nb, mixes, jobs, 3, cluster_ctas=16)


def test_single_cluster_drains_queue(torch_cuda, nb, mixes):
    jobs = mixes.ragged_mix(seed=14, count=20, logn=range(12, 18), limbs=(1, 4),
                            ops=((nb.OP_FORWARD, 1), (nb.OP_INVERSE, 1)))
    info, _ = run_batch_and_compare(torch_cuda, nb, mixes, jobs, 4, max_clusters=1)
    assert info.clusters == 1


def test_plain_launch_without_graph(torch_cuda, nb, mixes):
    jobs = mixes.ragged_mix(seed=15, count=16, logn=range(12, 17), limbs=(1, 4))
    run_batch_and_compare(torch_cuda, nb, mixes, jobs, 5, use_graph=False)


def test_multiply(torch_cuda, nb, mixes):
    jobs = mixes.ragged_mix(seed=16, count=24, logn=range(12, 18), limbs=(1, 4), bits=(30, 31),
                            ops=((nb.OP_MULTIPLY, 1),))
    info, _ = run_batch_and_compare(torch_cuda, nb, mixes, jobs, 6)
    assert info.multiply == 1


def test_mixed_ops_one_launch(torch_cuda, nb, mixes):
    jobs = mixes.ragged_mix(seed=17, count=60, logn=range(12, 18), limbs=(1, 5), bits=(30, 31),
                            ops=((nb.OP_FORWARD, 2), (nb.OP_INVERSE, 2), (nb.OP_MULTIPLY, 1)))
    assert len({j.op for j in jobs}) == 3
    run_batch_and_compare(torch_cuda, nb, mixes, jobs, 7)


def test_multiply_schoolbook_sample(torch_cuda, nb, mixes):
    """Sampled (job, limb, coefficient) triples against the O(N) schoolbook
    negacyclic coefficient mod q."""
    torch = torch_cuda
    jobs = mixes.ragged_mix(seed=18, count=6, logn=(12, 15, 16), limbs=(2, 3), bits=(30, 31),
                            ops=((nb.OP_MULTIPLY, 1),))
    data, ops = make_inputs(torch, mixes, jobs, 8)
    a_h = [host(a) for a in ops]
    b_h = [host(x) for x in data]
    with nb.Batch([(j.op, j.logN, j.moduli, x, a) for j, x, a in zip(jobs, data, ops)]) as b:
        b.run()
        torch.cuda.synchronize()
    rng = np.random.default_rng(5)
    for i, j in enumerate(jobs):
        c = host(data[i])
        for _ in range(4):
            l = int(rng.integers(0, j.limbs))
            k = int(rng.integers(0, 1 << j.logN))
            q = j.moduli[l][0]
            assert int(c[l, k]) == O.negacyclic_coeff(a_h[i][l], b_h[i][l], j.logN, q, k)


def test_oracle_sample_and_roundtrip_replay(torch_cuda, nb, mixes):
    """Forward batch then inverse batch, replayed three times (graph
    replays): identity each time; the first forward is checked against the
    oracle on sampled (job, limb) pairs."""
    torch = torch_cuda
    jobs = mixes.ragged_mix(seed=19, count=24, logn=range(12, 18), limbs=(1, 4), bits=(30, 31))
    data, _ = make_inputs(torch, mixes, jobs, 9)
    orig = [host(x).copy() for x in data]
    fwd = nb.Batch([(nb.OP_FORWARD, j.logN, j.moduli, x, None) for j, x in zip(jobs, data)])
    inv = nb.Batch([(nb.OP_INVERSE, j.logN, j.moduli, x, None) for j, x in zip(jobs, data)])
    for rep in range(3):
        fwd.run()
        torch.cuda.synchronize()
        if rep == 0:
            for i in range(0, len(jobs), 4):
                j = jobs[i]
                l = j.limbs - 1
                T = O.LimbTables(j.logN, [j.moduli[l]])
                assert np.array_equal(host(data[i])[l:l + 1], T.forward_mont(orig[i][l:l + 1]))
        inv.run()
        torch.cuda.synchronize()
        for i in range(len(jobs)):
            assert np.array_equal(host(data[i]), orig[i]), f"replay {rep} job {i}"
    fwd.close()
    inv.close()


def test_tables_shared_and_trimmed(torch_cuda, nb, mixes):
    torch = torch_cuda
    nb.tables_trim()
    base = nb.tables_device_bytes()
    jobs = mixes.ragged_mix(seed=20, count=8, logn=(13,), limbs=(2, 2))
    data, _ = make_inputs(torch, mixes, jobs, 10)
    b = nb.Batch([(j.op, j.logN, j.moduli, x, None) for j, x in zip(jobs, data)])
    held = nb.tables_device_bytes()
    distinct = len({m for j in jobs for m in j.moduli})
    # two tables of 2^13 (w, w') pairs per modulus + its 2 x 28-byte generator inputs
    assert held - base == distinct * ((1 << 13) * 16 + 56)
    nb.tables_trim()
    assert nb.tables_device_bytes() == held  # still used by the batch
    b.close()
    nb.tables_trim()
    assert nb.tables_device_bytes() == base


def test_batch_errors(torch_cuda, nb, mixes):
    torch = torch_cuda
    x = torch.zeros(2, 1 << 12, dtype=torch.int32, device="cuda")
    mods = mixes.prime_pool(12, 30, 4)[:2]
    with pytest.raises(nb.NttError) as e:
        nb.Batch([(nb.OP_MULTIPLY, 12, mods, x, None)])
    assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"
    with pytest.raises(nb.NttError) as e:
        nb.Batch([(nb.OP_FORWARD, 12, [(mods[0][0] + 2, 3), mods[1]], x, None)])
    assert e.value.name == "NTT_ERR_MODULUS"
    with pytest.raises(nb.NttError) as e:
        nb.Batch([(nb.OP_FORWARD, 17, mixes.prime_pool(17, 30, 1), x, None)], cluster_ctas=8)
    assert e.value.name == "NTT_ERR_UNSUPPORTED"


@pytest.mark.parametrize("logN", [15, 16])
def test_config4_fused_vs_unfused_multiply(torch_cuda, nb, mixes, logN):
    """Fused negacyclic multiply (one persistent launch) against the unfused
    plain calls (forward, forward, ntt_pointwise_mul, inverse) at the
    multiply configuration's shape: N = 2^15 / 2^16, 24 limbs of 30-bit
    primes; plus 64 sampled (pair, limb, coefficient) schoolbook checks."""
    torch = torch_cuda
    pairs, limbs = 3, 24
    mods = list(mixes.prime_pool(logN, 30, 24))
    job = mixes.MixJob(nb.OP_MULTIPLY, logN, mods)
    g = torch.Generator(device="cuda")
    g.manual_seed(40 + logN)
    a = torch.stack([mixes.uniform_device(torch, job, g) for _ in range(pairs)])
    b = torch.stack([mixes.uniform_device(torch, job, g) for _ in range(pairs)])
    a_h, b_h = host(a).copy(), host(b).copy()
    # unfused plain calls on copies
    p = nb.Plan(logN, mods)
    ta, tb = a.clone(), b.clone()
    p.forward_many(ta, pairs)
    p.forward_many(tb, pairs)
    p.pointwise_mul(tb, ta, tb, pairs)
    p.inverse_many(tb, pairs)
    # fused: one batch of multiply tiles
    with nb.Batch([(nb.OP_MULTIPLY, logN, mods, b[i], a[i]) for i in range(pairs)]) as bt:
        bt.run()
    torch.cuda.synchronize()
    assert torch.equal(b, tb)
    assert torch.equal(a, torch.from_numpy(a_h.view(np.int32)).cuda())  # operand untouched
    c = host(b)
    rng = np.random.default_rng(logN)
    for _ in range(64):
        i, l, k = int(rng.integers(pairs)), int(rng.integers(limbs)), int(rng.integers(1 << logN))
        assert int(c[i, l, k]) == O.negacyclic_coeff(a_h[i, l], b_h[i, l], logN, mods[l][0], k)
    p.close()


def test_pointwise_mul_matches_numpy(torch_cuda, nb, mixes):
    torch = torch_cuda
    mods = list(mixes.prime_pool(13, 31, 5))
    job = mixes.MixJob(nb.OP_FORWARD, 13, mods)
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    x = torch.stack([mixes.uniform_device(torch, job, g) for _ in range(2)])
    y = torch.stack([mixes.uniform_device(torch, job, g) for _ in range(2)])
    z = torch.empty_like(x)
    p = nb.Plan(13, mods)
    p.pointwise_mul(z, x, y, 2)
    torch.cuda.synchronize()
    for i in range(2):
        assert np.array_equal(host(z)[i], mont_pointwise(host(x)[i], host(y)[i], mods))
    p.close()


def test_multiply_spectrum_operand(torch_cuda, nb, mixes):
    """OP_MULTIPLY_SPECTRUM with the operand given as its forward transform
    equals OP_MULTIPLY with the operand itself (and the plain path)."""
    torch = torch_cuda
    jobs = mixes.ragged_mix(seed=21, count=20, logn=range(12, 18), limbs=(1, 4), bits=(30, 31),
                            ops=((nb.OP_MULTIPLY, 1),))
    data, ops = make_inputs(torch, mixes, jobs, 11)
    expect = [plain_expected(torch, nb, j, x, a) for j, x, a in zip(jobs, data, ops)]
    spectra = []
    for j, a in zip(jobs, ops):
        p = nb.Plan(j.logN, j.moduli)
        s = a.clone()
        p.forward(s)
        spectra.append(s)
        p.close()
    torch.cuda.synchronize()
    mixed = [(nb.OP_MULTIPLY_SPECTRUM if i % 2 == 0 else nb.OP_MULTIPLY, j.logN, j.moduli, x,
              spectra[i] if i % 2 == 0 else ops[i]) for i, (j, x) in enumerate(zip(jobs, data))]
    with nb.Batch(mixed) as b:
        b.run()
        torch.cuda.synchronize()
    for i, x in enumerate(data):
        assert np.array_equal(host(x), expect[i]), f"job {i}"
