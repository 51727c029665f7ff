"""Serving loop: continuous batching of NTT / INTT / multiply requests with
host buffers, an HBM budget and resident operands.  Needs a B200.

Each result must equal the plain per-call path on the same input (itself
pinned to the oracle), and a request's result must be the same when it runs
alone and when it runs inside a mixed stream of other requests.
"""
import threading
import time

import numpy as np
import pytest

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


def rand_poly(rng, job):
    q = np.array([m[0] for m in job.moduli], dtype=np.uint64)
    return (rng.integers(0, 1 << 62, size=(job.limbs, 1 << job.logN), dtype=np.uint64)
            % q[:, None]).astype(np.uint32)


def mont_pointwise(x, y, mods):
    out = np.empty_like(x)
    for l, (q, _) in enumerate(mods):
        rinv = pow(R32, q - 2, q)
        xy = (x[l].astype(np.uint64) * y[l].astype(np.uint64)) % np.uint64(q)
        out[l] = ((xy * np.uint64(rinv)) % np.uint64(q)).astype(np.uint32)
    return out


def plain(torch, nb, job, x, a=None):
    p = nb.Plan(job.logN, job.moduli)
    d = torch.from_numpy(x.view(np.int32)).cuda()
    if job.op == nb.OP_FORWARD:
        p.forward(d)
    elif job.op == nb.OP_INVERSE:
        p.inverse(d)
    else:
        fa = torch.from_numpy(a.view(np.int32)).cuda()
        p.forward(fa)
        p.forward(d)
        torch.cuda.synchronize()
        prod = mont_pointwise(fa.cpu().numpy().view(np.uint32), d.cpu().numpy().view(np.uint32),
                              job.moduli)
        d = torch.from_numpy(prod.view(np.int32)).cuda()
        p.inverse(d)
    torch.cuda.synchronize()
    p.close()
    return d.cpu().numpy().view(np.uint32)


def test_mixed_stream_matches_plain(torch_cuda, nb, mixes):
    torch = torch_cuda
    jobs = mixes.ragged_mix(seed=31, count=120, logn=range(12, 18), limbs=(1, 8), bits=(30, 31),
                            ops=((nb.OP_FORWARD, 2), (nb.OP_INVERSE, 2), (nb.OP_MULTIPLY, 1)))
    rng = np.random.default_rng(1)
    ins = [rand_poly(rng, j) for j in jobs]
    opnds = [rand_poly(rng, j) if j.op == nb.OP_MULTIPLY else None for j in jobs]
    outs = [np.empty_like(x) for x in ins]
    with nb.Server(hbm_budget_bytes=1 << 30) as srv:
        tickets = []
        # submissions arrive while earlier rounds run (two client threads)
        lock = threading.Lock()

        def client(idx):
            for i in idx:
                t = srv.submit(jobs[i].op, jobs[i].logN, jobs[i].moduli, ins[i], outs[i],
                               operand=opnds[i])
                with lock:
                    tickets.append(t)
                time.sleep(0.0005 * (i % 3))

        th = [threading.Thread(target=client, args=(range(k, len(jobs), 2),)) for k in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for t in tickets:
            srv.wait(t, 60.0)
        st = srv.stats()
    assert st["completed"] == len(jobs) and st["failed"] == 0
    assert st["rounds"] >= 2 and st["p99_ms"] >= st["p50_ms"] > 0
    for i, j in enumerate(jobs):
        assert np.array_equal(outs[i], plain(torch, nb, j, ins[i], opnds[i])), f"request {i}"


def test_alone_equals_in_mix(torch_cuda, nb, mixes):
    """The same request alone on an idle server, then in the middle of a
    burst of other requests of every kind: identical results."""
    jobs = mixes.ragged_mix(seed=32, count=200, logn=range(12, 18), limbs=(1, 6), bits=(30, 31),
                            ops=((nb.OP_FORWARD, 2), (nb.OP_INVERSE, 2), (nb.OP_MULTIPLY, 1)))
    rng = np.random.default_rng(2)
    probes = [j for j in jobs if j.op == nb.OP_MULTIPLY][:1] + \
             [j for j in jobs if j.op == nb.OP_FORWARD][:1] + \
             [j for j in jobs if j.op == nb.OP_INVERSE][:1]
    with nb.Server(hbm_budget_bytes=2 << 30) as srv:
        for pj in probes:
            x = rand_poly(rng, pj)
            a = rand_poly(rng, pj) if pj.op == nb.OP_MULTIPLY else None
            alone = np.empty_like(x)
            srv.wait(srv.submit(pj.op, pj.logN, pj.moduli, x, alone, operand=a), 60.0)
            ins = [rand_poly(rng, j) for j in jobs]
            ops = [rand_poly(rng, j) if j.op == nb.OP_MULTIPLY else None for j in jobs]
            outs = [np.empty_like(v) for v in ins]
            mixed = np.empty_like(x)
            ts = []
            for i, j in enumerate(jobs):
                ts.append(srv.submit(j.op, j.logN, j.moduli, ins[i], outs[i], operand=ops[i]))
                if i == len(jobs) // 2:
                    ts.append(srv.submit(pj.op, pj.logN, pj.moduli, x, mixed, operand=a))
            for t in ts:
                srv.wait(t, 60.0)
            assert np.array_equal(alone, mixed)
        st = srv.stats()
    assert st["mean_round_requests"] > 1.5  # the bursts were batched


def test_budget_admission(torch_cuda, nb, mixes):
    torch = torch_cuda
    budget = 24 << 20
    jobs = mixes.ragged_mix(seed=33, count=40, logn=(16,), limbs=(8, 16))  # 2..4 MiB each
    rng = np.random.default_rng(3)
    ins = [rand_poly(rng, j) for j in jobs]
    outs = [np.empty_like(x) for x in ins]
    with nb.Server(hbm_budget_bytes=budget, streams=2) as srv:
        big = mixes.ragged_mix(seed=34, count=1, logn=(17,), limbs=(48, 48))[0]  # 24 MiB + 256
        xb = np.zeros((big.limbs + 1, 1 << 17), dtype=np.uint32)
        with pytest.raises(nb.NttError) as e:
            srv.submit(nb.OP_FORWARD, 17, big.moduli + big.moduli[:1], xb, xb)
        assert e.value.name == "NTT_ERR_BUDGET"
        ts = [srv.submit(j.op, j.logN, j.moduli, ins[i], outs[i]) for i, j in enumerate(jobs)]
        for t in ts:
            srv.wait(t, 60.0)
        st = srv.stats()
    assert st["completed"] == len(jobs)
    assert st["arena_peak_bytes"] <= st["budget_bytes"] == budget
    assert st["rounds"] > 3  # the budget split the stream into several rounds
    for i in range(0, len(jobs), 7):
        assert np.array_equal(outs[i], plain(torch, nb, jobs[i], ins[i]))


def test_resident_operand(torch_cuda, nb, mixes):
    torch = torch_cuda
    j = mixes.ragged_mix(seed=35, count=1, logn=(14,), limbs=(5, 5),
                         ops=((nb.OP_MULTIPLY, 1),))[0]
    rng = np.random.default_rng(4)
    a = rand_poly(rng, j)
    with nb.Server(hbm_budget_bytes=256 << 20) as srv:
        h = srv.put(a)
        assert srv.stats()["resident_bytes"] >= a.nbytes
        xs = [rand_poly(rng, j) for _ in range(6)]
        outs = [np.empty_like(x) for x in xs]
        ts = [srv.submit(nb.OP_MULTIPLY, j.logN, j.moduli, x, o, operand_handle=h)
              for x, o in zip(xs, outs)]
        for t in ts:
            srv.wait(t, 60.0)
            assert srv.latency_ms(t) > 0
        srv.drop(h)
        assert srv.stats()["resident_bytes"] == 0
    for x, o in zip(xs, outs):
        assert np.array_equal(o, plain(torch, nb, j, x, a))


def test_resident_spectrum_operand(torch_cuda, nb, mixes):
    torch = torch_cuda
    j = mixes.ragged_mix(seed=37, count=1, logn=(15,), limbs=(3, 3),
                         ops=((nb.OP_MULTIPLY, 1),))[0]
    rng = np.random.default_rng(6)
    a = rand_poly(rng, j)
    with nb.Server(hbm_budget_bytes=256 << 20) as srv:
        h = srv.put_spectrum(j.logN, j.moduli, a)
        xs = [rand_poly(rng, j) for _ in range(5)]
        outs = [np.empty_like(x) for x in xs]
        ts = [srv.submit(nb.OP_MULTIPLY_SPECTRUM, j.logN, j.moduli, x, o, operand_handle=h)
              for x, o in zip(xs, outs)]
        for t in ts:
            srv.wait(t, 60.0)
        srv.drop(h)
    for x, o in zip(xs, outs):
        assert np.array_equal(o, plain(torch, nb, j, x, a))


def test_in_place_output_and_errors(torch_cuda, nb, mixes):
    j = mixes.ragged_mix(seed=36, count=1, logn=(12,), limbs=(3, 3))[0]
    rng = np.random.default_rng(5)
    x = rand_poly(rng, j)
    expect_in = x.copy()
    with nb.Server(hbm_budget_bytes=64 << 20) as srv:
        srv.wait(srv.submit(nb.OP_FORWARD, 12, j.moduli, x, x), 60.0)  # output == input
        srv.wait(srv.submit(nb.OP_INVERSE, 12, j.moduli, x, x), 60.0)
        assert np.array_equal(x, expect_in)
        with pytest.raises(nb.NttError) as e:
            srv.submit(nb.OP_FORWARD, 11, j.moduli, x, x)
        assert e.value.name == "NTT_ERR_UNSUPPORTED"
        with pytest.raises(nb.NttError) as e:
            srv.submit(nb.OP_MULTIPLY, 12, j.moduli, x, x)
        assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"
        with pytest.raises(nb.NttError) as e:
            srv.submit(nb.OP_FORWARD, 12, [(j.moduli[0][0] + 2, 3)] * 3, x, x)
        assert e.value.name == "NTT_ERR_MODULUS"
        with pytest.raises(nb.NttError) as e:
            srv.wait(123456, 0.1)
        assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"


def test_device_resident_requests_match_plain(torch_cuda, nb, mixes):
    """Requests on device buffers (device_buffers): transformed where they
    lie, in place or from a distinct input, mixed in one stream with
    host-buffer requests; every result equals the plain per-call path."""
    torch = torch_cuda
    jobs = mixes.ragged_mix(seed=35, count=60, logn=range(12, 18), limbs=(1, 6), bits=(30, 31),
                            ops=((nb.OP_FORWARD, 2), (nb.OP_INVERSE, 2), (nb.OP_MULTIPLY, 1)))
    rng = np.random.default_rng(5)
    ins = [rand_poly(rng, j) for j in jobs]
    opnds = [rand_poly(rng, j) if j.op == nb.OP_MULTIPLY else None for j in jobs]
    dev = lambda a: torch.from_numpy(a.view(np.int32)).cuda()
    outs, keep = [], []
    with nb.Server(hbm_budget_bytes=1 << 30) as srv:
        tickets = []
        for i, j in enumerate(jobs):
            if i % 3 == 2:  # host buffers
                o = np.empty_like(ins[i])
                tickets.append(srv.submit(j.op, j.logN, j.moduli, ins[i], o, operand=opnds[i]))
            else:
                x = dev(ins[i])
                o = x if i % 3 == 0 else torch.empty_like(x)  # in place / distinct output
                a = dev(opnds[i]) if opnds[i] is not None else None
                keep.append((x, a))
                tickets.append(srv.submit(j.op, j.logN, j.moduli, x, o, operand=a, device=True))
            outs.append(o)
        for t in tickets:
            srv.wait(t, 60.0)
        st = srv.stats()
    assert st["completed"] == len(jobs) and st["failed"] == 0
    for i, j in enumerate(jobs):
        got = outs[i] if isinstance(outs[i], np.ndarray) else outs[i].cpu().numpy().view(np.uint32)
        assert np.array_equal(got, plain(torch, nb, j, ins[i], opnds[i])), f"request {i}"


def test_device_buffers_must_be_aligned(torch_cuda, nb, mixes):
    torch = torch_cuda
    pool = mixes.prime_pool(12, 30, 2)
    x = torch.zeros(2 * (1 << 12) + 4, dtype=torch.int32, device="cuda")
    with nb.Server(hbm_budget_bytes=1 << 28) as srv:
        with pytest.raises(nb.NttError) as e:
            srv.submit(nb.OP_FORWARD, 12, pool, x[1:], x[1:], device=True)
        assert e.value.name == "NTT_ERR_MISALIGNED"
