"""Transform launches back to back with no host synchronisation between them.

Transform launches carry programmatic dependent launch (the split kernels,
which trigger the next launch at their start up to logN 16 and after the
phase exchange at logN 17, and the cluster kernels): such a launch may be
scheduled while the kernel before it in the stream drains, and the kernel
waits for that one's completion before it touches memory (pdl_wait in
pdl.cuh).  These chains feed each launch's output to the next, mix
in torch kernels (launched without the attribute) that read and rewrite the
buffers, and compare with the oracle and with the same chain synchronised
after every call.  Needs a B200.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def to_dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda().reshape(-1)


def to_host(t, shape):
    return t.cpu().numpy().view(np.uint32).reshape(shape)


@pytest.mark.parametrize("logN,limbs", [(16, 4), (17, 2), (15, 3), (13, 5), (11, 6)])
def test_dependent_chain_matches_oracle(torch_cuda, logN, limbs):
    torch = torch_cuda
    import ntt_b200 as nb
    mods = O.ascending_primes(logN, limbs, 974258177)
    T = O.LimbTables(logN, mods)
    x = O.uniform_limbs(logN, T.q, 31 * logN + limbs)
    F = T.forward_mont(x)
    s = torch.cuda.Stream()
    sh = s.cuda_stream
    with nb.Plan(logN, mods) as p:
        with torch.cuda.stream(s):
            d = to_dev(torch, x)
            for _ in range(10):  # 20 launches, each on the previous one's output
                p.forward(d, sh)
                p.inverse(d, sh)
            p.forward(d, sh)
            snap = d.clone()  # a torch kernel reads the forward's output
            p.inverse(d, sh)
            d.copy_(snap)  # a torch kernel rewrites the buffer the next launch reads
            p.inverse(d, sh)
            p.forward(d, sh)
        s.synchronize()
        assert np.array_equal(to_host(snap, x.shape), F)
        assert np.array_equal(to_host(d, x.shape), F)


def test_unsynchronised_chain_equals_synchronised(torch_cuda):
    """A fixed random sequence of roundtrips, products, products with a
    resident spectrum and scaled forwards over two buffers and two plans
    (the split kernels at 2^16, the cluster kernels at 2^13), once with a
    device synchronisation after every call and once with none."""
    torch = torch_cuda
    import ntt_b200 as nb
    rng = np.random.default_rng(77)
    ops = [rng.choice(["rt", "mul", "spec", "scaled", "swap"]) for _ in range(30)]
    polys = 2
    results = []
    for sync in (True, False):
        out = []
        s = torch.cuda.Stream()
        sh = s.cuda_stream
        for logN, limbs in ((16, 3), (13, 4)):
            mods = O.ascending_primes(logN, limbs, 974258177)
            T = O.LimbTables(logN, mods)
            xs = [np.stack([O.uniform_limbs(logN, T.q, 100 * k + p) for p in range(polys)])
                  for k in range(3)]
            with nb.Plan(logN, mods) as p, torch.cuda.stream(s):
                u, v, spec = (to_dev(torch, a) for a in xs)
                cs = to_dev(torch, np.array([3 + k for k in range(limbs)], dtype=np.uint32))
                p.forward_many(spec, polys, 0, sh)
                for op in ops:
                    if op == "rt":
                        p.forward_many(u, polys, 0, sh)
                        p.inverse_many(u, polys, 0, sh)
                    elif op == "mul":
                        p.multiply_many(v, u, polys, 0, sh)
                    elif op == "spec":
                        p.multiply_spectrum_many(spec, u, polys, 0, sh)
                    elif op == "scaled":
                        p.forward_scaled(u, cs, polys, 0, sh)
                        p.inverse_many(u, polys, 0, sh)
                    else:
                        u, v = v, u
                    if sync:
                        s.synchronize()
                s.synchronize()
                out.append((to_host(u, xs[0].shape), to_host(v, xs[0].shape)))
        results.append(out)
    for (u0, v0), (u1, v1) in zip(results[0], results[1]):
        assert np.array_equal(u0, u1) and np.array_equal(v0, v1)
