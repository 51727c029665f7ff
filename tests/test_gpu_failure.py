"""Failure detection on the GPU without a fault (needs a B200).

The transform kernels bound every mbarrier wait; on expiry they record it in
the plan's status word and return normally, and ntt_plan_check reports
NTT_ERR_TIMEOUT.  Here that wait runs on a barrier nothing ever completes
(no arrival, no copy in flight) with a short limit: it must give up, the
status must read as a timeout, and the context must stay usable.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_bounded_wait_expiry_is_reported_and_the_context_survives(torch_cuda):
    torch = torch_cuda
    import ntt_b200 as nb
    mods = O.ascending_primes(12, 2, int(2 ** 29.5))
    T = O.LimbTables(12, mods)
    x = O.uniform_limbs(12, T.q, 3)
    with nb.Plan(12, mods) as p:
        assert p.check() == 0
        p.selftest_wait_expiry(256)
        with pytest.raises(nb.NttError) as e:
            p.check()
        assert e.value.name == "NTT_ERR_TIMEOUT"
        assert p.check() == 0  # the word was cleared by the read
        d = torch.from_numpy(x.view(np.int32)).cuda()
        p.forward(d)
        p.inverse(d)
        torch.cuda.synchronize()
        assert np.array_equal(d.cpu().numpy().view(np.uint32), x)
        assert p.check() == 0


def test_wait_expiry_limits(torch_cuda):
    import ntt_b200 as nb
    mods = O.ascending_primes(12, 1, int(2 ** 29.5))
    with nb.Plan(12, mods) as p:
        for bad in (0, (1 << 16) + 1):
            with pytest.raises(nb.NttError) as e:
                p.selftest_wait_expiry(bad)
            assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"
