"""Speed against the reference's own GPU path on the same B200: its v04
launch_ntt / launch_intt (built unchanged for sm_100a in oracle/_ref), one
call per polynomial as its driver uses them (v04:980-1039), against this
library's one launch over the whole batch and its own per-call form, on the
same 64 polynomials of 2^16 x 16 limbs.  Results are checked equal first.
The batch form must beat the reference's per-call path in each direction,
and the per-call form must not be slower over a forward + inverse roundtrip.

The measured times are written as one JSON object to the file named by
$NTT_B200_COMPARE_OUT when it is set.  Needs a B200.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def events_ms(torch, fn, iters):
    fn()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(iters):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / iters


@pytest.mark.parametrize("moduli", ["reference-default", "ascending-30bit"])
def test_faster_than_reference_v04_gpu(torch_cuda, moduli):
    R = O.ref_lib()
    if R is None:
        pytest.skip("reference harness not built")
    torch = torch_cuda
    import ntt_b200 as nb
    logN, polys, iters = 16, 64, 10
    mods = (O.REFERENCE_DEFAULT_MODULI if moduli == "reference-default"
            else O.ascending_primes(16, 16, 974258177))
    T = O.LimbTables(logN, mods)
    L, N = len(mods), 1 << logN
    tw, itw = T.mont_tables()
    rng = np.random.default_rng(3)
    x = rng.integers(0, T.q[None, :, None], size=(polys, L, N), dtype=np.uint64).astype(np.uint32)

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()

    src = dev(x.reshape(-1))
    ref_d, ours = src.clone(), src.clone()
    tw_d, itw_d, q_d, qi_d = dev(tw), dev(itw), dev(T.q), dev(T.q_inv)
    r2_d, di_d = dev(T.r2), dev(T.degree_inv_mont)
    args = [tw_d.data_ptr(), itw_d.data_ptr(), q_d.data_ptr(), qi_d.data_ptr(),
            r2_d.data_ptr(), di_d.data_ptr(), L]
    # the same words first (every polynomial's forward transform)
    words = L * N
    for p in range(polys):
        a = ref_d.data_ptr() + 4 * p * words
        assert R.ref_gpu_launch_ntt16(a, tw_d.data_ptr(), q_d.data_ptr(), qi_d.data_ptr(),
                                      r2_d.data_ptr(), L) == 0
    plan = nb.Plan(logN, mods)
    plan.forward_many(ours, polys)
    torch.cuda.synchronize()
    assert torch.equal(ref_d, ours)
    ms = {}
    f_ntt, f_intt = ctypes.c_float(), ctypes.c_float()
    for name, restore in (("reference_per_call", None), ("reference_per_call_restore", src)):
        assert R.ref_gpu_time16(ref_d.data_ptr(), None if restore is None else restore.data_ptr(),
                                *args, polys, iters, ctypes.byref(f_ntt), ctypes.byref(f_intt)) == 0
        ms[name] = {"ntt": f_ntt.value, "intt": f_intt.value}
    ms["ours_batch"] = {"ntt": events_ms(torch, lambda: plan.forward_many(ours, polys), iters),
                        "intt": events_ms(torch, lambda: plan.inverse_many(ours, polys), iters)}
    views = [ours[p * words:(p + 1) * words] for p in range(polys)]

    def per_call(fn):
        def run():
            for v in views:
                fn(v)
        return run
    ms["ours_per_call"] = {"ntt": events_ms(torch, per_call(plan.forward), iters),
                           "intt": events_ms(torch, per_call(plan.inverse), iters)}
    plan.close()
    out = {"workload": f"{polys} polynomials of 2^{logN} x {L} limbs, {moduli} moduli",
           "ms_per_pass_over_all_polynomials": ms,
           "limb_ntt_per_s": {k: 2 * polys * L / ((v["ntt"] + v["intt"]) / 1000.0)
                              for k, v in ms.items()}}
    path = os.environ.get("NTT_B200_COMPARE_OUT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(out) + "\n")
    for k in ("ntt", "intt"):
        assert ms["ours_batch"][k] < ms["reference_per_call"][k]
    # one polynomial per call: a single wave of CTAs, latency-bound on both
    # sides (the forward alone is on par); the roundtrip must not be slower
    rt = {k: v["ntt"] + v["intt"] for k, v in ms.items()}
    assert rt["ours_per_call"] < rt["reference_per_call"]
