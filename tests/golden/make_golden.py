"""Generate tests/golden/golden.json from the reference's own compiled code.

Runs the reference's host functions (make_modulus_runtime,
make_twiddle_table, fill_random, cpu_ntt_butterfly, cpu_intt_butterfly from
src/v04_montgomery.cu, compiled unchanged by oracle/Makefile into
oracle/_ref/libntt_ref.so) and records small known-answer fixtures:
per-limb constants, full vectors for small N, and SHA-256 digests plus
sample words for the 2^16 x 16 configurations.  Needs the reference
checkout (run here, not on the GPU host):

    make -C oracle ref && python tests/golden/make_golden.py
"""
import ctypes
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

R = O.ref_lib()
if R is None:
    raise SystemExit("oracle/_ref/libntt_ref.so is not built (make -C oracle ref)")
P = O._ptr


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


def runtime(logN, q, g):
    o = (ctypes.c_uint32 * 8)()
    R.ref_modulus_runtime(logN, q, g, o)
    return list(o)


def ref_tables(logN, moduli):
    N = 1 << logN
    L = len(moduli)
    rts = [runtime(logN, q, g) for q, g in moduli]
    tw = np.empty((L, N), np.uint32)
    itw = np.empty((L, N), np.uint32)
    for i, rt in enumerate(rts):
        R.ref_twiddle_table(logN, rt[0], rt[4], P(tw[i]))
        R.ref_twiddle_table(logN, rt[0], rt[5], P(itw[i]))
    return rts, tw, itw


def ref_run(logN, moduli, seed_input=None):
    N = 1 << logN
    rts, tw, itw = ref_tables(logN, moduli)
    x = np.empty((len(moduli), N), np.uint32)
    for i, rt in enumerate(rts):
        R.ref_fill_random(P(x[i]), N, rt[0])
    f = x.copy()
    for i, rt in enumerate(rts):
        R.ref_cpu_ntt(P(f[i]), logN, rt[0], P(tw[i]))
    fm = np.stack([[R.ref_to_mont(int(v), rt[0]) for v in f[i]] if N <= 1024 else
                   O.to_mont_array(f[i], rt[0]) for i, rt in enumerate(rts)]).astype(np.uint32)
    rtp = f.copy()
    for i, rt in enumerate(rts):
        R.ref_cpu_intt(P(rtp[i]), logN, rt[0], P(itw[i]), rt[7])
    return rts, tw, itw, x, f, fm, rtp


out = {"generator": "tests/golden/make_golden.py", "source": "reference v04 host functions",
       "cases": []}

baseline16 = O.ascending_primes(16, 16, 974258177)
sets = {
    "reference_default_moduli": O.REFERENCE_DEFAULT_MODULI,
    "ascending_2^17_from_974258177": baseline16,
}
for name, mods in sets.items():
    for logN in (10, 12, 16):
        rts, tw, itw, x, f, fm, rtp = ref_run(logN, mods)
        case = {
            "name": f"{name}/logN{logN}", "logN": logN, "moduli": [list(m) for m in mods],
            "runtime": rts,
            "sha256": {"input": sha(x), "twiddles": sha(tw), "inv_twiddles": sha(itw),
                       "ntt": sha(f), "ntt_mont": sha(fm), "roundtrip": sha(rtp)},
            "samples": {"input_limb0": x[0, :8].tolist(), "ntt_limb0": f[0, :8].tolist(),
                        "ntt_limb_last": f[-1, :8].tolist(), "ntt_mont_limb0": fm[0, :8].tolist(),
                        "tw_limb0": tw[0, :8].tolist()},
        }
        out["cases"].append(case)
        print(case["name"], "ok")

# full small vectors, one 30-bit and one 31-bit modulus each
for logN in (1, 2, 3, 4, 5, 6, 8):
    for start in (int(2 ** 29.5), int(2 ** 30.5)):
        mods = O.ascending_primes(logN, 1, start)
        rts, tw, itw, x, f, fm, rtp = ref_run(logN, mods)
        out["cases"].append({
            "name": f"small/logN{logN}/q{mods[0][0]}", "logN": logN, "moduli": [list(mods[0])],
            "runtime": rts, "full": {"input": x[0].tolist(), "ntt": f[0].tolist(),
                                     "ntt_mont": fm[0].tolist(), "roundtrip": rtp[0].tolist(),
                                     "twiddles": tw[0].tolist(), "inv_twiddles": itw[0].tolist()}})

path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
with open(path, "w") as fh:
    json.dump(out, fh, separators=(",", ":"))
print("wrote", path, os.path.getsize(path), "bytes")
