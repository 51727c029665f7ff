"""The autotuner (include/ntt_b200_tune.h): sweep, then cache.

It replaces the reference's compile-time phase-triple choice
(DefaultNTTLaunchConfig<LogN>, src/ntt_config.h:62-73).  Checked here: the
sweep writes the cache file named by NTT_B200_TUNE_CACHE; a fresh process
reads it back and its plans pick the same configurations (marked tuned);
tuned plans stay bit-exact with the oracle.  Needs a B200.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.join(os.path.dirname(__file__), "..")

CHILD = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import ntt_b200 as nb
mods = [(m.qi, m.primitive_root) for m in nb.find_moduli(int(sys.argv[2]), int(sys.argv[3]), 1 << 29)]
with nb.Plan(int(sys.argv[2]), mods) as p:
    i = p.info
    print(json.dumps({"tuned": i.tuned, "fwd": i.fwd_config, "inv": i.inv_config}))
"""


@pytest.fixture()
def tune_cache(tmp_path, monkeypatch, torch_cuda):
    import ntt_b200 as nb
    path = tmp_path / "tune" / "cache.txt"
    monkeypatch.setenv("NTT_B200_TUNE_CACHE", str(path))
    nb.autotune_reload()
    yield nb, path
    monkeypatch.delenv("NTT_B200_TUNE_CACHE")
    nb.autotune_reload()


def test_sweep_writes_cache_and_a_fresh_process_reuses_it(tune_cache):
    nb, path = tune_cache
    logN, limbs = 16, 4
    r = nb.autotune(logN, limbs, polys=4, iters=2)
    cands = [i for i, c in enumerate(nb.kernel_configs()) if c.logN == logN]
    assert r.candidates == len(cands)
    assert r.fwd_index in cands and r.inv_index in cands
    assert r.fwd_us > 0 and r.inv_us > 0
    lines = [l.split() for l in path.read_text().splitlines()]
    mine = {l[3]: int(l[4]) for l in lines if int(l[1]) == logN}
    assert mine == {"fwd": r.fwd_index, "inv": r.inv_index}
    # a plan in this process and one in a fresh process both take the entry
    mods = [(m.qi, m.primitive_root) for m in nb.find_moduli(logN, limbs, 1 << 29)]
    with nb.Plan(logN, mods) as p:
        assert (p.info.tuned, p.info.fwd_config, p.info.inv_config) == (1, r.fwd_index, r.inv_index)
    out = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(logN), str(limbs)],
                         capture_output=True, text=True, env=dict(os.environ), timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    got = json.loads(out.stdout.strip().splitlines()[-1])
    assert got == {"tuned": 1, "fwd": r.fwd_index, "inv": r.inv_index}
    # forgetting the entries puts plans back on the defaults
    nb.autotune_forget()
    with nb.Plan(logN, mods) as p:
        assert p.info.tuned == 0


@pytest.mark.parametrize("logN,limbs", [(16, 4), (14, 2)])
def test_tuned_plans_are_bit_exact(tune_cache, logN, limbs):
    nb, _ = tune_cache
    torch = pytest.importorskip("torch")
    r = nb.autotune(logN, limbs, polys=2, iters=1)
    mods = O.ascending_primes(logN, limbs, int(2 ** 29.5))
    T = O.LimbTables(logN, mods)
    x = O.uniform_limbs(logN, T.q, 5)
    with nb.Plan(logN, mods) as p:
        assert (p.info.fwd_config, p.info.inv_config) == (r.fwd_index, r.inv_index)
        d = torch.from_numpy(x.view(np.int32)).cuda()
        p.forward(d)
        torch.cuda.synchronize()
        assert np.array_equal(d.cpu().numpy().view(np.uint32), T.forward_mont(x))
        p.inverse(d)
        torch.cuda.synchronize()
        assert np.array_equal(d.cpu().numpy().view(np.uint32), x)
