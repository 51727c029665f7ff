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
    # entries name configurations by their parameters, not catalogue indices
    cfgs = nb.kernel_configs()

    def sig(i):
        c = cfgs[i]
        return ",".join(str(v) for v in (c.logN, c.cluster_ctas, c.r1, c.words_log2, c.k1a, c.k2a,
                                         c.polys_per_job, c.exchange, c.k2b if c.exchange else 0))
    lines = [l.split() for l in path.read_text().splitlines()]
    mine = {l[3]: l[4] for l in lines if int(l[1]) == logN}
    assert mine == {"fwd": sig(r.fwd_index), "inv": sig(r.inv_index)}
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


def test_cache_entries_of_unknown_configurations_are_ignored(tune_cache):
    """A cache written by another build may name configurations this build
    does not compile (or bare catalogue indices of an older format): such
    entries are skipped, and plans stay on the defaults."""
    nb, path = tune_cache
    r = nb.autotune(14, 2, polys=2, iters=1)  # writes the file: learn this device's key
    dev = path.read_text().split()[0]
    path.write_text(f"{dev} 16 1 fwd 16,8,9,5,3,4,1,0,0 1.0\n"   # not compiled
                    f"{dev} 16 1 inv 26 1.0\n")                  # old index format
    nb.autotune_reload()
    mods = [(m.qi, m.primitive_root) for m in nb.find_moduli(16, 3, 1 << 29)]
    with nb.Plan(16, mods) as p:
        assert p.info.tuned == 0
    assert r.candidates > 0
