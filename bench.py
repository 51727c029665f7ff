"""Benchmark: RNS negacyclic NTT + INTT roundtrip at N = 2^16, 16 limbs.

One step = forward then inverse transform (two launches, in place) over a
batch of `--polys` polynomials of 2^16 x 16 uint32 limbs (4 MiB each; the
default 64 polynomials = 256 MiB, larger than the 126 MB L2, so every step
streams from HBM).  Moduli: the 16 ascending primes q == 1 mod 2^17 from
974258177, smallest generators; coefficients uniform in [0, q) from seed
1234.  Metric: limb-NTT/s, each limb forward or inverse transform counting
one (whole job, all ranks).

Launched with torchrun for N > 1: one rank per GPU, each transforming its
own batch (limbs and polynomials are independent: weak scaling, no
collective on the data path); time = max over ranks of the device-timed
region.  `--impl reference` times the reference's CPU implementation of the
same path (oracle/_ref: its unchanged cpu_ntt_butterfly /
cpu_intt_butterfly, limbs split over all host threads) on rank 0 only.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LOGN, LIMBS, FIRST_Q, SEED = 16, 16, 974258177, 1234
METRIC = "limb-NTT/s at 2^16x16 limbs"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--polys", type=int, default=64)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--e2e-chunks", type=int, default=8)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batched-steps", type=int, default=20)
    ap.add_argument("--plain-steps", type=int, default=5)
    ap.add_argument("--no-multiply", action="store_true")
    ap.add_argument("--multiply-steps", type=int, default=10)
    ap.add_argument("--no-compressed", action="store_true")
    ap.add_argument("--no-small", action="store_true")
    ap.add_argument("--no-u64", action="store_true")
    ap.add_argument("--compressed-steps", type=int, default=50)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=20000)
    ap.add_argument("--serve-loads", type=str, default="0.5,0.8,0.95")
    return ap.parse_args()


def moduli():
    """The 16 ascending primes q == 1 (mod 2^17) from 974258177 (the library's
    own search; the tests check it against the oracle's)."""
    import ntt_b200 as nb
    return [(m.qi, m.primitive_root) for m in nb.find_moduli(LOGN, LIMBS, FIRST_Q)]


# ---------------------------------------------------------------------------
# CPU reference / baseline
# ---------------------------------------------------------------------------

def cpu_roundtrip_rate(seconds, threads):
    """Reference CPU path (oracle/_ref when built here, else the oracle port)
    on one 2^16 x 16 polynomial per repetition, forward + inverse, limbs
    split over `threads` host threads; repeated for about `seconds`."""
    from oracle import oracle as O
    mods = O.ascending_primes(LOGN, LIMBS, FIRST_Q)
    T = O.LimbTables(LOGN, mods)
    x = O.uniform_limbs(LOGN, T.q, SEED)
    R = O.ref_lib()
    kind = "reference" if R is not None else "port"
    fn = R.ref_cpu_transform_limbs if R is not None else O.lib().oracle_transform_limbs
    P = O._ptr
    reps, t0 = 0, time.perf_counter()
    a = x.copy()
    while True:
        fn(P(a), LOGN, LIMBS, P(T.q), P(T.psi_tab), None, threads)
        fn(P(a), LOGN, LIMBS, P(T.q), P(T.inv_tab), P(T.degree_inv), threads)
        reps += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    if not np.array_equal(a, x):
        raise RuntimeError("CPU reference roundtrip is not the identity")
    return 2 * LIMBS * reps / el, kind, reps, el


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return  # other ranks exit 0 without work
    threads = os.cpu_count() or 1
    rates = []
    for _ in range(max(args.warmup, 0)):
        cpu_roundtrip_rate(0.0, threads)
    t_total = time.perf_counter()
    for _ in range(max(1, args.steps if args.steps <= 50 else 50)):
        r, kind, reps, el = cpu_roundtrip_rate(0.0, threads)
        rates.append(r)
    total = time.perf_counter() - t_total
    value = float(np.median(rates))
    steps = len(rates)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "limb-NTT/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * total / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": "NTT+INTT roundtrip, N=2^16, 16 limbs, 1 polynomial per step "
                               "(CPU: one 4 MiB polynomial per step)",
                   "moduli": f"16 ascending primes q=1 mod 2^17 from {FIRST_Q}", "seed": SEED},
        "cpu_baseline": {"value": value, "unit": "limb-NTT/s", "cores": threads, "kind": kind,
                         "sample": "one 2^16 x 16-limb polynomial forward+inverse per step"},
        "e2e": {"value": value, "unit": "limb-NTT/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clock / throttle sampling while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.dev)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [v.strip() for v in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(value_ms: float, device: str = "cuda") -> float:
    """The job's time: the slowest rank's (a no-op with one process)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value_ms)
    t = torch.tensor([float(value_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_env():
    """(world, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def relaunch_under_torchrun(gpus: int) -> int:
    """`--gpus N` (N > 1) started as a plain process: run this same command
    line as N ranks under torch.distributed.run (one process per GPU,
    rendezvous on 127.0.0.1) and return its exit status."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={gpus}", "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def init_ranks(args, backend="nccl"):
    """Join the process group of a multi-rank run (short timeout, so that a
    rank that never arrives ends the others' waits with an error); the
    world size must be the `--gpus` asked for."""
    import datetime
    import torch.distributed as dist
    world, rank, local = rank_env()
    if world != args.gpus:
        raise SystemExit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}")
    if world > 1:
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def run_ours(args):
    import torch
    import torch.distributed as dist

    world, rank, local = init_ranks(args)
    torch.cuda.set_device(local)
    import ntt_b200 as nb

    mods = moduli()
    plan = nb.Plan(LOGN, mods)
    N = 1 << LOGN
    P = args.polys
    words = P * LIMBS * N
    q = np.array([m[0] for m in mods], dtype=np.uint64)
    rng = np.random.default_rng(SEED + rank)
    x = rng.integers(0, q[None, :, None], size=(P, LIMBS, N), dtype=np.uint64).astype(np.uint32)
    host_in = torch.from_numpy(x.reshape(-1).view(np.int32)).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    d = torch.empty(words, dtype=torch.int32, device="cuda")
    d.copy_(host_in)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # sanity check of the timed path (bit-exact parity is the tests' job)
    with torch.cuda.stream(stream):
        plan.forward_many(d, P, 0, stream=sh)
        plan.inverse_many(d, P, 0, stream=sh)
    stream.synchronize()
    if not torch.equal(d, host_in.cuda()):
        raise RuntimeError("roundtrip is not the identity")

    # warm-up
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            plan.forward_many(d, P, 0, stream=sh)
            plan.inverse_many(d, P, 0, stream=sh)
    barrier()

    K = args.steps
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4 * K)]
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.25)
    barrier()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        t_start.record(stream)
        for k in range(K):
            ev[4 * k].record(stream)
            plan.forward_many(d, P, 0, stream=sh)
            ev[4 * k + 1].record(stream)
            ev[4 * k + 2].record(stream)
            plan.inverse_many(d, P, 0, stream=sh)
            ev[4 * k + 3].record(stream)
        t_end.record(stream)
    stream.synchronize()
    barrier()
    clocks = sampler.stop()
    elapsed_ms = t_start.elapsed_time(t_end)
    fwd_ms = np.array([ev[4 * k].elapsed_time(ev[4 * k + 1]) for k in range(K)])
    inv_ms = np.array([ev[4 * k + 2].elapsed_time(ev[4 * k + 3]) for k in range(K)])
    elapsed_max = max_over_ranks(elapsed_ms)

    # e2e through the public API with host buffers (pinned), copies timed.
    # The step's polynomials move in chunks on three streams -- host-to-device
    # copy, transforms, device-to-host copy -- so the two copy directions
    # (separate copy engines, full-duplex PCIe) and the transforms overlap;
    # every step still copies all P polynomials in and all results out.
    E = max(1, args.e2e_steps)
    chunks = max(1, min(args.e2e_chunks, P))
    bounds = [P * c // chunks for c in range(chunks + 1)]
    words_per_poly = LIMBS * N
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    host_out.zero_()
    barrier()
    e0.record(s_in)
    stream.wait_event(e0)
    s_out.wait_event(e0)
    done = [None] * chunks  # per chunk: its results have left the device
    for _ in range(E):
        for c in range(chunks):
            lo, hi = bounds[c] * words_per_poly, bounds[c + 1] * words_per_poly
            ev_in, ev_tr, ev_done = torch.cuda.Event(), torch.cuda.Event(), torch.cuda.Event()
            if done[c] is not None:  # the previous step's results of this chunk
                s_in.wait_event(done[c])
            with torch.cuda.stream(s_in):
                d[lo:hi].copy_(host_in[lo:hi], non_blocking=True)
                ev_in.record(s_in)
            stream.wait_event(ev_in)
            plan.forward_many(d[lo:hi], bounds[c + 1] - bounds[c], 0, stream=sh)
            plan.inverse_many(d[lo:hi], bounds[c + 1] - bounds[c], 0, stream=sh)
            ev_tr.record(stream)
            s_out.wait_event(ev_tr)
            with torch.cuda.stream(s_out):
                host_out[lo:hi].copy_(d[lo:hi], non_blocking=True)
                ev_done.record(s_out)
            done[c] = ev_done
    s_in.wait_stream(stream)
    s_in.wait_stream(s_out)
    e1.record(s_in)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    if not torch.equal(host_out, host_in):
        raise RuntimeError("e2e roundtrip is not the identity")

    # the plain per-call form of the same workload: one forward and one
    # inverse call per polynomial (the reference driver's usage pattern)
    views = [d[p * LIMBS * N:(p + 1) * LIMBS * N] for p in range(P)]

    def per_call_step():
        for v in views:
            plan.forward(v, sh)
            plan.inverse(v, sh)
    per_call_ms = device_time(torch, stream, per_call_step, max(3, K // 100), 3)
    per_call_ms = max_over_ranks(per_call_ms)
    # host time to submit one step's calls (the stream is idle at the start,
    # and 2P launches stay far below the launch queue's depth, so nothing
    # blocks): when it reaches the device time per launch, the per-call
    # figure is the host's submission rate, not the kernels'
    torch.cuda.synchronize()
    t_host = time.perf_counter()
    per_call_step()
    host_us_per_launch = (time.perf_counter() - t_host) * 1e6 / (2 * P)
    torch.cuda.synchronize()

    transforms = 2 * P * LIMBS * K * world
    value = transforms / (elapsed_max / 1000.0)
    e2e_value = 2 * P * LIMBS * E * world / (e2e_ms / 1000.0)

    # roofline of the dominant kernel: algorithmic bytes = read + write of
    # every word once per launch (8 bytes per coefficient)
    alg_bytes = 8.0 * P * LIMBS * N
    fwd_avg, inv_avg = float(fwd_ms.mean()), float(inv_ms.mean())
    dom, dom_ms = ("forward", fwd_avg) if fwd_avg >= inv_avg else ("inverse", inv_avg)
    kname = kernel_name(nb, plan.info, dom)
    achieved = alg_bytes / (dom_ms / 1000.0) / 1e9
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak, peak_src = json.load(open(peaks_path))["hbm_gbs"], "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tpath):
        tj = json.load(open(tpath))
        per = tj.get(dom)
        if per:
            traffic = per["bytes_per_coefficient"] * P * LIMBS * N

    # integer-multiply roofline of the same kernel: 3 32-bit multiplies per
    # Shoup butterfly (the normal->Montgomery and N^-1 folds ride on stage 0)
    int_peak = nb.measure_int_peak()
    muls = 3.0 * (N // 2) * LOGN * P * LIMBS
    int_achieved = muls / (dom_ms / 1000.0)

    out = {
        "metric": METRIC, "value": value, "unit": "limb-NTT/s", "n_gpus": world,
        "steps": K, "warmup": args.warmup, "ms_per_step": elapsed_max / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic",
        "config": {"workload": f"NTT+INTT roundtrip, N=2^16, 16 limbs, {P} polynomials per "
                               "rank per step (in place, one launch per direction)",
                   "moduli": f"16 ascending primes q=1 mod 2^17 from {FIRST_Q}",
                   "seed": SEED, "parallelism": f"dp{world} (independent polynomials)",
                   "l2": f"inputs {P * LIMBS * N * 4 >> 20} MiB per rank > 126 MB L2, "
                         "no flush needed"},
        "e2e": {"value": e2e_value, "unit": "limb-NTT/s",
                "h2d_bytes_per_step": P * LIMBS * N * 4, "d2h_bytes_per_step": P * LIMBS * N * 4,
                "steps": E,
                "pipeline": f"{chunks} chunks of polynomials on 3 streams (host-to-device copy, "
                            "forward + inverse, device-to-host copy)"},
        "gpu_launches": 2 * K,
        "per_call": {"value": 2 * P * LIMBS * world / (per_call_ms / 1000.0), "unit": "limb-NTT/s",
                     "ms_per_step": per_call_ms, "launches_per_step": 2 * P,
                     "device_us_per_launch": per_call_ms * 1000.0 / (2 * P),
                     "host_us_per_launch": host_us_per_launch,
                     "form": "one ntt_forward + one ntt_inverse call per polynomial "
                             "(Python through ctypes)"},
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_source": peak_src,
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "forward_ms": fwd_avg, "inverse_ms": inv_avg},
        "int_roofline": {"bound": "int-multiply", "kernel": kname,
                         "achieved": int_achieved / 1e12, "peak": int_peak / 1e12,
                         "unit": "T mul/s", "frac": int_achieved / int_peak,
                         "peak_source": "measured (ntt_measure_int_peak: Shoup mul.hi + "
                                        "2 mul.lo chains on every SM)",
                         "algorithmic_muls_per_launch": muls},
        "clocks": clocks,
    }
    info = plan.info
    out["config"]["kernel"] = {"cluster_ctas": info.cluster_ctas,
                               "threads_per_cta": info.threads_per_cta,
                               "smem_bytes": info.smem_bytes,
                               "phases": [info.effective.ntt_phase1.as_tuple(),
                                          info.effective.ntt_phase2.as_tuple()]}
    if not args.no_batched:
        out["batched"] = bench_batched(args, torch, nb, stream)
        out["gpu_launches_batched"] = 2 * (args.batched_steps + args.plain_steps *
                                           out["batched"]["polynomials"])
    if not args.no_multiply:
        out["fused_multiply"] = bench_multiply(args, torch, nb, stream)
    if not args.no_compressed:
        out["compressed_twiddles"] = bench_compressed(args, torch, nb, stream, d, P)
    if not args.no_small:
        out["small_sizes"] = bench_small(args, torch, nb, stream)
    if not args.no_u64:
        out["u64"] = bench_u64(args, torch, nb, stream)
    if not args.no_serve:
        out["serve"] = bench_serve(args, torch, nb)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, kind, reps, el = cpu_roundtrip_rate(args.cpu_seconds, threads)
        out["cpu_baseline"] = {"value": rate, "unit": "limb-NTT/s", "cores": threads,
                               "kind": kind,
                               "sample": f"{reps} forward+inverse roundtrips of one 2^16 x 16 "
                                         f"polynomial in {el:.1f} s"}
    out["summary"] = summary(out)  # last key: the compact figures survive a cut stdout tail
    if rank == 0:
        print(json.dumps(out))
    plan.close()
    if world > 1:
        dist.destroy_process_group()


def summary(out):
    """The headline figures of every leg in a few hundred bytes."""
    r = lambda v, n=3: None if v is None else round(float(v), n)
    s = {"value": r(out["value"], 1), "e2e": r(out["e2e"]["value"], 1),
         "roofline_frac": r(out["roofline"]["frac"]),
         "forward_ms": r(out["roofline"]["forward_ms"], 4),
         "inverse_ms": r(out["roofline"]["inverse_ms"], 4)}
    if "per_call" in out:
        s["per_call_value"] = r(out["per_call"]["value"], 1)
        s["per_call_us_per_launch_device_host"] = [r(out["per_call"]["device_us_per_launch"]),
                                                   r(out["per_call"]["host_us_per_launch"])]
    if "batched" in out:
        s["batched_value"] = r(out["batched"]["value"], 1)
        s["batched_speedup_vs_plain"] = r(out["batched"]["speedup_vs_plain"])
    if "fused_multiply" in out:
        fm = out["fused_multiply"]
        s["multiply_speedup_vs_unfused"] = r(fm["speedup_vs_unfused"])
        s["multiply_batch_tiles_speedup_vs_unfused"] = r(fm["batch_tiles"]["speedup_vs_unfused"])
        s["multiply_spectrum_speedup_vs_unfused"] = r(fm["spectrum"]["speedup_vs_unfused"])
        s["multiply_one_launch_speedup_vs_unfused"] = r(fm["one_launch"]["speedup_vs_unfused"])
    if "small_sizes" in out:
        s["small_warp_speedup_vs_shared"] = {k: r(v["speedup_vs_shared"])
                                             for k, v in out["small_sizes"].items()
                                             if isinstance(v, dict)}
    if "u64" in out:
        s["u64_value"] = r(out["u64"]["value"], 1)
        s["u64_hbm_frac"] = r(out["u64"]["roofline"]["frac"])
    if "compressed_twiddles" in out:
        ct = out["compressed_twiddles"]
        s["compressed_headline_ratio"] = r(ct["headline"]["speedup_vs_full"])
        s["compressed_table_bound_ratio"] = r(ct["table_bound"]["speedup_vs_full"])
    if "serve" in out:
        for leg in ("host", "device"):
            L = out["serve"][leg]
            b, p = L["batched"], L["per_call"]
            s[f"serve_{leg}_capacity_ratio"] = r(L["capacity_speedup_vs_per_call"])
            s[f"serve_{leg}_batched_rps"] = r(b["capacity"]["achieved_rps"], 1)
            s[f"serve_{leg}_p99_ms"] = [r(x["p99_ms"]) for x in b["poisson"]]
            s[f"serve_{leg}_per_call_p99_ms_at_half"] = r(p["poisson"][0]["p99_ms"])
    if "cpu_baseline" in out:
        s["cpu_baseline"] = r(out["cpu_baseline"]["value"], 1)
    return s


RAGGED = dict(seed=SEED, count=256, logn=tuple(range(12, 17)), limbs=(1, 48), bits=(30,))


def bench_u64(args, torch, nb, stream):
    """64-bit words: 16 polynomials of 2^16 x 16 limbs of primes below 2^60
    (ntt64_find_moduli from 2^59; 128 MiB > L2), step = forward + inverse,
    CUDA events.  Algorithmic bytes per launch: 16 per coefficient (read and
    write of 8-byte words); the kernels run the column and the row stages as
    two launches per direction, so their traffic is twice that."""
    sh = stream.cuda_stream
    logN, limbs, polys = 16, 16, 16
    mods = nb.find_moduli64(logN, limbs, 1 << 59)
    g = torch.Generator(device="cuda")
    g.manual_seed(SEED)
    x = torch.randint(0, 1 << 59, (polys * limbs << logN,), generator=g, device="cuda",
                      dtype=torch.int64)
    x0 = x.clone()
    p = nb.Plan64(logN, mods)
    with torch.cuda.stream(stream):
        p.forward_many(x, polys, 0, sh)
        p.inverse_many(x, polys, 0, sh)
    stream.synchronize()
    if not torch.equal(x, x0):
        raise RuntimeError("64-bit roundtrip is not the identity")
    del x0
    K = 50
    fwd = device_time(torch, stream, lambda: p.forward_many(x, polys, 0, sh), K, 3)
    inv = device_time(torch, stream, lambda: p.inverse_many(x, polys, 0, sh), K, 3)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = json.load(open(peaks_path))["hbm_gbs"] if os.path.exists(peaks_path) else 6650.0
    alg = 16.0 * polys * limbs * (1 << logN)
    dom = max(fwd, inv)
    p.close()
    return {"workload": f"{polys} x 2^{logN} x {limbs} limbs of primes below 2^60 (64-bit "
                        "words), forward + inverse",
            "value": 2 * polys * limbs / ((fwd + inv) / 1000.0), "unit": "limb-NTT/s",
            "forward_ms": fwd, "inverse_ms": inv,
            "roofline": {"bound": "hbm", "achieved": alg / (dom / 1000.0) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": alg / (dom / 1000.0) / 1e9 / peak,
                         "algorithmic_bytes_per_launch": alg,
                         "note": "two launches per direction: traffic is twice the "
                                 "algorithmic bytes"}}


def bench_small(args, torch, nb, stream):
    """Small limbs (logN 6 and 9, 16 limbs of 30-bit primes, 2048
    polynomials = 8 / 64 MiB), step = forward + inverse, CUDA events: the
    warp-per-limb kernel (registers, the last five stages through shfl.xor)
    against the shared-memory kernel (a CTA per limb, one shared-memory round
    and one barrier per stage).  Same words (checked)."""
    from ntt_b200 import mixes
    sh = stream.cuda_stream
    res = {}
    for logN in (6, 9):
        limbs, polys = 16, 2048
        mods = list(mixes.prime_pool(logN, 30, limbs))
        job = mixes.MixJob(nb.OP_FORWARD, logN, mods)
        g = torch.Generator(device="cuda")
        g.manual_seed(SEED + logN)
        x = torch.stack([mixes.uniform_device(torch, job, g) for _ in range(polys)])
        pw, ps = nb.Plan(logN, mods), nb.Plan(logN, mods)
        ps.set_small_kernel(nb.SMALL_SHARED)
        y = x.clone()
        with torch.cuda.stream(stream):
            pw.forward_many(x, polys, 0, sh)
            ps.forward_many(y, polys, 0, sh)
        stream.synchronize()
        if not torch.equal(x, y):
            raise RuntimeError("warp and shared-memory kernels differ")
        del y

        def step(p):
            return lambda: (p.forward_many(x, polys, 0, sh), p.inverse_many(x, polys, 0, sh))
        t_w = device_time(torch, stream, step(pw), 50, 5)
        t_s = device_time(torch, stream, step(ps), 50, 5)
        res[f"logN{logN}"] = {
            "workload": f"{polys} x 2^{logN} x {limbs} limbs, forward + inverse",
            "warp_ms": t_w, "shared_ms": t_s, "speedup_vs_shared": t_s / t_w,
            "warp_limb_ntt_per_s": 2 * polys * limbs / (t_w / 1000.0)}
        pw.close()
        ps.close()
    return res


def bench_compressed(args, torch, nb, stream, d, P):
    """Full against compressed twiddle tables (NTT_PLAN_COMPRESSED_TWIDDLES:
    3N/16 + 16 pairs per limb instead of N, the last four stages multiplying
    by two factors).  Two workloads, device-resident, step = forward +
    inverse, CUDA events:
      headline: the headline batch (64 x 2^16 x 16 limbs; 16 MiB of full
        tables, L2-resident either way): the compute cost of compression;
      table_bound: 4 plans of disjoint 32-limb chains of 30-bit primes at
        logN 17, one polynomial per call through each plan in turn (the
        per-ciphertext pattern of RNS schemes): full tables 4 x 2 x 32 MiB =
        256 MiB cycle through the 126 MB L2, compressed ones 48 MiB.
    Both forms give the same words (checked)."""
    sh = stream.cuda_stream
    K = args.compressed_steps
    res = {}
    # headline workload
    mods = moduli()
    pf = nb.Plan(16, mods)
    pc = nb.Plan(16, mods, compressed_twiddles=True)
    x = d.clone()
    with torch.cuda.stream(stream):
        pc.forward_many(x, P, 0, sh)
    y = d.clone()
    with torch.cuda.stream(stream):
        pf.forward_many(y, P, 0, sh)
    stream.synchronize()
    if not torch.equal(x, y):
        raise RuntimeError("compressed and full tables differ (headline)")
    del y

    def step(p):
        return lambda: (p.forward_many(x, P, 0, sh), p.inverse_many(x, P, 0, sh))
    t_full = device_time(torch, stream, step(pf), K, 3)
    t_comp = device_time(torch, stream, step(pc), K, 3)
    res["headline"] = {"workload": f"{P} x 2^16 x 16 limbs (default moduli), forward + inverse",
                       "full_ms": t_full, "compressed_ms": t_comp,
                       "speedup_vs_full": t_full / t_comp,
                       "table_bytes_full": pf.info.device_bytes,
                       "table_bytes_compressed": pc.info.device_bytes}
    pf.close()
    pc.close()
    # table-bound workload
    logN, limbs, chains = 17, 32, 4
    # disjoint chains: 32 primes q = 1 mod 2^18 span < 2^27, all below 2^30
    starts = [(1 << 29) + k * (1 << 27) for k in range(chains)]
    chain = [nb.find_moduli(logN, limbs, s0) for s0 in starts]
    plans_f = [nb.Plan(logN, c) for c in chain]
    plans_c = [nb.Plan(logN, c, compressed_twiddles=True) for c in chain]
    g = torch.Generator(device="cuda")
    g.manual_seed(SEED)
    polys = [torch.randint(0, 1 << 29, (limbs << logN,), generator=g, device="cuda",
                           dtype=torch.int32) for _ in range(chains)]
    chk = [p.clone() for p in polys]
    with torch.cuda.stream(stream):
        for p, v in zip(plans_c, polys):
            p.forward(v, sh)
        for p, v in zip(plans_f, chk):
            p.forward(v, sh)
    stream.synchronize()
    if not all(torch.equal(a, b) for a, b in zip(polys, chk)):
        raise RuntimeError("compressed and full tables differ (table-bound)")
    del chk

    def cycle(plans):
        def fn():
            for p, v in zip(plans, polys):
                p.forward(v, sh)
                p.inverse(v, sh)
        return fn
    t_full = device_time(torch, stream, cycle(plans_f), K, 3)
    t_comp = device_time(torch, stream, cycle(plans_c), K, 3)
    res["table_bound"] = {
        "workload": f"{chains} chains x 2^{logN} x {limbs} limbs of 30-bit primes, one "
                    "polynomial per call, forward + inverse through each plan in turn",
        "full_ms": t_full, "compressed_ms": t_comp, "speedup_vs_full": t_full / t_comp,
        "limb_ntt_per_s_full": 2 * chains * limbs / (t_full / 1000.0),
        "limb_ntt_per_s_compressed": 2 * chains * limbs / (t_comp / 1000.0),
        "table_bytes_full": sum(p.info.device_bytes for p in plans_f),
        "table_bytes_compressed": sum(p.info.device_bytes for p in plans_c)}
    for p in plans_f + plans_c:
        p.close()
    res["steps"] = K
    return res


def device_time(torch, stream, fn, steps, warmup):
    """Average device time (ms) of fn() over `steps` runs on `stream` after
    `warmup` untimed runs (CUDA events on the launching stream)."""
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            fn()
    stream.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
    stream.synchronize()
    return e0.elapsed_time(e1) / steps


def bench_batched(args, torch, nb, stream):
    """Ragged batch: 256 polynomials, logN uniform in 12..16, limbs uniform
    in 1..48, each with its own chain of 30-bit primes, uniform [0, q)
    coefficients.  Step = forward + inverse of every polynomial.  Batched
    form: two persistent launches (CUDA-graph replays); plain form: one
    ntt_forward + one ntt_inverse call per polynomial (512 launches)."""
    from ntt_b200 import mixes
    jobs = mixes.ragged_mix(**RAGGED)
    g = torch.Generator(device="cuda")
    g.manual_seed(SEED)
    data = [mixes.uniform_device(torch, j, g) for j in jobs]
    orig = [x.clone() for x in data]
    limbs = sum(j.limbs for j in jobs)
    words = sum(j.words for j in jobs)
    sh = stream.cuda_stream
    plans = [nb.Plan(j.logN, j.moduli) for j in jobs]

    def plain():
        for p, x in zip(plans, data):
            p.forward(x, sh)
            p.inverse(x, sh)

    bf = nb.Batch([(nb.OP_FORWARD, j.logN, j.moduli, x, None) for j, x in zip(jobs, data)])
    bi = nb.Batch([(nb.OP_INVERSE, j.logN, j.moduli, x, None) for j, x in zip(jobs, data)])

    def batched():
        bf.run(sh)
        bi.run(sh)

    w = max(3, args.warmup if args.warmup < 10 else 10)
    plain_ms = device_time(torch, stream, plain, args.plain_steps, w)
    batch_ms = device_time(torch, stream, batched, args.batched_steps, w)
    for x, o in zip(data, orig):  # every step is a roundtrip: data must be unchanged
        if not torch.equal(x, o):
            raise RuntimeError("batched / plain roundtrips changed the data")
    info = bf.info
    res = {
        "workload": "256 ragged polynomials: logN uniform 12..16, limbs uniform 1..48, own "
                    "chains of 30-bit primes q=1 mod 2N, uniform [0,q) coefficients; step = "
                    "forward + inverse of every polynomial",
        "polynomials": len(jobs), "limbs": limbs, "bytes": 4 * words,
        "value": 2 * limbs / (batch_ms / 1000.0), "unit": "limb-NTT/s",
        "ms_per_step": batch_ms, "launches_per_step": 2,
        "plain_per_call": {"value": 2 * limbs / (plain_ms / 1000.0), "unit": "limb-NTT/s",
                           "ms_per_step": plain_ms, "launches_per_step": 2 * len(jobs)},
        "speedup_vs_plain": plain_ms / batch_ms,
        "kernel": {"cluster_ctas": info.cluster_ctas, "clusters": info.clusters,
                   "groups": info.groups, "smem_bytes": info.smem_bytes},
        "steps": args.batched_steps, "plain_steps": args.plain_steps, "warmup": w,
        "l2": f"{4 * words >> 20} MiB of inputs > 126 MB L2",
    }
    bf.close()
    bi.close()
    for p in plans:
        p.close()
    return res


def kernel_name(nb, info, direction):
    """The kernel template a plan launches for one direction, as the launch
    list names it: split_kernel (phases meeting in place through L2) or
    fused_kernel (phases meeting in the cluster's shared memory)."""
    idx = info.fwd_config if direction == "forward" else info.inv_config
    c = nb.kernel_configs()[idx]
    if c.exchange == 1:
        return (f"split_kernel<SplitGeo<{c.logN}, {c.cluster_ctas.bit_length() - 1}, "
                f"{c.words_log2}, {c.k2a}, {c.k2b}>> ({direction})")
    return (f"fused_kernel ({direction}; {c.cluster_ctas} CTAs, r1 {c.r1}, "
            f"{1 << c.words_log2} words per thread)")


def bench_multiply(args, torch, nb, stream):
    """Fused negacyclic multiply: 128 pairs of 2^16 x 24-limb polynomials
    (24 ascending 30-bit primes q == 1 mod 2^17 above 2^29.5), uniform [0, q)
    coefficients; c = a * b into b's buffer.  Fused: ntt_multiply_many in its
    default form on this split plan -- NTT(b) with the split kernel, NTT(a)
    with the pointwise Montgomery product folded into its store into b (a
    cluster kernel: a is only read), INTT(b) with the split kernel (28 bytes
    per coefficient) -- and, as `one_launch`, the split multiply kernel (NTT(b),
    NTT(a), product and INTT per (pair, limb) in one launch: a read once, b
    read and written once, 12 bytes per coefficient).  Unfused: the plain calls
    forward_many(a), forward_many(b), pointwise_mul, inverse_many(b) (4
    launches, 36 bytes per coefficient; a is overwritten by its spectrum,
    which favours it).  Batch tiles: the same products as multiply tiles of
    the ragged-batch kernel (one launch; the serving path's form)."""
    from ntt_b200 import mixes
    logN, limbs, pairs = 16, 24, 128
    mods = list(mixes.prime_pool(logN, 30, limbs))
    job = mixes.MixJob(nb.OP_MULTIPLY, logN, mods)
    g = torch.Generator(device="cuda")
    g.manual_seed(SEED)
    a = torch.stack([mixes.uniform_device(torch, job, g) for _ in range(pairs)])
    b = torch.stack([mixes.uniform_device(torch, job, g) for _ in range(pairs)])
    sh = stream.cuda_stream
    p = nb.Plan(logN, mods)
    tiles = nb.Batch([(nb.OP_MULTIPLY, logN, mods, b[i], a[i]) for i in range(pairs)])
    # consistency of the forms on this workload (parity is the tests' job)
    b0 = b.clone()
    ta, tb = a.clone(), b.clone()
    with torch.cuda.stream(stream):
        p.forward_many(ta, pairs, 0, sh)
        p.forward_many(tb, pairs, 0, sh)
        p.pointwise_mul(tb, ta, tb, pairs, 0, sh)
        p.inverse_many(tb, pairs, 0, sh)
        tiles.run(sh)
    stream.synchronize()
    if not torch.equal(b, tb):
        raise RuntimeError("batch-tile and unfused multiply differ")
    pb = b0.clone()
    b3 = b0.clone()  # the three-launch form's operand (b holds the tiles' product by now)
    with torch.cuda.stream(stream):
        p.multiply_many(a, pb, pairs, 0, sh)
    stream.synchronize()
    if not torch.equal(pb, tb):
        raise RuntimeError("fused and unfused multiply differ")
    del b0

    def unfused():
        p.forward_many(ta, pairs, 0, sh)
        p.forward_many(tb, pairs, 0, sh)
        p.pointwise_mul(tb, ta, tb, pairs, 0, sh)
        p.inverse_many(tb, pairs, 0, sh)

    # the product with a resident spectrum (a transformed once, outside the
    # timed region): two launches on split plans against forward, pointwise,
    # inverse
    spec = a.clone()
    with torch.cuda.stream(stream):
        p.forward_many(spec, pairs, 0, sh)
        sb, su = b.clone(), b.clone()
        p.multiply_spectrum_many(spec, sb, pairs, 0, sh)
        p.forward_many(su, pairs, 0, sh)
        p.pointwise_mul(su, spec, su, pairs, 0, sh)
        p.inverse_many(su, pairs, 0, sh)
    stream.synchronize()
    if not torch.equal(sb, su):
        raise RuntimeError("spectrum product and its unfused form differ")

    def spec_unfused():
        p.forward_many(su, pairs, 0, sh)
        p.pointwise_mul(su, spec, su, pairs, 0, sh)
        p.inverse_many(su, pairs, 0, sh)

    w = 3
    spec_ms = device_time(torch, stream, lambda: p.multiply_spectrum_many(spec, sb, pairs, 0, sh),
                          args.multiply_steps, w)
    spec_unfused_ms = device_time(torch, stream, spec_unfused, args.multiply_steps, w)
    del su
    fused_ms = device_time(torch, stream, lambda: p.multiply_many(a, pb, pairs, 0, sh),
                           args.multiply_steps, w)
    # the one-launch form on the same (split) plan
    p3 = nb.Plan(logN, mods)
    p3.set_multiply_form(nb.MULTIPLY_ONE_LAUNCH)
    p3b = b3
    with torch.cuda.stream(stream):
        p3.multiply_many(a, p3b, pairs, 0, sh)
    stream.synchronize()
    if not torch.equal(p3b, tb):
        raise RuntimeError("one-launch and unfused multiply differ")
    one_ms = device_time(torch, stream, lambda: p3.multiply_many(a, p3b, pairs, 0, sh),
                           args.multiply_steps, w)
    p3.close()
    del p3b
    unfused_ms = device_time(torch, stream, unfused, args.multiply_steps, w)
    tiles_ms = device_time(torch, stream, lambda: tiles.run(sh), args.multiply_steps, w)
    products = pairs * limbs
    words = pairs * limbs << logN
    res = {
        "workload": f"{pairs} pairs of 2^{logN} x {limbs}-limb polynomials, 30-bit primes, "
                    "c = a*b negacyclic per limb into b",
        "value": products / (fused_ms / 1000.0), "unit": "limb-products/s",
        "limb_ntt_per_s": 3 * products / (fused_ms / 1000.0),
        "ms_per_step": fused_ms, "launches_per_step": 3,
        "form": "ntt_multiply_many (default form on split plans: split NTT(b), cluster NTT(a) "
                "with the product folded into its store into b, split INTT(b))",
        "algorithmic_bytes": 28 * words,
        "achieved_gbs": 28 * words / (fused_ms / 1000.0) / 1e9,
        "unfused": {"value": products / (unfused_ms / 1000.0), "ms_per_step": unfused_ms,
                    "launches_per_step": 4, "algorithmic_bytes": 36 * words},
        "speedup_vs_unfused": unfused_ms / fused_ms,
        "one_launch": {"form": "the split multiply kernel: NTT(b), NTT(a), product, INTT per "
                               "(pair, limb) in one launch",
                       "value": products / (one_ms / 1000.0), "ms_per_step": one_ms,
                       "launches_per_step": 1, "speedup_vs_unfused": unfused_ms / one_ms},
        "spectrum": {"form": "ntt_multiply_spectrum_many with NTT(a) resident: forward of b "
                             "with the product on its final store, inverse (2 launches)",
                     "value": products / (spec_ms / 1000.0), "ms_per_step": spec_ms,
                     "launches_per_step": 2, "unfused_ms": spec_unfused_ms,
                     "unfused_form": "forward(b), pointwise_mul, inverse(b) (3 launches)",
                     "speedup_vs_unfused": spec_unfused_ms / spec_ms},
        "batch_tiles": {"value": products / (tiles_ms / 1000.0), "ms_per_step": tiles_ms,
                        "launches_per_step": 1, "speedup_vs_unfused": unfused_ms / tiles_ms,
                        "cluster_ctas": tiles.info.cluster_ctas, "clusters": tiles.info.clusters},
        "steps": args.multiply_steps, "warmup": w,
    }
    tiles.close()
    p.close()
    return res


SERVE = dict(seed=SEED, logn=tuple(range(12, 18)), limbs=(1, 64), bits=(30, 31),
             ops=((0, 0.4), (1, 0.4), (2, 0.2)))


def bench_serve(args, torch, nb):
    """Serving stream: requests with logN uniform in 12..17, limbs uniform in
    1..64, 30/31-bit moduli chains, 40% NTT / 40% INTT / 20% multiply.
    Two legs: host buffers (pinned; each request's polynomial crosses PCIe
    both ways) and device-resident buffers (each request transformed where
    it lies in HBM: the GPU is the bound).  In each leg the batched server
    (rounds of up to 1024 tiles, 4 rounds in flight) is compared with the
    plain per-call form: the same server with one request per launch and
    the same 4 stream slots, so the ratio isolates batching.  Capacity = all
    requests submitted at once; then Poisson arrivals at fractions of that
    capacity (open loop), p50/p99 of submit -> result (in the host buffer,
    or on the device)."""
    from ntt_b200 import mixes
    jobs = mixes.ragged_mix(count=args.serve_requests, **SERVE)
    for lg in SERVE["logn"]:
        for b in SERVE["bits"]:
            nb.tables_preload(lg, mixes.prime_pool(lg, b, 96))
    gen = torch.Generator().manual_seed(SEED)
    limb_ntts = sum(j.limbs * (3 if j.op == nb.OP_MULTIPLY else 1) for j in jobs)
    pcie = sum(j.words * 4 * (3 if j.op == nb.OP_MULTIPLY else 2) for j in jobs)
    # host leg: inputs < 2^29 are valid for every op and modulus; outputs of
    # the same logN share one pinned buffer (their contents are not checked)
    hpool = {lg: torch.randint(0, 1 << 29, (64, 1 << lg), dtype=torch.int32, generator=gen)
                  .pin_memory().numpy().view(np.uint32) for lg in SERVE["logn"]}
    hsink = {lg: torch.empty((64, 1 << lg), dtype=torch.int32).pin_memory().numpy()
                  .view(np.uint32) for lg in SERVE["logn"]}
    # device leg: requests run in place on a ring of device slots per logN;
    # multiply operands come from a read-only device pool
    RING = 32
    dpool = {lg: torch.randint(0, 1 << 29, (64, 1 << lg), dtype=torch.int32, device="cuda")
             for lg in SERVE["logn"]}
    dring = {lg: torch.randint(0, 1 << 29, (RING, 64, 1 << lg), dtype=torch.int32,
                               device="cuda") for lg in SERVE["logn"]}

    def prepare(srv, device):
        out, k = [], {lg: 0 for lg in SERVE["logn"]}
        for j in jobs:
            if device:
                slot = dring[j.logN][k[j.logN] % RING][:j.limbs]
                k[j.logN] += 1
                x = o = slot
                a = dpool[j.logN][:j.limbs] if j.op == nb.OP_MULTIPLY else None
            else:
                x, o = hpool[j.logN][:j.limbs], hsink[j.logN][:j.limbs]
                a = x if j.op == nb.OP_MULTIPLY else None
            out.append(srv.request(j.op, j.logN, j.moduli, x, o, operand=a, device=device))
        return out

    def run(srv, reqs, rate):
        srv.stats(reset=True)
        rng = np.random.default_rng(SEED)
        gaps = rng.exponential(1.0 / rate, len(reqs)) if rate else None
        t_next = time.perf_counter()
        tickets = []
        for i, r in enumerate(reqs):
            if gaps is not None:
                t_next += gaps[i]
                while True:
                    dt = t_next - time.perf_counter()
                    if dt <= 0:
                        break
                    if dt > 2e-4:
                        time.sleep(dt - 1e-4)
            tickets.append(srv.submit_prepared(r))
        for t in tickets:
            srv.wait(t, 300.0)
        st = srv.stats(reset=True)
        return {"offered_rps": rate, "achieved_rps": len(reqs) / st["elapsed_s"],
                "limb_ntt_per_s": st["limb_ntt_per_s"], "p50_ms": st["p50_ms"],
                "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"], "max_ms": st["max_ms"],
                "rounds": st["rounds"], "mean_round_requests": st["mean_round_requests"],
                "arena_peak_bytes": st["arena_peak_bytes"], "elapsed_s": st["elapsed_s"]}

    def form(device, batched, loads):
        kw = {} if batched else {"max_round_requests": 1}
        with nb.Server(streams=4, **kw) as srv:
            reqs = prepare(srv, device)
            cap = run(srv, reqs, None)
            res = {"capacity": cap,
                   "poisson": [run(srv, reqs, f * cap["achieved_rps"]) for f in loads]}
            res["budget_bytes"] = srv.stats()["budget_bytes"]
        return res

    # correctness spot check of the served path against the plain path
    with nb.Server() as srv:
        for j in [j for j in jobs[:200] if j.limbs <= 8 and j.op != nb.OP_MULTIPLY][:6]:
            x = hpool[j.logN][:j.limbs].copy()
            o = np.empty_like(x)
            srv.wait(srv.submit(j.op, j.logN, j.moduli, x, o), 60.0)
            p = nb.Plan(j.logN, j.moduli)
            d = torch.from_numpy(x.view(np.int32)).cuda()
            (p.forward if j.op == nb.OP_FORWARD else p.inverse)(d)
            torch.cuda.synchronize()
            if not np.array_equal(d.cpu().numpy().view(np.uint32), o):
                raise RuntimeError("served result differs from the plain path")
            p.close()
    loads = [float(v) for v in args.serve_loads.split(",") if v]
    out = {"workload": f"{len(jobs)} requests: logN uniform 12..17, limbs uniform 1..64, "
                       "30/31-bit chains, 40% NTT / 40% INTT / 20% multiply",
           "limb_ntts": limb_ntts, "pcie_bytes_host_leg": pcie,
           "per_call_form": "the same server, one request per launch, same 4 stream slots"}
    for leg, device in (("host", False), ("device", True)):
        b = form(device, True, loads)
        p = form(device, False, [0.5])
        out[leg] = {"batched": b, "per_call": p,
                    "capacity_speedup_vs_per_call":
                        b["capacity"]["achieved_rps"] / p["capacity"]["achieved_rps"]}
    return out


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch_under_torchrun(args.gpus))
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
