"""Benchmark: LDA Gibbs sweeps on the B200 (Gibbs tokens/sec).

Workload: K=50 topics, V=10,000 words, D=2,000 documents with lengths
~ Poisson(200) (about 4e5 tokens), alpha=0.1, beta=0.01, tokens drawn from the
LDA generative process with seed 0; int32 token ids, assignments and counts.
One step = one augur_step of the schedule
ConjGibbs [theta] (*) ConjGibbs [phi] (*) DiscGibbs [z].

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (launched by torch.distributed.run) runs one independent chain per GPU
(replicas; LDA chains share nothing), value = all tokens / max-over-ranks time.
`--impl reference` times the reference's own CPU sampler (its cbits runtime
compiled from source, oracle/_ref) on all host cores, one chain per process.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

K_TOPICS, V_WORDS, D_DOCS, MEAN_LEN, ALPHA, BETA, DATA_SEED = 50, 10000, 2000, 200, 0.1, 0.01, 0
L2_FLUSH_BYTES = 512 << 20


def workload_config():
    return {"workload": "lda_gibbs_k50_v10000_d2000_len_poisson200", "K": K_TOPICS, "V": V_WORDS,
            "D": D_DOCS, "mean_doc_len": MEAN_LEN, "alpha": ALPHA, "beta": BETA,
            "schedule": "ConjGibbs [theta] (*) ConjGibbs [phi] (*) DiscGibbs [z]",
            "l2": "flushed between timed steps (512 MiB write)", "parallelism": None}


def corpus():
    from augurv2_b200.lda import synthetic_corpus
    return synthetic_corpus(K_TOPICS, V_WORDS, D_DOCS, MEAN_LEN, ALPHA, BETA, DATA_SEED)


# ---------------------------------------------------------------- clocks ----
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during timing."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ our arm ------
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def run_ours(args, rank, world, local_rank):
    import torch
    from augurv2_b200 import _native as N
    from augurv2_b200.lda import LdaGibbs

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    off, w = corpus()
    T = len(w)
    seed = 1000 + rank
    stream = torch.cuda.Stream()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    with torch.cuda.stream(stream):
        s = LdaGibbs(K_TOPICS, V_WORDS, off, w, ALPHA, BETA, seed=seed)
        s.sweep(max(3, args.warmup), stream=stream)
    stream.synchronize()

    # ---- timed: K sweeps, each bracketed by events, L2 flushed in between
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                flush.fill_(i & 0xFF)
                ev[i][0].record(stream)
                s.sweep(1, stream=stream)
                ev[i][1].record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    ms_t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = T * args.steps * world / (ms_max / 1e3)

    # ---- dominant kernel (z resample) timed alone for the roofline
    z_ms = time_z_kernel(s, stream, flush, reps=max(5, min(args.steps, 30)))
    alg_bytes = T * (4 + 4 + 8 + K_TOPICS * 8) + D_DOCS * K_TOPICS * 12
    hbm, peak_kind = measured_peaks()
    achieved = alg_bytes / (z_ms / 1e3) / 1e9

    # ---- end to end through the public API with host buffers
    e2e = run_e2e(args, off, w, seed, stream)
    s.close()

    line = None
    if rank == 0:
        cfg = workload_config()
        cfg["parallelism"] = "replicas%d" % world if world > 1 else "single"
        line = {
            "metric": "Gibbs tokens/sec (LDA)", "value": value, "unit": "tokens/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+int32", "data": "synthetic (LDA generative process, seed 0)",
            "config": cfg, "tokens_per_step": T,
            "gpu_launches": 4 * args.steps,
            "clocks": clocks.summary(),
            "roofline": {"bound": "hbm", "kernel": "lda_z_kernel", "achieved": achieved,
                         "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_source": peak_kind, "traffic": None,
                         "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": z_ms,
                         "note": "algorithmic bytes per token = 4 w + 4 z + 8 count RMW + 8K phi row"},
            "sweep_roofline_frac": (T * 442.0) / (ms_max / args.steps / 1e3) / 1e9 / hbm,
            "e2e": e2e,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(off, w, budget_s=args.cpu_seconds)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return line


def time_z_kernel(s, stream, flush, reps):
    import torch
    from augurv2_b200 import _native as N
    L = N.lib()
    z = s.z.clone()
    evs = []
    with torch.cuda.stream(stream):
        for i in range(reps + 2):
            flush.fill_(i & 0xFF)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            N.check(L.ab_lda_disc_z(s.D, s.K, s.V, N.ptr(s.doc_off), N.ptr(s.w), N.ptr(s.theta),
                                    N.ptr(s.phiT), N.ptr(z), None, None, s.seed, 0,
                                    N.stream_ptr(stream)), "disc_z")
            b.record(stream)
            evs.append((a, b))
    torch.cuda.synchronize()
    t = [a.elapsed_time(b) for a, b in evs[2:]]
    return sum(t) / len(t)


def run_e2e(args, off, w, seed, stream):
    """Same metric through the public Python API with host data: the corpus
    is uploaded from host memory inside the timed region, and every step
    copies the sample (theta, phi, z) back to host numpy arrays, as the
    reference's AugurInfer.samplen does (pyaugur/pyaugur/augurlib.py:195-222)."""
    import torch
    from augurv2_b200.lda import LdaGibbs
    steps = args.steps
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        s = LdaGibbs(K_TOPICS, V_WORDS, off, w, ALPHA, BETA, seed=seed)
        d2h = 0
        for _ in range(steps):
            s.sweep(1, stream=stream)
            th, ph, z = s.state()
            d2h = th.nbytes + ph.nbytes + z.nbytes
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    s.close()
    h2d = off.nbytes + w.nbytes + 8 * (K_TOPICS + V_WORDS)
    return {"value": len(w) * steps / dt, "unit": "tokens/s",
            "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step": d2h,
            "note": "corpus upload + graph capture inside the timed region; sample copied to host every step"}


# ------------------------------------------------------- CPU reference ------
def _ref_worker(args_tuple):
    kind, off, w, seed, warmup, steps, budget_s = args_tuple
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    o = O.Oracle(kind)
    D, K, V = len(off) - 1, K_TOPICS, V_WORDS
    theta, phi = np.full((D, K), 1.0 / K), np.full((K, V), 1.0 / V)
    z = np.zeros(len(w), np.int32)
    alpha, beta = np.full(K, ALPHA), np.full(V, BETA)
    for i in range(warmup):
        o.lda_sweeps(off, w, alpha, beta, theta, phi, z, seed, i, 1)
    t0 = time.perf_counter()
    n = 0
    while n < steps and (budget_s is None or n == 0 or time.perf_counter() - t0 < budget_s):
        o.lda_sweeps(off, w, alpha, beta, theta, phi, z, seed, warmup + n, 1)
        n += 1
    return n, time.perf_counter() - t0


def ref_kind():
    from oracle import oracle as O
    return "reference" if O.available("ref") else "port"


def cpu_baseline(off, w, budget_s=12.0):
    kind = ref_kind()
    lib = "ref" if kind == "reference" else "oracle"
    n, dt = _ref_worker((lib, off, w, 0, 0, 1000, budget_s))
    return {"value": len(w) * n / dt, "unit": "tokens/s", "cores": 1, "kind": kind,
            "sample": "%d full sweeps of the benchmark corpus (%d tokens) on 1 core, %.1f s" % (n, len(w), dt)}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    import multiprocessing as mp
    off, w = corpus()
    kind = ref_kind()
    lib = "ref" if kind == "reference" else "oracle"
    cores = os.cpu_count() or 1
    # each timed step is one full sweep per process; bounded so the run ends in minutes
    steps = max(1, min(args.steps, 40))
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        res = pool.map(_ref_worker, [(lib, off, w, 1000 + i, min(args.warmup, 1), steps, 60.0)
                                     for i in range(cores)])
    wall = time.perf_counter() - t0
    tokens = sum(n for n, _ in res) * len(w)
    tmax = max(dt for _, dt in res)
    value = tokens / tmax
    cfg = workload_config()
    cfg["parallelism"] = "%d independent CPU chains" % cores
    return {"impl": "reference", "metric": "Gibbs tokens/sec (LDA)", "value": value, "unit": "tokens/s",
            "n_gpus": world, "steps": steps, "warmup": min(args.warmup, 1),
            "ms_per_step": 1e3 * tmax / max(1, min(n for n, _ in res)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64+int32",
            "data": "synthetic (LDA generative process, seed 0)", "config": cfg,
            "cpu_baseline": {"value": value, "unit": "tokens/s", "cores": cores, "kind": kind,
                             "sample": "%d processes x %d sweeps of the benchmark corpus (%.1f s wall)"
                                       % (cores, steps, wall)},
            "e2e": {"value": value, "unit": "tokens/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        line = run_ours(args, rank, world, local_rank)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
