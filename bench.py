"""Benchmark: LDA Gibbs sweeps on the B200 (Gibbs tokens/sec).

Workload: K=50 topics, V=10,000 words, D=2,000 documents with lengths
~ Poisson(200) (about 4e5 tokens), alpha=0.1, beta=0.01, tokens drawn from the
LDA generative process with seed 0; int32 token ids, assignments and counts.
One step = one augur_step of the schedule
ConjGibbs [theta] (*) ConjGibbs [phi] (*) DiscGibbs [z].

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload lda|hlr_surrogate]

The default line also carries the other configurations, each measured in the
same run (and printable as its own line with --workload):
  hlr_surrogate  surrogate-gradient HMC on HLR (N=2,000,000 rows, D=512,
                 X ~ N(0,1) stored bf16, beta ~ Student-t(3), 256 chains,
                 L=10): min-ESS/s of the learned sampler and of plain
                 exact-gradient GPU HMC, and their ratio;
  hlr_small      HLR N=1000, D=10 plain HMC (1000 iterations, 10 leapfrog
                 steps of 0.01), min-ESS/s against the reference's cbits HMC;
  gmm            hmvgmm K=16, d=32, N=200,000 Gibbs sweeps, points/s against
                 the reference's assignment draw;
  hlr_nuts       64 HLR instances x 512 NUTS chains (max depth 10), min over
                 instances of min-ESS/s.

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
# DRAM bytes (read + write) of one launch of the sweep's z kernel on this
# workload, from the ncu capture summarised with its command in profiles/
# (phi and the count tables stay in L2)
Z_KERNEL_DRAM_BYTES = 5_137_408
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


def measured_tensor_peak(sustained=False):
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    key = "bf16_tflops_sustained" if sustained else "bf16_tflops"
    if os.path.exists(p):
        d = json.load(open(p))
        if key in d:
            return d[key], "measured"
    return (1400.0 if sustained else 1590.0), "fallback"


HLR_N, HLR_D, HLR_C, HLR_L, HLR_SEED = 2_000_000, 512, 256, 10, 5
_TUNER = None


def bench_tuner():
    """The launch-shape autotuner for this run: its cache lives in the run's
    working directory (a fresh box tunes once, outside every timed region)."""
    global _TUNER
    if _TUNER is None:
        from augurv2_b200 import autotune as T
        _TUNER = T.Autotuner(cache_path=os.path.join(os.getcwd(), ".augur_autotune.json"), reps=3, warmup=1)
    return _TUNER


def run_hlr_pass(n_rows, steps, warmup):
    """Exact batched HLR passes alone (log density + gradient for 256 chains
    at D=512 over n_rows bf16 rows): device time per pass and tensor-pipe
    throughput."""
    import torch
    from augurv2_b200 import hlrb as H
    X, y, beta = H.synthetic(n_rows, HLR_D, seed=HLR_SEED)
    d = H.HlrbData(X, y, prior="student_t", nu=3.0, scale=1.0)
    tuned = d.autotune(HLR_C, tuner=bench_tuner())
    th = torch.as_tensor(beta, device="cuda").repeat(HLR_C, 1).contiguous()
    work = d.workspace(HLR_C)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = {}
    for grad in (False, True):
        for _ in range(warmup):
            d.logp_grad(th, grad, work=work, err=err)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            d.logp_grad(th, grad, work=work, err=err)
        e1.record()
        torch.cuda.synchronize()
        out["grad" if grad else "logp"] = e0.elapsed_time(e1) / steps
    if int(err.item()) != 0:
        raise RuntimeError("device wait timed out in the HLR pass")
    mm = 2.0 * n_rows * HLR_D * HLR_C          # one N x D x C product
    peak, kind = measured_tensor_peak(sustained=False)
    return {"metric": "batched HLR exact pass (logp + grad, 256 chains)", "value": out["grad"], "unit": "ms",
            "higher_is_better": False, "logp_only_ms": out["logp"],
            "tflops": {"forward": mm / (out["logp"] / 1e3) / 1e12,
                       "forward+backward": 2 * mm / (out["grad"] / 1e3) / 1e12},
            "tensor_pipe_tflops": {"forward": 3 * mm / (out["logp"] / 1e3) / 1e12,
                                   "forward+backward": 5 * mm / (out["grad"] / 1e3) / 1e12},
            "note": "tflops: algorithmic 2 N D C per product; tensor_pipe_tflops: executed, 3 bf16 parts of "
                    "theta in the forward and 2 of the residual in the backward",
            "peak": peak, "peak_source": kind,
            "config": {"workload": "hlr_pass_n%d_d%d_c%d" % (n_rows, HLR_D, HLR_C), "N": n_rows, "D": HLR_D,
                       "chains": HLR_C, "launch_shape": tuned}}


# ---- config 1: small HLR, plain HMC (the reference's CPU case) -------------
def hlr_small_data(N_=1000, D=10, seed=0):
    """X ~ N(0,1), sigma^2 ~ InvGamma(1,1), beta ~ N(0, sigma^2 I), y ~ Bern(sigmoid(X beta))."""
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((N_, D))
    s2 = 1.0 / rng.gamma(1.0, 1.0)
    beta = rng.standard_normal(D) * np.sqrt(s2)
    y = (rng.random(N_) < 1.0 / (1.0 + np.exp(-(X @ beta)))).astype(np.int32)
    return X, y, beta, s2


def hlr_small_cpu_baseline(X, y, init, iters, budget_s=10.0):
    """The reference's own HMC (cbits h_augur_mcmc_hmc with the restated ll/grad,
    oracle/_ref) for one chain on one host core: min-ESS/s over (beta, sigma^2)."""
    from augurv2_b200.diagnostics import ess
    from oracle import oracle as O
    kind = "reference" if O.available("ref") else "port"
    o = O.Oracle("ref" if kind == "reference" else "oracle")
    m = O.HlrModel(X, y, has_b=False, vprior="invgamma", a0=1.0, s0=1.0)
    D = X.shape[1]
    idx = list(range(D)) + [D + 1]
    par = np.array(init, np.float64)
    draws = []
    t0 = time.time()
    for it in range(iters):
        O.hlr_hmc(o, m, par, idx, 0.1, 0.01, 0, it, 0, 0)
        draws.append(par[idx].copy())
        if time.time() - t0 > budget_s:
            break
    wall = time.time() - t0
    e = ess(np.asarray(draws)[:, None, :])
    return {"value": float(e.min() / wall), "unit": "min-ESS/s", "cores": 1, "kind": kind,
            "sample": "%d HMC iterations of one chain (10 leapfrog steps, eps 0.01), %.2f s" % (len(draws), wall)}


def run_hlr_small(iters=1000, chains=256, cpu=True):
    """HLR N=1000, D=10 (ighlr.rv: sigma^2 ~ InvGamma(1,1)), HMC over
    (beta, sigma^2) with simulation length 0.1 and step 0.01 (10 leapfrog
    steps), 1000 iterations, seed 0, on the per-chain engine: every chain's
    whole run is one kernel launch.  min-ESS/s over the 11 parameters."""
    import torch
    from augurv2_b200 import hlr as G
    from augurv2_b200.diagnostics import ess
    X, y, beta, s2 = hlr_small_data()
    D = X.shape[1]
    data = G.HlrData(X, y, has_b=False, vprior="invgamma", a0=1.0, s0=1.0, compat=True, x_dtype="f32")
    sched = [{"kind": "HMC", "block": ["theta", "v"], "simlen": 0.1, "eps": 0.01}]
    init = np.zeros(D + 2)
    init[:D] = beta
    init[D + 1] = s2
    idx = list(range(D)) + [D + 1]
    out = {}
    for C_ in (1, chains):
        # draws (one launch per iteration, recorded) ...
        ch = G.HlrChains(data, sched, C=C_, init=init, seed=0)
        rec = np.empty((iters, C_, len(idx)))
        for it in range(iters):
            ch.run(1)
            rec[it] = ch.pars[:, idx].cpu().numpy()
        e = ess(rec)
        # ... and the same iterations timed as one launch (identical states:
        # the random streams are keyed by iteration)
        ch2 = G.HlrChains(data, sched, C=C_, init=init, seed=0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        ch2.run(iters)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        same = bool(np.array_equal(ch2.pars[:, idx].cpu().numpy(), rec[-1]))
        out[C_] = {"min_ess": float(e.min()), "ms": ms, "min_ess_per_s": float(e.min() / (ms / 1e3)),
                   "us_per_iteration": ms * 1e3 / iters, "replay_identical": same}
    line = {"metric": "min-ESS/sec (HLR plain HMC, N=1000 D=10)", "value": out[chains]["min_ess_per_s"],
            "unit": "min-ESS/s", "chains": chains, "single_chain": out[1], "batched": out[chains],
            "config": {"workload": "hlr_hmc_n1000_d10", "N": 1000, "D": 10, "iterations": iters,
                       "leapfrog_steps": 10, "eps": 0.01, "seed": 0, "x_dtype": "f32",
                       "block": "theta, sigma^2"}}
    if cpu:
        line["cpu_baseline"] = hlr_small_cpu_baseline(X, y, init, iters)
        line["gain_single_chain_vs_cpu"] = out[1]["min_ess_per_s"] / line["cpu_baseline"]["value"]
    return line


# ---- config 4: many HLR instances, batched NUTS --------------------------------
NUTS_INST, NUTS_C, NUTS_DEPTH = 64, 512, 10


def nuts_instances(n_inst=NUTS_INST, seed=0):
    """N_i log-uniform in [1e3, 1e6], D_i uniform over {16, 64, 256}."""
    rng = np.random.default_rng(seed)
    Ns = np.exp(rng.uniform(np.log(1e3), np.log(1e6), n_inst)).astype(np.int64)
    Ds = rng.choice([16, 64, 256], n_inst)
    return [(int(n), int(d)) for n, d in zip(Ns, Ds)]


def run_hlr_group(scale=1.0, steps=10, warmup=3, n_inst=NUTS_INST, chains=NUTS_C):
    """The grouped HLR pass alone on the 64 config-4 instances with every N_i
    scaled by `scale` (scale 1: the NUTS workload's data, X ~ N(0,1) bf16):
    log density and gradient of 512 chains per instance at theta = the
    generating coefficients plus noise, one HlrGroup pass (theta split, the
    fused tensor-core kernel, finishing sums) for all instances; device time
    per pass and tensor-pipe throughput."""
    import torch
    from augurv2_b200 import hlrb as H
    specs = [(max(64, int(n * scale)), d) for n, d in nuts_instances(n_inst)]
    rng = np.random.default_rng(42)
    datas, ths, lps, gs = [], [], [], []
    for i, (Ni, Di) in enumerate(specs):
        g = torch.Generator(device="cuda")
        g.manual_seed(1000 + i)
        X = torch.randn((Ni, Di), generator=g, device="cuda").to(torch.bfloat16)
        beta = rng.standard_normal(Di).astype(np.float32) * 0.5
        t = X.float() @ torch.as_tensor(beta, device="cuda")
        y = (torch.rand(Ni, generator=g, device="cuda") < torch.sigmoid(t)).to(torch.int32)
        datas.append(H.HlrbData(X, y, prior="normal", var=1.0))
        ths.append(torch.as_tensor(beta[None] + 0.01 * rng.standard_normal((chains, Di)).astype(np.float32),
                                   device="cuda").contiguous())
        lps.append(torch.empty(chains, dtype=torch.float64, device="cuda"))
        gs.append(torch.empty((chains, Di), dtype=torch.float32, device="cuda"))
    grp = H.HlrGroup(datas, [chains] * len(datas))
    for i in range(len(datas)):
        grp.bind(i, ths[i], lps[i], gs[i])
    grp.set_active([True] * len(datas))
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    for _ in range(warmup):
        grp.logp_grad(err)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        grp.logp_grad(err)
    e1.record()
    torch.cuda.synchronize()
    if int(err.item()) != 0:
        raise RuntimeError("device wait timed out in the grouped HLR pass")
    ms = e0.elapsed_time(e1) / steps
    nd = float(sum(n * d for n, d in specs))
    alg = 4.0 * nd * chains                      # forward + backward products
    peak, kind = measured_tensor_peak(sustained=True)
    out = {"metric": "grouped HLR pass (logp + grad, 512 chains per instance, all instances)", "value": ms,
           "unit": "ms", "higher_is_better": False, "fused": grp.fused,
           "roofline": {"bound": "tensor", "kernel": "hlrf_kernel" if grp.fused else "grouped_gemm_kernel",
                        "achieved": alg / (ms / 1e3) / 1e12, "peak": peak, "unit": "TFLOP/s",
                        "frac": alg / (ms / 1e3) / 1e12 / peak, "peak_source": kind + " (sustained)",
                        "executed_tflops": 2.5 * alg / (ms / 1e3) / 1e12,
                        "note": "algorithmic 4 N D C per instance (forward and backward product); the pipe "
                                "executes 2.5x (3 bf16 parts of theta forward, 2 of the residual backward)"},
           "config": {"workload": "hlr_group_64_instances_c512", "scale": scale, "sum_N": int(sum(n for n, _ in specs)),
                      "sum_ND": int(nd), "D": "{16, 64, 256}", "chains": chains}}
    grp.close()
    return out


def nuts_cpu_baseline(per, chains, budget_s=12.0, max_nd=4_000_000):
    """The reference's NUTS on the host, one chain per core, for every
    instance of the run, from timed pieces of its own code: each NUTS leaf of
    the reference (cbits/augur_mcmclib.h:305-325, h_augur_nuts_build_tree)
    calls its gradient twice and its log density once, so the reference's
    seconds per leaf are at least 2 t_grad + t_ll of its cbits HLR functions
    (oracle/_ref), timed here on one core at a spread of instance sizes
    (those with N D <= max_nd) and fitted as a + b N D.  The same algorithm
    draws the same chain, so its leaves per draw (the GPU run's rounds per
    draw: one leaf per chain per round) and its effective samples per draw
    (the GPU run's min-ESS over its 512 chains' draws) carry over:
    min-ESS/s_ref(i) = (min-ESS_i / draws_i) / (leaves per draw_i x
    seconds per leaf_i).  A full reference NUTS iteration at these sizes runs
    for minutes (up to 2^10 leaves of an N D product), hence the pieces."""
    from oracle import oracle as O
    kind = "reference" if O.available("ref") else "port"
    o = O.Oracle("ref" if kind == "reference" else "oracle")
    sizes = sorted({(q["N"], q["D"]) for q in per if q["N"] * q["D"] <= max_nd}, key=lambda s: s[0] * s[1])
    if len(sizes) > 5:
        sizes = [sizes[int(round(i * (len(sizes) - 1) / 4))] for i in range(5)]
    rng = np.random.default_rng(5)
    pts = []
    t_start = time.perf_counter()
    for (Ni, Di) in sizes:
        X = rng.standard_normal((Ni, Di))
        y = (rng.random(Ni) < 0.5).astype(np.int32)
        m = O.HlrModel(X, y, has_b=False, vprior="invgamma", a0=1.0, s0=1.0)
        par = np.concatenate([rng.standard_normal(Di) * 0.1, [0.0, 1.0]])
        idx = list(range(Di))
        reps, t0 = 0, time.perf_counter()
        while reps < 3 or (time.perf_counter() - t0 < budget_s / (2 * len(sizes)) and reps < 200):
            O.hlr_grad(o, m, par, idx)
            O.hlr_grad(o, m, par, idx)
            O.hlr_ll(o, m, par, idx)
            reps += 1
        pts.append((Ni * Di, (time.perf_counter() - t0) / reps))
    nd = np.array([p[0] for p in pts], np.float64)
    tl = np.array([p[1] for p in pts])
    b, a = np.polyfit(nd, tl, 1) if len(pts) > 1 else (tl[0] / nd[0], 0.0)
    a = max(a, 0.0)
    rates = []
    for q in per:
        leaves_per_draw = q["rounds"] / max(1, q["draws_per_chain"])
        sec_leaf = a + b * q["N"] * q["D"]
        ess_per_draw = q["min_ess"] / (q["draws_per_chain"] * chains)
        rates.append(ess_per_draw / (leaves_per_draw * sec_leaf))
    worst = int(np.argmin(rates))
    return {"value": float(rates[worst]), "unit": "min-ESS/s", "cores": 1, "kind": kind,
            "per_instance_min_ess_per_s": [float(r) for r in rates],
            "worst_instance": {"N": per[worst]["N"], "D": per[worst]["D"]},
            "seconds_per_leaf_fit": {"a": float(a), "b_per_nd": float(b),
                                     "timed": [{"ND": int(n), "s": float(t)} for n, t in pts]},
            "sample": "the reference's cbits HLR gradient (x2) and log density per NUTS leaf, timed on one core "
                      "at %d instance sizes (%.1f s), fitted linear in N D; leaves and min-ESS per draw from the "
                      "GPU run of the same algorithm" % (len(pts), time.perf_counter() - t_start)}


def run_hlr_nuts(min_draws=48, max_rounds=2400, warmup_draws=16, n_inst=NUTS_INST, chains=NUTS_C,
                 hist_cap=128, variants=("reference", "standard"), cpu=True):
    """64 HLR instances (X ~ N(0,1) bf16, sigma^2 ~ InvGamma(1,1),
    beta ~ N(0, sigma^2 I), y ~ Bern(sigmoid(X beta)); sigma^2 held at its
    generating value), 512 NUTS chains each, max tree depth 10.  Every round
    every running instance advances all its chains to their next leaf and
    evaluates its log density and gradient there; a NutsGroup does this for
    all instances with one advance launch and one grouped tensor-core pass
    (theta split, the fused forward + residual + backward kernel whose work
    units of every instance share one persistent grid, and the finishing
    sums), captured as one CUDA graph, until every chain of every
    instance has `min_draws` draws (instances with deep trees run more
    rounds; finished instances leave the launches), after an untimed warm-up
    of `warmup_draws` draws per chain whose draws are discarded.  min-ESS/s per instance = min-ESS
    of its draws / the whole run's device time; the line reports the minimum
    over instances.  Each selection rule in `variants` runs on the same data
    and starting points; the first is the line's value (the reference's
    rule), the others are reported beside it."""
    import torch
    from augurv2_b200 import hlrb as H
    from augurv2_b200.diagnostics import ess
    specs = nuts_instances(n_inst)
    rng = np.random.default_rng(42)
    datas = []
    flops_round_i = []
    for i, (Ni, Di) in enumerate(specs):
        s2 = 1.0 / rng.gamma(1.0, 1.0)
        beta = (rng.standard_normal(Di) * np.sqrt(s2)).astype(np.float32)
        g = torch.Generator(device="cuda")
        g.manual_seed(1000 + i)
        X = torch.randn((Ni, Di), generator=g, device="cuda").to(torch.bfloat16)
        t = X.float() @ torch.as_tensor(beta, device="cuda")
        y = (torch.rand(Ni, generator=g, device="cuda") < torch.sigmoid(t)).to(torch.int32)
        w = (torch.sigmoid(t) * (1 - torch.sigmoid(t))).mean().item()
        eps = 0.6 / np.sqrt(Ni * w + 1.0 / s2)       # ~ 0.6 of the posterior scale
        d = H.HlrbData(X, y, prior="normal", var=s2)
        init = beta[None] + (0.1 * eps) * rng.standard_normal((chains, Di)).astype(np.float32)
        datas.append((d, eps, init))
        flops_round_i.append(4.0 * Ni * Di * chains)   # algorithmic: forward + backward product
    peak, kind = measured_tensor_peak(sustained=True)
    results = {}
    for variant in variants:
        insts = [H.BatchedNuts(d, chains, eps=eps, max_depth=NUTS_DEPTH, seed=7 + i, init=init, hist_cap=hist_cap,
                               variant=variant) for i, (d, eps, init) in enumerate(datas)]
        pool = H.NutsGroup(insts)
        # warm-up (untimed, draws discarded): the chains leave their common start
        pool.run(warmup_draws, max_rounds)
        pool.reset()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        rounds = pool.run(min_draws, max_rounds)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        per = []
        for i, nuts in enumerate(insts):
            dr = nuts.draws()
            inf = nuts.info()
            e = ess(dr) if dr.shape[0] >= 4 else np.zeros(nuts.D)
            per.append({"N": nuts.data.N, "D": nuts.D, "rounds": rounds[i], "draws_per_chain": int(dr.shape[0]),
                        "min_ess": float(e.min()), "mean_depth": float(inf[:, 5].mean()),
                        "min_ess_per_s": float(e.min() / (ms / 1e3))})
        worst = min(per, key=lambda q: q["min_ess_per_s"])
        ach = sum(f * r for f, r in zip(flops_round_i, rounds)) / (ms / 1e3) / 1e12
        results[variant] = {
            "value": worst["min_ess_per_s"], "unit": "min-ESS/s", "rounds_total": int(sum(rounds)),
            "seconds": ms / 1e3, "worst_instance": worst,
            "median_instance_min_ess_per_s": float(np.median([q["min_ess_per_s"] for q in per])),
            "total_draws": int(sum(q["draws_per_chain"] for q in per) * chains),
            "roofline": {"bound": "tensor", "kernel": "hlrf_kernel (fused forward + residual + backward, all "
                                                     "instances)", "achieved": ach,
                         "peak": peak, "unit": "TFLOP/s", "frac": ach / peak, "peak_source": kind + " (sustained)",
                         "note": "algorithmic 4 N D C per chain-round (forward and backward product); the tensor "
                                 "pipe executes 2.5x that (3 bf16 parts forward, 2 backward)"},
            "instances": per}
        pool.close()
        del pool, insts
        torch.cuda.empty_cache()
    head = dict(results[variants[0]])
    head.update({"metric": "min-ESS/sec per instance, min over 64 instances (batched NUTS, HLR)",
                 "selection_rule": variants[0], "min_draws_per_chain": min_draws,
                 "warmup_draws_per_chain": warmup_draws,
                 "other_rules": {v: {k: results[v][k] for k in ("value", "seconds", "median_instance_min_ess_per_s",
                                                                "worst_instance", "rounds_total")}
                                 for v in variants[1:]},
                 "config": {"workload": "hlr_nuts_64_instances_c512", "instances": n_inst, "chains": chains,
                            "max_depth": NUTS_DEPTH, "x_dtype": "bf16", "N": "log-uniform [1e3, 1e6]",
                            "D": "{16, 64, 256}", "prior": "normal(0, sigma^2), sigma^2 at its generating value",
                            "step_size": "0.6 / sqrt(N E[w] + 1/sigma^2) at the generating coefficients",
                            "schedule": "NutsGroup: one advance + one grouped fused pass (3 launches) per round "
                                        "for all running instances, one CUDA graph; rounds until %d draws per chain"
                                        % min_draws}})
    if cpu:
        head["cpu_baseline"] = nuts_cpu_baseline(results[variants[0]]["instances"], chains)
        head["gain_vs_cpu_core"] = head["value"] / head["cpu_baseline"]["value"]
    return head


# ---- config 3: Gaussian mixture Gibbs ----------------------------------------
GMM_N, GMM_K, GMM_D = 200_000, 16, 32


def gmm_data(N_=GMM_N, K=GMM_K, d=GMM_D, seed=0):
    """Means ~ N(0, 25 I), covariances ~ Wishart(d + 2, I) / (d + 2),
    weights ~ Dirichlet(1); y stored as float32."""
    rng = np.random.default_rng(seed)
    mus = rng.standard_normal((K, d)) * 5.0
    covs = []
    for _ in range(K):
        A = rng.standard_normal((d + 2, d))
        covs.append(A.T @ A / (d + 2))
    pis = rng.dirichlet(np.ones(K))
    z = rng.choice(K, size=N_, p=pis)
    Y = np.empty((N_, d))
    for k in range(K):
        m = z == k
        if m.any():
            Y[m] = mus[k] + rng.standard_normal((m.sum(), d)) @ np.linalg.cholesky(covs[k]).T
    return Y.astype(np.float32), z.astype(np.int32), mus, np.array(covs), pis


def gmm_cpu_baseline(Y, mus, covs, pis, n_points=1500):
    """The reference's DiscGibbs z (cbits augur_mvnormal_ll, which factors the
    covariance for every point and component) on a bounded sample of points."""
    from oracle import oracle as O
    kind = "reference" if O.available("ref") else "port"
    o = O.Oracle("ref" if kind == "reference" else "oracle")
    K, d = mus.shape
    g = O.GmmModel(Y[:n_points].astype(np.float64), K, np.zeros(d), 25.0 * np.eye(d), shared_cov=False,
                   alpha=np.ones(K), df=d + 2, scale0=np.eye(d))
    t0 = time.time()
    O.gmm_disc_z(o, g, pis, mus, covs, 0, 0)
    wall = time.time() - t0
    return {"value": n_points / wall, "unit": "points/s (assignment draw)", "cores": 1, "kind": kind,
            "sample": "DiscGibbs z over %d of the %d points (K=%d, d=%d), %.2f s" % (n_points, len(Y), K, d, wall)}


def run_gmm(steps=10, warmup=3, cpu=True):
    """hmvgmm.rv, K=16, d=32, N=200,000: one sweep = ConjGibbs [pis] (*)
    ConjGibbs [mu] (*) ConjGibbs [cov] (*) DiscGibbs [z] on the device."""
    import torch
    from augurv2_b200 import _native as Nn
    from augurv2_b200.gmm import GmmGibbs
    Y, z0, mus, covs, pis = gmm_data()
    K, d = GMM_K, GMM_D
    s = GmmGibbs(Y, K, np.zeros(d), 25.0 * np.eye(d), alpha=np.ones(K), df=d + 2, scale0=np.eye(d),
                 mu=mus, cov=covs, pis=pis, z=z0, seed=3)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    s.sweep(warmup)
    torch.cuda.synchronize()
    ms = 0.0
    for i in range(steps):
        flush.fill_(i & 0xFF)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        s.sweep(1)
        b.record()
        torch.cuda.synchronize()
        ms += a.elapsed_time(b)
    # the assignment draw alone: the sweep's screened launch (prep, binary32
    # screen, binary64 path for the queued points) and the all-binary64 kernel
    L = Nn.lib()
    zs = s.z.clone()
    times = {}
    for kind in ("screened", "binary64"):
        tot = 0.0
        for i in range(-1, steps):          # i = -1: untimed first launch
            flush.fill_(i & 0xFF)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            if kind == "screened":
                Nn.check(L.ab_gmm_disc_z_screened(GMM_N, d, K, 0, Nn.ptr(s.Y), Nn.ptr(s.pis), Nn.ptr(s.mu),
                                                  Nn.ptr(s.Linv), Nn.ptr(s.hdet), Nn.ptr(zs), s.seed, 10_000 + i, 0,
                                                  Nn.ptr(s.zscratch), Nn.stream_ptr()), "disc_z_screened")
            else:
                Nn.check(L.ab_gmm_disc_z(GMM_N, d, K, 0, Nn.ptr(s.Y), Nn.ptr(s.pis), Nn.ptr(s.mu), Nn.ptr(s.Linv),
                                         Nn.ptr(s.hdet), Nn.ptr(zs), s.seed, 10_000 + i, 0, Nn.stream_ptr()),
                         "disc_z")
            b.record()
            torch.cuda.synchronize()
            if i >= 0:
                tot += a.elapsed_time(b)
        times[kind] = tot / steps
    # points the screen left to the binary64 path in the last screened call
    # (the queue length after the component tables)
    qoff = int(L.ab_gmm_z_queue_offset(d, K))
    flops_pt = K * (d * d + 3 * d)     # triangular solve (d^2/2 FMAs) + centring and squares, per component
    zms = times["screened"]
    ach = GMM_N * flops_pt / (zms / 1e3) / 1e12
    fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12   # nominal B200 FP32 FMA rate at the measured SM clock
    line = {"metric": "GMM Gibbs points/sec (hmvgmm, K=16 d=32)", "value": GMM_N * steps / (ms / 1e3),
            "unit": "points/s", "ms_per_sweep": ms / steps, "steps": steps, "warmup": warmup,
            "roofline": {"bound": "fp32", "kernel": "gmm_zs_kernel (binary32-screened assignment draw)",
                         "achieved": ach, "peak": fp32_peak, "unit": "TFLOP/s", "frac": ach / fp32_peak,
                         "peak_source": "nominal (148 SMs x 128 FP32 FMA per clock at 1965 MHz; no measured "
                                        "FP32 peak)",
                         "launch_ms": zms, "binary64_kernel_ms": times["binary64"],
                         "points_to_binary64_path": int(s.zscratch[qoff:qoff + 4].view(torch.int32).item()),
                         "algorithmic_flops_per_point": flops_pt},
            "config": {"workload": "gmm_hmvgmm_n200000_k16_d32", "N": GMM_N, "K": K, "d": d,
                       "y_dtype": "f32", "l2": "flushed between timed sweeps"}}
    if cpu:
        line["cpu_baseline"] = gmm_cpu_baseline(Y, mus, covs, pis)
    return line


def chain_moments(sampler, n, burn=0):
    """Runs `burn` iterations of `sampler` (discarded), then `n` more,
    accumulating every chain's sum and sum of squares of theta on the device
    (float64), separately for the two halves of the window.  Returns the chain
    means [C, D], within-chain variances [C, D] and the two half-window chain
    means (for a stationarity check) as numpy arrays."""
    import torch
    C_, D = sampler.theta.shape
    for _ in range(burn):
        sampler.run(1)
    s1 = torch.zeros((2, C_, D), dtype=torch.float64, device="cuda")
    s2 = torch.zeros((C_, D), dtype=torch.float64, device="cuda")
    for i in range(n):
        sampler.run(1)
        t = sampler.theta.double()
        s1[int(2 * i >= n)] += t
        s2 += t * t
    h = torch.tensor([(n + 1) // 2, n // 2], dtype=torch.float64, device="cuda")
    halves = s1 / h[:, None, None]
    m = s1.sum(0) / n
    v = (s2 / n - m * m).clamp_min(0.0) * (n / (n - 1.0))
    return m.cpu().numpy(), v.cpu().numpy(), halves.cpu().numpy()


def exactness_stats(mom_s, mom_p):
    """Posterior means of two samplers of one posterior, compared in units of
    the posterior sd per coefficient.  Each sampler's Monte-Carlo error is
    estimated from the spread of its independent chains' means
    (var(grand mean) = var over chains of the chain means / C).  Reports the
    largest and median |difference|, the Monte-Carlo sd of the difference,
    and the root-mean-square bias over coefficients with the Monte-Carlo
    noise removed: sqrt(max(0, mean(d^2 - s^2))), with an approximate 95%
    upper bound (mean(d^2) has standard error sqrt(2/D) mean(d^2) when the
    difference is noise)."""
    (m_s, v_s, h_s), (m_p, v_p, h_p) = mom_s, mom_p
    C_, D = m_p.shape
    sd = np.sqrt(v_p.mean(0))

    def drift(h):
        # second-half minus first-half grand means, in posterior sd, with the
        # Monte-Carlo noise of the halves removed (rms over coefficients)
        dd = (h[1].mean(0) - h[0].mean(0)) / sd
        nn = np.sqrt(h[1].var(0, ddof=1) / C_ + h[0].var(0, ddof=1) / C_) / sd
        return float(np.sqrt(max(0.0, np.mean(dd * dd) - np.mean(nn * nn))))
    gs, gp = m_s.mean(0), m_p.mean(0)
    mc = np.sqrt(m_s.var(0, ddof=1) / C_ + m_p.var(0, ddof=1) / C_) / sd
    d = (gs - gp) / sd
    msq, nsq = float(np.mean(d * d)), float(np.mean(mc * mc))
    bias2 = msq - nsq
    upper2 = bias2 + 2.0 * np.sqrt(2.0 / D) * msq
    return {"posterior_mean_diff_in_sd": float(np.max(np.abs(d))),
            "posterior_mean_diff_in_sd_median": float(np.median(np.abs(d))),
            "posterior_mean_mc_sd": float(np.median(mc)),
            "posterior_mean_z_max": float(np.max(np.abs(d) / mc)),
            "posterior_mean_bias_rms_in_sd": float(np.sqrt(max(bias2, 0.0))),
            "posterior_mean_bias_rms_upper95_in_sd": float(np.sqrt(max(upper2, 0.0))),
            "posterior_sd_ratio_median": float(np.median(np.sqrt(v_s.mean(0)) / sd)),
            "drift_rms_in_sd": {"surrogate": drift(h_s), "plain": drift(h_p)}}


def ess_chain_means(mom):
    """Effective sample size per coefficient of C independent chains of n
    draws each from their chain means: var(chain mean) = sigma^2 tau / n, so
    ESS = C n / tau = C sigma^2 / var(chain mean) (sigma^2 the mean
    within-chain variance).  Valid when n is many autocorrelation times, which
    the burn-in and window lengths of the caller ensure."""
    m, v, _ = mom
    return m.shape[0] * v.mean(0) / np.maximum(m.var(0, ddof=1), 1e-300)


def run_hlr_surrogate(iters=100, warm=40, learn=240, train_every=8, train_steps=10, exact_plain=1000,
                      exact_sur=3000, exact_burn=(300, 600)):
    """Surrogate-gradient HMC vs plain exact-gradient HMC on the same data,
    chains, step-size rule and trajectory length.  Per-iteration device time
    by CUDA events over `iters` iterations of each (graph replays, the
    surrogate's periodic exact-gradient checks included).  Each sampler then
    runs a burn-in and a long window whose chain means give both the
    effective sample size (ess_chain_means) and the exactness comparison
    (posterior means of the two samplers in posterior sd, exactness_stats).
    The surrogate learns online (replay buffer, refitted linear part, Adam)
    for its first `learn` iterations only; afterwards its kernel is fixed and
    its error checks decide the fallback."""
    import torch
    from augurv2_b200 import hlrb as H

    X, y, beta = H.synthetic(HLR_N, HLR_D, seed=HLR_SEED)
    d = H.HlrbData(X, y, prior="student_t", nu=3.0, scale=1.0)
    tuned = d.autotune(HLR_C, tuner=bench_tuner())
    rs = np.random.default_rng(HLR_SEED)
    init = np.asarray(beta, np.float32)[None] + 1e-3 * rs.standard_normal((HLR_C, HLR_D)).astype(np.float32)

    # exact pass timing (forward = log density only; forward + backward)
    th = torch.as_tensor(init, device="cuda")
    work = d.workspace(HLR_C)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    pass_ms = {}
    for grad in (False, True):
        for _ in range(3):
            d.logp_grad(th, grad, work=work, err=err)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(10):
            d.logp_grad(th, grad, work=work, err=err)
        e1.record()
        torch.cuda.synchronize()
        pass_ms["grad" if grad else "logp"] = e0.elapsed_time(e1) / 10
    mm = 2.0 * HLR_N * HLR_D * HLR_C          # one N x D x C product
    peak, peak_kind = measured_tensor_peak(sustained=True)
    ach = 2 * mm / (pass_ms["grad"] / 1e3) / 1e12        # algorithmic: forward + backward product
    exe = 5 * mm / (pass_ms["grad"] / 1e3) / 1e12        # executed: 3 + 2 bf16 parts

    def timed(sampler, n):
        ms = 0.0
        for i in range(n):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            sampler.run(1)
            b.record()
            torch.cuda.synchronize()
            ms += a.elapsed_time(b)
        return ms / n

    plain = H.BatchedHmc(d, HLR_C, L=HLR_L, eps=2e-4, jitter=0.1, seed=11, init=init)
    eps = H.adapt_step_size(plain, warm)
    init = plain.theta.cpu().numpy()      # both samplers start from the warmed-up chains
    plain.capture()
    plain.reset_stats()
    ms_p = timed(plain, iters)
    acc_p = plain.accept_rate()[0]
    mom_p = chain_moments(plain, exact_plain, exact_burn[0])
    div_p = plain.divergences()
    del plain

    sur = H.SurrogateHmc(d, HLR_C, L=HLR_L, eps=eps, jitter=0.1, seed=12, init=init, train_every=train_every,
                         train_steps=train_steps, learn_iters=learn)
    sur.run(learn)                        # online learning: the warm-up
    eps_s = H.adapt_step_size(sur, warm // 2)
    sur.capture()
    sur.reset_stats()
    g0, l0 = sur.n_grad, sur.n_logp
    ms_s = timed(sur, iters)
    acc_s = sur.accept_rate()[0]
    passes = {"grad": sur.n_grad - g0, "logp_only": sur.n_logp - l0, "plain_grad": iters * HLR_L}
    mom_s = chain_moments(sur, exact_sur, exact_burn[1])
    div_s = sur.divergences()

    exact = exactness_stats(mom_s, mom_p)
    exact["iterations"] = {"plain": exact_plain, "surrogate": exact_sur}
    exact["burn_in"] = {"plain": exact_burn[0], "surrogate": exact_burn[1]}
    ess_p, ess_s = ess_chain_means(mom_p), ess_chain_means(mom_s)
    v_p = ess_p.min() / (exact_plain * ms_p / 1e3)
    v_s = ess_s.min() / (exact_sur * ms_s / 1e3)
    return {
        "metric": "min-ESS/sec (surrogate-gradient HMC, HLR)", "value": float(v_s), "unit": "min-ESS/s",
        "plain_hmc_value": float(v_p), "gain_vs_plain": float(v_s / v_p),
        "iterations_timed": iters, "chains": HLR_C, "leapfrog_steps": HLR_L,
        "step_size": {"plain": eps, "surrogate": eps_s},
        "ms_per_iteration": {"surrogate": ms_s, "plain": ms_p},
        "min_ess": {"surrogate": float(ess_s.min()), "plain": float(ess_p.min()),
                    "estimator": "chain means of 256 chains over the exactness windows"},
        "autocorrelation_time_max": {"surrogate": float(HLR_C * exact_sur / ess_s.min()),
                                     "plain": float(HLR_C * exact_plain / ess_p.min())},
        "accept": {"surrogate": float(acc_s), "plain": float(acc_p)},
        "surrogate_rel_err": sur.last_rel_err, "fallback": sur.fallback, "max_rel_err": sur.max_rel_err,
        "exact_passes": passes,
        "exactness": exact,
        "posterior_mean_diff_in_sd": exact["posterior_mean_diff_in_sd"],
        "divergences": {"surrogate": div_s, "plain": div_p},
        "exact_pass_ms": pass_ms,
        "roofline": {"bound": "tensor", "kernel": "gemm_kernel (forward + backward data passes)",
                     "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
                     "peak_source": peak_kind + " (sustained)",
                     "algorithmic_flops_per_pass": 2 * mm,
                     "executed_tflops": exe, "executed_frac": exe / peak,
                     "note": "algorithmic 2 x 2 N D C (forward and backward product); executed on the tensor "
                             "pipe 5 x 2 N D C: three bf16 parts of theta forward, two of the residual backward"},
        "config": {"workload": "hlr_surrogate_n2000000_d512_c256", "N": HLR_N, "D": HLR_D, "chains": HLR_C,
                   "x_dtype": "bf16", "prior": "student_t(3)",
                   "mlp": "512-256-256-512 gelu, bf16 weights, over a dense least-squares linear part",
                   "init": "generating coefficients + N(0, 1e-6), then the plain sampler's warm-up",
                   "launch_shape": tuned, "warmup": warm, "surrogate_learning_iterations": learn,
                   "train_every": train_every, "train_steps": train_steps},
    }


def max_over_ranks(x, dist, device):
    """x maximised over the ranks of the default process group (x itself
    without one): the job's time is its slowest rank's."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank, world, seconds):
    """Whole-job throughput of `world` replicas that each processed
    `units_per_rank` units, timed by the slowest rank."""
    return units_per_rank * world / seconds


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
    ms_max = max_over_ranks(ms, dist, "cuda")
    value = aggregate_rate(T * args.steps, world, ms_max / 1e3)

    # ---- dominant kernel (z resample) timed alone for the roofline
    z_ms = time_z_kernel(s, stream, flush, reps=max(5, min(args.steps, 30)))
    # the screened z kernel reads a binary32 phi row (4 K bytes) per token
    alg_bytes = T * (4 + 4 + 8 + K_TOPICS * 4) + D_DOCS * K_TOPICS * 12
    hbm, peak_kind = measured_peaks()
    achieved = alg_bytes / (z_ms / 1e3) / 1e9

    # ---- end to end through the public API with host buffers
    # end to end through the public API, three times; the median is reported
    # (a wall-clock region of tens of milliseconds sees host jitter)
    runs = []
    for _ in range(3):
        if dist:
            dist.barrier()
        r = run_e2e(args, off, w, seed, stream)
        # whole-job rate: every rank's tokens over the slowest rank's wall time
        r["value"] = aggregate_rate(T * args.steps, world, max_over_ranks(r.pop("seconds"), dist, "cuda"))
        runs.append(r)
    e2e = sorted(runs, key=lambda r: r["value"])[1]
    e2e["repeats"] = [r["value"] for r in runs]
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
            "gpu_launches": 5 * args.steps,
            "clocks": clocks.summary(),
            "roofline": {"bound": "hbm", "kernel": "lda_zf_kernel<7> (K=50, binary32-screened z draw)",
                         "achieved": achieved,
                         "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_source": peak_kind, "traffic": Z_KERNEL_DRAM_BYTES,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of "
                                           "this kernel on this workload (the capture summarised with its "
                                           "command in profiles/)",
                         "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": z_ms,
                         "note": "algorithmic bytes per token = 4 w + 4 z + 8 count RMW + 4K binary32 phi row, "
                                 "plus 12 D K per launch (theta rows, document counts)"},
            # the whole sweep against the 442 B/token byte model of the
            # binary64 formulation (4 w + 4 z + 8 (z, w) re-read + 8 count RMW
            # + 8K phi row, plus the count tables and draws per sweep)
            "sweep_roofline_frac": (T * 442.0) / (ms_max / args.steps / 1e3) / 1e9 / hbm,
            "sweep_critical_path": "phi first tries -> phi fix-up + normalise (theta beside them) -> z",
            "e2e": e2e,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(off, w, budget_s=args.cpu_seconds)
        if world == 1 and not args.no_secondary:
            # the other configurations, each measured in the same run (the
            # LDA line stands on its own if one of them fails)
            for key, fn in (("hlr_surrogate", lambda: run_hlr_surrogate(iters=args.hlr_iters,
                                                                         train_every=args.train_every,
                                                                         train_steps=args.train_steps,
                                                                         exact_plain=args.exact_plain,
                                                                         exact_sur=args.exact_sur)),
                            ("hlr_small", lambda: run_hlr_small(cpu=not args.no_cpu_baseline)),
                            ("gmm", lambda: run_gmm(cpu=not args.no_cpu_baseline)),
                            ("hlr_nuts", lambda: run_hlr_nuts(min_draws=args.nuts_draws,
                                                              max_rounds=args.nuts_rounds,
                                                              cpu=not args.no_cpu_baseline))):
                try:
                    line[key] = fn()
                except Exception as e:
                    line[key] = {"error": repr(e)[:300]}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return line


def time_z_kernel(s, stream, flush, reps):
    """Average duration of the production z launch - the binary32-screened
    kernel the sweep runs (ab_lda_disc_z_f32 on the sampler's own binary32
    copy of phi), with both count tables - L2 flushed and the topic-word table
    zeroed before each launch, outside its events."""
    import torch
    from augurv2_b200 import _native as N
    L = N.lib()
    Kq = L.ab_lda_phi32_stride(s.K)
    off32 = (int(L.ab_lda_phi_scratch_bytes(s.K, s.V)) + 255) & ~255
    phi32 = s.scratch[off32:off32 + 4 * s.V * Kq].view(torch.float32)
    z = s.z.clone()
    cdk = torch.zeros_like(s.cnt_dk)
    ckw = torch.zeros_like(s.cnt_kw)
    evs = []
    with torch.cuda.stream(stream):
        for i in range(reps + 2):
            flush.fill_(i & 0xFF)
            ckw.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            N.check(L.ab_lda_disc_z_f32(s.D, s.K, s.V, N.ptr(s.doc_off), N.ptr(s.w), N.ptr(s.theta),
                                        N.ptr(s.phiT), N.ptr(phi32), N.ptr(z), N.ptr(cdk), N.ptr(ckw), s.seed, 0,
                                        N.stream_ptr(stream)), "disc_z_f32")
            b.record(stream)
            evs.append((a, b))
    torch.cuda.synchronize()
    t = [a.elapsed_time(b) for a, b in evs[2:]]
    return sum(t) / len(t)


def run_e2e(args, off, w, seed, stream):
    """Same metric through the public Python API with host data: the corpus
    is uploaded from host memory inside the timed region, and every step
    copies the sample (theta, phi, z) back to host numpy arrays, as the
    reference's AugurInfer.samplen does (pyaugur/pyaugur/augurlib.py:195-222);
    LdaGibbs.samples overlaps each copy with the next sweep."""
    import torch
    from augurv2_b200.lda import LdaGibbs
    steps = args.steps
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        s = LdaGibbs(K_TOPICS, V_WORDS, off, w, ALPHA, BETA, seed=seed)
        d2h = 0
        for th, ph, z in s.samples(steps, stream=stream):
            d2h = th.nbytes + ph.nbytes + z.nbytes
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    s.close()
    h2d = off.nbytes + w.nbytes + 8 * (K_TOPICS + V_WORDS)
    return {"value": len(w) * steps / dt, "unit": "tokens/s", "seconds": dt,
            "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step": d2h,
            "note": "corpus upload + graph capture inside the timed region; sample copied to host every step (overlapping the next sweep)"}


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
    ap.add_argument("--no-secondary", action="store_true", help="skip the surrogate HLR measurement")
    ap.add_argument("--workload", default="lda",
                    choices=["lda", "hlr_surrogate", "hlr_pass", "hlr_small", "gmm", "hlr_nuts", "hlr_group"])
    ap.add_argument("--group-scale", type=float, default=1.0, help="hlr_group: factor on every instance's N")
    ap.add_argument("--nuts-rounds", type=int, default=2400, help="batched NUTS: round cap per instance")
    ap.add_argument("--nuts-draws", type=int, default=48, help="batched NUTS: draws per chain per instance")
    ap.add_argument("--hlr-n", type=int, default=HLR_N, help="rows for --workload hlr_pass")
    ap.add_argument("--hlr-iters", type=int, default=100)
    ap.add_argument("--train-every", type=int, default=8, help="surrogate: exact check + training period")
    ap.add_argument("--train-steps", type=int, default=10, help="surrogate: Adam steps per check")
    ap.add_argument("--exact-plain", type=int, default=1000,
                    help="surrogate exactness: iterations of the plain sampler's continuation (0: skip)")
    ap.add_argument("--exact-sur", type=int, default=3000,
                    help="surrogate exactness: iterations of the surrogate sampler's continuation")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    elif args.workload in ("hlr_small", "gmm"):
        import torch
        torch.cuda.set_device(local_rank)
        fn = run_hlr_small if args.workload == "hlr_small" else run_gmm
        line = fn(cpu=not args.no_cpu_baseline) if rank == 0 else None
    elif args.workload == "hlr_nuts":
        import torch
        torch.cuda.set_device(local_rank)
        line = run_hlr_nuts(min_draws=args.nuts_draws, max_rounds=args.nuts_rounds) if rank == 0 else None
    elif args.workload == "hlr_group":
        import torch
        torch.cuda.set_device(local_rank)
        line = run_hlr_group(args.group_scale, args.steps, args.warmup) if rank == 0 else None
    elif args.workload == "hlr_pass":
        import torch
        torch.cuda.set_device(local_rank)
        line = run_hlr_pass(args.hlr_n, args.steps, args.warmup) if rank == 0 else None
    elif args.workload == "hlr_surrogate":
        import torch
        torch.cuda.set_device(local_rank)
        line = run_hlr_surrogate(iters=args.hlr_iters, train_every=args.train_every,
                                 train_steps=args.train_steps, exact_plain=args.exact_plain,
                                 exact_sur=args.exact_sur) if rank == 0 else None
        if line is not None:
            line.update({"n_gpus": 1, "steps": args.hlr_iters, "warmup": 30, "higher_is_better": True,
                         "scaling": "weak", "vs_baseline": None, "dtype": "bf16 x3 parts, f32 accum, f64 energy",
                         "data": "synthetic (X ~ N(0,1) bf16, beta ~ Student-t(3), seed 5)"})
    else:
        line = run_ours(args, rank, world, local_rank)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
