"""Benchmark: input edges sparsified per second on one B200 (or N replicas under torchrun).

Workload (default): Erdos-Renyi G(n, p), n = 1,000,000, average degree 20 (m ~ 10M undirected edges),
weights uniform [0.5, 2] rounded to FP32, eps = 0.5, k = ceil(24 ln n / eps^2) = 1327 JL columns of
+-1/sqrt(k) Philox signs, PCG relative tolerance 1e-8 -- a single graph through the FP64 path.
A step is one full sparsification: device-resident input CSC -> device-resident L_H.

  python bench.py [--gpus N --steps K --warmup W]          # our GPU path
  python bench.py --impl reference [...]                    # the reference CPU path on the host cores
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (generator, kwargs, eps)
    "er_n1M_deg20": ("er", dict(n=1_000_000, avg_degree=20.0, wlo=0.5, whi=2.0, seed=1), 0.5),
    "grid2d_100": ("grid2d", dict(nx=100, ny=100), 0.5),
    "er_n100k_deg20": ("er", dict(n=100_000, avg_degree=20.0, wlo=0.5, whi=2.0, seed=1), 0.5),
    "er_n250k_deg20": ("er", dict(n=250_000, avg_degree=20.0, wlo=0.5, whi=2.0, seed=1), 0.5),
    # 3-D 7-point grids with log-uniform weights in [1e-3, 1e3] (the ill-conditioned mesh configuration)
    "grid3d_64": ("grid3d", dict(nx=64, ny=64, nz=64, lo=-3.0, hi=3.0, seed=2), 0.5),
    "grid3d_128": ("grid3d", dict(nx=128, ny=128, nz=128, lo=-3.0, hi=3.0, seed=2), 0.5),
    # the R-MAT configuration: scale 22, edge factor 16, (a, b, c) = (0.57, 0.19, 0.19), largest connected
    # component, LogNormal(0, 1) weights, eps 0.3 (k ~ 4000: the columns are solved in memory-sized batches)
    "rmat_s22": ("rmat", dict(scale=22, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=3), 0.3),
    "rmat_s18": ("rmat", dict(scale=18, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=3), 0.3),
}
PCG_TOL = 1e-8
# the arithmetic of each --precision: plain FP64; FP32 inner PCG inside FP64 refinement; FP64 PCG whose
# preconditioner (the triangular solves) runs in FP32
PREC_DTYPE = {"fp64": "f64", "mixed": "f32 inner PCG, f64 dots + refinement", "pc32": "f64 PCG, f32 preconditioner"}


def make_graph(S, name, rank=0):
    kind, kw, eps = WORKLOADS[name]
    kw = dict(kw)
    if kind == "er":
        kw["seed"] = kw["seed"] + rank
        return S.gen_er(kw["n"], kw["avg_degree"], kw["wlo"], kw["whi"], kw["seed"]), eps
    if kind == "grid3d":
        return S.gen_grid3d(kw["nx"], kw["ny"], kw["nz"], kw["lo"], kw["hi"], kw["seed"]), eps
    if kind == "rmat":
        return S.gen_rmat(kw["scale"], kw["edge_factor"], kw["a"], kw["b"], kw["c"], kw["seed"] + rank), eps
    return S.gen_grid2d(kw["nx"], kw["ny"]), eps


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    def __init__(self, device):
        self.device = device
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        def run():
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            try:
                p = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            except OSError:
                return
            while not self._stop.is_set():
                line = p.stdout.readline()
                if not line:
                    break
                self.samples.append([x.strip() for x in line.split(",")])
            p.terminate()
            try:
                p.wait(timeout=5)
            except Exception:
                p.kill()

        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        sm = []
        mx = None
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[1]))
                mx = float(s[2])
                for nm, val in zip(names, s[5:9]):
                    if val.lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM bytes per (Laplacian nonzero, 32-column tile) of one FP64 SpMM launch at ER n=1M, from the ncu
# capture of a one-tile solve of that graph (profiles/k_chunked_spmm_er_n1M_k32.md: 4.123 GB read + 0.287 GB
# written for nnz(L_G) = 21.003M nonzeros x 1 tile); every tile of a full launch does the same work
SPMM_TRAFFIC_PER_NNZ_TILE = 4.4093e9 / 21.003e6
SPMM_TILE = 32


def spmm_bytes(n, nnz_lap, k, s=8):
    # compulsory traffic of q = A p over k columns: row pointers, (index, value) per nonzero, read p, write q;
    # s = bytes per value (8 FP64, 4 for the FP32 inner solves of the mixed mode)
    return 8 * (n + 1) + nnz_lap * (4 + s) + 2 * n * k * s


def precond_bytes(n, nnz_l, k, s=8):
    # forward + backward triangular solves (each: pointers, L entries, read + write n x k) and D
    return 2 * (8 * (n + 1) + nnz_l * (4 + s) + 2 * n * k * s) + s * n


# ER sample sizes of the CPU legs (average degree 20, weights U[0.5, 2], the workload's generator and seed).
# The reference's factorization keeps its fill in a fixed edge pool of 5 nnz(L) entries (example.cc:336-337)
# and stops with "need more edge map capacity" (auxilliary.hpp:114-117) when it runs out: on ER with average
# degree 20 that happens from n = 650K on (the 1M workload always aborts), so the reference arm runs the
# largest size that completes, 600K, and steps down if a run there still aborts (the reference's fill
# sampler is seeded from random_device, example.cc:99-101).
REF_SAMPLE_LADDER = (600_000, 500_000, 400_000)
PORT_SAMPLE_N = 200_000
REF_UNAVAILABLE_AT_CONFIG = ("ER n=1M (the workload itself) aborts in the reference's factorization: assertion "
                             "'need more edge map capacity' (auxilliary.hpp:114-117; edge pool 5*nnz, "
                             "example.cc:336-337), log in profiles/reference_cpu_er_n1M_abort.md")


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as ora
    return ora


def cpu_baseline(eps, k_full, n_sample=PORT_SAMPLE_N, budget_cols=16):
    """The C port of every stage (the oracle) on one core over a bounded sample: ER n_sample, average degree
    20, the full pipeline with budget_cols of the k_full right-hand sides; the per-column cost (sketch, PCG
    solve, diff norms) is extrapolated to k_full.  Builds its input with the oracle's generator, so nothing
    of the library is involved."""
    ora = _oracle()
    v1, v2, w = ora.gen_er(n_sample, 20.0, 0.5, 2.0, 1)
    n = n_sample
    t0 = time.perf_counter()
    cp, ri, va = ora.laplacian(n, v1, v2, w)
    t_graph = time.perf_counter() - t0
    kc = budget_cols
    t0 = time.perf_counter()
    Y = ora.sketch(n, v1, v2, w, kc, 1.0 / math.sqrt(k_full), 0)
    t_sketch = time.perf_counter() - t0
    t0 = time.perf_counter()
    F = ora.Factor(n, cp, ri, va, 0, 4096, 64)
    t_fact = time.perf_counter() - t0
    t0 = time.perf_counter()
    Z, it, rel, rc = ora.pcg(n, cp, ri, va, F, Y, PCG_TOL, 0.0, 400)
    t_solve = time.perf_counter() - t0
    t0 = time.perf_counter()
    d = ora.diff_norms(v1, v2, Z)
    t_norms = time.perf_counter() - t0
    t0 = time.perf_counter()
    p = ora.probs(w, d, math.pow(eps, -2) * 4 * math.log(n), 1.0)
    ora.sample_apply(n, v1, v2, w, p, ora.coins(0, len(w)), 0, (cp, ri, va))
    t_tail = time.perf_counter() - t0
    per_col = (t_sketch + t_solve + t_norms) / kc
    total = t_graph + t_fact + per_col * k_full + t_tail
    measured = t_graph + t_fact + t_sketch + t_solve + t_norms + t_tail
    return {"value": len(w) / total, "unit": "edges/s", "cores": 1, "kind": "port",
            "sample": f"ER n={n} avg deg 20 (m={len(w)}), C port of every stage (the oracle), full pipeline with "
                      f"{kc} of k={k_full} right-hand sides, per-column cost extrapolated to k; measured "
                      f"{measured:.1f}s"}


def run_reference(args):
    """--impl reference: the reference's own CPU solver on this host's cores.

    The sample is the workload's graph family at the largest size the reference completes (ER n =
    REF_SAMPLE_N, average degree 20, k = the workload's 1327 columns).  One run of the reference solver
    (oracle/_ref/ref_solve: src/example.cc factorization_driver + include/custom_cg.hpp, all host threads)
    factors the Laplacian once and solves 2 (W + K) right-hand sides one after another, as the reference does
    (example.cc:551-568); the MKL shim records when each solve starts.  Warm-up step i covers right-hand sides
    2i and 2i + 1 and is discarded; timed step i covers the next pair.  A step's value is the input edges per
    second of the whole sparsification at k columns, extrapolated from that step's two solves:
        m / (assembly + set-up and factorization + k (solve + sketch + diff norms per column) + sampling)
    The Rust stages (Laplacian assembly, sketch, diff norms, probabilities, sampling) are the oracle's C port
    on one core.  Only oracle/ code runs here; nothing of the library is imported."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    _, kw, eps = WORKLOADS[args.workload]
    n_cfg = kw.get("n", 10_000)
    k = math.ceil(24 * math.log(n_cfg) / eps ** 2) if args.jl_cols <= 0 else args.jl_cols
    base = {"impl": "reference", "metric": "input edges sparsified/sec", "unit": "edges/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic"}
    ora = _oracle()
    import refsolver
    if args.workload != "er_n1M_deg20" and args.reference_n <= 0:
        print(json.dumps({**base, "unavailable": f"the reference arm samples the ER workload only "
                                                 f"(asked for {args.workload})"}), flush=True)
        return
    if not refsolver.available():
        # the reference's sources were not at hand where this tree was built: time the oracle port instead
        walls, vals = [], []
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            cb = cpu_baseline(eps, k, n_sample=100_000, budget_cols=4)
            if i >= args.warmup:
                walls.append((time.perf_counter() - t0) * 1e3)
                vals.append(cb["value"])
        v = statistics.median(vals)
        print(json.dumps({**base, "value": v, "ms_per_step": statistics.median(walls),
                          "config": {"workload": args.workload, "eps": eps, "k": k, "pcg_tol": PCG_TOL},
                          "unavailable_at_config": REF_UNAVAILABLE_AT_CONFIG,
                          "cpu_baseline": {**cb, "value": v},
                          "e2e": {"value": v, "unit": "edges/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    sizes = [args.reference_n] if args.reference_n > 0 else list(REF_SAMPLE_LADDER)
    threads = os.cpu_count()
    ncols = 2 * (args.warmup + args.steps)
    t_run0 = time.perf_counter()
    aborted = []
    for n in sizes:
        v1, v2, w = ora.gen_er(n, 20.0, 0.5, 2.0, 1)
        m = len(w)
        t0 = time.perf_counter()
        cp, ri, va = ora.laplacian(n, v1, v2, w)
        t_graph = time.perf_counter() - t0
        t0 = time.perf_counter()
        Y = ora.sketch(n, v1, v2, w, ncols, 1.0 / math.sqrt(k), 0)
        t_sketch_col = (time.perf_counter() - t0) / ncols
        try:
            status, secs, Z, starts = refsolver.solve(n, cp, ri, va, Y, threads=threads, timeout=3000,
                                                      timings=True)
            break
        except RuntimeError as e:
            msg = str(e).strip().splitlines()
            aborted.append(f"ER n={n}: {msg[-1][-240:] if msg else 'failed'}")
            sys.stderr.write(f"reference solver failed on ER n={n} avg deg 20:\n{e}\n")
    else:
        print(json.dumps({**base, "unavailable": "the reference solver failed on every sample size: " +
                                                 "; ".join(aborted)}), flush=True)
        return
    if status != 0 or len(starts) != ncols:
        print(json.dumps({**base, "unavailable": f"the reference solver did not converge on ER n={n} (status "
                                                 f"{status}, {len(starts)} of {ncols} solves started)"}),
              flush=True)
        return
    t_fact = float(starts[0])
    col_s = [float(b - a) for a, b in zip(starts[:-1], starts[1:])] + [float(secs - starts[-1])]
    t0 = time.perf_counter()
    d = ora.diff_norms(v1, v2, Z)
    t_norm_col = (time.perf_counter() - t0) / ncols
    t0 = time.perf_counter()
    p = ora.probs(w, d, math.pow(eps, -2) * 4 * math.log(n), 1.0)
    ora.sample_apply(n, v1, v2, w, p, ora.coins(0, m), 0, (cp, ri, va))
    t_tail = time.perf_counter() - t0
    wall = time.perf_counter() - t_run0
    vals, step_ms = [], []
    for i in range(args.warmup, args.warmup + args.steps):
        solve = 0.5 * (col_s[2 * i] + col_s[2 * i + 1])
        per_col = solve + t_sketch_col + t_norm_col
        vals.append(m / (t_graph + t_fact + k * per_col + t_tail))
        step_ms.append(2 * per_col * 1e3)
    v = statistics.median(vals)
    sample = (f"ER n={n} avg deg 20 (m={m}), the largest ER size the reference completes here; one run of the "
              f"reference's own solver (oracle/_ref: factorization_driver + example_pcg_solver, {threads} threads, "
              f"the reference's stopping rule) factoring once ({t_fact:.1f}s) and solving {ncols} right-hand sides "
              f"one after another (2 per step; the first {2 * args.warmup} are warm-up), per-column cost "
              f"extrapolated to k={k}; assembly, sketch, diff norms and sampling by the C port of the Rust stages "
              f"on 1 core; whole run {wall:.1f}s")
    line = {**base, "value": v, "ms_per_step": statistics.median(step_ms),
            "ms_per_sparsification_extrapolated": m / v * 1e3,
            "config": {"workload": args.workload, "eps": eps, "k": k, "pcg_tol": PCG_TOL,
                       "sample_n": n, "sample_m": m},
            "unavailable_at_config": REF_UNAVAILABLE_AT_CONFIG, "aborted_samples": aborted,
            "reference_solve_s_per_column_median": statistics.median(col_s), "reference_factor_s": t_fact,
            "cpu_baseline": {"value": v, "unit": "edges/s", "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": v, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def serving_mix(S, count, max_n, seed=4, precision="fp64", min_n=1000, eps_choices=(0.3, 0.5)):
    """The serving mix of seeded requests: random-geometric or ER graphs (equiprobable), n log-uniform in
    [min_n, max_n], average degree uniform in 8..32, weights uniform [0.1, 10] rounded to FP32, eps drawn from
    eps_choices (0.3 or 0.5).
    Every request asks for the autotuned factor without the dense tail (factor_max_degree = -1,
    dense_threshold = 0), so the server may batch it; the plain path runs the same parameters one request at a
    time."""
    import numpy as np
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        n = int(10 ** rng.uniform(math.log10(min_n), math.log10(max_n)))
        d = float(rng.integers(8, 33))
        eps = float(rng.choice(list(eps_choices)))
        G = S.gen_rgg(n, d, 0.1, 10.0, 1000 + i) if rng.random() < 0.5 else S.gen_er(n, d, 0.1, 10.0, 1000 + i)
        prm = S.SparsifierParameters.baseline(eps, pcg_tol=PCG_TOL, sampling_seed=i)
        prm.dense_threshold = 0
        prm.factor_max_degree = -1
        if precision == "mixed":
            prm.precision = S.SSP_PRECISION_MIXED
        reqs.append((G, prm))
    return reqs


def serve_measure(S, reqs, slots, max_batch, rate_frac=0.8, seed=5):
    """Closed loop (everything submitted at once) for the capacity, then Poisson arrivals at rate_frac of it;
    returns throughput, latency percentiles and the batching the server did."""
    import numpy as np
    m_total = sum(G.nnz // 2 for G, _ in reqs)

    def run_pass(srv, arrivals):
        t0 = time.perf_counter()
        tickets = [None] * len(reqs)

        def submitter():
            for i, (G, prm) in enumerate(reqs):
                delay = t0 + arrivals[i] - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                tickets[i] = srv.submit(G, prm)

        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        lat, batch = [], []
        for t in tickets:
            _, st, tm = srv.wait(t)
            lat.append(tm["latency_ms"])
            batch.append(tm["batch"])
        return time.perf_counter() - t0, lat, batch

    with S.Server(0, slots=slots, max_batch=max_batch) as srv:
        run_pass(srv, [0.0] * len(reqs))  # warm-up: workspaces grow, modules load
        cap_s, _, _ = run_pass(srv, [0.0] * len(reqs))
        rate = rate_frac * len(reqs) / cap_s
        rng = np.random.default_rng(seed)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs))).tolist()
        wall, lat, batch = run_pass(srv, arrivals)
        info = srv.info()
    return {"value": m_total / wall, "unit": "edges/s", "closed_loop_edges_per_s": m_total / cap_s,
            "arrivals": f"Poisson at {rate:.2f} req/s ({rate_frac} x closed-loop capacity)",
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(np.mean(lat)), "slots": slots, "max_batch": max_batch,
            "mean_batch": float(np.mean(batch)), "peak_batch": info["peak_batch"], "runs": info["batches"],
            "peak_inflight": info["peak_inflight"], "peak_inflight_bytes": info["peak_inflight_bytes"]}


def plain_measure(S, reqs):
    """The plain single-graph path: each request alone through ssp_sparsify on one context, back to back (the
    same parameters; with the default dense tail as well, reported beside)."""
    ctx = S.Context(0)
    try:
        ctx.sparsify(*reqs[0])  # warm-up
        t0 = time.perf_counter()
        for G, prm in reqs:
            ctx.sparsify(G, prm)
        wall = time.perf_counter() - t0
    finally:
        ctx.close()
    return sum(G.nnz // 2 for G, _ in reqs) / wall


def serving_section(S, count, max_n, slots=2, max_batch=64, min_n=1000, eps_choices=(0.3, 0.5)):
    """The serving mix on the plain path, through the server without batching (slots only) and with
    continuous batching, in FP64 and in mixed precision."""
    reqs = serving_mix(S, count, max_n, min_n=min_n, eps_choices=eps_choices)
    m_total = sum(G.nnz // 2 for G, _ in reqs)
    plain = plain_measure(S, reqs)
    # the library's default single-graph parameters (autotuned factor with the dense tail)
    plain_default = plain_measure(S, [(G, S.SparsifierParameters.baseline(p.epsilon, pcg_tol=PCG_TOL,
                                                                          sampling_seed=p.sampling_seed))
                                      for G, p in reqs])
    slots_only = serve_measure(S, reqs, 4, 1)
    batched = serve_measure(S, reqs, slots, max_batch)
    batched_mixed = serve_measure(S, serving_mix(S, count, max_n, precision="mixed", min_n=min_n,
                                                 eps_choices=eps_choices), slots, max_batch)
    return {"workload": "serving mix", "requests": count, "n_range": [min_n, max_n], "degree_range": [8, 32],
            "eps": list(eps_choices), "edges": m_total,
            "plain_fp64_edges_per_s": plain, "plain_fp64_default_params_edges_per_s": plain_default,
            "served_slots_only_fp64": slots_only,
            "served_batched_fp64": batched, "served_batched_mixed": batched_mixed,
            "batched_mixed_over_plain": batched_mixed["value"] / plain,
            "batched_fp64_over_plain": batched["value"] / plain,
            "batched_mixed_over_plain_default": batched_mixed["value"] / plain_default}


def serving_lite(S, count=48, max_n=20_000, slots=2, max_batch=64):
    """The serving mix at a bounded size for the default line: the plain FP64 path one request after another,
    then the request loop with continuous batching (closed loop for capacity, then Poisson arrivals at 0.8 of
    it) with p50/p99 latency."""
    reqs = serving_mix(S, count, max_n)
    plain = plain_measure(S, reqs)
    batched = serve_measure(S, reqs, slots, max_batch)
    return {"workload": "serving mix", "requests": count, "n_range": [1000, max_n], "degree_range": [8, 32],
            "eps": [0.3, 0.5], "edges": sum(G.nnz // 2 for G, _ in reqs), "dtype": "f64",
            "plain_fp64_edges_per_s": plain, "value": batched["value"], "unit": "edges/s",
            "p50_ms": batched["p50_ms"], "p99_ms": batched["p99_ms"], "served_batched_fp64": batched,
            "batched_over_plain": batched["value"] / plain,
            "batched_closed_loop_over_plain": batched["closed_loop_edges_per_s"] / plain}


def run_serve(args):
    """--serve: the serving mix through the persistent request loop (ssp_server_*), beside the plain path."""
    import spec_spars_b200 as S
    sec = serving_section(S, args.serve_requests, args.serve_max_n, args.serve_slots, args.serve_batch,
                          args.serve_min_n, tuple(float(x) for x in args.serve_eps.split(",")))
    best = sec["served_batched_mixed"] if args.precision == "mixed" else sec["served_batched_fp64"]
    line = {"metric": "serving mix: input edges sparsified/sec", "value": best["value"], "unit": "edges/s",
            "n_gpus": 1, "higher_is_better": True, "dtype": "f64" if args.precision == "fp64" else "mixed",
            "data": "synthetic", "config": {k: sec[k] for k in ("workload", "requests", "n_range", "degree_range",
                                                              "eps", "edges")},
            "p50_ms": best["p50_ms"], "p99_ms": best["p99_ms"], "serving": sec}
    print(json.dumps(line), flush=True)


def run_precond(args):
    """--precond-cols N: M^-1 applied to N seeded standard-normal columns with the workload's complete factor
    (stage entry point ssp_stage_precond, dense-tail threshold 4096), twice; prints the host-side seconds of
    each call.  For profiling the triangular solves alone."""
    import numpy as np
    import spec_spars_b200 as S
    G, _ = make_graph(S, args.workload)
    ctx = S.Context(0)
    _, L = S.stage_graph(ctx, G)
    R = np.random.default_rng(0).standard_normal((G.n, args.precond_cols))
    secs = []
    for _ in range(2):
        t = time.perf_counter()
        S.stage_precond(ctx, L, 0, R, 4096, 0)
        secs.append(time.perf_counter() - t)
    print(json.dumps({"workload": args.workload, "n": G.n, "columns": args.precond_cols, "seconds": secs}), flush=True)
    ctx.close()


def run_mtx(args):
    """--mtx: the Matrix Market path of sparsify_dataset on the workload's graph.  Timed: the GPU reader and
    writer (ssp_read_mtx_device / ssp_write_mtx_device, file in the page cache) and sparsify_dataset file to
    file; beside them the host reader and writer they replace (one pass each).  Both readers must return the
    same CSC and both writers the same bytes."""
    import tempfile
    import numpy as np
    import spec_spars_b200 as S
    G, eps = make_graph(S, args.workload)
    d = tempfile.mkdtemp(prefix="ssp_mtx_")
    src, out_h, out_d, out_s = (os.path.join(d, x) for x in ("g.mtx", "h.mtx", "d.mtx", "s.mtx"))
    S.write_mtx(src, G)
    size = os.path.getsize(src)
    ctx = S.Context(0)
    for _ in range(max(1, args.warmup)):
        ctx.read_mtx(src)
        ctx.write_mtx(out_d, G)
    t = time.perf_counter()
    for _ in range(args.steps):
        Hd = ctx.read_mtx(src)
    t_read = (time.perf_counter() - t) / args.steps
    t = time.perf_counter()
    for _ in range(args.steps):
        ctx.write_mtx(out_d, G)
    t_write = (time.perf_counter() - t) / args.steps
    wsize = os.path.getsize(out_d)
    S.sparsify_dataset(src, args.workload, out_s, eps, False, 0, 0, False)
    t = time.perf_counter()
    for _ in range(args.steps):
        st = S.sparsify_dataset(src, args.workload, out_s, eps, False, 0, 0, False)
    t_ds = (time.perf_counter() - t) / args.steps
    t = time.perf_counter()
    Hh = S.read_mtx(src)
    th_read = time.perf_counter() - t
    t = time.perf_counter()
    S.write_mtx(out_h, G)
    th_write = time.perf_counter() - t
    same_read = (np.array_equal(Hh.colptr, Hd.colptr) and np.array_equal(Hh.rowidx, Hd.rowidx)
                 and np.array_equal(Hh.values.view(np.uint64), Hd.values.view(np.uint64)))
    with open(out_h, "rb") as a, open(out_d, "rb") as b:
        same_write = a.read() == b.read()
    m = G.nnz // 2
    line = {"metric": "Matrix Market read: file bytes/sec", "value": size / t_read, "unit": "B/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "text -> f64",
            "data": "synthetic", "config": {"workload": args.workload, "file_bytes": size, "entries": int(G.nnz),
                                            "written_bytes": wsize, "page_cache": "file read from the page cache"},
            "read_s": t_read, "write_s": t_write, "write_bytes_per_s": wsize / t_write,
            "sparsify_dataset": {"s": t_ds, "edges_per_s": m / t_ds, "m_out": st.final_num_edges},
            "cpu_baseline": {"read_s": th_read, "write_s": th_write, "cores": 1, "kind": "port",
                             "sample": "the same file, host reader and writer (read_mtx / write_mtx restated)"},
            "same_csc": bool(same_read), "same_bytes": bool(same_write)}
    print(json.dumps(line), flush=True)
    for f in (src, out_h, out_d, out_s):
        os.remove(f)
    os.rmdir(d)


def spectral_check(S, ctx, LG, H, eps, st, probes=100):
    """probe_quadratic_form (experiments.rs:88-122) on the device: x^T L_H x against x^T L_G x for 100
    seeded uniform(-1, 1) probes, with the (1 +- eps) violation counts."""
    r = ctx.probe_quadratic_form(LG, H, eps, probes=probes, seed=11)
    return {"probes": r["probes"], "eps": eps, "upper_violations": r["upper_bound_violations"],
            "lower_violations": r["lower_bound_violations"], "max_rel_err": r["max_relative_error"],
            "mean_rel_err": r["mean_relative_error"], "kept_fraction": st["m_out"] / st["m_in"],
            "passed": r["upper_bound_violations"] == 0 and r["lower_bound_violations"] == 0}


def trsv_info(S, first, last):
    """How the preconditioner's level-launch shapes were chosen: measured on the first step (device ms spent),
    then taken from the context's cache; level launches at 8/16/32 columns per warp row."""
    src = {S.SSP_TRSV_RULE: "rule", S.SSP_TRSV_TUNED: "measured", S.SSP_TRSV_CACHED: "cached",
           S.SSP_TRSV_FORCED: "forced"}
    return {"first_step": src.get(first["trsv_shapes"], "?"), "timed_steps": src.get(last["trsv_shapes"], "?"),
            "ms_measuring": first["ms_trsv_tune"],
            "level_launches_w8_w16_w32": [last["trsv_levels_w8"], last["trsv_levels_w16"], last["trsv_levels_w32"]]}


def mesh_step(S, ctx, stream, name="grid3d_128"):
    """The ill-conditioned mesh configuration (3-D 7-point grid 128^3, weights log-uniform over six decades,
    eps 0.5, k = ceil(24 ln n / eps^2) = 1398, PCG tol 1e-8, FP64): one untimed step, one timed step (CUDA
    events on the library's stream), with the preconditioner's roofline (it dominates there) and the
    spectral check of the output."""
    import torch
    G, eps = make_graph(S, name)
    prm = S.SparsifierParameters.baseline(eps, pcg_tol=PCG_TOL)
    dev = torch.device("cuda", torch.cuda.current_device())
    cp = torch.from_numpy(G.colptr).to(dev)
    ri = torch.from_numpy(G.rowidx).to(dev)
    va = torch.from_numpy(G.values).to(dev)
    _, LG = S.stage_graph(ctx, G)
    torch.cuda.synchronize()
    _, st0 = ctx.sparsify_device(G.n, G.nnz, cp.data_ptr(), ri.data_ptr(), va.data_ptr(), prm)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    H_dev, st = ctx.sparsify_device(G.n, G.nnz, cp.data_ptr(), ri.data_ptr(), va.data_ptr(), prm)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    spec = spectral_check(S, ctx, LG, S.DeviceCSC(G.n, *H_dev), eps, st)
    peak, src = peaks()
    n, k = st["n"], st["k"]
    pc_ms = st["ms_precond"] / max(1, st["n_precond"])
    sp_ms = st["ms_spmm"] / max(1, st["n_spmm"])
    pb = precond_bytes(n, st["nnz_factor"], k)
    out = {"workload": name, "n": n, "m": st["m_in"], "eps": eps, "k": k, "pcg_tol": PCG_TOL, "dtype": "f64",
           "ms_per_step": ms, "value": st["m_in"] / (ms / 1000.0), "unit": "edges/s", "steps": 1, "warmup": 1,
           "kept_fraction": st["m_out"] / st["m_in"], "pcg_iters_max": st["pcg_max_iters_used"],
           "factor_nnz": st["nnz_factor"], "factor_levels": st["factor_levels"],
           "factor_max_degree_used": st["factor_max_degree_used"], "trsv_shapes": trsv_info(S, st0, st),
           "stages_ms": {x: st[x] for x in ("ms_assembly", "ms_sketch", "ms_factor", "ms_solve", "ms_leverage",
                                            "ms_sample", "ms_total")},
           "roofline": {"kernel": "precond (fwd+bwd level-set triangular solves, all k columns)", "bound": "hbm",
                        "achieved": pb / (pc_ms / 1000.0) / 1e9 if pc_ms > 0 else None, "peak": peak,
                        "unit": "GB/s", "peak_source": src, "avg_launch_ms": pc_ms, "algorithmic_bytes_per_launch": pb,
                        "frac": pb / (pc_ms / 1000.0) / 1e9 / peak if pc_ms > 0 else None,
                        "spmm_avg_ms": sp_ms},
           "spectral": spec}
    del cp, ri, va
    return out


def run_sharded(args, S, torch, dist, world, rank, local):
    """--gpus N (N > 1): ONE graph with its k JL columns split over the N ranks (spec_spars_b200.sharded's
    scheme): every rank factors the same graph, sketches and solves its tile-aligned share of the columns
    (ssp_shard_leverage), one NCCL all-reduce(sum) of the m per-edge partial squares, then every rank forms
    the same probabilities, coins and L_H (ssp_shard_finish).  Total work is fixed (strong scaling); value =
    the graph's input edges / (max over ranks of the device time per step)."""
    from spec_spars_b200.sharded import column_range
    G, eps = make_graph(S, args.workload)  # the same graph on every rank
    prm = S.SparsifierParameters.baseline(eps, pcg_tol=PCG_TOL)
    if args.jl_cols > 0:
        prm.jl_dim_override = args.jl_cols
    if args.precision == "mixed":
        prm.precision = S.SSP_PRECISION_MIXED
    elif args.precision == "pc32":
        prm.precision = S.SSP_PRECISION_PC32
    ctx = S.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    dev = torch.device("cuda", local)
    cp = torch.from_numpy(G.colptr).to(dev)
    ri = torch.from_numpy(G.rowidx).to(dev)
    va = torch.from_numpy(G.values).to(dev)
    Gd = S.DeviceCSC(G.n, G.nnz, cp.data_ptr(), ri.data_ptr(), va.data_ptr())
    m = ctx.num_edges(Gd)
    k = prm.jl_dim(G.n)
    c0, c1 = column_range(k, world, rank)
    sq = torch.zeros(max(m, 1), dtype=torch.float64, device=dev)

    def step():
        part = {}
        if c1 > c0:
            part = ctx.shard_leverage(Gd, prm, c0, c1, sq.data_ptr())
        else:
            sq.zero_()
        dist.all_reduce(sq, op=dist.ReduceOp.SUM)
        _, st = ctx.shard_finish(Gd, prm, sq.data_ptr(), device_out=True)
        return part, st

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    k0 = ctx.kernels_launched
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    dist.barrier()
    e0.record(stream)
    for _ in range(args.steps):
        part, st = step()
    e1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    clocks.stop()
    launches = ctx.kernels_launched - k0
    ms = e0.elapsed_time(e1) / args.steps
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    # end to end: host graph in, host L_H out, every step (the graph's H2D on every rank)
    Gh = G

    def step_host():
        if c1 > c0:
            ctx.shard_leverage(Gh, prm, c0, c1, sq.data_ptr())
        else:
            sq.zero_()
        dist.all_reduce(sq, op=dist.ReduceOp.SUM)
        return ctx.shard_finish(Gh, prm, sq.data_ptr())

    step_host()
    torch.cuda.synchronize()
    dist.barrier()
    h0 = torch.cuda.Event(enable_timing=True)
    h1 = torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    for _ in range(args.e2e_steps):
        H, _ = step_host()
    h1.record(stream)
    torch.cuda.synchronize()
    ems = h0.elapsed_time(h1) / max(1, args.e2e_steps)
    t = torch.tensor([ems], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ems = float(t.item())
    if rank == 0:
        line = {"metric": "input edges sparsified/sec", "value": m / (ms / 1000.0), "unit": "edges/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": PREC_DTYPE[args.precision],
                "data": "synthetic",
                "config": {"workload": args.workload, "n": G.n, "m": m, "eps": eps, "k": k, "pcg_tol": PCG_TOL,
                           "precision": args.precision,
                           "parallelism": f"JL columns split over {world} ranks, one NCCL all-reduce of m doubles",
                           "columns_rank0": [c0, c1],
                           "l2": "inputs and n-by-k working set larger than L2; no flush"},
                "gpu_launches": launches, "kept_fraction": st["m_out"] / st["m_in"],
                "pcg_iters_max": part.get("pcg_max_iters_used"), "clocks": clocks.summary(),
                "e2e": {"value": m / (ems / 1000.0), "unit": "edges/s",
                        "h2d_bytes_per_step": G.colptr.nbytes + G.rowidx.nbytes + G.values.nbytes,
                        "d2h_bytes_per_step": H.colptr.nbytes + H.rowidx.nbytes + H.values.nbytes,
                        "ms_per_step": ems}}
        print(json.dumps(line), flush=True)
    del sq
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="er_n1M_deg20", choices=list(WORKLOADS))
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed", "pc32"],
                    help="PCG arithmetic: fp64; mixed (FP32 inner solves inside FP64 refinement to the same tolerance); "
                         "pc32 (FP64 PCG with the preconditioner in FP32)")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the secondary mixed-precision measurement reported beside the FP64 headline")
    ap.add_argument("--jl-cols", type=int, default=0,
                    help="use this many JL columns instead of ceil(24 ln n / eps^2) (smaller profiling cases)")
    ap.add_argument("--serve", action="store_true", help="run the serving mix through the request loop")
    ap.add_argument("--serve-requests", type=int, default=64)
    ap.add_argument("--serve-max-n", type=int, default=100_000)
    ap.add_argument("--serve-min-n", type=int, default=1000)
    ap.add_argument("--serve-eps", default="0.3,0.5", help="comma-separated eps values the requests draw from")
    ap.add_argument("--serve-slots", type=int, default=2)
    ap.add_argument("--serve-batch", type=int, default=64)
    ap.add_argument("--mtx", action="store_true", help="time the GPU Matrix Market reader/writer and sparsify_dataset")
    ap.add_argument("--precond-cols", type=int, default=0,
                    help="apply the workload's complete preconditioner to this many columns, twice (profiling)")
    ap.add_argument("--mode", default="auto", choices=["auto", "sharded", "replicas"],
                    help="N > 1: split one graph's JL columns over the ranks (auto, sharded) or run N independent "
                         "replicas, one graph each (replicas)")
    ap.add_argument("--no-complete", dest="complete", action="store_false",
                    help="leave out the one-step complete-elimination measurement of the default line")
    ap.add_argument("--no-serving", dest="serving", action="store_false",
                    help="leave out the bounded serving-mix measurement of the default line")
    ap.add_argument("--no-mesh", dest="mesh", action="store_false",
                    help="skip the one-step grid3d_128 measurement reported beside the ER headline")
    ap.add_argument("--reference-n", type=int, default=0,
                    help="--impl reference: ER sample size (default: the largest size the reference completes)")
    args = ap.parse_args()
    if args.serve:
        run_serve(args)
        return
    if args.mtx:
        run_mtx(args)
        return
    if args.precond_cols > 0:
        run_precond(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist
    import spec_spars_b200 as S

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1 or args.mode == "sharded":
        import datetime
        # the communicator's set-up lines show the rank count (--mode sharded also runs on one rank, where
        # the all-reduce is the identity)
        os.environ.setdefault("NCCL_DEBUG", "INFO")
        os.environ.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
        for key, val in (("MASTER_ADDR", "127.0.0.1"), ("MASTER_PORT", "29511"), ("RANK", "0"), ("WORLD_SIZE", "1")):
            os.environ.setdefault(key, val)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        if args.mode != "replicas":
            run_sharded(args, S, torch, dist, world, rank, local)
            dist.destroy_process_group()
            return

    G, eps = make_graph(S, args.workload, rank)
    prm = S.SparsifierParameters.baseline(eps, pcg_tol=PCG_TOL)
    if args.jl_cols > 0:
        prm.jl_dim_override = args.jl_cols
    if args.precision == "mixed":
        prm.precision = S.SSP_PRECISION_MIXED
    elif args.precision == "pc32":
        prm.precision = S.SSP_PRECISION_PC32
    ctx = S.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    dev = torch.device("cuda", local)
    cp = torch.from_numpy(G.colptr).to(dev)
    ri = torch.from_numpy(G.rowidx).to(dev)
    va = torch.from_numpy(G.values).to(dev)
    torch.cuda.synchronize()

    def step():
        return ctx.sparsify_device(G.n, G.nnz, cp.data_ptr(), ri.data_ptr(), va.data_ptr(), prm)

    # L_G as the library forms it, for the spectral check of the timed steps' output (untimed)
    _, LG = S.stage_graph(ctx, G)
    warm = []
    for _ in range(args.warmup):
        _, st = step()
        warm.append(st)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    k0 = ctx.kernels_launched
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t_start.record(stream)
    stats = []
    for _ in range(args.steps):
        H_dev, st = step()
        stats.append(st)
    t_end.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks.stop()
    # "at verified eps": the last timed step's L_H, still in the context, against L_G on seeded probes
    spectral = spectral_check(S, ctx, LG, S.DeviceCSC(G.n, *H_dev), eps, stats[-1])
    launches = ctx.kernels_launched - k0
    ms = t_start.elapsed_time(t_end) / args.steps
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    m = stats[-1]["m_in"]
    value = m * world / (ms / 1000.0)

    # end to end through the public API with host buffers (H2D of the input, D2H of L_H, every step)
    e2e = None
    if args.e2e_steps > 0:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        h2d = G.colptr.nbytes + G.rowidx.nbytes + G.values.nbytes
        d2h = 0
        ctx.sparsify(G, prm)  # untimed: the host path's one-time set-up (its pinned staging ring)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.e2e_steps):
            H, st2 = ctx.sparsify(G, prm)
            d2h = H.colptr.nbytes + H.rowidx.nbytes + H.values.nbytes
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1) / args.e2e_steps
        if world > 1:
            t = torch.tensor([ems], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {"value": m * world / (ems / 1000.0), "unit": "edges/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": ems}

    st = stats[-1]
    n, k = st["n"], st["k"]
    peak, src = peaks()
    sp_ms = sum(s["ms_spmm"] for s in stats) / max(1, sum(s["n_spmm"] for s in stats))
    pc_ms = sum(s["ms_precond"] for s in stats) / max(1, sum(s["n_precond"] for s in stats))
    sp_tot = sum(s["ms_spmm"] for s in stats)
    pc_tot = sum(s["ms_precond"] for s in stats)
    vs = 4 if args.precision == "mixed" else 8
    if pc_tot >= sp_tot:
        kern, byts, kms = "precond (fwd+bwd level-set triangular solves, all k columns)", \
            precond_bytes(n, st["nnz_factor"], k, vs), pc_ms
    else:
        kern, byts, kms = "spmm (Laplacian x n-by-k block)", spmm_bytes(n, st["nnz_laplacian"], k, vs), sp_ms
    achieved = byts / (kms / 1000.0) / 1e9 if kms > 0 else None
    traffic = None
    if kern.startswith("spmm") and vs == 8:
        # scaled from the small-case capture by the units one launch processes
        traffic = SPMM_TRAFFIC_PER_NNZ_TILE * st["nnz_laplacian"] * math.ceil(k / SPMM_TILE)
    roof = {"kernel": kern, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if achieved else None, "traffic": traffic, "peak_source": src,
            # the DRAM bytes the launch really moves (traffic) per second, against the same peak
            "traffic_GBps": traffic / (kms / 1000.0) / 1e9 if traffic and kms > 0 else None,
            "traffic_frac": traffic / (kms / 1000.0) / 1e9 / peak if traffic and kms > 0 else None,
            "algorithmic_bytes_per_launch": byts, "avg_launch_ms": kms,
            "spmm_avg_ms": sp_ms, "precond_avg_ms": pc_ms,
            "spmm_GBps": spmm_bytes(n, st["nnz_laplacian"], k, vs) / (sp_ms / 1000.0) / 1e9 if sp_ms > 0 else None,
            "precond_GBps": precond_bytes(n, st["nnz_factor"], k, vs) / (pc_ms / 1000.0) / 1e9 if pc_ms > 0 else None}
    line = {"metric": "input edges sparsified/sec", "value": value, "unit": "edges/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": PREC_DTYPE[args.precision],
            "data": "synthetic",
            "config": {"workload": args.workload, "n": n, "m": m, "eps": eps, "k": k, "pcg_tol": PCG_TOL,
                       "precision": args.precision,
                       "l2": "inputs and n-by-k working set larger than L2; no flush",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "gpu_launches": launches,
            "stages_ms": {x: st[x] for x in ("ms_assembly", "ms_sketch", "ms_factor", "ms_solve", "ms_leverage",
                                             "ms_sample", "ms_total")},
            "kept_fraction": st["m_out"] / st["m_in"], "pcg_iters_max": st["pcg_max_iters_used"],
            "pcg_iters_mean": st["pcg_mean_iters"], "pcg_max_relres": st["pcg_max_relres"],
            "pcg_refinements": st["pcg_refinements"], "pcg_fp64_rounds": st["pcg_fp64_rounds"],
            "spmm_slabs": st["spmm_slabs"], "factor_nnz": st["nnz_factor"], "factor_levels": st["factor_levels"],
            "trsv_shapes": trsv_info(S, warm[0] if warm else stats[0], st),
            "roofline": roof, "spectral": spectral, "clocks": clocks.summary(), "e2e": e2e}
    if args.precision == "fp64" and not args.no_mixed:
        # the same workload with FP32 inner solves inside FP64 refinement (same PCG tolerance), beside the
        # plain FP64 headline; one untimed step, then two timed ones, on the same stream and clock rules
        prm.precision = S.SSP_PRECISION_MIXED
        step()
        torch.cuda.synchronize()
        m0 = torch.cuda.Event(enable_timing=True)
        m1 = torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        for _ in range(2):
            _, stm = step()
        m1.record(stream)
        torch.cuda.synchronize()
        mms = m0.elapsed_time(m1) / 2
        if world > 1:
            t = torch.tensor([mms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            mms = float(t.item())
        line["mixed_precision"] = {"value": m * world / (mms / 1000.0), "unit": "edges/s", "ms_per_step": mms,
                                   "dtype": "f32 inner PCG, f64 dots + refinement",
                                   "pcg_max_relres": stm["pcg_max_relres"], "pcg_iters_max": stm["pcg_max_iters_used"],
                                   "pcg_refinements": stm["pcg_refinements"], "spmm_slabs": stm["spmm_slabs"],
                                   "spmm_avg_ms": stm["ms_spmm"] / max(1, stm["n_spmm"])}
        prm.precision = S.SSP_PRECISION_FP64
    if args.complete and world == 1:
        # the reference's own preconditioner, complete elimination (example.cc:91-323), beside the autotuner's
        # choice: one timed step (23 s at ER 1M), with the fixed rule's level shapes so that no shape
        # measurement falls inside it
        deg = prm.factor_max_degree
        prm.factor_max_degree = 0
        old_tune = os.environ.get("SSP_TRSV_TUNE")
        os.environ["SSP_TRSV_TUNE"] = "0"
        torch.cuda.synchronize()
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        _, stc = step()
        c1.record(stream)
        torch.cuda.synchronize()
        cms = c0.elapsed_time(c1)
        if old_tune is None:
            del os.environ["SSP_TRSV_TUNE"]
        else:
            os.environ["SSP_TRSV_TUNE"] = old_tune
        line["complete_elimination"] = {
            "value": m / (cms / 1000.0), "unit": "edges/s", "ms_per_step": cms, "dtype": "f64", "steps": 1,
            "trsv_shapes": "rule",
            "pcg_iters_max": stc["pcg_max_iters_used"], "ms_factor": stc["ms_factor"],
            "factor_nnz": stc["nnz_factor"], "factor_levels": stc["factor_levels"],
            "precond_avg_ms": stc["ms_precond"] / max(1, stc["n_precond"]),
            "spmm_avg_ms": stc["ms_spmm"] / max(1, stc["n_spmm"]),
            "autotuned_choice": {"factor_max_degree": st["factor_max_degree_used"], "factor_nnz": st["nnz_factor"],
                                 "factor_levels": st["factor_levels"], "pcg_iters_max": st["pcg_max_iters_used"],
                                 "ms_factor": st["ms_factor"]}}
        prm.factor_max_degree = deg
    if args.mesh and world == 1 and args.workload == "er_n1M_deg20":
        # the mesh configuration beside the headline, on a released workspace (its n x k blocks are 141 GB)
        ctx.release_workspace()
        try:
            line["mesh_grid3d_128"] = mesh_step(S, ctx, stream)
        except Exception as e:  # reported, never fatal to the headline
            line["mesh_grid3d_128"] = {"error": f"{type(e).__name__}: {e}"[:400]}
    if args.serving and world == 1 and args.workload == "er_n1M_deg20":
        # the serving mix through the request loop, beside the headline (its own contexts; ours released)
        ctx.release_workspace()
        try:
            line["serving"] = serving_lite(S)
        except Exception as e:  # reported, never fatal to the headline
            line["serving"] = {"error": f"{type(e).__name__}: {e}"[:400]}
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(eps, k)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
