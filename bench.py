#!/usr/bin/env python
"""PageRank throughput on one B200 (or N replicas): RMAT scale 24.

Workload (the configuration the metric is quoted on): seeded RMAT graph,
scale 24 (16,777,216 vertices), edge factor 16, (a,b,c,d) =
(0.57, 0.19, 0.19, 0.05), self-loops and duplicate edges removed, int32 pull
CSR + out-degree; plain pull PageRank in FP32 with an FP64 L1 residual,
damping 0.85f, tolerance 1e-6, at most 100 sweeps, uniform 1/m start.

One step = one complete solve (score initialisation, every sweep until the
residual drops below the tolerance, scores scattered back to vertex order) on
the device-resident graph.  value = GTEPS = edges x sweeps / time, summed
over ranks (replicas, weak scaling).  The graph (1.07 GB of CSR) is larger
than L2, so no flush is needed between steps.

--impl reference times the reference's own OpenMP PRSolver
(src/pr/omp_base.cc, compiled from the reference tree into oracle/_ref) on
the same graph on the host cores: each step is a bounded sample of the same
solve (SAMPLE_SWEEPS sweeps over the full graph).
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SCALE, EDGE_FACTOR, SEED = 24, 16, 1
ABC = (0.57, 0.19, 0.19)
TOL, MAX_ITER = 1e-6, 100
DAMPING = np.float32(0.85)
SAMPLE_SWEEPS = 2            # reference / CPU-baseline sample: sweeps per call
CPU_BASELINE_BUDGET_S = 12.0  # CPU work for the cpu_baseline leg


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def pr_bytes_per_sweep(m, nnz):
    """Algorithmic bytes of one plain FP32 sweep: 4 nnz (column indices) +
    4 (m+1) (row offsets) + 12 m (contribution: read score, read degree,
    write contribution) + 4 m (contributions gathered, counted once) + 8 m
    (read old score, write new score)  =  4 nnz + 28 m + 4."""
    return 4 * nnz + 28 * m + 4


# The BF16 + FP32-refinement results are reported as a study, not as a form
# of the metric: a sweep here is bound by the latency and count of its gather
# requests, not by their bytes, so a BF16 sweep costs what an FP32 sweep
# costs, and the refinement back to the FP32 error needs as many FP32 sweeps
# as the plain solve would have taken from the BF16 start.
BF16_NOTE = ("measured, not a gain: BF16 halves gather bytes but the sweep is bound by "
             "request latency and count, so a BF16 sweep costs what an FP32 sweep costs; "
             "refining to the FP32 error then adds sweeps (time to solution >= plain)")

# Random 4-byte gathers served by L2 on one B200, whole GPU (requests/s):
# profiles/gather_rates.md, 289-296 G/s for L2-resident working sets.
L2_GATHER_RATE = 290e9


def spmv_bytes(m, nnz):
    """Aj + Ax (8 nnz) + row offsets (4 (m+1)) + x once (4 m) + y read/write (8 m)."""
    return 8 * nnz + 16 * m + 4


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.f = tempfile.TemporaryFile(mode="w+")

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.seek(0)
        rows = []
        for line in self.f:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 10 or (self.uuid and p[1] != self.uuid):
                continue
            rows.append(p)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[2]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[6:10]) if v.lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": float(rows[0][3]),
                "samples": len(rows), "power_w_max": max(float(r[4]) for r in rows),
                "reasons": reasons}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def init_dist(world, local, use_cuda=True, timeout_s=120):
    """One process per GPU (replicas): NCCL on GPUs, gloo on CPU; the group
    carries only barriers and the max-over-ranks timings.  None at N = 1."""
    if world <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist
    if use_cuda:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=timeout_s),
                                device_id=torch.device("cuda", local))
    else:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(x, dist, device=None):
    """The largest x over all ranks (the timing of a multi-rank step)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world, units_per_rank, seconds):
    """Whole-job rate of `world` replicas that each processed units_per_rank
    in (at most) `seconds`."""
    return world * units_per_rank / seconds


def cpu_reference_sample(rp, col, od, sweeps, budget_s, min_calls=1):
    """Time the reference's OpenMP PRSolver (oracle/_ref) or, without it, the
    oracle port, on the full graph, `sweeps` sweeps per call."""
    import oracle as O
    m = len(rp) - 1
    kind = "reference" if O.ref_available() else "port"
    total_t, total_sweeps, calls = 0.0, 0, 0
    while calls < min_calls or total_t < budget_s:
        s0 = np.full(m, np.float32(1.0) / np.float32(m), dtype=np.float32)
        t0 = time.perf_counter()
        if kind == "reference":
            _, printed, _ = O.ref_pr_solver(rp, col, od, scores=s0, tol=0.0, max_iter=sweeps)
            done = sweeps  # tol 0 never converges: exactly `sweeps` sweeps
        else:
            _, done, _ = O.pr_plain_f32(rp, col, od, scores=s0, tol=0.0, max_iter=sweeps)
        total_t += time.perf_counter() - t0
        total_sweeps += done
        calls += 1
        if calls >= 50:
            break
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    return {"gteps": len(col) * total_sweeps / total_t / 1e9, "kind": kind, "cores": cores,
            "calls": calls, "sweeps": total_sweeps, "seconds": total_t}


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    import oracle as O
    t0 = time.time()
    rp, col, od = O.rmat_graph(args.scale, EDGE_FACTOR, seed=SEED, abc=ABC)
    log(f"[reference] graph s{args.scale}: m={len(rp) - 1} nnz={len(col)} built in {time.time() - t0:.1f}s")
    kind = "reference" if O.ref_available() else "port"
    m = len(rp) - 1
    times = []
    for i in range(args.warmup + args.steps):
        s0 = np.full(m, np.float32(1.0) / np.float32(m), dtype=np.float32)
        t1 = time.perf_counter()
        if kind == "reference":
            O.ref_pr_solver(rp, col, od, scores=s0, tol=0.0, max_iter=SAMPLE_SWEEPS)
        else:
            O.pr_plain_f32(rp, col, od, scores=s0, tol=0.0, max_iter=SAMPLE_SWEEPS)
        dt = time.perf_counter() - t1
        if i >= args.warmup:
            times.append(dt)
    total = sum(times)
    gteps = len(col) * SAMPLE_SWEEPS * len(times) / total / 1e9
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    sample = (f"{SAMPLE_SWEEPS} sweeps of the full RMAT-{args.scale} graph per step "
              f"(OpenMP, {cores} threads); GTEPS per sweep is what a full solve sustains")
    line = {
        "impl": "reference", "metric": "pagerank_gteps_rmat24", "value": gteps, "unit": "GTEPS",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded RMAT)",
        "config": dict(workload_config(args.scale, m, len(col)),
                       workload=f"pagerank_rmat{args.scale}_ef{EDGE_FACTOR}_rate_sample",
                       sample=f"{SAMPLE_SWEEPS}-sweep rate sample (tol 0) per step of the "
                              f"full graph, not a tol {TOL:g} solve; the rate per sweep is "
                              "what a full solve sustains",
                       precision="plain fp32 (fp64 residual), reference OpenMP PRSolver"),
        "cpu_baseline": {"value": gteps, "unit": "GTEPS", "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": gteps, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(scale, m, nnz):
    return {"workload": f"pagerank_rmat{scale}_ef{EDGE_FACTOR}_tol1e-6",
            "graph": f"RMAT scale {scale}, edge factor {EDGE_FACTOR}, abc={ABC}, seed {SEED}, "
                     "scrambled ids, self-loops/duplicates removed",
            "m": m, "nnz": nnz, "tol": TOL, "max_iter": MAX_ITER, "damping": float(DAMPING),
            "precision": "plain fp32 (fp64 residual)",
            "l2": "inputs larger than L2 (CSR > 1 GB vs 126 MB L2): no flush between steps",
            "parallelism": "replicas (one independent solve per GPU)"}


def run_ours(args):
    import torch

    import gardenia_ocl_b200 as G
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    G.set_device(local)
    dist = init_dist(world, local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    t0 = time.time()
    csr = G.gen_rmat(args.scale, EDGE_FACTOR, seed=SEED, abc=ABC)
    m, nnz = csr.m, csr.nnz
    # The project autotuner picks the bins, hot prefix and kernel variant for
    # this degree distribution (timed on the graph, outside the timed region).
    # It also decides between the exact-order layout and the blocked one.
    tuned = None
    layout = {"blocked": True}  # untuned: the blocked form
    variant = 0
    if not args.no_tune:
        tuned = G.tune_graph(csr.rowptr, csr.col, csr.third, m=m, nnz=nnz, cache=args.tune_cache,
                             sweeps=5)
        layout = {k: tuned[k] for k in ("sell_max", "chunk", "chunk_min", "hot_entries",
                                        "blocked", "block_rows", "tile_words",
                                        "blocked_long")}
        variant = tuned["variant"]
        log(f"[ours] tuned: {tuned}")
    blocked = bool(layout.get("blocked"))
    kernel = "k_pr_blocked" if blocked else "k_pr_hot"
    g = G.Graph(csr.rowptr, csr.col, csr.third, m=m, nnz=nnz, batched=not args.no_forms,
                **layout)
    g.set_stream(stream.cuda_stream)
    log(f"[ours] rank {rank}: graph s{args.scale} m={m} nnz={nnz} layout={g.layout()} "
        f"ready in {time.time() - t0:.2f}s")
    scores = torch.empty(m, dtype=torch.float32, device=dev)
    init = float(np.float32(1.0) / np.float32(m))
    opts = G.options(tol=TOL, max_iter=MAX_ITER, damping=DAMPING, variant=variant)

    def step():
        scores.fill_(init)
        _, st = g.pagerank(scores, opts)
        return st

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    props = torch.cuda.get_device_properties(dev)
    uuid = getattr(props, "uuid", None)
    uuid = f"GPU-{uuid}" if uuid is not None and not str(uuid).startswith("GPU-") else uuid
    sampler = ClockSampler(str(uuid) if uuid else None)
    sampler.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    ev0.record(stream)
    for _ in range(args.steps):
        stats.append(step())
    ev1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist, dev)
    sweeps = sum(s.iterations for s in stats)
    launches = sum(s.gpu_launches for s in stats)
    gteps = replica_rate(world, nnz * sweeps, ms / 1e3) / 1e9
    loop_ms = sum(s.loop_ms for s in stats) / len(stats)
    sweeps_per_solve = sweeps / len(stats)
    per_sweep = pr_bytes_per_sweep(m, nnz)
    alg_bytes = per_sweep * sweeps_per_solve
    peak, peak_kind = load_peaks()
    achieved = alg_bytes / (loop_ms / 1e3) / 1e9
    traffic = load_traffic().get(f"{kernel}_rmat{args.scale}")
    roof = {"kernel": f"{kernel} (persistent: all sweeps of one solve)", "bound": "hbm",
            "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": (traffic["bytes_per_sweep"] * sweeps_per_solve) if traffic else None,
            "algorithmic_bytes_per_launch": alg_bytes,
            "bytes_per_sweep_formula": "4*nnz + 28*m + 4",
            "launch_ms": loop_ms}
    if traffic and traffic.get("l2_requests_per_sweep"):
        # The second ceiling of a gather: L1->L2 requests (one per scattered
        # sector) at the measured random-gather rate of profiles/gather_rates.md.
        req = traffic["l2_requests_per_sweep"]
        rate = req * sweeps_per_solve / (loop_ms / 1e3)
        roof["l2_requests"] = {"requests_per_sweep": req, "achieved": rate,
                               "peak": L2_GATHER_RATE, "unit": "requests/s",
                               "frac": rate / L2_GATHER_RATE,
                               "source": traffic.get("source", "")}
    resid = g.residual_f64(scores, DAMPING)
    accuracy = {"fp64_residual_l1": resid,
                "l1_error_bound_vs_fixed_point": resid / (1.0 - float(DAMPING)),
                "sweeps_per_solve": sweeps_per_solve}
    x_star, fp_it, fp_delta = fp64_fixed_point(torch, csr, m, scores)
    accuracy.update(errors_vs(x_star, scores))
    accuracy["fp64_fixed_point"] = {"how": "PyTorch FP64 sparse mat-vec on the GPU from the "
                                           "solver's result", "iterations": fp_it,
                                    "last_l1_change": fp_delta}

    # The same solve in the exact-order form (rows of <= 64 in-edges summed in
    # the reference's order) on the same graph, for comparison.
    exact = None
    for _ in range(3):
        scores.fill_(init)
        _, st = g.pagerank(scores, G.options(tol=TOL, max_iter=MAX_ITER, damping=DAMPING,
                                             variant=variant if not blocked else 0,
                                             form=G.FORM_EXACT))
        if exact is None or st.loop_ms < exact.loop_ms:
            exact = st
    exact_order = {"kernel": "k_pr_hot", "sweeps": exact.iterations, "loop_ms": exact.loop_ms,
                   "gteps": nnz * exact.iterations / (exact.loop_ms / 1e3) / 1e9,
                   "hbm_frac": per_sweep * exact.iterations / (exact.loop_ms / 1e3) / 1e9 / peak}

    line = {"metric": "pagerank_gteps_rmat24", "value": gteps, "unit": "GTEPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded RMAT generated on the GPU)",
            "config": workload_config(args.scale, m, nnz), "roofline": roof,
            "gpu_launches": launches, "clocks": clocks, "accuracy": accuracy,
            "tuning": tuned, "form": "blocked" if blocked else "exact", "exact_order": exact_order}

    # End to end through the reference-shaped C-ABI call with host buffers:
    # PageRank(m, nnz, row_offsets, column_indices, degree, scores) copies the
    # CSR in, builds the layout, solves and copies the scores back.
    if not args.no_e2e:
        h_rp = torch.empty(m + 1, dtype=torch.int32, pin_memory=True)
        h_col = torch.empty(nnz, dtype=torch.int32, pin_memory=True)
        h_od = torch.empty(m, dtype=torch.int32, pin_memory=True)
        h_sc = torch.empty(m, dtype=torch.float32, pin_memory=True)
        for h, d in ((h_rp, csr.rowptr), (h_col, csr.col), (h_od, csr.third)):
            G.lib().gpr_memcpy(G.C.c_void_p(h.data_ptr()), G.C.c_void_p(d.ptr), d.nbytes)
        na = [x.numpy() for x in (h_rp, h_col, h_od, h_sc)]
        e2e_steps = max(1, min(args.steps, 5))
        e_sweeps, e_time = 0, 0.0
        for i in range(1 + e2e_steps):
            na[3].fill(np.float32(1.0) / np.float32(m))
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            t1 = time.perf_counter()
            st = G.PageRank(m, nnz, na[0], na[1], na[2], na[3], tol=TOL, max_iter=MAX_ITER,
                            damping=DAMPING)
            dt = time.perf_counter() - t1
            if i > 0:
                e_sweeps += st.iterations
                e_time += dt
        e_time = max_over_ranks(e_time, dist, dev)
        line["e2e"] = {"value": replica_rate(world, nnz * e_sweeps, e_time) / 1e9, "unit": "GTEPS",
                       "h2d_bytes_per_step": 4 * (m + 1) + 4 * nnz + 4 * m + 4 * m,
                       "d2h_bytes_per_step": 4 * m, "ms_per_step": 1e3 * e_time / e2e_steps,
                       "call": "PageRank(m, nnz, row_offsets, column_indices, degree, scores) "
                               "via gpr_page_rank, pinned host buffers"}

    if not args.no_forms:
        line["forms"] = forms_leg(G, torch, dev, g, m, nnz, gteps / world, args, x_star,
                                  (csr.rowptr.to_numpy(), csr.third.to_numpy()))
        line["forms"]["bf16_study"]["pr_bf16_refined"]["time_to_solution_vs_plain"] = (
            (ms / args.steps) / line["forms"]["bf16_study"]["pr_bf16_refined"]["loop_ms"])
    if not args.no_multigraph:
        line["multigraph"] = multigraph_leg(G, torch, dev, stream, gteps / world, args)
    if not args.no_forms:
        line["ppr"] = ppr_leg(G, torch, dev, stream, args)

    if not args.no_s16:
        line["s16"] = s16_leg(G, torch, dev, stream, args)
    if rank == 0 and not args.no_ref_cuda:
        line["reference_cuda"] = reference_cuda_leg(G, torch, dev, csr, args)
        line["reference_cuda"]["gpr_pr_gteps"] = gteps / world
        if "pr_gather_warp" in line["reference_cuda"]:
            line["reference_cuda"]["gpr_vs_gather_warp"] = (
                gteps / world / line["reference_cuda"]["pr_gather_warp"]["gteps"])
            line["reference_cuda"]["gpr_vs_gather"] = (
                gteps / world / line["reference_cuda"]["pr_gather"]["gteps"])
    if not args.no_spmv:
        line["spmv"] = spmv_leg(G, torch, dev, stream, args)
        if "spmv_base" in line.get("reference_cuda", {}):
            line["reference_cuda"]["gpr_spmv_vs_base"] = (
                line["reference_cuda"]["spmv_base"]["ms"] / line["spmv"]["ms"])
    if not args.no_spmv:
        line["symgs"] = symgs_leg(G, torch, dev, args)
    if args.io and rank == 0:
        line["io"] = io_leg(G, args)

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle as O  # checker / baseline only
        rp = csr.rowptr.to_numpy()
        col = csr.col.to_numpy()
        od = csr.third.to_numpy()
        cb = cpu_reference_sample(rp, col, od, SAMPLE_SWEEPS, CPU_BASELINE_BUDGET_S)
        line["cpu_baseline"] = {"value": cb["gteps"], "unit": "GTEPS", "cores": cb["cores"],
                                "kind": cb["kind"],
                                "sample": f"{cb['calls']} calls x {SAMPLE_SWEEPS} sweeps of the "
                                          f"full RMAT-{args.scale} graph ({cb['seconds']:.1f} s)"}
        del O
    g.close()
    csr.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def pull_matrix(torch, csr, m, dev):
    """The in-CSR as a PyTorch FP64 sparse matrix, A[v, u] = 1 / outdeg[u]."""
    import warnings
    warnings.filterwarnings("ignore", message="Sparse")  # beta-status notices of torch.sparse
    rp = torch.from_numpy(csr.rowptr.to_numpy().astype(np.int64)).to(dev)
    col = torch.from_numpy(csr.col.to_numpy().astype(np.int64)).to(dev)
    od = torch.from_numpy(csr.third.to_numpy()).to(dev).double()
    return torch.sparse_csr_tensor(rp, col, (1.0 / od.clamp(min=1.0))[col], size=(m, m))


def fp64_fixed_point(torch, csr, m, x0, base=None, A=None):
    """FP64 fixed point of the plain recurrence x = base + d A x (A[v, u] =
    1 / outdeg[u] over the in-CSR, d = (double)0.85f, base (1 - d) / m, or
    per vertex (1 - d) / m_g for a batch of graphs, as the reference's FP64
    restatement), computed with PyTorch's FP64 sparse matrix-vector product
    on the GPU from x0 until the L1 change is below 1e-13.  A checker for the
    accuracy report: the solvers are not involved.  Returns (x, iterations,
    last L1 change)."""
    if A is None:
        A = pull_matrix(torch, csr, m, x0.device)
    d = float(np.float32(DAMPING))
    if base is None:
        base = (1.0 - d) / m
    x = x0.double()
    delta, k = float("inf"), 0
    while k < 400 and delta >= 1e-13:
        xn = base + d * torch.mv(A, x)
        delta = float((xn - x).abs().sum())
        x, k = xn, k + 1
    del A
    return x, k, delta


def ppr_fp64_fixed_point(torch, csr, m, seeds, x0):
    """FP64 fixed point of the batched personalized PageRank recurrence (the
    solver's): for vector q with seed s_q,
      x_q = d A x_q + [v == s_q] ((1 - d) + d * sum of x_q over out-degree-0 v),
    A[v, u] = 1 / outdeg[u] over the in-CSR, d = (double)0.85f, computed with
    PyTorch's FP64 sparse x dense product on the GPU from x0 (m x k) until
    every vector's L1 change is below 1e-13.  A checker only."""
    dev = x0.device
    A = pull_matrix(torch, csr, m, dev)
    dang = torch.from_numpy((csr.third.to_numpy() == 0).astype(np.float64)).to(dev)
    k = x0.shape[1]
    rows = torch.from_numpy(np.asarray(seeds, np.int64)).to(dev)
    cols = torch.arange(k, device=dev)
    d = float(np.float32(DAMPING))
    x = x0.double()
    delta, it = float("inf"), 0
    while it < 400 and delta >= 1e-13:
        xn = d * (A @ x)
        xn[rows, cols] += (1.0 - d) + d * (dang @ x)
        delta = float((xn - x).abs().sum(0).max())
        x, it = xn, it + 1
    del A
    return x


def errors_vs(x_star, s):
    """Max and L1 error of a float32 score vector against the FP64 fixed point."""
    e = (s.double() - x_star).abs()
    return {"l1_error_vs_fp64_fixed_point": float(e.sum()),
            "max_error_vs_fp64_fixed_point": float(e.max())}


def forms_leg(G, torch, dev, g, m, nnz, plain_gteps, args, x_star=None, g_host_degrees=None):
    """The forms the metric compares with the plain FP32 path, on the same
    graph: batched personalized PageRank (k seed vectors, one persistent
    launch) in FP32 and in BF16 with FP32 refinement.  Rates are edge-vector
    pairs per second over every vector of every sweep (nnz * k * sweeps /
    time of the sweep loop); `useful` counts only sweeps in which a vector was
    still updating."""
    out = {"plain_fp32_gteps": plain_gteps}
    # single-vector mixed form: BF16 contributions, then FP32 refinement
    scores = torch.empty(m, dtype=torch.float32, device=dev)
    best = None
    for _ in range(3):
        scores.fill_(float(np.float32(1.0) / np.float32(m)))
        _, st = g.pagerank(scores, G.options(tol=TOL, max_iter=MAX_ITER, damping=DAMPING,
                                             precision=G.PREC_BF16))
        if best is None or st.loop_ms < best.loop_ms:
            best = st
    resid = g.residual_f64(scores, DAMPING)
    study = {"note": BF16_NOTE}
    study["pr_bf16_refined"] = {
        "sweeps": best.iterations, "refine_sweeps": best.refine_iterations,
        "loop_ms": best.loop_ms, "gteps": nnz * best.iterations / (best.loop_ms / 1e3) / 1e9,
        "time_to_solution_vs_plain": None, "l1_error_bound_vs_fixed_point": resid / (1 - 0.85)}
    if x_star is not None:
        study["pr_bf16_refined"].update(errors_vs(x_star, scores))
    out["bf16_study"] = study
    # push direction (atomic scatter) on the same graph, FP32
    best = None
    for _ in range(3):
        scores.fill_(float(np.float32(1.0) / np.float32(m)))
        _, st = g.pagerank_push(scores, G.options(tol=TOL, max_iter=MAX_ITER, damping=DAMPING))
        if best is None or st.loop_ms < best.loop_ms:
            best = st
    out["pr_push_fp32"] = {"sweeps": best.iterations, "loop_ms": best.loop_ms,
                           "gteps": nnz * best.iterations / (best.loop_ms / 1e3) / 1e9,
                           "vs_plain_fp32": nnz * best.iterations / (best.loop_ms / 1e3) / 1e9
                           / plain_gteps}
    if x_star is not None:
        out["pr_push_fp32"].update(errors_vs(x_star, scores))
    rng = np.random.default_rng(5)
    rp_h, od_h = g_host_degrees
    pool = np.flatnonzero((np.diff(rp_h) > 0) & (od_h > 0)).astype(np.int32)
    for k, prec, name in ((8, G.PREC_FP32, "ppr_k8_fp32"), (32, G.PREC_FP32, "ppr_k32_fp32"),
                          (32, G.PREC_BF16, "ppr_k32_bf16_refined")):
        dest = study if prec == G.PREC_BF16 else out
        seeds = rng.choice(pool, k).astype(np.int32)
        buf = torch.empty(m * k, dtype=torch.float32, device=dev)
        best = None
        for _ in range(2):
            _, it, st = g.ppr(seeds, out=buf, tol=TOL, max_iter=MAX_ITER, precision=prec)
            if best is None or st.loop_ms < best[0].loop_ms:
                best = (st, it)
        st, it = best
        rate = nnz * k * st.iterations / (st.loop_ms / 1e3) / 1e9
        dest[name] = {"k": k,
                     "precision": "bf16+fp32 refinement" if prec == G.PREC_BF16 else "fp32",
                     "sweeps": st.iterations, "refine_sweeps": st.refine_iterations,
                     "loop_ms": st.loop_ms, "edge_vector_gteps": rate,
                     "useful_edge_vector_gteps": nnz * float(it.sum()) / (st.loop_ms / 1e3) / 1e9,
                     "vs_plain_fp32": rate / plain_gteps, "max_final_residual": st.residual}
        del buf
    return out


PPR_SCALE, PPR_KS = 22, (8, 32, 128)


def ppr_leg(G, torch, dev, stream, args):
    """Batched personalized PageRank on its own configuration: RMAT scale 22,
    edge factor 16 (same RMAT parameters), k = 8, 32 and 128 seed vectors,
    each seed drawn uniformly (seeded), teleport mass on the seed, tol 1e-6
    per vector, one persistent launch, FP32 and BF16 + FP32 refinement, and
    the FP32 solve again as a CUDA-graph loop of one launch per sweep.
    Rate: nnz x k x sweeps per second of the sweep loop (edge-vector pairs);
    the plain FP32 single-vector GTEPS on the same graph is the comparison."""
    csr = G.gen_rmat(PPR_SCALE, EDGE_FACTOR, seed=SEED, abc=ABC)
    m, nnz = csr.m, csr.nnz
    g = G.Graph(csr.rowptr, csr.col, csr.third, m=m, nnz=nnz, batched=True, blocked=True)
    g.set_stream(stream.cuda_stream)
    scores = torch.empty(m, dtype=torch.float32, device=dev)
    plains = {}
    for form, name in ((G.FORM_EXACT, "exact"), (G.FORM_BLOCKED, "blocked")):
        best = None
        for _ in range(4):
            scores.fill_(float(np.float32(1.0) / np.float32(m)))
            _, st = g.pagerank(scores, G.options(tol=TOL, max_iter=MAX_ITER, damping=DAMPING,
                                                 form=form))
            if best is None or st.loop_ms < best.loop_ms:
                best = st
        plains[name] = {"sweeps": best.iterations, "loop_ms": best.loop_ms,
                        "gteps": nnz * best.iterations / (best.loop_ms / 1e3) / 1e9}
    # the comparison: the faster single-vector FP32 form on the same graph
    plain = max(p["gteps"] for p in plains.values())
    out = {"workload": f"ppr_rmat{PPR_SCALE}_ef{EDGE_FACTOR}_tol1e-6", "m": m, "nnz": nnz,
           "seed_rule": "seeds drawn uniformly (seeded) from the vertices with in- and "
                        "out-edges (a seed without out-edges keeps its mass and stops after "
                        "one sweep)",
           "plain_fp32": dict(gteps=plain, forms=plains),
           "useful_rate": "nnz x (sum over vectors of the sweeps in which the vector still "
                          "updated) per second of the sweep loop",
           "edge_vector_rate": "nominal: nnz x k x the batch's sweeps per second; once half "
                               "of the vectors stop, the rest continue packed into a narrower "
                               "layout (gpr_pr_opts.ppr_repack), so later sweeps do less than "
                               "k vectors' work"}
    rp_h, od_h = csr.rowptr.to_numpy(), csr.third.to_numpy()
    pool = np.flatnonzero((np.diff(rp_h) > 0) & (od_h > 0)).astype(np.int32)
    rng = np.random.default_rng(22)
    for k in PPR_KS:
        seeds = rng.choice(pool, k).astype(np.int32)
        buf = torch.empty(m * k, dtype=torch.float32, device=dev)
        for prec, tag in ((G.PREC_FP32, "fp32"), (G.PREC_BF16, "bf16_refined")):
            dest = out if prec == G.PREC_FP32 else out.setdefault("bf16_study", {"note": BF16_NOTE})
            bst = None
            for _ in range(2):
                _, it, st = g.ppr(seeds, out=buf, tol=TOL, max_iter=MAX_ITER, precision=prec)
                if bst is None or st.loop_ms < bst[0].loop_ms:
                    bst = (st, it)
            st, it = bst
            rate = nnz * k * st.iterations / (st.loop_ms / 1e3) / 1e9
            useful = nnz * float(it.sum()) / (st.loop_ms / 1e3) / 1e9
            dest[f"k{k}_{tag}"] = {"sweeps": st.iterations, "refine_sweeps": st.refine_iterations,
                                  "vector_sweeps_min": int(it.min()),
                                  "vector_sweeps_mean": float(it.mean()), "loop_ms": st.loop_ms,
                                  "edge_vector_gteps": rate, "vs_plain_fp32": rate / plain,
                                  "useful_edge_vector_gteps": useful,
                                  "useful_vs_plain_fp32": useful / plain,
                                  "max_final_residual": st.residual}
            # errors of the last solve's vectors against the FP64 fixed point
            xk = buf.view(m, k)
            x_star = ppr_fp64_fixed_point(torch, csr, m, seeds, xk)
            e = (xk.double() - x_star).abs()
            dest[f"k{k}_{tag}"]["max_l1_error_vs_fp64_fixed_point"] = float(e.sum(0).max())
            dest[f"k{k}_{tag}"]["max_error_vs_fp64_fixed_point"] = float(e.max())
            del x_star, e
        # the same FP32 solve as a CUDA-graph loop (one launch per sweep)
        bst = None
        for _ in range(2):
            _, it, st = g.ppr(seeds, out=buf, tol=TOL, max_iter=MAX_ITER, loop=G.LOOP_GRAPH)
            if bst is None or st.loop_ms < bst.loop_ms:
                bst = st
        rate = nnz * k * bst.iterations / (bst.loop_ms / 1e3) / 1e9
        out[f"k{k}_fp32_graph_loop"] = {"sweeps": bst.iterations, "loop_ms": bst.loop_ms,
                                        "gpu_launches": bst.gpu_launches,
                                        "edge_vector_gteps": rate, "vs_plain_fp32": rate / plain}
        del buf
    g.close()
    csr.close()
    return out


S16_SCALE, S16_TOL, S16_MAX_ITER = 16, 1e-4, 100


def s16_leg(G, torch, dev, stream, args):
    """The small workload: plain PageRank on RMAT scale 16 (edge factor 16, same
    RMAT parameters), tol 1e-4, at most 100 sweeps, from 1/m.  On the GPU
    through the graph handle (device-resident graph: exact-order and blocked
    forms, device time of the solve) and end to end through PageRank() with
    host buffers; beside it the reference's own OpenMP PRSolver
    (src/pr/omp_base.cc, compiled into oracle/_ref) solving the same graph on
    the host cores (its full solve, wall time)."""
    import oracle as O  # checker / baseline only
    csr = G.gen_rmat(S16_SCALE, EDGE_FACTOR, seed=SEED, abc=ABC)
    m, nnz = csr.m, csr.nnz
    rp, col, od = csr.rowptr.to_numpy(), csr.col.to_numpy(), csr.third.to_numpy()
    out = {"workload": f"pagerank_rmat{S16_SCALE}_ef{EDGE_FACTOR}_tol1e-4", "m": m, "nnz": nnz}
    g = G.Graph(csr.rowptr, csr.col, csr.third, m=m, nnz=nnz, blocked=True)
    g.set_stream(stream.cuda_stream)
    scores = torch.empty(m, dtype=torch.float32, device=dev)
    for form, name in ((G.FORM_EXACT, "gpu_exact"), (G.FORM_BLOCKED, "gpu_blocked")):
        best = None
        for _ in range(5):
            scores.fill_(float(np.float32(1.0) / np.float32(m)))
            _, st = g.pagerank(scores, G.options(tol=S16_TOL, max_iter=S16_MAX_ITER,
                                                 damping=DAMPING, form=form))
            if best is None or st.solve_ms < best.solve_ms:
                best = st
        out[name] = {"sweeps": best.iterations, "solve_ms": best.solve_ms,
                     "loop_ms": best.loop_ms,
                     "gteps": nnz * best.iterations / (best.solve_ms / 1e3) / 1e9}
        if form == G.FORM_EXACT:
            s_gpu = scores.cpu().numpy()
    g.close()
    # end to end: PageRank() on host arrays (copies, layout build, solve, copy back)
    times, sweeps = [], 0
    for i in range(4):
        s_h = np.full(m, np.float32(1.0) / np.float32(m), dtype=np.float32)
        t0 = time.perf_counter()
        st = G.PageRank(m, nnz, rp, col, od, s_h, tol=S16_TOL, max_iter=S16_MAX_ITER,
                        damping=DAMPING)
        if i > 0:
            times.append(time.perf_counter() - t0)
            sweeps = st.iterations
    e2e = min(times)
    out["gpu_e2e"] = {"sweeps": sweeps, "ms": 1e3 * e2e, "gteps": nnz * sweeps / e2e / 1e9,
                      "call": "PageRank(m, nnz, row_offsets, column_indices, degree, scores)"}
    kind = "reference" if O.ref_available() else "port"
    times = []
    for i in range(4):
        t0 = time.perf_counter()
        if kind == "reference":
            ref, printed, _ = O.ref_pr_solver(rp, col, od, tol=S16_TOL, max_iter=S16_MAX_ITER)
            ref_sweeps = printed
        else:
            ref, ref_sweeps, _ = O.pr_plain_f32(rp, col, od, tol=S16_TOL, max_iter=S16_MAX_ITER)
        if i > 0:
            times.append(time.perf_counter() - t0)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    t = min(times)
    out["cpu_reference"] = {"kind": kind, "cores": cores, "sweeps": ref_sweeps, "ms": 1e3 * t,
                            "gteps": nnz * ref_sweeps / t / 1e9,
                            "note": "wall time of the full solve (its per-sweep printf included)"}
    out["max_abs_diff_gpu_vs_reference"] = float(np.abs(s_gpu - ref).max())
    out["gpu_device_vs_cpu_reference"] = out["gpu_exact"]["gteps"] / out["cpu_reference"]["gteps"]
    out["gpu_e2e_vs_cpu_reference"] = out["gpu_e2e"]["gteps"] / out["cpu_reference"]["gteps"]
    csr.close()
    return out


REF_CUDA_SWEEPS = 10


def reference_cuda_leg(G, torch, dev, csr24, args):
    """The reference's own CUDA solvers (src/pr/gather.cu thread per row,
    gather_warp.cu warp per row, src/spmv/base.cu thread per row), compiled
    unmodified for sm_100a into oracle/_ref, on this benchmark's graph and on
    the 27-point 128^3 stencil; times from their own Timer (the sweep loop,
    including its per-sweep device-to-host residual copy).  gpr's numbers on
    the same inputs beside them."""
    import oracle as O  # baseline only
    out = {}
    if not O.ref_gpu_available("gather"):
        return {"unavailable": "oracle/_ref CUDA solvers not built (needs the reference tree)"}
    rp, col, od = csr24.rowptr.to_numpy(), csr24.col.to_numpy(), csr24.third.to_numpy()
    nnz = len(col)
    for name in ("gather", "gather_warp"):
        _, it, ms, _ = O.ref_gpu_pr_solver(name, rp, col, od, tol=0.0, max_iter=REF_CUDA_SWEEPS)
        out[f"pr_{name}"] = {"sweeps": it, "ms": ms, "gteps": nnz * it / (ms / 1e3) / 1e9,
                             "workload": f"RMAT s{args.scale}, {REF_CUDA_SWEEPS} sweeps (tol 0)"}
    Ap, Aj, Ax = O.stencil27(128)
    m = len(Ap) - 1
    x, y0 = O.uniform_f32(m, 3), np.zeros(m, np.float32)
    O.ref_gpu_spmv_solver(Ap, Aj, Ax, x, y0)  # warm
    _, ms = O.ref_gpu_spmv_solver(Ap, Aj, Ax, x, y0)
    out["spmv_base"] = {"ms": ms, "gb_s": spmv_bytes(m, len(Aj)) / (ms / 1e3) / 1e9,
                        "workload": "27-point 128^3 stencil, one SpMV"}
    return out


MG_GRAPHS, MG_MMIN, MG_MMAX, MG_SEED, MG_MAX_ITER = 512, 1000, 500000, 1, 200


def multigraph_leg(G, torch, dev, stream, plain_gteps, args):
    """Uneven multi-graph batch: 512 seeded graphs, m_g log-uniform in
    [1e3, 5e5], half Erdos-Renyi (8 draws per vertex), half Chung-Lu power
    law (exponent 2.1, 16 draws per vertex), each solved to tol 1e-6 as plain
    PageRank of its own, all in one persistent launch, in FP32 (the blocked
    form: every graph's rows in blocks of source-ordered edges, fixed-point
    sums; the units form beside it) and in the BF16 + FP32 refinement form.
    Rate: sum over graphs of nnz_g x sweeps_g per second of the sweep loop;
    bytes: sum of (4 nnz_g + 28 m_g + 4) x sweeps_g."""
    t0 = time.time()
    A, voff = G.gen_multigraph(MG_GRAPHS, MG_MMIN, MG_MMAX, seed=MG_SEED)
    layouts, tuned = None, None
    if not args.no_tune:
        layouts, tuned = G.tune_multigraph(A.rowptr, A.col, A.third, voff, nnz=A.nnz,
                                           cache=args.tune_cache, sweeps=5)
        log(f"[ours] multigraph tuned: {tuned}")
    mg = G.MultiGraph(A.rowptr, A.col, A.third, voff, nnz=A.nnz, layouts=layouts, blocked=True)
    mg.set_stream(stream.cuda_stream)
    info = mg.info()
    rp = A.rowptr.to_numpy()
    nnz_g = (rp[voff[1:]] - rp[voff[:-1]]).astype(np.int64)
    m_g = np.diff(voff).astype(np.int64)
    log(f"[ours] multigraph: {info} ready in {time.time() - t0:.2f}s")
    scores = torch.empty(A.m, dtype=torch.float32, device=dev)
    init = torch.from_numpy(mg.initial_scores()).to(dev)
    peak, peak_kind = load_peaks()
    out = {"workload": f"multigraph_{MG_GRAPHS}_m{MG_MMIN}-{MG_MMAX}_tol1e-6",
           "graphs": MG_GRAPHS, "m": A.m, "nnz": A.nnz, "units": info["units"],
           "edge_slots": info["edge_slots"], "tol": TOL, "max_iter": MG_MAX_ITER,
           "tuning": tuned,
           "bins": sorted({(d["sell_max"], d["chunk_min"], d["chunk"]) for d in layouts})
           if layouts else "defaults"}
    x_star = None
    for prec, name, form in ((G.PREC_FP32, "fp32", G.FORM_AUTO),
                             (G.PREC_FP32, "fp32_units_form", G.FORM_EXACT),
                             (G.PREC_BF16, "bf16_refined", G.FORM_AUTO)):
        dest = out if prec == G.PREC_FP32 else out.setdefault("bf16_study", {"note": BF16_NOTE})
        best = None
        for _ in range(3):
            scores.copy_(init)
            _, it, res, st = mg.pagerank(scores, tol=TOL, max_iter=MG_MAX_ITER, damping=DAMPING,
                                         precision=prec, form=form)
            if best is None or st.loop_ms < best[0].loop_ms:
                best = (st, it.copy(), res.copy())
        st, it, res = best
        edges = float((nnz_g * it).sum())
        byts = float(((4 * nnz_g + 28 * m_g + 4) * it).sum())
        dest[name] = {"launch_sweeps": st.iterations, "refine_sweeps": st.refine_iterations,
                     "graph_sweeps_min": int(it.min()), "graph_sweeps_max": int(it.max()),
                     "converged": int((res < TOL).sum()), "loop_ms": st.loop_ms,
                     "solve_ms": st.solve_ms, "gteps": edges / (st.loop_ms / 1e3) / 1e9,
                     "vs_plain_single_graph": edges / (st.loop_ms / 1e3) / 1e9 / plain_gteps,
                     "achieved_gbs": byts / (st.loop_ms / 1e3) / 1e9,
                     "frac": byts / (st.loop_ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind,
                     "gpu_launches": st.gpu_launches,
                     "form": "blocked" if name == "fp32" else "units"}
        # every graph's errors against the batch's FP64 fixed point (each
        # graph with its own teleport (1 - d) / m_g); all graphs have m_g > 0
        if x_star is None:
            base = np.repeat((1.0 - float(np.float32(DAMPING))) / m_g, m_g)
            x_star, _, _ = fp64_fixed_point(torch, A, A.m, scores,
                                            base=torch.from_numpy(base).to(dev))
        e = (scores.double() - x_star).abs().cpu().numpy()
        dest[name]["max_l1_error_vs_fp64_fixed_point"] = float(np.add.reduceat(e, voff[:-1]).max())
        dest[name]["max_error_vs_fp64_fixed_point"] = float(e.max())
    del x_star
    # the FP32 solve again as a CUDA-graph loop (one launch per sweep)
    best = None
    for _ in range(2):
        scores.copy_(init)
        _, it, res, st = mg.pagerank(scores, tol=TOL, max_iter=MG_MAX_ITER, damping=DAMPING,
                                     loop=G.LOOP_GRAPH)
        if best is None or st.loop_ms < best[0].loop_ms:
            best = (st, it.copy())
    st, it = best
    edges = float((nnz_g * it).sum())
    out["fp32_graph_loop"] = {"launch_sweeps": st.iterations, "loop_ms": st.loop_ms,
                              "gteps": edges / (st.loop_ms / 1e3) / 1e9,
                              "gpu_launches": st.gpu_launches}
    mg.close()
    A.close()
    return out


def symgs_stencil(G, torch, dev, n=128):
    """The 27-point n^3 stencil, its 8-colour parity colouring and a SymGS
    handle, with x and b seeded uniform on the device."""
    A = G.gen_stencil27(n)
    m = A.m
    v = np.arange(m, dtype=np.int64)
    color = (v % n % 2) + 2 * ((v // n) % n % 2) + 4 * ((v // (n * n)) % 2)
    indices = np.argsort(color, kind="stable").astype(np.int32)
    offsets = np.zeros(9, dtype=np.int32)
    np.cumsum(np.bincount(color, minlength=8), out=offsets[1:])
    S = G.SymGS(A.rowptr, A.col, A.third, indices, offsets, m=m, nnz=A.nnz)
    x = torch.empty(m, dtype=torch.float32, device=dev)
    b = torch.empty(m, dtype=torch.float32, device=dev)
    G.gen_uniform(m, 31, x)
    G.gen_uniform(m, 32, b)
    return A, S, x, b, color


def symgs_leg(G, torch, dev, args):
    """Multicolour symmetric Gauss-Seidel (src/symgs) on the 27-point 128^3
    stencil with the 8-colour parity colouring (colour = x%2 + 2(y%2) +
    4(z%2): every neighbour differs by one in some coordinate), x and b
    seeded uniform.  One sweep = 8 colour passes forward + 8 backward; a pass
    that repeats the colour of the pass before it writes the same values and
    is skipped (14 passes per sweep after the first).  Bytes: per executed
    pass over colour c, 8 per off-diagonal entry of its rows + 24 per row
    (diagonal, row id, length, b, x read and write)."""
    A, S, x, b, color = symgs_stencil(G, torch, dev)
    m = A.m
    for _ in range(3):
        S.apply(x, b, sweeps=1)
    sweeps = 10
    ms = min(S.apply(x, b, sweeps=sweeps) for _ in range(3)) / sweeps
    # bytes of one pass over colour c: 8 per off-diagonal entry of its rows
    # plus 24 per row; a pass repeating the previous pass's colour is skipped
    deg = np.diff(A.rowptr.to_numpy()).astype(np.int64) - 1  # one diagonal per row
    nc = int(color.max()) + 1
    pass_bytes = [8 * int(deg[color == c].sum()) + 24 * int((color == c).sum()) for c in range(nc)]
    order = (list(range(nc)) + list(range(nc - 1, -1, -1))) * sweeps
    run = [c for i, c in enumerate(order) if i == 0 or c != order[i - 1]]
    byts = sum(pass_bytes[c] for c in run) / sweeps
    peak, kind = load_peaks()
    S.close()
    A.close()
    return {"workload": "symgs_stencil27_128^3_8colours", "m": m, "nnz": int(A.nnz),
            "ms_per_sweep": ms, "achieved_gbs": byts / (ms / 1e3) / 1e9,
            "frac": byts / (ms / 1e3) / 1e9 / peak, "peak_kind": kind,
            "passes_per_sweep": len(run) / sweeps,
            "bytes_formula": "sum over executed colour passes of 8*offdiag_nnz_c + 24*m_c"}


def spmv_leg(G, torch, dev, stream, args):
    """27-point 3-D Laplacian, 128^3 grid: y = A x (x seeded uniform, y = 0)."""
    A = G.gen_stencil27(128)
    M = G.Matrix(A.rowptr, A.col, A.third, m=A.m, nnz=A.nnz)
    x = torch.empty(A.m, dtype=torch.float32, device=dev)
    G.gen_uniform(A.m, 11, x)
    y = torch.zeros(A.m, dtype=torch.float32, device=dev)
    for _ in range(3):
        M.spmv(x, y, stream.cuda_stream)
    torch.cuda.synchronize()
    reps = 20
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(reps):
        M.spmv(x, y, stream.cuda_stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / reps
    peak, kind = load_peaks()
    b = spmv_bytes(A.m, A.nnz)
    M.close()
    A.close()
    return {"workload": "spmv_stencil27_128^3", "m": A.m, "nnz": A.nnz, "ms": ms,
            "gflops": 2 * A.nnz / (ms / 1e3) / 1e9, "achieved_gbs": b / (ms / 1e3) / 1e9,
            "frac": b / (ms / 1e3) / 1e9 / peak, "peak": peak, "peak_kind": kind,
            "bytes_formula": "8*nnz + 16*m + 4"}


IO_SCALE = 20


def io_leg(G, args):
    """Graph loading for the PR driver (src/pr/main.cc:23-24 reads the file
    twice: out-CSR, then the transposed in-CSR).  A seeded RMAT scale-20
    graph (edge factor 16, shuffled edge order) is written as a .gr file;
    timed: the reference's own read_graph twice (single-threaded, compiled
    from the reference into oracle/_ref: a CPU baseline), and
    read_graph_pr (one multithreaded parse, both CSRs built on the GPU).
    Both results are compared."""
    import shutil
    import tempfile

    import oracle as O  # CPU baseline only
    csr = G.gen_rmat(IO_SCALE, EDGE_FACTOR, seed=SEED, abc=ABC)
    m = csr.m
    rp, col = csr.rowptr.to_numpy(), csr.col.to_numpy()
    csr.close()
    dst = np.repeat(np.arange(m, dtype=np.int64), np.diff(rp))
    order = np.random.default_rng(9).permutation(len(col))
    src, dst = col.astype(np.int64)[order] + 1, dst[order] + 1
    d = tempfile.mkdtemp()
    path = os.path.join(d, f"rmat{IO_SCALE}.gr")
    try:
        with open(path, "w") as f:
            f.write(f"p sp {m} {len(col)}\n")
            f.write("".join(f"a {a} {b} 1\n" for a, b in zip(src.tolist(), dst.tolist())))
        size = os.path.getsize(path)
        out = {"file": f"RMAT scale {IO_SCALE} .gr, {len(col)} arcs, {size / 1e6:.0f} MB",
               "threads": len(os.sched_getaffinity(0))}
        if O.ref_available():
            t0 = time.perf_counter()
            orp, ocol, _, _, _ = O.ref_read_graph(path, False, False, False)
            irp, icol, _, _, _ = O.ref_read_graph(path, False, True, False)
            out["reference_two_reads_s"] = time.perf_counter() - t0
        best = None
        for _ in range(2):
            t0 = time.perf_counter()
            o, i = G.read_graph_pr(path)
            G.synchronize()
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
            if _ == 0 and "reference_two_reads_s" in out:
                out["identical_to_reference"] = bool(
                    np.array_equal(o.rowptr.to_numpy(), orp) and np.array_equal(o.col.to_numpy(), ocol)
                    and np.array_equal(i.rowptr.to_numpy(), irp)
                    and np.array_equal(i.col.to_numpy(), icol))
            o.close()
            i.close()
        out["one_parse_gpu_build_s"] = best
        if "reference_two_reads_s" in out:
            out["speedup"] = out["reference_two_reads_s"] / best
        return out
    finally:
        shutil.rmtree(d, ignore_errors=True)


def profile_solve(args):
    """One solve of exactly N sweeps on the benchmark graph (for ncu)."""
    import torch

    import gardenia_ocl_b200 as G
    csr = G.gen_rmat(args.scale, EDGE_FACTOR, seed=SEED, abc=ABC)
    blocked = args.profile_form == "blocked"
    g = G.Graph(csr.rowptr, csr.col, csr.third, m=csr.m, nnz=csr.nnz, blocked=blocked)
    scores = torch.full((csr.m,), float(np.float32(1.0) / np.float32(csr.m)),
                        dtype=torch.float32, device="cuda")
    loop = G.LOOP_PERSISTENT if args.profile_loop == "persistent" else G.LOOP_GRAPH
    _, st = g.pagerank(scores, G.options(tol=0.0, max_iter=args.profile_solve, damping=DAMPING,
                                         loop=loop,
                                         form=G.FORM_BLOCKED if blocked else G.FORM_EXACT))
    log(json.dumps({"m": csr.m, "nnz": csr.nnz, "layout": g.layout(), **st.as_dict()}))
    g.close()
    csr.close()
    return 0


def profile_multigraph(args):
    """One FP32 solve of exactly --profile-solve sweeps (tol 0) on the first
    --profile-multigraph graphs of the multi-graph batch (for ncu)."""
    import torch

    import gardenia_ocl_b200 as G
    A, voff = G.gen_multigraph(args.profile_multigraph, MG_MMIN, MG_MMAX, seed=MG_SEED)
    blocked = args.profile_form == "blocked"
    mg = G.MultiGraph(A.rowptr, A.col, A.third, voff, nnz=A.nnz, blocked=blocked)
    scores = torch.from_numpy(mg.initial_scores()).cuda()
    _, it, _, st = mg.pagerank(scores, tol=0.0, max_iter=args.profile_solve or 10,
                               damping=DAMPING,
                               form=G.FORM_BLOCKED if blocked else G.FORM_EXACT)
    log(json.dumps({"info": mg.info(), **st.as_dict()}))
    mg.close()
    A.close()
    return 0


def profile_ppr(args):
    """One batched PPR solve of --profile-ppr vectors, exactly --profile-solve
    sweeps (tol 0) on the RMAT graph of --scale (for ncu)."""
    import torch

    import gardenia_ocl_b200 as G
    csr = G.gen_rmat(args.scale, EDGE_FACTOR, seed=SEED, abc=ABC)
    g = G.Graph(csr.rowptr, csr.col, csr.third, m=csr.m, nnz=csr.nnz, batched=True)
    k = args.profile_ppr
    seeds = np.random.default_rng(22).integers(0, csr.m, k).astype(np.int32)
    buf = torch.empty(csr.m * k, dtype=torch.float32, device="cuda")
    _, it, st = g.ppr(seeds, out=buf, tol=0.0, max_iter=args.profile_solve or 3)
    log(json.dumps({"m": csr.m, "nnz": csr.nnz, "k": k, **st.as_dict()}))
    g.close()
    csr.close()
    return 0


def profile_spmv(args):
    """--profile-spmv calls of y += A x on the 27-point 128^3 stencil (for ncu)."""
    import torch

    import gardenia_ocl_b200 as G
    A = G.gen_stencil27(128)
    M = G.Matrix(A.rowptr, A.col, A.third, m=A.m, nnz=A.nnz)
    x = torch.empty(A.m, dtype=torch.float32, device="cuda")
    G.gen_uniform(A.m, 11, x)
    y = torch.zeros(A.m, dtype=torch.float32, device="cuda")
    for _ in range(args.profile_spmv):
        M.spmv(x, y)
    torch.cuda.synchronize()
    log(json.dumps({"m": A.m, "nnz": A.nnz, "calls": args.profile_spmv}))
    M.close()
    A.close()
    return 0


def profile_symgs(args):
    """One SymGS apply of exactly --profile-symgs sweeps on the 27-point 128^3
    stencil with the 8-colour parity colouring (for ncu)."""
    import torch

    import gardenia_ocl_b200 as G
    A, S, x, b, _ = symgs_stencil(G, torch, torch.device("cuda"))
    ms = S.apply(x, b, sweeps=args.profile_symgs)
    log(json.dumps({"m": A.m, "nnz": A.nnz, "sweeps": args.profile_symgs, "ms": ms}))
    S.close()
    A.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=SCALE)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-spmv", action="store_true")
    ap.add_argument("--no-forms", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-multigraph", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="default bins and kernel variant")
    ap.add_argument("--no-s16", action="store_true", help="skip the RMAT s16 (tol 1e-4) leg")
    ap.add_argument("--no-ref-cuda", action="store_true",
                    help="skip the reference's own CUDA solvers on the benchmark inputs")
    ap.add_argument("--io", action="store_true",
                    help="also time graph loading: the reference's two read_graph calls vs "
                         "one parse with the CSRs built on the GPU")
    ap.add_argument("--tune-cache", default=None, metavar="PATH",
                    help="autotuner cache file (default: none, tune on every run)")
    ap.add_argument("--profile-solve", type=int, default=0, metavar="SWEEPS",
                    help="build the graph and run one solve of exactly SWEEPS sweeps, "
                         "nothing else (the case profiled with ncu)")
    ap.add_argument("--profile-loop", choices=["persistent", "graph"], default="persistent",
                    help="sweep loop of --profile-solve")
    ap.add_argument("--profile-form", choices=["exact", "blocked"], default="exact",
                    help="sweep form of --profile-solve (k_pr_hot / k_pr_step or k_pr_blocked) "
                         "and of --profile-multigraph (k_multi or k_multi_blocked)")
    ap.add_argument("--profile-multigraph", type=int, default=0, metavar="GRAPHS",
                    help="build the first GRAPHS graphs of the multi-graph batch and run one "
                         "solve of --profile-solve sweeps (the case profiled with ncu)")
    ap.add_argument("--profile-ppr", type=int, default=0, metavar="K",
                    help="one batched PPR solve with K seed vectors and --profile-solve sweeps "
                         "on the RMAT graph of --scale (the case profiled with ncu)")
    ap.add_argument("--profile-symgs", type=int, default=0, metavar="SWEEPS",
                    help="one SymGS apply of SWEEPS sweeps on the 128^3 stencil "
                         "(the case profiled with ncu)")
    ap.add_argument("--profile-spmv", type=int, default=0, metavar="CALLS",
                    help="CALLS SpMV calls on the 128^3 stencil (the case profiled with ncu)")
    args = ap.parse_args()
    if args.profile_spmv:
        return profile_spmv(args)
    if args.profile_symgs:
        return profile_symgs(args)
    if args.profile_multigraph:
        return profile_multigraph(args)
    if args.profile_ppr:
        return profile_ppr(args)
    if args.profile_solve:
        return profile_solve(args)
    if args.warmup < 3:
        log("warm-up raised to 3 steps (minimum)")
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
