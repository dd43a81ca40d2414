#!/usr/bin/env python
"""Benchmark of the greedy selection hot path on B200.

Workload (one bench step): a complete forward selection on the seeded
generator "fwd-64k": holdout, n_train=65,536, n_val=32,768, p=60, k=10,
15 greedy steps (60+59+...+46 = 795 candidate scorings).  Metric:
candidate-evaluations per second, one evaluation being one
(validation row, training row, candidate feature) triple.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours:       inputs resident in HBM; each step = snn_run (initial distance
            matrix + 15 x [score, reduce, select, commit]) timed with CUDA
            events on the library's stream.  `e2e` repeats it through the
            public API from pinned host buffers (upload + run + result read).
reference:  speedynn's own CPU neighbour scan (get_k_nearest_neighbors_cpu,
            speedynn/lib/cpu.c:128-168, compiled from the reference sources
            into oracle/_ref) on a bounded sample of the same workload:
            sampled validation rows x all 65,536 training rows x the 53
            candidates of the eighth greedy step (the first seven features
            committed into the sampled rows' distances), one process per host
            core.  ms_per_step is the measured time of one such sample.

Besides the timed loop, the default run (one GPU, rank 0) also reports:
  oracle      the selection against the full-size oracle fixture of the same
              workload (tests/golden/config_*.npz: ordering and FP32 errors
              bit for bit, and each FP32 error against the all-FP64 pipeline);
  batched     the batch workload (320 problems) run once as one batch and once
              as the plain single-problem form, with identical results checked;
  cpu_baseline  the reference CPU scan on a bounded sample (as --impl reference).

N > 1 (torchrun): every rank runs its own selection problem (seed offset by
rank): independent problems, no collective on the data path; value sums all
ranks' evaluations over the slowest rank's time.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOAD = "fwd-64k"
# DRAM bytes per (validation row, training row) pair of one scoring launch, from an
# ncu capture of a seeded step (dram__bytes_read.sum + dram__bytes_write.sum =
# 544.2 + 8.3 MB for 8192 x 16384 pairs): the D stream read once plus the small
# X, bound and label traffic.
TRAFFIC_PER_PAIR = 552.44e6 / (8192 * 16384)
# The same for the 64-slot lists (k in (32, 64]), from a seeded step with k = 50
# on 15,000 x 30,000 pairs: 1845.4 + 29.9 MB.
TRAFFIC_PER_PAIR_K64 = 1875.35e6 / (15000 * 30000)
METRIC = "cand-evals/s (n_val*n_train*candidates per second), greedy forward selection"
UNIT = "cand-evals/s"


def workload_desc(k, steps, n_train, n_val, p, name=WORKLOAD):
    method = "backward elimination" if name.startswith("bwd") else "forward selection"
    gb = 4.0 * n_train * n_val / 1e9
    return {"workload": f"{name}: {method}, holdout, n_train={n_train}, n_val={n_val}, p={p}, k={k}, "
                        f"{steps} greedy steps (seeded synthetic generator)",
            "n_train": n_train, "n_val": n_val, "p": p, "k": k, "greedy_steps": steps,
            "l2": f"inputs larger than L2 (distance matrix {gb:.1f} GB)"}


def rank_seed(seed, rank):
    """Seed of rank `rank`'s problem: every rank solves its own selection."""
    return seed + 1000 * rank


def allmax(x, world):
    """Maximum of x over the ranks of the current process group (a float)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(evals_per_rank, ms_max, world):
    """Whole-job throughput: all ranks' evaluations over the slowest rank's time."""
    return world * evals_per_rank / (ms_max / 1000.0)


def scoring_kernel(kmax, option=0):
    """Name of the scoring kernel the library picks (option 0 = automatic)."""
    if option == 3 or (option == 0 and kmax <= 64):
        return "k_score_tma"
    return "k_score"


# FP32-pipe operations per evaluation in the roofline's work count: sub, mul,
# add and compare (the reference's scalar loop); the scorer's filter issues one
# packed sub and one packed FMA per evaluation plus a sign-bit OR.
OPS_PER_EVAL = 4


def fixture_path(name):
    return os.path.join(ROOT, "tests", "golden", f"config_{name.replace('-', '')}.npz")


def data_sha256(split):
    import hashlib
    h = hashlib.sha256()
    for a in (split.Xtrain, split.ytrain, split.Xval, split.yval):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def oracle_statement(name, split, res):
    """The run's selection against the committed full-size oracle fixture of
    the same workload (tests/golden/make_config_golden.py): ordering and FP32
    errors bit for bit over the fixture's steps, FP64 errors against the
    oracle's FP64 sums, and each FP32 error against the all-FP64 pipeline."""
    path = fixture_path(name)
    if not os.path.exists(path):
        return {"available": False, "why": f"no fixture {os.path.basename(path)}"}
    g = np.load(path)
    if str(g["data_sha256"]) != data_sha256(split):
        return {"available": False, "why": "generated inputs differ from the fixture's (generator changed)"}
    slots = [int(x) for x in g["slots"]]
    e32 = np.array([res["errors"][i] for i in slots], np.float32)
    o32 = np.array([g["errors"][i] for i in slots], np.float32)
    e64 = np.array([res["errors64"][i] for i in slots])
    o64 = np.array([g["errors64"][i] for i in slots])
    pipe = np.asarray(g["errors_fp64_pipeline"], np.float64)
    gap = np.abs(e32.astype(np.float64) - pipe) / pipe
    return {"available": True, "fixture": os.path.basename(path), "steps_compared": len(slots),
            "ordering_equal": bool(all(res["ordering"][i] == g["ordering"][i] for i in slots)),
            "errors_bit_equal": bool(np.array_equal(e32, o32)),
            "errors64_max_rel_vs_oracle": float(np.max(np.abs(e64 - o64) / o64)),
            "fp32_vs_fp64_pipeline": {"max_rel": float(gap.max()), "per_step_rel": [float(x) for x in gap],
                                      "fp64_pipeline": [float(x) for x in pipe]},
            "note": "fp64_pipeline = RMSE of each step's winner with FP64 distances, FP64 neighbour order and "
                    "FP64 predictions (oracle, all rows); max_rel = largest |FP32 error - FP64 pipeline| / FP64 "
                    "pipeline over the steps"}


def cand_evals(n_rows, n_cols, p, steps):
    return float(n_rows) * n_cols * sum(p - t for t in range(steps))


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), float(f[3]), f[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [r for r in rows if r[2] > 200.0] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in load for i in range(4) if r[3][i].lower().startswith("active")})
        return {"sm_mhz": float(np.median([r[0] for r in load])), "sm_max_mhz": float(max(r[1] for r in rows)),
                "power_w_max": float(max(r[2] for r in rows)), "samples": len(load), "reasons": reasons}


# ---------------------------------------------------------------------------
# CPU reference: speedynn's own neighbour scan over sampled validation rows
# ---------------------------------------------------------------------------
_W = {}


def _ref_worker_init(npz_path, k, committed):
    import ctypes
    from oracle import ref
    d = np.load(npz_path)
    _W["Xv"], _W["yv"], _W["Xt"], _W["yt"] = d["Xval"], d["yval"], d["Xtrain"], d["ytrain"]
    _W["k"] = k
    _W["committed"] = list(committed)
    _W["lib"] = ref.load()
    _W["ct"] = ctypes


def _ref_worker_run(rows):
    """Holdout scoring of validation rows ``rows`` with the reference's own
    get_k_nearest_neighbors_cpu: the rows are placed in front of the training
    block as fold 0 (num_per_fold = len(rows)), so each scans exactly the
    training points; then the kNN mean and squared error as cpu.c:56-66.
    The rows' distances hold the committed features, summed in commit order
    with the reference's rounding (cpu.c:217-231), and every other feature is
    a candidate."""
    ct = _W["ct"]
    L = _W["lib"]
    Xv, yv, Xt, yt, k = _W["Xv"], _W["yv"], _W["Xt"], _W["yt"], _W["k"]
    R = len(rows)
    Xp = np.ascontiguousarray(np.concatenate([Xv[rows], Xt]), np.float32)
    yp = np.concatenate([yv[rows], yt]).astype(np.float32)
    n, p = Xp.shape
    D = np.zeros((R, n), np.float32)
    for w in _W["committed"]:
        t = (Xp[:R, w][:, None] - Xp[None, :, w]).astype(np.float32)
        D = (D + (t * t).astype(np.float32)).astype(np.float32)
    cands = [c for c in range(p) if c not in _W["committed"]]
    ib = np.zeros(k, np.int32)
    db = np.zeros(k, np.float32)
    ip = ib.ctypes.data_as(ct.POINTER(ct.c_int))
    dp = db.ctypes.data_as(ct.POINTER(ct.c_float))
    ct.c_int.in_dll(L, "dim").value = p
    ct.c_int.in_dll(L, "num_training_patterns").value = n
    ct.c_int.in_dll(L, "k_max").value = k
    ct.c_void_p.in_dll(L, "training_patterns").value = Xp.ctypes.data
    ct.c_void_p.in_dll(L, "current_dist_matrix").value = D.ctypes.data
    sse = np.zeros(p, np.float64)
    t0 = time.perf_counter()
    for c in cands:
        for r in range(R):
            L.get_k_nearest_neighbors_cpu(r, 0, R, ip, dp, c, 1)
            pred = np.float32(yp[ib].sum(dtype=np.float32) / np.float32(k))
            sse[c] += float(yp[r] - pred) ** 2
    el = time.perf_counter() - t0
    ct.c_void_p.in_dll(L, "current_dist_matrix").value = None
    ct.c_void_p.in_dll(L, "training_patterns").value = None
    return el, float(R) * Xt.shape[0] * len(cands)


class RefCPU:
    """Process pool timing the reference's CPU scan; one process per core."""

    def __init__(self, split, k, rows_per_proc, committed=(), procs=None):
        import multiprocessing as mp
        self.procs = procs or len(os.sched_getaffinity(0))
        fd, self.npz = tempfile.mkstemp(suffix=".npz")
        os.close(fd)
        np.savez(self.npz, Xval=split.Xval, yval=split.yval, Xtrain=split.Xtrain, ytrain=split.ytrain)
        self.committed = list(committed)
        self.pool = mp.get_context("spawn").Pool(self.procs, initializer=_ref_worker_init,
                                                 initargs=(self.npz, k, self.committed))
        self.rows = rows_per_proc
        self.nval = split.Xval.shape[0]
        self.calls = 0

    def step(self):
        """One bounded sample: `procs` disjoint row blocks in parallel."""
        jobs = []
        for w in range(self.procs):
            start = ((self.calls * self.procs + w) * self.rows) % max(1, self.nval - self.rows)
            jobs.append(list(range(start, start + self.rows)))
        self.calls += 1
        t0 = time.perf_counter()
        res = self.pool.map(_ref_worker_run, jobs)
        wall = time.perf_counter() - t0
        evals = sum(r[1] for r in res)
        return evals, wall

    def close(self):
        self.pool.close()
        self.pool.join()
        os.unlink(self.npz)


def ref_available():
    return os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libspeedynn_ref.so"))


def port_cpu_rate(split, k, rows, committed=()):
    """Fallback CPU baseline: the oracle restatement (OpenMP, all cores)."""
    from oracle import oracle
    prob = oracle.Problem(split.Xtrain, split.ytrain, split.Xval, split.yval)
    p = split.Xtrain.shape[1]
    cands = [c for c in range(p) if c not in committed]
    t0 = time.perf_counter()
    oracle.step(prob, [k], list(committed), cands, rows=list(range(rows)), want_neighbours=False)
    el = time.perf_counter() - t0
    return float(rows) * split.Xtrain.shape[0] * len(cands) / el, el


# The reference arm and the CPU baseline sample the eighth greedy step: the
# first seven winners of the fwd-64k oracle fixture are committed (the first
# seven features otherwise), leaving 53 candidates, the selection's average.
REF_COMMITTED = 7


def ref_committed(name, split):
    path = fixture_path(name)
    if os.path.exists(path):
        g = np.load(path)
        if str(g["data_sha256"]) == data_sha256(split):
            return [int(x) for x in g["commit_order"][:REF_COMMITTED]]
    return list(range(REF_COMMITTED))


# ---------------------------------------------------------------------------
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args, world, rank):
    from speedynn_b200 import datagen
    if rank != 0:
        return 0
    split, k, steps = datagen.workload(WORKLOAD)
    n_train, n_val, p = split.Xtrain.shape[0], split.Xval.shape[0], split.Xtrain.shape[1]
    cfg = dict(workload_desc(k, steps, n_train, n_val, p), parallelism=f"independent problems x{world}")
    line = {"impl": "reference", "metric": METRIC, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": cfg}
    committed = ref_committed(WORKLOAD, split)
    n_cand = p - len(committed)
    if ref_available():
        rc = RefCPU(split, k, args.ref_rows, committed)
        for _ in range(args.warmup):
            rc.step()
        tot_e, tot_t = 0.0, 0.0
        for _ in range(args.steps):
            e, t = rc.step()
            tot_e += e
            tot_t += t
        rc.close()
        v = tot_e / tot_t
        kind = "reference"
        sample = (f"speedynn get_k_nearest_neighbors_cpu + kNN mean, {rc.procs} processes x {args.ref_rows} "
                  f"validation rows x {n_train} training rows x {n_cand} candidates (greedy step "
                  f"{len(committed) + 1}, {len(committed)} features committed) per bench step")
        cores = rc.procs
    else:
        el_tot = 0.0
        for _ in range(args.steps):
            v, el = port_cpu_rate(split, k, args.ref_rows, committed)
            el_tot += el
        tot_t = el_tot
        kind = "port"
        cores = len(os.sched_getaffinity(0))
        sample = f"oracle restatement, {args.ref_rows} validation rows x {n_train} x {n_cand} candidates"
    line.update({"value": v, "ms_per_step": 1000.0 * tot_t / max(1, args.steps),
                 "ms_per_step_note": "measured: one bounded sample (see cpu_baseline.sample) per bench step",
                 "ms_full_selection_extrapolated": 1000.0 * cand_evals(n_val, n_train, p, steps) / v,
                 "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
                 "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                 "gpu_launches": 0})
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, world, rank, local):
    import torch
    import torch.distributed as dist

    from speedynn_b200 import datagen
    from speedynn_b200.selector import Selector

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    name = args.workload
    w = dict(datagen.WORKLOADS[name])
    k, select = w.pop("k"), w.pop("select")
    backward = name.startswith("bwd")
    steps = w["p"] - select if backward else select  # backward keeps `select` features
    w["seed"] = rank_seed(w["seed"], rank)
    if args.rows_scale != 1.0:
        w["n_train"] = int(w["n_train"] * args.rows_scale)
        w["n_val"] = int(w["n_val"] * args.rows_scale)
    split = datagen.generate(**w)
    n_train, n_val, p = split.Xtrain.shape[0], split.Xval.shape[0], split.Xtrain.shape[1]
    evals = cand_evals(n_val, n_train, p, steps)

    sel = Selector(split.Xtrain, split.ytrain, split.Xval, split.yval, k_vals=[k],
                   num_features=select if backward else steps, method="backward" if backward else "forward",
                   device=local)
    sel.set_kernel(args.kernel)
    if args.seed_step is not None:
        sel.set_seed_step(args.seed_step)
    for _ in range(args.warmup):
        sel.run()

    gpu_index = local
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x for x in vis.split(",") if x.strip()]
        if local < len(ids):
            gpu_index = ids[local]
    clk = Clocks(gpu_index)
    barrier()
    clk.start()
    tot_ms = score_ms = commit_ms = setup_ms = 0.0
    score_n = commit_n = launches = 0
    step_score = np.zeros(steps)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sel.run()
        tm = sel.timing()
        tot_ms += tm["total_ms"]
        score_ms += tm["score_ms"]
        score_n += tm["score_launches"]
        commit_ms += tm["commit_ms"]
        commit_n += tm["commit_launches"]
        launches += tm["launches"]
        setup_ms += sel.setup_ms()
        step_score += sel.step_timing()[0][:steps]
    barrier()
    wall = time.perf_counter() - t0
    clocks = clk.stop()
    res = sel.results()
    # one more selection with the filter counters on (outside the timed region)
    sel.set_counters(True)
    sel.run()
    fc = sel.filter_counters()
    sel.set_counters(False)
    ms_step = allmax(tot_ms / args.steps, world)

    # end to end through the public API: pinned host inputs uploaded every step, results read back
    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        return t.numpy()
    hx, hy, hxv, hyv = pinned(split.Xtrain), pinned(split.ytrain), pinned(split.Xval), pinned(split.yval)
    h2d = hx.nbytes + hy.nbytes + hxv.nbytes + hyv.nbytes
    from speedynn_b200 import _lib
    from speedynn_b200._lib import _f32p, ptr
    L = _lib.lib()
    barrier()
    e0 = time.perf_counter()
    d2h = 0
    for _ in range(0 if args.no_e2e else args.steps):
        _lib.check(L.snn_load(sel._h, ptr(hx, _f32p), ptr(hy, _f32p), ptr(hxv, _f32p), ptr(hyv, _f32p)))
        _lib.check(L.snn_run(sel._h))
        r = sel.results()
        d2h = sum(v.nbytes for v in r.values() if isinstance(v, np.ndarray)) + 8
    barrier()
    e2e_s = allmax((time.perf_counter() - e0) / args.steps, world)
    sel.close()

    # roofline of the scoring kernel: FP32 pipe (OPS_PER_EVAL ops per evaluation) vs one D read
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    hbm_src = "measured" if "hbm_gbs" in peaks else "fallback"
    sm = torch.cuda.get_device_properties(local).multi_processor_count
    mhz = clocks.get("sm_mhz") or float(peaks.get("sm_max_mhz", 1965.0))
    fp32_peak = sm * 128 * mhz * 1e6 * 1e-12  # T ops/s of the FP32 pipe at the sampled clock
    avg_score_s = score_ms / max(1, score_n) / 1000.0
    evals_per_launch = evals / steps
    achieved_fp32 = OPS_PER_EVAL * evals_per_launch / avg_score_s * 1e-12
    bytes_per_launch = 4.0 * n_val * n_train
    achieved_hbm = bytes_per_launch / avg_score_s * 1e-9
    # the same over the steps that scan every column (forward holdout steps 1
    # and 2 take their lists from sorted feature values instead, for k <= 64)
    first_scan = 0 if backward else (2 if k <= 64 else 1)
    scan_evals = sum(float(n_val) * n_train * (p - t) for t in range(first_scan, steps))
    scan_s = float(step_score[first_scan:].sum()) / args.steps / 1000.0
    achieved_scan = OPS_PER_EVAL * scan_evals / scan_s * 1e-12 if scan_s > 0 else None

    line = {"metric": METRIC, "value": job_value(evals, ms_step, world), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(workload_desc(k, steps, n_train, n_val, p, name), parallelism=f"independent problems x{world}"),
            "greedy_step_ms": ms_step / steps,
            "breakdown_ms_per_step": {"score": score_ms / args.steps, "commit": commit_ms / args.steps,
                                      "initial_distance": setup_ms / args.steps,
                                      "other": (tot_ms - score_ms - commit_ms - setup_ms) / args.steps},
            "score_ms_per_greedy_step": [round(float(x) / args.steps, 3) for x in step_score],
            "wall_ms_per_step": 1000.0 * wall / args.steps,
            "e2e": None if args.no_e2e else {"value": world * evals / e2e_s, "unit": UNIT,
                                             "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": launches,
            "filter": {"row_chunks": fc["row_chunks"],
                       "flagged_frac": fc["flagged"] / fc["row_chunks"] if fc["row_chunks"] else None,
                       "passing_frac": fc["passed"] / fc["row_chunks"] if fc["row_chunks"] else None,
                       "note": "(row, 64-column chunk) pairs of the TMA-fed scorer's full passes in one selection "
                               "(counted in an extra untimed run); flagged = re-scored exactly, passing = held a "
                               "list update candidate"},
            "roofline": {"bound": "fp32", "kernel": scoring_kernel(k, args.kernel), "achieved": achieved_fp32,
                         "peak": fp32_peak,
                         "unit": "TFLOP/s", "frac": achieved_fp32 / fp32_peak,
                         "ops_per_eval": OPS_PER_EVAL,
                         "frac_scan_steps": achieved_scan / fp32_peak if achieved_scan else None,
                         "scan_steps_note": f"steps {first_scan + 1}..{steps} only (the scanning launches); the "
                                            "first steps of a forward holdout run are served from sorted "
                                            "feature values and count their evaluations without scanning them",
                         "frac_3op": 0.75 * achieved_fp32 / fp32_peak,
                         "evals_per_s_per_launch": evals_per_launch / avg_score_s,
                         "launch_ms": avg_score_s * 1000.0,
                         "peak_source": f"{sm} SMs x 128 FP32 lanes x {mhz:.0f} MHz (sampled median; "
                                        "MEASURED_PEAKS.json holds no FP32 figure); work = 4 FP32-pipe ops per "
                                        "evaluation (sub, mul, add, compare); frac_3op counts the 3 rounded "
                                        "arithmetic ops only",
                         "hbm_achieved_gbs": achieved_hbm, "hbm_peak_gbs": hbm, "hbm_peak_source": hbm_src,
                         "hbm_frac": achieved_hbm / hbm,
                         "traffic": args.traffic if args.traffic is not None else
                         (TRAFFIC_PER_PAIR_K64 if 32 < k <= 64 else TRAFFIC_PER_PAIR) * n_val * n_train,
                         "traffic_source": "command line" if args.traffic is not None else
                         ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one seeded k_score_tma launch on "
                          + ("the k = 50, 30000 x 15000 case (1875.4 MB, profiles/k_score_tma_k50_small_ncu.md)"
                             if 32 < k <= 64 else
                             "the 16384 x 8192 case (552.4 MB, profiles/k_score_tma_small_ncu.md)")
                          + ", scaled per (validation row, training row) pair")},
            "clocks": clocks,
            "result": {"ordering": [int(x) for x in res["ordering"][:steps]],
                       "errors": [float(x) for x in res["errors"][:steps]]}}
    if name != WORKLOAD:
        line["metric"] = METRIC.replace("greedy forward selection", "greedy backward elimination" if backward else
                                        "greedy forward selection") + f" ({name})"
    if rank == 0 and world == 1 and args.rows_scale == 1.0 and not args.no_oracle:
        line["oracle"] = oracle_statement(name, split, res)
    if rank == 0 and world == 1 and name == WORKLOAD and args.rows_scale == 1.0 and not args.no_batch:
        line["batched"] = batch_summary(args, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline and name == WORKLOAD:
        committed = ref_committed(name, split)
        n_cand = p - len(committed)
        if ref_available():
            rc = RefCPU(split, k, args.cpu_rows, committed)
            e, t = rc.step()
            rc.close()
            line["cpu_baseline"] = {"value": e / t, "unit": UNIT, "cores": rc.procs, "kind": "reference",
                                    "sample": f"speedynn get_k_nearest_neighbors_cpu + kNN mean, {rc.procs} "
                                              f"processes x {args.cpu_rows} validation rows x {n_train} x {n_cand} "
                                              f"candidates (greedy step {len(committed) + 1})"}
        else:
            v, el = port_cpu_rate(split, k, args.cpu_rows, committed)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": len(os.sched_getaffinity(0)), "kind": "port",
                                    "sample": f"oracle restatement, {args.cpu_rows} rows x {n_train} x {n_cand}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_plain(probs, batch_res, evals, batch_ms, world):
    """The plain single-problem form of the batch workload: the same problems
    one after another through the handle API (device time of each snn_run),
    with the selected features and errors checked against the batch's."""
    from speedynn_b200.selector import Selector

    plain_ms = 0.0
    same = True
    best_rate = 0.0
    by_k = {}  # k -> [evaluations, ms]: the plain form's rate per list length
    for pr, rb in zip(probs, batch_res):
        with Selector(pr["Xtrain"], pr["ytrain"], pr["Xval"], pr["yval"], k_vals=pr["k_vals"],
                      num_features=pr["num_features"], method=pr["method"]) as sel:
            r = sel.run()
            ms = sel.timing()["total_ms"]
            plain_ms += ms
        e = cand_evals(pr["Xval"].shape[0], pr["Xtrain"].shape[0], pr["Xtrain"].shape[1], pr["num_features"])
        best_rate = max(best_rate, e / (ms / 1000.0))
        acc = by_k.setdefault(int(max(pr["k_vals"])), [0.0, 0.0])
        acc[0] += e
        acc[1] += ms
        same = same and np.array_equal(r["ordering"], rb["ordering"]) and np.array_equal(r["errors"], rb["errors"])
    # a batch can at best run every problem at the rate the best single problem reaches alone
    ceiling_ms = 1000.0 * evals / best_rate
    return {"ms": plain_ms, "value": world * evals / (plain_ms / 1000.0), "batched_speedup": plain_ms / batch_ms,
            "identical_results": bool(same), "best_single_problem_rate": best_rate,
            "ceiling_ms": ceiling_ms, "ceiling_speedup": plain_ms / ceiling_ms,
            "rate_by_k": {str(k): v[0] / (v[1] / 1000.0) for k, v in sorted(by_k.items())},
            "note": "the problems one at a time (CUDA-event time of each selection, creates and uploads excluded); "
                    "ceiling: all evaluations at the best single problem's own rate"}


def batch_summary(args, local):
    """Batched vs plain on the batch workload (320 holdout problems), outside
    the timed loop of the default line: one warm-up batch, one measured batch
    (device time and end to end through snn_batch_*), then the same problems
    one at a time through the handle API, results compared."""
    from speedynn_b200 import datagen
    from speedynn_b200.batch import Batch

    probs = datagen.batch_workload(seed0=4000)
    evals = sum(cand_evals(pr["Xval"].shape[0], pr["Xtrain"].shape[0], pr["Xtrain"].shape[1], pr["num_features"])
                for pr in probs)
    b = Batch(probs)
    b.run()
    t0 = time.perf_counter()
    res = b.run()
    wall = time.perf_counter() - t0
    tm = b.timing()
    b.close()
    plain = run_plain(probs, res, evals, tm["run_ms"], 1)
    return {"workload": f"batch-64x5: {len(probs)} holdout forward selections, n_train 1,045..30,790, p=40, "
                        "k in {1,5,10,20}, 15 steps", "evals": evals,
            "batch_ms": tm["run_ms"], "batch_value": evals / (tm["run_ms"] / 1000.0),
            "batch_e2e_value": evals / wall, "batch_e2e_ms": 1000.0 * wall,
            "plain_ms": plain["ms"], "plain_value": plain["value"], "batched_speedup": plain["batched_speedup"],
            "identical_results": plain["identical_results"], "ceiling_speedup": plain["ceiling_speedup"],
            "best_single_problem_rate": plain["best_single_problem_rate"],
            "plain_rate_by_k": plain["rate_by_k"],
            "note": "batch_ms: union of the problems' CUDA-event intervals; batch_e2e: snn_batch_run wall time "
                    "(creates, uploads, runs, result reads, frees); plain: each problem's own selection time"}


def run_batch(args, world, rank, local):
    """One bench step = one snn_batch_run over the 320 holdout problems of the
    batch workload (64 pools x 5 seeded train/validation splits)."""
    import torch

    from speedynn_b200 import datagen
    from speedynn_b200.batch import Batch

    torch.cuda.set_device(local)
    probs = datagen.batch_workload(seed0=4000 + 1000 * rank, scale_rows=args.rows_scale)
    evals = sum(cand_evals(pr["Xval"].shape[0], pr["Xtrain"].shape[0], pr["Xtrain"].shape[1], pr["num_features"])
                for pr in probs)
    d_bytes = sum(4.0 * pr["Xval"].shape[0] * pr["Xtrain"].shape[0] for pr in probs)
    b = Batch(probs)
    for _ in range(args.warmup):
        b.run()
    clk = Clocks(local)
    clk.start()
    run_ms = 0.0
    wall = 0.0
    waves = 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        res = b.run()
        wall += time.perf_counter() - t0
        tm = b.timing()
        run_ms += tm["run_ms"]
        waves = tm["waves"]
    clocks = clk.stop()
    b.close()
    ms = run_ms / args.steps
    h2d = sum(pr["Xtrain"].nbytes + pr["ytrain"].nbytes + pr["Xval"].nbytes + pr["yval"].nbytes for pr in probs)
    n_tr = [pr["Xtrain"].shape[0] for pr in probs]
    line = {"metric": METRIC + " (batch-64x5)", "value": world * evals / (ms / 1000.0), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"batch-64x5: {len(probs)} holdout forward selections (64 pools, n_train "
                                   f"log-uniform in [1024, 40000] -> {min(n_tr)}..{max(n_tr)}, n_val = n_train/2, "
                                   f"p=40, k in {{1,5,10,20}}, 15 steps, 5 seeded splits each)",
                       "problems": len(probs), "distance_matrices_gb": d_bytes / 1e9, "waves": waves,
                       "l2": "inputs larger than L2", "parallelism": "one CUDA stream per problem"},
            "e2e": {"value": world * evals / (wall / args.steps), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(sum(pr["Xtrain"].shape[1] * 28 + 8 for pr in probs))},
            "clocks": clocks}
    if not args.no_plain and args.steps > 0:
        line["plain"] = run_plain(probs, res, evals, ms, world)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--ref-rows", type=int, default=64, help="validation rows per process per reference step")
    ap.add_argument("--cpu-rows", type=int, default=96, help="validation rows per process for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--rows-scale", type=float, default=1.0,
                    help="scale n_train and n_val (small cases for profiler captures; not the bench workload)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end pass (profiler captures)")
    ap.add_argument("--no-plain", action="store_true",
                    help="batch workload: skip running the problems one at a time for comparison")
    ap.add_argument("--kernel", type=int, default=0, help="scoring kernel: 0 auto, 1 rows per lane, 3 TMA-fed row tiles")
    ap.add_argument("--seed-step", type=int, default=None,
                    help="first forward step scored from seed bounds (library option; default: the library's)")
    ap.add_argument("--no-oracle", action="store_true", help="skip the comparison with the full-size oracle fixture")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batch-vs-plain comparison that the default workload's line carries")
    ap.add_argument("--workload", default=WORKLOAD,
                    choices=["fwd-64k", "bwd-50k", "fwd-200k", "batch-64x5"],
                    help="fwd-64k (the headline), bwd-50k (backward, p=120 -> 20), fwd-200k (80 GB distance matrix, "
                         "k=50), batch-64x5 (320 holdout problems in one batch)")
    ap.add_argument("--traffic", type=float, default=None,
                    help="ncu dram bytes per scoring launch, scaled to this workload (reported as roofline.traffic)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference(args, world, rank)
    if args.workload.startswith("batch"):
        return run_batch(args, world, rank, local)
    return run_ours(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
