#!/usr/bin/env python
"""Benchmark: certified BM-ADMM solves per second at n = 18 (1 % menu density), abs gap 1e-5.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--dtype float64|mixed] [--impl rumb|reference]
    python bench.py --profile-case ITERS [--dtype ...]   # one solve capped at ITERS iterations, for
                                                          # profilers; prints no bench line
    python bench.py --workload bootstrap_n20             # batched bootstrap draws vs one at a time
    python bench.py --workload paper                     # paper instances beside the reference's times
    python bench.py --workload pricing --steps 20        # Flow-CG pricing sweeps alone
    python bench.py --workload pricing_large             # pricing calls at n = 28, 30, 32 (pairwise)
    python bench.py --workload dsr_n25                   # p_hat's solve at the learned warm start's
                                                          # shape (n = 25), time-boxed

Workload "n18_d1pct_k50": every menu of 18 alternatives with >= 2 members kept with probability
0.01 (2,627 menus, 23,650 observed cells), p_hat from a Dirichlet(1) mixture of 50 random linear
orders with Multinomial(500) noise per menu, seed 0 (rumb.instances). A step is one certified
solve from the cold start: float64 upper and lower bound every 50 iterations until ub - lb <=
1e-5 (rel_tol off), i.e. the reference's RUM.calculate_distance(method="bm_admm") bracket.

value   solves/s with the instance already in HBM (device pointers), all ranks summed
e2e     the same through the C ABI from host buffers: rows uploaded and p_fit read back per solve
roofline, for the kernel with the largest time share over 20 iterations and one check (after 2000
        untimed iterations), captured as a CUDA graph with events around every kernel and
        replayed: algorithmic bytes per launch / its launch time, against MEASURED_PEAKS.json
        hbm_gbs; traffic = DRAM bytes per launch from the committed ncu summary of the same kernel
        source (profiles/), null when there is none for the source built now
reference_kernels   one certified solve of the same workload by the reference's own float64
        kernels (its source strings compiled by NVRTC, replayed with its host sequence:
        baseline/ref_replay.py), and value / its solves/s
gpu_launches   the library's own count of the kernels the timed solves launched
mixed_state    the same certified solve with a float32 state until its bracket stalls, then float64
        (rumb_bm_params dtype RUMB_MIXED; the bounds are float64 throughout)
bootstrap      the metric's second half: p_hat certified, then 4 draws of the n = 20 panel solved to
        abs 5e-4 batched against 2 of the same draws one at a time (bootstrap_leg), and the screen
        of 10,000 draws
cpu_baseline   the oracle (C restatement of the reference's iteration and certificate) on the host,
        a bounded sample of iterations extrapolated to solves/s by this run's iteration count

--impl reference times the reference's CPU path -- the oracle port, all host threads -- on a
bounded sample per step, extrapolated by the iteration count of the reference's own kernels on the
same workload, and prints its line with "impl": "reference" and "extrapolated": true.

Multi-GPU: a single solve does not shard (the prox couples every alternative of a menu each
iteration), so N GPUs run N replicas of the solve (weak scaling, no collective on the data path);
NCCL carries only the barrier and the max-over-ranks step time.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rum-testing-gpu_b200"))

import numpy as np  # noqa: E402

WORKLOAD = "n18_d1pct_k50"
METRIC = "n=18 BM-ADMM certified solves/s at abs gap 1e-5"
ABS_TOL = 1e-5
CHECK = 50
# iterations run before the profiled ones: the roofline kernel is timed mid-solve
PROFILE_WARMUP = 2000
PROFILES = os.path.join(ROOT, "profiles")


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# the kernel sources whose digest a committed ncu summary must match for its DRAM figure to count
KERNEL_SOURCES = {"prox": ("prox.cu", "prox.cuh"), "xform": ("xform.cuh",)}


def source_digest(kernel):
    import hashlib
    files = next((v for k, v in KERNEL_SOURCES.items() if kernel.startswith(k)), None)
    if files is None:
        return None
    h = hashlib.sha256()
    for f in files:
        h.update(open(os.path.join(ROOT, "rum-testing-gpu_b200", "csrc", f), "rb").read())
    return h.hexdigest()[:16]


def kernel_traffic(kernel):
    """(DRAM bytes read + written per launch, summary file) of `kernel` from the committed ncu
    summaries in profiles/: a summary names `kernel:`, `source_sha256:` and
    `dram_bytes_per_launch:` on lines of their own, and counts only when its digest is the digest of
    the kernel source built now; otherwise (None, None)."""
    want = source_digest(kernel)
    if want is None or not os.path.isdir(PROFILES):
        return None, None
    for f in sorted(os.listdir(PROFILES)):
        if not f.endswith(".md"):
            continue
        kv = {}
        for line in open(os.path.join(PROFILES, f)):
            line = line.strip().strip("`")
            for key in ("kernel:", "source_sha256:", "dram_bytes_per_launch:"):
                if line.startswith(key):
                    kv[key[:-1]] = line[len(key):].strip()
        if kv.get("kernel") == kernel and kv.get("source_sha256") == want and "dram_bytes_per_launch" in kv:
            return float(kv["dram_bytes_per_launch"]), f
    return None, None


def reference_kernels_leg(n, menu, alt, p, beta):
    """One certified float64 solve of the workload by the reference's own kernels (its source
    strings NVRTC-compiled into baseline/_ref and replayed with its host sequence: one_iter as a
    CUDA graph with its calibrated butterfly plan, the float64 push and lower bound every `check`
    iterations with the runner's hooks, solver/bm_admm/solver.py:148-377,
    solver/rum_solver.py:879-905), timed on the wall clock with the device synchronized on both
    sides; setup (compilation, calibration, cold start) excluded."""
    sys.path.insert(0, os.path.join(ROOT, "baseline"))
    import ref_replay
    if not ref_replay.available():
        return {"unavailable": "baseline/_ref not built: the reference's source tree was absent at build time"}
    import torch
    r = ref_replay.BMReplay(n, menu, alt, p, beta)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = r.solve(abs_tol=ABS_TOL, check=CHECK, lb_every=1)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    del r
    torch.cuda.empty_cache()
    return {"impl": "the reference's float64 solve_kadmm_v2 kernels, replayed on this GPU",
            "s_per_solve": wall, "solves_per_s": 1.0 / wall, "iters": int(res["iters"]),
            "checks": int(res["checks"]), "ms_per_iter": 1e3 * res["iter_s"] / max(1, res["iters"]),
            "ms_per_check": 1e3 * res["check_s"] / max(1, res["checks"]), "ub": res["ub"], "lb": res["lb"],
            "stop": res["stop_reason"]}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def instance():
    from rumb.instances import config_instance
    n, menu, alt, p = config_instance(WORKLOAD, seed=0)
    return n, menu.astype(np.uint32), alt.astype(np.int32), p.astype(np.float64)


def beta_rule(mp):
    from rumb.params import bm_beta_default
    return bm_beta_default(mp)


# ------------------------------------------------------------------ CPU paths (oracle)
def cpu_sample(n, menu, alt, p, threads, iters_per_solve, checks_per_solve, sample_iters):
    """(solves/s, description, threads used): the oracle's iteration and float64 check, timed on a
    bounded sample and scaled to one certified solve."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    used = O.set_threads(threads)
    bm = O.BMOracle(n, menu, alt, p, beta=beta_rule(p.size))
    bm.iterate(1)
    t0 = time.perf_counter()
    bm.iterate(sample_iters)
    t_it = (time.perf_counter() - t0) / sample_iters
    t0 = time.perf_counter()
    O.push_ub64(n, bm.x2, bm.obs, bm.p)
    O.fw_lb64(n, bm.obs, bm.x2[bm.obs], bm.p)
    t_chk = time.perf_counter() - t0
    per_solve = iters_per_solve * t_it + checks_per_solve * t_chk
    desc = ("%d float64 ADMM iterations + 1 float64 check (push + lower bound) of %s on %d thread(s): "
            "%.1f ms/iteration, %.1f ms/check, extrapolated to %d iterations and %d checks per certified solve"
            % (sample_iters, WORKLOAD, used, 1e3 * t_it, 1e3 * t_chk, iters_per_solve, checks_per_solve))
    return 1.0 / per_solve, desc, used


def run_reference(args, rank):
    """The reference arm: the reference's CPU path (the oracle port of its iteration and float64
    check) on every host thread, on a bounded sample of iterations per step, extrapolated to a
    certified solve by the iteration and check counts of the reference's own float64 kernels on
    this workload (one solve replayed on the GPU before the timed steps)."""
    if rank != 0:
        return
    n, menu, alt, p = instance()
    beta = beta_rule(p.size)
    iters = checks = None
    source = None
    try:
        import torch
        if torch.cuda.is_available():
            leg = reference_kernels_leg(n, menu, alt, p, beta)
            if "iters" in leg:
                iters, checks = leg["iters"], leg["checks"]
                source = "counted by one certified solve of the reference's own float64 kernels (replayed on the GPU)"
            else:
                source = leg.get("unavailable")
    except Exception as e:                                  # no GPU or no reference kernels: say so
        source = "reference kernels unavailable (%s)" % str(e).splitlines()[0][:120]
    if iters is None:
        line = {"impl": "reference", "unavailable": "the iteration count of a certified solve needs the reference's "
                "kernels on a GPU: " + (source or "no GPU")}
        print(json.dumps(line), flush=True)
        return
    vals = []
    desc, used = "", 0
    sample = 10
    for i in range(args.warmup + args.steps):
        v, desc, used = cpu_sample(n, menu, alt, p, 0, iters, checks, sample_iters=sample)
        if i >= args.warmup:
            vals.append(v)
    value = statistics.mean(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "extrapolated": True, "sample_iters": sample, "iters_per_solve": iters, "checks_per_solve": checks,
            "iters_source": source,
            "config": {"workload": WORKLOAD, "n": n, "cells": int(p.size), "abs_tol": ABS_TOL, "check": CHECK,
                       "iters_per_solve": iters},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": used, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def pricing_sweeps(ctx, stream, sweeps=20):
    """Flow-CG pricing at n = 18, 0.5 % menus (workload n18_d05pct_k50): the uint24, uint16 and mask
    sweeps over the cover lists and the uint24 sweep scanning rows (one full Bellman-Ford pass over
    the lattice plus the backtrace, read back each sweep), timed with CUDA events on the bench
    stream; seeded float32 scores resident on the GPU."""
    import torch
    from rumb import _lib, flow_cg
    from rumb.instances import config_instance
    n, menu, alt, p = config_instance("n18_d05pct_k50", seed=0)
    menus, alts, p32, offsets, _ = flow_cg.prepare_choice_data(menu, alt, p, n)
    scores = torch.from_numpy(np.random.default_rng(0).standard_normal(menus.size).astype(np.float32)).cuda()
    out = {"workload": "n18_d05pct_k50", "rows": int(menus.size), "subset_tests_per_sweep": int(menus.size) << (n - 1)}
    for mode, lists in (("u24", True), ("u16", True), ("mask", True), ("u24", False)):
        pr = _lib.Pricer(ctx, n, menus, offsets, mode=mode, lists=lists)
        for _ in range(3):
            pr.price_device(scores.data_ptr())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(sweeps):
            pr.price_device(scores.data_ptr())
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / sweeps
        entries = pr.list_entries
        if lists:
            out["cover_list_entries"] = entries
        # the cover lists read per sweep: n 2^(n-1) + 1 uint32 offsets and the uint16 entries
        list_bytes = 4 * ((n << (n - 1)) + 1) + 2 * entries if entries >= 0 else 0
        out[mode if lists else mode + "_row_scan"] = {
            "ms_per_sweep": ms, "sweeps_per_s": 1e3 / ms,
            "subset_tests_per_s": out["subset_tests_per_sweep"] / (ms * 1e-3),
            "list_bytes_per_sweep": list_bytes, "list_gb_per_s": list_bytes / (ms * 1e-3) / 1e9}
        pr.close()
    # the reference's own pricing kernels on the same scores (layer launches only: a lower bound)
    sys.path.insert(0, os.path.join(ROOT, "baseline"))
    import ref_replay
    if ref_replay.available():
        ref = ref_replay.time_pricing(menus, offsets, scores.cpu().numpy(), n)
        out["reference_kernels"] = {"u24_ms_per_sweep": ref["u24_layers_ms"], "u16_ms_per_sweep": ref["u16_layers_ms"],
                                    "mask_ms_per_sweep": ref["mask_layers_ms"],
                                    "note": "the reference's layer kernels alone (no backtrace, no reads): a lower "
                                            "bound of its sweep"}
        for mode in ("u24", "u16", "mask"):
            out["speedup_vs_reference_" + mode] = ref[mode + "_layers_ms"] / out[mode]["ms_per_sweep"]
    return out


def run_pricing(args, rank):
    """Workload pricing: the Flow-CG pricing sweeps of n18_d05pct_k50 alone (cover lists in the
    u24, u16 and mask storages, and the row scan for comparison), one JSON line."""
    if rank != 0:
        return
    import torch
    from rumb import _lib
    ctx = _lib.Context(0)
    stream = torch.cuda.current_stream()
    res = pricing_sweeps(ctx, stream, sweeps=max(args.steps, 1))
    print(json.dumps({"metric": "Flow-CG pricing sweeps/s (n = 18, 0.5 % menus)", "value": res["u24"]["sweeps_per_s"],
                      "unit": "sweeps/s", "n_gpus": 1, "higher_is_better": True, "dtype": "u24",
                      "data": "synthetic", "config": {"workload": "n18_d05pct_k50"}, "pricing": res}), flush=True)


def run_bootstrap(args, rank, batch_draws=8, single_draws=4):
    """Workload bootstrap_n20: bootstrap_leg with 8 batched and 4 one-at-a-time draws, as its own line."""
    if rank != 0:
        return
    print(json.dumps(bootstrap_leg(batch_draws, single_draws)), flush=True)


def bootstrap_leg(batch_draws, single_draws):
    """The bootstrap half of the metric (n20_d1pct_panel520: n = 20, 1 % menus, a 520-respondent
    panel of 30 menus each, K = 30): certify p_hat, then solve open draws to abs 5e-4 from p_hat's
    state, batched (rumb_bm_solve_batch, all draws resident) against one at a time (Session.solve),
    both float64. Wall time around each phase with the device synchronized on both sides; the
    one-at-a-time draws are the batch's first draws, so the per-draw iterations compare directly."""
    import torch
    from rumb import RUM
    from rumb import bootstrap as BS
    from rumb.instances import config_instance
    n, m, a, p, panel = config_instance("n20_d1pct_panel520")
    rum = RUM(m, a, p, num_alternatives=n)
    boot = rum.bootstrap(panel=panel, B=batch_draws, weights="multinomial", seed=0, method="bm_admm",
                         method_args={"dtype": "float64"})
    boot._certify()
    idx = np.arange(batch_draws)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    boot.solve_draws(idx, stops=False)
    torch.cuda.synchronize()
    tb = time.perf_counter() - t0
    P = BS.perturb(boot.p_hat, boot.draws.rows(np.arange(single_draws)), boot.r_n, boot.eps_n)
    its = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for j in range(single_draws):
        r = boot.session.solve(P[j], abs_tol=boot.abs_tol, rel_tol=0.0, warm=True, max_time=600.0)
        its.append(int(r.iterations))
    torch.cuda.synchronize()
    ts = time.perf_counter() - t0
    # the screen of 10,000 draws of this panel (rows, perturbation, ||P_b - p_fit|| and ||p_b - p_hat||):
    # on the GPU over all draws, and the host builder (rumb.draws, block by block) on a sample
    from rumb import _lib
    from rumb.rum_solver import context
    D = BS.Draws(panel, m, a, p, B=10000, weights="multinomial", seed=0)
    r_n, eps_n, _ = BS.scaling(D.R)
    fit = boot.session.fit
    gd = _lib.DrawRows(context(), D.W, D.lists, D.p_hat)
    gd.screen(fit, eps_n * r_n)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    gd.screen(fit, eps_n * r_n)
    torch.cuda.synchronize()
    t_gpu = time.perf_counter() - t0
    sample = 512
    t0 = time.perf_counter()
    for lo in range(0, sample, 256):
        rows = D.rows(np.arange(lo, lo + 256))
        P = BS.perturb(D.p_hat, rows, r_n, eps_n)
        np.sqrt(np.einsum("ij,ij->i", P - fit, P - fit))
        np.sqrt(np.einsum("ij,ij->i", rows - D.p_hat, rows - D.p_hat))
    t_host = (time.perf_counter() - t0) * D.B / sample
    gd.close()
    screen = {"draws": D.B, "rows": D.M, "gpu_s": t_gpu, "host_s": t_host, "host_sample_draws": sample,
              "host_threads": 1}
    return {"metric": "n=20 bootstrap draws/s at abs gap 5e-4 (batched vs one at a time)",
            "value": batch_draws / tb, "unit": "draws/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "n20_d1pct_panel520", "batch_draws": batch_draws, "abs_tol": boot.abs_tol,
                       "slots": boot.last_batch["slots"], "iters_batched": boot.iters[idx].tolist()},
            "one_at_a_time": {"value": single_draws / ts, "unit": "draws/s", "draws": single_draws,
                              "iters": its},
            "ratio_batched_over_one_at_a_time": (batch_draws / tb) / (single_draws / ts),
            "target": "5x (batched float32 + learned warm start against one-at-a-time float64); not met: float32 "
                      "cannot certify abs 5e-4 on these distances (about 110) and one draw's kernels already "
                      "fill the GPU at n = 20",
            "screen": screen}


# published RTX 5090 figures for the paper instances (the reference's records)
PAPER = {
    "bm_admm_n20_d1pct": {"seconds": 45.09, "iterations": 7800, "bracket": [18.603539524, 18.621794959],
                          "record": "replication/feasibility_in_density/results/cert_bm_admm_n20_d1pct.json"},
    "flow_cg_n18_d1pct": {"seconds": 15.86, "columns": 848, "record": "data/opt_refs.json (key n18_d1pct)"},
}


# the reference's published large-n pricing times (RTX 5090, pairwise instances):
# solver/flow_cg/MEMORY.md:61 (mask sweep) and :67-69 (one column at n = 32)
LARGE_N_PUBLISHED = {"mask_sweep_ms": {20: 0.4, 28: 39.0, 30: 170.0},
                     "column_s_n32": {"mask": 0.70, "f32": 0.70, "u16": 0.72},
                     "column_s_n33": {"f32": 1.62, "u16": 1.72}}


PRICING_LARGE = ((20, ("mask", "f32", "f32_stream", "u16")), (28, ("mask", "f32", "f32_stream", "u16")),
                 (30, ("mask", "f32", "f32_stream", "u16")), (32, ("mask", "f32", "f32_stream", "u16")),
                 (33, ("mask", "f32")))


def run_pricing_large(args, rank, sweeps=3):
    """Workload pricing_large: one pricing call (sweep, backtrace or readout, read-back) on the
    reference's pairwise instances at n = 20 to 33, in mask storage (the tile sweep: 5 * 2^n bytes,
    20 GiB at n = 32, 40 GiB at n = 33), float32 storage (by mask where it fits, the same bits),
    float32 forced to two rank-indexed layers (f32_stream) and uint16 storage (rows scanned per
    subset above n = 26, where the cover lists are not built), seeded float32 scores; beside the
    reference's published RTX 5090 times for the same instances. --pricing-n / --pricing-modes
    restrict the list (one small case for a profiler)."""
    if rank != 0:
        return
    import torch
    from rumb import _lib, flow_cg
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import paper_instances as PI
    sys.path.insert(0, os.path.join(ROOT, "baseline"))
    import ref_replay
    ctx = _lib.Context(0)
    out = {}
    only_n = {int(v) for v in args.pricing_n.split(",")} if args.pricing_n else None
    only_modes = set(args.pricing_modes.split(",")) if args.pricing_modes else None
    for n, modes in PRICING_LARGE:
        if only_n is not None and n not in only_n:
            continue
        modes = [m for m in modes if only_modes is None or m in only_modes]
        cd, _ = PI.gen_pairwise(n)
        menus, alts, p32, offsets, _ = flow_cg.prepare_choice_data(cd[:, 0], cd[:, 1], cd[:, 2], n)
        scores = np.random.default_rng(n).standard_normal(menus.size).astype(np.float32)
        row = {}
        for mode in modes:
            pr = _lib.Pricer(ctx, n, menus, offsets, mode="f32" if mode == "f32_stream" else mode,
                             stream=mode == "f32_stream")
            pr.price(scores)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(sweeps):
                pr.price(scores)
            torch.cuda.synchronize()
            row[mode + "_ms"] = 1e3 * (time.perf_counter() - t0) / sweeps
            pr.close()
        if n <= 28 and ref_replay.available():
            # the reference's own layer kernels on the same B200 and scores (launches only)
            ref = ref_replay.time_pricing(menus, offsets, scores, n, reps=2)
            row["reference_kernels_ms"] = {"u24": ref["u24_layers_ms"], "u16": ref["u16_layers_ms"],
                                           "mask": ref["mask_layers_ms"]}
        out["n%d" % n] = row
    ctx.close()
    print(json.dumps({"metric": "Flow-CG pricing call at large n (pairwise), ms", "unit": "ms", "n_gpus": 1,
                      "higher_is_better": False, "data": "the reference's pairwise instances (regenerated)",
                      "runs": out, "reference_rtx5090": LARGE_N_PUBLISHED}), flush=True)


def run_learned_n10(args, rank):
    """Workload learned_n10: the learned warm start at shapes whose distances are large against the
    network's error (n = 10 panels of 200 respondents x 20 menus and 120 x 30, K = 8 / 6): 128
    draws, the first 96 train the network, the last 32 are solved to abs 5e-4 seeded by it (lower
    bound at the prediction and, with y0_state, the start state's fitted cells) and without it;
    reports the Frank-Wolfe bound at the prediction against the one at p_hat's fit, iterations
    both ways and the draws' decisions against the band."""
    if rank != 0:
        return
    from rumb import RUM
    from rumb import bootstrap as BS
    from rumb.instances import panel_instance
    from rumb.rum_solver import context
    runs = []
    for (dens, resp, per, K, seed) in ((0.5, 200, 20, 8, 3), (1.0, 120, 30, 6, 4)):
        panel, (m, a, p) = panel_instance(10, dens, resp, per, K, seed=seed)
        rum = RUM(m, a, p, num_alternatives=10)
        ntr, nte = 96, 32
        kw = dict(panel=panel, B=ntr + nte, weights="multinomial", seed=0, method="bm_admm",
                  method_args={"dtype": "float64"})
        row = {"rows": int(p.size)}
        for y0_state in (False, True):
            boot = rum.bootstrap(learned=True, train_draws=ntr, mlp_epochs=300, y0_state=y0_state, **kw)
            plain = rum.bootstrap(**kw)
            for b in (boot, plain):
                b._certify()
            idx = np.arange(ntr + nte)
            boot.solve_draws(idx, stops=False)
            plain.solve_draws(idx, stops=False)
            te = idx[ntr:]
            g, ctx = rum._geom, context()
            P = BS.perturb(boot.p_hat, boot.draws.rows(te), boot.r_n, boot.eps_n)
            yp = boot.predict_fit(P)
            lb_net = [ctx.fw_lb64(10, g.menu, g.alternative, yp[j], P[j]) for j in range(nte)]
            lb_hat = [ctx.fw_lb64(10, g.menu, g.alternative, boot.session.fit, P[j]) for j in range(nte)]
            dec = BS.decide(boot.L[te], boot.U[te], *boot.tau)
            row["y0_state" if y0_state else "lb_seed"] = dict(
                iters_learned=int(boot.iters[te].sum()), iters_plain=int(plain.iters[te].sum()),
                lb_at_prediction_median=float(np.median(lb_net)), lb_at_p_hat_fit_median=float(np.median(lb_hat)))
        row.update(p_hat_bracket=[boot.L0, boot.U0], band=list(boot.tau),
                   distance_min_median_max=[float(np.min(plain.U[te])), float(np.median(plain.U[te])),
                                            float(np.max(plain.U[te]))],
                   decided_below_above_open=[int((dec == BS.BELOW).sum()), int((dec == BS.ABOVE).sum()),
                                             int((dec == BS.UNDECIDED).sum())])
        runs.append(row)
    print(json.dumps({"metric": "learned warm start at n = 10 panels: iterations of 32 seeded draws against plain",
                      "unit": "iterations", "n_gpus": 1, "data": "synthetic", "runs": runs}), flush=True)


def run_dsr_n25(args, rank, seconds=90.0):
    """Workload dsr_n25 (n25_dsr301_panel520: n = 25, alternative 0 observed on 301 menus, a
    520-respondent panel, K = 40; the learned warm start's configuration): p_hat's own certified
    solve to abs 5e-4, bounded by `seconds` per state dtype, from the cold start. It measures what a
    bootstrap at this shape must first do once -- certify p_hat -- and what one iteration costs
    (8 slabs of 2^24 x 25 values), the reference's record being that its bm_admm did not certify
    this shape in 4 hours (replication/empirical_dsr_n25/README.md:57-58)."""
    if rank != 0:
        return
    import torch
    from rumb import _lib
    from rumb.instances import config_instance
    n, m, a, p, _panel = config_instance("n25_dsr301_panel520")
    ctx = _lib.Context(0)
    beta = beta_rule(p.size)
    prob = ctx.bm_problem(n, m.astype(np.uint32), a.astype(np.int32), p)
    out = {}
    for dt in ("float32", "float64"):
        par = ctx.bm_params(beta, check=CHECK, abs_tol=5e-4, rel_tol=None, dtype=dt, max_iter=10 ** 7,
                            time_limit=seconds, stall_checks=0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r, _, _ = ctx.bm_solve(prob, par, want_fit=False)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        out[dt] = {"seconds": wall, "iters": int(r["iters"]), "ms_per_iter": 1e3 * r["solve_s"] / max(1, r["iters"]),
                   "lb": r["lb"], "ub": r["ub"], "gap": r["ub"] - r["lb"], "stop": r["stop_reason"],
                   "setup_s": r["setup_s"]}
    ctx.close()
    print(json.dumps({"metric": "n=25 DSR p_hat certified solve, bounded (abs 5e-4)", "unit": "s", "n_gpus": 1,
                      "data": "synthetic", "config": {"workload": "n25_dsr301_panel520", "cells": int(p.size),
                                                      "time_box_s": seconds, "abs_tol": 5e-4},
                      "runs": out}), flush=True)


def run_paper(args, rank):
    """Workload paper: the reference's certified runs on two of its paper instances, regenerated
    from its generator (sha256 fingerprints checked): BM-ADMM on n20_d1pct (104,885 cells) in
    float64, rel 1e-3, bounds every 200 iterations; Flow-CG on n18_d1pct (23,568 cells), rel 1e-3.
    Prints the library's times beside the reference's published RTX 5090 times (its records)."""
    if rank != 0:
        return
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import paper_instances as PI
    from rumb import RUM
    out = {}
    for key, n, cat, method, margs in (("bm_admm_n20_d1pct", 20, "d1pct", "bm_admm", {"dtype": "float64", "check": 200}),
                                      ("flow_cg_n18_d1pct", 18, "d1pct", "flow_cg", None)):
        cd, mp = PI.get_instance(n, cat)
        rum = RUM(cd[:, 0].astype(np.int64), cd[:, 1].astype(np.int64), cd[:, 2], num_alternatives=n)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = rum.calculate_distance(method=method, method_args=margs, abs_tol=0.0, rel_tol=1e-3, max_time=600)
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
        out[key] = {"seconds": sec, "lb": r.lb, "ub": r.ub, "iterations": r.iterations, "unit": r.iteration_unit,
                    "status": r.status, "cells": int(mp), "fingerprint": PI.fingerprint(cd),
                    "reference_rtx5090": PAPER[key], "speedup_vs_published": PAPER[key]["seconds"] / sec}
    line = {"metric": "paper instances: certified solve seconds (rel 1e-3)", "value": out["bm_admm_n20_d1pct"]["seconds"],
            "unit": "s", "higher_is_better": False, "n_gpus": 1, "data": "the reference's paper instances (regenerated)",
            "runs": out}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--dtype", default="float64", choices=["float64", "mixed", "float32"])
    ap.add_argument("--impl", default="rumb", choices=["rumb", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--no-bootstrap", action="store_true", help="skip the bootstrap leg of the bench line")
    ap.add_argument("--pricing-n", default="", help="pricing_large: comma-separated n to run (default all)")
    ap.add_argument("--pricing-modes", default="", help="pricing_large: comma-separated storages to run")
    ap.add_argument("--workload", default="bm_n18", choices=["bm_n18", "bootstrap_n20", "paper", "pricing", "pricing_large", "dsr_n25",
                             "learned_n10"],
                    help="bootstrap_n20: the batched-draw comparison; paper: the reference's certified runs on "
                         "its paper instances beside its published times (each prints its own line)")
    ap.add_argument("--profile-case", type=int, default=0, metavar="ITERS",
                    help="run one solve capped at ITERS iterations (for ncu) and print no bench line")
    args = ap.parse_args()
    rank, world, local = _env_int("RANK", 0), _env_int("WORLD_SIZE", 1), _env_int("LOCAL_RANK", 0)

    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "bootstrap_n20":
        run_bootstrap(args, rank)
        return
    if args.workload == "paper":
        run_paper(args, rank)
        return
    if args.workload == "pricing":
        run_pricing(args, rank)
        return
    if args.workload == "dsr_n25":
        run_dsr_n25(args, rank)
        return
    if args.workload == "learned_n10":
        run_learned_n10(args, rank)
        return
    if args.workload == "pricing_large":
        run_pricing_large(args, rank)
        return

    import torch
    import torch.distributed as dist
    from rumb import _lib

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    n, menu, alt, p = instance()
    mp = p.size
    beta = beta_rule(mp)
    ctx = _lib.Context(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    d_menu = torch.from_numpy(menu.view(np.int32)).cuda()
    d_alt = torch.from_numpy(alt).cuda()
    d_p = torch.from_numpy(p).cuda()
    prob_dev = _lib.BMProblem(n, mp, d_menu.data_ptr(), d_alt.data_ptr(), d_p.data_ptr(), 1)
    prob_host = ctx.bm_problem(n, menu, alt, p)
    # checks overlapped with the next interval (rumb_bm_params.overlap_check): the same certified
    # bracket, reached one interval (50 iterations) later, with the float64 check off the critical path
    par = ctx.bm_params(beta, check=CHECK, abs_tol=ABS_TOL, rel_tol=None, dtype=args.dtype, max_iter=10 ** 7,
                        time_limit=600, overlap_check=True)
    if args.profile_case > 0:
        par.max_iter = args.profile_case
        r, _, _ = ctx.bm_solve((prob_dev, None), par, want_fit=False)
        torch.cuda.synchronize()
        print("profile case: %d iterations, %d kernel launches, stop %s" % (r["iters"], r["launches"],
                                                                           r["stop_reason"]))
        return
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")       # > 126 MB of L2

    def solve(dev):
        if dev:
            r, _, _ = ctx.bm_solve((prob_dev, None), par, want_fit=False)
        else:
            r, _, _ = ctx.bm_solve(prob_host, par, want_fit=True)
        return r

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(dev, k):
        ms, res = [], None
        timed.launches = 0
        for _ in range(k):
            with torch.cuda.stream(stream):
                flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            res = solve(dev)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            timed.launches += int(res["launches"])
        return ms, res

    for _ in range(args.warmup):
        last = solve(True)
    barrier()
    with ClockSampler(local) as clk:
        ms_dev, res = timed(True, args.steps)
        launches_dev = timed.launches
        barrier()
    clocks = clk.summary()
    barrier()
    ms_e2e, res_e2e = timed(False, args.steps)
    barrier()
    step_ms = sum(ms_dev) / len(ms_dev)
    e2e_ms = sum(ms_e2e) / len(ms_e2e)
    if world > 1:
        t = torch.tensor([step_ms, e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_ms, e2e_ms = float(t[0]), float(t[1])

    # the same solve with a float32 state until its bracket stalls, float64 to the end (informative;
    # `value` stays the float64 state), timed the same way on rank 0
    mixed = None
    if rank == 0 and args.dtype == "float64":
        par_m = ctx.bm_params(beta, check=CHECK, abs_tol=ABS_TOL, rel_tol=None, dtype="mixed", max_iter=10 ** 7,
                              time_limit=600, overlap_check=True)
        for _ in range(2):
            ctx.bm_solve((prob_dev, None), par_m, want_fit=False)
        ms_m, res_m = [], None
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            res_m, _, _ = ctx.bm_solve((prob_dev, None), par_m, want_fit=False)
            e1.record(stream)
            e1.synchronize()
            ms_m.append(e0.elapsed_time(e1))
        mixed = {"solves_per_s": 1e3 / (sum(ms_m) / len(ms_m)), "ms_per_step": sum(ms_m) / len(ms_m),
                 "iters_per_solve": int(res_m["iters"]), "iters_float32": int(res_m["iters_f32"]),
                 "ub": res_m["ub"], "lb": res_m["lb"], "stop": res_m["stop_reason"]}

    # roofline of the dominant kernel: 20 iterations and one check after PROFILE_WARMUP iterations,
    # captured as a CUDA graph with CUDA events around every kernel and replayed (rumb_bm_profile)
    prof = ctx.bm_profile((prob_dev, None), par, iters=20, warmup=PROFILE_WARMUP)
    top = max(prof, key=lambda k: k["total_ms"])
    tot = sum(k["total_ms"] for k in prof)
    per_launch_ms = top["total_ms"] / top["launches"]
    if not per_launch_ms > 0:
        raise RuntimeError("the kernel profile timed nothing: %s" % prof)
    peak, peak_kind = load_peaks()
    achieved = top["bytes_per_launch"] / (per_launch_ms * 1e-3) / 1e9
    traffic, traffic_src = kernel_traffic(top["name"])
    # the reference's own float64 kernels on the same workload and GPU (rank 0, after the timing)
    ref_leg = None
    if rank == 0:
        try:
            ref_leg = reference_kernels_leg(n, menu, alt, p, beta)
        except Exception as e:
            ref_leg = {"unavailable": str(e).splitlines()[0][:200]}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    with torch.cuda.stream(stream):
        pricing = pricing_sweeps(ctx, stream)
    cpu = None
    if not args.no_cpu:
        v, desc, used = cpu_sample(n, menu, alt, p, 1, int(res["iters"]), int(res["n_push"]), sample_iters=40)
        cpu = {"value": v, "unit": "solves/s", "cores": used, "kind": "port", "sample": desc}
    boot = None
    if not args.no_bootstrap:
        try:
            boot = bootstrap_leg(4, 2)
        except Exception as e:
            boot = {"unavailable": str(e).splitlines()[0][:200]}
    value = world * 1e3 / step_ms
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"float64": "f64", "mixed": "f32+f64", "float32": "f32"}[args.dtype],
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": n, "cells": int(mp), "menus": int(np.unique(menu).size),
                   "abs_tol": ABS_TOL, "rel_tol": None, "check": CHECK, "beta": beta,
                   "iters_per_solve": int(res["iters"]), "iters_float32": int(res["iters_f32"]),
                   "checks_per_solve": int(res["n_push"]),
                   "ub": res["ub"], "lb": res["lb"], "state_dtype": args.dtype,
                   "l2": "flushed (256 MB write) before every timed solve; state slabs exceed L2",
                   "check_overlap": True,
                   "parallelism": "replicas x%d" % world},
        "e2e": {"value": world * 1e3 / e2e_ms, "unit": "solves/s", "h2d_bytes_per_step": int(mp * 16),
                "d2h_bytes_per_step": int(mp * 8 + 64 * res_e2e["n_push"] + 104)},
        "roofline": {"bound": "hbm", "kernel": top["name"], "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "share": top["total_ms"] / tot if tot > 0 else None,
                     "bytes_per_launch": top["bytes_per_launch"], "launch_ms": per_launch_ms,
                     "timing": ("CUDA events around each kernel inside the replayed CUDA graph" if top.get("graph")
                                else "CUDA events around eager launches"),
                     "traffic": traffic, "traffic_source": traffic_src,
                     "source_sha256": source_digest(top["name"])},
        # one iteration's kernels under graph replay (the check's plain transforms left out)
        "iteration_ms": sum(k["total_ms"] for k in prof if ",plain>" not in k["name"]) / 20.0,
        "reference_kernels": ref_leg,
        "mixed_state": dict(mixed, speedup_vs_reference_kernels=(mixed["solves_per_s"] * ref_leg["s_per_solve"]
                                                                 if ref_leg and "s_per_solve" in ref_leg else None))
        if mixed else None,
        "speedup_vs_reference_kernels": (value * ref_leg["s_per_solve"]
                                         if ref_leg and "s_per_solve" in ref_leg else None),
        "kernels": [{"name": k["name"], "share": round(k["total_ms"] / tot, 4),
                     "us_per_launch": round(1e3 * k["total_ms"] / k["launches"], 2),
                     "gbs": round(k["bytes_per_launch"] / (k["total_ms"] / k["launches"] * 1e-3) / 1e9, 1)}
                    for k in sorted(prof, key=lambda k: -k["total_ms"])[:8]],
        "gpu_launches": int(launches_dev),
        "cpu_baseline": cpu,
        "flow_cg_pricing": pricing,
        "bootstrap": boot,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
