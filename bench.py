"""Benchmark of the linking-number hot path on B200.

One step = the certificate's linking-number stage over every potential loop
pair of the workload: tree build + Barnes–Hut traversal (+ beta retry, margin
check and FP64 recompute) with the discretized polylines already in HBM.
Metric: certificate ms and segment-pair throughput, Gsegpair/s =
sum over pairs of n_i * n_j (post-Discretize segment counts, the
direct-sum-equivalent work) / step time; the same numerator for every method.

Default workload: random closed polymer loops, 200 loops x 50,000 Gaussian
steps (10M segments), centres uniform in a cube of side 400, quadrupole BH,
beta = 2 — seeded synthetic data. N > 1 (torchrun): every rank runs its own
seeded instance (weak scaling, no data-path collective); the time is the max
over ranks.

--impl reference times the reference's CPU algorithm (the oracle port, the
reference itself cannot be built here) on the host cores with all threads,
each step a seeded sample of the same workload's pairs.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "certificate ms & Gsegpair/s (exact certs): mixed+learned BH vs plain FP64 GPU"
UNIT = "Gsegpair/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
# Algorithmic bytes per evaluated Barnes–Hut node pair: two FP32 node records
# of the reference-minimal layout (c_M 3 + C_D 9 + C_Q 27 + centre 3 + radius
# 1 + 3 norms = 46 values x 4 B = 184 B each).
BH_BYTES_PER_NODE_PAIR = 2 * 184
# Per node pair the traversal hands to the exact list: the two centres and
# radii it classified (2 x (3 + 1) x 8 B).
BH_BYTES_PER_EXACT_ENTRY = 2 * 32


def _peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return PEAKS_FALLBACK, "fallback"


def _workload_curves(name: str, seed: int, loops: int, steps: int):
    """The seeded curves of a workload (numpy only: loads no native library)."""
    from fastlinkingnumbers_b200 import workloads as W
    if name == "polymer" and (loops, steps) != (200, 50000):
        off, xyz = W.polymer(seed=seed, n_loops=loops, n_steps=steps)
        desc = (f"polymer loops: {loops} x {steps}-step closed Gaussian walks "
                f"({loops * steps / 1e6:g}M segments), cube 400")
    else:
        off, xyz, desc = W.named(name, seed)
    cfg = {"workload": desc, "loops": int(len(off) - 1)}
    if name == "polymer":
        cfg["steps_per_loop"] = steps
    cfg.update({"method": "barneshut (quadrupole, beta 2, beta_limit 10)", "seed": seed,
                "l2": "inputs and per-step trees larger than L2 (no flush needed)"})
    return off, xyz, cfg


def make_workload(name: str, seed: int, loops: int = 200, steps: int = 50000, engine=None):
    from fastlinkingnumbers_b200 import Model
    off, xyz, cfg = _workload_curves(name, seed, loops, steps)
    m = Model().SetCurves(3, -np.diff(off).astype(np.int32), xyz)
    t0 = time.perf_counter()
    poff, pxyz, pairs, rounds = m.Prepare(True, engine=engine)
    cfg["prepare_ms"] = round(1e3 * (time.perf_counter() - t0), 1)
    cfg["_raw"] = (off, xyz)  # the curves before Discretize (popped before printing)
    cfg["prepare_on"] = "host" if engine is None else "gpu"
    cfg["discretize_rounds"] = int(rounds)
    cfg["segments_after_discretize"] = int(poff[-1])
    cfg["pairs"] = int(len(pairs))
    return poff, pxyz, pairs, cfg


def certificate_text(ncurves: int, pairs, lk) -> str:
    """The certificate file of a set of linking numbers, as the library writes
    it (src/linking_number_certificate.cpp:294-322): the curve count, then
    "i,j,lk" for every pair whose rounded value is not 0, i < j, sorted."""
    r = np.round(np.asarray(lk, dtype=np.float64))
    keep = ~(np.abs(r) < 0.25)
    ij = np.sort(np.asarray(pairs, dtype=np.int64)[keep], axis=1)
    rows = sorted(zip(ij[:, 0].tolist(), ij[:, 1].tolist(), r[keep].astype(np.int64).tolist()))
    return f"{ncurves}\n" + "".join(f"{i},{j},{v}\n" for i, j, v in rows)


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region.

    nvidia-smi is started before the warm-up steps (its start-up competes with
    the process's own driver calls), and only the samples whose timestamps
    fall between mark() and stop() are kept (all of them if none does)."""

    def __init__(self, index: int, interval_ms: int = 200):
        self.path = tempfile.mktemp(suffix=".csv")
        self.t0 = None
        q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", str(interval_ms)],
                                      stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def mark(self):
        """The timed region starts now."""
        self.t0 = datetime.datetime.now()

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        t1 = datetime.datetime.now()
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                sm_mhz, max_mhz = float(parts[2]), float(parts[3])
            except ValueError:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f")
            except ValueError:
                ts = None
            rows.append((ts, sm_mhz, max_mhz, [k for k, v in zip(names, parts[6:10]) if v.lower() == "active"]))
        os.unlink(self.path)
        inside = [r for r in rows if self.t0 is not None and r[0] is not None and self.t0 <= r[0] <= t1]
        use = inside or rows
        sm = [r[1] for r in use]
        mx = [r[2] for r in use]
        reasons = sorted({k for r in use for k in r[3]})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(sm), "samples_in_timed_region": len(inside)}


def cpu_sample_run(poff, pxyz, pairs, target_s: float, seed: int, nthreads: int, oracle=None):
    """Times the oracle (the reference's CPU algorithm: loop-pair parallel,
    serial depth-first Barnes–Hut with the beta retry; built -O3
    -march=native like the reference) on a seeded sample of pairs sized for
    about target_s seconds; returns (Gsegpair/s, info)."""
    from oracle import pyoracle
    o = oracle if oracle is not None else pyoracle.Oracle(native=True).set_polylines(poff, pxyz)
    rng = np.random.default_rng(seed)
    order = rng.permutation(len(pairs))
    n = np.diff(poff).astype(np.float64)
    done, t_total, work, k = 0, 0.0, 0.0, max(nthreads, 1)
    while done < len(order):
        sel = pairs[order[done:done + k]]
        t0 = time.perf_counter()
        o.eval_pairs(pyoracle.BARNES_HUT, sel, bh_parallel=False, nthreads=nthreads)
        dt = time.perf_counter() - t0
        t_total += dt
        work += float(np.sum(n[sel[:, 0]] * n[sel[:, 1]]))
        done += len(sel)
        if t_total >= target_s:
            break
        k = int(max(nthreads, min(4 * k, len(sel) * max(1.0, (target_s - t_total) / max(dt, 1e-3)))))
    return work / t_total / 1e9, {"pairs": done, "seconds": round(t_total, 2), "segment_pairs": work}


def run_reference(args, rank):
    """The reference's CPU path, restated by the oracle, end to end on the
    host: the oracle generates nothing itself, so the seeded curves come from
    the workload generator (numpy); the oracle then runs the reference's
    potential-link search and Discretize, and each step times its Barnes-Hut
    over a seeded sample of the pairs. No product library is loaded."""
    if rank != 0:
        return
    from oracle import pyoracle
    off, xyz, cfg = _workload_curves(args.workload, args.seed, args.loops, args.loop_steps)
    o = pyoracle.Oracle(native=True).set_curves(pyoracle.SEG_POLYLINE, -np.diff(off).astype(np.int32), xyz)
    del xyz
    t0 = time.perf_counter()
    o.prepare(True)
    cfg["prepare_ms"] = round(1e3 * (time.perf_counter() - t0), 1)
    cfg["prepare_on"] = "host (oracle)"
    cfg["discretize_rounds"] = int(o.rounds)
    poff, pxyz = o.polylines()
    pairs = o.pairs()
    cfg["segments_after_discretize"] = int(poff[-1])
    cfg["pairs"] = int(len(pairs))
    threads = pyoracle.max_threads(native=True)
    # Each step is a bounded sample, sized so that the whole run stays within
    # about four minutes.
    per_step = min(args.cpu_seconds, max(3.0, 240.0 / max(1, args.steps + args.warmup)))
    vals = []
    for s in range(args.warmup + args.steps):
        v, info = cpu_sample_run(poff, pxyz, pairs, per_step, args.seed + 17, threads, oracle=o)
        if s >= args.warmup:
            vals.append((v, info))
    v = float(np.mean([x[0] for x in vals]))
    info = vals[-1][1]
    sample = (f"{info['pairs']} seeded random pairs of {len(pairs)} ({info['segment_pairs']:.3g} "
              f"segment pairs, {info['seconds']} s) per step, Barnes-Hut beta 2 with retry, oracle port of "
              f"the reference built -O3 -march=native")
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * float(np.mean([x[1]["seconds"] for x in vals])), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": dict(cfg, parallelism=f"replicas x{args.gpus}"),
        "impl_details": {"method": "barneshut", "precision": "f64",
                         "tree": "reference kd-median", "traversal": "serial depth-first per pair",
                         "prepare": "oracle potential-link search + Discretize (host)"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from fastlinkingnumbers_b200 import Engine, _native as N

    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    stream = torch.cuda.current_stream()
    eng = Engine(local_rank, stream.cuda_stream)
    poff, pxyz, pairs, cfg = make_workload(args.workload, args.seed + rank, args.loops, args.loop_steps, engine=eng)
    raw_curves = cfg.pop("_raw")
    prm = N.default_params(precision=N.PREC_MIXED if args.precision == "mixed" else N.PREC_FP64,
                           bh_tree=args.bh_tree, bh_schedule=args.bh_schedule, bh_bucket=args.bh_bucket)
    tune = None
    if args.bh_occupancy:
        prm.bh_occupancy = args.bh_occupancy
    if args.fp64_margin is not None:
        prm.fp64_margin = args.fp64_margin
    if args.bh_budget:
        prm.bh_budget = args.bh_budget
    elif args.autotune and args.method == "barneshut":
        # Round budget only: the same node pairs, so results change only in the
        # rounding of partial sums (beta stays the reference's 2). Tuned on a
        # seeded sample of the pairs, untimed.
        prm, tune = eng.autotune(pxyz, poff, pairs, tune_beta=False, sample_pairs=2048, params=prm,
                                 tune_bucket=bool(args.autotune_bucket) and not args.bh_bucket)
    d_xyz = torch.from_numpy(pxyz).cuda()
    d_off = torch.from_numpy(poff).cuda()
    d_pairs = torch.from_numpy(pairs).cuda()
    npairs = len(pairs)
    d_lk = torch.zeros(npairs, dtype=torch.float64, device="cuda")
    d_err = torch.zeros(npairs, dtype=torch.float64, device="cuda")
    d_flags = torch.zeros(npairs, dtype=torch.int32, device="cuda")
    n = np.diff(poff).astype(np.float64)
    units = float(np.sum(n[pairs[:, 0]] * n[pairs[:, 1]]))

    def step():
        eng.linking_numbers_device(d_xyz.data_ptr(), d_off.data_ptr(), len(poff) - 1,
                                   d_pairs.data_ptr(), npairs, d_lk.data_ptr(), d_err.data_ptr(),
                                   d_flags.data_ptr(), method=args.method, params=prm)
        return eng.stats()

    clocks = ClockSampler(local_rank, args.clock_interval_ms)
    for w in range(args.warmup):
        t0 = time.perf_counter()
        s = step()
        print(f"[bench] warmup {w}: {1e3 * (time.perf_counter() - t0):.1f} ms wall, main kernel "
              f"{s['ms_main_kernel']:.1f} ms, tree {s['ms_tree_build']:.1f} ms, far {s['bh_far_evals']:.3g}, "
              f"leaf {s['bh_leaf_evals']:.3g}, retried {s['beta_retried']}, escalated {s['bh_escalated']}, "
              f"fp64 {s['fp64_recomputed']}, launches {s['kernel_launches']}, timeouts {s['bh_wait_timeouts']}",
              file=sys.stderr, flush=True)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    clocks.mark()
    ev0.record(stream)
    st = []
    for _ in range(args.steps):
        st.append(step())
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    lk = d_lk.cpu().numpy()
    flags = d_flags.cpu().numpy()
    value = world * units / (ms * 1e-3) / 1e9
    # One untimed step with each round's exact list after its traversal on one
    # stream (bh_exact_serial; the same results bit for bit): each kernel's
    # own CUDA-event time, which the overlapped timed steps cannot give.
    alone = None
    if args.method == "barneshut" and args.bh_schedule == 0:
        prm_serial = type(prm).from_buffer_copy(prm)
        prm_serial.bh_exact_serial = 1
        eng.linking_numbers_device(d_xyz.data_ptr(), d_off.data_ptr(), len(poff) - 1, d_pairs.data_ptr(), npairs,
                                   d_lk.data_ptr(), d_err.data_ptr(), d_flags.data_ptr(), method=args.method,
                                   params=prm_serial)
        alone = eng.stats()
        assert np.array_equal(d_lk.cpu().numpy(), lk), "the serial exact list changed the sums"

    # End to end through the host-array entry point: H2D of the polylines and
    # pairs, the whole stage, D2H of the per-pair results, every step.
    h_xyz = torch.from_numpy(pxyz).pin_memory().numpy()
    h_off = torch.from_numpy(poff).pin_memory().numpy()
    h_pairs = torch.from_numpy(pairs).pin_memory().numpy()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        elk, _, _ = eng.linking_numbers(h_xyz, h_off, h_pairs, args.method, params=prm)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    assert np.array_equal(np.round(elk), np.round(lk)), "host and device entry points disagree"

    s_last = st[-1]
    peaks, peak_kind = _peaks()
    main_ms = float(np.mean([s["ms_main_kernel"] for s in st]))
    if args.method == "barneshut":
        # The dominant kernel is the traversal (bh_traverse); the exact-list
        # kernel (bh_buckets) is timed separately by the library.
        exact_ms = float(np.mean([s["ms_exact"] for s in st]))
        # The traversal launches are timed by their own events (the exact list
        # runs beside them on a second stream, so main - exact understates them).
        trav_ms = float(np.mean([s["ms_traverse"] for s in st]))
        if trav_ms <= 0:
            trav_ms = main_ms - exact_ms
        far = float(np.mean([s["bh_far_evals"] for s in st]))
        ent = float(np.mean([s["bh_exact_entries"] for s in st]))
        seg_exact = float(np.mean([s["bh_leaf_evals"] for s in st]))
        node_pairs = far + ent
        alg = BH_BYTES_PER_NODE_PAIR * far + BH_BYTES_PER_EXACT_ENTRY * ent
        sm_ghz = (clk.get("sm_mhz") or 1965.0) / 1e3
        fp32_bound = 148 * 128 * sm_ghz / 45.0  # G segment pairs / s
        achieved = alg / (trav_ms * 1e-3) / 1e9
        traffic = args.traffic_bytes_per_node_pair * node_pairs if args.traffic_bytes_per_node_pair else None
        dram_gbs = traffic / (trav_ms * 1e-3) / 1e9 if traffic else None
        roof = {"bound": "hbm", "kernel": "bh_traverse", "achieved": achieved,
                "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                "frac_basis": "algorithmic bytes (2 x 184 B per far node pair, 2 x 32 B per exact entry)",
                "peak_source": peak_kind, "traffic": traffic,
                "algorithmic_bytes_per_launch": alg, "far_node_pairs_per_step": far,
                "exact_node_pairs_per_step": ent, "ms_per_launch": trav_ms,
                "dram_gbs": dram_gbs, "dram_frac": dram_gbs / peaks["hbm_gbs"] if dram_gbs else None,
                "limiter": "L1 wavefronts and dependent-load latency (node records are re-read from L1/L2); "
                           "DRAM runs at dram_frac of the copy peak",
                "alone": None if alone is None else {
                    "note": "one untimed step with each exact list after its traversal on one stream",
                    "traversal_ms": alone["ms_traverse"],
                    "achieved": alg / (alone["ms_traverse"] * 1e-3) / 1e9,
                    "frac": alg / (alone["ms_traverse"] * 1e-3) / 1e9 / peaks["hbm_gbs"],
                    "exact_ms": alone["ms_exact"],
                    "exact_Gsegpair_per_s": seg_exact / (alone["ms_exact"] * 1e-3) / 1e9,
                    "passes_ms": alone["ms_main_kernel"]},
                "exact_kernel": {"kernel": "bh_buckets", "ms_per_step": exact_ms,
                                 "segment_pairs_per_step": seg_exact,
                                 "Gsegpair_per_s": seg_exact / (exact_ms * 1e-3) / 1e9 if exact_ms > 0 else None,
                                 "bound": "fp32 issue",
                                 "bound_Gsegpair_per_s": fp32_bound,
                                 "frac": (seg_exact / (exact_ms * 1e-3) / 1e9) / fp32_bound if exact_ms > 0 else None,
                                 "bound_note": "45 FP32 FMA-pipe ops + 2 MUFU per segment pair (the algorithmic "
                                               "count): 148 SMs x 128 lanes x SM clock / 45"},
                "note": ("per step (all traversal rounds, CUDA events around each launch): algorithmic "
                         "bytes = 2 x 184 B FP32 node record per far-field node pair + 2 x 32 B (centre, "
                         "radius) per node pair handed to the exact list; traffic = DRAM read+write per "
                         "node pair from the small-case ncu captures in "
                         "profiles/bh_traverse_bh_buckets_polymer_6M.md x node pairs; node records are "
                         "mostly re-read from L1/L2: the kernel is bound by L1 wavefronts and latency, not "
                         "by HBM. In the timed steps each round's exact list runs beside the next "
                         "traversal on a second stream, so a traversal launch's events include the time "
                         "the two kernels share the SMs; 'alone' times them one after the other")}
    else:
        roof = {"bound": "fp32-issue", "kernel": "direct_" + args.precision, "ms_per_launch": main_ms,
                "segment_pairs_per_s": units / (main_ms * 1e-3)}
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded)",
        "config": dict(cfg, parallelism=f"replicas x{world}"),
        "impl_details": {"method": args.method, "precision": args.precision,
                         "tree": "curve-order" if args.bh_tree == 0 else "reference kd-median",
                         "schedule": ["rounds, fused evaluation", "persistent queue", "rounds, split evaluation"][args.bh_schedule],
                         "exact_bucket_segments": 1 if (args.bh_tree == 1 or args.bh_schedule != 0)
                         else (prm.bh_bucket or 8),
                         "round_budget": prm.bh_budget or 256,
                         "traversal_ctas_per_sm": prm.bh_occupancy or 5},
        "certificate_ms": ms,
        "autotune": tune,
        "e2e": {"value": world * units / (e2e_ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(pxyz.nbytes + poff.nbytes + pairs.nbytes),
                "d2h_bytes_per_step": int(npairs * (8 + 8 + 4))},
        "gpu_launches": int(sum(s["kernel_launches"] for s in st)),
        "roofline": roof,
        "clocks": clk,
        "stats": {"pairs": npairs, "segment_pairs": units, "beta_retried": s_last["beta_retried"],
                  "retry_ms": s_last["ms_retry"], "front_records": s_last["bh_front_records"],
                  "front_pairs_kept_far": s_last["bh_far_reused"], "front_pairs_opened": s_last["bh_far_subtracted"],
                  "retry_from_roots": s_last["bh_retry_from_roots"], "rounds": s_last["bh_rounds"],
                  "escalated": s_last["bh_escalated"], "wait_timeouts": s_last["bh_wait_timeouts"],
                  "fp64_recomputed": s_last["fp64_recomputed"], "tree_build_ms": s_last["ms_tree_build"],
                  "far_evals": s_last["bh_far_evals"], "leaf_evals": s_last["bh_leaf_evals"],
                  "nonzero_links": int(np.sum(np.round(lk) != 0)), "flags_recomputed": int(np.sum(flags & 1))},
        # Each timed step as the library saw it: device time of the call
        # (events around it), of its Barnes-Hut passes, and host wall time.
        "timed_steps": {"call_ms": [round(s["ms_kernels"], 2) for s in st],
                        "passes_ms": [round(s["ms_main_kernel"], 2) for s in st],
                        "tree_ms": [round(s["ms_tree_build"], 2) for s in st],
                        "wall_ms": [round(s["ms_total"], 2) for s in st]},
    }
    fx = os.path.join(REPO, "tests", "golden", "configs", args.workload + ".npz")
    if args.method == "barneshut" and os.path.exists(fx) and rank == 0:
        # The FP64 direct-sum certificate of this workload (every pair), when
        # one was made for it: the integers must agree byte for byte.
        z = np.load(fx)
        meta = json.loads(str(z["meta"]))
        if meta["seed"] == args.seed and meta["pairs"] == npairs and (args.loops, args.loop_steps) == (200, 50000):
            from fastlinkingnumbers_b200 import workloads as W
            want = open(os.path.join(REPO, "tests", "golden", "configs", args.workload + ".txt")).read()
            result["fp64_certificate"] = {
                "certificate_equal": W.certificate_text(len(poff) - 1, pairs, lk) == want,
                "max_abs_dev_vs_fp64": float(np.abs(lk - z["lk"]).max()),
                "fp64_direct_kernel_s": meta.get("fp64_kernel_s")}
    if rank == 0 and world == 1 and args.direct_sample > 0:
        # Plain FP64 GPU direct sum and the mixed direct sum on a seeded sample
        # of pairs, extrapolated by segment pairs (the full FP64 direct sum of
        # this workload takes minutes).
        rng = np.random.default_rng(args.seed + 5)
        sel = pairs[rng.permutation(npairs)[:args.direct_sample]]
        w = float(np.sum(n[sel[:, 0]] * n[sel[:, 1]]))
        out = {}
        for prec, name in ((N.PREC_FP64, "fp64"), (N.PREC_MIXED, "mixed")):
            eng.linking_numbers(pxyz, poff, sel, "directsum", precision=prec)
            s = eng.stats()
            out[name] = {"sample_pairs": int(len(sel)), "kernel_ms": s["ms_main_kernel"],
                         "Gsegpair_per_s": w / (s["ms_main_kernel"] * 1e-3) / 1e9,
                         "extrapolated_certificate_ms": s["ms_main_kernel"] * units / w}
        result["direct_sum_sample"] = out
        result["speedup_vs_fp64_direct"] = out["fp64"]["extrapolated_certificate_ms"] / ms
    if rank == 0 and world == 1 and args.learned_leg and args.method == "barneshut":
        # The learned opening criterion, trained on another seed of the same
        # workload family, on this workload: one step, against the plain one.
        from fastlinkingnumbers_b200 import LearnedCriterion
        t0 = time.perf_counter()
        if args.workload == "held_out_20M":
            from fastlinkingnumbers_b200 import workloads as W
            toff, txyz, tpairs = W.walk_pairs(seed=args.seed + 1000)
            trained_on = "20 pairs of interleaved 100,000-step closed walks (seed %d)" % (args.seed + 1000)
        else:
            toff, txyz, tpairs, _ = make_workload(args.workload, args.seed + 1000, args.loops, args.loop_steps, engine=eng)
            trained_on = f"seed {args.seed + 1000} of the same workload family (held out)"
        model = LearnedCriterion.train(eng, txyz, toff, tpairs, params=prm)
        train_s = time.perf_counter() - t0
        eng.set_learned(model)
        try:
            runs = []
            for _ in range(2):
                step()
                runs.append((eng.stats(), d_lk.cpu().numpy()))
        finally:
            eng.set_learned(None)
        sl, llk = min(runs, key=lambda r: r[0]["ms_kernels"])
        info = model.info()
        result["learned_leg"] = {
            "trained_on": trained_on,
            "train": {k: info[k] for k in ("recorded", "samples", "log10_tau", "s_min", "val_loss",
                                           "val_coverage", "ms_collect", "ms_train")},
            "train_wall_s_incl_workload": round(train_s, 2),
            "certificate_ms": sl["ms_kernels"], "main_kernel_ms": sl["ms_main_kernel"],
            "node_pairs": sl["bh_far_evals"] + sl["bh_exact_entries"],
            "plain_node_pairs": node_pairs, "plain_certificate_ms": ms,
            "beta_retried": sl["beta_retried"], "escalated": sl["bh_escalated"],
            "fp64_recomputed": sl["fp64_recomputed"],
            "same_integers_as_plain": bool(np.array_equal(np.round(llk), np.round(lk))),
            "max_abs_diff_vs_plain": float(np.abs(llk - lk).max()),
        }
    if rank == 0 and world == 1 and args.cli_leg:
        # End to end through the flag-compatible CLI: a fresh process loads
        # the BCC, prepares on the GPU, runs Barnes-Hut and writes the
        # certificate (wall clock, so it includes CUDA start-up).
        from fastlinkingnumbers_b200 import workloads as W
        from fastlinkingnumbers_b200._native import LIB_DIR
        # The CLI is a second process on the same GPU: this process's engine
        # buffers (grow-only; about 100 GB on the 134M-segment batch) and
        # torch's cached blocks are released first. Nothing below uses them.
        eng.close()
        torch.cuda.empty_cache()
        with tempfile.TemporaryDirectory() as td:
            path, cert = os.path.join(td, "w.bcc"), os.path.join(td, "cert.txt")
            W.write_bcc(path, raw_curves)
            walls, failed = [], None
            for _ in range(2):
                t0 = time.perf_counter()
                r = subprocess.run([os.path.join(LIB_DIR, "verifycurves"), "--input", path, "--output", cert],
                                   capture_output=True, text=True)
                if r.returncode != 0:
                    # The leg is reported, not fatal: the JSON line still prints.
                    failed = f"exit {r.returncode}: " + (r.stderr.strip().splitlines() or [""])[-1][:300]
                    break
                walls.append(round(time.perf_counter() - t0, 3))
            cli_text = None if failed else open(cert).read()
        entries = None if failed else len(cli_text.strip().splitlines()) - 1
        result["cli_e2e"] = {"command": "verifycurves --input <workload>.bcc --output cert.txt",
                             "wall_s": walls, "certificate_entries": entries,
                             "same_certificate_bytes_as_bench": None if failed else
                             cli_text == certificate_text(len(poff) - 1, pairs, lk)}
        if failed:
            result["cli_e2e"]["error"] = failed
    if rank == 0 and world == 1 and args.cpu_seconds > 0:
        from oracle import pyoracle
        thr = pyoracle.max_threads(native=True)
        v, info = cpu_sample_run(poff, pxyz, pairs, args.cpu_seconds, args.seed + 17, thr)
        result["cpu_baseline"] = {
            "value": v, "unit": UNIT, "cores": thr, "kind": "port",
            "sample": f"{info['pairs']} seeded random pairs ({info['segment_pairs']:.3g} segment "
                      f"pairs) in {info['seconds']} s; oracle port of the reference's BH, built -O3 "
                      f"-march=native"}
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="polymer",
                    choices=["polymer", "held_out_20M", "mixed_batch", "chain_mail", "ring_chain"])
    ap.add_argument("--method", default="barneshut", choices=["barneshut", "directsum"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--bh-tree", type=int, default=0)
    ap.add_argument("--bh-schedule", type=int, default=0, help="0 rounds (fused evaluation), 1 persistent queue, 2 rounds (split evaluation)")
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--loops", type=int, default=200)
    ap.add_argument("--loop-steps", type=int, default=50000)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--direct-sample", type=int, default=64)
    ap.add_argument("--traffic-bytes-per-node-pair", type=float, default=66.4,
                    help="DRAM bytes per node pair measured by ncu on the polymer workload (0: none)")
    ap.add_argument("--cli-leg", type=int, default=1,
                    help="also time the verifycurves CLI end to end on the workload written as BCC")
    ap.add_argument("--bh-bucket", type=int, default=0,
                    help="node pairs of at most this many segments a side are summed exactly; 0 = 8, 1 = leaf pairs only")
    ap.add_argument("--bh-budget", type=int, default=0,
                    help="fixed Barnes-Hut round budget (skips the autotuner); 0 = tuned")
    ap.add_argument("--autotune", type=int, default=1,
                    help="tune the Barnes-Hut round budget on a sample of the pairs before timing")
    ap.add_argument("--fp64-margin", type=float, default=None,
                    help="margin to the rounding boundary below which a pair is recomputed in FP64 (default 0.25)")
    ap.add_argument("--bh-occupancy", type=int, default=0,
                    help="CTAs per SM of the traversal kernels (5, 6 or 7; 0 = the library's default or the "
                         "autotuner's choice)")
    ap.add_argument("--autotune-bucket", type=int, default=1,
                    help="let the autotuner also choose the exact-bucket size (unless --bh-bucket is given)")
    ap.add_argument("--clock-interval-ms", type=int, default=200,
                    help="nvidia-smi sampling interval of the clocks record")
    ap.add_argument("--learned-leg", type=int, default=1,
                    help="also train the learned opening criterion on another seed and time one step with it")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
