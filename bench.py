#!/usr/bin/env python3
"""Benchmark of the B200 ForceAtlas2 engine on the plain Barnes-Hut workload.

Workload (one "step" = one ForceAtlas2 iteration of the whole graph):
  R-MAT scale 20, 16,777,216 edge draws, a=.57 b=.19 c=.19 (seed 0), self-loops
  and repeated undirected edges removed (N = 646,567 nodes, E = 15,702,443
  edges with this generator); positions uniform in [-1e4, 1e4]^2 (srandom(1234) + the reference's
  randomizePositions); strong gravity, scale 10, gravity 1, theta 1.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is device-timed iterations/s with the graph resident in HBM (CUDA
events on the engine's stream around K iterations, max over ranks, summed
over ranks: with N > 1 every rank lays out its own replica of the graph, the
single-graph path does not shard).  `e2e` is the same metric through the
public C ABI with host buffers: per step, the positions are copied in from
pinned host memory, one iteration runs and the positions are copied back
(fa2_step_host: the three in one call, one host synchronisation).
`--impl reference` times the reference's own CPU ForceAtlas2
(CPUForceAtlas2::doStep, built from its sources into oracle/_ref) on the same
graph and positions, one iteration per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FA2 iters/s on R-MAT 1M/16M: plain BH vs learned-correction at equal force RMSE"
UNIT = "iters/s"
SCALE, DRAWS = 20, 16_777_216
K_R, K_G, STRONG = 10.0, 1.0, True
WIDTH = 2.0e4
# R-MAT workloads: scale, edge draws, side of the square of the initial
# positions.  rmat23 is the large run: 8.4M ids, 134M draws, U[-1e5,1e5]^2.
RMAT = {"rmat20": (SCALE, DRAWS, WIDTH), "rmat23": (23, 134_217_728, 2.0e5)}
FP64_SAMPLES = 4096
FP64_EVERY, FP64_CHECKS = 50, 4
# kernels per iteration besides the sort passes: attract, keys, tree_count, emit,
# traverse, displace; the sort is 8 passes, or 6 passes and a fix-up pass after
# shallow trees (fa2_stats.sort_passes); the quadrupole walk adds the moment
# scan and the per-cell a2 kernel
KERNELS_PER_ITER = 6
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one k_attract
# launch at this workload, from an ncu capture of
#   ncu --set full --clock-control none -k regex:k_attract -s 4 -c 1 \
#       python bench.py --steps 5 --warmup 3 --no-cpu-baseline --no-extras --no-correction
ATTRACT_TRAFFIC_BYTES = 144_444_160


def clocks_sampler(device: int, path: str):
    try:
        return subprocess.Popen(
            ["nvidia-smi", f"--id={device}",
             "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
             "--format=csv,noheader,nounits", "-lms", "200"],
            stdout=open(path, "w"), stderr=subprocess.DEVNULL)
    except Exception:
        return None


def clocks_summary(path: str):
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    try:
        for line in open(path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
    except OSError:
        pass
    if not sm:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons)}


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier_max(world, value: float) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ------------------------------------------------------------------ reference --

def run_reference(args, world, rank):
    if rank != 0:
        return
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libref_cpu.so is not built (needs the "
                                         "reference sources at build time)"}))
        return
    from gpugraphlayout_b200 import synth
    s, t = synth.rmat_edges(SCALE, DRAWS, seed=0)
    og = O.Graph(s, t)
    rg = O.RefGraph(graph=og)
    ref = O.RefCPUFA2(rg, WIDTH, WIDTH, 1234, True, STRONG, K_G, K_R)
    for _ in range(args.warmup):
        ref.step(1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ref.step(1)
    dt = time.perf_counter() - t0
    v = args.steps / dt
    sample = (f"{args.warmup}+{args.steps} full iterations of CPUForceAtlas2::doStep "
              f"(Barnes-Hut, 1 thread) on the whole workload graph")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": workload_config(og.n, og.m),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def workload_config(n, m, theta=1.0, multipole=1, workload="rmat20", learned=False):
    walk = ("plain Barnes-Hut" if multipole == 1 else "Barnes-Hut with the quadrupole term")
    if learned:
        walk += (" with the learned far-field correction (MLP trained on R-MAT scale 16 "
                 "layouts, FP64 targets)")
    scale, draws, width = RMAT[workload]
    return {"workload": f"R-MAT scale {scale} ({draws:,} draws, a=.57 b=.19 c=.19, seed 0), "
                        f"N={n:,} E={m:,}; positions U[-{width / 2:g},{width / 2:g}]^2; "
                        f"strong gravity, scale 10, gravity 1, theta {theta:g}; {walk}",
            "nodes": n, "edges": m, "l2": "per-iteration working set larger than L2 "
                                          "(padded CSR alone exceeds 126 MB)",
            "parallelism": "replicas (one graph per GPU)"}


def cpu_baseline_sample(og, xy):
    """The reference CPU ForceAtlas2 on the workload graph: 3 iterations after
    one untimed one (~10-30 s of single-thread CPU work at scale 20)."""
    from oracle import oracle as O
    if not O.ref_available():
        return None
    rg = O.RefGraph(graph=og)
    ref = O.RefCPUFA2(rg, WIDTH, WIDTH, 1234, True, STRONG, K_G, K_R)
    ref.set_positions(xy)
    ref.step(1)
    it = 3
    t0 = time.perf_counter()
    ref.step(it)
    dt = time.perf_counter() - t0
    return {"value": it / dt, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"{it} iterations of CPUForceAtlas2::doStep (Barnes-Hut, 1 thread) on "
                      f"the full workload graph after 1 untimed iteration"}


# ----------------------------------------------------------------------- ours --

CORRECTION_SAMPLES = 4096
GUARD_EVERY, GUARD_SAMPLES = 25, 512
CORRECTION_THETAS = (1.2, 1.4, 1.5, 1.6, 1.7, 1.8, 2.0)
# The learned correction: trained on R-MAT scale 16 (1,048,576 draws) from
# 200 layout snapshots of a plain run, evaluated on the workload at these
# (theta, multipole) walks against the plain walk at theta 1.
TRAIN_SCALE, TRAIN_DRAWS = 16, 1 << 20
LEARNED = ((1.2, 1), (1.5, 1), (1.6, 1), (1.7, 1), (2.0, 1), (2.0, 2))
EQUAL_RMSE_TARGET = 1.5  # the speed-up at equal or lower error the design aims at


def train_learned(eng_device, combos=LEARNED):
    """One MLP per (theta, multipole) of `combos`, trained on the engine's
    own layouts of the scale-16 R-MAT graph (gpugraphlayout_b200.learn)."""
    from gpugraphlayout_b200 import UGraph, synth
    from gpugraphlayout_b200.learn import train_correction
    s_raw, t_raw = synth.rmat_edges(TRAIN_SCALE, TRAIN_DRAWS, seed=0)
    g = UGraph.from_pairs(s_raw, t_raw)
    s, t = g.edges()
    out = {}
    for theta, mp in combos:
        out[(theta, mp)] = train_correction(g.num_nodes(), s, t, theta=theta, multipole=mp,
                                            strong_gravity=STRONG, gravity=K_G, scale=K_R,
                                            width=WIDTH, device=eng_device)
    return out, {"graph": f"R-MAT scale {TRAIN_SCALE} ({TRAIN_DRAWS:,} draws, seed 0)",
                 "nodes": g.num_nodes(), "edges": g.num_edges()}


def snapshot(eng):
    """The layout state a step starts from: positions, global speed, speed
    efficiency and the previous forces."""
    return eng.get_positions(), eng.speed_state()


def restore(eng, S):
    """Back to a snapshot.  Positions alone are not enough: a step repeated
    from the same positions sees no swing, so the speed rule raises the
    global speed as far as it may, and the layout that follows is shaken
    for tens of iterations (its walk up to 40 % slower)."""
    P, (gs, se, fp) = S
    eng.set_positions(P)
    eng.set_speed_state(gs, se, fp)


def timed_from(eng, S, k):
    """k steps from snapshot S, timed twice: the step time without per-kernel
    events, then the kernels' times with them.  Both iteration graphs are
    captured beforehand (one untimed step each, then the snapshot again)."""
    restore(eng, S)
    eng.step(1)
    restore(eng, S)
    eng.step_timed(1)
    restore(eng, S)
    ms, _ = eng.step_timed(k, kernels=False)
    restore(eng, S)
    _, kms = eng.step_timed(k)
    return ms, kms


def correction_report(eng, n, steps, device=0):
    """Far-field accuracy against cost at the current layout: the reference's
    monopole walk at theta 1 beside the quadrupole walk at larger theta.  Each
    configuration computes one step's repulsion from the same state S
    (positions and speed state); the error is the relative RMSE against the
    exact FP64 all-pairs sum over CORRECTION_SAMPLES sampled nodes, and the
    cost is the mean step and walk (traverse + quadrupole sums) time over a
    few steps from S.  Outside the
    timed region; the engine is left at theta 1, multipole 1."""
    S = snapshot(eng)
    rng = np.random.default_rng(3)
    samples = np.sort(rng.choice(n, min(CORRECTION_SAMPLES, n), replace=False)).astype(np.uint32)
    exact = eng.exact_repulsion(samples)
    k = max(3, min(steps, 10))
    rows = []
    for theta, mp in [(1.0, 1)] + [(t, 2) for t in CORRECTION_THETAS]:
        eng.set_approximation(theta, mp)
        restore(eng, S)
        eng.step(1)
        tot, ga = eng.forces()
        rep = (tot - ga)[samples].astype(np.float64)
        err = float(np.sqrt(((rep - exact) ** 2).sum() / (exact ** 2).sum()))
        visits = eng.stats()["visits"]
        ms, kms = timed_from(eng, S, k)
        rows.append({"theta": theta, "multipole": mp, "rel_rmse": err, "visits": visits,
                     "ms_per_step": ms / k,
                     "walk_ms": kms.get("traverse", 0.0) + kms.get("quadrupole", 0.0),
                     "moments_ms": kms.get("moments", 0.0),
                     "quadrupole_ms": kms.get("quadrupole", 0.0)})
    base = rows[0]

    # the learned correction on the same positions, samples and FP64 sums
    models, train_graph = train_learned(device)
    learned = []
    from gpugraphlayout_b200 import Fa2Error
    for (theta, mp), (mlp, info) in models.items():
        eng.set_approximation(theta, mp)
        eng.set_learned_correction(mlp)
        try:
            restore(eng, S)
            eng.step(1)
            tot, ga = eng.forces()
            rep = (tot - ga)[samples].astype(np.float64)
            err = float(np.sqrt(((rep - exact) ** 2).sum() / (exact ** 2).sum()))
            st1 = eng.stats()
            visits, pairs = st1["visits"], st1["learned_pairs"]
            ms, kms = timed_from(eng, S, k)
        except Fa2Error as ex:  # recorded, not fatal: the next configuration starts afresh
            learned.append({"theta": theta, "multipole": mp, "error": str(ex),
                            "device_error": eng.stats()["device_error"]})
            eng.set_learned_correction(None)
            restore(eng, S)
            continue
        learned.append({"theta": theta, "multipole": mp, "rel_rmse": err, "visits": visits,
                        "pairs": pairs,
                        "ms_per_step": ms / k,
                        "walk_ms": kms.get("traverse", 0.0) + kms.get("quadrupole", 0.0),
                        "moments_ms": kms.get("moments", 0.0),
                        "mlp_and_tail_ms": kms.get("learn", 0.0),
                        "training": {kk: info[kk] for kk in ("samples", "snapshots", "final_loss",
                                                             "collect_s", "fit_s")}})
        eng.set_learned_correction(None)
    eng.set_approximation(1.0, 1)
    ran = [r for r in learned if "error" not in r]
    ok_l = [r for r in ran if r["rel_rmse"] <= base["rel_rmse"]]
    best_l = min(ok_l, key=lambda r: r["ms_per_step"]) if ok_l else None
    fastest_l = min(ran, key=lambda r: r["ms_per_step"]) if ran else None
    learned_guarded = None
    if best_l is not None:
        steps_g = 4 * GUARD_EVERY
        ms_plain, _ = timed_from(eng, S, steps_g)
        eng.set_approximation(best_l["theta"], best_l["multipole"])
        eng.set_learned_correction(models[(best_l["theta"], best_l["multipole"])][0])
        eng.set_accuracy_guard(GUARD_EVERY, GUARD_SAMPLES)
        ms, _ = timed_from(eng, S, steps_g)
        gd = eng.accuracy_guard()
        eng.set_accuracy_guard(0, 0)
        eng.set_learned_correction(None)
        eng.set_approximation(1.0, 1)
        learned_guarded = {"theta": best_l["theta"], "multipole": best_l["multipole"],
                           "every": GUARD_EVERY, "samples": GUARD_SAMPLES, "steps": steps_g,
                           "ms_per_step": ms / steps_g, "plain_ms_per_step": ms_plain / steps_g,
                           "speedup_vs_plain": ms_plain / ms, **gd}
    learned_report = {
        "mlp": "12 -> 64 -> 64 -> 2, BF16 weights and activations, FP32 accumulation "
               "(tcgen05, accumulators in tensor memory); trained with the FP32 training "
               "kernels on FP64 exact targets",
        "training_graph": train_graph,
        "configs": learned,
        "equal_rmse_speedup": (None if best_l is None else
                               {"theta": best_l["theta"], "multipole": best_l["multipole"],
                                "step": base["ms_per_step"] / best_l["ms_per_step"],
                                "target": EQUAL_RMSE_TARGET,
                                "met": base["ms_per_step"] / best_l["ms_per_step"]
                                >= EQUAL_RMSE_TARGET}),
        "fastest": (None if fastest_l is None else
                    {"theta": fastest_l["theta"], "multipole": fastest_l["multipole"],
                     "step": base["ms_per_step"] / fastest_l["ms_per_step"],
                     "rel_rmse": fastest_l["rel_rmse"]}),
        "guarded": learned_guarded,
    }

    ok = [r for r in rows[1:] if r["rel_rmse"] <= base["rel_rmse"]]
    best = min(ok, key=lambda r: r["ms_per_step"]) if ok else None
    guarded = None
    if best is not None:
        # the corrected walk as a user runs it: with the accuracy guard
        # checking it against the FP64 sum every GUARD_EVERY steps
        steps_g = 4 * GUARD_EVERY
        eng.set_approximation(1.0, 1)
        ms_plain, _ = timed_from(eng, S, steps_g)
        eng.set_approximation(best["theta"], 2)
        eng.set_accuracy_guard(GUARD_EVERY, GUARD_SAMPLES)
        ms, _ = timed_from(eng, S, steps_g)
        gd = eng.accuracy_guard()
        eng.set_accuracy_guard(0, 0)
        # the same steps from the same positions with the plain walk
        guarded = {"theta": best["theta"], "every": GUARD_EVERY, "samples": GUARD_SAMPLES,
                   "steps": steps_g, "ms_per_step": ms / steps_g,
                   "plain_ms_per_step": ms_plain / steps_g,
                   "speedup_vs_plain": ms_plain / ms, **gd}
    eng.set_approximation(1.0, 1)
    restore(eng, S)
    return {
        "samples": len(samples), "exact": "fp64 all-pairs on the GPU",
        "configs": rows,
        "equal_rmse_speedup": (None if best is None else
                               {"theta": best["theta"], "multipole": 2,
                                "step": base["ms_per_step"] / best["ms_per_step"],
                                "walk": base["walk_ms"] / best["walk_ms"]}),
        "guarded": guarded,
        "learned": learned_report,
    }


def fp64_checks(eng, n, checks=FP64_CHECKS):
    """The large run's accuracy record: every FP64_EVERY steps, the repulsion
    of the next step on FP64_SAMPLES sampled nodes against the exact FP64
    all-pairs sum at the same positions (computed on the GPU)."""
    rng = np.random.default_rng(5)
    samples = np.sort(rng.choice(n, min(FP64_SAMPLES, n), replace=False)).astype(np.uint32)
    out = []
    for c in range(checks):
        eng.step(FP64_EVERY - 1)
        exact = eng.exact_repulsion(samples)
        eng.step(1)
        tot, ga = eng.forces()
        rep = (tot - ga)[samples].astype(np.float64)
        err = float(np.sqrt(((rep - exact) ** 2).sum() / (exact ** 2).sum()))
        out.append({"after_steps": (c + 1) * FP64_EVERY, "rel_rmse": err})
    return {"samples": len(samples), "every": FP64_EVERY, "checks": out}


def run_ours(args, world, rank, local, fp64_n=FP64_CHECKS, correction=True):
    """The R-MAT workload's record (rank 0; None on the other ranks)."""
    from gpugraphlayout_b200 import Engine, UGraph, kernel_names, random_positions, synth
    scale, draws, width = RMAT[args.workload]
    large = args.workload != "rmat20"
    s_raw, t_raw = synth.rmat_edges(scale, draws, seed=0)
    g = UGraph.from_pairs(s_raw, t_raw)
    n, m = g.num_nodes(), g.num_edges()
    s, t = g.edges()
    xy0 = random_positions(n, width, width, 1234)
    eng = Engine(n, s, t, strong_gravity=STRONG, gravity=K_G, scale=K_R, device=local,
                 theta=args.theta, multipole=args.multipole)
    learned = getattr(args, "learned", None)
    plain = args.theta == 1.0 and args.multipole == 1 and learned is None
    eng.set_positions(xy0)
    train_info = None
    if learned is not None:
        # the workload with the learned correction at theta `learned`,
        # trained first (outside the timed region) on the scale-16 graph
        models, _ = train_learned(local, ((learned, args.multipole),))
        mlp, train_info = models[(learned, args.multipole)]
        eng.set_approximation(learned, args.multipole)
        eng.set_learned_correction(mlp)

    import torch
    torch.cuda.set_device(local)
    # warm-up: both captured iteration graphs (the plain one of fa2_step and
    # the one with timing events of fa2_step_timed) are built here, not in a
    # timed region
    eng.step(1)
    eng.step_timed(max(args.warmup, 3))
    clk_path = os.path.join(tempfile.gettempdir(), f"fa2_clocks_{rank}.csv")
    sampler = clocks_sampler(local, clk_path)
    time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize()
    ms, _ = eng.step_timed(args.steps, kernels=False)
    torch.cuda.synchronize()
    barrier(world)
    if sampler:
        sampler.terminate()
        sampler.wait()
    ms_max = barrier_max(world, ms)
    value = world * args.steps / (ms_max / 1000.0)
    # per-kernel times inside the iteration graph, from a copy of it with an
    # event around every kernel (those events cost time of their own, so the
    # timed steps above run without them)
    _, kms = eng.step_timed(min(args.steps, 20))
    st = eng.stats()

    # per-kernel times with every kernel running alone (the attraction is
    # otherwise spread over the tree build's gaps): the roofline denominators
    iso_steps = min(args.steps, 10)
    eng.set_overlap(False)
    eng.step(1)
    eng.step_timed(3)
    _, kms_iso = eng.step_timed(iso_steps)
    eng.set_overlap(True)
    eng.step(1)  # the plain graph again after the overlap switch

    # end to end through the C ABI with pinned host buffers
    host = torch.empty((n, 2), dtype=torch.float32, pin_memory=True)
    host.numpy()[:] = eng.get_positions()
    ptr = host.data_ptr()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        # positions in from pinned memory, one iteration, positions out
        eng.step_host(ptr, 1, ptr)
    e2e_s = barrier_max(world, time.perf_counter() - t0)
    e2e = world * args.steps / e2e_s

    if rank != 0:
        eng.close()
        return None
    # the correction report compares against the plain walk, so it runs only
    # when the plain walk is the workload, and only at N = 1 (with N > 1 the
    # other ranks have left; their GPUs are not held for it)
    correction = (correction_report(eng, n, args.steps, local)
                  if (correction and plain and not large and not args.no_correction
                      and world == 1) else None)
    fp64 = fp64_checks(eng, n, fp64_n) if large else None
    names = kernel_names()
    pk, pk_kind = peaks()
    hbm = float(pk["hbm_gbs"])
    # algorithmic bytes per launch: the attraction reads both directions of
    # every edge (4 B ids), the row offsets and each node's own position, and
    # writes its force, 8E + 20N + 4 (each neighbour position is gathered
    # from L2, not counted; the row padding and the mass read are not
    # algorithmic either)
    attract_bytes = 8 * m + 20 * n + 4
    disp_bytes = 40 * n
    trav_ms = kms_iso.get("traverse", 0.0)
    kernels = {}
    for nm in names:
        kernels[nm] = {"ms": kms.get(nm, 0.0), "ms_alone": kms_iso.get(nm, 0.0)}
    att_ms = kms_iso["attract"]
    kernels["attract"].update(bytes=attract_bytes,
                              gbs=attract_bytes / (att_ms * 1e6) if att_ms else None)
    dsp_ms = kms_iso["displace"]
    kernels["displace"].update(bytes=disp_bytes,
                               gbs=disp_bytes / (dsp_ms * 1e6) if dsp_ms else None)
    inter = st["interactions"]
    kernels["traverse"].update(interactions=inter, visits=st["visits"],
                               interactions_per_s=inter / (trav_ms * 1e-3) if trav_ms else None)
    dom = max(names, key=lambda k: kms_iso.get(k, 0.0))
    att_gbs = kernels["attract"]["gbs"] or 0.0
    roofline = {"kernel": "attract", "bound": "hbm", "achieved": att_gbs, "peak": hbm,
                "unit": "GB/s", "frac": att_gbs / hbm,
                "traffic": ATTRACT_TRAFFIC_BYTES, "traffic_unit": "bytes per launch",
                "note": f"peak = {pk_kind} HBM copy bandwidth; achieved = algorithmic bytes / "
                        f"the kernel's CUDA-event time running alone; dominant kernel by time "
                        f"is '{dom}' ({kms_iso.get(dom, 0.0):.3f} ms/launch alone)"}
    # The walk is bound by instruction issue and dependent-load latency, not by
    # HBM or tensor cores: its work is 10 FP32 operations per interaction,
    # reported against the nominal FP32 rate of the SMs.
    fp32_peak = 148 * 128 * 2 * float(pk.get("sm_max_mhz", 1965.0)) * 1e6 / 1e12
    trav_tflops = 10.0 * inter / (trav_ms * 1e-3) / 1e12 if trav_ms else 0.0
    roofline_traverse = {"kernel": "traverse", "bound": "fp32 issue / load latency",
                         "achieved": trav_tflops, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": trav_tflops / fp32_peak, "flop_per_interaction": 10,
                         "note": "peak = nominal FP32 (148 SMs x 128 lanes x 2 x max SM clock)"}
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": workload_config(n, m, args.theta if learned is None else learned,
                                  args.multipole, args.workload, learned is not None),
        "clocks": clocks_summary(clk_path),
        # + moment scan and per-cell a2 (quadrupole walk), + the cells'
        # children moments, MLP and tail (learned correction)
        "gpu_launches": (KERNELS_PER_ITER + st["sort_passes"] + (st["sort_passes"] < 8)
                         + (2 if args.multipole == 2 else 0)
                         + (3 if learned is not None else 0)) * args.steps,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 8 * n,
                "d2h_bytes_per_step": 8 * n},
        "roofline": roofline,
        "roofline_traverse": roofline_traverse,
        "kernels": kernels,
        "tree": {"nodes": st["tree_nodes"], "cells": st["tree_cells"],
                 "max_level": st["max_level"]},
        "far_field_correction": correction,
    }
    if fp64 is not None:
        out["fp64_checks"] = fp64
    if train_info is not None:
        out["learned_training"] = {k: train_info[k] for k in ("samples", "snapshots", "final_loss",
                                                               "collect_s", "fit_s")}
        out["learned_pairs"] = st["learned_pairs"]
    if large:
        # ncu's DRAM count above was taken at scale 20
        out["roofline"]["traffic"] = None
        out["cpu_baseline_skipped"] = ("one CPUForceAtlas2::doStep at this size takes minutes; "
                                       "the reference CPU baseline is in the rmat20 line")
    eng.close()
    if world == 1 and not args.no_cpu_baseline and not large:
        from oracle import oracle as O
        out["cpu_baseline"] = cpu_baseline_sample(O.Graph(s_raw, t_raw), xy0)
    return out


# ---------------------------------------------------------------- batched --

BATCH_GRAPHS = 4096
BATCH_METRIC = ("FA2 batch iters/s: 4096 SBM graphs (nodes log-uniform 50-20000) "
                "laid out together")


def batch_config(graphs, world):
    n = sum(g[0] for g in graphs)
    m = sum(len(g[1]) for g in graphs)
    return {"workload": f"{len(graphs)} stochastic block models, nodes log-uniform in "
                        "[50, 20000], 2-32 equal blocks, p_in 0.05, p_out 0.002, mean degree "
                        "capped at 40 (seed 0); positions U[-5000,5000]^2 (srandom per graph); "
                        "weak gravity, scale 2, gravity 1, theta 1",
            "graphs": len(graphs), "nodes": n, "edges": m,
            "l2": f"per-iteration working set ({(16 * n + 8 * m) / 1e6:.0f} MB) larger than L2",
            "parallelism": f"graphs sharded over {world} rank(s), no collective"}


def batch_cpu_baseline(graphs, sample_ids):
    """The reference's CPU ForceAtlas2 on a sample of the batch's graphs, 2
    iterations each after 1 untimed; the batch's time per iteration is
    extrapolated from the sample by seconds per node (the sample spans the
    size range)."""
    from oracle import oracle as O
    if not O.ref_available():
        return None
    t_sum, n_sum = 0.0, 0
    for i in sample_ids:
        n, lo, hi = graphs[i]
        g = O.Graph(lo, hi)
        ref = O.RefCPUFA2(O.RefGraph(graph=g), 10000.0, 10000.0, 1234, True, False, 1.0, 2.0)
        ref.step(1)
        t0 = time.perf_counter()
        ref.step(2)
        t_sum += (time.perf_counter() - t0) / 2
        n_sum += g.n
        del ref
    total_n = sum(g[0] for g in graphs)
    per_iter = t_sum / n_sum * total_n
    return {"value": 1.0 / per_iter, "unit": "batch iters/s", "cores": 1, "kind": "reference",
            "sample": f"2 iterations of CPUForceAtlas2::doStep (1 thread) on {len(sample_ids)} of "
                      f"the graphs ({n_sum} nodes), extrapolated by seconds per node to all "
                      f"{total_n} nodes"}


def run_batched(args, world, rank, local):
    """The batched workload's record (rank 0; None on the other ranks)."""
    import torch
    from gpugraphlayout_b200 import BatchEngine, random_positions, shard, synth
    graphs = synth.sbm_batch(BATCH_GRAPHS, seed=0)
    parts = shard.partition(shard.graph_costs(graphs), world)
    mine = parts[rank]
    eng = BatchEngine([graphs[i] for i in mine], strong_gravity=False, gravity=1.0, scale=2.0,
                      device=local)
    xy = np.concatenate([random_positions(graphs[i][0], 10000.0, 10000.0, 1234 + i)
                         for i in mine]) if mine else np.zeros((0, 2), np.float32)
    eng.set_positions(xy)
    torch.cuda.set_device(local)
    eng.step(max(args.warmup, 3))
    # CTA sizes picked by measurement on this batch (the layout state is kept)
    tuned = eng.autotune(2)
    # a step call runs a graph captured once per iteration count: the counts
    # the timed loops use are captured here
    eng.step_timed(args.steps)
    eng.step(1)
    sizes = [graphs[i][0] for i in mine]
    classes = (any(s <= tuned["split"] for s in sizes) + any(s > tuned["split"] for s in sizes))
    clk_path = os.path.join(tempfile.gettempdir(), f"fa2_clocks_b{rank}.csv")
    sampler = clocks_sampler(local, clk_path)
    time.sleep(0.3)
    barrier(world)
    torch.cuda.synchronize()
    ms = eng.step_timed(args.steps)
    torch.cuda.synchronize()
    barrier(world)
    if sampler:
        sampler.terminate()
        sampler.wait()
    ms_max = barrier_max(world, ms)
    value = args.steps / (ms_max / 1000.0)

    # end to end through the C ABI: positions in from pinned host memory, one
    # iteration, positions out
    host = torch.empty((max(eng.n, 1), 2), dtype=torch.float32, pin_memory=True)
    host.numpy()[: eng.n] = eng.get_positions()
    ptr = host.data_ptr()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.set_positions_ptr(ptr)
        eng.step(1)
        eng.get_positions_ptr(ptr)
    e2e = args.steps / barrier_max(world, time.perf_counter() - t0)
    eng.close()
    if rank != 0:
        return None
    pk, pk_kind = peaks()
    hbm = float(pk["hbm_gbs"])
    n_all = sum(g[0] for g in graphs)
    m_all = sum(len(g[1]) for g in graphs)
    # compulsory bytes of one iteration of every graph: CSR ids (2 per edge),
    # offsets, positions and previous forces read and written, mass
    bytes_iter = 8 * m_all + 4 * n_all + 16 * n_all + 16 * n_all + 4 * n_all
    achieved = bytes_iter * value / 1e9
    out = {
        "metric": BATCH_METRIC, "value": value, "unit": "batch iters/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": batch_config(graphs, world),
        "graph_iters_per_s": value * len(graphs),
        "clocks": clocks_summary(clk_path),
        # one persistent launch per size class runs all the timed iterations
        "gpu_launches": classes,
        "autotune": tuned,
        "e2e": {"value": e2e, "unit": "batch iters/s", "h2d_bytes_per_step": 8 * n_all // world,
                "d2h_bytes_per_step": 8 * n_all // world},
        "roofline": {"kernel": "batch", "bound": "hbm", "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": achieved / hbm, "traffic": None,
                     "note": f"peak = {pk_kind} HBM copy bandwidth; achieved = compulsory bytes "
                             "of one iteration of every graph / time; the per-graph pipeline is "
                             "latency-bound (one CTA per graph), so this is a lower bound"},
    }
    if world == 1 and not args.no_cpu_baseline:
        sizes = np.array([g[0] for g in graphs])
        sample = [int(i) for i in np.argsort(sizes)[:: len(graphs) // 8][:8]]
        out["cpu_baseline"] = batch_cpu_baseline(graphs, sample)
    return out


# Wall-clock budget of the default run: the sub-records are skipped once the
# run has taken this long (their graphs take tens of seconds to build).
EXTRAS_BUDGET_S = 240.0
SUB_STEPS, SUB_WARMUP = 10, 3


def _compact(rec, keys):
    return {k: rec[k] for k in keys if k in rec}


CONFIG1_ITERS = 500


def config1_record(local, no_cpu_baseline):
    """The CPU baseline configuration: Barabasi-Albert, 10,000 nodes, m = 3,
    seed 0; positions U[-1000,1000]^2; weak gravity, scale 80, gravity 1;
    500 iterations, on the engine (device-timed, and end to end through the
    C ABI) and on the reference's CPUForceAtlas2 from the same positions,
    with both final layouts' statistics."""
    from gpugraphlayout_b200 import Engine, UGraph, random_positions, synth
    from gpugraphlayout_b200.layout_stats import summary
    s_raw, t_raw = synth.ba_edges(10000, 3, seed=0)
    g = UGraph.from_pairs(s_raw, t_raw)
    n, m = g.num_nodes(), g.num_edges()
    s, t = g.edges()
    xy0 = random_positions(n, 2000.0, 2000.0, 1234)
    eng = Engine(n, s, t, strong_gravity=False, gravity=1.0, scale=80.0, device=local)
    eng.set_positions(xy0)
    eng.step(5)  # warm-up (both captured graphs), then the run starts again
    eng.step_timed(5)  # from the same state
    eng.set_positions(xy0)
    eng.set_speed_state(1.0, 1.0)
    ms, _ = eng.step_timed(CONFIG1_ITERS, kernels=False)
    ours_xy = eng.get_positions()
    eng.set_speed_state(1.0, 1.0)
    t0 = time.perf_counter()
    eng.set_positions(xy0)
    eng.step(CONFIG1_ITERS)
    eng.get_positions()
    e2e_s = time.perf_counter() - t0
    eng.close()
    rec = {"workload": f"Barabasi-Albert n=10,000 m=3 seed 0 (N={n:,} E={m:,}); positions "
                       "U[-1000,1000]^2; weak gravity, scale 80, gravity 1, theta 1; "
                       f"{CONFIG1_ITERS} iterations",
           "value": CONFIG1_ITERS / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms / CONFIG1_ITERS,
           "e2e": {"value": CONFIG1_ITERS / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 8 * n,
                   "d2h_bytes_per_step": 8 * n,
                   "note": "positions in once and out once around the 500 iterations"},
           "layout": {"ours": summary(ours_xy, s, t, 64)}}
    if not no_cpu_baseline:
        from oracle import oracle as O
        if O.ref_available():
            og = O.Graph(s_raw, t_raw)
            ref = O.RefCPUFA2(O.RefGraph(graph=og), 2000.0, 2000.0, 1234, True, False, 1.0,
                              80.0)
            ref.set_positions(xy0)
            t0 = time.perf_counter()
            ref.step(CONFIG1_ITERS)
            dt = time.perf_counter() - t0
            rec["cpu_baseline"] = {
                "value": CONFIG1_ITERS / dt, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": f"{CONFIG1_ITERS} iterations of CPUForceAtlas2::doStep (Barnes-Hut, "
                          "1 thread) on the whole graph, from the same positions"}
            rec["layout"]["reference_cpu"] = summary(ref.positions(), og.sources, og.targets, 64)
    return rec


def extras(args, local, out, t_start):
    """The batched (4096 SBM graphs), the large (R-MAT scale 23) and the CPU
    baseline (BA 10k) workloads, measured in the same run as compact
    sub-records of the default line."""
    import argparse as _ap
    sub = _ap.Namespace(**vars(args))
    sub.steps, sub.warmup, sub.no_cpu_baseline = SUB_STEPS, SUB_WARMUP, args.no_cpu_baseline
    keys = ("metric", "value", "unit", "steps", "warmup", "ms_per_step", "config", "clocks",
            "gpu_launches", "e2e", "roofline", "cpu_baseline", "autotune", "graph_iters_per_s",
            "fp64_checks", "tree", "cpu_baseline_skipped")
    if time.perf_counter() - t_start < EXTRAS_BUDGET_S:
        try:
            sub.workload = "batched"
            out["batched"] = _compact(run_batched(sub, 1, 0, local), keys)
        except Exception as e:  # a failed sub-record leaves the main line intact
            out["batched"] = {"error": repr(e)}
    else:
        out["batched"] = {"skipped": "over the default run's wall-clock budget"}
    if time.perf_counter() - t_start < EXTRAS_BUDGET_S:
        try:
            sub.workload = "rmat23"
            sub.no_cpu_baseline = True
            rec = run_ours(sub, 1, 0, local, fp64_n=1, correction=False)
            rec["kernels_ms_alone"] = {k: v["ms_alone"] for k, v in rec.get("kernels", {}).items()
                                       if v.get("ms_alone")}
            out["rmat23"] = _compact(rec, keys + ("kernels_ms_alone",))
        except Exception as e:
            out["rmat23"] = {"error": repr(e)}
    else:
        out["rmat23"] = {"skipped": "over the default run's wall-clock budget"}
    try:
        out["config1"] = config1_record(local, args.no_cpu_baseline)
    except Exception as e:
        out["config1"] = {"error": repr(e)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-correction", action="store_true",
                    help="leave out the far-field correction report (theta sweep, learned rows)")
    ap.add_argument("--learned", type=float, default=None,
                    help="rmat20: time the workload with the learned correction at this theta "
                         "(trained first on R-MAT scale 16)")
    ap.add_argument("--no-extras", action="store_true",
                    help="rmat20 at N=1 only: leave out the batched and rmat23 sub-records")
    ap.add_argument("--theta", type=float, default=1.0,
                    help="Barnes-Hut opening parameter of the rmat20 workload (reference: 1)")
    ap.add_argument("--multipole", type=int, default=1, choices=[1, 2],
                    help="1: cells as point masses (reference); 2: with the quadrupole term")
    ap.add_argument("--workload", default="rmat20", choices=["rmat20", "rmat23", "batched"],
                    help="rmat20: the R-MAT scale-20 graph (default); rmat23: the large "
                         "R-MAT scale-23 run; batched: 4096 SBM graphs")
    args = ap.parse_args()
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.workload == "batched":
            if args.impl == "reference":
                if rank == 0:
                    print(json.dumps({"impl": "reference", "unavailable": "the batched workload "
                                      "has no reference arm; its cpu_baseline is in the "
                                      "default arm's line"}))
            else:
                out = run_batched(args, world, rank, local)
                if out is not None:
                    print(json.dumps(out))
        elif args.impl == "reference" and args.workload != "rmat20":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "one CPUForceAtlas2::doStep "
                                  "at R-MAT scale 23 takes minutes; the reference arm runs on "
                                  "the rmat20 workload"}))
        elif args.impl == "reference":
            run_reference(args, world, rank)
        else:
            t_start = time.perf_counter()
            out = run_ours(args, world, rank, local)
            if (out is not None and world == 1 and args.workload == "rmat20"
                    and not args.no_extras):
                extras(args, local, out, t_start)
            if out is not None:
                print(json.dumps(out))
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
