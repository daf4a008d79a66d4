#!/usr/bin/env python
"""Benchmark of the B200 SPH step: particle-steps/s on the two-phase
submerged-soil workload (912,016 particles: 4.0 m x 1.0 m domain, dx 0.002 m,
soil block 1.0 m x 0.4 m under 0.8 m of water, FP32 pair arithmetic with FP64
positions/time/leapfrog state).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one full leapfrog step of time_integration (declarations_sph.f90:525)
over both phases, neighbour search included.  Prints one JSON line (rank 0).

Under torchrun (N > 1) every rank steps its own replica of the workload on
its own GPU (the step has no exchange between replicas: weak scaling, no
collective on the data path); the timed region is bracketed by a barrier
and device synchronisation on every rank and the time is the max over ranks.

--impl reference times the reference's CPU path on the host cores: the C
restatement of the serial Fortran step (the reference itself has no C/CUDA
code and no Fortran compiler exists here), on a bounded sub-domain sample of
the same workload at the same spacing.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s at 1M particles (two-phase water/soil SPH step, 1 B200)"
UNIT = "particle-steps/s"
WORKLOAD = "two_phase_912k"

# Algorithmic HBM bytes per particle of each kernel in FP32 mode: the
# particle's own data read once and its results written once (neighbour
# records are re-read from L1/L2 and not counted).  The leapfrog predictor
# runs inside `gather`; the cross pairs and the corrector run inside the last
# pass of each phase (`water_pass_b`, `soil_pass`), so their state traffic is
# counted there.
CORRECTOR_WATER = 16 + 8 + 4 + 16 + 8 + 16 + 8 + 32 + 16 + 4   # rho, rho_min, drho, vof, vof_min, v_min, av, x rw, v, itype
CORRECTOR_SOIL = 16 + 4 + 64 + 16 + 16 + 8 + 32 + 16 + 4 + 4    # rho, rho_min, drho, p/s rw, ds, dp, v_min, av, x rw, v, itype, fail
ALG_BYTES = {
    # perm, xs, hs, recA, c, rho, vof, itype -> c, drho, p, s(3), recB, countiac
    "water_pass_a": 4 + 16 + 8 + 16 + 8 + 8 + 8 + 4 + 8 + 4 + 8 + 24 + 32 + 4,
    # perm, xs, hs, recA, recB, itype -> dv, av, dvof, vof2, countiac + corrector
    "water_pass_b": 4 + 16 + 8 + 16 + 32 + 4 + 8 + 8 + 4 + 4 + 4 + CORRECTOR_WATER,
    # perm, xs, hs, recA, recB, itype, p, s(3), eps_p rw, fail -> dv, av, drho, ds(3), dp, c, t(3), vcc, countiac;
    # rho -> vof + corrector
    "soil_pass": 4 + 16 + 8 + 16 + 32 + 4 + 8 + 24 + 16 + 4 + 8 + 8 + 4 + 12 + 4 + 8 + 12 + 4 + 4 + 8 + 8 + CORRECTOR_SOIL,
}
# Whole-step algorithmic bytes per particle-step (FP32 pair data, FP64 state):
# the compulsory state read + write once per step plus the cell key; water:
# x 32, v 16, rho 8, drho 8, dv 16, mass 4, type 4, key 8, vof 8, dvof 8;
# soil: the same without vof/dvof, plus vof 8, stress and p 32, their rates 32.
# The roofline of the dominant kernel charges its phase's full per-step bytes
# to it (neighbour re-reads and the per-pass record traffic are not counted).
STEP_BYTES = {"water": 112, "soil": 168}
# FP32 peak of the part (148 SMs x 128 FP32 lanes x 2 flops per FMA per clock)
FP32_LANES_PER_SM = 128


def clocks_sampler(stop, out):
    cmd = ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
           "--format=csv,noheader,nounits", "-lms", "200"]
    try:
        p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except OSError:
        return
    def reader():
        for line in p.stdout:
            out.append(line.strip())
    t = threading.Thread(target=reader, daemon=True)
    t.start()
    stop.wait()
    p.terminate()
    try:
        p.wait(timeout=5)
    except Exception:
        p.kill()
    t.join(timeout=2)


def summarize_clocks(lines, device_index):
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for l in lines:
        f = [x.strip() for x in l.split(",")]
        if len(f) < 9 or f[0] != str(device_index):
            continue
        try:
            sm.append(float(f[1])); mx.append(float(f[2]))
        except ValueError:
            continue
        for n, v in zip(names, f[5:9]):
            if v.lower().startswith("active"):
                reasons.add(n)
    if not sm:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_issue():
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_issue.json")) as f:
            return json.load(f)["warp_instructions_per_particle"]
    except Exception:
        return {}


def ncu_traffic():
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def ncu_flops():
    """FP32 flops per pair-end of each pass (ncu's executed FADD + FMUL +
    2 FFMA, over the neighbour pairs each pass evaluated), from
    profiles/ncu_flops.json."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_flops.json")) as f:
            return json.load(f)["fp32_flops_per_pair_end"]
    except Exception:
        return {}


# A sample of the workload with the same spacing and physics and the same
# water:soil particle ratio (88.4 : 11.6, virtual particles included):
# 51,508 water and 6,758 soil particles.
def workload_config(workload: str, forchheimer_b: float, world: int) -> dict:
    """The `config` of both arms' JSON lines (the same dict for the same run)."""
    sizes = {WORKLOAD: (912016, 806008, 106008), "two_phase_456k": (508016, 404008, 104008)}
    if workload not in sizes:
        return {"workload": workload, "parallelism": f"replicas{world}"}
    n, nw, ns = sizes[workload]
    return {"workload": workload, "particles": n, "water": nw, "soil": ns, "dx": 0.002, "skf": 1,
            "parallelism": f"replicas{world}",
            "drag": ("darcy (the reference's law)" if forchheimer_b == 0
                     else "darcy-forchheimer b=%g s^2/m^2" % forchheimer_b),
            "l2": "inputs larger than L2 (state ~%.0f MB)" % (n * 250 / 1e6)}


SUBDOMAIN = dict(width=1.0, height=0.25, block_w=0.21, block_h=0.1, water_h=0.2)
SUBDOMAIN_TEXT = "1.0 m x 0.2 m water, 0.21 m x 0.1 m soil block, dx 0.002 m, water:soil 88.4:11.6 as the workload"


def _oracle_worker(args):
    """One serial oracle on its own copy of the sub-domain; every worker
    starts its timed steps behind the same barrier."""
    steps, warmup, barrier = args
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, ROOT)
    from oracle import Oracle
    from sources_b200 import scenes
    s = scenes.two_phase(**SUBDOMAIN)
    o = Oracle(s)
    rc = o.time_integration(warmup)
    barrier.wait()
    t0 = time.perf_counter()
    rc = rc or o.time_integration(steps)
    return s.n_particles, time.perf_counter() - t0, rc


def host_cores() -> int:
    """Host threads this process may run on (SPHG_HOST_CORES caps it)."""
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    cap = int(os.environ.get("SPHG_HOST_CORES", "0") or 0)
    return min(n, cap) if cap > 0 else n


def oracle_throughput(steps: int, warmup: int, cores: int):
    """The serial C restatement of the reference step (the reference's own
    path is serial) on every host core at once: one independent instance per
    core, each on its own copy of a 58,266-particle sub-domain of the workload.
    Aggregate particle-steps/s = all instances' particle-steps / the slowest
    instance's time (all start together).  Spawned processes: no fork after
    the CUDA context exists."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    barrier = mgr.Barrier(cores)
    with ctx.Pool(cores) as pool:
        res = pool.map(_oracle_worker, [(steps, warmup, barrier)] * cores)
    mgr.shutdown()
    if any(r[2] for r in res):
        raise RuntimeError(f"oracle step failed: {[r[2] for r in res]}")
    n = res[0][0]
    dt = max(r[1] for r in res)
    return n, dt, n * steps * cores / dt


def cpu_baseline(steps: int, cores: int | None = None):
    """The oracle port of the serial reference step, one instance per host
    core on a sub-domain sample of the workload (same spacing and physics),
    and the same sample on one core alone (the reference's serial path)."""
    cores = cores or host_cores()
    n, dt, v = oracle_throughput(steps, 1, cores)
    _, dt1, v1 = oracle_throughput(steps, 1, 1)
    return {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"serial C restatement of the Fortran step, one instance per core on {cores} cores, each "
                      f"{steps} leapfrog steps of its own {n}-particle sub-domain of the workload ({SUBDOMAIN_TEXT})",
            "seconds": dt,
            "serial": {"value": v1, "unit": UNIT, "cores": 1, "seconds": dt1}}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    cores = host_cores()
    try:
        n, dt, v = oracle_throughput(args.steps, args.warmup, cores)
    except RuntimeError as e:
        print(json.dumps({"impl": "reference", "unavailable": str(e)}))
        return 0
    sample = (f"serial C restatement of the Fortran step (the reference has no compilable C/CUDA and no Fortran "
              f"compiler is present), one instance per host core on {cores} cores; each step is one leapfrog step "
              f"of every instance's own {n}-particle sub-domain of the workload ({SUBDOMAIN_TEXT})")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (deterministic lattice scene)",
            "config": workload_config(args.workload, args.forchheimer_b, world),
            "precision": "fp64 (the reference's arithmetic)",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ensemble(args, rank, world, torch, dist):
    """256 scenes (Philox-keyed seeds 0..255: dam-breaks, dry and submerged
    collapses of 2k-60k particles at dx 0.004 m), each kind packed into one
    context, cell factor and reorder interval autotuned per group."""
    from sources_b200 import ensemble, replicas
    t0 = time.perf_counter()
    ens = ensemble.Ensemble(ensemble.specs(256))
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream()
    ens.set_stream(stream.cuda_stream)
    ens.time_integration(args.warmup)
    torch.cuda.synchronize()
    replicas.barrier(dist if world > 1 else None)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ens.time_integration(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = replicas.max_over_ranks(e0.elapsed_time(e1), dist if world > 1 else None, device="cuda")
    n = ens.n_particles
    groups = {g.kind: {"scenes": len(g.members), "particles": g.scene.n_particles, "tuning": list(g.tuning),
                       "autotune_ms_per_step": {",".join(map(str, k)): v for k, v in ens.tuning_table.get(g.kind, {}).items()}}
              for g in ens.groups}
    ens.close()
    if rank == 0:
        print(json.dumps({"metric": "particle-steps/s, 256-scene batched ensemble", "value":
                          replicas.weak_scaling_value(world, n, args.steps, ms), "unit": UNIT, "n_gpus": world,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                          "higher_is_better": True, "scaling": "weak", "dtype": "f32",
                          "config": {"workload": "ensemble_256", "scenes": 256, "particles": n, "groups": groups,
                                     "setup_s": setup_s}}))
    return 0


def learned_arm(solver, scene, torch, plain_value, strides):
    """The learned stepper on the same scene, beside the plain solver: a
    history of 5 strides (k = 10 steps) from the plain solver, then `strides`
    learned strides timed end to end (graph search, network, stride update and
    the fallback-gate sums, wall clock with a synchronisation per stride), and
    the plain solver's own strides from the same state, timed the same way,
    as the yardstick of the speed and of the position error."""
    import numpy as np
    from sources_b200 import learn
    if not os.path.exists(learn.DEFAULT_WEIGHTS):
        return {"unavailable": "no trained weights at sources_b200/data/learned_weights.npz"}
    net = learn.MPNet.from_state(dict(np.load(learn.DEFAULT_WEIGHTS)))
    x0 = torch.from_numpy(np.concatenate([P.x for P in scene.phases])).to("cuda")   # the initial lattice
    hist = learn.scene_rollout(solver, scene, "submerged", learn.HIST, x0=x0)
    learn.LearnedStepper(net, hist, learn.HIST, "net").step()        # warm-up: buffers, graph
    st = learn.LearnedStepper(net, hist, learn.HIST, "net")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(strides):
        st.step()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    n = hist.X.shape[1]
    # the plain solver's strides from the same state, timed the same way (wall clock, a
    # synchronisation per stride, the positions kept after each stride); its final
    # positions are the yardstick of the learned ones
    sizes = [P.n for P in scene.phases]
    xp = torch.empty((n, 2), dtype=torch.float64, device="cuda")
    solver.set_stream(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(strides):
        solver.time_integration(learn.K_STRIDE)
        a = 0
        for k, nk in enumerate(sizes):
            solver.export_xv(k + 1, xp[a:a + nk].data_ptr(), None)
            a += nk
        torch.cuda.synchronize()
    wall_plain = time.perf_counter() - t0
    real = hist.nodes["type"] != learn.GNN_BOUNDARY
    d = ((st.x - xp).norm(dim=1).cpu().numpy()[real]) / hist.dx
    value = n * strides * learn.K_STRIDE / wall
    return {"value": value, "unit": UNIT, "vs_plain": value / plain_value, "stride_steps": learn.K_STRIDE,
            "strides": strides, "ms_per_stride": wall / strides * 1e3,
            "plain_ms_per_stride_same_timing": wall_plain / strides * 1e3, "vs_plain_same_timing": wall_plain / wall,
            "edges": int(st.batch.E),
            "position_error_dx": {"mean": float(d.mean()), "p99": float(np.percentile(d, 99)),
                                  "max": float(d.max())},
            "weights": "sources_b200/data/learned_weights.npz (trained on the 4 mm ensemble)",
            "network": f"message passing, {learn.LAYERS} layers, width {learn.L_WIDTH}, bf16 tcgen05"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=100, help="steps of the end-to-end reference loop")
    ap.add_argument("--full-state-steps", type=int, default=5,
                    help="steps of the end-to-end run that copies the full state every step")
    ap.add_argument("--cpu-steps", type=int, default=60)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-stepper arm")
    ap.add_argument("--fp64-steps", type=int, default=20, help="steps of the FP64-mode timing (0: skip)")
    ap.add_argument("--learned-strides", type=int, default=5)
    ap.add_argument("--forchheimer-b", type=float, default=0.0,
                    help="Forchheimer coefficient of the water-soil drag [s^2/m^2] (0: the reference's Darcy law)")
    ap.add_argument("--workload", default=WORKLOAD, choices=[WORKLOAD, "two_phase_456k", "ensemble_256"],
                    help="two_phase_456k: the same scene 2.0 m wide (for profiler captures); "
                         "ensemble_256: 256 uneven scenes stepped as three batched groups")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)

    import numpy as np
    import torch
    import torch.distributed as dist

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    from sources_b200 import Solver, build, replicas, scenes
    from sources_b200.abi import SPHG_FP32, Stats

    build.build()
    if args.workload == "ensemble_256":
        return run_ensemble(args, rank, world, torch, dist)
    if args.workload == WORKLOAD:
        scene = scenes.two_phase(precision=SPHG_FP32, forchheimer_b=args.forchheimer_b)
    else:
        scene = scenes.two_phase(width=2.0, precision=SPHG_FP32, forchheimer_b=args.forchheimer_b)
    n = scene.n_particles
    stream = torch.cuda.current_stream()
    solver = Solver(scene)
    solver.set_stream(stream.cuda_stream)

    solver.time_integration(args.warmup)
    torch.cuda.synchronize()

    # ---- device-resident timed region
    samples, stop = [], threading.Event()
    th = threading.Thread(target=clocks_sampler, args=(stop, samples), daemon=True)
    th.start()
    time.sleep(0.3)
    launches0 = solver.kernel_report()["launches"]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    solver.time_integration(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    launches = solver.kernel_report()["launches"] - launches0
    # per-kernel CUDA-event times on the library's stream over a second window
    # of the same K steps (events between launches would slow the headline one)
    solver.profile(True)
    solver.time_integration(args.steps)
    rep = solver.kernel_report()
    solver.profile(False)
    stop.set()
    th.join(timeout=10)
    clocks = summarize_clocks(samples, local)
    ms = replicas.max_over_ranks(ms, dist if world > 1 else None, device="cuda")
    value = replicas.weak_scaling_value(world, n, args.steps, ms)

    # ---- dominant kernel and its roofline
    kern = rep["kernels"]
    top = max(kern.items(), key=lambda kv: kv[1][1])
    top_name, (top_launches, top_ms) = top[0], top[1]
    avg_ms = top_ms / max(top_launches, 1)

    def phase_n(name):
        return scene.phases[1].n if name == "soil_pass" else scene.phases[0].n

    def step_bytes_of(name):   # the per-step bytes of the particles the kernel covers
        return STEP_BYTES["soil" if name == "soil_pass" else "water"] * phase_n(name)

    units = phase_n(top_name)
    alg = step_bytes_of(top_name)
    peak, peak_kind = measured_peak_hbm()
    achieved = alg / (avg_ms / 1000.0) / 1e9
    tr = ncu_traffic().get(top_name)
    step_bytes = STEP_BYTES["water"] * scene.phases[0].n + STEP_BYTES["soil"] * scene.phases[1].n
    step_ms = ms / args.steps
    # issue roofline of the same kernel: warp instructions per launch (ncu count
    # per particle x particles) over the live launch time, against 4 schedulers
    # x 1 warp-instruction per clock per SM at the SM clock seen under load
    ipp = ncu_issue()
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    issue_peak = sms * 4 * mhz * 1e6
    fp32_peak = sms * FP32_LANES_PER_SM * 2 * mhz * 1e6
    st = solver.stats()
    pair_ends = {"water_pass_a": 2 * st.niac[0], "water_pass_b": 2 * st.niac[0] + st.niac[2],
                 "soil_pass": 2 * st.niac[1] + st.niac[2]}
    fpp = ncu_flops()

    def issue(name, ms_launch, particles):
        if name not in ipp:
            return None
        inst = ipp[name] * particles
        return {"warp_inst_per_launch": inst, "achieved": inst / (ms_launch / 1000.0), "peak": issue_peak,
                "unit": "warp-inst/s", "frac": inst / (ms_launch / 1000.0) / issue_peak}

    def fp32(name, ms_launch):
        if name not in fpp or name not in pair_ends:
            return None
        fl = fpp[name] * pair_ends[name]
        return {"flops_per_pair_end": fpp[name], "pair_ends_per_launch": int(pair_ends[name]),
                "achieved": fl / (ms_launch / 1000.0) / 1e12, "peak": fp32_peak / 1e12, "unit": "TFLOP/s",
                "frac": fl / (ms_launch / 1000.0) / fp32_peak}

    def launch_ms(k):
        return kern[k][1] / max(kern[k][0], 1)

    roofline = {"bound": "hbm", "kernel": top_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind, "traffic": tr,
                "alg_bytes_per_launch": alg,
                "alg_bytes_basis": "per-step state bytes of the particles the kernel covers: 112 B per water "
                                   "particle-step, 168 B per soil particle-step",
                "avg_launch_ms": avg_ms,
                "issue": issue(top_name, avg_ms, units),
                "fp32": fp32(top_name, avg_ms),
                "step": {"alg_bytes": step_bytes, "achieved_gbs": step_bytes / (step_ms / 1000.0) / 1e9,
                         "frac": step_bytes / (step_ms / 1000.0) / 1e9 / peak},
                "kernels_ms_per_step": {k: v[1] / args.steps for k, v in kern.items()},
                "passes": {k: {"alg_bytes": step_bytes_of(k), "avg_ms": launch_ms(k),
                               "achieved_gbs": step_bytes_of(k) / (launch_ms(k) / 1000.0) / 1e9,
                               "frac": step_bytes_of(k) / (launch_ms(k) / 1000.0) / 1e9 / peak,
                               "per_pass_bytes": ALG_BYTES[k] * phase_n(k),
                               "per_pass_frac": ALG_BYTES[k] * phase_n(k) / (launch_ms(k) / 1000.0) / 1e9 / peak,
                               "traffic": ncu_traffic().get(k),
                               "issue": issue(k, launch_ms(k), phase_n(k)),
                               "fp32": fp32(k, launch_ms(k))}
                           for k in ALG_BYTES if k in kern}}

    # ---- end to end through the C ABI with pinned host buffers
    def pinned(shape, dtype):
        t = torch.zeros(shape, dtype=torch.float64 if dtype == np.float64 else torch.int32, pin_memory=True)
        return t.numpy()
    host = [P.copy(alloc=pinned) for P in scene.phases]
    for k in range(len(host)):
        solver.download(k + 1, into=host[k])
    torch.cuda.synchronize()
    state_bytes = sum(P.nbytes() for P in host)
    stats_bytes = ctypes.sizeof(Stats)

    def timed(fn):
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        return replicas.max_over_ranks(time.perf_counter() - t0, dist if world > 1 else None, device="cuda")

    # The reference's own host loop (declarations_sph.f90:535-885): the input
    # state goes in once, every step is one call whose statistics come back,
    # the full state comes out at the output step.
    def reference_loop():
        for k, P in enumerate(host):
            solver.upload(k + 1, P)
        for _ in range(args.e2e_steps):
            solver.time_integration(1)
            solver.stats()
        for k in range(len(host)):
            solver.download(k + 1, into=host[k])

    # A host that owns every array and hands all of them over every step.
    def full_state():
        for _ in range(args.full_state_steps):
            for k, P in enumerate(host):
                solver.upload(k + 1, P)
            solver.time_integration(1)
            for k in range(len(host)):
                solver.download(k + 1, into=host[k])

    e2e_s = timed(reference_loop)
    full_s = timed(full_state)
    K = args.e2e_steps
    e2e = {"value": world * n * K / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": (state_bytes + K * 16) / K,
           "d2h_bytes_per_step": (state_bytes + K * stats_bytes) / K, "steps": K,
           "mode": "the reference's time loop through the C ABI on pinned host arrays: upload the full state, "
                   "then every step one sphg_time_integration call (itimestep and time in, status out) and its "
                   "statistics read back (sphg_stats), then download the full state (the output step)",
           "full_state_every_step": {"value": world * n * args.full_state_steps / full_s, "unit": UNIT,
                                     "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
                                     "steps": args.full_state_steps,
                                     "mode": "every step: upload the full state, one step, download the full state"}}

    # ---- the FP64 parity mode on the same scene (every field and sum in double)
    fp64 = None
    if args.fp64_steps > 0:
        from sources_b200.abi import SPHG_FP64
        s64 = scene.copy()
        s64.params.precision = SPHG_FP64
        with Solver(s64) as g64:
            g64.set_stream(stream.cuda_stream)
            g64.time_integration(3)
            torch.cuda.synchronize()
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f0.record(stream)
            g64.time_integration(args.fp64_steps)
            f1.record(stream)
            torch.cuda.synchronize()
            ms64 = replicas.max_over_ranks(f0.elapsed_time(f1), dist if world > 1 else None, device="cuda")
        fp64 = {"value": replicas.weak_scaling_value(world, n, args.fp64_steps, ms64), "unit": UNIT,
                "ms_per_step": ms64 / args.fp64_steps, "steps": args.fp64_steps, "warmup": 3, "dtype": "f64",
                "mode": "FP64 parity mode: pair arithmetic, rates and state all in double"}

    learned = None
    if not args.no_learned and args.workload == WORKLOAD:
        learned = learned_arm(solver, scene, torch, value / world, args.learned_strides)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args.cpu_steps)

    solver.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (deterministic lattice scene, no dataset)",
                "config": workload_config(args.workload, args.forchheimer_b, world),
                "precision": "fp32 pairs / fp64 state",
                "pairs": {"water": int(st.niac[0]), "soil": int(st.niac[1]), "cross": int(st.niac[2])},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clocks, "learned": learned, "fp64_mode": fp64}
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
