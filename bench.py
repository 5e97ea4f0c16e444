"""Benchmark: particle-steps/s of Velocity-Verlet steps with Barnes-Hut gravity.

Workload (default): N = 2^20 equal-mass Plummer sphere (a = 1, G = 1, seed =
rank), theta = 0.5, eps = 0.01, dt = 1e-3, leaf capacity 8, FP32-compensated
pair terms with FP64 state.  One step = one Velocity-Verlet tick on the device:
bounding cube, descent keys, radix sort, octree + centre of mass, theta walk,
kick/drift.  The walk is the group walk (one interaction list per cell group of
at most 64 bodies); --walk body times the per-body walk, and the other walk is
timed beside the default one in the JSON line.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one rank per GPU): every rank integrates its own
independent system (replicas, weak scaling; the path has no exchange step);
time is the max over ranks.  `--impl reference` times the reference's CPU
algorithm (the C++ oracle restatement: serial pointer-octree build + threaded
walk, two force evaluations per tick as the reference schedule runs them) on
the host cores, rank 0 only: whole ticks of all N bodies, as many of the
requested steps as fit in REFERENCE_BUDGET_S, with the count it ran.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
for _p in (REPO, os.path.join(REPO, "phys-rs_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = ("particle-steps/s, 1M-body BH θ=0.5: FP32-comp vs FP64 GPU at ≤1e-6 accel error")
FLOPS_PER_INTERACTION = 20  # Nyland, Harris & Prins (GPU Gems 3, ch. 31)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="bh",
                    choices=["bh", "galaxy", "ensemble", "direct", "adjoint", "bh_shared"],
                    help="bh: 2^20 Plummer Barnes-Hut (default; one replica per GPU); "
                         "galaxy: 2^24 disk+halo BH; ensemble: 16384 small systems; "
                         "direct: 1024-body direct sum; adjoint: 4096-body trajectory "
                         "gradient; bh_shared: one 2^20 Plummer system split by targets "
                         "over the GPUs (all-gather of accelerations per evaluation)")
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--leaf-cap", type=int, default=8)
    ap.add_argument("--walk", default="group", choices=["body", "group"],
                    help="Barnes-Hut walk: per body (the reference's) or per 64-body group")
    ap.add_argument("--theta", type=float, default=None)
    ap.add_argument("--eps", type=float, default=None)
    ap.add_argument("--dt", type=float, default=None)
    ap.add_argument("--ens-steps", type=int, default=10000, help="ensemble steps per bench step")
    ap.add_argument("--adj-steps", type=int, default=1000,
                    help="Verlet steps per trajectory gradient (adjoint workload)")
    ap.add_argument("--no-extras", action="store_true", help="skip FP64 comparison and accuracy")
    ap.add_argument("--quick", action="store_true",
                    help="device-resident timing only (no e2e, extras, CPU baseline): profiling")
    ap.add_argument("--precision", default="f32c", choices=["f32c", "f64", "f64_exact"],
                    help="with --quick: the precision of the timed Barnes-Hut steps (the full "
                         "line always times F32C, the metric's form)")
    a = ap.parse_args()
    if a.precision != "f32c" and not a.quick:
        ap.error("--precision other than f32c needs --quick")
    defaults = {  # n, theta, eps, dt per workload shape
        "bh": (1 << 20, 0.5, 0.01, 1e-3), "galaxy": (1 << 24, 0.6, 0.02, 5e-4),
        "bh_shared": (1 << 20, 0.5, 0.01, 1e-3),
        "ensemble": (16384, 0.5, 1e-3, 1e-4), "direct": (1024, 0.5, 0.01, 1e-3),
        "adjoint": (4096, 0.5, 0.01, 1e-3)}[a.workload]
    a.n = a.n if a.n is not None else defaults[0]
    a.theta = a.theta if a.theta is not None else defaults[1]
    a.eps = a.eps if a.eps is not None else defaults[2]
    a.dt = a.dt if a.dt is not None else defaults[3]
    return a


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference_tick_sampled(pos, vel, m, args, sample, rng, nthreads):
    """One reference Velocity-Verlet tick at full N on the host, with the
    walk timed on `sample` random targets and scaled to N (two force
    evaluations per tick, src/main.rs:109,128).  Used only where a full tick
    takes minutes (the 2^24 galaxy).  Returns seconds per tick and the parts."""
    import oracle
    n = len(m)
    targets = np.sort(rng.choice(n, size=min(sample, n), replace=False))
    t0 = time.perf_counter()
    _, tm = oracle.bh_forces_targets(pos, m, 1.0, args.eps, args.theta, targets,
                                     nthreads=nthreads)
    wall = time.perf_counter() - t0
    build_s, walk_s = tm[0], tm[1] * n / len(targets)
    t1 = time.perf_counter()
    x = pos + vel * args.dt
    _ = vel + x * 0.5 * args.dt
    vv_s = time.perf_counter() - t1
    eval_s = build_s + walk_s
    return 2.0 * eval_s + vv_s, {"build_s": build_s, "walk_s_scaled": walk_s, "vv_s": vv_s,
                                 "sample_targets": len(targets), "wall_s": wall}


def cpu_reference_eval(pos, m, args, nthreads):
    """One whole barnes_hut_gravity_system force evaluation of all N bodies
    on the host: the serial pointer-octree build and the threaded walk of
    every target (gravity_tree.rs:260-338).  Returns (seconds, build_s,
    walk_s), all measured."""
    import oracle
    tm = np.zeros(2)
    t0 = time.perf_counter()
    oracle.bh_forces(pos, m, 1.0, args.eps, args.theta, nthreads=nthreads, timings=tm)
    return time.perf_counter() - t0, float(tm[0]), float(tm[1])


def cpu_reference_tick(pos, vel, m, args, nthreads):
    """One reference Velocity-Verlet tick of all N bodies on the host, as the
    reference schedule runs it (src/main.rs:103-140): force pass, position
    step, force pass, velocity step, each force pass a whole Barnes-Hut
    evaluation.  Returns the measured seconds."""
    import oracle
    t0 = time.perf_counter()
    oracle.vv_run(pos, vel, m, 1.0, args.eps, args.dt, 1, method="bh", theta=args.theta,
                  nthreads=nthreads)
    return time.perf_counter() - t0


# Host seconds the reference arm spends in its timed ticks: each full tick
# of 2^20 bodies takes several seconds, so the arm runs as many of the
# requested ticks as fit and states the number it ran.
REFERENCE_BUDGET_S = 90.0


def run_reference(args, ws, rank):
    import oracle
    oracle.lib()
    if rank != 0:
        return 0
    import physgpu.ics as ics
    nthreads = oracle.ncpu()
    if args.workload == "galaxy":
        pos, vel, m = ics.galaxy(args.n, seed=0)
        rng = np.random.default_rng(1)
        for _ in range(args.warmup):
            cpu_reference_tick_sampled(pos, vel, m, args, 16384, rng, nthreads)
        ticks, parts = [], None
        for _ in range(args.steps):
            t, parts = cpu_reference_tick_sampled(pos, vel, m, args, 16384, rng, nthreads)
            ticks.append(t)
        t_tick = sum(ticks) / len(ticks)
        steps, warmup, extra = args.steps, args.warmup, {}
        sample = ("per tick: serial pointer-octree build of all %d bodies + threaded walk of "
                  "%d random targets scaled to N, x2 force evaluations per tick; last tick %s" % (
                      args.n, parts["sample_targets"],
                      json.dumps({k: round(v, 4) for k, v in parts.items()})))
    else:
        pos, vel, m = ics.plummer(args.n, seed=0)
        # warm-up: one whole force evaluation, timed by parts
        eval_s, build_s, walk_s = cpu_reference_eval(pos, m, args, nthreads)
        warmup = 1
        steps = max(1, min(args.steps, int(REFERENCE_BUDGET_S // (2.0 * eval_s))))
        ticks = [cpu_reference_tick(pos, vel, m, args, nthreads) for _ in range(steps)]
        t_tick = sum(ticks) / len(ticks)
        one_eval_tick = t_tick - eval_s
        extra = {"steps_requested": args.steps, "warmup_requested": args.warmup,
                 "tick_s": ticks,
                 "one_evaluation": {"eval_s": eval_s, "build_s": build_s, "walk_s": walk_s,
                                    "tick_s": one_eval_tick,
                                    "value": args.n / one_eval_tick,
                                    "note": "the same tick with one force evaluation, as the "
                                            "device path runs it (the reference schedule's two "
                                            "passes per tick are at the same positions)"}}
        sample = ("%d whole reference ticks of all %d bodies (serial pointer-octree build + "
                  "threaded walk of every target, two force evaluations per tick, "
                  "src/main.rs:109,128), each timed; no scaling" % (steps, args.n))
    value = args.n / t_tick
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "particle-steps/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": warmup,
        "ms_per_step": t_tick * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Plummer)",
        "config": dict(workload_config(args, precision="f64", leaf_cap=1),
                       l2="not applicable (host cores)"),
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": nthreads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    line.update(extra)
    print(json.dumps(line), flush=True)
    return 0


def workload_config(args, precision, leaf_cap, walk="body"):
    galaxy = args.workload == "galaxy"
    return {"workload": ("barnes_hut_galaxy_n%d" if galaxy else "barnes_hut_plummer_n%d") % args.n,
            "n": args.n, "theta": args.theta, "eps": args.eps, "G": 1.0, "dt": args.dt,
            "leaf_cap": leaf_cap, "precision": precision,
            "walk": ("per body (the reference's criterion per target)" if walk == "body" else
                     "per 64-body group (criterion at the group box's nearest point)"),
            "ics": ("30% exponential disk (R_d=1, sech^2 z0=0.1) + 70% NFW halo (r_s=3, cut 30), "
                    "seed=rank" if galaxy else "Plummer a=1, equal masses 1/N, seed=rank"),
            "l2": "flushed between timed steps (256 MiB write)"}


# DRAM bytes (read + write) of one launch of the dominant kernel for the
# default workload (N = 2^20 Plummer, theta 0.5, leaf capacity 8, F32C), each
# from one ncu capture of this binary at full size:
#   group walk, geval_kernel<true>: dram__bytes_read.sum 471.8 MB +
#     dram__bytes_write.sum 52.1 MB;
#   per-body walk, walk2_kernel: 131.8 MB + 25.3 MB.
WALK_TRAFFIC_BYTES = {"group": 523.97e6, "body": 157.05e6}


def walk_traffic(args):
    if (args.workload, args.n, args.theta, args.leaf_cap) == ("bh", 1 << 20, 0.5, 8):
        return WALK_TRAFFIC_BYTES[args.walk]
    return None


def run_ours(args, ws, rank, local):
    import torch

    import physgpu
    import physgpu.dist as dist
    import physgpu.ics as ics
    from physgpu import BARNES_HUT, F32C, F64, make_params

    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local))
    ctx = physgpu.Context(local)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    if args.workload == "galaxy":
        pos, vel, m = ics.galaxy(args.n, seed=rank)
    else:
        pos, vel, m = ics.plummer(args.n, seed=rank)
    n = args.n
    flags = physgpu.GROUP_WALK if args.walk == "group" else 0
    p32 = make_params(1.0, args.eps, args.theta, BARNES_HUT, F32C, args.leaf_cap, flags)
    p_timed = p32 if args.precision == "f32c" else make_params(
        1.0, args.eps, args.theta, BARNES_HUT, physgpu.PRECISIONS[args.precision],
        args.leaf_cap, flags)
    p64 = make_params(1.0, args.eps, args.theta, BARNES_HUT, F64, args.leaf_cap, flags)

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed_steps(params, k, flush=True):
        """k ticks, each bracketed by CUDA events on the library's stream,
        L2 flushed between ticks; returns (total_ms, walk_ms_list, interactions)."""
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(k)]
        walk, inter = [], []
        with torch.cuda.stream(stream):
            for i in range(k):
                if flush:
                    flush_buf.fill_(i & 0xff)
                evs[i][0].record(stream)
                ctx.verlet_steps(params, args.dt, 1)
                evs[i][1].record(stream)
                t = ctx.timings()
                walk.append(t["walk_ms"])
                inter.append(t["interactions"])
                eval_ms.append(t["walk_eval_ms"])
                eval_inter.append(t["walk_eval_interactions"])
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in evs), walk, inter

    # ---- device-resident value: F32C ----
    eval_ms, eval_inter = [], []  # group walk: list-evaluation kernel (per timed step)
    ctx.upload(pos, vel, m)
    for _ in range(args.warmup):
        ctx.verlet_steps(p_timed, args.dt, 1)
    launches0 = ctx.timings()["launches"]
    clocks = Clocks(local)
    clocks.start()
    barrier()
    tot_ms, walk_ms, inter = timed_steps(p_timed, args.steps)
    geval_ms, geval_inter = list(eval_ms), list(eval_inter)
    barrier()
    clk = clocks.stop()
    launches = ctx.timings()["launches"] - launches0
    t_max_ms = dist.max_over_ranks(tot_ms, device="cuda")
    value = ws * n * args.steps / (t_max_ms * 1e-3)
    tm = ctx.timings()

    if args.quick:
        if rank == 0:
            print(json.dumps({"quick": True, "value": value, "ms_per_step": t_max_ms / args.steps,
                              "walk_ms": statistics.median(walk_ms),
                              "interactions": statistics.median(inter),
                              "timings": ctx.timings()}), flush=True)
        ctx.close()
        return 0

    # ---- e2e through the C ABI with pinned host buffers ----
    def pinned(k):
        return torch.empty(k, dtype=torch.float64, pin_memory=True)

    X = [pinned(n) for _ in range(3)]
    V = [pinned(n) for _ in range(3)]
    A = [pinned(n) for _ in range(3)]
    M = pinned(n)
    for k in range(3):
        X[k].copy_(torch.from_numpy(np.ascontiguousarray(pos[:, k])))
        V[k].copy_(torch.from_numpy(np.ascontiguousarray(vel[:, k])))
    M.copy_(torch.from_numpy(m))
    ctx.upload(pos, vel, m)
    ctx.gravity_accel(p32, download=False)
    ptr = lambda t: ctypes.cast(t.data_ptr(), ctypes.POINTER(ctypes.c_double))
    lib.phys_state_download(ctx.h, None, None, None, None, None, None, *[ptr(a) for a in A])
    h2d = n * 8 * 10
    d2h = n * 8 * 9

    def e2e_step():
        # one tick on host state in one call: upload of x, v, m and the
        # Acceleration component, the tick, x, v, a back in place (the
        # positions' copy back overlaps the force pass: page-locked arrays)
        st = lib.phys_verlet_tick_host(ctx.h, ctypes.byref(p32), args.dt, n,
                                       *[ptr(a) for a in X], *[ptr(a) for a in V], ptr(M),
                                       *[ptr(a) for a in A])
        if st:
            raise physgpu.PhysError(st, lib.phys_last_error(ctx.h).decode())

    for _ in range(max(1, args.warmup)):
        e2e_step()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = dist.max_over_ranks(e0.elapsed_time(e1), device="cuda")
    e2e_value = ws * n * args.steps / (e2e_ms * 1e-3)

    extras = {}
    if not args.no_extras:
        # ---- FP64 form of the same step (same tree, same workload) ----
        ctx.upload(pos, vel, m)
        for _ in range(args.warmup):
            ctx.verlet_steps(p64, args.dt, 1)
        barrier()
        t64, walk64, _ = timed_steps(p64, args.steps)
        extras["fp64_ms_per_step"] = t64 / args.steps
        extras["fp64_walk_ms"] = statistics.median(walk64)
        extras["speedup_f32c_vs_fp64_step"] = t64 / tot_ms
        # ---- accuracy: F32C vs F64 on the same tree, initial positions ----
        ctx.upload(pos, vel, m)
        a64 = ctx.gravity_accel(p64)
        a32 = ctx.gravity_accel(p32)
        e = np.linalg.norm(a32 - a64, axis=1) / np.linalg.norm(a64, axis=1)
        extras["accel_err_f32c_vs_fp64_same_tree"] = {
            "median": float(np.median(e)), "p99": float(np.quantile(e, 0.99)),
            "max": float(e.max())}
        # ---- BH truncation vs the f64 direct sum on a 65,536-body subsample ----
        sub = np.sort(np.random.default_rng(7).choice(n, size=min(65536, n), replace=False))
        pd = make_params(1.0, args.eps, args.theta, physgpu.DIRECT, F64, 1)
        t0 = time.perf_counter()
        ad = ctx.direct_accel_targets(pd, sub)
        extras["direct_f64_subsample_s"] = time.perf_counter() - t0
        for name, a in (("f32c_bh", a32), ("f64_bh", a64)):
            e = np.linalg.norm(a[sub] - ad, axis=1) / np.linalg.norm(ad, axis=1)
            extras["accel_err_%s_vs_f64_direct_subsample" % name] = {
                "median": float(np.median(e)), "p99": float(np.quantile(e, 0.99)),
                "max": float(e.max()), "targets": int(len(sub))}
        pcap1 = make_params(1.0, args.eps, args.theta, BARNES_HUT, F32C, 1, flags)
        ctx.upload(pos, vel, m)
        for _ in range(2):
            ctx.verlet_steps(pcap1, args.dt, 1)
        c1, _, _ = timed_steps(pcap1, max(2, args.steps // 2))
        extras["leaf_cap1_ms_per_step"] = c1 / max(2, args.steps // 2)
        # ---- the other walk (per body <-> per group), F32C and F64 ----
        other = "body" if args.walk == "group" else "group"
        oflags = physgpu.GROUP_WALK if other == "group" else 0
        for prec, name in ((F32C, "f32c"), (F64, "fp64")):
            po = make_params(1.0, args.eps, args.theta, BARNES_HUT, prec, args.leaf_cap, oflags)
            ctx.upload(pos, vel, m)
            for _ in range(2):
                ctx.verlet_steps(po, args.dt, 1)
            ko = max(2, args.steps // 2)
            to, wo, io = timed_steps(po, ko)
            extras["%s_walk_%s_ms_per_step" % (other, name)] = to / ko
            extras["%s_walk_%s_walk_ms" % (other, name)] = statistics.median(wo)
            extras["%s_walk_%s_interactions" % (other, name)] = statistics.median(io)
            if prec == F32C:
                ctx.upload(pos, vel, m)  # the direct sum above is at the initial positions
                ao = ctx.gravity_accel(po)
                e = np.linalg.norm(ao[sub] - ad, axis=1) / np.linalg.norm(ad, axis=1)
                extras["accel_err_%s_walk_f32c_vs_f64_direct_subsample" % other] = {
                    "median": float(np.median(e)), "p99": float(np.quantile(e, 0.99)),
                    "max": float(e.max())}

        # ---- the bit-exact reference form (F64_EXACT: the reference's walk,
        # insertion-order centre of mass, reference op order), leaf capacity 1 ----
        pex = make_params(1.0, args.eps, args.theta, BARNES_HUT, physgpu.F64_EXACT, 1, 0)
        ctx.upload(pos, vel, m)
        ctx.verlet_steps(pex, args.dt, 1)
        tex, wex, _ = timed_steps(pex, 2)
        extras["exact_f64_bh_ms_per_step"] = tex / 2
        extras["exact_f64_bh_walk_ms"] = statistics.median(wex)
        extras["exact_f64_bh_tree_ms"] = ctx.timings()["tree_ms"]

    # ---- roofline of the dominant kernel (the walk) ----
    fp32_tf, fp32x2_tf, fp64_tf = ctx.probe_peaks()
    fp32_peak = max(fp32_tf, fp32x2_tf)
    walk_med = statistics.median(walk_ms)
    inter_med = statistics.median(inter)
    peak_source = ("measured live: max of FFMA and packed FFMA2 loops on all SMs "
                   "(FMA = 2 flops); ffma %.1f, ffma2 %.1f" % (fp32_tf, fp32x2_tf))
    phases = {k: round(tm[k], 4) for k in ("bbox_ms", "keys_ms", "sort_ms", "tree_ms", "walk_ms")}
    if args.walk == "group":
        # the dominant kernel is the list evaluation: its own events and count
        ev_med = statistics.median(geval_ms)
        ev_inter = statistics.median(geval_inter)
        achieved = FLOPS_PER_INTERACTION * ev_inter / (ev_med * 1e-3) / 1e12
        roof = {"kernel": "geval_kernel<true> (f32c group-walk list evaluation)", "bound": "fp32",
                "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved / fp32_peak, "peak_source": peak_source,
                "flops_per_interaction": FLOPS_PER_INTERACTION,
                "interactions_per_launch": ev_inter, "kernel_ms": ev_med,
                "walk_phase_ms": walk_med, "walk_phase_interactions": inter_med,
                "traffic": walk_traffic(args), "fp64_peak_tflops": fp64_tf,
                "phase_ms_last_step": phases}
    else:
        achieved = FLOPS_PER_INTERACTION * inter_med / (walk_med * 1e-3) / 1e12
        roof = {"kernel": "walk2_kernel (f32c)", "bound": "fp32", "achieved": achieved,
                "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                "peak_source": peak_source, "flops_per_interaction": FLOPS_PER_INTERACTION,
                "interactions_per_launch": inter_med, "walk_ms": walk_med,
                "traffic": walk_traffic(args), "fp64_peak_tflops": fp64_tf,
                "phase_ms_last_step": phases}

    # ---- CPU baseline (rank 0, N=1): reference algorithm on a bounded sample ----
    cpu = None
    if rank == 0 and ws == 1 and args.workload == "bh":
        import oracle
        oracle.lib()
        nth = oracle.ncpu()
        t_tick = cpu_reference_tick(pos, vel, m, args, nth)
        cpu = {"value": n / t_tick, "unit": "particle-steps/s", "cores": nth, "kind": "port",
               "sample": ("one whole reference tick of all %d bodies, measured: serial "
                          "pointer-octree build + threaded walk of every target, two force "
                          "evaluations per tick (src/main.rs:109,128); %.2f s" % (n, t_tick))}

    if rank == 0:
        line = {
            "metric": METRIC if args.workload == "bh" else
            "particle-steps/s, %d-body galaxy BH θ=%g, FP32-comp" % (n, args.theta),
            "value": value, "unit": "particle-steps/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32c",
            "data": "synthetic (seeded %s; no dataset)" % (
                "Plummer sphere" if args.workload == "bh" else "exponential disk + NFW halo"),
            "config": workload_config(args, "f32c (f32 pair terms, two-sum, f64 state)",
                                      args.leaf_cap, args.walk),
            "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "call": "phys_verlet_tick_host (page-locked "
                    "host arrays; x, v, m, a in, x, v, a back)"},
            "gpu_launches": launches, "clocks": clk, "roofline": roof, "cpu_baseline": cpu,
            "interactions_per_step": inter_med, "nodes": tm["nodes"], "tree_depth_max": tm["max_depth"],
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def _line(args, ws, metric, value, unit, ms, dtype, config, **kw):
    d = {"metric": metric, "value": value, "unit": unit, "n_gpus": ws, "steps": args.steps,
         "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
         "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded; no dataset)",
         "config": config}
    d.update(kw)
    return d


def run_other(args, ws, rank, local):
    """Ensemble, direct-sum, adjoint and shared Barnes-Hut workload shapes
    (one device per rank).  The ensemble's systems are split over the ranks
    and the shared system's targets too (strong scaling); the direct and
    adjoint shapes run one independent replica per rank."""
    import torch

    import physgpu
    import physgpu.dist as dist
    import physgpu.ics as ics
    from physgpu import BARNES_HUT, DIRECT, F32C, F64, F64_EXACT, GROUP_WALK, make_params

    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local))
    ctx = physgpu.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    fp32_tf, fp32x2_tf, fp64_tf = ctx.probe_peaks()

    def timed(fn, k):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(k)]
        with torch.cuda.stream(stream):
            for i in range(k):
                evs[i][0].record(stream)
                fn()
                evs[i][1].record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in evs]

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()

    clocks = Clocks(local)
    line = None
    if args.workload == "ensemble":
        # one ensemble for the whole job; its systems are split over the ranks
        # (longest first to the least-loaded rank, by N(N-1)) with no exchange
        import physgpu.dist as pdist
        off_all, pos_all, vel_all, m_all = ics.ensemble(args.n, seed=0)
        nb_all = int(off_all[-1])
        mine = pdist.shard_systems(off_all, rank, ws)
        off, body = pdist.subset_csr(off_all, mine)
        pos, vel, m = pos_all[body], vel_all[body], m_all[body]
        ns = np.diff(off)
        pairs = int(np.sum(ns * (ns - 1)))
        nb = int(off[-1])
        p = make_params(1.0, args.eps, precision=F32C)
        ctx.ensemble_load(off, pos, vel, m)
        best, tune = ctx.ensemble_autotune(p, args.dt, 16)
        for _ in range(args.warmup):
            ctx.ensemble_run(p, args.dt, args.ens_steps, group=best)
        barrier()
        l0 = ctx.timings()["launches"]
        clocks.start()
        ms = timed(lambda: ctx.ensemble_run(p, args.dt, args.ens_steps, group=best), args.steps)
        clk = clocks.stop()
        t = dist.max_over_ranks(sum(ms), device="cuda")
        value = nb_all * args.ens_steps * args.steps / (t * 1e-3)
        ach = 20.0 * pairs * args.ens_steps * args.steps / (sum(ms) * 1e-3) / 1e12
        cpu = None
        if rank == 0 and ws == 1:
            import oracle
            sel = np.arange(0, args.n, max(1, args.n // 512))
            import physgpu.dist as pdist
            sub, body = pdist.subset_csr(off, sel)
            cs = 20
            t0 = time.perf_counter()
            oracle.ensemble_run(sub, pos[body], vel[body], m[body], 1.0, args.eps, args.dt, cs,
                                nthreads=oracle.ncpu())
            dtc = time.perf_counter() - t0
            cpu = {"value": len(body) * cs / dtc, "unit": "particle-steps/s",
                   "cores": oracle.ncpu(), "kind": "port",
                   "sample": "%d of %d systems (every %d-th), %d reference ticks each" % (
                       len(sel), args.n, max(1, args.n // 512), cs)}
        line = _line(args, ws, "particle-steps/s, batched ensemble of %d systems (N in [3,64]), "
                     "FP32-comp forces, FP64 state" % args.n, value, "particle-steps/s",
                     t / args.steps, "f32c",
                     {"workload": "ensemble_%d_systems" % args.n, "bodies": nb_all,
                      "systems_per_rank": "split over %d rank(s) by N(N-1), no exchange" % ws,
                      "steps_per_bench_step": args.ens_steps, "eps": args.eps, "dt": args.dt,
                      "config": best, "config_meaning": "lanes per system (1 = by size) | "
                      "warps per block << 8", "autotune_ms": {str(k): v for k, v in tune.items()},
                      "launch": "one persistent launch per run, captured in a CUDA graph",
                      "l2": "state (%.1f MB) stays on chip for a whole run" % (nb * 80 / 1e6)},
                     interactions_per_s=pairs * args.ens_steps * args.steps / (sum(ms) * 1e-3),
                     roofline={"kernel": "ensemble_kernel (config 0x%x)" % best, "bound": "fp32",
                               "achieved": ach, "peak": max(fp32_tf, fp32x2_tf),
                               "unit": "TFLOP/s", "frac": ach / max(fp32_tf, fp32x2_tf),
                               "flops_per_interaction": 20, "traffic": None},
                     cpu_baseline=cpu, clocks=clk, scaling="strong",
                     gpu_launches=ctx.timings()["launches"] - l0)
    elif args.workload == "direct":
        pos, vel, m = ics.plummer(args.n, seed=rank)
        out = {}
        for name, prec in (("f64_exact", F64_EXACT), ("f64", F64), ("f32c", F32C)):
            p = make_params(1.0, args.eps, method=DIRECT, precision=prec)

            def run100():
                ctx.upload(pos, vel, m)
                ctx.verlet_steps(p, args.dt, 100)
            for _ in range(args.warmup):
                run100()
            barrier()
            clocks.start()
            ms = timed(run100, args.steps)
            clk = clocks.stop()
            out[name] = (dist.max_over_ranks(sum(ms), device="cuda"), clk)
        t, clk = out["f64_exact"]
        n = args.n
        value = ws * n * 100 * args.steps / (t * 1e-3)
        cpu = None
        if rank == 0 and ws == 1:
            import oracle
            t0 = time.perf_counter()
            oracle.vv_run(pos, vel, m, 1.0, args.eps, args.dt, 10, method="direct")
            dtc = (time.perf_counter() - t0) / 10
            cpu = {"value": n / dtc, "unit": "particle-steps/s", "cores": 1, "kind": "port",
                   "sample": "10 reference ticks (2 direct-sum evaluations each; 1024 targets "
                             "run as one rayon task, so one core)"}
        line = _line(args, ws, "particle-steps/s, %d-body Plummer direct sum f64, 100 VV steps"
                     % n, value, "particle-steps/s", t / args.steps, "f64",
                     {"workload": "direct_plummer_n%d_100_steps" % n, "eps": args.eps,
                      "dt": args.dt, "precision": "f64_exact (bit-identical to the reference)",
                      "bench_step": "upload + 100 Velocity-Verlet ticks on the device"},
                     variants_ms_per_step={k: v[0] / args.steps for k, v in out.items()},
                     cpu_baseline=cpu, clocks=clk)
    elif args.workload == "bh_shared":
        # one system for the whole job, split by targets: every rank holds
        # and integrates all bodies, builds the same tree, evaluates the
        # groups of its share of the key order, and one all-gather of the
        # shares' accelerations (24 bytes per body) completes each evaluation
        n = args.n
        pos, vel, m = ics.plummer(n, seed=0)
        p = make_params(1.0, args.eps, args.theta, BARNES_HUT, F32C, args.leaf_cap, GROUP_WALK)
        flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        ctx.upload(pos, vel, m)
        ex = dist.SharedEvaluation(ctx)
        ex.evaluate(p)

        def tick():
            ctx.vv_position_step(args.dt)
            ex.evaluate(p)
            ctx.vv_velocity_step(args.dt)
        for _ in range(args.warmup):
            tick()
        barrier()
        l0 = ctx.timings()["launches"]
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        clocks.start()
        with torch.cuda.stream(stream):
            for i in range(args.steps):
                flush_buf.fill_(i & 0xff)
                evs[i][0].record(stream)
                tick()
                evs[i][1].record(stream)
        torch.cuda.synchronize()
        clk = clocks.stop()
        launches = ctx.timings()["launches"] - l0
        ms = [a.elapsed_time(b) for a, b in evs]
        t = dist.max_over_ranks(sum(ms), device="cuda")
        value = n * args.steps / (t * 1e-3)
        x_final, _, _ = ctx.download()
        line = _line(args, ws, METRIC, value, "particle-steps/s", t / args.steps, "f32c",
                     dict(workload_config(args, precision="f32c", leaf_cap=args.leaf_cap,
                                          walk="group"),
                          workload="barnes_hut_plummer_n%d_shared" % n,
                          ics="Plummer a=1, equal masses 1/N, seed=0 (one system on all ranks)",
                          parallelism="one system, targets split over %d rank(s) by key "
                                      "order; all-gather of the shares' accelerations" % ws,
                          l2="flushed between timed steps (256 MiB write)"),
                     scaling="strong", clocks=clk, gpu_launches=launches,
                     exchange_bytes_per_evaluation=24 * physgpu.share_chunk(n, ws) * ws,
                     checksum_final_x=float(np.abs(x_final).sum()),
                     note="same trajectory as one GPU bit for bit (tests/test_share_gpu.py)")
    elif args.workload == "adjoint":
        n, nsteps = args.n, args.adj_steps
        pos, vel, m = ics.plummer(n, seed=rank)
        p = make_params(1.0, args.eps, precision=F64)
        rng = np.random.default_rng(rank + 100)
        ctx.upload(pos, vel + rng.normal(0.0, 0.01, vel.shape), m)
        _, targets = ctx.trajectory_loss(p, args.dt, nsteps, np.zeros((n, 3)), final=True)
        ctx.upload(pos, vel, m)
        for _ in range(args.warmup):
            ctx.adjoint(p, args.dt, nsteps, targets, checkpoint=32)
        barrier()
        clocks.start()
        ms = timed(lambda: ctx.adjoint(p, args.dt, nsteps, targets, checkpoint=32), args.steps)
        clk = clocks.stop()
        t = dist.max_over_ranks(sum(ms), device="cuda")
        value = ws * args.steps / (t * 1e-3)
        line = _line(args, ws, "trajectory gradients/s, %d-body Plummer, %d VV steps, f64 "
                     "adjoint with checkpoint 32" % (n, nsteps), value, "gradients/s",
                     t / args.steps, "f64",
                     {"workload": "adjoint_plummer_n%d_%d_steps" % (n, nsteps), "eps": args.eps,
                      "dt": args.dt, "checkpoint": 32,
                      "work_per_gradient": "%d force evaluations + %d Jacobian-vector "
                                           "products of the direct sum" % (2 * nsteps + 1,
                                                                           nsteps + 1)},
                     particle_steps_per_s=ws * n * nsteps * args.steps / (t * 1e-3),
                     cpu_baseline=None, clocks=clk,
                     note="the reference has no differentiation: no CPU baseline")
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def run_reference_other(args, ws, rank):
    import oracle
    oracle.lib()
    if rank != 0:
        return 0
    import physgpu.ics as ics
    if args.workload == "adjoint":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference has no differentiation of trajectories"}), flush=True)
        return 0
    ticks = []
    if args.workload == "ensemble":
        import physgpu.dist as pdist
        off, pos, vel, m = ics.ensemble(args.n, seed=0)
        sel = np.arange(0, args.n, max(1, args.n // 512))
        sub, body = pdist.subset_csr(off, sel)
        for k in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            oracle.ensemble_run(sub, pos[body], vel[body], m[body], 1.0, args.eps, args.dt, 20)
            if k >= args.warmup:
                ticks.append((time.perf_counter() - t0) / 20)
        value = len(body) / (sum(ticks) / len(ticks))
        sample = "%d of %d systems, 20 ticks per step" % (len(sel), args.n)
    else:
        pos, vel, m = ics.plummer(args.n, seed=0)
        for k in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            oracle.vv_run(pos, vel, m, 1.0, args.eps, args.dt, 10, method="direct")
            if k >= args.warmup:
                ticks.append((time.perf_counter() - t0) / 10)
        value = args.n / (sum(ticks) / len(ticks))
        sample = "10 reference ticks per step"
    line = {"impl": "reference", "metric": args.workload, "value": value,
            "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(ticks) / len(ticks),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": {"workload": args.workload, "n": args.n},
            "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": oracle.ncpu(),
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        if args.workload in ("bh", "galaxy", "bh_shared"):
            return run_reference(args, ws, rank)
        return run_reference_other(args, ws, rank)
    if args.workload in ("bh", "galaxy"):
        return run_ours(args, ws, rank, local)
    return run_other(args, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
