#!/usr/bin/env python3
"""Benchmark: MLS-MPM fluid substep + diffuse update, particle-updates/s.

Workload (one "step" = one substep of the scene, all passes incl. diffuse):
  dam_break_1m — 128^3 grid, 1,048,576 particles (seeded-jitter dam break,
  block 40% of the width x 60% of the height), diffuse pool 262,144.
Multi-GPU (torchrun): every rank simulates its own independent scene (seed =
rank) — scene sharding with no data-path collective; `value` sums all ranks'
particle-updates over the max-over-ranks device time ("scaling": "weak").
The batched and served comparisons shard their scene mix and job stream over
the ranks (mls_mpm_b200.shard), one batch or serving loop per GPU.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mls-mpm_b200"))

import numpy as np  # noqa: E402

METRIC = "particle-updates/s @1M (frac HBM roofline)"
UNIT = "particle-updates/s"
WORKLOAD = "dam_break_1m"


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured hbm_gbs (MEASURED_PEAKS.json)"
    return 6650.0, "fallback 6.65 TB/s"


# Algorithmic bytes per unit of each phase (reference vec4/affine9 layouts):
# per particle: P2G_MASS 20 (pos 16 + mass 4), P2G_MOM 76 (pos 16 + vel 16 +
# C 36 + mass 4 + density 4), G2P 84 (pos 16 in; pos 16 + vel 16 + C 36 out);
# per cell: P2G_MASS 4 (mass i32 write), P2G_MOM 16 (mass read 4 + momentum
# i32 write 12), UPDATE_GRID 28 (momentum+mass read 16, velocity write 12),
# G2P 12 (velocity read).  Sum: 180 B per particle + 60 B per cell.
PHASE_BYTES = {"p2g_mass": (20, 4), "p2g_mom": (76, 16), "update_grid": (0, 28), "g2p": (84, 12)}

# Bytes of one scene's uniform block in the device scene table (grid dims and
# ranges, Params 80 B, WallParams 336 B, HandParams 80 B, hand box): what a
# frame that changes any uniform uploads.
SCENE_DESC_BYTES = 576


class ClockSampler:
    """NVML sampling of SM clock and throttle reasons while running."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x1: "gpu_idle", 0x2: "applications_clocks_setting",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, index):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._h = None

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for bit, name in self.REASONS.items():
                    if r & bit and name != "gpu_idle":
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.01)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        if self._h is not None:
            self._stop.set()
            self._t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_reference_rate(scene, substeps, threads, budget_s=None, warmup=1):
    """Times the reference pin (the reference's WGSL compiled on the host) or,
    when it is absent, the oracle restatement, over `substeps` substeps of
    `scene` with diffuse after `warmup` untimed ones.  Returns (updates/s,
    kind, steps run, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle as O
    import scenarios
    kind = "reference" if O.ref_available() else "port"
    impl = "ref" if kind == "reference" else "oracle"
    sc = scenarios.Scenario(scene.name, scene, substeps + warmup, diffuse_max=scene.diffuse_max)
    st = O.new_state(scene, scene.diffuse_max)
    frames = sc.frames()
    for _ in range(warmup):
        P, W, H, dims, gen, adv = next(frames)
        O.substep(st, P, W, H, dims, gen, adv, threads=threads, impl=impl)
    t0 = time.perf_counter()
    done = 0
    for P, W, H, dims, gen, adv in frames:
        O.substep(st, P, W, H, dims, gen, adv, threads=threads, impl=impl)
        done += 1
        if budget_s and time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return scene.n * done / dt, kind, done, dt


def run_config(workload, scene, ws):
    """The `config` object of both arms' lines."""
    return {"workload": workload, "grid": list(scene.grid), "particles": scene.n,
            "diffuse_pool": scene.diffuse_max, "substeps_per_step": 1,
            "parallelism": f"scene-sharded x{ws}" if ws > 1 else "single scene",
            "l2": l2_note(scene.n, scene.cells, scene.diffuse_max)}


def run_reference_arm(args, ws, rank):
    from mls_mpm_b200 import scenes
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    scene = scenes.WORKLOADS[args.workload](seed=0)
    # warm-up steps are untimed; each timed step is one full substep of the
    # scene; the run is capped at ~240 s of CPU time (the sample is stated)
    rate, kind, done, secs = cpu_reference_rate(scene, args.steps, threads, budget_s=240.0, warmup=args.warmup)
    sample = f"{done} substeps of the {args.workload} scene ({scene.n:,} particles + {scene.diffuse_max:,} " \
             f"diffuse pool) on {threads} host threads"
    line = {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": done,
            "warmup": args.warmup, "ms_per_step": 1e3 * secs / max(done, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+i32", "data": "synthetic",
            "impl": "reference",
            "config": run_config(args.workload, scene, ws),
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-vs-one-at-a-time comparison")
    ap.add_argument("--no-served", action="store_true", help="skip the served-vs-per-job comparison")
    ap.add_argument("--no-drift", action="store_true", help="skip the f32-vs-f64 drift report")
    ap.add_argument("--batched-only", action="store_true",
                    help="run only the batched-vs-one-at-a-time comparison and print it (for profiling)")
    ap.add_argument("--workload", default=WORKLOAD)
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference_arm(args, ws, rank)
    if args.batched_only:
        import torch
        torch.cuda.set_device(local)
        print(json.dumps({"batched": batched_comparison(local, substeps=args.steps, warmup=args.warmup)}))
        return 0

    import torch
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from mls_mpm_b200 import DiffuseGPU, FluidGPU, scenes
    from mls_mpm_b200.abi import check
    scene = scenes.WORKLOADS[args.workload](seed=rank)

    def make(render=False):
        """One simulation of the workload; identical copies follow the same
        trajectory, so the device-timed, per-phase and end-to-end numbers all
        cover the same substeps [W, W+K).  render: the renderer takes its
        buffers at start-up (as fluid-renderer.js binds them once), before
        the warm-up."""
        fl = FluidGPU.from_scene(scene, device=local)
        if scene.diffuse_max:
            DiffuseGPU(scene.diffuse_max).initGPU(local, fl)
        if render:
            for name in ("pos", "vel", "density"):
                fl.get_buffer(name)
        for _ in range(args.warmup):
            fl.simFrame()
        fl.sync()
        return fl

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    clocks = ClockSampler(local)
    # (1) device-timed region: exactly K substeps, inputs resident in HBM
    fl = make()
    lib, h = fl._lib, fl._scene
    sptr = ctypes.c_void_p()
    check(lib.mpm_get_stream(h, ctypes.byref(sptr)), "mpm_get_stream")
    stream = torch.cuda.ExternalStream(sptr.value, device=torch.device("cuda", local))
    c0, c1 = ctypes.c_uint64(), ctypes.c_uint64()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    lib.mpm_launch_count(h, ctypes.byref(c0))
    with clocks:
        e0.record(stream)
        for _ in range(args.steps):
            check(lib.mpm_step(h, 1), "mpm_step")
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    lib.mpm_launch_count(h, ctypes.byref(c1))
    n_launch = c1.value - c0.value
    fl.destroy()

    # (2) end to end through the public API over the same substeps, as the
    # reference's frame drives it (main.js:504-528): per step the host moves
    # the hand (fluid-gpu.js:479-527; a small cylinder sweeping the empty top
    # corner of the domain, so every frame carries new uniforms, uploaded from
    # pinned memory), steps the scene, takes the particle position, velocity
    # and density buffers the renderer draws from (fluid-renderer.js:315-328;
    # zero-copy device pointers in the reference layout), queues the diffuse
    # alive-count readback (diffuse-gpu.js:172-176) and polls it (178-188)
    # without waiting; the clock stops after the last readback has landed.
    # The same loop without the render buffers is reported beside it.
    def e2e_run(render):
        fl = make(render)
        X, Y, Z = scene.grid
        barrier()
        t0 = time.perf_counter()
        for s in range(args.steps):
            hz = Z - 14.0 + 2.0 * math.sin(0.1 * s)
            fl.updateHand([X - 14.0, Y - 12.0, hz], [0.0, 0.0, 0.5], 3.0, 0.2, True, [X - 14.0, Y - 12.0, Z + 40.0])
            fl.simFrame()
            if render:
                for name in ("pos", "vel", "density"):
                    fl.get_buffer(name)
            if fl.diffuse is not None:
                fl.diffuse.requestDebugReadback()
                fl.diffuse.pollDebug()
        fl.sync()
        if fl.diffuse is not None:
            fl.diffuse.pollDebug()
        secs = max_over_ranks(time.perf_counter() - t0)
        fl.destroy()
        return secs

    e2e_s = e2e_run(render=True)
    e2e_plain_s = e2e_run(render=False)

    # (3) per-phase device time over the same substeps (CUDA events on the scene stream),
    # after the end-to-end run so that both timed loops follow each other
    fl = make()
    lib, h = fl._lib, fl._scene
    lib.mpm_profile_enable(h, 1)
    lib.mpm_profile_read(h, None, None, 1)
    for _ in range(args.steps):
        check(lib.mpm_step(h, 1), "mpm_step")
    pm = (ctypes.c_double * 10)()
    pc = (ctypes.c_uint64 * 10)()
    check(lib.mpm_profile_read(h, pm, pc, 1), "mpm_profile_read")
    names = [lib.mpm_phase_name(i).decode() for i in range(10)]
    fl.destroy()

    h2d = SCENE_DESC_BYTES   # the scene's uniform block, changed by the hand every frame
    d2h = 4 if scene.diffuse_max else 0

    n = scene.n
    total_updates = n * args.steps * ws
    value = total_updates / (ms / 1e3)
    e2e_value = total_updates / e2e_s
    peak, peak_src = measured_peaks()
    G = scene.cells
    phase_ms = {names[i]: pm[i] / pc[i] for i in range(10) if pc[i]}
    dom = max((k for k in phase_ms if k in PHASE_BYTES), key=lambda k: phase_ms[k])
    bn, bg = PHASE_BYTES[dom]
    dom_bytes = bn * n + bg * G
    achieved = dom_bytes / (phase_ms[dom] * 1e-3) / 1e9
    sub_bytes = 180 * n + 60 * G
    sub_ms = ms / args.steps
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None, "peak_source": peak_src,
                "algorithmic_bytes_per_launch": dom_bytes, "avg_launch_ms": phase_ms[dom]}
    traffic = _profile_traffic(dom, args.workload)
    if traffic:
        roofline["traffic"] = traffic
    # the same kernel's issue-slot use (sm__inst_issued, ncu): what bounds it
    issue = _profile_value("issue_active_per_launch", dom, args.workload)
    if issue is not None:
        roofline["issue_active"] = issue
        roofline["issue_note"] = ("fraction of issue slots used, from the committed ncu summary: the particle "
                                  "kernels are issue/latency-bound, not HBM-bound")
    # issue roofline: the kernel's warp instructions (committed ncu summary)
    # against 4 issue slots per SM per clock over its live launch time
    winst = _profile_value("warp_inst_per_launch", dom, args.workload)
    csum = clocks.summary()
    if winst is not None and csum.get("sm_mhz"):
        props = torch.cuda.get_device_properties(local)
        slots = 4.0 * props.multi_processor_count * csum["sm_mhz"] * 1e6 * phase_ms[dom] * 1e-3
        roofline["issue_roofline"] = {"warp_instructions": winst, "issue_slots": slots, "frac": winst / slots,
                                      "note": "warp instructions / (4 x SMs x median SM clock x live launch time)"}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sub_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+i32", "data": "synthetic",
            "config": run_config(args.workload, scene, ws),
            "roofline": roofline,
            "substep_roofline": {"achieved": sub_bytes / (sub_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                                 "frac": sub_bytes / (sub_ms * 1e-3) / 1e9 / peak,
                                 "algorithmic_bytes": sub_bytes, "note": "180 B/particle + 60 B/cell"},
            "phase_ms": phase_ms,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "render_buffers": "particle pos, vel and density taken every frame (reference layout, device)",
                    "without_render_buffers": total_updates / e2e_plain_s},
            "gpu_launches": n_launch,
            "clocks": clocks.summary()}

    if rank == 0 and not args.no_drift:
        line["drift_f32_vs_f64"] = drift_report(local)
    if not args.no_batched:
        line["batched"] = batched_comparison(local, ws=ws, rank=rank, reduce_max=max_over_ranks)
    if not args.no_served:
        line["served"] = served_comparison(local, ws=ws, rank=rank)

    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cpu_scene = scenes.WORKLOADS[args.workload](seed=0)
        rate, kind, done, secs = cpu_reference_rate(cpu_scene, 40, threads, budget_s=20.0)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
                                "sample": f"{done} substeps of {args.workload} ({secs:.1f} s) on {threads} threads"}
    if dist is not None:
        dist.barrier()
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def drift_report(local, substeps=100, checkpoints=(1, 10, 100), threads=None):
    """f32 drift: the dam_break_64 scene advanced on the GPU (its f32 state is
    bit-identical to the f32 oracle) against the same passes evaluated in
    binary64 (the oracle instantiated for double), after 1, 10 and 100
    substeps.  Positions in cells."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle as O
    import scenarios
    from mls_mpm_b200 import FluidGPU
    threads = threads or os.cpu_count() or 1
    sc = scenarios.dam_break_64(substeps)
    fl = FluidGPU.from_scene(sc.scene, device=local)
    ref = O.to_f64(O.new_state(sc.scene))
    rows = []
    for t, (P, W, H, dims, gen, adv) in enumerate(sc.frames(), 1):
        fl.simFrame()
        O.substep(ref, P, W, H, dims, impl="f64", threads=threads)
        if t in checkpoints:
            g = fl.read("pos")[:, :3].astype(np.float64)
            r = ref["pos"][:, :3]
            d = np.abs(g - r)
            gv = fl.read("vel")[:, :3].astype(np.float64)
            dv = np.abs(gv - ref["vel"][:, :3])
            rows.append({"substep": t, "pos_max_abs": float(d.max()), "pos_rms": float(np.sqrt((d * d).mean())),
                         "vel_max_abs": float(dv.max()),
                         "vel_max_rel": float((dv / np.maximum(np.abs(ref["vel"][:, :3]), 1e-3)).max())})
    fl.destroy()
    return {"workload": "dam_break_64 (65,536 particles, 64^3)", "reference": "same passes in binary64",
            "note": "GPU f32 state is bit-identical to the f32 oracle at every substep", "checkpoints": rows}


def batched_comparison(local, substeps=200, warmup=20, count=64, seed=0, ws=1, rank=0, reduce_max=None):
    """The batched workload (scenes.batch_mix: 64 scenes, 200 substeps) run as
    one batch (one launch per kernel per substep for all scenes, CUDA graph,
    autotuned launch shape) and one scene at a time through the single-scene
    path (the same kernels, each scene's `substeps` substeps in turn on its own
    stream).  Both are device-timed with CUDA events after `warmup` substeps
    (the autotuner's trials fall in the batch's warm-up).  With ws ranks each
    rank runs its share of the scenes (shard.assign on particle-updates) in
    both arms; times are the max over ranks."""
    import torch
    from mls_mpm_b200 import abi, scenes, shard
    from mls_mpm_b200.abi import check
    from mls_mpm_b200.batch import Batch, default_params
    from mls_mpm_b200.fluid_gpu import FluidGPU

    reduce_max = reduce_max or (lambda x: x)
    full = scenes.batch_mix(count, seed)
    n_all = sum(s.n for s in full)
    cells_all = sum(s.cells for s in full)
    mine = shard.my_items([shard.scene_cost(s, substeps) for s in full], ws, rank)
    mix = [full[i] for i in mine]
    n_tot = sum(s.n for s in mix)
    cells = sum(s.cells for s in mix)
    dev = torch.device("cuda", local)
    # batched
    b = Batch(max(1, n_tot), max(1, cells), max(1, len(mix)), device=local, flags=abi.BATCH_AUTOTUNE)
    for s in mix:
        b.add(default_params(s.grid, s.n, b.lib), s.pos, s.mass, s.vel, s.affine)
    b.step(warmup)
    b.sync()
    st = torch.cuda.ExternalStream(b.stream(), device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = b.info().launches
    e0.record(st)
    b.step(substeps)
    e1.record(st)
    e1.synchronize()
    batched_ms = reduce_max(e0.elapsed_time(e1))
    info = b.info()
    launches = info.launches - l0
    shape = (info.item_blocks, info.grid_blocks)
    b.close()
    # one scene at a time
    alone_ms = 0.0
    alone_launches = 0
    for s in mix:
        fl = FluidGPU.from_scene(s, device=local)
        lib, h = fl._lib, fl._scene
        check(lib.mpm_step(h, warmup), "mpm_step")
        fl.sync()
        sp = ctypes.c_void_p()
        check(lib.mpm_get_stream(h, ctypes.byref(sp)), "mpm_get_stream")
        ss = torch.cuda.ExternalStream(sp.value, device=dev)
        c0, c1 = ctypes.c_uint64(), ctypes.c_uint64()
        lib.mpm_launch_count(h, ctypes.byref(c0))
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(ss)
        check(lib.mpm_step(h, substeps), "mpm_step")
        a1.record(ss)
        a1.synchronize()
        alone_ms += a0.elapsed_time(a1)
        lib.mpm_launch_count(h, ctypes.byref(c1))
        alone_launches += c1.value - c0.value
        fl.destroy()
    alone_ms = reduce_max(alone_ms)
    updates = n_all * substeps
    sub_bytes = 180 * n_all + 60 * cells_all
    peak, _ = measured_peaks()
    peak *= ws
    return {"workload": f"batch_mix: {count} scenes, {n_all} particles, {cells_all} cells, seed {seed}"
                        + (f"; scene-sharded over {ws} GPUs (max over ranks)" if ws > 1 else ""),
            "substeps": substeps, "warmup": warmup,
            "batched": {"value": updates / (batched_ms / 1e3), "unit": UNIT, "ms_per_substep": batched_ms / substeps,
                        "gpu_launches": launches, "launch_shape": {"item_blocks": shape[0], "grid_blocks": shape[1]},
                        "hbm_frac": sub_bytes / (batched_ms / substeps * 1e-3) / 1e9 / peak},
            "one_at_a_time": {"value": updates / (alone_ms / 1e3), "unit": UNIT,
                              "ms_per_substep_all_scenes": alone_ms / substeps, "gpu_launches": alone_launches},
            "speedup": alone_ms / batched_ms}


def served_comparison(local, rates=(50.0, 200.0, 2000.0), count=64, seed=0, budget_gb=150.0, ws=1, rank=0):
    """The served workload: `count` jobs (scenes.serve_job) arriving as a
    Poisson stream at each rate, run by the serving loop (admission against an
    HBM budget, resident scenes batched every substep) and by the plain
    per-job path (one job at a time in arrival order through the single-scene
    path).  Plain-path latencies come from each job's device-timed service
    time played through the same arrival times in FIFO order.  With ws ranks
    each rank serves its share of the stream (shard.assign on
    particle-updates, arrival times kept); throughput is all ranks' updates
    over the slowest rank's wall time, latencies are pooled."""
    import torch
    from mls_mpm_b200 import abi, scenes, shard
    from mls_mpm_b200.abi import check
    from mls_mpm_b200.batch import default_params
    from mls_mpm_b200.fluid_gpu import FluidGPU
    from mls_mpm_b200.server import Server

    all_jobs = [scenes.serve_job(seed, i) for i in range(count)]
    mine = shard.shard_jobs(all_jobs, ws, rank)
    jobs = [all_jobs[i] for i in mine]
    updates_all = sum(sc.n * k for sc, k in all_jobs)
    dev = torch.device("cuda", local)
    free, _ = torch.cuda.mem_get_info(dev)
    budget = int(min(budget_gb * 1e9, free - 12e9))
    cpp = max(sc.cells / sc.n for sc, _ in all_jobs)
    out = {"workload": f"serve_job x{count}: {sum(sc.n for sc, _ in all_jobs)} particles, "
                       f"{updates_all} particle-updates, seed {seed}"
                       + (f"; job stream sharded over {ws} GPUs" if ws > 1 else ""),
           "budget_bytes": budget, "budget_note": f"min({budget_gb:g} GB, free device memory - 12 GB) per GPU",
           "rates": {}}
    # plain per-job path: service time of each job alone (device-timed)
    service = []
    for sc, k in jobs:
        fl = FluidGPU.from_scene(sc, device=local)
        lib, h = fl._lib, fl._scene
        sp = ctypes.c_void_p()
        check(lib.mpm_get_stream(h, ctypes.byref(sp)), "mpm_get_stream")
        ss = torch.cuda.ExternalStream(sp.value, device=dev)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(ss)
        check(lib.mpm_step(h, k), "mpm_step")
        a1.record(ss)
        a1.synchronize()
        service.append(a0.elapsed_time(a1) / 1e3)
        fl.destroy()
    srv = Server(budget, scene_capacity=max(64, count), cells_per_particle=cpp, device=local)
    try:
        for rate in rates:
            arr_all = scenes.poisson_arrivals(rate, count, seed)
            arr = [float(arr_all[i]) for i in mine]
            ids = [srv.submit(default_params(sc.grid, sc.n, srv.lib), sc.pos, sc.mass, k, t, vel4=sc.vel)
                   for (sc, k), t in zip(jobs, arr)]
            st = srv.run()
            lat = []
            for j in ids:
                r = srv.job(j)
                lat.append(r.finish_s - r.arrival_s)
            # plain path, FIFO through the same arrivals
            fin, plat = 0.0, []
            for t, sv in zip(arr, service):
                fin = max(fin, t) + sv
                plat.append(fin - t)
            parts = shard.gather({"updates": int(st.particle_updates), "wall": st.wall_s, "lat": lat,
                                  "plain_wall": fin, "plain_lat": plat, "mean_active": st.mean_active,
                                  "max_active": st.max_active, "substeps": int(st.substeps),
                                  "launches": int(st.launches)})
            served_updates = sum(p["updates"] for p in parts)
            wall = max(p["wall"] for p in parts)
            plain_wall = max(p["plain_wall"] for p in parts)
            lat_all = [x for p in parts for x in p["lat"]]
            plat_all = [x for p in parts for x in p["plain_lat"]]
            out["rates"][f"{rate:g}"] = {
                "served": {"value": served_updates / wall, "unit": UNIT,
                           "p50_latency_s": float(np.percentile(lat_all, 50)),
                           "p99_latency_s": float(np.percentile(lat_all, 99)),
                           "wall_s": wall, "mean_active_scenes": st.mean_active,
                           "max_active_scenes": st.max_active, "substeps": st.substeps,
                           "gpu_launches": sum(p["launches"] for p in parts)},
                "plain_per_job": {"value": updates_all / plain_wall, "unit": UNIT,
                                  "p50_latency_s": float(np.percentile(plat_all, 50)),
                                  "p99_latency_s": float(np.percentile(plat_all, 99)), "wall_s": plain_wall},
                "speedup": (served_updates / wall) / (updates_all / plain_wall)}
        out["capacity"] = {"particles": st.particle_capacity, "cells": st.cell_capacity}
    finally:
        srv.close()
    return out


# kernel that carries each timed phase (for the DRAM traffic of its ncu summary)
PHASE_KERNEL = {"p2g_mass": "k_p2g_mass_chunks", "p2g_mom": "k_p2g_mom_chunks", "g2p": "k_g2p_chunks",
                "update_grid": "k_update_tiles"}


def l2_note(n, cells, pool):
    """How the timed substeps stand against the 126 MB L2: the state read and
    written every substep (particles 72 B: position, velocity, affine,
    density; grid cells 32 B: i32 mass and momentum, float4 velocity; diffuse
    slots 48 B)."""
    mb = lambda b: b / 2**20
    p, g, d = 72 * n, 32 * cells, 48 * pool
    rel = ">" if p + g + d > 126e6 else "<="
    return (f"working set {rel} 126 MB L2 (particles {mb(p):.0f} MB + grids {mb(g):.0f} MB + pool {mb(d):.0f} MB); "
            "no flush")


def _profile_value(key, phase, workload):
    """The value of a `<key> <kernel> <workload> <value>` line of the committed
    ncu summaries under profiles/ for the phase's kernel, or None."""
    kernel = PHASE_KERNEL.get(phase)
    d = os.path.join(ROOT, "profiles")
    if not kernel or not os.path.isdir(d):
        return None
    for f in sorted(os.listdir(d)):
        if not f.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(d, f)):
            parts = line.split()
            if len(parts) == 4 and parts[0] == key and parts[1] == kernel and parts[2] == workload:
                return float(parts[3])
    return None


def _profile_traffic(phase, workload=WORKLOAD):
    """DRAM bytes (read + write) per launch of the phase's kernel, from the
    `dram_bytes_per_launch <kernel> <workload> <bytes>` lines, or None."""
    v = _profile_value("dram_bytes_per_launch", phase, workload)
    return int(v) if v is not None else None


if __name__ == "__main__":
    sys.exit(main())
