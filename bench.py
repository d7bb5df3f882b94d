"""Narrow-phase microbenchmark: 1,048,576 shape pairs in seven algorithm
batches (sphere-sphere, sphere-capsule, capsule-capsule, sphere-box,
capsule-box, box-box, hull-box), FP32, seeded synthetic inputs.

One step = one pass of the six ReactPhysics3D narrow-phase algorithms over
the whole pair set (seven kernel launches, one per batch), inputs resident in
device memory, L2 flushed between steps.  Each rank runs its own pair set
(pairs are independent: weak scaling, no data-path collective).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `--impl reference` times the reference
engine's own CPU algorithms (built from its sources into oracle/_ref) on the
host cores over a bounded sample of the same workload.
"""
import argparse
import ctypes as C
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
T_START = time.perf_counter()

from reactphysics3d_b200 import _abi as A  # noqa: E402
from reactphysics3d_b200 import scenes  # noqa: E402

METRIC = "narrowphase pairs/sec"
UNIT = "pairs/s"
WORKLOAD = "narrowphase microbenchmark: 1,048,576 pairs in 7 algorithm batches (FP32)"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


# Measured DRAM traffic per pair of a batch (both of its launches): ncu
# dram__bytes_read.sum + dram__bytes_write.sum of `python bench.py --pairs
# 262144 --steps 2 --warmup 1 --no-cpu --no-e2e --no-learned` (37,449 pairs
# per batch): hull-box 2.76 + 5.28 MB, box-box 5.85 + 2.77 MB.
TRAFFIC_PER_PAIR = {"hull_box": (2.76e6 + 5.26e6 + 0.02e6) / 37449, "box_box": (5.54e6 + 0.31e6 + 2.77e6) / 37449}


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def peaks():
    try:
        with open(PEAKS_FILE) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """SM clock and throttle reasons sampled through NVML (read-only queries)
    every 20 ms while the timed region runs; nvidia-smi is the fallback."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.sm, self.mx, self.bits = [], [], 0
        self._stop = threading.Event()
        self.t = None

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[self.gpu]) if vis and vis.split(",")[0].isdigit() else self.gpu
            h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self.mx.append(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))

            def run():
                while not self._stop.is_set():
                    try:
                        self.sm.append(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                        self.bits |= int(pynvml.nvmlDeviceGetCurrentClocksEventReasons(h))
                    except Exception:
                        pass
                    self._stop.wait(0.02)
            self.t = threading.Thread(target=run, daemon=True)
            self.t.start()
        except Exception:
            self.t = None

    def stop(self):
        if self.t is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"], "samples": 0}
        self._stop.set()
        self.t.join(timeout=2)
        reasons = sorted(k for k, b in self.REASONS.items() if self.bits & b)
        return {"sm_mhz": statistics.median(self.sm) if self.sm else None,
                "sm_max_mhz": max(self.mx) if self.mx else None, "reasons": reasons, "samples": len(self.sm)}


# Algorithmic bytes per pair (unit of the HBM roofline): inputs read
# (shape indices 8 B + two shape records 64 B + four float4 transform rows
# 64 B) + outputs written (flag + count 2 B + 48 B per reported contact).
IN_BYTES_PER_PAIR = 8 + 64 + 64


def run_ours(args):
    import torch
    from reactphysics3d_b200 import engine

    rank, local_rank, world = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"

    sc = scenes.narrowphase_scene(total_pairs=args.pairs, seed=args.seed + rank)
    ctx = engine.Context(local_rank)
    mesh = ctx.create_convex_mesh(sc.hull_vertices, sc.hull_faces)
    ctx.create_convex_mesh_shape(mesh)
    ctx.set_shapes(sc.shapes)
    names = list(sc.batches.keys())
    dpairs = {nm: engine.DevicePairs(sc.batches[nm][1], device=dev) for nm in names}
    douts = {nm: engine.DeviceContacts(sc.batches[nm][1].n, device=dev) for nm in names}
    algos = {nm: sc.batches[nm][0] for nm in names}
    stream = ctx.torch_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2

    def one_step(evs=None):
        for k, nm in enumerate(names):
            if evs is not None:
                evs[k][0].record(stream)
            ctx.narrowphase_device(algos[nm], dpairs[nm], douts[nm])
            if evs is not None:
                evs[k][1].record(stream)

    # everything below is queued on the library's stream (torch made current
    # on it), so the kernels need no cross-stream ordering
    torch.cuda.synchronize()
    torch.cuda.set_stream(stream)
    for _ in range(args.warmup):
        flush.zero_()
        one_step()
    ctx.synchronize()

    sampler = ClockSampler(local_rank)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler.start()
    launches0 = ctx.kernel_launches()
    step_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    batch_ev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in names]
                for _ in range(args.steps)]
    for s in range(args.steps):
        flush.zero_()
        step_ev[s][0].record(stream)
        one_step(batch_ev[s])
        step_ev[s][1].record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    torch.cuda.set_stream(torch.cuda.default_stream())
    launches = ctx.kernel_launches() - launches0
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(b) for a, b in step_ev]
    batch_ms = {nm: [batch_ev[s][k][0].elapsed_time(batch_ev[s][k][1]) for s in range(args.steps)]
                for k, nm in enumerate(names)}
    total_ms = float(sum(step_ms))
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    pairs_total = sc.n_pairs * world
    value = pairs_total / (ms_per_step / 1e3)

    # ---- per-kernel roofline of the dominant kernel ----------------------
    mean_batch = {nm: float(np.mean(v)) for nm, v in batch_ms.items()}
    dom = max(mean_batch, key=mean_batch.get)
    host_out = {nm: douts[nm].nb_contacts.cpu().numpy() for nm in names}
    n_dom = sc.batches[dom][1].n
    contacts_dom = int(host_out[dom].astype(np.int64).sum())
    alg_bytes = n_dom * (IN_BYTES_PER_PAIR + 2) + contacts_dom * 48
    hbm_peak, peak_src = peaks()
    achieved = alg_bytes / (mean_batch[dom] / 1e3) / 1e9
    share = {nm: round(mean_batch[nm] / sum(mean_batch.values()), 4) for nm in names}
    label = ("narrowphase_kernel<7> + narrowphase_warp_kernel<mesh-box>" if algos[dom] == 6
             else f"narrowphase_kernel<{algos[dom]}>")
    roofline = {"bound": "hbm", "kernel": f"{label} ({dom})", "achieved": round(achieved, 2),
                "peak": hbm_peak, "unit": "GB/s", "frac": round(achieved / hbm_peak, 5), "traffic": None,
                "peak_source": peak_src, "kernel_ms": round(mean_batch[dom], 4), "share": share,
                "note": "FP32 SAT/GJK kernels are issue/latency-bound; HBM fraction is reported because no "
                        "FP32 CUDA-core peak is in MEASURED_PEAKS.json"}
    if args.traffic_bytes:
        roofline["traffic"] = args.traffic_bytes
    elif dom in TRAFFIC_PER_PAIR:
        # DRAM bytes (read + write) of the batch's launches from an ncu capture
        # of the 262,144-pair case, scaled by the pairs of this launch
        roofline["traffic"] = round(TRAFFIC_PER_PAIR[dom] * n_dom)
        roofline["traffic_source"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the same batch in the "
                                      "262,144-pair case (37,449 pairs), scaled by pairs")

    # ---- end to end through the host-memory C-ABI call -------------------
    e2e, pinned = None, None
    if not args.no_e2e:
        pinned = {}
        for nm in names:
            hp = sc.batches[nm][1]
            pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
            pp = A.HostPairs(pin(hp.shape1), pin(hp.shape2), pin(hp.pos1), pin(hp.rot1), pin(hp.pos2), pin(hp.rot2))
            ho = A.HostContacts(hp.n)
            for f in ("is_colliding", "nb_contacts", "normal_depth", "local1", "local2"):
                setattr(ho, f, torch.from_numpy(getattr(ho, f)).pin_memory().numpy())
            pinned[nm] = (pp, ho)
        # the whole narrow-phase input per call (testNarrowPhaseCollision):
        # the batches overlap, the contacts come back packed and the library's
        # host threads write them into the outputs
        step_batches = [(algos[nm], pinned[nm][0], pinned[nm][1]) for nm in names]
        call = ctx.narrowphase_input_call(step_batches)
        for _ in range(max(1, args.warmup)):
            call()
        h2d = sum(p.shape1.nbytes + p.shape2.nbytes + p.pos1.nbytes + p.rot1.nbytes + p.pos2.nbytes + p.rot2.nbytes
                  for p, _ in pinned.values())
        t0 = time.perf_counter()
        for _ in range(args.steps):
            call()
        e2e_s = (time.perf_counter() - t0) / args.steps
        # device-to-host bytes: flags and counts, and the contacts in use
        d2h = 0
        for nm in names:
            _, ho = pinned[nm]
            d2h += 2 * ho.n + 48 * int(ho.nb_contacts.astype(np.int64).sum())
        e2e_val = sc.n_pairs / e2e_s
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([e2e_s], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_val = pairs_total / float(t.item())
        e2e = {"value": round(e2e_val, 1), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e2e_s * 1e3, 4),
               "api": "rp3dg_narrowphase_input_host (all seven batches per call, pinned host buffers; the "
                      "batch descriptors built once, one C call per step)"}

    # ---- the headline's CPU baseline, then the other sections --------------
    # Every section below is guarded: an exception or the time budget records
    # {"error": ...} / {"skipped": ...} in its place instead of losing the
    # headline line.  A section that ends in a collective (many worlds) runs
    # on every rank; the single-world sections are replicas, run by rank 0.
    t_bench0 = T_START
    sections = {}
    solo = rank == 0
    cpu_ok = rank == 0 and not args.no_cpu

    def section(name, enabled, fn, every_rank=False):
        if not enabled:
            return None
        if not (every_rank or solo):
            return None
        left = args.budget_s - (time.perf_counter() - t_bench0)
        if left < 0 and not every_rank:
            sections[name] = {"skipped": f"time budget of {args.budget_s:.0f} s spent before this section"}
            return sections[name]
        t0 = time.perf_counter()
        try:
            r = fn()
        except Exception as e:  # recorded, never fatal for the headline
            r = {"error": f"{type(e).__name__}: {str(e)[:400]}"}
        if isinstance(r, dict):
            r["section_seconds"] = round(time.perf_counter() - t0, 2)
        sections[name] = r
        ctx.set_shapes(sc.shapes)   # the narrow-phase workload's table again
        return r

    cpu = section("cpu_baseline", cpu_ok and world == 1, lambda: cpu_baseline(sc, args))
    sections.pop("cpu_baseline", None)
    section("fp32_roofline", not args.no_fp32, lambda: fp32_section(ctx, sc, names, algos, dpairs, douts, mean_batch,
                                                                   args, dev, roofline))
    section("fp64_error", not args.no_cpu and not args.no_fp64, lambda: fp64_error_section(ctx, sc, names, algos, args, dev))
    section("manifolds", not args.no_manifolds,
            lambda: manifold_section(ctx, sc, names, algos, dpairs, douts, args, dev, pinned))
    section("dynamics", not args.no_dynamics, lambda: dynamics_section(ctx, args, dev, cpu_ok and world == 1))
    section("broadphase", not args.no_broadphase, lambda: broadphase_section(ctx, args, dev))
    section("world_step", not args.no_world, lambda: world_section(ctx, args, cpu_ok))
    section("many_worlds", not args.no_worlds, lambda: many_worlds_section(ctx, args, cpu_ok, rank, world),
            every_rank=True)
    section("learned_axis", not args.no_learned, lambda: learned_axis_section(ctx, sc, args, dev))
    section("many_worlds_1000_steps", not args.no_worlds and world == 1,
            lambda: worlds_long_section(ctx, args, cpu_ok))
    section("terrain_world", not args.no_terrain, lambda: terrain_section(ctx, args, cpu_ok))
    section("graph_coloured_solver", not args.no_terrain and not args.no_colored,
            lambda: colored_solver_section(ctx, args))

    line = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "pairs_per_gpu": sc.n_pairs, "batches": names,
                       "seed": args.seed, "l2": "flushed between steps (256 MB write)",
                       "parallelism": f"independent pair sets per rank x{world}"},
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu,
            "gpu_launches": int(launches),
            "clocks": clocks, "batch_ms": {k: round(v, 4) for k, v in mean_batch.items()}}
    line.update(sections)
    line["bench_seconds"] = round(time.perf_counter() - t_bench0, 1)
    if rank == 0:
        print(json.dumps(line), flush=True)
    try:
        ctx.close()
    except Exception:
        pass
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def fp64_error_section(ctx, sc, names, algos, args, dev):
    """Error of the GPU's FP32 contacts against the reference's double build
    (IS_RP3D_DOUBLE_PRECISION_ENABLED, oracle/_ref/librp3d_ref_f64.so) on the
    first args.fp64_sample pairs of every batch, fresh caches: the share of
    pairs on the same path (same colliding flag and contact count), then per
    contact the largest component error of the normal, the depth error and
    the largest component error of the two local points (metres), median and
    max.  The same sample through the reference's float build is checked
    bit for bit against the GPU, so these errors are the reference's own
    FP32 errors."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import reflib
    if not (reflib.have_ref("f64") and reflib.have_ref("f32")):
        return {"skipped": "reference builds (oracle/_ref) absent"}
    r32, r64 = reflib.RefEngine("f32"), reflib.RefEngine("f64")
    for e in (r32, r64):
        m = e.create_convex_mesh(sc.hull_vertices, sc.hull_faces)
        e.create_convex_mesh_shape(m)
    threads = _threads()
    res, identical = {}, True
    worst = {"normal": 0.0, "depth": 0.0, "point": 0.0}
    for nm in names:
        algo, pairs = sc.batches[nm]
        k = min(pairs.n, args.fp64_sample)
        ours = ctx.narrowphase_host(algo, pairs.slice(0, k))
        f32, _ = r32.narrowphase(algo, sc.shapes, pairs.slice(0, k), nthreads=threads)
        f64, _ = r64.narrowphase(algo, sc.shapes, pairs.slice(0, k), nthreads=threads)
        identical &= all(v == 0 for v in reflib.compare_contacts(ours, f32, k).values())
        same = (ours.is_colliding == f64.is_colliding) & (ours.nb_contacts == f64.nb_contacts)
        mask = ours.valid_mask() & same[None, :]
        nd = np.abs(ours.normal_depth.astype(np.float64) - f64.normal_depth)[mask]
        pt = np.maximum(np.abs(ours.local1.astype(np.float64) - f64.local1)[mask][:, :3].max(1),
                        np.abs(ours.local2.astype(np.float64) - f64.local2)[mask][:, :3].max(1))
        ne, de = nd[:, :3].max(1) if len(nd) else np.zeros(1), nd[:, 3] if len(nd) else np.zeros(1)
        pt = pt if len(pt) else np.zeros(1)
        q = lambda v: {"median": float(f"{np.median(v):.3g}"), "max": float(f"{v.max():.3g}")}
        res[nm] = {"pairs": k, "same_path": round(float(same.mean()), 6), "contacts": int(mask.sum()),
                   "normal": q(ne), "depth_m": q(de), "local_point_m": q(pt)}
        worst["normal"] = max(worst["normal"], float(ne.max()))
        worst["depth"] = max(worst["depth"], float(de.max()))
        worst["point"] = max(worst["point"], float(pt.max()))
    return {"oracle": "reference double build (IS_RP3D_DOUBLE_PRECISION_ENABLED), outputs rounded to float",
            "sample": f"first {args.fp64_sample} pairs of every batch, fresh caches", "batches": res,
            "max_error": {k: float(f"{v:.3g}") for k, v in worst.items()},
            "tolerance": {"normal": 1e-3, "depth_m": 1e-4, "local_point_m": 1e-3, "same_path": 0.999},
            "bit_identical_to_reference_f32_on_sample": bool(identical)}


def manifold_section(ctx, sc, names, algos, dpairs, douts, args, dev, pinned):
    """The convex manifold step after the narrow phase (reduction to <= 4
    points, de-duplication, last-frame update): device time of the reduction
    kernel on each batch's narrow-phase output (restored before every
    repetition, outside the timed events), its HBM roofline, and the host-array
    call that runs narrow phase + reduction and copies back only kept slots."""
    import torch
    from reactphysics3d_b200 import engine
    stream = ctx.torch_stream()
    reps = max(3, min(args.steps, 20))
    per = {}
    tot_ms, tot_bytes = 0.0, 0
    with torch.cuda.stream(stream):
        for nm in names:
            src = douts[nm]
            n = src.n
            work = engine.DeviceContacts(n, device=dev)
            kept = torch.empty((n, 4), dtype=torch.uint8, device=dev)
            nb = src.nb_contacts.to(torch.int64)
            ms = []
            for r in range(reps + 2):
                for f in ("is_colliding", "nb_contacts", "normal_depth", "local1", "local2"):
                    getattr(work, f).copy_(getattr(src, f))
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                ctx.reduce_contacts_device(dpairs[nm], work, kept)
                b.record(stream)
                if r >= 2:
                    ms.append((a, b))
            ctx.synchronize()
            t = float(np.mean([x.elapsed_time(y) for x, y in ms]))
            m = work.nb_contacts.to(torch.int64)
            # per pair: flag, count, orientation, cache flag byte, kept row, count
            # written; per raw point its local1 (16 B); per kept point 48 B read
            # and 48 B written
            alg = n * (1 + 1 + 16 + 1 + 4 + 1) + int(nb.sum()) * 16 + int(m.sum()) * 96
            per[nm] = {"ms": round(t, 4), "pairs_with_more_than_4": int((nb > 4).sum()),
                       "points_in": int(nb.sum()), "points_kept": int(m.sum()),
                       "achieved_gbs": round(alg / (t / 1e3) / 1e9, 1)}
            tot_ms += t
            tot_bytes += alg
    hbm_peak, _ = peaks()
    out = {"kernel": "contacts_reduce_kernel", "batches": per, "ms_per_step": round(tot_ms, 4),
           "pairs_per_s": round(sc.n_pairs / (tot_ms / 1e3), 1),
           "roofline": {"bound": "hbm", "achieved": round(tot_bytes / (tot_ms / 1e3) / 1e9, 1), "peak": hbm_peak,
                        "unit": "GB/s", "frac": round(tot_bytes / (tot_ms / 1e3) / 1e9 / hbm_peak, 4)}}
    if pinned is not None:
        for _ in range(2):
            for nm in names:
                ctx.narrowphase_manifolds_host(algos[nm], *pinned[nm], want_kept=False)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            for nm in names:
                ctx.narrowphase_manifolds_host(algos[nm], *pinned[nm], want_kept=False)
        dt = (time.perf_counter() - t0) / args.steps
        out["e2e_narrowphase_plus_manifolds"] = {"value": round(sc.n_pairs / dt, 1), "unit": UNIT,
                                                 "ms_per_step": round(dt * 1e3, 4),
                                                 "api": "rp3dg_narrowphase_manifolds_host (pinned host buffers)"}
    return out


DYNAMICS_FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", "np_dynamics.npz")


def dynamics_section(ctx, args, dev, with_cpu):
    """Dynamics stage of a world step (inertia, velocities, contact solver
    with 6 velocity iterations and split impulses, positions, state) for many
    independent worlds in one call: the reference worlds captured in
    tests/golden/np_dynamics.npz, replicated to args.dyn_worlds worlds.
    Device time per stage with CUDA events; the C restatement on one host
    core for the same worlds as the CPU figure."""
    import torch
    from reactphysics3d_b200 import dynamics as D
    z = np.load(DYNAMICS_FIXTURE)
    names = sorted({k.split("/")[0] for k in z.files})
    caps = [{k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(n + "/")} for n in names]
    base = [D.world_from_capture(c) for c in caps]
    reps = (args.dyn_worlds + len(base) - 1) // len(base)
    worlds = (base * reps)[: args.dyn_worlds]
    batch, _ = D.batch_worlds(worlds)
    params = D.params_from_capture(caps[0])
    cnt = batch.counts
    stream = ctx.torch_stream()
    # inputs are restored from a pristine device copy before every step
    # (outside the timed events), so each step solves the captured state
    src = D.DynWorld(batch.a, batch.nb_enabled, batch.nc_enabled, device=dev)
    work = D.DynWorld(batch.a, batch.nb_enabled, batch.nc_enabled, device=dev)
    steps = max(3, min(args.steps, 20))
    evs = []
    launches0 = ctx.kernel_launches()
    with torch.cuda.stream(stream):
        for s_ in range(steps + 2):
            for k in work.a:
                work.a[k].copy_(src.a[k])
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            ctx.dynamics_step(params, work)
            b.record(stream)
            if s_ >= 2:
                evs.append((a, b))
        ctx.synchronize()
    launches = (ctx.kernel_launches() - launches0) // (steps + 2)
    ms = float(np.mean([x.elapsed_time(y) for x, y in evs]))
    out = {"workload": f"{len(worlds)} worlds (reference captures of tests/golden/np_dynamics.npz, replicated)",
           "bodies": cnt["bodies"], "manifolds": cnt["manifolds"], "points": cnt["points"], "islands": cnt["islands"],
           "kernels_per_stage": int(launches), "ms_per_stage": round(ms, 4),
           "world_steps_per_s": round(len(worlds) / (ms / 1e3), 1),
           "bodies_per_s": round(cnt["bodies"] / (ms / 1e3), 1)}
    if with_cpu:
        import ctypes as C
        sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests"))
        import reflib
        if reflib.have_ref("f32"):
            # the reference's own dynamics stage (inertia, velocities,
            # solveContactsAndConstraints, positions, state) on the captured
            # worlds, rebuilt and stepped to their captured step
            sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden"))
            from make_golden import DYNAMICS_CASES
            per_case = []
            for kind, seed, nsteps, nx, ny, nz, variety in DYNAMICS_CASES:
                secs = []
                for _ in range(3):
                    w = reflib.RefWorld(kind=kind, seed=seed, nx=nx, ny=ny, nz=nz, variety=variety)
                    w.step(n=nsteps)
                    w.apply_forces(seed + 1)
                    secs.append(float(w.capture()["dyn_seconds"][0]))
                per_case.append(float(np.median(secs)))
            # the GPU's worlds are the captures replicated in equal numbers
            per_world = float(np.mean(per_case))
            out["cpu_baseline"] = {"value": round(1.0 / per_world, 1), "unit": "world-steps/s", "cores": 1,
                                   "kind": "reference",
                                   "sample": f"the {len(DYNAMICS_CASES)} captured worlds: the reference's dynamics "
                                             "stage of their captured step (median of 3 runs each), mean over the "
                                             "worlds, one core"}
        lib = C.CDLL(reflib.PORT_LIB)
        D.bind(lib, "rp3do_dynamics_step")
        n_cpu = max(len(base), len(worlds) // 16)
        cb, _ = D.batch_worlds(worlds[:n_cpu])
        t0 = time.perf_counter()
        b_, c_, m_, p_, i_ = cb.structs()
        lib.rp3do_dynamics_step(C.byref(params), C.byref(b_), C.byref(c_), C.byref(m_), C.byref(p_), C.byref(i_))
        dt_cpu = time.perf_counter() - t0
        port = {"value": round(n_cpu / dt_cpu, 1), "unit": "world-steps/s", "cores": 1, "kind": "port",
                "sample": f"{n_cpu} of the worlds, one stage, C restatement (oracle), one core"}
        if "cpu_baseline" in out:
            out["port_baseline"] = port
        else:
            out["cpu_baseline"] = port
    return out


def world_section(ctx, args, with_cpu):
    """The whole world step (PhysicsWorld::update) on the plain box pile:
    1,000 dynamic boxes falling onto a static ground, 300 steps at 1/60 s,
    through rp3dg_world_update (host API; synchronous, so wall-clock time is
    the metric).  The reference engine (oracle/_ref, built from its sources)
    steps the same world on one host core (it is single-threaded); the final
    states are compared bit for bit, and both against the reference's FP64
    build.  A second run with phase profiling gives the per-phase split."""
    from reactphysics3d_b200 import engine
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import reflib
    sc = scenes.box_pile()
    n = args.world_steps
    dt = float(np.float32(1.0 / 60.0))
    w = engine.World(ctx, sc)
    w.update(dt, 1)                  # first step: pair creation for every collider
    launches0 = ctx.kernel_launches()
    t0 = time.perf_counter()
    w.update(dt, n - 1)
    ctx.synchronize()
    sec = time.perf_counter() - t0
    launches = (ctx.kernel_launches() - launches0) / (n - 1)
    st = w.stats()
    ours = w.bodies()
    w.close()
    wp = engine.World(ctx, sc)
    wp.set_profiling(True)
    wp.update(dt, n)
    phases = {k: round(v / n, 4) for k, v in wp.phase_times().items()}
    wp.close()
    # the same pile with the graph-coloured solver (not the drop-in: another
    # constraint order, so other results), by residual and resting height
    wc = engine.World(ctx, sc)
    wc.set_solver(engine.SOLVER_GRAPH_COLORED, True)
    wc.update(dt, 1)
    t0 = time.perf_counter()
    res = []
    for _ in range(n - 1):
        wc.update(dt)
        res.append(wc.solver_stats())
    csec = time.perf_counter() - t0
    col_y = float(np.mean(wc.bodies()[0][:, 1]))
    wc.close()
    out = {"workload": "plain box pile: 1,000 boxes (half-extents U[0.25,0.75], density 1, friction 0.3, "
                       "restitution 0) on a 10x10x10 grid, 2 m spacing, lowest layer at y=2, +-0.1 m jitter, "
                       "random orientations, static ground box 50x0.5x50 at y=0; 300 steps at 1/60 s, "
                       "6 velocity iterations, sleeping on",
           "steps": n, "world_steps_per_s": round((n - 1) / sec, 1), "ms_per_step": round(1e3 * sec / (n - 1), 4),
           "kernels_per_step": round(launches, 1), "phase_ms_per_step": phases,
           "final_stats": st, "api": "rp3dg_world_update",
           "graph_coloured_solver": {
               "note": "not the drop-in: the constraints solved colour by colour, so the pile ends elsewhere",
               "world_steps_per_s": round((n - 1) / csec, 1),
               "residual_rms_last20": float(f"{np.mean([t['residual_rms'] for t in res[-20:]]):.4g}"),
               "colors_max": int(max(t["colors"] for t in res)),
               "mean_resting_height_m": round(col_y, 3),
               "exact_mean_resting_height_m": round(float(np.mean(ours[0][:, 1])), 3)}}
    if with_cpu and reflib.have_ref("f32"):
        r = reflib.RefScene(sc, "f32")
        r.update(dt, 1)
        t0 = time.perf_counter()
        r.update(dt, n - 1)
        rsec = time.perf_counter() - t0
        ref = r.bodies()
        out["cpu_baseline"] = {"value": round((n - 1) / rsec, 1), "unit": "world-steps/s", "cores": 1,
                               "kind": "reference", "sample": f"the same world, steps 2-{n}, PhysicsWorld::update "
                                                              "of the reference float build (single-threaded engine)"}
        out["bit_identical_to_reference"] = all(np.array_equal(a, b) for a, b in zip(ours, ref))
        if reflib.have_ref("f64"):
            r64 = reflib.RefScene(sc, "f64")
            r64.update(dt, n)
            d = np.linalg.norm(ours[0].astype(np.float64) - r64.bodies()[0], axis=1)
            out["fp64_position_deviation_m"] = {"median": round(float(np.median(d)), 5), "max": round(float(d.max()), 4),
                                                "note": "same for the reference float build (bit-identical); "
                                                        "a 1,000-body pile is chaotic"}
    return out


def many_worlds_section(ctx, args, with_cpu, rank=0, world=1):
    """Many independent worlds stepped together: 4,096 worlds of U[20, 200]
    dynamic boxes and spheres (sizes U[0.2, 1]) and 1-4 ragdolls (15 capsules,
    10 ball-and-socket + 4 hinge joints, 60-degree cones, +-60-degree hinge
    limits) falling onto a static ground each (scenes.many_worlds), dt 1/120,
    through one rp3dg_world_update per step of the whole group (wall clock,
    synchronous; the worlds' broad-phase trees are on the device, their
    reinsertions and queries on the GPU).  60 untimed steps, then 60 timed.  With N ranks the worlds
    are split into N contiguous blocks balanced by body count
    (reactphysics3d_b200.shard), each rank steps its block with
    cpu_count // N host threads, and the time is the slowest rank's (strong
    scaling: the 4,096 worlds are the whole job).  The reference engine
    steps a sample of the same worlds over the same steps on every host core
    (one PhysicsWorld per thread at a time, its own PhysicsCommon each), and
    the sampled worlds' final states are compared bit for bit."""
    from reactphysics3d_b200 import engine, shard
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import reflib
    n = args.n_worlds
    dt = float(np.float32(1.0 / 120.0))
    warm, timed = 60, 60
    raw_all = scenes.many_worlds(n, seed=args.seed, merge=False)
    lo, hi = shard.rank_block([len(s_.bodies) for s_ in raw_all], rank, world)
    shapes, scs = scenes.merge_shapes(raw_all[lo:hi])
    threads = max(1, (os.cpu_count() or 1) // world)
    ok, err = True, None
    try:
        g = engine.WorldGroup(ctx, scs, shapes, threads=threads)
        g.autotune(rounds=2)             # 18 of the warm-up steps: island scheduling (results unchanged)
        g.update(dt, warm)
        tuning = g.tuning()
        launches0 = ctx.kernel_launches()
        step_ms = []
        for _ in range(timed):
            t0 = time.perf_counter()
            g.update(dt)
            step_ms.append(1e3 * (time.perf_counter() - t0))
        sec = 1e-3 * sum(step_ms)
        launches = (ctx.kernel_launches() - launches0) / timed
    except Exception as e:   # every rank still takes part in the gather below
        ok, err, sec = False, f"{type(e).__name__}: {str(e)[:300]}", float("inf")
    sec_all = shard.max_over_ranks(sec)
    all_ok = all(shard.gather_objects(ok))
    if not all_ok:
        return {"error": err or "another rank failed", "rank_block": [lo, hi]}
    st = g.stats()
    g.set_profiling(True)
    g.update(dt, 5)
    phases = {k: round(v / 5, 3) for k, v in g.phase_times().items() if not k.startswith("m.")}
    out = {"workload": f"{n} independent worlds, U[20,200] boxes and spheres each (sizes U[0.2,1]) and 1-4 ragdolls "
                       "(15 capsules, 10 ball-and-socket + 4 hinge joints, 60-degree cones, +-60-degree hinge limits) "
                       "above a static ground box, random orientations, dt 1/120; steps 61-120 timed",
           "worlds": n, "bodies": int(sum(len(s_.bodies) for s_ in raw_all)),
           "world_steps_per_s": round(n * timed / sec_all, 1), "ms_per_step": round(1e3 * sec_all / timed, 3),
           "median_ms_per_step": round(float(np.median(step_ms)), 3), "min_ms_per_step": round(min(step_ms), 3),
           "note": "host-side bookkeeping runs on the box's shared host cores; the median and minimum step show "
                   "how much of the mean is host contention",
           "ranks": world, "scaling": "strong (the worlds are split over the ranks)",
           "rank0_block": [lo, hi], "kernels_per_step": round(launches, 1), "host_threads_per_rank": threads,
           "phase_ms_per_step": phases, "autotuned_scheduling": tuning,
           "device_trees": g.device_trees,
           "stats_at_step_120": st, "api": "rp3dg_world_update (world group)"}
    if with_cpu and reflib.have_ref("f32"):
        raw = raw_all[lo:hi]
        threads = _threads()
        nn = len(raw)
        sample = list(range(0, nn, max(1, nn // (8 * threads))))[: 8 * threads]
        refs = [reflib.RefScene(raw[k]) for k in sample]
        # warm-up steps on all threads, then the timed steps
        def run(idx, steps):
            for i in idx:
                refs[i].update(dt, steps)
        chunks = [list(range(t, len(refs), threads)) for t in range(threads)]
        ths = [threading.Thread(target=run, args=(c, warm)) for c in chunks]
        [t_.start() for t_ in ths]
        [t_.join() for t_ in ths]
        t0 = time.perf_counter()
        ths = [threading.Thread(target=run, args=(c, timed)) for c in chunks]
        [t_.start() for t_ in ths]
        [t_.join() for t_ in ths]
        rsec = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round(len(refs) * timed / rsec, 1), "unit": "world-steps/s", "cores": threads,
                               "kind": "reference",
                               "sample": f"{len(refs)} of the worlds, steps 61-120, PhysicsWorld::update of the "
                                         "reference float build, one world per thread at a time"}
        same, dev, spread = True, 0.0, 0.0
        for j, k in enumerate(sample[:16]):
            refs[j].update(dt, 5)   # the group ran 5 more (profiled) steps
            same &= all(np.array_equal(a, b) for a, b in zip(g.bodies(k), refs[j].bodies()))
            pr = refs[j].bodies()[0].astype(np.float64)
            dev = max(dev, float(np.abs(g.bodies(k)[0] - pr).max()))
            if reflib.have_ref("f64"):
                r64 = reflib.RefScene(raw[k], "f64")
                r64.update(dt, warm + timed + 5)
                spread = max(spread, float(np.abs(r64.bodies()[0] - pr).max()))
        out["bit_identical_sample"] = bool(same)
        out["parity"] = {"max_position_deviation_m": round(dev, 6),
                         "reference_fp32_vs_fp64_deviation_m": round(spread, 6),
                         "note": "16 sampled worlds after 125 steps; ragdoll cone / hinge limits use acos / atan2, "
                                 "whose last bit differs between CUDA and the host C library, so worlds whose limits "
                                 "engage are tolerance-level (worlds without limits are bit-identical: "
                                 "tests/test_world_gpu.py)"}
    digest = [np.asarray(g.bodies(k)[0], np.float64).sum() for k in range(0, hi - lo, 97)]
    g.close()
    if world == 1:
        try:
            out["two_groups_in_flight"] = _two_groups(raw_all, dt, warm, timed, digest)
        except Exception as e:
            out["two_groups_in_flight"] = {"error": f"{type(e).__name__}: {str(e)[:300]}"}
    return out


def _two_groups(raw, dt, warm, timed, digest):
    """The same worlds as two groups (halves balanced by body count), each on
    its own context and half the host threads, stepped from two host threads
    at once: one group's host bookkeeping runs while the other's kernels do.
    Same steps (autotuning, warm-up, timed, 5 more) as the single group, whose
    sampled final positions they must reproduce."""
    import threading
    from reactphysics3d_b200 import engine, shard
    n = len(raw)
    blocks = [shard.rank_block([len(s_.bodies) for s_ in raw], r, 2) for r in range(2)]
    threads = max(1, (os.cpu_count() or 2) // 2)
    parts = []
    for lo, hi in blocks:
        c = engine.Context(0)
        shapes, scs = scenes.merge_shapes(raw[lo:hi])
        g = engine.WorldGroup(c, scs, shapes, threads=threads)
        g.autotune(rounds=2)
        parts.append((c, g, lo, hi))

    def run(steps):
        ths = [threading.Thread(target=g.update, args=(dt, steps)) for _, g, _, _ in parts]
        t0 = time.perf_counter()
        [t_.start() for t_ in ths]
        [t_.join() for t_ in ths]
        return time.perf_counter() - t0
    run(warm)
    sec = run(timed)
    run(5)
    got = []
    for k in range(0, n, 97):
        for _, g, lo, hi in parts:
            if lo <= k < hi:
                got.append(np.asarray(g.bodies(k - lo)[0], np.float64).sum())
    for c, g, _, _ in parts:
        g.close()
        c.close()
    return {"world_steps_per_s": round(n * timed / sec, 1), "ms_per_step": round(1e3 * sec / timed, 3),
            "groups": 2, "host_threads_per_group": threads,
            "same_states_as_one_group": bool(np.array_equal(np.asarray(got), np.asarray(digest))),
            "note": "not a library mode: two rp3dg_world_update calls in flight from two host threads, one "
                    "context each; the timed region is the same 60 steps of all worlds"}


def terrain_section(ctx, args, with_cpu):
    """The single large world: 100,000 bodies (40% boxes with half-extents
    U[0.2,0.6], 30% spheres with radius U[0.2,0.5], 30% capsules of radius
    0.2 and half-height 0.3) on a jittered 3-D lattice with 1.5 m spacing above
    a 256 x 256-cell height field of 1 m cells whose heights are a seeded sum
    of 8 sines (wave numbers in [0.05, 0.5] rad/m, total amplitude 2 m),
    stepped at 1/60 s through rp3dg_world_update (wall clock, synchronous).
    Steps 2-21 (the bodies fall, the first ones land) are timed on both
    engines, the reference on one host core (it is single-threaded), and the
    states after step 21 compared bit for bit; the GPU then continues to step
    60 and times steps 61-80, when most bodies rest on the terrain and on each
    other (the contact-heavy regime: ~2 million triangle tests, ~10^5
    manifolds, one island of ~10^5 manifolds)."""
    from reactphysics3d_b200 import engine
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import reflib
    n_bodies = args.terrain_bodies
    sc = scenes.heightfield_world(n_bodies=n_bodies, cols=257, rows=257, seed=5)
    dt = float(np.float32(1.0 / 60.0))
    w = engine.World(ctx, sc)
    w.update(dt, 1)
    t0 = time.perf_counter()
    w.update(dt, 20)
    sec_early = time.perf_counter() - t0
    ours21 = w.bodies()
    st21 = w.stats()
    rays = scenes.terrain_rays(sc, args.rays)
    ray_out, ray_hits = raycast_measure(ctx, w, rays)
    w.update(dt, 39)
    launches0 = ctx.kernel_launches()
    t0 = time.perf_counter()
    w.update(dt, 20)
    sec = time.perf_counter() - t0
    launches = (ctx.kernel_launches() - launches0) / 20
    st = w.stats()
    ours80 = w.bodies()
    w.set_profiling(True)
    w.update(dt, 3)
    phases = {k: round(v / 3, 3) for k, v in w.phase_times().items() if not k.startswith("m.")}
    w.close()
    out = {"workload": f"{n_bodies:,} bodies (40% boxes, 30% spheres, 30% capsules) on a 1.5 m jittered lattice above a "
                       "256x256-cell height field (1 m cells, 8 seeded sines, amplitude 2 m), dt 1/60; "
                       "steps 61-80 timed",
           "bodies": n_bodies, "world_steps_per_s": round(20 / sec, 3), "ms_per_step": round(1e3 * sec / 20, 2),
           "kernels_per_step": round(launches, 1), "host_threads": os.cpu_count() or 1,
           "phase_ms_per_step": phases, "stats_at_step_80": st,
           "early_steps_2_21": {"world_steps_per_s": round(20 / sec_early, 3), "stats_at_step_21": st21},
           "api": "rp3dg_world_update"}
    if with_cpu and reflib.have_ref("f32"):
        r = reflib.RefScene(sc, "f32")
        r.update(dt, 1)
        t0 = time.perf_counter()
        r.update(dt, 20)
        rsec = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round(20 / rsec, 3), "unit": "world-steps/s", "cores": 1, "kind": "reference",
                               "sample": "the same world, steps 2-21, PhysicsWorld::update of the reference float "
                                         "build (single-threaded engine); compare early_steps_2_21"}
        out["bit_identical_to_reference_at_step_21"] = all(np.array_equal(a, b) for a, b in zip(ours21, r.bodies()))
        # the reference's PhysicsWorld::raycast on a sample of the same rays,
        # same state (step 21); its hits compared with the GPU's bit for bit
        ns = min(len(rays), args.ray_sample)
        t0 = time.perf_counter()
        rh, rc = r.raycast(rays[:ns], A.RAYCAST_CLOSEST, 1)
        rsec = time.perf_counter() - t0
        gh, gc = ray_hits
        ray_out["cpu_baseline"] = {"value": round(ns / rsec, 1), "unit": "rays/s", "cores": 1, "kind": "reference",
                                   "sample": f"the first {ns:,} rays, PhysicsWorld::raycast with a closest-hit "
                                             "callback, reference float build, one host core"}
        k = gc[:ns] > 0
        ray_out["bit_identical_to_reference_sample"] = bool(np.array_equal(gc[:ns], rc) and
                                                            gh[:ns][k].tobytes() == rh[k].tobytes())
        # after the landing: the reference continues to step 80 (~10^5
        # manifolds, one large island) and its states are compared again
        n_ref = args.terrain_ref_steps
        if n_ref > 21:
            t0 = time.perf_counter()
            r.update(dt, min(n_ref, 80) - 21)
            out["reference_steps_22_to_80_seconds"] = round(time.perf_counter() - t0, 1)
            out["bit_identical_to_reference_at_step_80"] = all(np.array_equal(a, b)
                                                               for a, b in zip(ours80, r.bodies()))
    out["raycast_at_step_21"] = ray_out
    return out


def colored_solver_section(ctx, args):
    """The graph-coloured contact solver (RP3DG_SOLVER_GRAPH_COLORED, not the
    drop-in) against the exact-order solver on the 100,000-body terrain world:
    each solver steps its own copy of the world to args.colored_steps (the
    bodies settle into one island of ~10^5 manifolds), the last 20 steps are
    timed, and every step records the velocity constraint residual over the
    contact points and the bodies' kinetic + potential energy."""
    from reactphysics3d_b200 import engine
    n_bodies = args.terrain_bodies
    sc = scenes.heightfield_world(n_bodies=n_bodies, cols=257, rows=257, seed=5)
    dt = float(np.float32(1.0 / 60.0))
    steps = args.colored_steps
    out = {"workload": f"{n_bodies:,}-body terrain world (as terrain_world), steps 1-{steps}, last 20 timed",
           "note": "the graph-coloured solver changes the constraint order, so its results differ from the "
                   "reference's; it is reported by residual and energy beside the exact (drop-in) solver"}
    for name, solver in (("exact", engine.SOLVER_EXACT), ("graph_coloured", engine.SOLVER_GRAPH_COLORED)):
        w = engine.World(ctx, sc)
        w.set_solver(solver, True)
        trace = []
        for s_ in range(steps - 20):
            w.update(dt)
            trace.append(w.solver_stats())
        t0 = time.perf_counter()
        for s_ in range(20):
            w.update(dt)
            trace.append(w.solver_stats())
        sec = time.perf_counter() - t0
        w.set_profiling(True)
        w.update(dt, 2)
        ph = w.phase_times()
        st = w.stats()
        w.close()
        e = np.array([t["kinetic_energy"] + t["potential_energy"] for t in trace])
        res = np.array([t["residual_rms"] for t in trace[-20:]])
        out[name] = {"world_steps_per_s": round(20 / sec, 3), "ms_per_step": round(1e3 * sec / 20, 2),
                     "dynamics_ms_per_step": round(ph.get("dynamics", 0.0) / 2, 3),
                     "residual_rms_last20": float(f"{res.mean():.4g}"),
                     "residual_max_last20": float(f"{max(t['residual_max'] for t in trace[-20:]):.4g}"),
                     "energy_J": {f"step_{k}": round(float(e[k - 1]), 1) for k in (1, steps // 2, steps)},
                     "kinetic_energy_J_last": round(float(trace[-1]["kinetic_energy"]), 2),
                     "largest_energy_rise_J_per_step": round(float(np.max(np.diff(e))) if len(e) > 1 else 0.0, 3),
                     "colors_last": int(trace[-1]["colors"]), "islands": st["islands"],
                     "manifolds": st["manifolds"]}
    return out


def worlds_long_section(ctx, args, with_cpu):
    """Parity of the many-worlds workload over its full length: a sample of
    its worlds (every (n / sample)-th world of the same seeded batch) stepped
    as one group for args.worlds_long_steps steps at 1/120 s, then every
    sampled world's body states compared with the reference's float build
    (bit for bit; ragdoll cone / hinge limits use acos / atan2, whose last bit
    differs between CUDA and the host C library, so a world whose limits
    engaged is held to a tolerance instead) and with the reference's double
    build, whose distance to the float build is the spread the tolerance is
    stated against.  The same sample with the ragdolls' limits off (no acos /
    atan2 on the path) is compared bit for bit over the same steps."""
    from reactphysics3d_b200 import engine
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import reflib
    if not (with_cpu and reflib.have_ref("f32") and reflib.have_ref("f64")):
        return {"skipped": "reference builds (oracle/_ref) absent or CPU legs disabled"}
    n, ns, steps = args.n_worlds, args.worlds_long_sample, args.worlds_long_steps
    dt = float(np.float32(1.0 / 120.0))
    idx = list(range(0, n, max(1, n // ns)))[:ns]
    threads = _threads()

    def run_sample(raw, precisions):
        shapes, scs = scenes.merge_shapes([raw[k] for k in idx])
        g = engine.WorldGroup(ctx, scs, shapes, threads=threads)
        t0 = time.perf_counter()
        g.update(dt, steps)
        gpu_s = time.perf_counter() - t0
        ours = [g.bodies(j) for j in range(len(idx))]
        g.close()
        refs = {p: [reflib.RefScene(raw[k], p) for k in idx] for p in precisions}

        def run(chunk):
            for p, j in chunk:
                refs[p][j].update(dt, steps)
        jobs = [(p, j) for p in precisions for j in range(len(idx))]
        ths = [threading.Thread(target=run, args=(jobs[t::threads],)) for t in range(threads)]
        t0 = time.perf_counter()
        [t_.start() for t_ in ths]
        [t_.join() for t_ in ths]
        return ours, refs, gpu_s, time.perf_counter() - t0

    ours, refs, gpu_s, ref_s = run_sample(scenes.many_worlds(n, seed=args.seed, merge=False), ("f32", "f64"))
    same, within, dev_max, spread_max = 0, 0, 0.0, 0.0
    for j in range(len(idx)):
        a = refs["f32"][j].bodies()
        if all(np.array_equal(x, y) for x, y in zip(ours[j], a)):
            same += 1
        p32 = a[0].astype(np.float64)
        dev = float(np.abs(ours[j][0].astype(np.float64) - p32).max())
        spread = float(np.abs(refs["f64"][j].bodies()[0] - p32).max())
        within += dev <= spread
        dev_max, spread_max = max(dev_max, dev), max(spread_max, spread)
    ours_nl, refs_nl, _, _ = run_sample(scenes.many_worlds(n, seed=args.seed, merge=False, limits=False), ("f32",))
    same_nl = sum(all(np.array_equal(x, y) for x, y in zip(ours_nl[j], refs_nl["f32"][j].bodies()))
                  for j in range(len(idx)))
    return {"workload": f"{len(idx)} of the {n} many-worlds worlds (every {max(1, n // ns)}-th), {steps} steps at "
                        "1/120 s as one group",
            "worlds": len(idx), "steps": steps, "gpu_seconds": round(gpu_s, 2),
            "reference_seconds_f32_and_f64": round(ref_s, 2), "reference_threads": threads,
            "bit_identical_worlds": same, "worlds_within_fp32_fp64_spread": int(within),
            "max_position_deviation_m": float(f"{dev_max:.3g}"),
            "max_reference_fp32_vs_fp64_deviation_m": float(f"{spread_max:.3g}"),
            "limits_off": {"note": "the same worlds with the ragdolls' cone and hinge limits off",
                           "bit_identical_worlds": int(same_nl), "worlds": len(idx)}}


def raycast_measure(ctx, w, rays, reps=5):
    """rp3dg_world_raycast_device on device-resident rays (kernel time by CUDA
    events, after a first call that also builds the tree tables) and
    rp3dg_world_raycast on host arrays (wall clock, copies included)."""
    import torch
    dev = torch.device("cuda", 0)
    n = len(rays)
    d_rays = torch.from_numpy(rays.view(np.uint8)).to(dev)
    d_hits = torch.empty(n * A.RAYCAST_HIT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    d_cnt = torch.empty(n, dtype=torch.int32, device=dev)
    t0 = time.perf_counter()
    w.raycast_device(d_rays.data_ptr(), n, d_hits.data_ptr(), d_cnt.data_ptr())
    first = time.perf_counter() - t0
    ms = [w.raycast_device(d_rays.data_ptr(), n, d_hits.data_ptr(), d_cnt.data_ptr()) for _ in range(reps)]
    t0 = time.perf_counter()
    for _ in range(reps):
        hits, counts = w.raycast(rays, A.RAYCAST_CLOSEST, 1)
    e2e = (time.perf_counter() - t0) / reps
    kms = float(np.median(ms))
    out = {"rays": n, "mode": "closest hit", "rays_per_s": round(n / (kms * 1e-3), 1), "kernel_ms": round(kms, 3),
           "first_call_ms": round(1e3 * first, 3),
           "e2e": {"rays_per_s": round(n / e2e, 1), "ms": round(1e3 * e2e, 3),
                   "h2d_bytes": int(rays.nbytes), "d2h_bytes": int(hits.nbytes + counts.nbytes)},
           "hit_rays": int((counts > 0).sum()),
           "api": "rp3dg_world_raycast_device / rp3dg_world_raycast"}
    return out, (hits[:, 0], counts)


def broadphase_section(ctx, args, dev):
    """Broad phase of a single large world: 100,000 colliders (40% boxes, 30%
    spheres, 30% capsules, sizes of the large-world workload) on a jittered
    50 x 40 x 50 lattice with 1.5 m spacing, random orientations: the fat-AABB
    update of every collider (after a small random displacement, so part of
    them are reinserted) and the overlapping-pair search, device time with
    CUDA events."""
    import torch
    from reactphysics3d_b200 import broadphase as BP
    rng = np.random.default_rng(args.seed + 17)
    nx, ny, nz = 50, 40, 50
    n = nx * ny * nz
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    pos = (g * 1.5 + rng.uniform(-0.1, 0.1, (n, 3))).astype(np.float32)
    kind = rng.choice([2, 0, 1], size=n, p=[0.4, 0.3, 0.3]).astype(np.int32)
    table = np.zeros(n, A.SHAPE_DTYPE)
    table["kind"] = kind
    table["params"][:, 0] = np.where(kind == 0, rng.uniform(0.2, 0.5, n), np.where(kind == 1, 0.2, rng.uniform(0.2, 0.6, n)))
    table["params"][:, 1] = np.where(kind == 1, 0.3, rng.uniform(0.2, 0.6, n))
    table["params"][:, 2] = rng.uniform(0.2, 0.6, n)
    q = rng.normal(size=(n, 4)).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    wpos = np.zeros((n, 4), np.float32); wpos[:, :3] = pos
    ctx.set_shapes(table)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    shape, wp, wo = T(np.arange(n, dtype=np.int32)), T(wpos), T(q)
    body = T(np.arange(n, dtype=np.int32))
    fmin = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    fmax = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    moved = torch.zeros(n, dtype=torch.uint8, device=dev)
    force = T(np.ones(n, np.uint8))
    bp0 = BP.make(n, n, 0, shape=shape, body=body, world_position=wp, world_orientation=wo, force_reinsert=force,
                  fat_min=fmin, fat_max=fmax, moved=moved)
    ctx.broadphase_update(bp0)           # initial fat AABBs
    wpos2 = wpos.copy()
    wpos2[:, :3] += rng.normal(scale=0.02, size=(n, 3)).astype(np.float32)
    wp2 = T(wpos2)
    bp = BP.make(n, n, 0, shape=shape, body=body, world_position=wp2, world_orientation=wo, fat_min=fmin,
                 fat_max=fmax, moved=moved)
    fmin0, fmax0 = fmin.clone(), fmax.clone()
    stream = ctx.torch_stream()
    reps = max(3, min(args.steps, 20))
    cap = 4 * n
    res = {}
    for method, axis in (("lbvh", -1), ("sweep_x", 0)):
        ev_u, ev_p = [], []
        with torch.cuda.stream(stream):
            for r in range(reps + 2):
                fmin.copy_(fmin0); fmax.copy_(fmax0)
                a0, a1, a2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
                a0.record(stream)
                ctx.broadphase_update(bp)
                a1.record(stream)
                cnt, pairs = ctx.broadphase_pairs(bp, cap, axis=axis, device=True)
                a2.record(stream)
                if r >= 2:
                    ev_u.append((a0, a1)); ev_p.append((a1, a2))
            ctx.synchronize()
        c = int(cnt.item())
        pr = pairs[:c].cpu().numpy().astype(np.int64)
        res[method] = {"pairs": c, "update_ms": float(np.mean([x.elapsed_time(y) for x, y in ev_u])),
                       "pairs_ms": float(np.mean([x.elapsed_time(y) for x, y in ev_p])),
                       "set": np.sort(pr[:, 0] * n + pr[:, 1])}
    lb, sw = res["lbvh"], res["sweep_x"]
    tu, tp = lb["update_ms"], lb["pairs_ms"]
    return {"workload": "one world, 100,000 colliders (40% boxes, 30% spheres, 30% capsules) on a 50x40x50 "
                        "lattice, 1.5 m spacing, 2 cm random displacement",
            "colliders": n, "reinserted": int(moved.sum().item()), "pairs": lb["pairs"],
            "method": "LBVH (Morton keys, Karras tree, refit, warp-cooperative traversal)",
            "update_ms": round(tu, 4), "pairs_ms": round(tp, 4),
            "colliders_per_s": round(n / ((tu + tp) / 1e3), 1),
            "sweep_and_prune_pairs_ms": round(sw["pairs_ms"], 4),
            "same_pair_set_as_sweep": bool(np.array_equal(lb["set"], sw["set"]))}


def learned_axis_section(ctx, sc, args, dev):
    """Learned separating-axis proposal vs plain SAT on the box-box and
    hull-box batches of the workload (the polyhedron pairs): train the MLP on
    labels from a fresh full-SAT frame, then time both variants on that frame
    (fresh caches) and on the next frame (moved poses, caches of the previous
    frame: the temporal-coherence path), checking contacts are bit-identical."""
    import torch
    from reactphysics3d_b200 import engine
    names = [nm for nm in ("box_box", "hull_box") if nm in sc.batches]
    mlp = engine.AxisMLP(ctx, seed=args.seed)
    stream = ctx.torch_stream()
    frames = {}
    xs, ys = [], []
    rng = np.random.default_rng(args.seed + 7)
    for nm in names:
        algo, pairs = sc.batches[nm]
        p1 = pairs.slice(0, pairs.n)
        p1.cache = A.fresh_cache(p1.n)
        dp = engine.DevicePairs(p1, device=dev)
        out = engine.DeviceContacts(p1.n, device=dev)
        ctx.narrowphase_device(algo, dp, out)
        xs.append(mlp.features(dp))
        ys.append(mlp.labels(dp, out))
        ctx.synchronize()
        c1 = dp.host_cache()
        p2 = _moved(p1, rng)
        p2.cache = _next_cache(c1, out.is_colliding.cpu().numpy())
        frames[nm] = (algo, A.fresh_cache(p1.n), p1, p2)
    x, y = torch.cat(xs), torch.cat(ys)
    perm = torch.randperm(x.shape[0], generator=torch.Generator().manual_seed(args.seed)).to(dev)
    x, y = x[perm].contiguous(), y[perm].contiguous()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    engine.train_axis_mlp(ctx, mlp, x, y, epochs=args.learned_epochs, batch=4096, lr=3e-3, seed=args.seed)
    ctx.synchronize()
    train_s = time.perf_counter() - t0
    pred = mlp.predict(x).cpu().numpy()
    acc = float(np.mean(pred == y.cpu().numpy()))

    def timed(frame, learned_on, reps=5):
        res = {}
        for nm in names:
            algo, fresh, p1, p2 = frames[nm]
            src = p1 if frame == 1 else p2
            dp = engine.DevicePairs(src, device=dev)
            cache0 = dp.cache.clone()
            out = engine.DeviceContacts(src.n, device=dev)
            mlp.enable(learned_on)
            ms = []
            for r in range(reps + 1):
                dp.cache.copy_(cache0)
                torch.cuda.synchronize()
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                ev0.record(stream)
                ctx.narrowphase_device(algo, dp, out)
                ev1.record(stream)
                ctx.synchronize()
                if r > 0:
                    ms.append(ev0.elapsed_time(ev1))
            mlp.enable(False)
            res[nm] = (float(np.median(ms)), out.to_host())
        return res

    report = {"train_samples": int(x.shape[0]), "train_epochs": args.learned_epochs,
              "train_seconds": round(train_s, 3), "train_accuracy": round(acc, 4)}
    identical = True
    for frame in (1, 2):
        plain = timed(frame, False)
        mlp.stats(clear=True)
        learn = timed(frame, True)
        tested, confirmed = mlp.stats(clear=True)
        n = sum(frames[nm][2].n for nm in names)
        for nm in names:
            mism = _compare(plain[nm][1], learn[nm][1])
            identical = identical and mism == 0
        pl_ms = sum(plain[nm][0] for nm in names)
        le_ms = sum(learn[nm][0] for nm in names)
        report[f"frame{frame}"] = {
            "cache": "fresh" if frame == 1 else "previous frame",
            "plain_pairs_per_s": round(n / (pl_ms / 1e3), 1), "learned_pairs_per_s": round(n / (le_ms / 1e3), 1),
            "plain_ms": {nm: round(plain[nm][0], 4) for nm in names},
            "learned_ms": {nm: round(learn[nm][0], 4) for nm in names},
            "speedup": round(pl_ms / le_ms, 3),
            "proposals_tested": int(tested // 6), "proposals_confirmed": int(confirmed // 6),
            "confirmed_rate": round(confirmed / max(1, 6 * n), 4)}
    report["contacts_bit_identical"] = bool(identical)
    return report


def _moved(p, rng, dpos=0.02, drot=0.02):
    q = A.HostPairs(p.shape1, p.shape2, p.pos1.copy(), p.rot1.copy(), p.pos2.copy(), p.rot2.copy())
    q.pos2[:, :3] += rng.uniform(-dpos, dpos, (p.n, 3)).astype(np.float32)
    r = q.rot2.astype(np.float64) + rng.uniform(-drot, drot, (p.n, 4))
    q.rot2[:] = (r / np.linalg.norm(r, axis=1, keepdims=True)).astype(np.float32)
    return q


def _next_cache(cache, colliding):
    c = cache.copy()
    c["flags"] |= A.LF_IS_VALID
    c["flags"] &= ~np.uint8(A.LF_WAS_COLLIDING)
    c["flags"] |= np.where(colliding != 0, A.LF_WAS_COLLIDING, 0).astype(np.uint8)
    return c


def _compare(a, b):
    if not (np.array_equal(a.is_colliding, b.is_colliding) and np.array_equal(a.nb_contacts, b.nb_contacts)):
        return 1
    m = a.valid_mask()
    bad = 0
    for f in ("normal_depth", "local1", "local2"):
        bad += int(np.sum(getattr(a, f)[m].view(np.uint32) != getattr(b, f)[m].view(np.uint32)))
    return bad


def _reference_engine():
    """The reference's own algorithms (oracle/_ref, built from its sources);
    the C restatement (oracle/librp3d_oracle.so) when the reference build is
    absent.  Returns (engine, kind)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import reflib
    if reflib.have_ref("f32"):
        return reflib.RefEngine("f32"), "reference"
    if not os.path.exists(reflib.PORT_LIB):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True, stdout=subprocess.DEVNULL)
    return reflib.PortEngine(), "port"


def _threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def fp32_section(ctx, sc, names, algos, dpairs, douts, mean_batch, args, dev, roofline):
    """FP32 roofline of every batch: the batch's inputs go once through the
    event-counting build of the kernels (rp3dg_narrowphase_count_events,
    untimed), the path events times the static op table
    (reactphysics3d_b200.roofline) give the reference's FP32 operations for
    those pairs, and dividing by the batch's timed device time gives the
    achieved rate.  The peak is this device's multiply + add rate measured by
    the library's microkernel (the kernels are compiled without FMA
    contraction, so fused multiply-adds are not available to them); the FMA
    rate is reported beside it.  The headline roofline becomes the dominant
    batch's FP32 roofline, with its HBM figures kept under "hbm"."""
    from reactphysics3d_b200 import engine
    from reactphysics3d_b200 import roofline as RF
    peak = ctx.measure_fp32_peak(fused=False) / 1e12
    peak_fma = ctx.measure_fp32_peak(fused=True) / 1e12
    per, tot_ops, tot_ms = {}, 0.0, 0.0
    for nm in names:
        scratch = engine.DeviceContacts(dpairs[nm].n, device=dev)
        ev = ctx.narrowphase_count_events(algos[nm], dpairs[nm], scratch)
        ops = RF.fp32_ops(algos[nm], ev)
        ms = mean_batch[nm]
        per[nm] = {"fp32_ops": round(ops), "ops_per_pair": round(ops / dpairs[nm].n, 1), "kernel_ms": round(ms, 4),
                   "achieved_tflops": round(ops / (ms * 1e-3) / 1e12, 3),
                   "frac": round(ops / (ms * 1e-3) / 1e12 / peak, 4), "events": RF.named(ev)}
        tot_ops += ops
        tot_ms += ms
    dom = max(mean_batch, key=mean_batch.get)
    hbm = {k: roofline[k] for k in ("bound", "achieved", "peak", "unit", "frac", "peak_source") if k in roofline}
    d = per[dom]
    roofline.update({"bound": "fp32", "achieved": d["achieved_tflops"], "peak": round(peak, 2), "unit": "TFLOP/s",
                     "frac": d["frac"], "peak_source": "measured: rp3dg_measure_fp32_peak, separate FP32 multiplies "
                                                       "and adds (the kernels' arithmetic: no FMA contraction)",
                     "fma_peak": round(peak_fma, 2), "frac_of_fma_peak": round(d["achieved_tflops"] / peak_fma, 4),
                     "algorithmic_flops": "reference code-path operations: path events x static op table "
                                          "(reactphysics3d_b200/roofline.py)",
                     "hbm": hbm,
                     "whole_step": {"achieved_tflops": round(tot_ops / (tot_ms * 1e-3) / 1e12, 3),
                                    "frac": round(tot_ops / (tot_ms * 1e-3) / 1e12 / peak, 4)}})
    roofline.pop("note", None)
    return {"peak_tflops_mul_add": round(peak, 2), "peak_tflops_fma": round(peak_fma, 2), "batches": per}


def cpu_baseline(sc, args, sample_frac=None, repeats=1):
    """Time the reference engine's algorithms on the host cores over a bounded
    sample (every batch cut to the same fraction) of the workload."""
    eng, kind = _reference_engine()
    m = eng.create_convex_mesh(sc.hull_vertices, sc.hull_faces)
    eng.create_convex_mesh_shape(m)
    threads = _threads() if kind == "reference" else 1
    frac = sample_frac if sample_frac is not None else args.cpu_sample
    total_pairs, total_s = 0, 0.0
    for nm, (algo, pairs) in sc.batches.items():
        k = max(threads, int(pairs.n * frac))
        sub = pairs.slice(0, k)
        if kind == "reference":
            _, sec = eng.narrowphase(algo, sc.shapes, sub, nthreads=threads, repeats=repeats)
        else:
            t0 = time.perf_counter()
            eng.narrowphase(algo, sc.shapes, sub)
            sec = time.perf_counter() - t0
        total_pairs += k
        total_s += sec
    return {"value": round(total_pairs / total_s, 1), "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"first {frac:.0%} of every batch ({total_pairs} pairs), testCollision on pre-filled "
                      f"NarrowPhaseInfoBatch, one batch slice per thread",
            "seconds": round(total_s, 3)}


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    sc = scenes.narrowphase_scene(total_pairs=args.pairs, seed=args.seed)
    vals = []
    base = None
    # each step is one pass of the reference's algorithms over the sample; the
    # value is the median over the (at least 5) timed steps, which damps the
    # load of other processes on the shared host
    steps = max(5, args.steps)
    for s in range(args.warmup + steps):
        r = cpu_baseline(sc, args, repeats=1)
        if s >= args.warmup:
            vals.append(r["value"])
            base = r
    value = float(np.median(vals))
    base["value"] = round(value, 1)
    base["steps_timed"] = steps
    base["spread"] = {"min": round(min(vals), 1), "max": round(max(vals), 1)}
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * args.pairs / value, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "pairs_per_gpu": args.pairs, "seed": args.seed,
                       "sample": base["sample"]},
            "cpu_baseline": base,
            "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--pairs", type=int, default=scenes.TOTAL_PAIRS)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--cpu-sample", type=float, default=0.25)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--traffic-bytes", type=float, default=None)
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-manifolds", action="store_true")
    ap.add_argument("--no-dynamics", action="store_true")
    ap.add_argument("--no-broadphase", action="store_true")
    ap.add_argument("--dyn-worlds", type=int, default=4096)
    ap.add_argument("--no-world", action="store_true")
    ap.add_argument("--no-worlds", action="store_true")
    ap.add_argument("--no-terrain", action="store_true")
    ap.add_argument("--terrain-bodies", type=int, default=100000)
    ap.add_argument("--rays", type=int, default=1 << 20)
    ap.add_argument("--ray-sample", type=int, default=20000)
    ap.add_argument("--n-worlds", type=int, default=4096)
    ap.add_argument("--world-steps", type=int, default=300)
    ap.add_argument("--learned-epochs", type=int, default=4)
    ap.add_argument("--budget-s", type=float, default=1500.0,
                    help="sections that would start after this many seconds are skipped (recorded as such)")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--fp64-sample", type=int, default=20000)
    ap.add_argument("--terrain-ref-steps", type=int, default=80,
                    help="the reference steps the large world this far and its states are compared with the GPU's")
    ap.add_argument("--no-colored", action="store_true")
    ap.add_argument("--colored-steps", type=int, default=200)
    ap.add_argument("--worlds-long-steps", type=int, default=1000)
    ap.add_argument("--worlds-long-sample", type=int, default=64)
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: start the ranks through torch's launcher
        # (rendezvous on the loopback address) and pass every argument on
        import socket
        s = socket.socket()
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
        s.close()
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
        sys.exit(subprocess.run(cmd).returncode)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
