"""Step one of the generated worlds on the GPU and print its statistics.

    python -m reactphysics3d_b200.run_world terrain --bodies 100000 --cols 257 --steps 156
    python -m reactphysics3d_b200.run_world pile --steps 300 --phases
    python -m reactphysics3d_b200.run_world terrain --bodies 20000 --steps 21 --rays 1048576
    python -m reactphysics3d_b200.run_world worlds --worlds 4096 --dt 0.008333334 --steps 70 --phases

Scenes: `pile` (scenes.box_pile), `mixed` (scenes.mixed_world), `terrain`
(scenes.heightfield_world: --bodies bodies over a --cols x --cols height
field), `ragdolls` (scenes.ragdoll_world), `worlds` (--worlds independent
worlds of scenes.many_worlds stepped as one group, rp3dg_world_group_create;
--host-trees keeps their broad-phase trees on the host).  The world is created, stepped
--steps times at --dt and synchronised; nothing else is launched, so kernel
launch counts (for a profiler's skip / count options) follow from the step
count.  --phases prints the per-phase host / device times per step
(rp3dg_world_set_profiling) of the last --phase-steps steps.  --rays casts
that many rays (scenes.terrain_rays for a terrain, closest hit) --ray-reps
times through rp3dg_world_raycast after the steps (one raycast kernel launch
each).
"""
import argparse
import json
import time

from . import engine, scenes


def make_scene(args):
    if args.scene == "pile":
        return scenes.box_pile(seed=args.seed if args.seed is not None else 1)
    if args.scene == "mixed":
        return scenes.mixed_world(seed=args.seed if args.seed is not None else 2)
    if args.scene == "ragdolls":
        return scenes.ragdoll_world(n_ragdolls=args.bodies or 8, seed=args.seed if args.seed is not None else 23)
    n = args.bodies or 100000
    seed = args.seed if args.seed is not None else (31 if n < 50000 else 5)
    return scenes.heightfield_world(n_bodies=n, cols=args.cols, rows=args.cols, seed=seed)


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("scene", choices=["pile", "mixed", "terrain", "ragdolls", "worlds"])
    ap.add_argument("--worlds", type=int, default=4096)
    ap.add_argument("--host-trees", action="store_true")
    ap.add_argument("--bodies", type=int, default=None)
    ap.add_argument("--cols", type=int, default=257)
    ap.add_argument("--seed", type=int, default=None)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--dt", type=float, default=1.0 / 60.0)
    ap.add_argument("--threads", type=int, default=None)
    ap.add_argument("--phases", action="store_true")
    ap.add_argument("--phase-steps", type=int, default=5)
    ap.add_argument("--rays", type=int, default=0)
    ap.add_argument("--ray-reps", type=int, default=1)
    args = ap.parse_args()
    ctx = engine.Context(0)
    if args.scene == "worlds":
        shapes, scs = scenes.many_worlds(args.worlds, seed=args.seed if args.seed is not None else 7)
        w = engine.WorldGroup(ctx, scs, shapes, threads=args.threads)
        if args.host_trees:
            w.set_device_trees(False)
        sc = scs[0]
    else:
        sc = make_scene(args)
        w = engine.World(ctx, sc, threads=args.threads)
    n_plain = args.steps - (min(args.phase_steps, args.steps) if args.phases else 0)
    t0 = time.perf_counter()
    w.update(args.dt, n_plain)
    ctx.synchronize()
    sec = time.perf_counter() - t0
    out = {"scene": f"{args.worlds} worlds" if args.scene == "worlds" else sc.name, "steps": args.steps,
           "ms_per_step": round(1e3 * sec / max(n_plain, 1), 3), "stats": w.stats()}
    if args.scene == "worlds":
        out["device_trees"] = w.device_trees
    if args.phases and args.steps > n_plain:
        w.set_profiling(True)
        w.update(args.dt, args.steps - n_plain)
        out["phase_ms_per_step"] = {k: round(v / (args.steps - n_plain), 3) for k, v in w.phase_times().items()}
    if args.rays:
        if not sc.heightfields:
            raise SystemExit("--rays needs the terrain scene")
        rays = scenes.terrain_rays(sc, args.rays)
        t0 = time.perf_counter()
        for _ in range(args.ray_reps):
            hits, counts = w.raycast(rays)
        out["raycast"] = {"rays": args.rays, "reps": args.ray_reps, "hit_rays": int((counts > 0).sum()),
                          "ms_per_call": round(1e3 * (time.perf_counter() - t0) / args.ray_reps, 3)}
    print(json.dumps(out))
    w.close()
    ctx.close()


if __name__ == "__main__":
    main()
