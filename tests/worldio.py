"""World trajectories in a compact, comparable form: per step the overlapping
pair ids (in array order) and the solver's contact manifolds, each as a count
and a 64-bit digest, plus the body state at checkpoints.  Used by the golden
world fixture (tests/golden/make_golden.py world) and the world tests."""
import hashlib

import numpy as np

from reactphysics3d_b200 import scenes

# name -> (scene factory, kwargs, steps, checkpoint every)
WORLD_CASES = {
    "pile125": (scenes.box_pile, dict(nx=5, ny=5, nz=5, seed=3), 240, 60),
    "mixed100": (scenes.mixed_world, dict(nx=5, ny=4, nz=5, seed=5), 200, 50),
    "ragdolls4": (scenes.ragdoll_world, dict(n_ragdolls=4, seed=23, limits=False, boxes=6), 240, 60),
    # boxes, spheres and capsules falling onto a height-field terrain
    "terrain60": (scenes.heightfield_world, dict(n_bodies=60, cols=24, rows=24, seed=11), 240, 60),
    # a scaled terrain on a tilted, shifted static body
    "terrain_tilt": (scenes.heightfield_world,
                     dict(n_bodies=40, cols=18, rows=21, cell=1.25, y_scale=0.7, seed=12,
                          terrain_position=(0.5, -0.3, 0.25),
                          terrain_orientation=(0.0499792, 0.0, 0.0299875, 0.9983002)), 200, 50),
    # convex hulls (two scales) with boxes, spheres and capsules
    "hulls75": (scenes.hull_world, dict(nx=5, ny=3, nz=5, seed=9), 240, 60),
    # the testbed's joints scene: ball-and-socket chain, motorised slider
    # with limits, motorised hinge, fixed joints; slider speeds set every step
    "mechanisms4": (scenes.mechanism_world, dict(n_mechanisms=4, seed=31), 240, 60),
}
DT = np.float32(1.0 / 60.0)
# cases whose joints' motors are driven between steps: name -> f(world, step)
DRIVERS = {
    "mechanisms4": lambda world, step: [world.set_motor_speed(j, v)
                                        for j, v in scenes.mechanism_motor_speeds(4, step, DT)],
}


def digest(*arrays):
    h = hashlib.blake2b(digest_size=8)
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return np.frombuffer(h.digest(), dtype=np.uint64)[0]


def make_scene(name):
    f, kw, steps, every = WORLD_CASES[name]
    return f(**kw), steps, every


def trajectory(world, steps, every, driver=None):
    """Step `world` (engine.World or reflib.RefScene) and record the trace;
    driver(world, step) runs before each update."""
    rec = {k: [] for k in ("pair_n", "pair_h", "man_n", "pt_n", "man_h", "pt_h")}
    ckpt = {k: [] for k in ("pos", "ori", "lv", "av", "sleep")}
    for s in range(steps):
        if driver is not None:
            driver(world, s)
        world.update(float(DT))
        p = world.pairs()
        b1, b2, k, nd, l1, l2 = world.contacts()
        rec["pair_n"].append(len(p))
        rec["pair_h"].append(digest(p))
        rec["man_n"].append(len(b1))
        rec["pt_n"].append(len(nd))
        rec["man_h"].append(digest(b1, b2, k))
        rec["pt_h"].append(digest(nd, l1, l2))
        if (s + 1) % every == 0 or s + 1 == steps:
            for key, v in zip(ckpt, world.bodies()):
                ckpt[key].append(v)
    out = {k: np.array(v, dtype=np.uint64 if k.endswith("_h") else np.int64) for k, v in rec.items()}
    out.update({"ckpt_" + k: np.stack(v) for k, v in ckpt.items()})
    return out


def first_mismatch(got, exp):
    """(step, field) of the first per-step difference, or None."""
    for s in range(len(exp["pair_n"])):
        for k in ("pair_n", "pair_h", "man_n", "pt_n", "man_h", "pt_h"):
            if got[k][s] != exp[k][s]:
                return s, k
    return None
