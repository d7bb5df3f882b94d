"""The FP32 op table of the narrow-phase roofline (reactphysics3d_b200/roofline.py)
against the event list of the kernels (csrc/rp3dg_internal.h NpEvent) and
the C ABI (include/rp3dg.h)."""
import os
import re

import numpy as np

from reactphysics3d_b200 import roofline as RF

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _enum_names():
    text = open(os.path.join(ROOT, "reactphysics3d_b200", "csrc", "rp3dg_internal.h")).read()
    body = text[text.index("enum NpEvent"):]
    body = body[:body.index("};")]
    return [m.lower() for m in re.findall(r"^\s*EV_(\w+)", body, re.M)]


def test_events_follow_the_kernels_enum():
    assert _enum_names() == RF.EVENTS


def test_table_size_matches_the_c_abi():
    h = open(os.path.join(ROOT, "include", "rp3dg.h")).read()
    assert int(re.search(r"#define RP3DG_NP_EVENTS (\d+)", h).group(1)) == RF.NB_EVENTS
    assert len(RF.EVENTS) <= RF.NB_EVENTS


def test_every_event_has_a_positive_cost():
    for algo in range(1, 7):
        t = RF.op_table(algo)
        assert t.shape == (RF.NB_EVENTS,)
        used = t[:len(RF.EVENTS)]
        closed = [RF.EVENTS.index("closed_form"), RF.EVENTS.index("closed_form_contact")]
        for k, v in enumerate(used):
            if k in closed and algo > 3:
                assert v == 0
            else:
                assert v > 0, (algo, RF.EVENTS[k])
        assert np.all(t[len(RF.EVENTS):] == 0)


def test_ops_are_linear_in_the_events():
    rng = np.random.default_rng(0)
    a = rng.integers(0, 1000, RF.NB_EVENTS)
    b = rng.integers(0, 1000, RF.NB_EVENTS)
    for algo in (1, 4, 6):
        assert RF.fp32_ops(algo, a + b) == RF.fp32_ops(algo, a) + RF.fp32_ops(algo, b)


def test_primitive_costs():
    # Quaternion * Vector3: 3 x (3 mul + 2 add) + (3 mul + 2 add) + 3 x (4 mul + 3 add)
    assert RF.QV == 15 + 5 + 21
    assert RF.TV == RF.QV + 3
    # Transform * Transform: the rotated position (20 + 3 x 8) and the quaternion product (4 x 7)
    assert RF.TT == 20 + 24 + 28
