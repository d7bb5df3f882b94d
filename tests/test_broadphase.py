"""Broad phase, CPU side: the C restatement (fat-AABB update, overlapping
pairs) against the reference's own broad phase, through the committed
fixture and live."""
import numpy as np
import pytest

import bpio
import dynio
import reflib

GOLDEN = reflib.ROOT + "/tests/golden/np_dynamics.npz"


@pytest.fixture(scope="module")
def fixture():
    return np.load(GOLDEN)


def _check_capture(port, cap):
    u = bpio.update_case(cap)
    fmin, fmax, moved = bpio.oracle_update(port.lib, bpio.shapes(cap), u)
    assert np.array_equal(fmin.view(np.uint32), u["exp_min"].view(np.uint32))
    assert np.array_equal(fmax.view(np.uint32), u["exp_max"].view(np.uint32))
    assert np.array_equal(moved, u["exp_moved"])
    p = bpio.pairs_case(cap)
    got = bpio.oracle_pairs(port.lib, p["fat_min"], p["fat_max"], p["body"], None, p["category"], p["mask"])
    assert bpio.pair_set(got, len(got), p["index"]) == p["expected"]
    return moved.sum(), len(p["expected"])


def test_oracle_matches_reference_fixture(port, fixture):
    filtered = 0
    for n in dynio.cases(fixture):
        cap = dynio.capture(fixture, n)
        _check_capture(port, cap)
        filtered += int(np.any(cap["bp_bits"][:, 1] != 0xffff))
    assert filtered >= 1   # a case with category / mask filters


@pytest.mark.skipif(not reflib.have_ref("f32"), reason="reference build oracle/_ref not present")
@pytest.mark.parametrize("kind,seed,steps,variety", [(1, 31, 5, 3), (0, 32, 120, 2), (1, 33, 400, 3)])
def test_oracle_matches_reference_live(port, kind, seed, steps, variety):
    w = reflib.RefWorld(kind=kind, seed=seed, nx=6, ny=3, nz=6, variety=variety)
    w.step(n=steps)
    moved, pairs = _check_capture(port, w.capture())
    assert pairs > 0
