"""Far-from-origin precision (RBPS_PRECISION_FP32_POS64): a world's bodies
are stored in float relative to a per-world double origin (the centre of the
box around its initial body positions).

* A world of box towers 1e4 m from the origin in FP32_POS64 steps bit for
  bit like the same world translated by that origin to the global origin in
  plain FP32: the relative frame removes the offset exactly.
* The state read back is in absolute coordinates (get_state, get_state_all,
  step_io), set_state takes absolute coordinates, and contact points come
  back absolute too.
* Against the same towers at the origin, plain FP32 at 1e4 m (float spacing
  1 mm there) departs from them, FP32_POS64 not at all.
"""
import ctypes as C

import numpy as np
import pytest

from rbps_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def _towers(offset, n_worlds=4, height=16, seed=3, mass_ratio=1.0e-3):
    return scenes.config4(seed=seed, n_worlds=n_worlds, height=height, offset=offset, mass_ratio=mass_ratio)


def _translated(sc):
    """The scene with every world moved so its relative-frame origin (centre
    of the box around its body positions) sits at the global origin."""
    worlds, origins = [], []
    for w in sc.worlds:
        p = w.bodies["position"]
        o = 0.5 * (p.min(0) + p.max(0))
        b = w.bodies.copy()
        b["position"] = p - o
        worlds.append(scenes.WorldSpec(b, w.forces, w.colliders, w.joints, w.hulls))
        origins.append(o)
    return scenes.Scene(sc.name, sc.timestep, sc.substeps, sc.steps, worlds), origins


def test_relative_frame_equals_translated_world(rbps):
    sc = _towers(1.0e4)
    tr, origins = _translated(sc)
    far = rbps.Batch.from_scene(sc, abi.PRECISION_FP32_POS64, abi.SOLVE_COLORED)
    near = rbps.Batch.from_scene(tr, abi.PRECISION_FP32, abi.SOLVE_COLORED)
    for _ in range(3):
        far.step(20)
        near.step(20)
        for w in range(len(sc.worlds)):
            a, b = far.state(w), near.state(w)
            np.testing.assert_array_equal(a["orientation"], b["orientation"])
            np.testing.assert_array_equal(a["linear_velocity"], b["linear_velocity"])
            np.testing.assert_array_equal(a["position"], b["position"] + origins[w])


def test_absolute_io(rbps):
    sc = _towers(1.0e4, n_worlds=2, height=4)
    b = rbps.Batch.from_scene(sc, abi.PRECISION_FP32_POS64, abi.SOLVE_COLORED)
    b.set_dump(True)
    x0 = np.concatenate([w.bodies["position"] for w in sc.worlds])
    got = b.state_all()["position"]
    np.testing.assert_allclose(got, x0, rtol=0, atol=1e-5)
    st = b.state(1)
    st["position"] = st["position"] + np.array([0.0, 0.25, 0.0])
    b.set_state(1, st)
    np.testing.assert_allclose(b.state(1)["position"], st["position"], rtol=0, atol=1e-5)
    b.step(1)
    c = b.contacts(1)
    assert len(c) and np.abs(c["point_on_a"][:, 0] - sc.worlds[1].bodies["position"][0, 0]).max() < 2.0
    n, _ = b.total_bodies()
    f = np.ascontiguousarray(np.concatenate([w.forces for w in sc.worlds]))
    pos, rot = np.zeros((n, 3)), np.zeros((n, 4))
    b.step_io(f.ctypes.data, pos.ctypes.data, rot.ctypes.data)
    b.synchronize()
    np.testing.assert_allclose(pos, b.state_all()["position"], rtol=0, atol=0)


def test_frame_error(rbps):
    """Towers 1e4 m out against the same towers translated to the origin,
    20 steps, each precision mode: FP32_POS64 shows no difference at all,
    plain FP32 (float spacing 1 mm at 1e4 m) a clear one.  FP64 differs too
    (1.6 cm measured), but not through position round-off: the reference's
    SAP keys are floats, so at 1e4 m the pair order -- and with it the order
    of the sequential contact solve -- is not the one at the origin."""
    sc = _towers(1.0e4, n_worlds=8, height=16, mass_ratio=1.0)
    tr, origins = _translated(sc)
    shift = np.concatenate([np.repeat(o[None], len(w.bodies), 0) for o, w in zip(origins, sc.worlds)])
    dev = {}
    for name, prec, mode in (("fp64", abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER),
                             ("fp32", abi.PRECISION_FP32, abi.SOLVE_COLORED),
                             ("pos64", abi.PRECISION_FP32_POS64, abi.SOLVE_COLORED)):
        far = rbps.Batch.from_scene(sc, prec, mode)
        near = rbps.Batch.from_scene(tr, abi.PRECISION_FP32 if prec == abi.PRECISION_FP32_POS64 else prec, mode)
        far.step(20)
        near.step(20)
        dev[name] = float(np.abs(far.state_all()["position"] - (near.state_all()["position"] + shift)).max())
    assert dev["pos64"] == 0.0, dev
    assert dev["fp32"] > 1e-4, dev
    assert np.isfinite(dev["fp64"]), dev
