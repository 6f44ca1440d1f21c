"""FP32 against FP64 on the batched workload's own scene (config 3: uneven
box/sphere worlds, each with a 13-link revolute chain, dt 1/120, 4
substeps), through the C ABI.

- The premise of every comparison: the FP64 reference-order engine equals
  the reference (compiled from its own sources) bit for bit on worlds of
  the bench's scene, every step.
- Cold start without initial overlap: one FP32 step (reference order and
  colored) within 1e-5 relative of FP64 in every world.
- Settled (the state the bench times): the reference's own revolute chains
  have broken by then (they fold up when they hit the ground, in the
  reference itself), and the piles are in contact everywhere, so one step
  amplifies any change of the state.  The gate is therefore relative to
  the problem's conditioning: the FP32 reference-order error, over the
  bodies outside each world's jointed component, stays within a small
  factor of the error FP64 itself makes from the same state moved by one
  float32 ulp per coordinate (the largest of three draws of the signs), and
  nearly every body is within 1e-5 (about as many as in those moved FP64
  runs).
- Colored FP32 over 60 steps from the settled state: energy and momentum
  change, deepest contact and joint attachment gaps stay close to FP64
  reference order's.
"""
import numpy as np
import pytest

from rbps_b200 import abi, metrics as M, scenes

pytestmark = pytest.mark.gpu

_CACHE = {}


def _bench_scene(n):
    if "sc" not in _CACHE:
        _CACHE["sc"] = scenes.config3(seed=0, n_worlds=4096)
    sc = _CACHE["sc"]
    return scenes.Scene(sc.name, sc.timestep, sc.substeps, sc.steps, sc.worlds[:n])


def _run(rbps, sc, prec, solve, steps=1, dump=False):
    b = rbps.Batch.from_scene(sc, prec, solve)
    b.set_state_check(False)
    if dump and steps > 1:
        b.step(steps - 1)
    if dump:
        b.set_dump(True)
    b.step(1 if dump else steps)
    st = [b.state(w) for w in range(len(sc.worlds))]
    con = [b.contacts(w) for w in range(len(sc.worlds))] if dump else None
    b.close()
    return st, con


def _settled(rbps, n):
    key = ("settled", n)
    if key not in _CACHE:
        sub = _bench_scene(n)
        st, _ = _run(rbps, sub, abi.PRECISION_FP32, abi.SOLVE_COLORED, steps=245)
        _CACHE[key] = (sub, st)
    return _CACHE[key]


def test_fp64_matches_reference_on_bench_worlds(rbps, ref):
    """32 worlds of the bench's own scene, FP64 reference order against the
    live reference engine: bit for bit, 5 steps."""
    sub = _bench_scene(32)
    b = rbps.Batch.from_scene(sub, abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER)
    refs = [ref.RefWorld(w, sub.timestep, sub.substeps) for w in sub.worlds]
    for step in range(5):
        b.step(1)
        for w, rw in enumerate(refs):
            rw.step(1)
            rs, st = rw.state(), b.state(w)
            for k in ("position", "orientation", "linear_velocity", "angular_velocity"):
                np.testing.assert_array_equal(st[k], rs[k], err_msg=f"step {step + 1} world {w} {k}")
    b.close()


def test_fp32_cold_start_without_overlap_within_1e5(rbps):
    sc = scenes.config3_separated(seed=0, n_worlds=48)
    base, _ = _run(rbps, sc, abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER)
    for solve in (abi.SOLVE_REFERENCE_ORDER, abi.SOLVE_COLORED):
        st, _ = _run(rbps, sc, abi.PRECISION_FP32, solve)
        e = [float(M.state_error(a, r).max()) for a, r in zip(st, base)]
        assert max(e) <= 1e-5, (solve, max(e))


def test_fp32_settled_error_within_float_conditioning(rbps):
    sub, st0 = _settled(rbps, 64)
    settled = scenes.with_state(sub, st0)
    base, c64 = _run(rbps, settled, abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER, dump=True)
    f32, _ = _run(rbps, settled, abi.PRECISION_FP32, abi.SOLVE_REFERENCE_ORDER)
    # FP64 from the state moved by one float ulp per coordinate, three draws
    # of the signs: the conditioning baseline is the largest of the three
    ulps = []
    for seed in range(3):
        pert = scenes.with_state(settled, [M.perturb_ulp(s, seed=seed) for s in st0])
        ulps.append(_run(rbps, pert, abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER)[0])
    e32, eulp, within, within_ulp, total = [], [], 0, 0, 0
    for w in range(len(sub.worlds)):
        if not np.isfinite(base[w]["position"]).all():
            continue
        keep = np.ones(len(st0[w]["position"]), bool)
        keep[M.jointed_component(settled.worlds[w], c64[w])] = False
        a = M.state_error(f32[w], base[w])[keep]
        u = np.max([M.state_error(ulp[w], base[w])[keep] for ulp in ulps], axis=0)
        if len(a):
            e32.append(a.max())
            eulp.append(u.max())
            within += int((a <= 1e-5).sum())
            within_ulp += int((u <= 1e-5).sum())
            total += len(a)
    e32, eulp = np.array(e32), np.array(eulp)
    assert len(e32) >= 60
    assert np.median(e32) <= 3.0 * np.median(eulp), (np.median(e32), np.median(eulp))
    assert np.percentile(e32, 90) <= 5.0 * np.percentile(eulp, 90), (np.percentile(e32, 90),
                                                                      np.percentile(eulp, 90))
    # nearly every body within 1e-5, about as many as FP64 from the moved state
    assert within / total >= 0.95, within / total
    assert within / total >= within_ulp / total - 0.03, (within / total, within_ulp / total)


def test_colored_drift_tracks_fp64(rbps):
    sub, st0 = _settled(rbps, 64)
    settled = scenes.with_state(sub, st0)
    n = len(sub.worlds)
    e0 = sum(M.world_energy(settled.worlds[w], st0[w]) for w in range(n))
    p0 = sum(M.world_momentum(settled.worlds[w], st0[w]) for w in range(n))
    mass = sum(float(w.bodies["mass"][w.bodies["type"] == abi.BODY_DYNAMIC].sum()) for w in settled.worlds)
    steps = 60
    res = {}
    for name, prec, solve in (("fp64", abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER),
                              ("fp32_colored", abi.PRECISION_FP32, abi.SOLVE_COLORED)):
        st, con = _run(rbps, settled, prec, solve, steps=steps, dump=True)
        assert all(np.isfinite(s["position"]).all() for s in st), name
        e = sum(M.world_energy(settled.worlds[w], st[w]) for w in range(n))
        p = sum(M.world_momentum(settled.worlds[w], st[w]) for w in range(n))
        gaps = np.concatenate([M.joint_gaps(settled.worlds[w], st[w]) for w in range(n)])
        depth = max(float(c["penetration_depth"].max()) for c in con if len(c))
        res[name] = ((e - e0) / abs(e0), float(np.linalg.norm(p - p0)) / (mass * 9.81 * steps * sub.timestep),
                     float(np.median(gaps)), depth)
    (e64, m64, g64, d64), (e32, m32, g32, d32) = res["fp64"], res["fp32_colored"]
    assert abs(e32 - e64) <= 0.05, res
    assert abs(m32 - m64) <= 0.25 * max(m64, 0.02), res
    assert abs(g32 - g64) <= 0.35 * g64 + 0.01, res
    assert d32 <= d64 + 0.05, res
