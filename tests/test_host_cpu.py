"""Host-side logic, without a GPU: seeded scene generation, the bench's
multi-rank aggregation on two gloo ranks, the byte model, and the
reference arm of bench.py end to end on a small world count."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from rbps_b200 import abi, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

from helpers import load_golden  # noqa: E402


def _same_spec(a, b):
    for f in ("bodies", "colliders", "joints"):
        x, y = getattr(a, f), getattr(b, f)
        assert x.dtype == y.dtype and len(x) == len(y)
        for name in x.dtype.names:
            np.testing.assert_array_equal(x[name], y[name], err_msg=f"{f}.{name}")
    np.testing.assert_array_equal(a.forces, b.forces)


def test_config3_is_deterministic_and_shaped():
    a = scenes.config3(seed=5, n_worlds=64)
    b = scenes.config3(seed=5, n_worlds=64)
    c = scenes.config3(seed=6, n_worlds=64)
    assert (a.timestep, a.substeps) == (1.0 / 120.0, 4)
    for wa, wb in zip(a.worlds, b.worlds):
        _same_spec(wa, wb)
    assert any(len(wa.bodies) != len(wc.bodies) for wa, wc in zip(a.worlds, c.worlds))
    for w in a.worlds:
        n_chain = int((w.colliders["shape"] == abi.SHAPE_CAPSULE).sum())
        n_free = len(w.bodies) - 1 - n_chain  # minus the static ground body
        assert 8 <= n_free <= 512
        assert n_chain == 13 and len(w.joints) == 12
        assert (w.joints["type"] == abi.JOINT_REVOLUTE).all()
        assert int((w.colliders["shape"] == abi.SHAPE_PLANE).sum()) == 1


def test_config3_body_counts_are_log_uniform():
    sc = scenes.config3(seed=0, n_worlds=1024)
    n = np.array([len(w.bodies) - 14 for w in sc.worlds], np.float64)
    assert n.min() >= 8 and n.max() <= 512
    # log-uniform on [8, 512]: log2(n) roughly uniform on [3, 9], mean near 6
    assert abs(np.log2(n).mean() - 6.0) < 0.15


def test_config0_composition():
    sc = scenes.config0(seed=0)
    w = sc.worlds[0]
    shapes = w.colliders["shape"]
    assert int((shapes == abi.SHAPE_BOX).sum()) == 256
    assert int((shapes == abi.SHAPE_SPHERE).sum()) == 256
    assert int((shapes == abi.SHAPE_PLANE).sum()) == 1
    assert (sc.timestep, sc.substeps) == (1.0 / 60.0, 10)
    dyn = w.bodies["type"] == abi.BODY_DYNAMIC
    assert np.allclose(w.forces[dyn][:, 1], -9.81 * w.bodies["mass"][dyn])


@pytest.mark.parametrize("name,factory", [
    ("boxsphere64_seed1", lambda: scenes.small_world(seed=1, n=64)),
    ("capsules32_seed2", lambda: scenes.capsule_world(seed=2, n=32)),
    ("chain13_seed3", lambda: scenes.chain_world(seed=3, n_bodies=12)),
])
def test_scene_factories_reproduce_fixture_inputs(name, factory):
    _, g = load_golden(name)
    spec = factory()
    for f in ("bodies", "colliders", "joints"):
        x, y = getattr(spec, f), g[f]
        assert len(x) == len(y)
        for fld in x.dtype.names:
            np.testing.assert_array_equal(x[fld], y[fld], err_msg=f"{f}.{fld}")


def test_bytes_model():
    # per step: substeps * (336 N + 704 C + 88 P_cand + 1116 J) + 208 N_coll + 56 P
    assert bench.bytes_model(10, 4, 3, 5, 7, 2, 11) == 4 * (3360 + 2112 + 440 + 2232) + 2288 + 392


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        t = bench.reduce_over_ranks(10.0 + rank, "max", ws)     # per-rank device time
        n = bench.reduce_over_ranks(100 * (rank + 1), "sum", ws)  # per-rank dynamic bodies
        seed = bench.rank_seed(7, rank)
        # the batched workload: one set of worlds, split as bench.py splits it
        from rbps_b200 import shard
        full = scenes.config3(seed=3, n_worlds=48 * ws)
        mine, idx = shard.shard_scene(full, ws, rank)
        bodies = sum(w.n_bodies for w in mine.worlds)
        total = bench.reduce_over_ranks(bodies, "sum", ws)
        hi = bench.reduce_over_ranks(bodies, "max", ws)
        lo = -bench.reduce_over_ranks(-bodies, "max", ws)
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump({"t": t, "n": n, "seed": seed, "idx": idx.tolist(), "total": total, "hi": hi, "lo": lo,
                       "full_total": full.n_bodies, "max_world": max(w.n_bodies for w in full.worlds)}, f)
    finally:
        dist.destroy_process_group()


def test_multirank_aggregation_gloo(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    r = [json.load(open(tmp_path / f"r{k}.json")) for k in range(2)]
    assert r[0]["t"] == r[1]["t"] == 11.0        # time: max over ranks
    assert r[0]["n"] == r[1]["n"] == 300.0       # work: sum over ranks
    assert r[0]["seed"] != r[1]["seed"]          # single-world replicas draw their own worlds
    # the batched worlds: one set, split exactly once, balanced by bodies
    idx = sorted(r[0]["idx"] + r[1]["idx"])
    assert idx == list(range(96))
    assert r[0]["total"] == r[0]["full_total"]
    assert r[0]["hi"] - r[0]["lo"] <= r[0]["max_world"]


def test_partition_balance_and_order():
    from rbps_b200 import shard
    rng = np.random.default_rng(0)
    counts = np.floor(np.exp(rng.uniform(np.log(8), np.log(513), 4096))).astype(int) + 14
    for n in (1, 2, 3, 8):
        parts = shard.partition_worlds(counts, n)
        assert len(parts) == n
        allidx = np.sort(np.concatenate(parts))
        np.testing.assert_array_equal(allidx, np.arange(len(counts)))
        loads = [int(counts[p].sum()) for p in parts]
        assert max(loads) - min(loads) <= counts.max()
        for p in parts:
            assert (np.diff(p) > 0).all()  # worlds keep their order within a rank
    np.testing.assert_array_equal(shard.partition_worlds(counts, 1)[0], np.arange(len(counts)))


def test_reduce_single_rank_is_identity():
    assert bench.reduce_over_ranks(3.5, "max", 1) == 3.5
    assert bench.reduce_over_ranks(3.5, "sum", 1) == 3.5


def test_reference_arm_json_line(ref):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--worlds", "32",
                          "--steps", "3", "--warmup", "3"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT, env={**os.environ, "RBPS_BENCH_REF_SECONDS": "4"})
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling", "dtype",
                "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["config"]["workload"] == bench.WORKLOAD
