#!/usr/bin/env python
"""Batched-world step throughput on B200: body-substeps/s.

Workload: 4,096 independent worlds, bodies per world log-uniform in [8,512]
(random boxes and spheres, sizes U[0.2,0.5] m) plus one 13-link revolute
capsule chain per world, over a ground plane; dt = 1/120 s, 4 substeps, FP32
state, graph-coloured Gauss-Seidel; all worlds step in one launch per step.
Seeded synthetic scene (rbps_b200.scenes.config3); under torchrun the N
ranks split one set of 4,096 x N worlds by balanced body count
(rbps_b200.shard: weak scaling, no collective on the step path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl rbps|reference]

Prints one JSON line (rank 0).  `value` = whole-job body-substeps/s from CUDA
events on the step stream (max over ranks); `e2e` = the same metric through
rbps_batch_step_io_async with page-locked host buffers, over the same steps
(the batch is rewound to a device snapshot taken after the warm-up): every
step copies its forces in and its poses out, on copy streams that overlap
the neighbouring steps' compute, and the timed region ends after the last
step's poses are on the host; `roofline` = the step kernel against the
measured HBM copy bandwidth with the algorithmic byte model below;
`cpu_baseline` = the reference engine (oracle/_ref, built from the
reference's own sources) on a bounded sample of the same worlds, all host
threads; `plain_gpu` = the plain per-world GPU path (one batch per world,
same colored solver) on a sample of the same worlds from the same state.
`--impl reference` times the reference CPU engine alone.

`--workload collision_stress` runs the single 65,536-body world of spheres,
boxes, capsules and convex hulls instead (scenes.config1), `--workload
joint_heavy` the single world of 1,024 hanging 32-capsule chains on ball
joints (scenes.config2); their lines add SAP pairs/s and GJK pairs/s.
`--workload precision_stress` steps 256 box towers 1e4 m from the origin
(scenes.config4) in FP32, FP32_POS64 and FP64 and reports drift, penetration
and energy change per mode.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "body-substeps/s (batched FP32, 4096 uneven worlds + 13-link revolute chain each, 1 B200)"
UNIT = "body-substeps/s"
WORKLOAD = "config3_batched_uneven_worlds"


def bytes_model(n_dyn, substeps, contacts, candidates, pairs, joints, colliders):
    """Algorithmic bytes of one step (FP32 SoA, every compulsory element once
    per phase that touches it):
      per dynamic body per substep     336 B  (integrate 128R+104W, velocity update 56R+48W)
      per contact point per substep    704 B  (position solve, velocity solve, narrowphase emit)
      per narrowphase candidate / sub   88 B
      per revolute joint per substep  1116 B  (4 rows, errors, damping)
      per collider per frame           208 B  (AABB / fat update, endpoint sort, sweep)
      per SAP pair per frame            56 B
    """
    per_sub = n_dyn * 336 + contacts * 704 + candidates * 88 + joints * 1116
    return substeps * per_sub + colliders * 208 + pairs * 56


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def reduce_over_ranks(x, op, ws):
    """x (a float) reduced over the process group: op "max" or "sum"; the
    identity at one rank.  NCCL reduces a CUDA tensor, gloo a CPU one."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def rank_seed(seed, rank):
    """Single-world workloads do not shard: each rank steps its own replica
    (same distribution, independent draw)."""
    return seed + rank


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id=None):
        self.bus_id = bus_id  # PCI bus number (int) of the timed device, None = all rows
        self.proc = None
        self.out = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(prefix="rbps_clocks_", suffix=".csv")
            self.out = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.out.close()
        path = self.path
        rows = []
        with open(path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 10:
                    continue
                if self.bus_id is not None:
                    try:
                        if int(parts[1].split(":")[1], 16) != int(self.bus_id):
                            continue
                    except (IndexError, ValueError):
                        pass
                rows.append(parts)
        os.remove(path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[6 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_reference_run(scene, preroll, warmup, steps, max_seconds, threads):
    """The reference engine (oracle/_ref, built from the reference's own
    sources) on the host cores, one World per thread at a time, on a prefix
    of the scene's worlds sized to about max_seconds: `preroll` + `warmup`
    untimed steps, then timed chunks of steps until at least `steps` steps
    and half of max_seconds have passed.  Returns (body-substeps/s,
    description of the sample)."""
    from oracle import ref
    worlds = scene.worlds
    # calibrate on a small prefix (falling bodies); resting piles cost ~3x more
    probe = [ref.RefWorld(w, scene.timestep, scene.substeps) for w in worlds[:256]]
    t = ref.step_worlds(probe, 2, threads)
    dyn_probe = sum(w.n_dynamic for w in worlds[:256])
    rate = dyn_probe * scene.substeps * 2 / max(t, 1e-9)
    per_dyn = scene.substeps * (2.0 * preroll + 3.0 * (warmup + 2 * steps)) / rate  # seconds per dynamic body
    total_dyn, n = 0, 0
    for w in worlds:
        if n >= 64 and (total_dyn + w.n_dynamic) * per_dyn > max_seconds:
            break
        total_dyn += w.n_dynamic
        n += 1
    del probe
    sample = worlds[:n]
    refs = [ref.RefWorld(w, scene.timestep, scene.substeps) for w in sample]
    t_pre = ref.step_worlds(refs, preroll + warmup, threads) if preroll + warmup else 0.0
    secs, done = 0.0, 0
    chunk = max(1, min(steps, 10))
    while done < steps or (secs < 0.5 * max_seconds and done < 20 * steps):
        secs += ref.step_worlds(refs, chunk, threads)
        done += chunk
    n_dyn = sum(w.n_dynamic for w in sample)
    value = n_dyn * scene.substeps * done / secs
    info = (f"{n} of {len(worlds)} worlds ({n_dyn} dynamic bodies), {preroll} pre-roll + {warmup} untimed steps "
            f"({t_pre:.1f} s), then {done} timed steps in {secs:.2f} s on {threads} threads")
    return value, info


def plain_gpu_run(scene, batch, n_sample, steps, warmup, stream):
    """The plain per-world GPU path on the same worlds: each world its own
    batch with the same FP32 colored solver (one world per launch sequence,
    no batching across worlds), the sample worlds stepped one after another
    on the same stream.  Each plain world starts from the batched run's
    current state, so both paths time the same regime.  Returns
    (body-substeps/s, description)."""
    import torch
    import rbps_b200
    from rbps_b200 import abi
    idx = list(range(min(n_sample, len(scene.worlds))))
    plain = []
    for w in idx:
        sub = type(scene)(scene.name, scene.timestep, scene.substeps, scene.steps, [scene.worlds[w]])
        b = rbps_b200.Batch.from_scene(sub, abi.PRECISION_FP32, abi.SOLVE_COLORED, stream=stream.cuda_stream)
        b.set_state(0, batch.state(w))
        plain.append(b)
    for b in plain:
        b.step(warmup)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        for b in plain:
            b.step(1)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    n_dyn = sum(scene.worlds[w].n_dynamic for w in idx)
    for b in plain:
        b.close()
    value = n_dyn * scene.substeps * steps / (ms / 1e3)
    return value, (f"{len(idx)} of {len(scene.worlds)} worlds ({n_dyn} dynamic bodies), one batch per world, "
                   f"FP32 colored, {warmup} untimed + {steps} timed steps from the batched state")


ERROR_MODES = (("fp64", "PRECISION_FP64", "SOLVE_REFERENCE_ORDER"),
               ("fp32_reference_order", "PRECISION_FP32", "SOLVE_REFERENCE_ORDER"),
               ("fp32_colored", "PRECISION_FP32", "SOLVE_COLORED"))


def _run_modes(scene, stream, steps=1, dump=False, modes=ERROR_MODES):
    """Each mode's batch of `scene`, stepped `steps` times: {name: (states,
    contacts of the last substep or None)}.  The failure check is off:
    worlds where the reference itself goes non-finite are counted below."""
    import rbps_b200
    from rbps_b200 import abi
    out = {}
    for name, prec, solve in modes:
        b = rbps_b200.Batch.from_scene(scene, getattr(abi, prec), getattr(abi, solve), stream=stream.cuda_stream)
        b.set_state_check(False)
        if dump and steps > 1:
            b.step(steps - 1)
        if dump:
            b.set_dump(True)
        b.step(1 if dump else steps)
        st = [b.state(w) for w in range(len(scene.worlds))]
        con = [b.contacts(w) for w in range(len(scene.worlds))] if dump else None
        b.close()
        out[name] = (st, con)
    return out


def _one_step(scene, runs, base, against, ok, comp=None):
    """Per-world one-step errors of each run against `base`, as summaries
    (max over a world's bodies; with comp, also over the bodies outside
    each world's jointed component) plus the fraction of bodies within
    1e-5."""
    from rbps_b200 import metrics as M
    out = {}
    for name, st in runs.items():
        e_all, e_out, b_in, b_n = [], [], 0, 0
        for w in range(len(scene.worlds)):
            if not ok[w]:
                continue
            e = M.state_error(st[w], base[w])
            e_all.append(float(e.max()))
            b_in += int((e <= 1e-5).sum())
            b_n += len(e)
            if comp is not None:
                m = np.ones(len(e), bool)
                m[comp[w]] = False
                e_out.append(float(e[m].max()) if m.any() else 0.0)
        r = {"max_over_world": M.summary(e_all), "bodies_within_1e-5": b_in / max(b_n, 1)}
        if comp is not None:
            r["max_over_world_outside_jointed_component"] = M.summary(e_out)
        out[name] = r
    out["against"] = against
    return out


def error_vs_fp64(scene, n_worlds, settled_states, stream, drift_steps=60):
    """Errors of the FP32 modes against the FP64 reference-order engine
    (the device engine that equals the reference bit for bit), on the first
    n_worlds worlds:
      cold_start   one step from the scene's initial state;
      settled      one step from `settled_states` (the first timed step's
                   state), over all bodies and over the bodies outside
                   each world's jointed component (the revolute chain and
                   whatever touches it); beside them the FP64 engine
                   started from the same state moved by one float32 ulp per
                   coordinate, which measures how strongly one step
                   amplifies the smallest change a float state can carry;
      drift        `drift_steps` steps from the settled state per mode:
                   relative change of total energy, change of total linear
                   momentum over the gravity impulse M g T, deepest contact
                   and joint attachment gaps at the end.
    Worlds where the reference itself goes non-finite are counted, not
    compared."""
    from rbps_b200 import metrics as M, scenes
    sub = type(scene)(scene.name, scene.timestep, scene.substeps, scene.steps, scene.worlds[:n_worlds])
    out = {"worlds": n_worlds,
           "against": "FP64 reference order (bit-identical to the reference engine)"}
    # cold start
    runs = _run_modes(sub, stream)
    base = runs["fp64"][0]
    ok = [bool(np.isfinite(s["position"]).all() and np.isfinite(s["orientation"]).all()) for s in base]
    out["fp64_nonfinite_worlds"] = int(len(ok) - sum(ok))
    out["cold_start"] = _one_step(sub, {k: runs[k][0] for k in ("fp32_colored", "fp32_reference_order")}, base,
                                  "state after step 1 from the initial state", ok)
    # settled: the timed state
    settled = scenes.with_state(sub, settled_states[:n_worlds])
    runs = _run_modes(settled, stream, dump=True)
    base, c64 = runs["fp64"]
    ok = [bool(np.isfinite(s["position"]).all() and np.isfinite(s["orientation"]).all()) for s in base]
    comp = [M.jointed_component(settled.worlds[w], c64[w]) for w in range(n_worlds)]
    pert = scenes.with_state(settled, [M.perturb_ulp(s) for s in settled_states[:n_worlds]])
    ulp = _run_modes(pert, stream, modes=ERROR_MODES[:1])["fp64"][0]
    gaps0 = [M.joint_gaps(settled.worlds[w], settled_states[w]) for w in range(n_worlds)]
    out["settled"] = _one_step(settled, {"fp32_colored": runs["fp32_colored"][0],
                                         "fp32_reference_order": runs["fp32_reference_order"][0],
                                         "fp64_one_ulp_perturbed_start": ulp},
                               base, "state after one step from the first timed step's state", ok, comp)
    out["settled"]["chains_broken_worlds"] = int(sum(len(g) and g.max() > 0.1 for g in gaps0))
    out["settled"]["jointed_component_bodies_median"] = float(np.median([len(c) for c in comp]))
    # drift from the settled state
    e0 = sum(M.world_energy(settled.worlds[w], settled_states[w]) for w in range(n_worlds))
    p0 = sum(M.world_momentum(settled.worlds[w], settled_states[w]) for w in range(n_worlds))
    mass = sum(float(w.bodies["mass"][w.bodies["type"] == 1].sum()) for w in settled.worlds)
    impulse = mass * 9.81 * drift_steps * scene.timestep
    drift = {"steps": drift_steps}
    for name, (st, con) in _run_modes(settled, stream, steps=drift_steps, dump=True).items():
        fin = [bool(np.isfinite(s["position"]).all()) for s in st]
        ws = [w for w in range(n_worlds) if fin[w]]
        e = sum(M.world_energy(settled.worlds[w], st[w]) for w in ws)
        p = sum(M.world_momentum(settled.worlds[w], st[w]) for w in ws)
        gaps = np.concatenate([M.joint_gaps(settled.worlds[w], st[w]) for w in ws])
        depth = max((float(con[w]["penetration_depth"].max()) for w in ws if len(con[w])), default=0.0)
        drift[name] = {"energy_rel": (e - e0) / abs(e0), "momentum_over_gravity_impulse": float(np.linalg.norm(p - p0) / impulse),
                       "max_penetration_m": depth, "joint_gap_median_m": float(np.median(gaps)) if len(gaps) else 0.0,
                       "joint_gap_max_m": float(gaps.max()) if len(gaps) else 0.0, "nonfinite_worlds": len(fin) - len(ws)}
    out["drift_from_settled"] = drift
    return out


SINGLE_WORLD = {
    "collision_stress": ("config1_collision_stress",
                         "body-substeps/s (collision stress: 65,536 mixed bodies incl. convex hulls, one world)"),
    "joint_heavy": ("config2_joint_heavy",
                    "body-substeps/s (joint-heavy: 1,024 chains x 32 capsules on ball joints with 60 deg cones, "
                    "one world)"),
}


def single_world(args, ws, rank, local):
    """One large world, FP32 colored, on the whole cooperative grid:
      collision_stress  65,536 spheres, boxes, capsules and convex hulls
                        over 200^3 m (scenes.config1), 10 substeps
      joint_heavy       1,024 hanging chains of 32 capsules on ball joints
                        with 60 degree cones (scenes.config2), 8 substeps
    K timed steps.  Reports body-substeps/s, SAP pairs/s and GJK pairs/s."""
    import torch
    import rbps_b200
    from rbps_b200 import abi, scenes
    torch.cuda.set_device(local)
    workload, metric = SINGLE_WORLD[args.workload]
    if args.workload == "collision_stress":
        scene = scenes.config1(seed=rank_seed(args.seed, rank))
    else:
        scene = scenes.config2(seed=rank_seed(args.seed, rank))
        # Once neighbouring chains tangle (1 m apart), their capsule contacts
        # pump energy into the chains -- the oracle shows the same (mean
        # speed 13 m/s and 1.6M SAP pairs by step 90 on 64 chains) -- so the
        # timed window is the first 30 steps after the warm-up.
        args.steps = min(args.steps, 30)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    # the chains swing into their neighbours (1 m apart) and tangle: their
    # SAP pairs grow past the default 8 per object within ~20 steps
    pair_cap = 1 << 21 if args.workload == "joint_heavy" else 0
    batch = rbps_b200.Batch.from_scene(scene, abi.PRECISION_FP32, abi.SOLVE_COLORED, device=local,
                                       stream=stream.cuda_stream, max_pairs_per_world=pair_cap,
                                       block_threads=args.block)
    batch.step(args.warmup)
    batch.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pairs = gjk = 0
    ms = 0.0
    for _ in range(args.steps):  # one step at a time: the per-step counters are read between steps
        ev0.record(stream)
        batch.step(1)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms += ev0.elapsed_time(ev1)
        st = batch.stats()
        pairs += st["pairs"]
        gjk += st["gjk_pairs"]
    batch.synchronize()
    n_tot, n_dyn = batch.total_bodies()
    ms = reduce_over_ranks(ms, "max", ws)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            from oracle import ref
            t0 = time.time()
            rw = ref.RefWorld(scene.worlds[0], scene.timestep, scene.substeps)
            t_build = time.time() - t0
            ref.step_worlds([rw], 1, 1)  # warm-up step
            secs, done = 0.0, 0
            while done < 2 or secs < 0.5 * args.cpu_seconds:
                secs += ref.step_worlds([rw], 1, 1)
                done += 1
            cpu = {"value": n_dyn * scene.substeps * done / secs, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"the same world in oracle/_ref (one World, one thread), built in {t_build:.1f} s, "
                             f"1 untimed + {done} timed steps from the initial state in {secs:.2f} s"}
        except Exception as e:  # the oracle library is missing
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"unavailable: {e}"}
    n_dyn_all = reduce_over_ranks(n_dyn, "sum", ws)
    pairs_all = reduce_over_ranks(pairs, "sum", ws)
    gjk_all = reduce_over_ranks(gjk, "sum", ws)
    if rank == 0:
        sec = ms / 1e3
        line = {"metric": metric,
                "value": n_dyn_all * scene.substeps * args.steps / sec, "unit": UNIT, "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": workload, "bodies": n_tot, "joints": len(scene.worlds[0].joints),
                           "substeps": scene.substeps,
                           "dt": scene.timestep, "seed": args.seed, "team": "cooperative grid, one launch per phase",
                           "timing": "each step bracketed by CUDA events; counters read between steps"},
                "cpu_baseline": cpu,
                "sap_pairs_per_s": pairs_all / sec, "gjk_pairs_per_s": gjk_all / sec,
                "sap_pairs_per_step": pairs_all / args.steps / ws, "gjk_pairs_per_step": gjk_all / args.steps / ws,
                "gpu_launches": int(batch.stats()["kernel_launches"]) * args.steps}
        print(json.dumps(line), flush=True)
    batch.close()


def tower_energy(scene, st, g=9.81):
    """Kinetic + potential energy of every dynamic body, summed (the ground
    plane of each world at its static body's height)."""
    e = 0.0
    off = 0
    for w in scene.worlds:
        n = len(w.bodies)
        dyn = w.bodies["type"] == 1  # RBPS_BODY_DYNAMIC
        x = st["position"][off:off + n]
        v = st["linear_velocity"][off:off + n]
        om = st["angular_velocity"][off:off + n]
        q = st["orientation"][off:off + n]
        m = w.bodies["mass"]
        I = w.bodies["inertia"][:, :3]
        # body-frame angular velocity: conj(q) * omega * q
        qw, qv = q[:, :1], -q[:, 1:]
        t = 2.0 * np.cross(qv, om)
        ob = om + qw * t + np.cross(qv, t)
        y0 = w.bodies["position"][~dyn][:, 1].min() if (~dyn).any() else 0.0
        ke = 0.5 * m * (v * v).sum(1) + 0.5 * (I * ob * ob).sum(1)
        pe = m * g * (x[:, 1] - y0)
        e += float((ke + pe)[dyn].sum())
        off += n
    return e


def precision_stress(args, ws, rank, local):
    """256 worlds, each a 64-box tower (half-extent 0.5 m, masses alternating
    1:1000) 1e4 m from the origin on its own ground plane, friction 0.8,
    20 substeps (scenes.config4).  Steps the same scene in FP32 (colored),
    FP32_POS64 (colored, positions relative to a per-world double origin)
    and FP64 (reference order: the device engine that matches the oracle
    bit for bit) and reports, per mode, throughput, the largest body
    displacement from the initial stack, the deepest contact in the last
    step and the relative change of total energy (the 1:1000 towers fall in
    every mode, the reference's FP64 solver included), and the frame error:
    the largest position difference after 200 steps between the towers
    where they are and the same towers moved to the origin, in the same
    mode (FP32_POS64 against FP32 at the origin).  FP32's float spacing at
    1e4 m is 1 mm, which also freezes small horizontal motions there.
    """
    import torch
    import rbps_b200
    from rbps_b200 import abi, scenes
    torch.cuda.set_device(local)
    steps = args.steps
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    def run(scene):
        x0 = np.concatenate([w.bodies["position"] for w in scene.worlds])
        st0 = {"position": x0, "orientation": np.concatenate([w.bodies["orientation"] for w in scene.worlds]),
               "linear_velocity": np.zeros_like(x0), "angular_velocity": np.zeros_like(x0)}
        e0 = tower_energy(scene, st0)
        modes = {}
        for name, prec, solve in (("fp32", abi.PRECISION_FP32, abi.SOLVE_COLORED),
                                  ("fp32_pos64", abi.PRECISION_FP32_POS64, abi.SOLVE_COLORED),
                                  ("fp64", abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER)):
            batch = rbps_b200.Batch.from_scene(scene, prec, solve, device=local, stream=stream.cuda_stream)
            n_tot, n_dyn = batch.total_bodies()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            ev0.record(stream)
            batch.step(steps - 1)
            ev1.record(stream)
            torch.cuda.synchronize()
            ms = ev0.elapsed_time(ev1)
            batch.set_dump(True)
            batch.step(1)
            st = batch.state_all(("position", "orientation", "linear_velocity", "angular_velocity"))
            depth = 0.0
            for w in range(0, len(scene.worlds), 16):
                c = batch.contacts(w)
                if len(c):
                    depth = max(depth, float(c["penetration_depth"].max()))
            finite = bool(np.isfinite(st["position"]).all())
            modes[name] = {"ms_per_step": ms / max(steps - 1, 1),
                           "body_substeps_per_s": n_dyn * scene.substeps * (steps - 1) / (ms / 1e3),
                           "max_displacement_m": float(np.abs(st["position"] - x0).max()) if finite else None,
                           "max_penetration_m": depth,
                           "energy_drift": (tower_energy(scene, st) - e0) / abs(e0) if finite else None,
                           "finite": finite}
            batch.close()
        return modes

    scene = scenes.config4(seed=rank_seed(args.seed, rank))
    modes = run(scene)

    # frame error: the same towers moved to the origin, 200 steps each way
    near_worlds, shift = [], []
    for w in scene.worlds:
        p = w.bodies["position"]
        o = 0.5 * (p.min(0) + p.max(0))
        b = w.bodies.copy()
        b["position"] = p - o
        near_worlds.append(scenes.WorldSpec(b, w.forces, w.colliders, w.joints, w.hulls))
        shift.append(np.repeat(o[None], len(p), 0))
    near = scenes.Scene(scene.name, scene.timestep, scene.substeps, scene.steps, near_worlds)
    shift = np.concatenate(shift)
    for name, prec, solve in (("fp32", abi.PRECISION_FP32, abi.SOLVE_COLORED),
                              ("fp32_pos64", abi.PRECISION_FP32_POS64, abi.SOLVE_COLORED),
                              ("fp64", abi.PRECISION_FP64, abi.SOLVE_REFERENCE_ORDER)):
        a = rbps_b200.Batch.from_scene(scene, prec, solve, device=local, stream=stream.cuda_stream)
        b = rbps_b200.Batch.from_scene(near, abi.PRECISION_FP32 if prec == abi.PRECISION_FP32_POS64 else prec, solve,
                                       device=local, stream=stream.cuda_stream)
        a.step(200)
        b.step(200)
        d = np.abs(a.state_all()["position"] - (b.state_all()["position"] + shift))
        modes[name]["frame_error_200_steps_m"] = float(d.max())
        a.close()
        b.close()
    if rank == 0:
        line = {"metric": "body-substeps/s (precision stress: 256 worlds x 64-box towers 1e4 m from the origin, "
                          "FP32_POS64)",
                "value": modes["fp32_pos64"]["body_substeps_per_s"], "unit": UNIT, "n_gpus": ws, "steps": steps,
                "warmup": 0, "ms_per_step": modes["fp32_pos64"]["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "config4_precision_stress", "worlds": len(scene.worlds),
                           "bodies_per_world": len(scene.worlds[0].bodies), "substeps": scene.substeps,
                           "dt": scene.timestep, "offset_m": 1.0e4, "seed": args.seed,
                           "timing": "steps 1..K-1 of a fresh scene per mode; step K with dumps for the depths"},
                "modes": modes}
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="rbps", choices=["rbps", "reference"])
    ap.add_argument("--worlds", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=0, help="0 = as many as --steps")
    ap.add_argument("--cpu-seconds", type=float, default=30.0)
    ap.add_argument("--preroll", type=int, default=240,
                    help="untimed steps before the warm-up (240 = 2 s simulated: the bodies have landed)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--error-worlds", type=int, default=256,
                    help="worlds in the error report against FP64 (0 = skip it)")
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--autotune", type=int, default=1, help="1: run the launch-shape autotuner before timing")
    ap.add_argument("--plain-worlds", type=int, default=64,
                    help="worlds in the plain per-world GPU sample (0 = skip it)")
    ap.add_argument("--workload", default="batched",
                    choices=["batched", "collision_stress", "joint_heavy", "precision_stress"])
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    ws, rank, local = dist_info()
    from rbps_b200 import abi, scenes
    threads = os.cpu_count() or 1

    if args.impl == "reference":
        if rank != 0:
            return
        scene = scenes.config3(seed=args.seed, n_worlds=args.worlds)
        budget = float(os.environ.get("RBPS_BENCH_REF_SECONDS", "150"))
        value, info = cpu_reference_run(scene, args.preroll, args.warmup, args.steps, max_seconds=budget,
                                        threads=threads)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": {"workload": WORKLOAD, "worlds": args.worlds, "substeps": 4, "dt": 1 / 120,
                           "preroll_steps": args.preroll, "solver": "reference sequential Gauss-Seidel (CPU)"},
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                                 "sample": info},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device")
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import rbps_b200
    if args.workload in SINGLE_WORLD or args.workload == "precision_stress":
        (precision_stress if args.workload == "precision_stress" else single_world)(args, ws, rank, local)
        if ws > 1:
            torch.distributed.destroy_process_group()
        return

    # one set of worlds * ranks worlds, split across the ranks by balanced
    # body count (weak scaling: each rank keeps about `worlds` worlds)
    from rbps_b200 import shard
    scene, _ = shard.shard_scene(scenes.config3(seed=args.seed, n_worlds=args.worlds * ws), ws, rank)
    stream = torch.cuda.Stream()  # a real stream: the legacy NULL stream would not order our launches
    torch.cuda.set_stream(stream)
    free0 = torch.cuda.mem_get_info(local)[0]
    batch = rbps_b200.Batch.from_scene(scene, abi.PRECISION_FP32, abi.SOLVE_COLORED, device=local,
                                       stream=stream.cuda_stream, block_threads=args.block)
    torch.cuda.synchronize()
    dev_bytes = int(free0 - torch.cuda.mem_get_info(local)[0])
    n_tot, n_dyn = batch.total_bodies()
    n_coll = sum(len(w.colliders) for w in scene.worlds)
    n_joints = sum(len(w.joints) for w in scene.worlds)

    def barrier():
        if ws > 1:
            torch.distributed.barrier()

    # pre-roll to the resting regime, then warm-up (both untimed)
    if args.preroll:
        batch.step(args.preroll)
    batch.step(args.warmup)
    # launch shapes picked by the project autotuner on these worlds (untimed;
    # it rewinds the batch to where it started)
    tune = batch.autotune(trial_steps=3) if args.autotune else None
    # the e2e leg rewinds here, so that both legs time the same steps
    snap = batch.snapshot()
    batch.synchronize()

    # timed region: K steps, device events on the step stream
    bus = None
    try:
        bus = torch.cuda.get_device_properties(local).pci_bus_id
    except Exception:
        pass
    clocks = ClockSampler(bus)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    batch.step(args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    batch.synchronize()  # raises if the device reported an error during the timed steps
    barrier()
    ms = reduce_over_ranks(ev0.elapsed_time(ev1), "max", ws)
    st = batch.stats()
    n_dyn_all = reduce_over_ranks(n_dyn, "sum", ws)  # scenes differ per rank
    n_tot_all = reduce_over_ranks(n_tot, "sum", ws)
    value = n_dyn_all * scene.substeps * args.steps / (ms / 1e3)
    ms_step = ms / args.steps

    # roofline of the step kernel (one launch per step)
    bmodel = bytes_model(n_dyn, scene.substeps, st["contacts"], st["candidates"], st["pairs"], n_joints, n_coll)
    peak, peak_kind = measured_peaks()
    achieved = bmodel / (ms_step / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "step_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tr = json.load(f)
        # DRAM bytes of one step (all its launches) from ncu on a smaller batch, scaled by dynamic bodies
        traffic = tr["dram_bytes_per_step"] * n_dyn / tr["dynamic_bodies"]

    # end-to-end through the C ABI: forces in, poses out, pinned host buffers
    f_host = torch.empty((n_tot, 3), dtype=torch.float64, pin_memory=True)
    f_host.copy_(torch.from_numpy(np.concatenate([w.forces for w in scene.worlds])))
    p_host = torch.empty((n_tot, 3), dtype=torch.float64, pin_memory=True)
    q_host = torch.empty((n_tot, 4), dtype=torch.float64, pin_memory=True)
    # two pose buffers, alternating: every step's poses land on the host
    # (torch.empty_like would not pin them: a pageable target turns the copy synchronous)
    p_host2 = torch.empty((n_tot, 3), dtype=torch.float64, pin_memory=True)
    q_host2 = torch.empty((n_tot, 4), dtype=torch.float64, pin_memory=True)
    batch.step_io_async(f_host.data_ptr(), p_host.data_ptr(), q_host.data_ptr())  # stage buffers
    batch.restore(snap)  # back to the first timed step
    batch.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e2e_steps = args.steps if args.e2e_steps <= 0 else args.e2e_steps
    for k in range(e2e_steps):
        p_out, q_out = (p_host, q_host) if k % 2 == 0 else (p_host2, q_host2)
        batch.step_io_async(f_host.data_ptr(), p_out.data_ptr(), q_out.data_ptr())
    batch.synchronize()  # the last step's poses are on the host
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = reduce_over_ranks(e0.elapsed_time(e1), "max", ws)
    e2e_value = n_dyn_all * scene.substeps * e2e_steps / (e2e_ms / 1e3)
    finite = bool(np.isfinite(p_host.numpy()).all() and np.isfinite(p_host2.numpy()).all())

    err1 = None
    if rank == 0 and args.error_worlds > 0:
        batch.restore(snap)  # the first timed step's state
        nw = min(args.error_worlds, len(scene.worlds))
        settled = [batch.state(w) for w in range(nw)]
        err1 = error_vs_fp64(scene, nw, settled, stream)

    plain = None
    if args.plain_worlds > 0:
        pv, pinfo = plain_gpu_run(scene, batch, args.plain_worlds, min(args.steps, 20), args.warmup, stream)
        pv = reduce_over_ranks(pv, "sum", ws)  # every rank samples its own worlds
        plain = {"value": pv, "unit": UNIT, "sample": pinfo, "batched_over_plain": value / pv}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            cv, info = cpu_reference_run(scene, args.preroll, args.warmup, min(args.steps, 40), args.cpu_seconds,
                                         threads)
            cpu = {"value": cv, "unit": UNIT, "cores": threads, "kind": "reference", "sample": info}
        except Exception as e:  # the oracle library is missing
            cpu = {"value": None, "unit": UNIT, "cores": threads, "kind": "reference", "sample": f"unavailable: {e}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "worlds_per_gpu": args.worlds, "bodies_per_gpu": n_tot,
                           "dynamic_bodies_per_gpu": n_dyn, "substeps": scene.substeps, "dt": scene.timestep,
                           "precision": "fp32", "solver": "graph-coloured Gauss-Seidel",
                           "preroll_steps": args.preroll,
                           "timed_steps": f"{args.preroll + args.warmup + 1}..{args.preroll + args.warmup + args.steps}",
                           "device_bytes": dev_bytes,
                           "l2": f"inputs larger than L2: {dev_bytes / 1e6:.0f} MB of world state and scratch "
                                 "touched every step (L2 126 MB)",
                           "parallelism": f"worlds split over {ws} rank(s) by balanced body count",
                           "worlds_total": args.worlds * ws, "seed": args.seed,
                           "autotune": tune,
                           "state_finite": finite},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                             "algorithmic_bytes_per_step": bmodel,
                             "kernel": f"one step = {st['kernel_launches'] // max(args.steps, 1)} phase-kernel launches"},
                "cpu_baseline": cpu,
                "plain_gpu": plain,
                "error_vs_fp64": err1,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(n_tot_all) * 24,
                        "d2h_bytes_per_step": int(n_tot_all) * 56, "steps": e2e_steps,
                        "window": "the same steps as value (device snapshot after the warm-up, restored)"},
                "clocks": clk,
                "gpu_launches": int(st["kernel_launches"]),
                "cuda_graph": bool(st["graph"]),
                "stats_last_step": {"pairs": st["pairs"], "candidates": st["candidates"],
                                    "contacts": st["contacts"], "max_colors": st["max_colors"],
                                    "serial_overflow": st["serial_overflow"]}}
        print(json.dumps(line), flush=True)
    batch.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
