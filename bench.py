#!/usr/bin/env python
"""TreePM particle-steps/s of the bimetric (m+ / m-) step on a B200.

Workload (one "step" = one full KDK TreePM step of every particle):
  2 x 224^3 = 22,478,848 particles (11,239,424 m+, 11,239,424 m-) on a 224^3
  lattice per species (the m- lattice offset by half a cell) with seeded
  Zel'dovich displacements (P(k) ~ k^-2.5 exp(-(k/k_c)^2), k_c = half the
  lattice Nyquist, rms 0.3 spacing, delta- = -delta+), L = 250 Mpc, PM grid
  512^3, mu = M-/M+ = 19, theta = 0.5, r_s = 1.25 cells, r_cut = 4.5 r_s
  widened by --cut-tail-ppm (default 440: the short-range cut at 6 r_s, where
  the p99 force error against the FP64 periodic sum is <= 1e-3; the plain cut
  is timed beside it as `config_cut`), Plummer softening = mean spacing / 30,
  dt = 0.005 Gyr, Hubble drag from the FP64 Janus expansion at z = 4.
  Synthetic data; positions (360 MB per copy) are larger than L2, so no flush
  is needed between steps.

`python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]`
prints ONE JSON line on rank 0.  N > 1 (torchrun): every rank advances its own
independent box (different seed): replicas, weak scaling, no collective on the
data path; time = max over ranks.

--impl reference times the reference's CPU TreePM path (src/treepm/*.rs,
restated in C under oracle/ because the Rust crate cannot be built here) on
the host cores, each step a bounded sample of the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "janus-sim_b200"))

METRIC = "TreePM particle-steps/s at 2x224^3"
UNIT = "particle-steps/s"

# flops per interaction of the short-range force, each exp, rcp and rsqrt
# counted as one flop: a particle pair inside r_cut (split kernel S(x) by
# A&S 7.1.26) 40; a monopole + quadrupole node 100.  The distance test of
# every candidate, and the force the cell walk computes and discards for
# candidates outside r_cut, are overhead and not counted as useful work.
FLOPS_PAIR = 40.0
FLOPS_NODE = 100.0
# DRAM bytes of one k_walk_cell launch per particle, from ncu on the 2x112^3
# case at the same density and cut (profiles/k_walk_cell_2x112.md: 206.6 MB
# read + 65.5 MB written for 2,809,856 particles); it grows with N
WALK_DRAM_BYTES_PER_PARTICLE = 96.8
# Force errors |a - a_ref| / |a_ref| (p50, p99) of this engine on B200 at the
# benchmark configs, recorded by tests/test_gpu_accuracy_full.py (65,536
# seeded targets against the FP64 periodic sum, "full", and the truncated
# split model, "split"; the reference-kernel restatement for compatibility
# mode).  The bench does not run the FP64 oracle itself: these are the last
# recorded values, reported beside the speed they were measured with.
ACCURACY_B200 = {
    "source": "tests/test_gpu_accuracy_full.py on B200 (recorded, not re-run by the bench)",
    "metric": "p50, p99 of |a - a_ref| / |a_ref| over 65,536 targets",
    "production_2x224": {
        "cut_tail_440ppm_vs_full": [3.28e-05, 5.64e-04],
        "cut_4.5rs_vs_split": [2.48e-05, 4.26e-04],
        "cut_4.5rs_vs_full": [1.46e-03, 2.15e-02],
    },
    "clustered_2x128": {
        "theta_0.3_vs_split": [3.10e-06, 2.03e-04], "theta_0.3_tail_440ppm_vs_full": [1.23e-05, 1.61e-04],
        "theta_0.5_vs_split": [2.81e-05, 6.72e-04], "theta_0.5_tail_440ppm_vs_full": [4.02e-05, 3.75e-04],
        "theta_0.7_vs_split": [2.08e-04, 2.36e-03], "theta_0.7_tail_440ppm_vs_full": [2.09e-04, 2.13e-03],
    },
    "small_2x32_rcompat_vs_reference_kernels": [2.60e-07, 1.69e-06],
}


def workload(n_side=224, L=250.0, M=512):
    n_tot = 2 * n_side ** 3
    r_s = 1.25 * L / M
    return dict(n_side=n_side, L=L, M=M, mu=19.0, theta=0.5, r_s=r_s, r_cut=4.5 * r_s,
                eps=(L / n_tot ** (1.0 / 3.0)) / 30.0, dt=0.005, z=4.0, n_total=n_tot)


def hubble_at(z):
    from janus_treepm import expansion
    return expansion.state_at_redshift(z)[2]


def max_over_ranks(value, ws, device):
    """The largest value over all ranks (every rank's device time of the same
    timed region; the job's time is the slowest rank's)."""
    if ws <= 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_treepm_step(sample_div=4, seed=42, threads=None, r_cut=None):
    """One reference-CPU TreePM step (update + compute_all_forces + kick/drift)
    on a bounded sample of the workload: the same density, r_s, cut,
    softening and theta in a box of side L/sample_div (N/sample_div^3
    particles, PM grid M/sample_div).  Returns (particles, seconds, cores)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from janus_treepm import ics
    w = workload()
    n_side = w["n_side"] // sample_div
    L = w["L"] / sample_div
    M = w["M"] // sample_div
    pp, vp, pm, vm = ics.zeldovich_lattice(n_side, L, seed=seed)
    pos = np.concatenate([pp, pm]).astype(np.float64)
    vel = np.concatenate([vp, vm]).astype(np.float64)
    n = len(pp)
    mass = np.concatenate([np.full(n, 1.0), np.full(n, w["mu"])]) * 1e-3
    sg = np.concatenate([np.ones(n, np.int8), -np.ones(n, np.int8)])
    t0 = time.perf_counter()
    acc, tu, tf = O.cpu_treepm_forces(pos, mass, sg, r_cut or w["r_cut"], M, L, w["theta"], w["eps"])
    vel += acc * w["dt"]
    pos += vel * w["dt"]
    dt = time.perf_counter() - t0
    return len(pos), dt, (threads or os.cpu_count())


def reference_gpu_step(n_side, grid, steps=3):
    """The reference's own GPU TreePM step on this GPU: its kernels (the kernel
    text of src/nbody_gpu_twopass.rs and cuda/cufft_wrapper.cu, compiled for
    sm_100a into oracle/_ref/libref_gpu.so) in step_treepm_gpu's launch order
    (oracle/refgpu/replay.cu), on the same seeded workload, in a child
    process.  A yardstick beside the CPU baseline; None when the library was
    not built (it needs the reference checkout at build time)."""
    lib = os.path.join(ROOT, "oracle", "_ref", "libref_gpu.so")
    if not os.path.exists(lib):
        return None
    try:
        out = subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "refgpu", "time_refgpu.py"),
                              "--n-side", str(n_side), "--grid", str(grid), "--steps", str(steps)],
                             capture_output=True, text=True, timeout=600)
        line = [x for x in out.stdout.splitlines() if x.startswith("{")]
        if out.returncode != 0 or not line:
            return {"error": (out.stderr or out.stdout)[-300:]}
        r = json.loads(line[-1])
        r["kind"] = "reference"
        r["value"] = r.pop("particle_steps_per_s")
        r["unit"] = UNIT
        return r
    except Exception as e:   # the yardstick never fails the bench
        return {"error": str(e)[:300]}


def counted_step(s, step):
    """One more step with the pair counters on (a diagnostic that the timed
    steps run without: one instruction per candidate pair of the cell walk),
    outside the timed region; its timings give the pairs, nodes and
    candidates of a step."""
    s.set_counters(True)
    step()
    tm = s.timings()
    s.set_counters(False)
    return tm


def run_clustered(J, ics, steps, warmup, H, dt, cut_tail_ppm=0, theta=0.5):
    """The clustered workload: 2x128^3 particles, 80 % in 512 Plummer spheres
    (scale radii log-uniform 0.05-1 Mpc, species alternating by sphere) + 20 %
    uniform background, L = 100 Mpc, PM 256^3, theta 0.5, mu 19, r_s = 1.25
    cells, cut 4.5 r_s (or widened by cut_tail_ppm), softening spacing/30.
    Most cells are too crowded for the cell walk, so the LBVH build and the
    Barnes-Hut group walk (multipoles) do the near field.  Device time of K
    KDK steps after W warm-up steps; the tree walk's FP32 roofline beside it."""
    n_side, L, M = 128, 100.0, 256
    n = n_side ** 3
    r_s = 1.25 * L / M
    pp, pm = ics.plummer_spheres(n, L, n_spheres=512, seed=42)
    cfg = J.Config(box_L=L, pm_grid=M, theta=theta, softening=(L / (2 * n) ** (1 / 3)) / 30, r_s=r_s,
                   r_cut=4.5 * r_s, mu=19.0, G_mass_plus=1.0e-3, cut_tail_ppm=cut_tail_ppm)
    s = J.Solver(cfg)
    s.set_state(pp, None, pm, None)
    for _ in range(warmup):
        s.step(dt, H, 1.0, 1)
    dev, stages = 0.0, {}
    for _ in range(steps):
        s.step(dt, H, 1.0, 1)
        tm = s.timings()
        dev += tm["total_ms"]
        for k, v in tm.items():
            stages[k] = stages.get(k, 0.0) + v
    counted = counted_step(s, lambda: s.step(dt, H, 1.0, 1))
    s.close()
    walk_ms = stages["walk_ms"] / steps - stages.get("interp_ms", 0.0) / steps
    flops = counted["pair_interactions"] * FLOPS_PAIR + counted["node_interactions"] * FLOPS_NODE
    return {"workload": f"2x{n_side}^3 in 512 Plummer spheres + 20 % background, L={L:g} Mpc, PM {M}^3, "
                        f"theta {theta}, mu 19, cut {J.short_cut(cfg) / r_s:.3g} r_s",
            "value": 2 * n * steps / (dev * 1e-3), "unit": UNIT, "ms_per_step": dev / steps,
            "stages_ms_per_step": {k: round(v / steps, 4) for k, v in stages.items() if k.endswith("_ms")},
            "pairs_per_step": counted["pair_interactions"],
            "nodes_per_step": counted["node_interactions"],
            "walk_tflops": flops / (walk_ms * 1e-3) / 1e12 if walk_ms > 0 else None,
            "steps": steps, "warmup": warmup}


def ensemble_boxes(n_boxes=64, seed=7):
    """The batched-ensemble workload: n_boxes independent boxes, n per species
    log-uniform in [16, 96] (N = n^3 per species), L ~ U(50, 300) Mpc, PM grid
    = next power of two >= 2n (32..256), mu ~ U(5, 30), eta ~ U(1.00, 1.10)
    (eta enters only the expansion factors, not the force path), seeded
    Zel'dovich ICs (seed 1000 + box), the 2x224^3 workload's theta / r_s / r_cut / softening
    rules and mass density."""
    rng = np.random.default_rng(seed)
    boxes = []
    for b in range(n_boxes):
        n = int(round(np.exp(rng.uniform(np.log(16), np.log(96)))))
        L = float(rng.uniform(50.0, 300.0))
        M = 1 << int(np.ceil(np.log2(2 * n)))
        mu = float(rng.uniform(5.0, 30.0))
        eta = float(rng.uniform(1.0, 1.1))
        boxes.append(dict(n=n, L=L, M=M, mu=mu, eta=eta, seed=1000 + b))
    return boxes


def box_config(J, bx):
    r_s = 1.25 * bx["L"] / bx["M"]
    spacing = bx["L"] / bx["n"]
    # the 2x224^3 workload's mass per particle scaled to the same mean density
    gm = 1.0e-3 * (spacing / (250.0 / 224.0)) ** 3
    return J.Config(box_L=bx["L"], pm_grid=bx["M"], theta=0.5,
                    softening=bx["L"] / (2 * bx["n"] ** 3) ** (1.0 / 3.0) / 30.0, r_s=r_s,
                    r_cut=4.5 * r_s, mu=bx["mu"], G_mass_plus=gm, mode=J.JT_ACCURATE,
                    integrator=J.JT_KDK)


def run_ensemble(J, ics, n_boxes, steps, warmup, H, dt):
    """Batched steps of the ensemble vs the same boxes one at a time through
    single handles (the plain path).  Device time of each call from its CUDA
    events; wall time beside it."""
    import torch
    boxes = ensemble_boxes(n_boxes)
    states = [ics.zeldovich_lattice(bx["n"], bx["L"], seed=bx["seed"]) for bx in boxes]
    n_part = sum(2 * bx["n"] ** 3 for bx in boxes)
    # batched
    B = J.Batch()
    ids = [B.add(box_config(J, bx), *st) for bx, st in zip(boxes, states)]
    for _ in range(warmup):
        B.step(ids, dt, H, 1.0, 1)
    torch.cuda.synchronize()
    dev, t0 = 0.0, time.perf_counter()
    stages = {}
    for _ in range(steps):
        B.step(ids, dt, H, 1.0, 1)
        tm = B.timings()
        dev += tm["total_ms"]
        for k, v in tm.items():
            stages[k] = stages.get(k, 0.0) + v
    torch.cuda.synchronize()
    wall_b = time.perf_counter() - t0
    mem = B.memory()
    # the same steps replayed as CUDA graphs (captured once for the set)
    B.set_graphs(True)
    B.step(ids, dt, H, 1.0, 1)
    torch.cuda.synchronize()
    dev_g, t0 = 0.0, time.perf_counter()
    for _ in range(steps):
        B.step(ids, dt, H, 1.0, 1)
        dev_g += B.timings()["total_ms"]
    torch.cuda.synchronize()
    wall_g = time.perf_counter() - t0
    B.close()
    # plain: one handle per box, stepped one after another
    solvers = []
    for bx, st in zip(boxes, states):
        s = J.Solver(box_config(J, bx))
        s.set_state(*st)
        solvers.append(s)
    for _ in range(warmup):
        for s in solvers:
            s.step(dt, H, 1.0, 1)
    torch.cuda.synchronize()
    dev_p, t0 = 0.0, time.perf_counter()
    for _ in range(steps):
        for s in solvers:
            s.step(dt, H, 1.0, 1)
            dev_p += s.timings()["total_ms"]
    torch.cuda.synchronize()
    wall_p = time.perf_counter() - t0
    for s in solvers:
        s.close()
    v_b = n_part * steps / (dev * 1e-3)
    v_p = n_part * steps / (dev_p * 1e-3)
    return {
        "workload": f"{n_boxes} boxes, n per species log-uniform 16..96 ({n_part} particles), "
                    f"L U(50,300), PM 32..256, mu U(5,30)",
        "value": v_b, "unit": UNIT, "ms_per_step": dev / steps,
        "wall_value": n_part * steps / wall_b,
        "graph_value": n_part * steps / (dev_g * 1e-3), "graph_wall_value": n_part * steps / wall_g,
        "plain_value": v_p, "plain_ms_per_step": dev_p / steps,
        "plain_wall_value": n_part * steps / wall_p,
        "speedup_vs_plain": v_b / v_p, "speedup_vs_plain_wall": wall_p / wall_b,
        "launches_per_step": stages.get("launches", 0) / steps,
        "stages_ms_per_step": {k: round(v / steps, 4) for k, v in stages.items() if k.endswith("_ms")},
        "device_bytes": {"persistent": mem[0], "scratch": mem[1]},
        "steps": steps,
    }


def run_ensemble_sharded(J, ics, n_boxes, steps, warmup, H, dt, rank, ws):
    """The ensemble sharded across the ranks (janus_treepm.shard): each rank
    steps its share of the boxes (a cost-balanced partition every rank
    computes alike) as one batch on its GPU, with no exchange; the device
    time is the max over ranks, the value all boxes' particle-steps over it
    (strong scaling: the total work stays fixed as N grows), and rank 0
    gathers each rank's boxes, particles and time.  Every rank calls it."""
    import torch
    from janus_treepm import shard
    boxes = ensemble_boxes(n_boxes)
    costs = [shard.box_cost(2 * bx["n"] ** 3, bx["M"]) for bx in boxes]
    shares = shard.partition(costs, ws)
    mine = shares[rank]
    n_part = sum(2 * bx["n"] ** 3 for bx in boxes)
    dev = 0.0
    if mine:
        B = J.Batch()
        ids = [B.add(box_config(J, boxes[i]), *ics.zeldovich_lattice(boxes[i]["n"], boxes[i]["L"],
                                                                       seed=boxes[i]["seed"]))
               for i in mine]
        for _ in range(warmup):
            B.step(ids, dt, H, 1.0, 1)
        torch.cuda.synchronize()
        for _ in range(steps):
            B.step(ids, dt, H, 1.0, 1)
            dev += B.timings()["total_ms"]
        torch.cuda.synchronize()
        B.close()
    dev_max = max_over_ranks(dev, ws, "cuda")
    metrics = shard.gather({"rank": rank, "boxes": len(mine),
                            "particles": sum(2 * boxes[i]["n"] ** 3 for i in mine),
                            "ms_per_step": dev / steps}, ws)
    if rank != 0:
        return None
    ld = shard.loads(costs, shares)
    return {
        "workload": f"{n_boxes} boxes, n per species log-uniform 16..96 ({n_part} particles), "
                    f"L U(50,300), PM 32..256, mu U(5,30), sharded by box over {ws} ranks",
        "value": n_part * steps / (dev_max * 1e-3), "unit": UNIT, "ms_per_step": dev_max / steps,
        "scaling": "strong", "ranks": ws, "per_rank": metrics,
        "cost_max_over_mean": max(ld) / (sum(ld) / len(ld)), "steps": steps,
    }


def run_serving_sharded(J, ics, n_small, n_big, steps, H, dt, rank, ws, budget_gb=150.0):
    """The serving workload's jobs sharded across the ranks
    (janus_treepm.shard, the cost of a job from its particles and grid):
    each rank serves its share on its GPU as a saturated run (every request
    at t = 0) under its own budget; the makespan is the max over ranks, and
    rank 0 gathers each rank's jobs, requests served and makespan.  Every
    rank calls it."""
    from janus_treepm import shard
    jobs = serving_jobs(J, ics, n_small, n_big, H, dt)
    costs = [shard.box_cost(p, cfg.pm_grid) for cfg, _, p in jobs]
    shares = shard.partition(costs, ws)
    mine = [jobs[i] for i in shares[rank]]
    wall, served = 0.0, 0
    if mine:
        wall, st = serve_once(J, mine, steps, None, H, dt, budget_gb, seed=11)
        served = int(st["requests_served"])
    wall_max = max_over_ranks(wall, ws, "cuda")
    metrics = shard.gather({"rank": rank, "jobs": len(mine), "requests": served, "makespan_s": wall}, ws)
    if rank != 0:
        return None
    total_ps = float(sum(p for _, _, p in jobs) * steps)
    ld = shard.loads(costs, shares)
    return {
        "workload": f"{n_small} ensemble-style jobs + {n_big} jobs of 2x256^3 (L=300, PM 512^3), "
                    f"{steps} steps each, {budget_gb:g} GB HBM budget per rank, sharded by job over "
                    f"{ws} ranks, saturated (every request at t = 0)",
        "particle_steps": total_ps, "saturated_value": total_ps / wall_max, "unit": UNIT,
        "makespan_s": wall_max, "scaling": "strong", "ranks": ws, "per_rank": metrics,
        "cost_max_over_mean": max(ld) / (sum(ld) / len(ld)),
    }


def serving_jobs(J, ics, n_small, n_big, H, dt, seed=11):
    """The serving workload's jobs: n_small boxes sized as the ensemble's plus
    n_big boxes of 2x256^3 (L = 300 Mpc, PM 512^3).  The big jobs share one
    Zel'dovich realisation, each moved by a random periodic shift and axis
    permutation (generating eight 256^3 fields would take minutes of host
    time).  Returns [(config, state, particles)]."""
    rng = np.random.default_rng(seed)
    jobs = []
    for bx in ensemble_boxes(n_small, seed=seed):
        jobs.append((box_config(J, bx), ics.zeldovich_lattice(bx["n"], bx["L"], seed=bx["seed"]),
                     2 * bx["n"] ** 3))
    if n_big:
        base = ics.zeldovich_lattice(256, 300.0, seed=seed)
        cfg = box_config(J, dict(n=256, L=300.0, M=512, mu=19.0))
        for _ in range(n_big):
            shift = rng.uniform(-150.0, 150.0, 3).astype(np.float32)
            perm = rng.permutation(3)
            st = []
            for k, a in enumerate(base):
                a = a[:, perm]
                if k % 2 == 0:
                    a = ((a + shift + 150.0) % 300.0 - 150.0).astype(np.float32)
                st.append(np.ascontiguousarray(a))
            jobs.append((cfg, tuple(st), 2 * 256 ** 3))
    return jobs


def serve_once(J, jobs, steps, rate, H, dt, budget_gb, seed):
    """One serving run: every job wants `steps` steps; requests arrive as one
    Poisson stream of the given rate (requests/s; None = all at t = 0), request
    k of a job in round k, jobs in a random order per round."""
    rng = np.random.default_rng(seed)
    S = J.Server(int(budget_gb * (1 << 30)))
    for cfg, st, _ in jobs:
        S.add_job(cfg, *st, steps=steps, dt=dt, hubble=H)
    order = np.concatenate([rng.permutation(len(jobs)) for _ in range(steps)])
    if rate is None:
        t = np.zeros(len(order))
    else:
        t = np.cumsum(rng.exponential(1.0 / rate, len(order)))
        t -= t[0]
    t0 = time.perf_counter()
    S.serve(t, order)
    wall = time.perf_counter() - t0
    st = S.stats()
    st["stages_ms"] = {k: round(v, 3) for k, v in S.timings().items() if k.endswith("_ms")}
    S.close()
    return wall, st


def run_serving(J, ics, n_small, n_big, steps, rates, H, dt, budget_gb=150.0):
    """Serving loop: a saturated run (every request at t = 0) measures the
    server's capacity in requests/s, then Poisson runs at the given fractions
    of it report p50/p99 per-request latency and throughput.  The plain-path
    estimate runs a seeded sample of the jobs one at a time through handles
    (load the state, take every step) and scales it by particle-steps."""
    import torch
    jobs = serving_jobs(J, ics, n_small, n_big, H, dt)
    parts = [p for _, _, p in jobs]
    total_ps = float(sum(parts) * steps)
    # plain path: jobs one at a time through a handle, each as a served job
    # runs (load the state, take all its steps): a seeded sample of 16 small
    # jobs and one big job, timed and scaled by particle-steps
    def plain_time(sel):
        t = 0.0
        for cfg, st, _ in sel:
            s = J.Solver(cfg)
            s.set_state(*st)
            s.accel()   # plans and the walk autotuner outside the timed region
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.set_state(*st)
            s.step(dt, H, 1.0, steps)
            torch.cuda.synchronize()
            t += time.perf_counter() - t0
            s.close()
        return t
    small_jobs = [j for j in jobs if j[2] != 2 * 256 ** 3]
    pick = np.random.default_rng(5).choice(len(small_jobs), min(16, len(small_jobs)), replace=False)
    sample = [small_jobs[k] for k in pick]
    t_small = plain_time(sample)
    plain_s = t_small * sum(j[2] for j in small_jobs) / sum(j[2] for j in sample)
    if n_big:
        plain_s += n_big * plain_time([jobs[-1]])
    out = {"workload": f"{n_small} ensemble-style jobs + {n_big} jobs of 2x256^3 (L=300, PM 512^3), "
                       f"{steps} steps each, {budget_gb:g} GB HBM budget",
           "particle_steps": total_ps, "plain_value_estimate": total_ps / plain_s, "runs": []}
    wall, st = serve_once(J, jobs, steps, None, H, dt, budget_gb, seed=11)
    cap = st["requests_served"] / wall
    out["capacity_requests_per_s"] = cap
    out["saturated_value"] = total_ps / wall
    out["saturated_gpu_busy_frac"] = st["busy_s"] / wall
    out["saturated_vs_plain"] = (total_ps / wall) / (total_ps / plain_s)
    out["saturated_swaps_trims"] = [int(st["swapped_out"]), int(st["trims"])]
    out["saturated_host_s"] = {"admit": st["admit_s"], "evict": st["evict_s"], "steps": st["busy_s"],
                               "steps_device": st["step_device_s"], "wall": wall,
                               "batched_steps": int(st["batched_steps"]),
                               "max_jobs_per_step": int(st["max_jobs_per_step"]),
                               "reserved_gb": st["reserved_gb"]}
    out["saturated_stages_ms"] = st["stages_ms"]
    for frac in rates:
        wall, st = serve_once(J, jobs, steps, frac * cap, H, dt, budget_gb, seed=12)
        out["runs"].append({
            "rate_vs_capacity": frac, "arrival_rate_per_s": frac * cap,
            "value": total_ps / wall, "unit": UNIT, "makespan_s": wall,
            "vs_plain": (total_ps / wall) / (total_ps / plain_s),
            "p50_latency_ms": 1e3 * st["p50_latency_s"], "p99_latency_ms": 1e3 * st["p99_latency_s"],
            "max_latency_ms": 1e3 * st["max_latency_s"], "gpu_busy_frac": st["busy_s"] / wall,
            "requests": int(st["requests_served"]), "batched_steps": int(st["batched_steps"]),
            "max_jobs_per_step": int(st["max_jobs_per_step"]),
            "admission_waits": int(st["admission_waits"]), "swapped_out": int(st["swapped_out"]),
            "trims": int(st["trims"]), "admit_s": st["admit_s"], "evict_s": st["evict_s"],
            "steps_device_s": st["step_device_s"], "peak_device_gb": st["peak_device_bytes"] / 1e9})
    return out


def config_of(w, args, short_cut, ws):
    """The `config` object of both arms' JSON lines (the same workload)."""
    return {"workload": f"TreePM KDK step 2x{w['n_side']}^3, L={w['L']:g} Mpc, "
                        f"PM {w['M']}^3, mu=19, theta=0.5, r_s=1.25 cells, "
                        f"short-range cut {short_cut / w['r_s']:.3g} r_s, accurate mode",
            "cut_tail_ppm": args.cut_tail_ppm,
            "l2": "inputs larger than L2 (no flush)",
            "parallelism": "replicas" if ws > 1 else "single"}


def short_cut_of(w, args):
    """The engine's short-range cut for the workload (r_cut, or widened by
    --cut-tail-ppm): the same formula as jt_config_short_cut, here without
    loading the library (the reference arm)."""
    from math import erfc, exp
    if args.cut_tail_ppm <= 0:
        return w["r_cut"]
    tol = 1e-6 * args.cut_tail_ppm
    lo, hi = 0.0, 8.0
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        if erfc(mid) + 1.1283791670955126 * mid * exp(-mid * mid) > tol:
            lo = mid
        else:
            hi = mid
    return max(w["r_cut"], 2.0 * w["r_s"] * hi)


def run_reference(args, ws, rank):
    """The reference's CPU TreePM path (src/treepm: TreePMForce::update +
    compute_all_forces, then the kick and drift), restated in C with OpenMP
    over all host cores (oracle/ref_cpu_treepm.c; the Rust crate cannot be
    built here).  Each of the W + K steps is one full step of a bounded
    sample of the workload (2x112^3 particles in a box half the side: the
    same density, r_s, cut, softening and theta), so the run ends in a few
    minutes; one full-size 2x224^3 step is timed once after them as a check
    that the sample's rate is the workload's."""
    if rank != 0:
        return 0
    w = workload(args.n_side, 250.0 * args.n_side / 224.0, args.grid)
    div = args.cpu_sample_div
    cut = short_cut_of(w, args)
    for k in range(args.warmup):
        cpu_treepm_step(div, seed=100 + k, r_cut=cut)
    tot_n, tot_t, cores = 0, 0.0, os.cpu_count()
    for k in range(args.steps):
        n, t, cores = cpu_treepm_step(div, seed=42 + k, r_cut=cut)
        tot_n += n
        tot_t += t
    v = tot_n / tot_t
    full = None
    if not args.no_full_reference_step:
        nf, tf, _ = cpu_treepm_step(1, seed=42, r_cut=cut)
        full = {"particles": nf, "seconds": tf, "value": nf / tf, "unit": UNIT,
                "what": "one full-size 2x224^3 step of the same code, outside the timed steps"}
    sample = (f"2x{w['n_side'] // div}^3 particles, L={w['L'] / div:g} Mpc, PM "
              f"{w['M'] // div}^3 (the workload's density, r_s, cut, eps, theta in a box "
              f"1/{div} the side); one full step per sample, {cores} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Zel'dovich lattice)",
        "config": config_of(w, args, cut, ws),
        "reference_path": "src/treepm (TreePMForce update + compute_all_forces), C restatement "
                          "with OpenMP (oracle/ref_cpu_treepm.c)",
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "full_size_step": full,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, ws, rank, local):
    import torch
    import janus_treepm as J
    from janus_treepm import ics
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist_
        dist_.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    w = workload(args.n_side, 250.0 * args.n_side / 224.0, args.grid)
    H = hubble_at(w["z"])
    seed = 42 + rank
    pp, vp, pm, vm = ics.zeldovich_lattice(w["n_side"], w["L"], seed=seed)
    n = len(pp)
    cfg = J.Config(box_L=w["L"], pm_grid=w["M"], theta=w["theta"], softening=w["eps"],
                   r_s=w["r_s"], r_cut=w["r_cut"], mu=w["mu"], G_mass_plus=1.0e-3,
                   mode=J.JT_ACCURATE, integrator=J.JT_KDK, cut_tail_ppm=args.cut_tail_ppm)
    short_cut = J.short_cut(cfg)
    s = J.Solver(cfg)
    s.set_state(pp, vp, pm, vm)
    peak_fp32 = J.fp32_peak_tflops()

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()

    for _ in range(args.warmup):
        s.step(w["dt"], H, 1.0, 1)
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    t_wall = time.perf_counter()
    dev_ms = 0.0
    stages = {}
    for _ in range(args.steps):
        s.step(w["dt"], H, 1.0, 1)
        tm = s.timings()
        dev_ms += tm["total_ms"]
        for k, v in tm.items():
            stages[k] = stages.get(k, 0.0) + v
    barrier()
    wall = time.perf_counter() - t_wall
    clk = clocks.stop()
    counted = counted_step(s, lambda: s.step(w["dt"], H, 1.0, 1))
    dev_ms = max_over_ranks(dev_ms, ws, "cuda")
    K = args.steps
    value = ws * 2 * n * K / (dev_ms * 1e-3)

    # the same step at the plain cut r_cut = 4.5 r_s (p99 force error 4e-4
    # against the split model it integrates, 2e-2 against the full periodic
    # sum): a second handle, timed the same way
    config_cut = None
    if args.config_cut_steps > 0 and args.cut_tail_ppm > 0:
        cfg0 = J.Config(box_L=w["L"], pm_grid=w["M"], theta=w["theta"], softening=w["eps"],
                        r_s=w["r_s"], r_cut=w["r_cut"], mu=w["mu"], G_mass_plus=1.0e-3,
                        mode=J.JT_ACCURATE, integrator=J.JT_KDK, cut_tail_ppm=0)
        s0 = J.Solver(cfg0)
        s0.set_state(pp, vp, pm, vm)
        for _ in range(3):
            s0.step(w["dt"], H, 1.0, 1)
        barrier()
        d0, st0 = 0.0, {}
        for _ in range(args.config_cut_steps):
            s0.step(w["dt"], H, 1.0, 1)
            tm = s0.timings()
            d0 += tm["total_ms"]
            for k, v in tm.items():
                st0[k] = st0.get(k, 0.0) + v
        barrier()
        s0.close()
        d0 = max_over_ranks(d0, ws, "cuda")
        K0 = args.config_cut_steps
        config_cut = {"cut": "4.5 r_s", "value": ws * 2 * n * K0 / (d0 * 1e-3), "unit": UNIT,
                      "ms_per_step": d0 / K0, "steps": K0, "warmup": 3,
                      "stages_ms_per_step": {k: round(v / K0, 4) for k, v in st0.items() if k.endswith("_ms")}}

    # end to end through the C ABI with pinned host buffers: every step
    # uploads the state a KDK step starts from (positions, velocities and the
    # accelerations at those positions), steps once, and reads the same three
    # back into the pinned buffers, which the next step uploads again
    # (jt_step_host: one call per step, the positions coming back during the
    # force pass)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    cur = [pin(a) for a in (pp, vp, pm, vm)]
    acc = [pin(np.zeros_like(pp)), pin(np.zeros_like(pm))]
    s.set_state(*cur)
    s.step(w["dt"], H, 1.0, 1)
    s.get_state(out=cur)
    s.get_accel(out=acc)
    s.step_host(cur[0], cur[1], acc[0], cur[2], cur[3], acc[1], w["dt"], H, 1.0)
    barrier()
    t0 = time.perf_counter()
    for _ in range(K):
        s.step_host(cur[0], cur[1], acc[0], cur[2], cur[3], acc[1], w["dt"], H, 1.0)
    barrier()
    e2e_t = time.perf_counter() - t0
    e2e_t = max_over_ranks(e2e_t, ws, "cuda")
    e2e = ws * 2 * n * K / e2e_t
    bytes_state = 2 * n * 3 * 4 * 3     # positions, velocities, accelerations; both species

    # the PM interpolation (k_b_interp, timed alone by its own events inside
    # the step).  Algorithmic bytes: positions in (16 B) and one float4 per
    # particle and interlaced grid out, and every value of the 3 x NG force
    # grids read once (tiles staged in shared memory)
    interp_ms = stages.get("interp_ms", 0.0) / K
    G = w["M"] ** 3
    interp_bytes = 16.0 * 2 * n + 16.0 * 2 * 2 * n + 4.0 * 3 * 2 * G

    # roofline of the dominant kernel: the near-field cell walk (FP32 pipe),
    # timed alone by its own events (the walk stage also holds the cell list
    # build and the tree walk of flagged particles, none at this density)
    walk_ms = (stages["cellwalk_ms"] if stages.get("cellwalk_ms", 0.0) > 0 else stages["walk_ms"]) / K
    pairs = counted["pair_interactions"]
    nodes = counted["node_interactions"]
    cands = counted["candidates"]
    achieved = (pairs * FLOPS_PAIR + nodes * FLOPS_NODE) / (walk_ms * 1e-3) / 1e12
    Gc = w["M"] * w["M"] * (w["M"] // 2 + 1)
    ks_ms = stages["kspace_ms"] / K
    ngrid = 2   # interlaced (the accurate default): reads 2 spectra, writes 6
    ks_gbs = 32.0 * ngrid * Gc / (ks_ms * 1e-3) / 1e9
    hbm_peak = 6550.7
    try:
        hbm_peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        hbm_src = "measured"
    except Exception:
        hbm_src = "fallback"
    walk_traffic = WALK_DRAM_BYTES_PER_PARTICLE * 2 * n if args.grid * 224 == 512 * args.n_side else None
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        npart, tcpu, cores = cpu_treepm_step(args.cpu_sample_div, r_cut=short_cut)
        cpu = {"value": npart / tcpu, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"one reference-CPU TreePM step (oracle/ref_cpu_treepm.c) on "
                         f"2x{w['n_side'] // args.cpu_sample_div}^3 particles in a box "
                         f"1/{args.cpu_sample_div} the side (same density, r_s, cut, "
                         f"eps, theta), {tcpu:.1f} s"}
    launches = stages.get("launches", 0)
    walk_tuning = J.walk_tuning()
    # the headline handle's memory back to the device before the other legs
    # (the serving loop reserves a 150 GiB budget)
    s.close()
    ensemble = None
    serving = None
    if ws > 1 and args.ensemble_boxes > 0:   # every rank: the boxes shard across them
        ensemble = run_ensemble_sharded(J, ics, args.ensemble_boxes, args.ensemble_steps, 3, H, w["dt"],
                                        rank, ws)
    if ws > 1 and args.serve_jobs > 0:       # every rank: the jobs shard across them
        serving = run_serving_sharded(J, ics, args.serve_jobs, args.serve_big, args.serve_steps, H, w["dt"],
                                      rank, ws)
    ref_gpu = None
    if rank == 0 and ws == 1 and not args.no_reference_gpu:
        ref_gpu = reference_gpu_step(args.n_side, args.grid)
    clustered = None
    if rank == 0 and ws == 1 and args.clustered_steps > 0:
        clustered = run_clustered(J, ics, args.clustered_steps, 3, H, w["dt"], args.cut_tail_ppm)
        if clustered.get("walk_tflops"):
            clustered["walk_frac_fp32"] = clustered["walk_tflops"] / peak_fp32
    if rank == 0 and ws == 1 and args.ensemble_boxes > 0:
        ensemble = run_ensemble(J, ics, args.ensemble_boxes, args.ensemble_steps, 3, H, w["dt"])
    if rank == 0 and ws == 1 and args.serve_jobs > 0:
        try:
            serving = run_serving(J, ics, args.serve_jobs, args.serve_big, args.serve_steps,
                                  [float(r) for r in args.serve_rates.split(",")], H, w["dt"])
        except J.JanusError as e:
            serving = {"error": str(e)}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K,
            "warmup": args.warmup, "ms_per_step": dev_ms / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Zel'dovich lattice)",
            "config": config_of(w, args, short_cut, ws),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": bytes_state * ws,
                    "d2h_bytes_per_step": bytes_state * ws},
            "roofline": {"bound": "fp32", "kernel": "k_walk_cell", "achieved": achieved,
                         "peak": peak_fp32, "unit": "TFLOP/s", "frac": achieved / peak_fp32,
                         "traffic": walk_traffic,
                         "peak_source": "measured (jt_fp32_peak FMA kernel, same run)",
                         "work": f"{pairs:.4g} pairs x {FLOPS_PAIR:g} + {nodes:.4g} nodes x "
                                 f"{FLOPS_NODE:g} flop per step ({cands:.4g} candidates tested)"},
            "roofline_hbm": {"bound": "hbm",
                             "kernel": ("k_zfft_kspace (z transforms of the 2 density and 6 force spectra "
                                        "fused with the k-space step)" if w["M"] == 512 and
                                        os.environ.get("JT_ZFFT", "1") != "0" else "k_b_kspace"),
                             "bytes": 32.0 * ngrid * Gc, "ms": ks_ms, "achieved": ks_gbs,
                             "peak": hbm_peak, "unit": "GB/s", "frac": ks_gbs / hbm_peak,
                             "peak_source": hbm_src},
            "roofline_deposit": {"bound": "hbm", "kernel": "k_b_deposit (+ grid zeroing, tile ranges)",
                                 "ms": stages["deposit_ms"] / K, "bytes": 16.0 * 2 * n + 4.0 * 2 * G,
                                 "achieved": (16.0 * 2 * n + 4.0 * 2 * G) / (stages["deposit_ms"] / K * 1e-3) / 1e9,
                                 "peak": hbm_peak, "unit": "GB/s",
                                 "frac": (16.0 * 2 * n + 4.0 * 2 * G) / (stages["deposit_ms"] / K * 1e-3) / 1e9
                                 / hbm_peak,
                                 "peak_source": hbm_src},
            "roofline_interp": {"bound": "hbm", "kernel": "k_b_interp (tiled PM interpolation)",
                                "ms": interp_ms, "bytes": interp_bytes,
                                "achieved": interp_bytes / (interp_ms * 1e-3) / 1e9 if interp_ms > 0 else None,
                                "peak": hbm_peak, "unit": "GB/s",
                                "frac": interp_bytes / (interp_ms * 1e-3) / 1e9 / hbm_peak if interp_ms > 0 else None,
                                "peak_source": hbm_src},
            "stages_ms_per_step": {k: round(v / K, 4) for k, v in stages.items()
                                   if k.endswith("_ms")},
            "wall_ms_per_step": 1e3 * wall / K,
            "clocks": clk,
            "gpu_launches": int(launches),
            "walk_autotune": walk_tuning,
            "cpu_baseline": cpu,
            "reference_gpu": ref_gpu,
            "config_cut": config_cut,
            "accuracy": ACCURACY_B200,
            "clustered": clustered,
            "ensemble": ensemble,
            "serving": serving,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n-side", type=int, default=224)
    ap.add_argument("--grid", type=int, default=512)
    ap.add_argument("--cpu-sample-div", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ensemble-boxes", type=int, default=64)
    ap.add_argument("--ensemble-steps", type=int, default=5)
    ap.add_argument("--serve-jobs", type=int, default=256)
    ap.add_argument("--serve-big", type=int, default=8)
    ap.add_argument("--serve-steps", type=int, default=4)
    ap.add_argument("--serve-rates", default="0.5,1.0")
    ap.add_argument("--clustered-steps", type=int, default=5,
                    help="steps of the clustered workload leg (0: skip)")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference's own GPU step (oracle/refgpu) beside the CPU baseline")
    ap.add_argument("--no-full-reference-step", action="store_true",
                    help="reference arm: skip the one full-size step timed after the samples")
    ap.add_argument("--cut-tail-ppm", type=int, default=440,
                    help="widen the short-range cut until S(r / 2 r_s) = ppm * 1e-6 (0: r_cut = "
                         "4.5 r_s).  440 (cut 6 r_s) keeps p99 force error <= 1e-3 against the FP64 "
                         "periodic sum (tests/test_gpu_accuracy_full.py)")
    ap.add_argument("--config-cut-steps", type=int, default=5,
                    help="also time this many steps at the plain cut 4.5 r_s (0: skip)")
    args = ap.parse_args()
    ws, rank, local = dist()
    if args.impl == "reference":
        return run_reference(args, ws, rank)
    return run_ours(args, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
