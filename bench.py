"""Benchmark: ns/day of the 64 000-ion LJ + PME melt on B200 (one process per GPU).

Workload (plain form): 32 000 Na+ / 32 000 Cl- ions at 0.0375 per cubic Angstrom
(L = 119.5 A), LJ eps = 0.01 eV, sigma = 2.8 A, r_c = 9 A; SPME r_c = 9 A,
erfc(alpha r_c) = 1e-5, mesh spacing 1 A (120^3), order 5; FP32 forces;
velocity-Verlet NVE at dt = 1 fs from a 1200 K Maxwell-Boltzmann start.
Inputs are seeded synthetic (no dataset exists for this path).

One step = one captured CUDA-graph replay of the full MD step (kick + drift,
device list decision, conditional build / prune, pair pass beside the mesh
transform, gather + scatter + kick).  Each timed step is bracketed by CUDA
events on the launching stream and preceded by an L2 flush (a 256 MiB write);
the timed region is bracketed by a barrier and device synchronisation, and the
max over ranks is reported.  With several GPUs every rank runs its own replica
(the system does not shard; no collective in the step).

--impl reference times the CPU restatement of the same step (the reference has
no CPU force path) on all host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "ns/day @64k-ion LJ+PME: learned-coarse vs plain, equal force error, 1 B200"
N_IONS = 64000
RHO = 0.0375
RC = 9.0
DT_FS = 1.0
T_INIT = 1200.0
BUFFER, PRUNE = 2.5, 0.7
E5_SPACING, E5_ORDER = 0.75, 6   # plain form at <= 1e-5 relative RMS force error against the Ewald sum
SEED = 2026
SELF_FORCE_TABLE = 16            # learned form: coarse-mesh self-force table size per axis


def ns_per_day(ms_per_step: float, dt_fs: float = DT_FS) -> float:
    return (1000.0 / ms_per_step) * dt_fs * 86400.0 * 1e-6


def make_system(pd, n_ions: int = N_IONS):
    L = (n_ions / RHO) ** (1.0 / 3.0)
    pos, q, box = pd.synthetic.ionic_melt(n_ions, L, 2.2, seed=SEED)
    m = pd.synthetic.melt_masses(q)
    v = pd.synthetic.maxwell_boltzmann(m, T_INIT, seed=SEED + 1, kB=pd.synthetic.KB_EV)
    return pos, q, m, v, box


def forces(pd, buffer=BUFFER, prune=PRUNE):
    lj = pd.LennardJones(epsilon=0.01, sigma=2.8, cutoff=RC, pairs="neighborlist",
                         neighborlist=pd.ClusterPairList(buffer=buffer, prune_buffer=prune))
    el = pd.PME(coulomb_prefactor=pd.synthetic.COULOMB_EV_A, real_cutoff=RC, real_space_tolerance=1e-5,
                mesh_spacing=1.0, order=5)
    return [lj, el]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms; the summary keeps the samples taken
    inside the timed region (the ``with`` block), which starts only once the sampler writes rows."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            import tempfile
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            deadline = time.time() + 15.0   # the first row shows that the sampler is running
            while time.time() < deadline and os.path.getsize(self.path) == 0 and self.proc.poll() is None:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        self.t0 = time.time()
        return self

    def __exit__(self, *a):
        self.t1 = time.time()
        if self.proc is not None:
            time.sleep(0.15)   # let the samples of the region's last moments be written
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        import datetime
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in open(self.path):
            p = [s.strip() for s in line.split(",")]
            if len(p) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(p[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(p[2]), float(p[3]), float(p[4]) if p[4] not in ("[N/A]", "") else 0.0,
                             p[6:10]))
            except ValueError:
                continue
        os.unlink(self.path)
        inside = [r for r in rows if self.t0 is not None and self.t0 - 0.025 <= r[0] <= self.t1 + 0.025]
        window = "timed region"
        if not inside:   # a region shorter than the sampling period: the samples nearest to it
            inside = sorted(rows, key=lambda r: abs(r[0] - 0.5 * (self.t0 + self.t1)))[:2]
            window = "nearest to the timed region"
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[k] for r in inside for k in range(4) if r[4][k].lower() == "active"})
        return {"sm_mhz": statistics.median(r[1] for r in inside), "sm_max_mhz": max(r[2] for r in inside),
                "power_w_max": max(r[3] for r in inside), "samples": len(inside), "window": window,
                "region_s": round(self.t1 - self.t0, 3), "reasons": reasons}


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, v: float) -> float:
    """The largest value over the ranks (NCCL on the GPUs; gloo on host tensors)."""
    if world <= 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cpu" if dist.get_backend() == "gloo" else "cuda"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def time_pairs_kernel(pd, st, reps=50):
    """Pair pass alone (same stream, warm): average launch time and the algorithmic work per launch."""
    import torch
    s = st.stream
    eng = st.cluster
    with torch.cuda.stream(s):
        for _ in range(3):
            eng.pairs(energy=False, stream=s)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for _ in range(reps):
            eng.pairs(energy=False, stream=s)
        b.record(s)
    b.synchronize()
    ms = a.elapsed_time(b) / reps
    # the timed passes accumulated into the slot forces: a first kick-free evaluation consumes (and clears)
    # them, a second one restores the forces of the current positions
    st.evaluate_forces_into_f(False)
    st.evaluate_forces_into_f(False)
    return ms


def pair_count(pos, box, rc):
    """Pairs inside r_c (Newton-3, counted once) from a cell grid on the host."""
    L = np.asarray(box, float)
    n = len(pos)
    nc = np.maximum((L // rc).astype(int), 3)
    cell = np.floor((pos / L + 0.5) % 1.0 * nc).astype(int) % nc
    cid = cell[:, 0] + nc[0] * (cell[:, 1] + nc[1] * cell[:, 2])
    order = np.argsort(cid, kind="stable")
    starts = np.searchsorted(cid[order], np.arange(nc.prod() + 1))
    total = 0
    for c in range(nc.prod()):
        ia = order[starts[c]:starts[c + 1]]
        if len(ia) == 0:
            continue
        cx, cy, cz = c % nc[0], (c // nc[0]) % nc[1], c // (nc[0] * nc[1])
        nb = []
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    cc = ((cx + dx) % nc[0]) + nc[0] * (((cy + dy) % nc[1]) + nc[1] * ((cz + dz) % nc[2]))
                    nb.append(order[starts[cc]:starts[cc + 1]])
        jb = np.concatenate(nb)
        d = pos[ia][:, None, :] - pos[jb][None, :, :]
        d -= L * np.round(d / L)
        r2 = (d * d).sum(-1)
        total += int(((r2 < rc * rc) & (r2 > 0)).sum())
    return total // 2


def cpu_baseline_run(pd, ora, steps_budget_s=15.0, max_steps=None):
    """The CPU restatement of the step (FP64, all host cores): ms per step on a bounded number of steps."""
    pos, q, m, v, box = make_system(pd)
    alpha = pd.splits.alpha_from_tolerance(RC, 1e-5)
    K = pd.splits.resolve_mesh(None, 1.0, box, 5)
    cpu = ora.CpuMelt(pos, v, q, m, box, C=pd.synthetic.COULOMB_EV_A, alpha=alpha, rc=RC, K=K, P=5,
                      lj=dict(sigma=2.8, eps=0.01, rc=RC), workers=-1)
    dt = DT_FS / pd.synthetic.TIME_UNIT_FS
    t0 = time.perf_counter()
    cpu.step(dt)   # warm-up step
    first = time.perf_counter() - t0
    nsteps = max(1, int(steps_budget_s / max(first, 1e-3)))
    if max_steps is not None:
        nsteps = max(1, min(nsteps, max_steps))
    t0 = time.perf_counter()
    for _ in range(nsteps):
        cpu.step(dt)
    el = time.perf_counter() - t0
    ms = 1000.0 * el / nsteps
    return ms, nsteps, os.cpu_count()


def run_ell_workload(pd, args, world, rank):
    """LJ fluid (fcc at rho 0.8442, T 0.72, r_c 2.5, skin 0.3, NVE dt 0.005) or 2D WCA disks (packing 0.7,
    eps 10, Langevin gamma 50, kT 1, dt 2e-4) on the ELL route; lists rebuilt at most every 10 steps.
    Prints atom-steps/s (a configuration run, not the headline metric)."""
    import torch
    if args.workload in ("lj1m", "lj4k"):
        ncell = 64 if args.workload == "lj1m" else 10
        pos, box = pd.synthetic.fcc_lattice(ncell, 0.8442, 0.05)
        m = np.ones(len(pos))
        v = pd.synthetic.maxwell_boltzmann(m, 0.72, seed=SEED)
        force = pd.LennardJones(epsilon=1.0, sigma=1.0, cutoff=2.5, pairs="neighborlist",
                                neighborlist=pd.CellList(buffer=0.3, capacity=96, rebuild_interval=10))
        methods, dt = [pd.ConstantVolume()], 0.005
        desc = f"3D LJ fluid N={len(pos)} rho=0.8442 r_c=2.5 skin 0.3, NVE dt=0.005"
    else:
        pos, box = pd.synthetic.hex_random_2d(1024, 0.7, 1.0, 0.25, seed=SEED)
        m = np.ones(len(pos))
        v = pd.synthetic.maxwell_boltzmann(m, 1.0, seed=SEED, dim=2)
        force = pd.WCA(epsilon=10.0, sigma=1.0, pairs="neighborlist",
                       neighborlist=pd.CellList(buffer=0.4, capacity=32, rebuild_interval=10))
        methods, dt = [pd.Langevin(gamma=50.0, kT=1.0)], 2e-4
        desc = f"2D WCA disks N={len(pos)} packing 0.7 eps 10, Langevin gamma 50 kT 1, dt=2e-4"
    system = pd.ParticleSystem(pos, box, masses=m, velocities=v)
    sim = pd.Simulation(system, pd.Integrator(dt=dt, forces=[force], methods=methods), seed=SEED)
    st = sim.state
    pd.evaluate_forces_into_f(sim)
    if args.profile:
        st.step(args.warmup, use_graph=False)
        st.step(args.steps, use_graph=False)
        st.synchronize()
        print(json.dumps({"profile": desc, "steps": args.steps, "list": st._ell_check()}))
        return
    st.step(args.warmup)
    st.synchronize()
    pre = st._ell_check()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    e0.record(st.stream)
    st.step(args.steps)
    e1.record(st.stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(world, e0.elapsed_time(e1)) / args.steps
    post = st._ell_check()
    if rank == 0:
        print(json.dumps({"metric": "atom-steps/s", "value": world * st.n * 1000.0 / ms, "unit": "atom-steps/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                          "higher_is_better": True, "dtype": "f32", "data": "synthetic",
                          "config": {"workload": desc, "route": "ELL (cell list rows)",
                                     "timed_builds": post["builds"] - pre["builds"], "lanes": post["lanes"],
                                     "cap": post["cap"], "l2": "not flushed"}}))


def pairs_within(pos, box, rc):
    """Pairs closer than rc (each counted once), periodic, from a k-d tree on the host."""
    from scipy.spatial import cKDTree
    L = np.asarray(box, float)
    p = np.asarray(pos, float) % L
    return int(len(cKDTree(p, boxsize=L).query_pairs(rc, output_type="ndarray")))


def load_peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        return {}


def fp32_peak_tflops(peaks):
    import torch
    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    return nsm * 128 * 2 * float(peaks.get("sm_max_mhz", 1965.0)) * 1e6 / 1e12


def ell_config(pd, name, steps, warmup, peaks):
    """One uncharged configuration on the ELL route, measured for the default bench line: atom-steps/s of
    the captured step, the row pair kernel against the FP32 rate (algorithmic work: pairs inside r_c,
    Newton-3 counted once, 20 flop per 3D LJ/WCA force pair, 16 in 2D) and the row build against HBM
    (algorithmic bytes: positions read, rows and counts written)."""
    import torch
    if name in ("lj4k", "lj1m"):
        ncell = 64 if name == "lj1m" else 10
        pos, box = pd.synthetic.fcc_lattice(ncell, 0.8442, 0.05)
        m = np.ones(len(pos))
        v = pd.synthetic.maxwell_boltzmann(m, 0.72, seed=SEED)
        force = pd.LennardJones(epsilon=1.0, sigma=1.0, cutoff=2.5, pairs="neighborlist",
                                neighborlist=pd.CellList(buffer=0.3, capacity=96, rebuild_interval=10))
        methods, dt, rc, fpair = [pd.ConstantVolume()], 0.005, 2.5, 20
        desc = f"3D LJ fluid N={len(pos)} rho=0.8442 T=0.72 r_c=2.5 skin 0.3, NVE dt=0.005"
    else:
        pos, box = pd.synthetic.hex_random_2d(1024, 0.7, 1.0, 0.25, seed=SEED)
        m = np.ones(len(pos))
        v = pd.synthetic.maxwell_boltzmann(m, 1.0, seed=SEED, dim=2)
        force = pd.WCA(epsilon=10.0, sigma=1.0, pairs="neighborlist",
                       neighborlist=pd.CellList(buffer=0.4, capacity=32, rebuild_interval=10))
        methods, dt, rc, fpair = [pd.Langevin(gamma=50.0, kT=1.0)], 2e-4, 2 ** (1 / 6), 16
        desc = f"2D WCA disks N={len(pos)} packing 0.7 eps 10, Langevin gamma 50 kT 1, dt=2e-4"
    sim = pd.Simulation(pd.ParticleSystem(pos, box, masses=m, velocities=v),
                        pd.Integrator(dt=dt, forces=[force], methods=methods), seed=SEED)
    st = sim.state
    pd.evaluate_forces_into_f(sim)
    st.step(warmup)
    st.synchronize()
    pre = st._ell_check()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st.stream)
    st.step(steps)
    e1.record(st.stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    post = st._ell_check()
    n = st.n
    # the row pair kernel alone and the row build alone (same stream, warm)
    ell, s = st.ell, st.stream
    xs = [t for t in (st.x, st.y, st.z) if t is not None]
    f = [torch.empty(n, device="cuda") for _ in range(len(xs))]
    pad = [None] * (3 - len(xs))
    reps = 20
    with torch.cuda.stream(s):
        for _ in range(3):
            ell.forces(*xs, *pad, *f, *pad, stream=s)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for _ in range(reps):
            ell.forces(*xs, *pad, *f, *pad, stream=s)
        b.record(s)
        b.synchronize()
        pair_ms = a.elapsed_time(b) / reps
        for _ in range(2):
            ell.request(stream=s)
            ell.update(*xs, *pad, stream=s)
        a.record(s)
        for _ in range(reps):
            ell.request(stream=s)
            ell.update(*xs, *pad, stream=s)
        b.record(s)
        b.synchronize()
        build_ms = a.elapsed_time(b) / reps
    entries = int(ell.counts_host().astype(np.int64).sum())
    P = st.positions()
    npairs = pairs_within(P if P.shape[1] == 3 else np.c_[P, np.zeros(len(P))],
                          box if len(box) == 3 else (box[0], box[1], 10.0), rc)
    fp32 = fp32_peak_tflops(peaks)
    achieved = npairs * fpair / (pair_ms * 1e-3) / 1e12
    dim = len(box)
    build_bytes = 4 * dim * n + 4 * entries + 4 * n
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    gbs = build_bytes / (build_ms * 1e-3) / 1e9
    return {"metric": "atom-steps/s", "value": n * 1000.0 / ms, "unit": "atom-steps/s", "ms_per_step": ms,
            "steps": steps, "warmup": warmup, "workload": desc, "route": "ELL (cell list rows)",
            "timed_builds": post["builds"] - pre["builds"], "lanes": post["lanes"], "cap": post["cap"],
            "l2": "warm (step graph replayed back to back)",
            "roofline": {"kernel": "row pair kernel (force only)", "bound": "fp32", "achieved": achieved,
                         "peak": fp32, "unit": "TFLOP/s", "frac": achieved / fp32, "per_launch_ms": pair_ms,
                         "pairs_within_rc": npairs, "flop_per_pair": fpair,
                         "peak_source": "nominal FP32 FMA rate at sm_max_mhz"},
            "row_build": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                          "per_build_ms": build_ms, "algorithmic_bytes": build_bytes,
                          "note": "positions read, row entries and counts written (cell binning not counted)",
                          "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback"}}


def batch_config(pd, steps, warmup, peaks, replicas=512):
    """The 512 LJ/WCA replicas as one batch (skin 0.45, lanes by the autotuner) for the default bench line:
    atom-steps/s of the captured batched step and the batched pair kernel against the FP32 rate."""
    import torch
    specs = pd.synthetic.replica_set(replicas, seed=SEED)
    systems = pd.batch.make_systems(specs)
    b = pd.batch.BatchedReplicas(systems, skin=0.45)
    b.evaluate()
    tune = b.autotune_lanes()
    b.step(warmup, 0.005)
    b.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(b.stream)
    b.step(steps, 0.005)
    e1.record(b.stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    if b.status()["error"]:
        raise RuntimeError(f"batch rows failed: {b.status()}")
    ntot = sum(sy["n"] for sy in systems)
    npairs = 0
    for k, sy in enumerate(systems):
        pos = np.stack([b.replica(k, t).double().cpu().numpy() for t in (b.x, b.y, b.z)], 1)
        npairs += pairs_within(pos, sy["box"], 2.5 if sy["kind"] == "lj" else 2 ** (1 / 6))
    pair_ms = tune["ms"][tune["lanes"]]
    fp32 = fp32_peak_tflops(peaks)
    achieved = npairs * 20 / (pair_ms * 1e-3) / 1e12
    return {"metric": "atom-steps/s", "value": ntot * 1000.0 / ms, "unit": "atom-steps/s", "ms_per_step": ms,
            "steps": steps, "warmup": warmup,
            "workload": f"{replicas} LJ/WCA 3D replicas (total {ntot}), skin 0.45, one launch per stage, NVE dt 0.005",
            "lanes": tune["lanes"], "l2": "warm",
            "roofline": {"kernel": "k_batch_pairs (force only)", "bound": "fp32", "achieved": achieved, "peak": fp32,
                         "unit": "TFLOP/s", "frac": achieved / fp32, "per_launch_ms": pair_ms,
                         "pairs_within_rc": npairs, "flop_per_pair": 20,
                         "peak_source": "nominal FP32 FMA rate at sm_max_mhz"}}


def profiled_traffic(name: str):
    """DRAM bytes per launch (read + write) of one ncu capture, from its committed summary."""
    import re
    try:
        txt = (ROOT / "profiles" / name).read_text()
    except OSError:
        return None
    m = re.search(r"dram bytes per launch \(read \+ write\) \| (\d+)", txt)
    return int(m.group(1)) if m else None


def time_md_steps(st, dt, steps, warmup, flush, no_flush):
    """Device time per captured NVE step (CUDA events on the step stream, L2 flushed between steps)."""
    import torch
    s = st.stream
    st.step(warmup, use_graph=True)
    st.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        for k in range(steps):
            if not no_flush:
                flush.fill_(float(k))
            starts[k].record(s)
            st.engine.step(1, dt, energy_last=False, use_graph=True, stream=s)
            ends[k].record(s)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in zip(starts, ends)) / steps


def run_learned_form(pd, args, st, system, dt, flush):
    """The learned coarse-mesh form on the same melt.

    Training data: ``args.snapshots`` snapshots of the running fine-mesh simulation ``st`` (one every
    ``args.snapshot_stride`` steps), target = fine-mesh minus coarse-mesh (2.0 A, order 4) forces; the radial
    weight is fitted by least squares, the network trained by Adam (fused tensor-core training kernel).  Held-out
    snapshots later in the run give the relative RMS electrostatic force error of each form against the FP64
    Ewald sum on the GPU.  Then the NVE step of coarse PME + correction (and of coarse PME alone) is timed like
    the plain step."""
    import torch
    n, box = st.n, st.box
    spec = st.solver.spec
    st.evaluate_forces_into_f(False)
    t0 = time.perf_counter()
    tr = pd.learned.CoarseMeshTrainer(n, box, st.q, st.typ, spec, coarse_spacing=2.0, coarse_order=4, seed=SEED,
                                      self_force_table=SELF_FORCE_TABLE)
    for _ in range(args.snapshots):
        st.step(args.snapshot_stride, use_graph=True)
        st.synchronize()
        tr.add_snapshot(st.x, st.y, st.z)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t0
    t0 = time.perf_counter()
    coef = tr.fit_radial()
    tr.build_dataset()
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    losses = tr.train(epochs=args.epochs, lr=2e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    # held-out snapshots: relative RMS electrostatic force error vs the FP64 Ewald sum
    ones = pd.learned.MLPNetwork(pd.learned.init_params(0, s0=1.0, out_scale=0.0))
    q = st.q.double()
    # the plain form on a mesh fine enough for 1e-5 relative RMS force error against the Ewald sum
    spec_e5 = pd.ElectrostaticsSpec(coulomb_prefactor=spec.coulomb_prefactor, real_cutoff=spec.real_cutoff,
                                    alpha=spec.alpha, order=E5_ORDER, mesh_spacing=E5_SPACING)
    solver_e5 = pd.ElectrostaticsSolver(spec_e5, box, st.q.double().cpu().numpy(), nmax=n)
    raw = pd.ElectrostaticsSolver(tr.coarse_spec, box, st.q.double().cpu().numpy(), nmax=n)   # self force kept
    # the configuration's PPPM variant: ik differentiation, alias order 2, same mesh and order as the SPME
    spec_ik = pd.ElectrostaticsSpec(coulomb_prefactor=spec.coulomb_prefactor, real_cutoff=spec.real_cutoff,
                                    alpha=spec.alpha, influence="p3m_ik", order=5, mesh_spacing=1.0, alias_order=2)
    solver_ik = pd.ElectrostaticsSolver(spec_ik, box, st.q.double().cpu().numpy(), nmax=n)
    errs = {"plain_fine": [], "plain_pppm_ik": [], "plain_e5": [], "coarse": [], "coarse_self": [], "coarse_radial": [], "learned": [],
            "ceiling_per_ion_scalar": []}
    held = []   # (positions, reciprocal Ewald force, RMS of the full Ewald force) per held-out snapshot
    for _ in range(args.heldout):
        st.step(100, use_graph=True)
        st.synchronize()
        x, y, z = st.x, st.y, st.z
        rq = torch.stack([x.double(), y.double(), z.double(), q], 1).contiguous()
        Fk, _ = pd.learned.ewald_oracle(rq, box, spec.C, spec.alpha, digits=10, parts=2)
        Ft, _ = pd.learned.ewald_oracle(rq, box, spec.C, spec.alpha, digits=10, parts=3)
        den = torch.sqrt((Ft ** 2).sum())
        held.append(((x.clone(), y.clone(), z.clone()), Fk, den, Ft))
        fine = tr.mesh_forces(tr.fine, x, y, z).double()
        coarse = tr.mesh_forces(tr.coarse, x, y, z).double()
        V = tr.corr.correction(ones, x, y, z, tr.q, tr.typ)[:, :3].double()
        # the best any per-ion scalar s_i on the radial vector V_i can do: least squares per ion,
        # s_i* = R_i . V_i / |V_i|^2 with R_i the exact residual of the self-force-free coarse mesh
        R = Fk - coarse
        s_star = (R * V).sum(1) / (V * V).sum(1).clamp_min(1e-300)
        forms = {"plain_fine": fine, "plain_pppm_ik": tr.mesh_forces(solver_ik, x, y, z).double(),
                 "plain_e5": tr.mesh_forces(solver_e5, x, y, z).double(),
                 "coarse": tr.mesh_forces(raw, x, y, z).double(), "coarse_self": coarse,
                 "coarse_radial": coarse + V,
                 "learned": coarse + tr.corr.correction(tr.net, x, y, z, tr.q, tr.typ)[:, :3].double(),
                 "ceiling_per_ion_scalar": coarse + s_star[:, None] * V}
        for k, f in forms.items():
            errs[k].append(float(torch.sqrt(((f - Fk) ** 2).sum()) / den))
    err = {k: float(np.mean(v)) for k, v in errs.items()}
    # the timed learned step, from the current state of the fine-mesh run
    el = pd.PME(coulomb_prefactor=pd.synthetic.COULOMB_EV_A, real_cutoff=RC, real_space_tolerance=1e-5,
                mesh_spacing=2.0, order=4)
    sys2 = pd.ParticleSystem(st.positions(), box, types=system.types, typeids=system.typeids, masses=system.masses,
                             charges=system.charges, velocities=st.velocities())
    forces2 = forces(pd, args.buffer, args.prune)[:1] + [el]
    st2 = pd.Simulation(sys2, pd.Integrator(dt=dt, forces=forces2)).state
    st2.evaluate_forces_into_f(False)
    ms_coarse = time_md_steps(st2, dt, args.steps, args.warmup, flush, args.no_flush)
    st2.solver.set_self_force_removal(SELF_FORCE_TABLE)
    st2.engine.set_learned(tr.corr, None)   # the radial term alone: the learned form's lower bound in time
    st2.evaluate_forces_into_f(False)
    ms_radial = time_md_steps(st2, dt, args.steps, args.warmup, flush, args.no_flush)
    st2.engine.set_learned(tr.corr, tr.net)
    st2.evaluate_forces_into_f(False)
    ms_learned = time_md_steps(st2, dt, args.steps, args.warmup, flush, args.no_flush)
    el5 = pd.PME(coulomb_prefactor=pd.synthetic.COULOMB_EV_A, real_cutoff=RC, real_space_tolerance=1e-5,
                 mesh_spacing=E5_SPACING, order=E5_ORDER)
    st3 = pd.Simulation(sys2, pd.Integrator(dt=dt, forces=forces(pd, args.buffer, args.prune)[:1] + [el5])).state
    st3.evaluate_forces_into_f(False)
    ms_e5 = time_md_steps(st3, dt, args.steps, args.warmup, flush, args.no_flush)
    lst = tr.corr.status()
    if tr.net.error() or lst["error"]:
        raise RuntimeError(f"learned correction failed during the timed run (network {tr.net.error()}, rows {lst})")
    # the metric as stated: the cheapest plain mesh setting whose error is at or below the learned form's
    equal = equal_error_comparison(pd, args, tr, spec, box, sys2, dt, flush, held, err["learned"], ms_learned,
                                   ms_coarse)
    ms_ik, mesh_ik = plain_step_ms(pd, args, sys2, dt, flush, "p3m_ik", 1.0, 5)
    # ESP at the 1e-5 rules (width 8, spacing pi r_c / c): the reference's cheapest form at that accuracy
    e_esp, mesh_esp, sp_esp = esp_error(pd, held, box, st.q.double().cpu().numpy(), dt, 1e-5)
    ms_esp = esp_step_ms(pd, args, sys2, dt, flush, 1e-5)
    return {"ms_per_step": ms_learned, "value": ns_per_day(ms_learned),
            "learned_vs_plain_equal_error": equal,
            "esp_at_1e-5": {"ms_per_step": ms_esp, "value": ns_per_day(ms_esp), "unit": "ns/day",
                            "mesh": f"ESP tolerance 1e-5: {'x'.join(str(k) for k in mesh_esp)}, width {sp_esp.order}, "
                                    f"spacing {sp_esp.mesh_spacing:.3f} A, split shape {sp_esp.split_shape:.3f}, "
                                    f"window shape {sp_esp.window_shape:.3f}",
                            "force_error_vs_fp64_ewald": e_esp,
                            "error_note": "total Coulomb force (prolate real space + mesh) against the full FP64 "
                                          "Ewald force, over its RMS"},
            "pppm_ik": {"ms_per_step": ms_ik, "value": ns_per_day(ms_ik), "unit": "ns/day",
                        "mesh": f"P3M-ik 1.0 A ({'x'.join(str(k) for k in mesh_ik)}), order 5, alias order 2 "
                                "(the configuration's PPPM variant)",
                        "force_error_vs_fp64_ewald": err["plain_pppm_ik"]},
            "coarse_only": {"ms_per_step": ms_coarse, "value": ns_per_day(ms_coarse)},
            "coarse_radial_no_network": {"ms_per_step": ms_radial, "value": ns_per_day(ms_radial),
                                         "note": "coarse mesh, self force removed, fitted radial term (s = 1): "
                                                 "descriptors and rows without the network"},
            "plain_e5": {"ms_per_step": ms_e5, "value": ns_per_day(ms_e5),
                         "mesh": f"SPME {E5_SPACING} A ({'x'.join(str(k) for k in solver_e5.mesh)}), order {E5_ORDER}"},
            "force_error_vs_fp64_ewald": err,
            "error_note": "relative RMS electrostatic force error (mesh part of each form against the FP64 "
                          "reciprocal Ewald sum, over the RMS of the full Ewald force; the real-space part is "
                          "common to all forms)",
            "mesh": "coarse PME 2.0 A (60^3), order 4; fine 1.0 A (120^3), order 5",
            "forms_note": "coarse: the coarse mesh alone (also the timed coarse_only step); coarse_self: its "
                          "self force removed (table %d^3); coarse_radial: plus the fitted radial term (s = 1); "
                          "learned: plus the trained network (the timed learned step)" % SELF_FORCE_TABLE,
            "training": {"snapshots": args.snapshots, "stride_steps": args.snapshot_stride, "epochs": args.epochs,
                         "mse_per_epoch": losses, "radial_coef": [float(c) for c in coef],
                         "seconds": {"snapshots": t_gen, "dataset": t_data, "adam": t_train},
                         "heldout_snapshots": args.heldout},
            "descriptor_rows": {"builds": lst["builds"], "cap": lst["cap"]}}


PLAIN_SWEEP = {"kinds": ("spme", "p3m_ad", "p3m_ik"), "spacings": (2.5, 2.25, 2.0, 1.75, 1.5, 1.25, 1.0),
               "orders": (3, 4, 5, 6)}


def mesh_error(pd, tr, solver, held):
    """Mean relative RMS force error of a mesh solver's forces against the reciprocal FP64 Ewald sum on the
    held-out snapshots (over the RMS of the full Ewald force)."""
    import torch
    e = []
    for (x, y, z), Fk, den, _ in held:
        f = tr.mesh_forces(solver, x, y, z).double()
        e.append(float(torch.sqrt(((f - Fk) ** 2).sum()) / den))
    return float(np.mean(e))


ESP_TOLERANCES = (3e-3, 1e-3, 1e-4)   # ESP settings of the equal-error sweep (workflow rules per tolerance; the
#                                      rules give no valid window above about 3e-3)


def esp_error(pd, held, box, q64, dt, tol):
    """Mean relative RMS error of the ESP solver's total Coulomb force (prolate real space + mesh) against
    the full FP64 Ewald force on the held-out snapshots (the prolate split differs from the Gaussian one, so
    the comparison is of total forces).  Returns (error, mesh dims)."""
    import torch
    el = pd.ESP(coulomb_prefactor=pd.synthetic.COULOMB_EV_A, real_cutoff=RC, tolerance=tol)
    st = None
    e = []
    for (x, y, z), _, den, Ft in held:
        if st is None:
            pos = torch.stack([x, y, z], 1).double().cpu().numpy()
            system = pd.ParticleSystem(pos, box, charges=q64, masses=np.ones(len(q64)))
            st = pd.Simulation(system, pd.Integrator(dt=dt, forces=[el])).state
        else:
            st.x.copy_(x)
            st.y.copy_(y)
            st.z.copy_(z)
            torch.cuda.synchronize()
        st.evaluate_forces_into_f(False)
        F = torch.stack([st.fx, st.fy, st.fz], 1).double()
        e.append(float(torch.sqrt(((F - Ft) ** 2).sum()) / den))
    return float(np.mean(e)), st.solver.mesh, st.solver.spec


def esp_step_ms(pd, args, sys2, dt, flush, tol):
    """Device time of the captured NVE step of the melt with LJ + ESP at a tolerance."""
    el = pd.ESP(coulomb_prefactor=pd.synthetic.COULOMB_EV_A, real_cutoff=RC, tolerance=tol)
    st = pd.Simulation(sys2, pd.Integrator(dt=dt, forces=forces(pd, args.buffer, args.prune)[:1] + [el])).state
    st.evaluate_forces_into_f(False)
    return time_md_steps(st, dt, min(args.steps, 40), args.warmup, flush, args.no_flush)


def plain_step_ms(pd, args, sys2, dt, flush, kind, spacing, order):
    """Device time of the captured NVE step of the melt with a plain mesh setting (LJ + real space + mesh)."""
    kw = dict(coulomb_prefactor=pd.synthetic.COULOMB_EV_A, real_cutoff=RC, real_space_tolerance=1e-5,
              mesh_spacing=spacing, order=order)
    el = pd.PME(**kw) if kind == "spme" else pd.PPPM(differentiation="ad" if kind == "p3m_ad" else "ik",
                                                      alias_order=2, **kw)
    st = pd.Simulation(sys2, pd.Integrator(dt=dt, forces=forces(pd, args.buffer, args.prune)[:1] + [el])).state
    st.evaluate_forces_into_f(False)
    return time_md_steps(st, dt, min(args.steps, 40), args.warmup, flush, args.no_flush), st.solver.mesh


def equal_error_comparison(pd, args, tr, spec, box, sys2, dt, flush, held, target, ms_learned, ms_coarse):
    """The headline metric as stated: learned coarse-mesh form against the cheapest plain form at equal force
    error.  Every plain setting of the sweep (SPME, P3M-AD, P3M-ik over mesh spacing and order, same split)
    has its held-out error measured; at each kind and order the coarsest spacing at or below the learned
    form's error is timed as a full NVE step, and the fastest of those is the plain side.  Also reported: the
    step-time ceiling of the learned form (a free, perfect correction: plain_ms / coarse_only_ms)."""
    n = tr.n
    q64 = tr.q.double().cpu().numpy()
    sweep = []
    for kind in PLAIN_SWEEP["kinds"]:
        for order in PLAIN_SWEEP["orders"]:
            for h in PLAIN_SWEEP["spacings"]:   # coarsest first
                sp = pd.ElectrostaticsSpec(coulomb_prefactor=spec.coulomb_prefactor, real_cutoff=spec.real_cutoff,
                                           alpha=spec.alpha, influence=kind, order=order, mesh_spacing=h,
                                           alias_order=2)
                solver = pd.ElectrostaticsSolver(sp, box, q64, nmax=n)
                e = mesh_error(pd, tr, solver, held)
                sweep.append({"kind": kind, "spacing": h, "order": order,
                              "mesh": "x".join(str(k) for k in solver.mesh), "error": e})
                solver.close()
                if e <= target:
                    break
    for tol in ESP_TOLERANCES:   # coarsest first
        e, mesh, sp = esp_error(pd, held, box, q64, dt, tol)
        sweep.append({"kind": "esp", "tolerance": tol, "spacing": round(sp.mesh_spacing, 4), "order": sp.order,
                      "mesh": "x".join(str(k) for k in mesh), "error": e,
                      "error_note": "total Coulomb force against the full Ewald force"})
        if e <= target:
            break
    timed = []
    for c in sweep:
        if c["error"] <= target:
            if c["kind"] == "esp":
                ms = esp_step_ms(pd, args, sys2, dt, flush, c["tolerance"])
            else:
                ms, _ = plain_step_ms(pd, args, sys2, dt, flush, c["kind"], c["spacing"], c["order"])
            c["ms_per_step"] = ms
            timed.append(c)
    best = min(timed, key=lambda c: c["ms_per_step"]) if timed else None
    out = {"error": target, "learned_ms": ms_learned, "coarse_only_ms": ms_coarse,
           "sweep": sweep, "note": "errors: mesh part against the FP64 reciprocal Ewald sum on the held-out "
                                   "snapshots; each timed setting is the coarsest spacing of its kind and "
                                   "order at or below the learned form's error"}
    if best is not None:
        out.update(plain_setting=f"{best['kind']} {best['spacing']} A ({best['mesh']}), order {best['order']}",
                   plain_error=best["error"], plain_ms=best["ms_per_step"],
                   ratio=best["ms_per_step"] / ms_learned,
                   ratio_note="plain_ms / learned_ms: above 1 the learned form is faster at equal error",
                   step_time_ceiling=best["ms_per_step"] / ms_coarse)
    return out


def profile_learned(pd, args, system, box, dt):
    """Profiling run of the learned form (no timing): coarse PME (2.0 A, order 4) with the correction attached,
    --warmup then --steps directly launched steps, each followed by one fused training batch and an Adam step
    over that step's descriptors, so that a launch list or a capture sees every learned-form kernel."""
    import torch
    el = pd.PME(coulomb_prefactor=pd.synthetic.COULOMB_EV_A, real_cutoff=RC, real_space_tolerance=1e-5,
                mesh_spacing=2.0, order=4)
    st = pd.Simulation(system, pd.Integrator(dt=dt, forces=forces(pd, args.buffer, args.prune)[:1] + [el])).state
    st.solver.set_self_force_removal(SELF_FORCE_TABLE)
    lc = pd.learned.LearnedCorrection(st.n, box)
    lc.set_radial(np.linspace(0.01, -0.02, lc.nb))
    net = pd.learned.MLPNetwork(pd.learned.init_params(SEED, s0=1.0, out_scale=0.1))
    st.engine.set_learned(lc, net)
    st.evaluate_forces_into_f(False)
    ab = torch.stack([torch.rand(st.n, device="cuda"), torch.randn(st.n, device="cuda")], 1).contiguous()
    X = torch.empty((st.n, 32), dtype=torch.bfloat16, device="cuda")
    for k in range(args.warmup + args.steps):
        st.step(1, use_graph=False)
        st.synchronize()
        lc.descriptors(st.x, st.y, st.z, st.q, st.typ, X=X)
        net.train_batch(X, ab, 2.0 / (3 * st.n))
        net.adam(1e-4)
    torch.cuda.synchronize()
    print(json.dumps({"profile": "melt64k learned-form eager steps + training batches", "steps": args.steps,
                      "warmup": args.warmup, "rows": lc.status(), "network_error": net.error()}))


def run_batch_workload(pd, args, world, rank):
    """512 independent 3D LJ / WCA replicas (N log-uniform in [500, 20 000], density 0.70-0.90, T 0.6-1.2,
    r_c 2.5 (LJ) or 2^(1/6) (WCA), NVE dt 0.005) as one batch: one launch per stage over all
    replicas, the step captured into one CUDA graph, lanes per row chosen by the autotuner.  Reported:
    aggregate atom-steps/s of the batch and of the loop of single-system ELL engines (one captured step per
    replica, launched one after another on one stream)."""
    import torch
    # one set of replicas for the whole job, split across the ranks by cost (no collective in the step)
    all_specs = pd.synthetic.replica_set(args.replicas, seed=SEED)
    mine = pd.batch.partition_by_cost(all_specs, world)[rank]
    specs = [all_specs[k] for k in mine]
    systems = pd.batch.make_systems(specs)
    ntot = sum(s["n"] for s in systems)
    dt = 0.005
    if args.profile:
        b = pd.batch.BatchedReplicas(systems, skin=0.3)
        b.evaluate()
        b.step(args.warmup, dt, use_graph=False)
        b.step(args.steps, dt, use_graph=False)
        b.synchronize()
        if rank == 0:
            print(json.dumps({"profile": "batch512 eager steps", "steps": args.steps, "rows": b.status()}))
        return
    # autotuner: list skin (rows longer vs rebuilt less often) and lanes per row, each candidate timed on
    # a short run of this batch
    trials = {}
    for skin in (0.3, 0.45, 0.6):
        bt = pd.batch.BatchedReplicas(systems, skin=skin)
        bt.evaluate()
        lanes = bt.autotune_lanes()
        bt.step(5, dt)
        bt.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(bt.stream)
        bt.step(30, dt)
        a1.record(bt.stream)
        a1.synchronize()
        trials[skin] = (a0.elapsed_time(a1) / 30, lanes["lanes"])
        bt.close()
        del bt
        torch.cuda.empty_cache()
    best_skin = min(trials, key=lambda k: trials[k][0])
    b = pd.batch.BatchedReplicas(systems, skin=best_skin, lanes=trials[best_skin][1])
    b.evaluate()
    tune = {"skin": best_skin, "lanes": b.lanes,
            "trials_ms": {f"skin {k}, lanes {v[1]}": v[0] for k, v in trials.items()}}
    b.step(args.warmup, dt)
    b.synchronize()
    pre = b.status()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        e0.record(b.stream)
        b.step(args.steps, dt)
        e1.record(b.stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(world, e0.elapsed_time(e1) / args.steps)
    post = b.status()
    if post["error"]:
        raise RuntimeError(f"batch rows failed: {post}")
    # the loop of single-system engines on the same replicas
    loop_steps = max(3, min(args.steps, 20))
    engines = []
    s = torch.cuda.Stream()
    for sy in systems:
        kw = dict(model="lj", cutoff=2.5) if sy["kind"] == "lj" else dict(model="wca")
        eng = pd.ELLEngine(sy["n"], sy["box"], skin=best_skin, capacity=int(b.cap), interval=100, lanes=b.lanes,
                           **kw)
        f32 = dict(dtype=torch.float32, device="cuda")
        state = {k: torch.tensor(sy["positions"][:, d], **f32) for d, k in enumerate("xyz")}
        state.update({k: torch.tensor(sy["velocities"][:, d], **f32) for d, k in enumerate(("vx", "vy", "vz"))})
        state.update({k: torch.zeros(sy["n"], **f32) for k in ("fx", "fy", "fz", "epot")})
        state["vir"] = torch.zeros((sy["n"], 6), **f32)
        state["inv_mass"] = 1.0
        md = pd.ELLDeviceEngine(eng, state)
        md.evaluate(stream=s)
        engines.append((eng, md))
    for _, md in engines:
        md.step(args.warmup, dt, stream=s)
    torch.cuda.synchronize()
    l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0.record(s)
    for _ in range(loop_steps):
        for _, md in engines:
            md.step(1, dt, stream=s)
    l1.record(s)
    torch.cuda.synchronize()
    loop_ms = l0.elapsed_time(l1) / loop_steps
    job_atoms = sum(s["n"] for s in all_specs)
    if rank == 0:
        print(json.dumps({"metric": "atom-steps/s", "value": job_atoms * 1000.0 / ms, "unit": "atom-steps/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                          "higher_is_better": True, "scaling": "strong", "dtype": "f32", "data": "synthetic",
                          "config": {"workload": f"{args.replicas} LJ/WCA 3D replicas, N log-uniform [500, 20000] "
                                                 f"(total {job_atoms}), rho 0.70-0.90, T 0.6-1.2, r_c 2.5 / 2^(1/6), "
                                                 f"skin {best_skin} (tuned), NVE dt 0.005, one launch per stage over "
                                                 "all replicas",
                                     "parallelism": f"replicas split by cost over {world} GPUs",
                                     "rank0_replicas": len(specs), "rank0_atoms": ntot,
                                     "l2": "warm (batch working set per rank)"},
                          "autotune": tune, "rebuilds_timed": post["builds"] - pre["builds"],
                          "loop_of_single_systems": {"value": world * ntot * 1000.0 / loop_ms, "ms_per_step": loop_ms,
                                                     "steps": loop_steps, "note": "rank 0's replicas x ranks"},
                          "clocks": clk.summary()}))


def melts_sizes(nmelts: int, rank: int = 0):
    """Sizes of the batched charged melts: N log-uniform in [2 000, 32 000], even (half +1, half -1)."""
    import __graft_entry__ as ge
    return ge.load_package().batch.melt_sizes(nmelts, SEED + 64 + rank)


def melts_measure(pd, ns, steps, warmup, skin, buffer, prune, world=1, compare=True, shape=None):
    """The charged melts as one batch (one launch per force stage, the step one captured graph, lanes per row
    and spread tile by the autotuner), and, with ``compare``, each melt's own captured single-system step
    replayed concurrently on 16 streams and one after another.  Returns the result dict (ms per step,
    atom-steps/s)."""
    import torch
    dt = DT_FS / pd.synthetic.TIME_UNIT_FS
    total = sum(ns)
    systems = pd.batch.melt_systems(ns, rho=RHO, T=T_INIT, seed=SEED)
    alpha = pd.splits.alpha_from_tolerance(RC, 1e-5)
    el = dict(alpha=alpha, C=pd.synthetic.COULOMB_EV_A, rc=RC, order=5, kind="spme", spacing=1.0)
    if shape is None:
        # autotuner: row-list skin (longer rows against fewer partial rebuilds), then lanes per row x spread
        # tile on whole captured steps of the batch itself
        trials = {}
        for sk in ((skin,) if skin is not None else (0.8, 1.2, 1.6)):
            bt = pd.batch.BatchedReplicas(systems, skin=sk, electrostatics=el)
            bt.evaluate()
            tb = bt.autotune(dt)
            trials[sk] = (min(tb["ms"].values()), tb)
            bt.close()
            del bt
            torch.cuda.empty_cache()
        skin = min(trials, key=lambda k: trials[k][0])
        tuned = dict(trials[skin][1], skin=skin, skin_trials_ms={str(k): v[0] for k, v in trials.items()})
        batch = pd.batch.BatchedReplicas(systems, skin=skin, electrostatics=el)
        batch.evaluate()
        batch.set_lanes(tuned["lanes"])
        batch.set_spread_tile(*tuned["spread_tile"])
    else:   # a fixed (lanes per row, spread tile), e.g. the autotuner's earlier choice for a launch list
        skin = 1.0 if skin is None else skin
        batch = pd.batch.BatchedReplicas(systems, skin=skin, electrostatics=el)
        batch.evaluate()
        batch.set_lanes(shape[0])
        batch.set_spread_tile(*shape[1:])
        tuned = {"lanes": shape[0], "spread_tile": list(shape[1:]), "skin": skin, "fixed": True}
    batch.step(warmup, dt)
    torch.cuda.synchronize()
    s0 = batch.stream
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(s0)
    batch.step(steps, dt)
    t1.record(s0)
    torch.cuda.synchronize()
    st = batch.status()
    if st["error"]:
        raise RuntimeError(f"batched melts: list error {st['error']}")
    ms_batch = max_over_ranks(world, t0.elapsed_time(t1) / steps)
    info = batch.mesh_info()
    out = {"metric": "atom-steps/s", "value": world * total * 1000.0 / ms_batch, "unit": "atom-steps/s",
           "ms_per_step": ms_batch, "steps": steps, "warmup": warmup,
           "workload": f"{len(ns)} charged melts, N log-uniform [2000, 32000] (total {total}), 0.0375 A^-3, "
                       f"LJ + SPME 1 A order 5, NVE 1 fs",
           "path": "batched: one launch per force stage, one captured graph per step",
           "skin": skin, "fft_plans": info["groups"], "mesh_nodes": info["nodes"], "list_builds": st["builds"],
           "autotune": tuned, "l2": "inputs larger than L2 (rows and grids)"}
    del batch
    torch.cuda.empty_cache()
    if not compare:
        return out
    states = []
    for sysd in systems:
        system = pd.ParticleSystem(sysd["positions"], sysd["box"], types=["Na", "Cl"],
                                   typeids=np.where(sysd["charges"] > 0, 1, 2), masses=sysd["masses"],
                                   charges=sysd["charges"], velocities=sysd["velocities"])
        sst = pd.Simulation(system, pd.Integrator(dt=dt, forces=forces(pd, buffer, prune))).state
        sst.evaluate_forces_into_f(False)
        states.append(sst)
    nstream = 16
    streams = [torch.cuda.Stream() for _ in range(nstream)]

    def replay(nsteps, concurrent):
        # system k always replays on stream k % 16 (its captured graph is bound to that stream); the
        # sequential replay chains the systems with events, the concurrent one lets them overlap
        prev = None
        for _ in range(nsteps):
            for k, sst in enumerate(states):
                s = streams[k % nstream]
                if not concurrent and prev is not None:
                    s.wait_event(prev)
                sst.engine.step(1, dt, energy_last=False, use_graph=True, stream=s)
                if not concurrent:
                    prev = torch.cuda.Event()
                    prev.record(s)

    replay(warmup, True)
    torch.cuda.synchronize()
    for conc in (False, True):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(streams[0])
        for s in streams[1:]:
            s.wait_event(a)
        replay(steps, conc)
        for s in streams[1:]:
            ev = torch.cuda.Event()
            ev.record(s)
            streams[0].wait_event(ev)
        b.record(streams[0])
        torch.cuda.synchronize()
        ms = max_over_ranks(world, a.elapsed_time(b) / steps)
        key = "concurrent_replay" if conc else "sequential_replay"
        out[key] = {"ms_per_step": ms, "value": world * total * 1000.0 / ms,
                    "path": ("each melt's captured single-system step, 16 streams" if conc
                             else "each melt's captured single-system step, one after another")}
    for sst in states:
        if sst.cluster.statistics()["error"]:
            raise RuntimeError("cluster list error during the melts run")
    out["batched_vs_sequential"] = out["sequential_replay"]["ms_per_step"] / ms_batch
    out["batched_vs_concurrent"] = out["concurrent_replay"]["ms_per_step"] / ms_batch
    return out


def run_melts_workload(pd, args, world, rank):
    """64 independent charged melts (the 64 000-ion melt's density, LJ and SPME settings, 1 A mesh, order 5)
    as one batch, against each melt's own captured step replayed concurrently and one after another."""
    ns = melts_sizes(args.melts, rank)
    shape = None if args.melt_shape is None else tuple(int(v) for v in args.melt_shape.split("x"))
    if args.profile:
        # eager steps (no graph) so that a profiler sees every launch: set-up, one force evaluation with its
        # full build, then warm-up and timed steps of the same batch and shape
        import torch
        shape = (1, 64) if shape is None else shape
        systems = pd.batch.melt_systems(ns, rho=RHO, T=T_INIT, seed=SEED)
        el = dict(alpha=pd.splits.alpha_from_tolerance(RC, 1e-5), C=pd.synthetic.COULOMB_EV_A, rc=RC, order=5,
                  kind="spme", spacing=1.0)
        b = pd.batch.BatchedReplicas(systems, skin=1.2 if args.melt_skin is None else args.melt_skin,
                                     lanes=shape[0], electrostatics=el)
        b.set_spread_tile(*shape[1:])
        b.evaluate()
        dt = DT_FS / pd.synthetic.TIME_UNIT_FS
        b.step(args.warmup, dt, use_graph=False)
        b.step(args.steps, dt, use_graph=False)
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"profile": "melts64 eager steps", "steps": args.steps, "shape": shape,
                              "rows": b.status(), "mesh": b.mesh_info()}))
        return
    res = melts_measure(pd, ns, args.steps, args.warmup, args.melt_skin, args.buffer, args.prune, world=world,
                        compare=not args.no_compare, shape=shape)
    if rank == 0:
        line = {"metric": res.pop("metric"), "value": res.pop("value"), "unit": res.pop("unit"), "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res.pop("ms_per_step"),
                "higher_is_better": True, "scaling": "weak", "dtype": "f32", "data": "synthetic",
                "config": {"workload": res.pop("workload"), "parallelism": f"replicas x{world}"}}
        line.update(res)
        print(json.dumps(line))


def run_reference(args, world, rank):
    """--impl reference: the CPU restatement on the host cores (rank 0 only)."""
    if rank != 0:
        return
    import __graft_entry__ as ge
    pd = ge.load_package()
    ora = ge.load_oracle()
    budget = 120.0
    pos, q, m, v, box = make_system(pd)
    alpha = pd.splits.alpha_from_tolerance(RC, 1e-5)
    K = pd.splits.resolve_mesh(None, 1.0, box, 5)
    cpu = ora.CpuMelt(pos, v, q, m, box, C=pd.synthetic.COULOMB_EV_A, alpha=alpha, rc=RC, K=K, P=5,
                      lj=dict(sigma=2.8, eps=0.01, rc=RC), workers=-1)
    dt = DT_FS / pd.synthetic.TIME_UNIT_FS
    t0 = time.perf_counter()
    for _ in range(max(1, min(args.warmup, 2))):
        cpu.step(dt)
    per = (time.perf_counter() - t0) / max(1, min(args.warmup, 2))
    steps = max(1, min(args.steps, int(budget / max(per, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(steps):
        cpu.step(dt)
    ms = 1000.0 * (time.perf_counter() - t0) / steps
    val = ns_per_day(ms)
    cores = os.cpu_count()
    out = {"impl": "reference", "metric": METRIC, "value": val, "unit": "ns/day", "n_gpus": args.gpus,
           "steps": steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded ionic melt)",
           "config": {"workload": "ionic melt N=64000 LJ+SPME 120^3 order 5, NVE dt=1 fs", "form": "plain"},
           "cpu_baseline": {"value": val, "unit": "ns/day", "cores": cores, "kind": "port",
                            "sample": f"{steps} full MD steps of the 64k-ion melt on the CPU restatement "
                                      f"(requested {args.steps}; capped to ~{int(budget)} s)"},
           "e2e": {"value": val, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="pdb200", choices=["pdb200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-flush", action="store_true", help="(diagnostic) do not flush L2 between steps")
    ap.add_argument("--buffer", type=float, default=BUFFER, help="cluster list buffer (Angstrom)")
    ap.add_argument("--prune", type=float, default=PRUNE, help="prune buffer (Angstrom)")
    ap.add_argument("--replicas", type=int, default=512, help="replicas of the batch512 workload")
    ap.add_argument("--melts", type=int, default=64, help="charged melts of the melts64 workload")
    ap.add_argument("--melt-skin", type=float, default=None,
                    help="row-list skin of the batched melts (Angstrom); default: the autotuner's choice")
    ap.add_argument("--melt-shape", default=None,
                    help="melts64: lanes per row x ions per spread tile [x threads per ion], e.g. 1x64x4, "
                         "instead of the autotuner's choice")
    ap.add_argument("--no-compare", action="store_true",
                    help="melts64: time the batched path only (no single-system replays), e.g. for a launch list")
    ap.add_argument("--workload", default="melt64k",
                    choices=["melt64k", "melt512k", "lj1m", "wca2d1m", "lj4k", "batch512", "melts64"],
                    help="melt64k: the headline run; melt512k: the same forms at 512 000 ions (L = 239 A); lj4k / "
                         "lj1m (3D LJ fluid, ELL route, NVE) and wca2d1m (2D WCA disks, ELL route, Langevin) and "
                         "batch512 (batched replicas) time the other configurations (not the headline metric)")
    ap.add_argument("--snapshots", type=int, default=2000, help="training snapshots of the learned form")
    ap.add_argument("--snapshot-stride", type=int, default=2, help="fine-mesh steps between training snapshots")
    ap.add_argument("--epochs", type=int, default=4, help="Adam epochs of the learned form")
    ap.add_argument("--heldout", type=int, default=4, help="held-out snapshots for the force errors")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned coarse-mesh form")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the short runs of the other configurations (LJ 4k / 1M, 2D WCA 1M, 512 replicas)")
    ap.add_argument("--form", default="plain", choices=["plain", "learned"],
                    help="with --profile: profile the plain step or the learned coarse-mesh step")
    ap.add_argument("--profile", action="store_true",
                    help="profiling run for ncu: the same workload, --warmup then --steps directly launched steps "
                         "(no graph, no timing, no baseline), so a launch list sees every kernel")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch
    import __graft_entry__ as ge
    pd = ge.load_package()
    pd.build()
    L = pd._native.lib()
    if args.workload == "batch512":
        run_batch_workload(pd, args, world, rank)
        return
    if args.workload == "melts64":
        run_melts_workload(pd, args, world, rank)
        return
    if args.workload not in ("melt64k", "melt512k"):
        run_ell_workload(pd, args, world, rank)
        return
    n_ions = 512000 if args.workload == "melt512k" else N_IONS
    if args.workload == "melt512k":
        args.no_cpu_baseline = True   # one FP64 CPU step of 512 000 ions takes minutes
        args.snapshots = min(args.snapshots, 500)   # 256 M training rows, as many as 4000 snapshots at 64 k
        args.heldout = min(args.heldout, 2)         # the FP64 real-space sum is all-pairs
    pos, q, m, v, box = make_system(pd, n_ions)
    system = pd.ParticleSystem(pos, box, types=["Na", "Cl"], typeids=np.where(q > 0, 1, 2), masses=m, charges=q,
                               velocities=v)
    dt = DT_FS / pd.synthetic.TIME_UNIT_FS
    sim = pd.Simulation(system, pd.Integrator(dt=dt, forces=forces(pd, args.buffer, args.prune)))
    st = sim.state
    s = st.stream
    pd.evaluate_forces_into_f(sim, energy=False)
    if args.profile and args.form == "learned":
        profile_learned(pd, args, system, box, dt)
        return
    if args.profile:
        st.step(args.warmup, use_graph=False)
        st.synchronize()
        st.step(args.steps, use_graph=False)
        st.synchronize()
        if rank == 0:
            print(json.dumps({"profile": "melt64k eager steps", "steps": args.steps, "warmup": args.warmup,
                              "list": st.cluster.statistics()}))
        return
    # the pair kernel's CTA shape (parts per super-cluster x warps per part) by the autotuner: the pair
    # pass alone, then whole captured steps for each shape (the pair pass shares the GPU with the mesh
    # chain, so the fastest pass alone need not give the fastest step); the timed pair passes
    # accumulated into the slot forces, two evaluations restore the forces
    tune = st.cluster.autotune_pairs(stream=s)
    st.evaluate_forces_into_f(False)
    st.evaluate_forces_into_f(False)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    step_ms = {}
    for key in tune["ms"]:   # timed like the measurement below: L2 flushed before every step
        ns_, w_ = (int(v) for v in key.split("x"))
        st.cluster.set_pair_shape(ns_, w_)
        step_ms[key] = time_md_steps(st, dt, 40, 3, flush, args.no_flush)
    best = min(step_ms, key=step_ms.get)
    st.cluster.set_pair_shape(*(int(v) for v in best.split("x")))
    tune["step_ms"] = step_ms
    tune["nsplit"], tune["warps"] = (int(v) for v in best.split("x"))
    # where the pair pass starts in the step (after the prune, the mesh spread or the forward transform),
    # timed the same way: a later start leaves the critical mesh chain more of the GPU
    sched_ms = {}
    for mode in (0, 1, 2):
        st.engine.set_schedule(mode)
        sched_ms[mode] = time_md_steps(st, dt, 40, 3, flush, args.no_flush)
    best_sched = min(sched_ms, key=sched_ms.get)
    st.engine.set_schedule(best_sched)
    tune["schedule_step_ms"] = {("after prune", "after spread", "after forward FFT")[k]: v for k, v in sched_ms.items()}
    tune["pair_wait"] = best_sched
    # kernels of one eager step: the always-run part (the prune kernel included: it is launched every
    # step and returns at once unless the device decision asks for a prune) plus the build kernels, which
    # the captured graph launches only inside its conditional node on steps that rebuild the list
    c0 = L.pd_launch_count()
    st.step(1, use_graph=False)
    st.synchronize()
    kernels_eager = int(L.pd_launch_count() - c0)
    KERNELS_BUILD = 9
    kernels_always = kernels_eager - KERNELS_BUILD
    # warm-up (graph capture on the first replay)
    st.step(args.warmup, use_graph=True)
    st.synchronize()
    pre = st.cluster.statistics()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        with torch.cuda.stream(s):
            for k in range(args.steps):
                if not args.no_flush:
                    flush.fill_(float(k))
                starts[k].record(s)
                st.engine.step(1, dt, energy_last=False, use_graph=True, stream=s)
                ends[k].record(s)
        torch.cuda.synchronize()
    barrier(world)
    total_ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends))
    total_ms = max_over_ranks(world, total_ms)
    ms_step = total_ms / args.steps
    value = world * ns_per_day(ms_step)
    stats = st.cluster.statistics()
    if stats["error"]:
        raise RuntimeError(f"cluster list error {stats['error']} during the run")
    clocks = clk.summary()
    timed_builds = stats["builds"] - pre["builds"]
    timed_prunes = stats["prunes"] - pre["prunes"]
    gpu_launches = kernels_always * args.steps + KERNELS_BUILD * timed_builds

    # end to end through the C ABI with pinned host buffers: every step copies the state (x, v) in from
    # pinned host memory and copies the stepped state back (the step's result)
    n = st.n
    hxv = torch.empty(6 * n, dtype=torch.float32, pin_memory=True).numpy()   # positions then velocities
    hx, hv = hxv[:3 * n], hxv[3 * n:]
    hx[:] = torch.cat([st.x, st.y, st.z]).cpu().numpy()
    hv[:] = torch.cat([st.vx, st.vy, st.vz]).cpu().numpy()
    e2e_steps = max(20, args.steps // 4)
    for _ in range(3):
        st.engine.step_host(hx, hv, 1, dt, stream=s, energy=False)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        st.engine.step_host(hx, hv, 1, dt, stream=s, energy=False)
    e2e_ms = 1000.0 * (time.perf_counter() - t0) / e2e_steps
    e2e_ms = max_over_ranks(world, e2e_ms)

    # roofline of the dominant kernel: the fused pair pass (FP32 pipe)
    pair_ms = time_pairs_kernel(pd, st)
    npairs = pair_count(st.positions(), box, RC)
    nf = len(st.solver.coulomb_polynomial().pf)
    flop_pair = 20 + 16 * 0 + (2 * (nf - 1) + 8)
    flops = npairs * flop_pair
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    fp32_peak = nsm * 128 * 2 * float(peaks.get("sm_max_mhz", 1965.0)) * 1e6 / 1e12   # TFLOP/s (no measured FP32 figure)
    achieved = flops / (pair_ms * 1e-3) / 1e12
    roofline = {"kernel": "k_pairs<LJ uniform, Coulomb polynomial, force only>", "bound": "fp32",
                "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                "traffic": profiled_traffic("k_pairs_melt64k.md"), "per_launch_ms": pair_ms,
                "pairs_within_rc": npairs, "flop_per_pair": flop_pair,
                "peak_source": "nominal FP32 FMA rate at sm_max_mhz (MEASURED_PEAKS.json has no FP32 figure)"}

    learned = None
    if not args.no_learned:
        learned = run_learned_form(pd, args, st, system, dt, flush)
        learned["value"] = world * learned["value"]
        learned["coarse_only"]["value"] = world * learned["coarse_only"]["value"]
        learned["coarse_radial_no_network"]["value"] = world * learned["coarse_radial_no_network"]["value"]
        learned["plain_e5"]["value"] = world * learned["plain_e5"]["value"]
        learned["pppm_ik"]["value"] = world * learned["pppm_ik"]["value"]
        learned["esp_at_1e-5"]["value"] = world * learned["esp_at_1e-5"]["value"]
        learned["ms_per_step"] = max_over_ranks(world, learned["ms_per_step"])
    # the headline is the learned form only where it reaches the plain form's force error
    form = "plain: fine-mesh SPME (learned coarse-mesh form measured under forms.learned_coarse)"
    if learned is not None:
        e = learned["force_error_vs_fp64_ewald"]
        if e["learned"] <= e["plain_fine"]:
            value = learned["value"]
            ms_step = learned["ms_per_step"]
            form = "learned coarse-mesh: coarse SPME + network at or below the plain form's force error"
    configs = None
    if not args.no_configs:
        configs = {"config0_lj4k": ell_config(pd, "lj4k", 200, args.warmup, peaks),
                   "config1a_lj1m": ell_config(pd, "lj1m", 30, args.warmup, peaks),
                   "config1b_wca2d1m": ell_config(pd, "wca2d1m", 30, args.warmup, peaks),
                   "config4_batch512": batch_config(pd, 30, args.warmup, peaks),
                   "config4_melts64": melts_measure(pd, melts_sizes(64), 20, args.warmup, None, args.buffer,
                                                    args.prune)}
        for c in configs.values():
            c["value"] = world * c["value"]
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        ora = ge.load_oracle()
        cms, csteps, cores = cpu_baseline_run(pd, ora)
        cpu = {"value": ns_per_day(cms), "unit": "ns/day", "cores": cores, "kind": "port",
               "sample": f"{csteps} full MD steps of the same 64k-ion melt on the FP64 CPU restatement "
                         f"(OpenMP pair sums, threaded FFT)"}
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "ns/day", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ionic melt, 1200 K start)",
               "config": {"workload": f"ionic melt N={n} (L={box[0]:.1f} A) LJ+SPME r_c=9 A, "
                                      f"{'x'.join(str(k) for k in st.solver.mesh)} order 5, NVE dt=1 fs",
                          "form": form, "parallelism": f"replicas x{world}",
                          "aggregate": ("value = ns/day summed over the independent replicas, one per GPU"
                                        if world > 1 else "one system"),
                          "list_buffer_A": args.buffer, "prune_buffer_A": args.prune,
                          "pair_shape": {"nsplit": tune["nsplit"], "warps": tune["warps"],
                                         "pair_pass_ms": tune["ms"], "step_ms": tune["step_ms"]},
                          "schedule": {"pair_wait": tune["pair_wait"], "step_ms": tune["schedule_step_ms"]},
                          "l2": "flushed (256 MiB write) before every timed step" if not args.no_flush else "warm",
                          "timed_builds": timed_builds, "timed_prunes": timed_prunes},
               "roofline": roofline, "cpu_baseline": cpu,
               "forms": {"plain": {"value": world * ns_per_day(total_ms / args.steps), "unit": "ns/day",
                                   "ms_per_step": total_ms / args.steps,
                                   "mesh": f"SPME 1.0 A ({'x'.join(str(k) for k in st.solver.mesh)}), order 5 "
                                           "(the configuration's settings)"},
                         "plain_at_1e-5_vs_ewald": learned.pop("plain_e5") if learned else None,
                         "pppm_ik": learned.pop("pppm_ik") if learned else None,
                         "esp_at_1e-5": learned.pop("esp_at_1e-5") if learned else None,
                         "learned_vs_plain_equal_error": learned.pop("learned_vs_plain_equal_error")
                         if learned else None,
                         "learned_coarse": learned},
               "e2e": {"value": world * ns_per_day(e2e_ms), "unit": "ns/day", "h2d_bytes_per_step": 24 * n,
                       "d2h_bytes_per_step": 24 * n, "ms_per_step": e2e_ms},
               "configs": configs,
               "gpu_launches": gpu_launches,
               "kernels": {"every_step": kernels_always, "per_build": KERNELS_BUILD,
                           "cufft_per_step": "2 transforms (library kernels, not counted)"},
               "clocks": clocks}
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
