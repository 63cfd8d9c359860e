"""Benchmark of the 2D active multi-phase-field step on B200.

Workload (one GPU): 2D periodic lattice 2048 x 2048, 1024 cells of radius
R = 12, centres from the sequential periodic initialiser with minimum
separation 2R, tanh-disk seeds, reference default coefficients, binary32 phi
with the exact Q5.27 aggregate. A "step" is one time step of every cell (one
fused kernel launch). Throughput is site-cell updates/s counted over the
reference's window (144^2 sites per class-0 cell).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl pfb|reference]

Multi-GPU: one process per GPU (torchrun); every rank runs an independent
replica of the workload with its own seed (the path has no exchange step), so
scaling is weak and the value is the total over ranks divided by the slowest
rank's device time.

``--impl reference`` times the reference's algorithm on the host cores: the
reference has no CPU solver, so this is the OpenMP restatement in oracle/
(the same code as the ``cpu_baseline`` leg), run on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "phase-field-gh200_b200"))

L_SIDE = 2048
N_CELLS = 1024
RADIUS = 12.0
WORKLOAD = ("2D periodic 2048x2048, 1024 cells R=12, min-separation 2R sequential centres, "
            "tanh disks, default coefficients (dt=0.01, lambda=7, kappa=10, mu=1, xi=1500, "
            "tau=1e4, v_A=0.01, M=0.5), f32 phi, Q5.27 aggregate")
FALLBACK_HBM_GBS = 6650.0
# the 2D single-system workloads: side, cells, description, L2 statement
WORKLOADS_2D = {
    "c2": (L_SIDE, N_CELLS, WORKLOAD,
           "inputs larger than L2: two 340 MB phi pools; per-step working set 85 MB phi read + "
           "85 MB phi written + 3 x 16.8 MB aggregate slots; no flush between steps"),
    "c1": (512, 64, WORKLOAD.replace("2048x2048, 1024 cells", "512x512, 64 cells"),
           "the whole state (two 21 MB phi pools, three 1 MB aggregate slots) fits in the 126 MB "
           "L2, so a 256 MiB buffer is written before every timed step and each step is timed "
           "alone (CUDA events around it); the L2-resident graph replay is reported beside it"),
}


def rank_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Largest value over all ranks (device times are taken as the slowest
    rank's); identity without a process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(sites_per_rank_step: int, steps: int, world: int, max_ms: float) -> float:
    """Site-cell updates/s of the whole job: every rank advances its own
    replica by `steps`; the job takes as long as its slowest rank."""
    return world * sites_per_rank_step * steps / (max_ms / 1000.0)


def workload_params(seed: int, wl: str = "c2"):
    from pfb200.sim2d import SimParams2D
    L, N = WORKLOADS_2D[wl][:2]
    return SimParams2D(L=L, num_cells=N, target_radius=RADIUS, seed=seed)


def workload_centres(p):
    import pfb200
    return pfb200.palmieri_centres(p.num_cells, p.L, 2.0 * p.target_radius, p.seed)


def sites_per_step(cells) -> int:
    """Reference window of every cell: 144^2 sites per class-0 cell."""
    return int(len(cells)) * 144 * 144


def algorithmic_bytes(cells, L: int, phi_bytes: int = 4) -> int:
    """sum_n A_n * 2 * phi_bytes (read phi^n + write phi^{n+1} over the
    processed window) + L^2 * 8 B (one read and one write of the u32
    aggregate)."""
    import pfb200
    area = sum(pfb200.CLASSES[int(c)][0] * pfb200.CLASSES[int(c)][1] for c in cells["cls"])
    return int(area * 2 * phi_bytes + L * L * 8)


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.lines: list[str] = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-i", str(self.device), "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def mark(self):
        return len(self.lines)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)

    def summary(self, start: int, end: int) -> dict:
        rows = []
        for ln in self.lines[start:end] or self.lines[-3:]:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) >= 8:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][1]) if rows[0][1].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def read_peak_hbm():
    f = REPO / "MEASURED_PEAKS.json"
    try:
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s"


def read_ncu_traffic(wl: str = "c2"):
    """DRAM bytes per launch of the step kernel from the committed ncu summary
    of the same workload (profiles/k_step2d_<workload>.md), or None."""
    f = REPO / "profiles" / f"k_step2d_{wl}.md"
    if not f.exists():
        return None
    for ln in f.read_text().splitlines():
        if ln.startswith("dram_bytes_per_launch:"):
            try:
                return int(float(ln.split(":", 1)[1].split()[0]))
            except ValueError:
                return None
    return None


def oracle_workload_state(seed: int, wl: str = "c2"):
    """A 2D workload's initial state built by the oracle alone (placement,
    fresh-start draws and tanh seeds restated from the reference's host code
    and k_init_tiles), so the CPU legs load no library of this package."""
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle2d
    p = workload_params(seed, wl)
    cx, cy = oracle2d.palmieri_centres(p.num_cells, p.L, 2.0 * p.target_radius, p.seed)
    cells, phi = oracle2d.init_state(p.to_c(), cx, cy, oracle2d.fresh_cells(p.to_c()))
    return p, cells, phi


def cpu_time_steps(p, cells, phi, warmup: int, steps: int):
    """Time `steps` consecutive time steps of the whole workload on the
    oracle's OpenMP restatement (all host threads), as one timed region after
    `warmup` untimed steps; returns (site-cell updates/s, seconds, threads)."""
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle2d
    threads = os.cpu_count() or 1
    o = oracle2d.OracleSim(p.to_c(), cells, phi, step=0)
    o.advance(max(1, warmup), threads)  # warms the caches and the thread pool
    t0 = time.perf_counter()
    o.advance(steps, threads)
    dt = time.perf_counter() - t0
    o.close()
    return sites_per_step(cells) * steps / dt, dt, threads


def c2_config(a, sites: int) -> dict:
    """The workload description both arms print (identical by construction)."""
    L, N, text, l2 = WORKLOADS_2D[a.workload]
    return {"workload": text, "L": L, "cells": N, "radius": RADIUS,
            "sites_per_step": sites, "window": "reference class-0 window 144^2",
            "l2": l2, "parallelism": f"replicas x{a.gpus}"}


def run_reference_arm(a):
    """Reference arm: the reference's update on the host cores. The reference
    has no CPU solver, so this is the OpenMP restatement of its update in
    oracle/ (pinned to the reference's own kernel and host code), over the
    whole c2 workload: W untimed steps, then K steps timed as one region on
    every host thread. The state comes from the oracle's own restatement of
    the reference's initialiser; nothing of this package is loaded."""
    rank, world, _ = rank_env()
    if rank != 0:
        return 0
    wl = a.workload if a.workload in WORKLOADS_2D else "c2"
    a.workload = wl
    p, cells, phi = oracle_workload_state(1234, wl)
    warm = min(a.warmup, 5)
    value, secs, threads = cpu_time_steps(p, cells, phi, warm, a.steps)
    sites = sites_per_step(cells)
    sample = (f"{a.steps} consecutive time steps of the whole workload after {warm} untimed "
              f"ones ({secs:.2f} s on {threads} threads)")
    line = {
        "impl": "reference", "metric": "site-cell updates/s", "value": value,
        "unit": "site-cell updates/s", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1000.0 * secs / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": c2_config(a, sites),
        "implementation": "CPU OpenMP restatement of the reference update (oracle/)",
        "cpu_baseline": {"value": value, "unit": "site-cell updates/s", "cores": threads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "site-cell updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# 3D workload (--workload c3): periodic 256^3, 512 cells R = 10, B = 64
# ---------------------------------------------------------------------------
WORKLOAD3D = ("3D periodic 256^3, 512 cells R=10 (V0=4/3 pi R^3), lambda=7, brick B=64 "
              "(the automatic edge; B=48 is rejected at lambda=7), min-separation 2R sequential "
              "centres (cell 0 at the box centre), tanh spheres with the calibrated seed radius, "
              "default coefficients, f32 phi, Q5.27 aggregate")


WORKLOAD3D_SLAB = ("3D substrate slab 256x256x128 (Nz = 32 is rejected because the slab "
                   "needs Nz > B), 187 cells R=10 (rho_A = N pi R^2 / 256^2 = 0.90; the same "
                   "cells per area as the periodic run would need rho_A = 2.45), hemispherical "
                   "V0 = 2/3 pi R^3, lambda=7, B=80 (at the automatic B=64 the packing exhausts "
                   "the support margin after 20 steps, where the reference promotes bricks), "
                   "centres on "
                   "the substrate (z = -1/2) sequential with minimum separation R (2R cannot "
                   "pack rho_A = 0.9), default coefficients, f32 phi, Q5.27 aggregate")


def workload3d(seed: int, wl: str = "c3"):
    import pfb200
    if wl == "c3s":
        # B = 80: at the automatic 64 the dense slab exhausts the brick's support
        # margin after 20 steps (the reference then promotes bricks, which this
        # build does not), so the base brick is raised as the reference's
        # --brick-edge allows
        p = pfb200.SimParams3D(Nx=256, Ny=256, Nz=128, geometry="slab", num_cells=187,
                               target_radius=10.0, lambda_=7.0, B=80, seed=seed)
        c = pfb200.sequential_centres(187, 256.0, 10.0, seed, planar_z=-0.5)
        return p, c
    p = pfb200.SimParams3D(Nx=256, Ny=256, Nz=256, num_cells=512, target_radius=10.0,
                           lambda_=7.0, B=64, seed=seed)
    c = pfb200.sequential_centres(512, 256.0, 20.0, seed, first_at_centre=True)
    return p, c.astype(np.float32).astype(np.float64)


def read_ncu_traffic3d(wl: str = "c3"):
    f = REPO / "profiles" / f"k_step3d_{wl}.md"
    if not f.exists():
        return None
    for ln in f.read_text().splitlines():
        if ln.startswith("dram_bytes_per_step:"):
            try:
                return int(float(ln.split(":", 1)[1].split()[0]))
            except ValueError:
                return None
    return None


def run_3d(a):
    """One step = the reference Sim3D sequence (measure, motion, clear,
    update, repair/finalize/restore/advance); throughput counts the B^3
    brick of every cell (the reference's window)."""
    import torch
    import pfb200
    rank, world, local = rank_env()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    p, c = workload3d(1234 + rank, a.workload)
    if a.brick_edge:
        p.B = a.brick_edge
    p.phi_storage = a.phi_storage
    sim = pfb200.Sim3D(p, c, device=local)
    if a.fused3d == "off":
        sim.set_fused(False)
    elif a.fused3d == "on":
        sim.set_fused(True)
    if a.order3d == "slot":
        sim.set_order(False)
    fused = sim.fused
    B, N = sim.B, p.num_cells
    sites = N * B ** 3
    phi_b = 2 if a.phi_storage else 4
    alg = sites * 2 * phi_b + p.Nx * p.Ny * p.Nz * 8
    slab = a.workload == "c3s"
    ext = torch.cuda.ExternalStream(sim.stream, device=local)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(local)

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    sim.advance(a.warmup)
    sim.sync()
    barrier()
    m0 = clocks.mark()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    sim.advance(a.steps)
    e1.record(ext)
    sim.sync()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, f"cuda:{local}")
    time.sleep(0.15)
    m1 = clocks.mark()
    e2e = None
    if not a.no_e2e:
        from pfb200._abi import check, lib
        cells_out = torch.empty((N, 256), dtype=torch.uint8).pin_memory()
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(ext)
        for _ in range(a.steps):
            check(lib().pfb_sim3d_advance(sim._h, 1), "advance")
            check(lib().pfb_sim3d_get_cells(sim._h, cells_out.data_ptr()), "get_cells")
        f1.record(ext)
        sim.sync()
        barrier()
        el = max_over_ranks(f0.elapsed_time(f1) / 1000.0, dist, f"cuda:{local}")
        e2e = {"value": world * sites * a.steps / el, "unit": "site-cell updates/s",
               "h2d_bytes_per_step": 0, "d2h_bytes_per_step": cells_out.numel(),
               "steps": a.steps,
               "note": "state built on the device from host centres at creation; every step "
                       "reads the 512 cell records back through pfb_sim3d_get_cells"}
    clocks.stop()
    flags = sim.flags()
    if rank == 0:
        ms_step = ms / a.steps
        peak, peak_src = read_peak_hbm()
        achieved = alg / (ms_step / 1000.0) / 1e9
        cpu = None
        if world == 1 and a.cpu_steps > 0 and a.phi_storage == 0:
            cpu = cpu_sample3d(p, sim, threads=0)
        line = {
            "metric": "site-cell updates/s", "value": world * sites * a.steps / (ms / 1000.0),
            "unit": "site-cell updates/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": ("f32", "f32 arithmetic, f16 phi storage",
                      "f32 arithmetic, bf16 phi storage")[a.phi_storage], "data": "synthetic",
            "config": {"workload": WORKLOAD3D_SLAB if slab else WORKLOAD3D,
                       "domain": [p.Nx, p.Ny, p.Nz], "geometry": p.geometry, "cells": N,
                       "radius": 10.0, "B": B, "sites_per_step": sites,
                       "step": "fused measure + motion + update launch" if fused else
                               "separate measure, motion and update launches",
                       "visit_order": a.order3d,
                       "phi_storage": ("binary32", "binary16", "bfloat16")[a.phi_storage],
                       "l2": "inputs larger than L2: two %d MB phi pools and two %d MB "
                             "aggregate slots; no flush between steps" % (
                                 N * B ** 3 * phi_b // 2 ** 20, p.Nx * p.Ny * p.Nz * 4 // 2 ** 20),
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": read_ncu_traffic3d(a.workload) if not a.phi_storage else None,
                         "kernel": ("pfb::p3::k_step3d<%d, %d> (one step)" % (
                             pfb200.lib().pfb3d_step_cluster(B), 1 if slab else 0)) if fused else
                                   ("pfb::p3::k_measure3d<%d> + k_update3d<%d> (one step)" % (
                                       pfb200.lib().pfb3d_step_cluster(B) or 4, 1 if slab else 0)),
                         "algorithmic_bytes_per_launch": alg, "peak_source": peak_src,
                         "duration_source": "CUDA events over the timed region / steps"},
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks.summary(m0, m1),
            "gpu_launches": a.steps * (8 if fused else 10),
            "flags": pfb200.flags_report3(flags),
        }
        print(json.dumps(line), flush=True)
    sim.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def cpu_sample3d(p, sim, threads: int):
    """One full step of the 3D workload on the OpenMP restatement (oracle/)."""
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle3d
    st = oracle3d.OracleState3D(p, sim.layout, sim.B, sim.cells(), sim.phi(), sim.S())
    n = os.cpu_count() or 1
    t0 = time.perf_counter()
    st.advance(1, threads)
    dt = time.perf_counter() - t0
    return {"value": p.num_cells * sim.B ** 3 / dt, "unit": "site-cell updates/s", "cores": n,
            "kind": "port", "sample": f"one full time step of the same 3D workload ({dt:.1f} s) "
                                      "on the OpenMP restatement of the update"}


# ---------------------------------------------------------------------------
# Batched ensemble (--workload ce): 64 independent 2D replicas of mixed size
# ---------------------------------------------------------------------------
WORKLOAD_CE = ("64 independent 2D periodic replicas, lattice side drawn from {256, 384, 512, "
               "768, 1024} (the reference refuses 256, below its largest window 286; here a "
               "256 side uses the classes whose window fits it), packing rho ~ U[0.5, 0.9], "
               "N = clamp(round(rho L^2 / (pi R^2)), 16, 400), "
               "R = 12, min-separation R sequential centres, per-replica seeds base + r, "
               "default coefficients, f32 phi; one launch per step for all replicas")


def ensemble_systems(base_seed: int, count: int = 64):
    import math
    import pfb200
    rng = np.random.default_rng(base_seed)
    ps, cs = [], []
    for r in range(count):
        L = int(rng.choice([256, 384, 512, 768, 1024]))
        rho = float(rng.uniform(0.5, 0.9))
        N = int(min(400, max(16, round(rho * L * L / (math.pi * RADIUS ** 2)))))
        p = pfb200.SimParams2D(L=L, num_cells=N, target_radius=RADIUS, seed=base_seed + r)
        ps.append(p)
        cs.append(pfb200.palmieri_centres(N, L, RADIUS, p.seed))
    return ps, cs


def run_ensemble(a):
    import torch
    import pfb200
    rank, world, local = rank_env()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    ps, cs = ensemble_systems(1234 + 64 * rank, a.replicas)
    for p in ps:
        p.phi_storage = a.phi_storage
    ens = pfb200.Ensemble2D(ps, cs, device=local)
    chosen = ens.autotune(12)
    sites = sum(p.num_cells for p in ps) * 144 * 144
    phi_b = 2 if a.phi_storage else 4
    alg = sum(p.num_cells * 144 * 144 * 2 * phi_b + p.L * p.L * 8 for p in ps)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(local)

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier()
    m0 = clocks.mark()
    ms_step = ens.bench(a.warmup, a.steps)  # device time (CUDA events), graph replay
    m1 = clocks.mark()
    ms_serial = ens.bench(3, max(6, a.steps // 10), serial=True)
    barrier()
    ms_step = max_over_ranks(ms_step, dist, f"cuda:{local}")
    # ---- end to end through the public API with host buffers (wall clock):
    # every replica's state uploaded from pinned memory once, every step the
    # trajectory records of all replicas read back, the final fields read back
    e2e = None
    if not a.no_e2e:
        from pfb200._abi import TRAJ_DTYPE, check, lib
        views = [ens.system(r) for r in range(len(ps))]
        up = [(torch.from_numpy(v.cells().view(np.uint8).copy()).pin_memory(),
               torch.from_numpy(np.ascontiguousarray(v.phi())).pin_memory()) for v in views]
        outs = [torch.empty_like(u[1]).pin_memory() for u in up]
        chunk = 30
        total = ens.total_cells
        # two halves of a page-locked ring of all systems' records: the host
        # reads one while the device fills the other
        ring = torch.empty((2, chunk, total * TRAJ_DTYPE.itemsize), dtype=torch.uint8).pin_memory()
        halves = [ring[h].numpy().view(TRAJ_DTYPE).reshape(chunk, total) for h in range(2)]
        ext_e = torch.cuda.ExternalStream(ens.stream, device=local)
        done_ev = [torch.cuda.Event(), torch.cuda.Event()]
        track = []
        step0 = ens.step
        e2e_steps = chunk * max(2, min(a.steps, 600) // chunk)
        ens.sync()
        barrier()
        t0 = time.perf_counter()
        for v, (c_h, p_h) in zip(views, up):
            check(lib().pfb_sim2d_set_state(v._h, c_h.data_ptr(), p_h.data_ptr(), step0),
                  "set_state")
        for c in range(e2e_steps // chunk):
            ens.advance_record(chunk, 1, halves[c % 2])
            done_ev[c % 2].record(ext_e)
            if c:
                done_ev[(c - 1) % 2].synchronize()
                f = halves[(c - 1) % 2]
                track.append((f["cx"].mean(axis=1), f["cy"].mean(axis=1)))
        for v, o in zip(views, outs):
            check(lib().pfb_sim2d_get_phi(v._h, o.data_ptr()), "get_phi")
        ens.sync()
        el = max_over_ranks(time.perf_counter() - t0, dist, f"cuda:{local}")
        f = halves[(e2e_steps // chunk - 1) % 2]
        track.append((f["cx"].mean(axis=1), f["cy"].mean(axis=1)))
        assert len(track) * chunk == e2e_steps
        h2d = sum(c.numel() + p_.numel() * p_.element_size() for c, p_ in up)
        d2h = total * TRAJ_DTYPE.itemsize * e2e_steps + sum(o.numel() * o.element_size() for o in outs)
        e2e = {"value": world * sites * e2e_steps / el, "unit": "site-cell updates/s",
               "h2d_bytes_per_step": h2d / e2e_steps, "d2h_bytes_per_step": d2h / e2e_steps,
               "steps": e2e_steps,
               "note": "host wall clock; states of all replicas uploaded from pinned memory, "
                       "one batched launch per step, every replica's trajectory records of every "
                       "step written to a page-locked ring (pfb_ens2d_advance_record, 30-step "
                       "chunks, two halves read on the host while the next chunk runs), final "
                       "fields read back"}
    cpu = None
    if world == 1 and a.cpu_steps > 0 and a.phi_storage == 0:
        # one time step of every replica on the OpenMP restatement (oracle/)
        sys.path.insert(0, str(REPO / "oracle"))
        import oracle2d
        tot, secs, thr = 0, 0.0, os.cpu_count() or 1
        for r, p in enumerate(ps):
            v = ens.system(r)
            o = oracle2d.OracleSim(p.to_c(), v.cells(), v.phi(), step=ens.step)
            o.advance(1, thr)
            t1 = time.perf_counter()
            o.advance(1, thr)
            secs += time.perf_counter() - t1
            o.close()
            tot += p.num_cells * 144 * 144
        cpu = {"value": tot / secs, "unit": "site-cell updates/s", "cores": thr, "kind": "port",
               "sample": f"one time step of each of the {len(ps)} replicas after one untimed "
                         f"({secs:.2f} s on {thr} threads) on the OpenMP restatement"}
    clocks.stop()
    flags = sum(int(ens.system(r).flags().sum()) for r in range(len(ps)))
    if rank == 0:
        peak, peak_src = read_peak_hbm()
        achieved = alg / (ms_step / 1000.0) / 1e9
        line = {
            "metric": "site-cell updates/s", "value": world * sites / (ms_step / 1000.0),
            "unit": "site-cell updates/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": ("f32", "f32 arithmetic, f16 phi storage",
                      "f32 arithmetic, bf16 phi storage")[a.phi_storage],
            "data": "synthetic",
            "config": {"workload": WORKLOAD_CE, "replicas": len(ps),
                       "phi_storage": ("binary32", "binary16", "bfloat16")[a.phi_storage],
                       "cells_total": sum(p.num_cells for p in ps), "sites_per_step": sites,
                       "sides": sorted({p.L for p in ps}), "cluster_ctas_per_cell": chosen,
                       "autotuned": True, "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "pfb::k_step2d_batch<%d%s>" % (
                             chosen, ("", ", __half", ", __nv_bfloat16")[a.phi_storage]),
                         "algorithmic_bytes_per_launch": alg, "peak_source": peak_src,
                         "duration_source": "CUDA events over the timed region / steps"},
            "replicas_one_at_a_time": {"ms_per_step": ms_serial,
                                       "batched_speedup": ms_serial / ms_step},
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks.summary(m0, m1),
            "gpu_launches": a.steps, "flags_total": flags,
        }
        print(json.dumps(line), flush=True)
    ens.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


WORKLOAD_CS = ("passive relaxation (v_A = 0) of a 1024^2 periodic lattice with 400 cells of "
               "radius 12 (rho 0.17, min separation 2R, seed 999): time until the step residual "
               "max |dphi/dt| reaches the target, plain explicit steps against steps with jumps "
               "of the learned surrogate judged by the plain solver")


def profile_conv_layers(local, batch=512, repeats=20):
    """One JSON line per U-Net layer shape (channels in -> out, crop edge):
    the median CUDA-event time of one pfb_conv3x3_forward (bias, ReLU,
    bfloat16 output) over `repeats` launches after 3 warm-up ones, L2
    flushed by a 256 MB write before each, with the persistent
    warp-specialised kernel (pipeline mode 2) and with one tile per CTA
    (mode 0); the useful FLOPs and the activation bytes in and out give the
    rates."""
    import torch
    import pfb200
    from pfb200 import check
    L = pfb200.lib()
    dev = f"cuda:{local}"
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    try:
        for cin, cout, h in ((32, 32, 64), (32, 32, 32), (16, 32, 64), (32, 16, 64), (32, 16, 32),
                             (16, 32, 32), (16, 16, 64)):
            p2 = (h + 2) * (h + 2)
            g = torch.Generator(device=dev).manual_seed(cin * 100 + cout + h)
            x = torch.randn(batch, p2, cin, device=dev, generator=g).to(torch.bfloat16)
            w = torch.randn(cout, cin, 3, 3, device=dev, generator=g) * 0.1
            wp = torch.zeros(9 * cin * cout, dtype=torch.bfloat16, device=dev)
            check(L.pfb_conv3x3_pack(w.data_ptr(), wp.data_ptr(), cin, cout, 0, None), "pack")
            bias = torch.randn(cout, device=dev, generator=g)
            y = torch.empty(batch, p2, cout, dtype=torch.bfloat16, device=dev)
            row = {"layer": f"{cin}->{cout}", "crop": h, "batch": batch}
            for mode in (0, 2):
                check(L.pfb_conv_set_pipeline(mode), "pipeline")
                times = []
                for it in range(3 + repeats):
                    flush.zero_()
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record()
                    check(L.pfb_conv3x3_forward(x.data_ptr(), y.data_ptr(), None, wp.data_ptr(),
                                                bias.data_ptr(), None, batch, h, h, cin, cout, 1,
                                                stream), "forward")
                    e1.record()
                    torch.cuda.synchronize()
                    if it >= 3:
                        times.append(e0.elapsed_time(e1) * 1e3)
                times.sort()
                us = times[len(times) // 2]
                key = "persistent" if mode else "tile_per_cta"
                row[key + "_us"] = us
                row[key + "_tflops"] = 2.0 * batch * h * h * 9 * cin * cout / us / 1e6
                row[key + "_gbs"] = batch * p2 * (cin + cout) * 2 / us / 1e3
            print(json.dumps(row), flush=True)
    finally:
        L.pfb_conv_set_pipeline(1)
    return 0


def run_surrogate(a):
    """The surrogate workload: training data from plain-solver pairs (10 runs x
    5 pairs x 400 cells = 20,000 crops, increments over 8,000 steps, inputs
    with the rate over the previous 100 steps), Adam training of the U-Net,
    then time-to-relaxed of a fresh system, plain against
    surrogate-accelerated (median wall time of three runs each). One GPU
    (other ranks exit)."""
    import torch
    import pfb200
    from pfb200 import surrogate as sg
    rank, world, local = rank_env()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    pfb200.lib().pfb_conv_set_pipeline(a.conv_pipeline)
    if a.profile_layers:
        return profile_conv_layers(local)
    if a.profile_forward:
        net = sg.Surrogate2D(max_batch=512, seed=1, device=local)
        ms = net.bench_forward(512, 3)
        x = torch.zeros((512, sg.PADDED, sg.IN_CH), dtype=torch.bfloat16, device=f"cuda:{local}")
        t = torch.zeros((512, sg.CROP, sg.CROP), dtype=torch.float32, device=f"cuda:{local}")
        idx = torch.arange(512, dtype=torch.int32, device=f"cuda:{local}")
        for _ in range(2):
            net.train_step(x, t, idx, 1e-4)
        net.sync()
        print(json.dumps({"profile_forward_ms": ms, "batch": 512,
                          "tflops": sg.forward_flops(512) / (ms / 1000.0) / 1e12,
                          "conv_pipeline": a.conv_pipeline}), flush=True)
        net.close()
        return 0
    interval, history, heal = 8000, 100, 100
    p = sg.relaxation_params()
    data = sg.make_dataset(p, runs=10, pairs_per_run=5, interval=interval, device=local,
                           history=history)
    net = sg.Surrogate2D(max_batch=512, seed=1, device=local)
    for _ in range(3):
        net.bench_forward(512, 5)  # warm-up
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    m0 = clocks.mark()
    fwd_ms = net.bench_forward(512, 50)
    m1 = clocks.mark()
    t0 = time.perf_counter()
    hist = sg.train(net, data, steps=a.train_steps, batch=256, log_every=1000)
    train_s = time.perf_counter() - t0

    def run(use_net):
        t1 = time.perf_counter()
        q = sg.relaxation_params(seed=999)
        cx, cy = pfb200.palmieri_centres(q.num_cells, q.L, 2 * q.target_radius, q.seed)
        sim = pfb200.Sim2D(q, cx, cy, device=local)
        r = sg.relax(sim, a.target, a.max_steps, net=net if use_net else None,
                     interval=interval, heal=heal, history=history)
        phi = sim.phi()  # final state back to the host
        total = time.perf_counter() - t1
        flags = sim.flags()
        sim.close()
        return r, total, phi.nbytes, flags

    def median_of(use_net, k=a.repeats):
        runs = sorted((run(use_net) for _ in range(k)), key=lambda x: x[0].seconds)
        return runs[k // 2], [x[0].seconds for x in runs]

    (plain, plain_total, _, _), plain_all = median_of(False)
    (sur, sur_total, phi_bytes, flags), sur_all = median_of(True)
    clocks.stop()
    peaks = json.loads((REPO / "MEASURED_PEAKS.json").read_text()) \
        if (REPO / "MEASURED_PEAKS.json").exists() else {}
    peak = float(peaks.get("bf16_tflops", 1590.0))
    achieved = sg.forward_flops(512) / (fwd_ms / 1000.0) / 1e12
    # kernels of one jump: extract, 8 convolutions, pool, upsample, take, insert, moments, scatter
    launches = sur.solver_steps + len(sur.history) + 15 * (sur.jumps_accepted + sur.jumps_rejected)
    line = {
        "metric": "time-to-relaxed", "value": sur.seconds, "unit": "s", "n_gpus": 1,
        "steps": sur.solver_steps, "warmup": 0, "ms_per_step": 1000.0 * sur.seconds / sur.solver_steps,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 solver; bf16 network with f32 accumulation", "data": "synthetic",
        "config": {"workload": WORKLOAD_CS, "L": p.L, "cells": p.num_cells, "radius": p.target_radius,
                   "target_residual": a.target, "residual": "max over cells and sites of "
                   "|phi^{k+1} - phi^k| / dt, checked every 500 steps",
                   "jump_interval_steps": interval, "rate_history_steps": history,
                   "heal_steps": heal, "repeats": f"median of {a.repeats} wall times",
                   "max_solver_steps": a.max_steps,
                   "dataset": f"{data.x.shape[0]} crops from 10 fresh runs x 5 pairs ({data.seconds:.1f} s)",
                   "train_steps": a.train_steps, "batch": 256,
                   "l2": "solver inputs larger than L2 (two 133 MB phi pools)"},
        "reached": sur.reached, "residual": sur.residual,
        "plain": {"seconds": plain.seconds, "reached": plain.reached, "residual": plain.residual,
                  "solver_steps": plain.solver_steps, "all_seconds": plain_all},
        "surrogate": {"seconds": sur.seconds, "reached": sur.reached, "residual": sur.residual,
                      "solver_steps": sur.solver_steps, "jumps_accepted": sur.jumps_accepted,
                      "jumps_rejected": sur.jumps_rejected,
                      "equivalent_steps": sur.equivalent_steps, "all_seconds": sur_all},
        "speedup_vs_plain": plain.seconds / sur.seconds,
        "solver_step_ratio": plain.solver_steps / sur.solver_steps,
        "training": {"seconds": train_s, "crops_per_s": a.train_steps * 256 / train_s,
                     "dataset_seconds": data.seconds,
                     "loss_first": hist[0][1], "loss_last": hist[-1][1]},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None,
                     "kernel": "pfb::k_conv3x3_fwd (U-Net forward, 512 crops, 8 layers)",
                     "flops_per_launch": sg.forward_flops(512),
                     "peak_source": "measured (MEASURED_PEAKS.json bf16_tflops, burst)",
                     "duration_source": "CUDA events, 50 forward passes"},
        "cpu_baseline": None,
        "e2e": {"value": sur_total, "unit": "s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": phi_bytes / max(1, sur.solver_steps),
                "plain_seconds": plain_total,
                "note": "fresh system from host centres to the relaxed phi pool back on the host"},
        "clocks": clocks.summary(m0, m1),
        "gpu_launches": launches,
        "flags": pfb200.flags_report(flags),
    }
    print(json.dumps(line), flush=True)
    net.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--warmup", type=int, default=60)
    ap.add_argument("--impl", default="pfb", choices=["pfb", "reference"])
    ap.add_argument("--cluster", type=int, default=0,
                    help="CTAs per cell (2, 4 or 8; 0: 2 for c2, 4 for c1)")
    ap.add_argument("--variant", type=int, default=0, help="kernel variant (0 = default)")
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--replicas", type=int, default=64,
                    help="ensemble workload: the first R of its 64 replicas (profiling cases)")
    ap.add_argument("--phi-storage", type=int, default=0, choices=[0, 1, 2],
                    help="2D phi pools: 0 binary32 (reference layout), 1 binary16, 2 bfloat16")
    ap.add_argument("--cpu-steps", type=int, default=int(os.environ.get("PFB_CPU_STEPS", "40")),
                    help="most time steps of the CPU baseline leg (one timed region)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="c2", choices=["c2", "c1", "c3", "c3s", "ce", "cs"],
                    help="c2: 2D 2048^2 / 1024 cells (default); c1: 2D 512^2 / 64 cells; "
                         "c3: 3D periodic 256^3 / 512 cells; c3s: 3D slab 256x256x128 / 187 "
                         "cells; ce: batched ensemble of 64 mixed-size 2D replicas; cs: passive "
                         "relaxation of 1024^2 / 400 cells, plain against the learned surrogate")
    ap.add_argument("--fused3d", choices=("auto", "on", "off"), default="auto",
                    help="3D: one fused measure + motion + update launch per step (auto: the "
                         "driver's default, the separate launches)")
    ap.add_argument("--order3d", choices=("morton", "slot"), default="morton",
                    help="3D: visit cells in the Morton order of their bricks or in slot order")
    ap.add_argument("--brick-edge", type=int, default=0,
                    help="c3/c3s: brick edge B (0: the automatic edge, 64 at lambda 7, R 10)")
    ap.add_argument("--target", type=float, default=1e-3,
                    help="cs: residual max |dphi/dt| that counts as relaxed")
    ap.add_argument("--train-steps", type=int, default=8000, help="cs: Adam steps")
    ap.add_argument("--repeats", type=int, default=3, help="cs: relaxations per method (median)")
    ap.add_argument("--max-steps", type=int, default=150000,
                    help="cs: plain solver steps after which a relaxation gives up")
    ap.add_argument("--conv-pipeline", type=int, default=1, choices=[0, 1, 2],
                    help="cs: forward convolution kernel: 2 persistent warp-specialised for every "
                         "channel pair, 1 for the 32 -> 32 pair only, 0 one tile per CTA")
    ap.add_argument("--profile-layers", action="store_true",
                    help="cs: time each U-Net layer shape's forward convolution with both kernels "
                         "and exit")
    ap.add_argument("--profile-forward", action="store_true",
                    help="cs: only 3 forward passes and 2 training steps of the U-Net on 512 "
                         "zero crops (a short command for ncu)")
    a = ap.parse_args()
    if a.warmup < 3:
        a.warmup = 3
    if a.impl == "reference":
        return run_reference_arm(a)
    if a.workload in ("c3", "c3s"):
        return run_3d(a)
    if a.workload == "ce":
        return run_ensemble(a)
    if a.workload == "cs":
        return run_surrogate(a)

    import torch
    import pfb200

    rank, world, local = rank_env()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    device = local
    torch.cuda.set_device(device)

    if a.cluster == 0:  # measured best per workload: 2 for c2, 4 for c1
        a.cluster = 4 if a.workload == "c1" else 2
    p = workload_params(1234 + rank, a.workload)
    p.phi_storage = a.phi_storage
    cx, cy = workload_centres(p)
    sim = pfb200.Sim2D(p, cx, cy, device=device, cluster=a.cluster, use_graph=not a.no_graph,
                       variant=a.variant)
    init_cells = sim.cells()
    init_phi = sim.phi() if (rank == 0 and world == 1) or not a.no_e2e else None
    alg = algorithmic_bytes(init_cells, p.L, 2 if a.phi_storage else 4)
    sites = sites_per_step(init_cells)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(device)

    ext = torch.cuda.ExternalStream(sim.stream, device=device)
    clocks = ClockSampler(device)
    clocks.start()
    time.sleep(0.3)

    sim.advance(a.warmup)
    sim.sync()
    barrier()
    m0 = clocks.mark()
    graph_ms = None
    if a.workload == "c1":
        # L2-resident state: flush before every step, each step timed alone
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{device}")
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(a.steps)]
        with torch.cuda.stream(ext):
            for b0, b1 in evs:
                flush.fill_(1)
                b0.record(ext)
                sim.advance(1)
                b1.record(ext)
        sim.sync()
        barrier()
        ms = sum(b0.elapsed_time(b1) for b0, b1 in evs)
        graph_ms = sim.bench(12, max(600, a.steps))
        del flush
    else:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        sim.advance(a.steps)
        e1.record(ext)
        sim.sync()
        barrier()
        ms = e0.elapsed_time(e1)
    time.sleep(0.15)
    m1 = clocks.mark()
    ms = max_over_ranks(ms, dist, f"cuda:{device}")
    flags = sim.flags()
    final_cells = sim.cells()
    value = whole_job_rate(sites, a.steps, world, ms)
    ms_step = ms / a.steps

    # ---- end to end through the public API with host buffers -------------
    e2e = None
    if not a.no_e2e:
        from pfb200._abi import TRAJ_DTYPE, check, lib
        pin_cells = torch.from_numpy(init_cells.view(np.uint8).copy()).pin_memory()
        pin_phi = torch.from_numpy(init_phi).pin_memory() if init_phi is not None else None
        chunk = 60
        # two halves of a page-locked ring: the host reads one while the
        # device fills the other
        ring = torch.empty((2, chunk, p.num_cells * TRAJ_DTYPE.itemsize), dtype=torch.uint8).pin_memory()
        halves = [ring[h].numpy().view(TRAJ_DTYPE).reshape(chunk, p.num_cells) for h in range(2)]
        phi_out = torch.empty((p.num_cells, 288, 288), dtype=torch.float32).pin_memory()
        L = lib()
        e2e_steps = chunk * max(1, a.steps // chunk)
        done_ev = [torch.cuda.Event(), torch.cuda.Event()]
        track = []  # mean cell position of every recorded step, read on the host
        barrier()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(ext)
        check(L.pfb_sim2d_set_state(sim._h, pin_cells.data_ptr(), pin_phi.data_ptr(), 0),
              "set_state")
        for c in range(e2e_steps // chunk):
            sim.advance_record(chunk, 1, halves[c % 2])
            done_ev[c % 2].record(ext)
            if c:
                done_ev[(c - 1) % 2].synchronize()
                f = halves[(c - 1) % 2]
                track.append((f["cx"].mean(axis=1), f["cy"].mean(axis=1)))
        check(L.pfb_sim2d_get_phi(sim._h, phi_out.data_ptr()), "get_phi")
        f1.record(ext)
        sim.sync()
        f = halves[(e2e_steps // chunk - 1) % 2]
        track.append((f["cx"].mean(axis=1), f["cy"].mean(axis=1)))
        barrier()
        el = max_over_ranks(f0.elapsed_time(f1) / 1000.0, dist, f"cuda:{device}")
        h2d = pin_cells.numel() + pin_phi.numel() * 4
        d2h = p.num_cells * TRAJ_DTYPE.itemsize * e2e_steps + phi_out.numel() * 4
        assert len(track) * chunk == e2e_steps
        e2e = {"value": world * sites * e2e_steps / el, "unit": "site-cell updates/s",
               "h2d_bytes_per_step": h2d / e2e_steps, "d2h_bytes_per_step": d2h / e2e_steps,
               "steps": e2e_steps,
               "note": "state uploaded from pinned host memory once; the trajectory records "
                       "of every step copied to a page-locked ring (pfb_sim2d_advance_record, "
                       "60-step chunks, two halves) and read on the host while the next chunk "
                       "runs; final phi pool read back"}
    clocks.stop()

    if rank == 0:
        peak, peak_src = read_peak_hbm()
        achieved = alg / (ms_step / 1000.0) / 1e9
        traffic = read_ncu_traffic(a.workload) if a.phi_storage == 0 else None
        cpu = None
        if world == 1 and a.cpu_steps > 0:
            # the procedure of --impl reference with this run's warm-up and step
            # count, the steps capped to keep the default run short
            cw, cs = min(a.warmup, 5), min(a.steps, a.cpu_steps)
            v, dt, thr = cpu_time_steps(p, init_cells, init_phi, cw, cs)
            cpu = {"value": v, "unit": "site-cell updates/s", "cores": thr, "kind": "port",
                   "sample": f"{cs} consecutive time steps of the whole workload after {cw} "
                             f"untimed ones ({dt:.2f} s on {thr} threads), the measurement "
                             "of --impl reference"}
        line = {
            "metric": "site-cell updates/s", "value": value, "unit": "site-cell updates/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": ("f32", "f32 arithmetic, f16 phi storage",
                      "f32 arithmetic, bf16 phi storage")[a.phi_storage],
            "data": "synthetic",
            "config": c2_config(a, sites),
            "implementation": {"cluster_ctas_per_cell": a.cluster, "kernel_variant": a.variant,
                               "cuda_graph": not a.no_graph,
                               "phi_storage": ("binary32", "binary16",
                                               "bfloat16")[a.phi_storage]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "pfb::k_step2d<%d, %s, 0, true>" % (
                             a.cluster, ("float", "__half", "__nv_bfloat16")[a.phi_storage]),
                         "algorithmic_bytes_per_launch": alg,
                         "peak_source": peak_src,
                         "duration_source": "CUDA events over the timed region / steps"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clocks.summary(m0, m1),
            # one step kernel per step, plus one bound-settling kernel per advance call
            "gpu_launches": a.steps + (a.steps if a.workload == "c1" else 1),
            "flags": pfb200.flags_report(flags),
            "cells_class_histogram": np.bincount(final_cells["cls"], minlength=6).tolist(),
        }
        if graph_ms is not None:
            line["l2_resident_graph_replay"] = {
                "ms_per_step": graph_ms, "value": sites / (graph_ms / 1000.0),
                "note": "the same steps replayed as six-step CUDA graphs with the state held in L2 "
                        "(no flush): the configuration's steady state in a long run"}
        print(json.dumps(line), flush=True)
    sim.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
