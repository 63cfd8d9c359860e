"""Learned relaxation surrogate of the 2D update (``include/pfb200_surrogate.h``):
the U-Net on tcgen05 convolutions, its training data from plain-solver pairs,
training, and a relaxation driver in which the plain solver judges every
surrogate jump by its residual and is the fallback. No counterpart in the
reference, which relaxes with the explicit step only.

Device buffers are torch tensors (memory only); every computation is a call
into ``libpfb200.so``.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from ._abi import check, lib
from .sim2d import Sim2D, SimParams2D, fatal, palmieri_centres

CROP = 64
PADDED = (CROP + 2) * (CROP + 2)
IN_CH = 16


def _torch():
    import torch
    return torch


class Surrogate2D:
    """The U-Net (pfb_sur2d) on one device."""

    def __init__(self, max_batch: int = 256, seed: int = 1, device: int = 0):
        h = lib().pfb_sur2d_create(max_batch, seed, device)
        if not h:
            raise RuntimeError("pfb_sur2d_create failed: " + lib().pfb_last_error().decode())
        self._h = h
        self.max_batch = max_batch
        self.device = device

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().pfb_sur2d_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - interpreter teardown order
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_params(self) -> int:
        return int(lib().pfb_sur2d_num_params(self._h))

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.num_params, np.float32)
        check(lib().pfb_sur2d_get_params(self._h, out.ctypes.data), "get_params")
        return out

    def set_params(self, flat: np.ndarray) -> None:
        flat = np.ascontiguousarray(flat, np.float32)
        assert flat.size == self.num_params
        check(lib().pfb_sur2d_set_params(self._h, flat.ctypes.data), "set_params")

    def train_step(self, x_all, t_all, idx, lr: float, want_loss: bool = True):
        loss = C.c_double()
        check(lib().pfb_sur2d_train_step(self._h, x_all.data_ptr(), t_all.data_ptr(),
                                         idx.data_ptr(), int(idx.numel()), lr,
                                         C.byref(loss) if want_loss else None), "train_step")
        return loss.value if want_loss else None

    def predict(self, x0, dphi, batch: int) -> None:
        check(lib().pfb_sur2d_predict(self._h, x0.data_ptr(), dphi.data_ptr(), batch), "predict")

    def jump(self, sim: Sim2D, history: int = 0) -> None:
        """Jump every cell of `sim`; with history > 0 the network also sees
        the rate over that many plain steps, which the jump takes first."""
        if history > 0:
            check(lib().pfb_sur2d_jump_history(self._h, sim._h, history,
                                               1.0 / (history * sim.params.dt)), "jump")
        else:
            check(lib().pfb_sur2d_jump(self._h, sim._h), "jump")

    def sync(self) -> None:
        check(lib().pfb_sur2d_sync(self._h), "sync")

    def bench_forward(self, batch: int, iters: int) -> float:
        ms = C.c_double()
        check(lib().pfb_sur2d_bench_forward(self._h, batch, iters, C.byref(ms)), "bench_forward")
        return ms.value


def forward_flops(batch: int) -> float:
    """Multiply-add work of one forward pass as the kernels run it (padded
    channels and the two computed border columns of every row included), x 2."""
    full, half = 64 * 66, 32 * 34
    macs = full * 9 * (16 * 32 + 32 * 32 * 4 + 32 * 16) + half * 9 * 32 * 32 * 2
    return 2.0 * macs * batch


def relaxation_params(L: int = 1024, N: int = 400, R: float = 12.0, seed: int = 1) -> SimParams2D:
    """Passive relaxation (no active speed) at the given lattice and cells."""
    return SimParams2D(L=L, num_cells=N, target_radius=R, seed=seed, v_A=0.0)


@dataclass
class Dataset:
    x: object  # torch bf16 (n, 66 * 66, 16) on the device
    t: object  # torch f32 (n, 64, 64): phi increment over `interval` steps
    interval: int
    runs: int
    pairs_per_run: int
    seconds: float


def make_dataset(p: SimParams2D, runs: int, pairs_per_run: int, interval: int,
                 seed0: int = 100, device: int = 0, history: int = 0) -> Dataset:
    """Plain-solver pairs: for each run (fresh start, seed seed0 + r), crops of
    every cell at steps 0, interval, 2 interval, ... and the increment of
    phi_n on the same crop `interval` steps later. With history > 0 each
    input is taken `history` steps after the crop that gives its rate
    channel (the pairs are then interval + history steps apart)."""
    t = _torch()
    dev = f"cuda:{device}"
    N = p.num_cells
    n = runs * pairs_per_run * N
    x_all = t.zeros((n, PADDED, IN_CH), dtype=t.bfloat16, device=dev)
    t_all = t.zeros((n, CROP, CROP), dtype=t.float32, device=dev)
    pc = t.zeros((N, CROP, CROP), dtype=t.float32, device=dev)
    org = t.zeros((N, 2), dtype=t.int32, device=dev)
    t0 = time.perf_counter()
    k = 0
    for r in range(runs):
        q = SimParams2D(**{**p.__dict__, "seed": seed0 + r})
        cx, cy = palmieri_centres(N, q.L, 2 * q.target_radius, q.seed)
        sim = Sim2D(q, cx, cy, device=device)
        for _ in range(pairs_per_run):
            check(lib().pfb_sur2d_extract(sim._h, x_all[k:k + N].data_ptr(), pc.data_ptr(),
                                          org.data_ptr()), "extract")
            if history > 0:
                sim.advance(history)
                prev = pc.clone()
                check(lib().pfb_sur2d_extract_at(sim._h, org.data_ptr(), prev.data_ptr(),
                                                 1.0 / (history * q.dt),
                                                 x_all[k:k + N].data_ptr(), pc.data_ptr()),
                      "extract_at")
            sim.advance(interval)
            check(lib().pfb_sur2d_crop_phi(sim._h, org.data_ptr(), pc.data_ptr(),
                                           t_all[k:k + N].data_ptr()), "crop_phi")
            k += N
        sim.sync()
        if fatal(sim.flags()):
            raise RuntimeError("a training run raised a fatal flag")
        sim.close()
    t.cuda.synchronize(device)
    return Dataset(x_all, t_all, interval, runs, pairs_per_run, time.perf_counter() - t0)


def train(net: Surrogate2D, data: Dataset, steps: int, batch: int, lr: float = 5e-4,
          seed: int = 0, log_every: int = 100) -> list[tuple[int, float]]:
    """Adam with a cosine-decayed learning rate on random batches; returns
    (step, loss) every log_every steps."""
    t = _torch()
    n = data.x.shape[0]
    g = t.Generator(device="cpu").manual_seed(seed)
    dev = data.x.device
    hist = []
    for s in range(steps):
        idx = t.randint(0, n, (batch,), generator=g, dtype=t.int32).to(dev)
        want = (s % log_every == 0) or s == steps - 1
        cur = lr * 0.5 * (1.0 + np.cos(np.pi * s / steps))
        loss = net.train_step(data.x, data.t, idx, cur, want)
        if want:
            hist.append((s, loss))
    net.sync()
    return hist


@dataclass
class RelaxResult:
    reached: bool
    residual: float
    solver_steps: int       # plain steps taken (judging branches included)
    equivalent_steps: int   # plain steps kept plus `interval` per accepted jump
    seconds: float          # wall time, synchronised at every check
    jumps_accepted: int = 0
    jumps_rejected: int = 0
    history: list = field(default_factory=list)  # (solver steps, seconds, residual)


def relax(sim: Sim2D, target: float, max_solver_steps: int, check_every: int = 500,
          net: Surrogate2D | None = None, interval: int = 2000, heal: int = 200,
          history: int = 0, retry_every: int = 0) -> RelaxResult:
    """Relax `sim` until the step residual max |dphi / dt| <= target, or until
    max_solver_steps plain steps were taken.

    Plain: check_every steps between residual measurements. With `net`, each
    segment is judged by the plain solver: from a saved state it first takes
    `history + heal` plain steps and measures the residual, then returns to
    the saved state, jumps by the network (trained on `interval`-step
    increments; the jump takes the `history` steps of its rate input first),
    takes `heal` steps and measures again. The jump is kept only if
    its residual is lower and no fatal flag was raised; otherwise the state is
    restored and the run continues with the plain solver alone, trying the
    network again after retry_every plain steps (never when 0)."""
    t0 = time.perf_counter()
    res = RelaxResult(False, float("inf"), 0, 0, 0.0)
    r, _ = sim.residual_step()
    res.solver_steps += 1
    res.equivalent_steps += 1
    use_net = net is not None
    retry_at = -1
    while True:
        res.history.append((res.solver_steps, time.perf_counter() - t0, r))
        if r <= target:
            res.reached = True
            break
        if res.solver_steps >= max_solver_steps:
            break
        if net is not None and not use_net and retry_at >= 0 and res.solver_steps >= retry_at:
            use_net = True
        if use_net:
            sim.save()
            sim.advance(history + heal - 1)
            r_plain, _ = sim.residual_step()
            sim.restore()
            net.jump(sim, history)
            sim.advance(heal - 1)
            r_jump, _ = sim.residual_step()
            res.solver_steps += 2 * (history + heal)
            if r_jump < r_plain and not fatal(sim.flags()):
                res.jumps_accepted += 1
                res.equivalent_steps += interval + history + heal
                r = r_jump
                continue
            sim.restore()
            res.jumps_rejected += 1
            use_net = False
            retry_at = res.solver_steps + retry_every if retry_every > 0 else -1
        sim.advance(check_every - 1)
        r, _ = sim.residual_step()
        res.solver_steps += check_every
        res.equivalent_steps += check_every
    res.residual = r
    res.seconds = time.perf_counter() - t0
    return res
