"""Batched ensemble of independent 2D systems advanced by one kernel launch
per step (``pfb_ens2d_*`` in ``include/pfb200.h``)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._abi import TRAJ_DTYPE, Params2D, check, lib
from .sim2d import Sim2D, SimParams2D


class Ensemble2D:
    def __init__(self, params: list[SimParams2D], centres: list[tuple[np.ndarray, np.ndarray]],
                 *, device: int = 0, cluster: int = 0):
        R = len(params)
        assert R == len(centres) and R > 0
        for p in params:
            p.validate()
        self.params = params
        self._pc = (Params2D * R)(*[p.to_c() for p in params])
        self._cx = [np.ascontiguousarray(c[0], dtype=np.float32) for c in centres]
        self._cy = [np.ascontiguousarray(c[1], dtype=np.float32) for c in centres]
        cxp = (C.c_void_p * R)(*[a.ctypes.data for a in self._cx])
        cyp = (C.c_void_p * R)(*[a.ctypes.data for a in self._cy])
        h = lib().pfb_ens2d_create(R, self._pc, cxp, cyp, device)
        if not h:
            raise RuntimeError("pfb_ens2d_create failed: " + lib().pfb_last_error().decode())
        self._h = h
        if cluster:
            self.set_cluster(cluster)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().pfb_ens2d_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - interpreter teardown order
        try:
            self.close()
        except Exception:
            pass

    def __len__(self) -> int:
        return len(self.params)

    def set_cluster(self, k: int) -> None:
        check(lib().pfb_ens2d_set_cluster(self._h, k), "set_cluster")

    def autotune(self, steps: int = 12) -> int:
        k = C.c_int()
        check(lib().pfb_ens2d_autotune(self._h, steps, C.byref(k)), "autotune")
        return k.value

    def advance(self, steps: int) -> None:
        check(lib().pfb_ens2d_advance(self._h, steps), "advance")

    @property
    def total_cells(self) -> int:
        return int(sum(p.num_cells for p in self.params))

    @property
    def stream(self) -> int:
        return int(lib().pfb_ens2d_stream(self._h) or 0)

    def advance_record(self, steps: int, every: int, ring: np.ndarray) -> None:
        """Advance every system `steps` steps; frame k % len(ring) of `ring`
        (a C-contiguous (frames, total_cells) TRAJ_DTYPE array, ideally in
        page-locked memory) receives the trajectory records of all systems,
        system 0 first, after every `every`-th step. Valid after sync()."""
        if ring.dtype != TRAJ_DTYPE or ring.ndim != 2 or ring.shape[1] != self.total_cells or \
                not ring.flags.c_contiguous:
            raise ValueError("ring must be a C-contiguous (frames, total_cells) TRAJ_DTYPE array")
        check(lib().pfb_ens2d_advance_record(self._h, steps, every, ring.ctypes.data, ring.shape[0]),
              "advance_record")

    def advance_serial(self, steps: int) -> None:
        check(lib().pfb_ens2d_advance_serial(self._h, steps), "advance_serial")

    def sync(self) -> None:
        check(lib().pfb_ens2d_sync(self._h), "sync")

    @property
    def step(self) -> int:
        return int(lib().pfb_ens2d_step(self._h))

    def bench(self, warmup: int, steps: int, serial: bool = False) -> float:
        ms = C.c_double()
        check(lib().pfb_ens2d_bench(self._h, warmup, steps, int(serial), C.byref(ms)), "bench")
        return ms.value

    def system(self, r: int) -> Sim2D:
        """System r as a (non-owning) Sim2D for reading its state."""
        h = lib().pfb_ens2d_system(self._h, r)
        if not h:
            raise IndexError(lib().pfb_last_error().decode())
        return Sim2D._view(h, self.params[r])
