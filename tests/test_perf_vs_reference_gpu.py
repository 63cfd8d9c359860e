"""Step time of the B200 kernel against the reference's own CUDA kernel
(compiled for sm_100a from the reference sources into oracle/_ref), on the same
device state: the 2048² / 1024-cell workload of bench.py and the 512² / 64-cell
case. Both run through caller-owned buffers (DeviceState2D) on the default
stream and are timed with CUDA events after a warm-up; the B200 kernel must
not be slower."""
import ctypes as C

import numpy as np
import pytest

import pfb200
import oracle2d
from helpers2d import DeviceState2D, params

pytestmark = pytest.mark.gpu

CASES = {
    "2048sq_1024cells": dict(L=2048, N=1024, min_sep=24.0, slack=1.0),
    "512sq_64cells": dict(L=512, N=64, min_sep=24.0, slack=1.25),
}


def _time_steps(ds, launch, steps):
    import torch
    for _ in range(5):
        ds.step_with(launch)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        ds.step_with(launch)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


@pytest.mark.skipif(not oracle2d.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("case", list(CASES))
def test_step_time_vs_reference_kernel(case):
    c = CASES[case]
    p = params(c["L"], c["N"], seed=1234)
    cx, cy = pfb200.palmieri_centres(p.num_cells, p.L, c["min_sep"], p.seed)
    sim = pfb200.Sim2D(p, cx, cy)
    cells, phi = sim.cells(), sim.phi()
    sim.close()

    def launch_pfb(a):
        return pfb200.lib().pfb_step2d_launch(C.byref(a), 0, None)

    grid = oracle2d.rlib().ref2d_grid(0)

    def launch_ref(a):
        return oracle2d.rlib().ref2d_launch_step(C.byref(a), grid, None)

    steps = 200
    t_pfb = _time_steps(DeviceState2D(p, cells, phi), launch_pfb, steps)
    t_ref = _time_steps(DeviceState2D(p, cells, phi), launch_ref, steps)
    print(f"\n[{case}] pfb {t_pfb * 1e3:.1f} us/step, reference kernel {t_ref * 1e3:.1f} us/step,"
          f" speed-up {t_ref / t_pfb:.2f}x")
    assert np.isfinite(t_pfb) and np.isfinite(t_ref)
    assert t_pfb <= t_ref * c["slack"]
