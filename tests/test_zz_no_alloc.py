"""pfb_conv3x3_wgrad_noalloc: the weight gradient for callers that cannot
allocate device memory for this library (hosts whose device memory belongs to
their own pool allocator and that forbid a raw cudaMalloc). Its partial sums
live in a fixed 4 MiB array inside the library instead of a caller workspace.

Checked through the C ABI against pfb_conv3x3_wgrad (caller workspace) on two
calls in a row with different shapes, so the second call runs on the scratch
contents the first left behind, within the tolerance of the weight-gradient
tests (1e-5 of the sum of absolute terms, plus 1e-5). This file is collected
last so that a run stopping at its first failure has run everything else."""
import numpy as np
import pytest

import conv_oracle as co
import pfb200
from pfb200 import check, lib

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _bf16(a):
    t = _torch()
    return t.from_numpy(np.ascontiguousarray(a, np.float32)).to(t.bfloat16).cuda().contiguous()


def _case(seed, B, H, W, cx, cy):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((B, H, W, cx))
    dy = rng.standard_normal((B, H, W, cy))
    return _bf16(co.to_padded(x)), _bf16(co.to_padded(dy))


def _with_workspace(xd, dyd, B, H, W, cx, cy):
    t = _torch()
    nbytes = lib().pfb_conv3x3_wgrad_workspace(B, H, W, cx, cy)
    ws = t.zeros(nbytes // 4, dtype=t.float32, device="cuda")
    dw = t.zeros((cy, cx, 3, 3), dtype=t.float32, device="cuda")
    db = t.zeros(cy, dtype=t.float32, device="cuda")
    check(lib().pfb_conv3x3_wgrad(xd.data_ptr(), dyd.data_ptr(), ws.data_ptr(), nbytes,
                                  dw.data_ptr(), db.data_ptr(), B, H, W, cx, cy, None), "wgrad")
    return dw, db


def test_noalloc_matches_workspace_entry_point_on_two_calls():
    t = _torch()
    cases = [(1, 40, 64, 64, 32, 32), (2, 24, 32, 32, 16, 32)]
    for seed, B, H, W, cx, cy in cases:
        xd, dyd = _case(seed, B, H, W, cx, cy)
        dw = t.full((cy, cx, 3, 3), 3.0, dtype=t.float32, device="cuda")
        db = t.full((cy,), 3.0, dtype=t.float32, device="cuda")
        check(lib().pfb_conv3x3_wgrad_noalloc(xd.data_ptr(), dyd.data_ptr(), dw.data_ptr(),
                                              db.data_ptr(), B, H, W, cx, cy, None), "noalloc")
        rw, rb = _with_workspace(xd, dyd, B, H, W, cx, cy)
        t.cuda.synchronize()
        x = xd.float().cpu().numpy()
        dy = dyd.float().cpu().numpy()
        sw, sb = co.conv3x3_wgrad(np.abs(co.from_padded(x, H, W)), np.abs(co.from_padded(dy, H, W)))
        got_w, got_b = dw.cpu().numpy(), db.cpu().numpy()
        ref_w, ref_b = rw.cpu().numpy(), rb.cpu().numpy()
        assert np.all(np.abs(got_w - ref_w) <= 1e-5 * sw + 1e-5)
        assert np.all(np.abs(got_b - ref_b) <= 1e-5 * sb + 1e-5)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    xd, dyd = _case(3, 2, 8, 8, 32, 32)
    with pytest.raises(pfb200.PfbError, match="scratch"):
        # 57 images of 64 x 64 with 32 -> 32 channels need more than 4 MiB
        check(lib().pfb_conv3x3_wgrad_noalloc(xd.data_ptr(), dyd.data_ptr(), xd.data_ptr(), None,
                                              57, 64, 64, 32, 32, None), "noalloc")
