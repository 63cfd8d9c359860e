"""ctypes signatures of the surrogate entry points (``include/pfb200_surrogate.h``)."""
from __future__ import annotations

import ctypes as C

from . import _abi

P = C.c_void_p
I = C.c_int

_abi._SIGS.update({
    "pfb_conv3x3_forward": (I, [P, P, P, P, P, P, I, I, I, I, I, I, P]),
    "pfb_conv3x3_pack": (I, [P, P, I, I, I, P]),
    "pfb_conv3x3_wgrad_workspace": (C.c_size_t, [I, I, I, I, I]),
    "pfb_conv3x3_wgrad": (I, [P, P, P, C.c_size_t, P, P, I, I, I, I, I, P]),
    "pfb_conv3x3_wgrad_noalloc": (I, [P, P, P, P, I, I, I, I, I, P]),
    "pfb_conv_status": (I, [C.POINTER(C.c_uint), I]),
    "pfb_conv_set_pipeline": (C.c_int, [C.c_int]),
    "pfb_sim2d_residual_step": (I, [P, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "pfb_sur2d_extract": (I, [P, P, P, P]),
    "pfb_sur2d_extract_at": (I, [P, P, P, C.c_float, P, P]),
    "pfb_sur2d_jump_history": (I, [P, P, I, C.c_float]),
    "pfb_sur2d_crop_phi": (I, [P, P, P, P]),
    "pfb_sur2d_insert": (I, [P, P, P]),
    "pfb_sur2d_create": (P, [I, C.c_ulonglong, I]),
    "pfb_sur2d_destroy": (None, [P]),
    "pfb_sur2d_num_params": (C.c_longlong, [P]),
    "pfb_sur2d_get_params": (I, [P, P]),
    "pfb_sur2d_set_params": (I, [P, P]),
    "pfb_sur2d_get_grads": (I, [P, P]),
    "pfb_sur2d_predict": (I, [P, P, P, I]),
    "pfb_sur2d_loss_grad": (I, [P, P, P, P, I, C.POINTER(C.c_double)]),
    "pfb_sur2d_train_step": (I, [P, P, P, P, I, C.c_float, C.POINTER(C.c_double)]),
    "pfb_sur2d_sync": (I, [P]),
    "pfb_sur2d_jump": (I, [P, P]),
    "pfb_sur2d_bench_forward": (I, [P, I, I, C.POINTER(C.c_double)]),
})
