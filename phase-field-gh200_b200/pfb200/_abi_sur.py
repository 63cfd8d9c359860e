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
})
