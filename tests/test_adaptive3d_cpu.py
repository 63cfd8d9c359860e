"""Tier rules of adaptive 3D bricks (growth and centred crop) against the
values of the reference's brick-class test
(tests/3d/brick_classes_cpu_test.cpp:27-62)."""
import ctypes as C

import pfb200


def test_tier_rules_match_reference_values():
    """Values of the reference's brick-class test
    (tests/3d/brick_classes_cpu_test.cpp:27-62)."""
    L = pfb200.lib()
    for cur, mx, want in ((144, 512, 176), (176, 512, 208), (208, 512, 240), (152, 512, 192),
                          (224, 250, 248), (224, 231, 0), (224, 224, 0), (145, 512, 0), (0, 512, 0)):
        assert L.pfb3d_next_brick_edge(cur, mx) == want, (cur, mx)
    def shrink(cur, mn, lo, hi):
        a = (C.c_int * 3)(*lo) if lo is not None else None
        b = (C.c_int * 3)(*hi)
        return L.pfb3d_shrink_brick_edge(cur, mn, a, b)
    assert shrink(224, 144, (80,) * 3, (143,) * 3) == 144
    assert shrink(224, 144, (32,) * 3, (191,) * 3) == 192
    assert shrink(224, 144, (8, 80, 80), (100, 143, 143)) == 224
    assert shrink(224, 152, (64,) * 3, (159,) * 3) == 152
    assert shrink(224, 144, (80,) * 3, (-1,) * 3) == 224
    assert shrink(224, 144, None, (143,) * 3) == 224
