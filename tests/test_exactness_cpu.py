"""CPU checks of the numerical facts the GPU activation test relies on.

1. The reference activates a block when kern(d2) > 0, i.e. fl(d2 / 2.25) < 1
   (src/driver/sparse_ops3d_tp.cpp:15-21, 35).  That is the same predicate as
   d2 < 2.25 for every double d2, which lets the GPU drop the division.
2. The FP32 fast path computes d^2 from the cell-local fraction; its error must
   stay far below the 1e-5 band inside which the exact FP64 test decides.
"""
import numpy as np


def test_division_free_activation_predicate():
    x = np.float64(2.25)
    below, above = [x], [x]
    for _ in range(2000):
        below.append(np.nextafter(below[-1], -np.inf))
        above.append(np.nextafter(above[-1], np.inf))
    vals = np.array(below + above + list(np.random.default_rng(0).uniform(0.0, 4.5, 100000)), np.float64)
    assert np.array_equal(vals / np.float64(2.25) < 1.0, vals < 2.25)


def test_fp32_fraction_distance_error_is_inside_the_band():
    rng = np.random.default_rng(1)
    g = rng.uniform(0.0, 512.0, 200000)  # grid coordinates up to a 512^3 lattice
    i0 = np.floor(g)
    fr32 = (g - i0).astype(np.float32)
    worst = 0.0
    for o in range(4):  # candidates i0-1 .. i0+2: d = fr + 1 - o
        d32 = fr32 + np.float32(1 - o)
        d64 = g - (i0 - 1 + o)
        worst = max(worst, float(np.max(np.abs((d32 * d32).astype(np.float64) - d64 * d64))))
    # three axes add up, plus two FP32 additions of sums below 4.5 (half an
    # ulp each); the total must sit well inside the 1e-5 band half-width
    sum_rounding = 2 * float(np.spacing(np.float32(4.5))) / 2
    assert 3 * worst + sum_rounding < 1e-5 / 4
