"""CPU check of the numerical fact the GPU activation test relies on:

the reference activates a block when kern(d2) > 0, i.e. fl(d2 / 2.25) < 1
(src/driver/sparse_ops3d_tp.cpp:15-21, 35).  That is the same predicate as
d2 < 2.25 for every double d2, which lets the GPU drop the division.
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
