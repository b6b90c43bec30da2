"""Inputs of the treecode golden vectors (tests/golden/bltc_*.npz), shared by
make_golden_bltc.py and the tests that check against them."""
import numpy as np

EPS = 1e-4
# name: (levels, degree, leaf_size, proxy_degree, theta)
CASES = {"L3_leaf16_n8": (3, 3, 16, 8, 0.7), "L4_leaf64_n6": (4, 3, 64, 6, 0.5),
         "L4_d2_leaf36_n10": (4, 2, 36, 10, 0.8)}


def pots_of(x, y, z):
    """A smooth vorticity-like field on the grid."""
    lat, lon = np.arcsin(np.clip(z, -1, 1)), np.arctan2(y, x)
    return np.sin(lat) - 0.5 * np.sin(lat) * np.cos(lat) ** 4 * 30 * np.cos(4 * lon) + 0.3 * np.sin(3 * x + 2 * y)


def down_in(Pf, qx):
    """Three proxy-target fields, smooth in the panel and proxy indices."""
    p, k = np.meshgrid(np.arange(Pf), np.arange(qx), indexing="ij")
    return [np.cos(0.37 * p + 1.3 * k + f) for f in range(3)]


def divs_of(x, y, z):
    """A smooth divergence-like field on the grid."""
    return 0.4 * np.cos(2 * x - z) + 0.2 * y * z
