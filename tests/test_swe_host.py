"""Host-side pieces of the shallow-water path, on the CPU: the hashed
grid-point map against the reference's own cubed_sphere_2d_to_1d output, and
the configuration key for the height-Laplacian factor."""
import os

import numpy as np
import pytest

from conftest import GOLDEN


def test_grid_point_map_matches_reference(sb):
    for name in ("swe_L3.npz", "swe_L4_d2.npz"):
        gd = dict(np.load(os.path.join(GOLDEN, name)))
        m, counts = sb.cubed_sphere_2d_to_1d(gd["x"], gd["y"], gd["z"], int(gd["degree"]))
        assert np.array_equal(m, gd["map"]), name
        assert np.array_equal(counts, gd["counts"]), name


def test_grid_point_map_counts_at_levels_7():
    import importlib

    sb = importlib.import_module("spectral_bslpm_b200")
    g = sb.build_grid(7, 3, exact_cc=False)
    m, counts = sb.cubed_sphere_2d_to_1d(g.x, g.y, g.z, 3)
    A = g.x.shape[0]
    assert len(counts) == A * 9 + 2  # distinct points of the cubed-sphere grid
    # 8 cube corners are shared by 3 panels; other panel corners by 4, edge points by 2
    assert np.bincount(counts).tolist() == [0, A * 4, A * 4, 8, A - 6]
    assert counts.sum() == A * 16


def test_g_over_a_default_and_namelist(sb, tmp_path):
    cfg = sb.config_default()
    assert cfg.g_over_a == 9.81 / 6371000.0
    p = tmp_path / "namelist.txt"
    p.write_text("levels=4\ng_over_a=1.0\nend\n")
    cfg = sb.read_run_config(str(p))
    assert cfg.levels == 4 and cfg.g_over_a == 1.0


def test_forcing_namelist_keys(sb, tmp_path):
    """forcing=1 with forcing_type ssw / ssw2 (src/io_utils.cpp:69-74)."""
    p = tmp_path / "namelist.txt"
    for text, want in (("forcing=1\nforcing_type=ssw2\nend\n", sb.FORCING_SSW2),
                       ("forcing_type=ssw\nforcing=1\nend\n", sb.FORCING_SSW),
                       ("forcing=0\nforcing_type=ssw\nend\n", sb.FORCING_NONE)):
        p.write_text(text)
        assert sb.read_run_config(str(p)).forcing == want
    p.write_text("forcing=1\nforcing_type=other\nend\n")
    with pytest.raises(sb.SbslpmError):
        sb.read_run_config(str(p))
