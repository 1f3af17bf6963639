"""The VTK XML writers of util/io_utils.py (the reference's output formats,
io_utils.py:29-139) round-trip through their reader.  CPU only."""
import os

import numpy as np


def test_vti_4channel_roundtrip(tmp_path):
    from util.io_utils import read_vtk, write_vtks_4channel_smoke
    rng = np.random.default_rng(0)
    w = rng.normal(size=(5, 4, 3)).astype(np.float32)
    smoke = rng.uniform(size=(5, 4, 3, 4)).astype(np.float32)
    write_vtks_4channel_smoke(w, smoke, str(tmp_path), 7)
    d = read_vtk(os.path.join(tmp_path, "field_0007.vti"))
    assert d["_extent"] == [0, 4, 0, 3, 0, 2]
    # points in x-fastest order, as vtk's numpy_to_vtk(ravel(order="F"))
    np.testing.assert_array_equal(d["vorticity"], w.ravel(order="F"))
    assert d["smoke"].shape == (60, 4)
    np.testing.assert_array_equal(d["smoke"][1], smoke[1, 0, 0])
    np.testing.assert_array_equal(d["smoke"][5], smoke[0, 1, 0])
    np.testing.assert_array_equal(d["smoke"][20], smoke[0, 0, 1])


def test_vtu_particles_roundtrip(tmp_path):
    from util.io_utils import read_vtk, write_to_vtks_lp
    pos = np.random.default_rng(1).uniform(size=(11, 3)).astype(np.float32)
    speed = np.arange(11, dtype=np.float32)
    write_to_vtks_lp(pos, {"speed": speed}, {"vel": pos * 2}, os.path.join(tmp_path, "field_003"))
    d = read_vtk(os.path.join(tmp_path, "field_003.vtu"))
    assert d["_npoints"] == 11
    np.testing.assert_array_equal(d["points"], pos)
    np.testing.assert_array_equal(d["connectivity"], np.arange(11))
    np.testing.assert_array_equal(d["offsets"], np.arange(1, 12))
    assert (d["types"] == 1).all()
    np.testing.assert_array_equal(d["speed"], speed)
    np.testing.assert_array_equal(d["vel"], pos * 2)
