"""Input formats of the reference, read the way existing cases write them.

map.xyz (src/io.rs:60-68, 121-143): whitespace-separated 0/1 tokens, one line
per image row, blank lines between z-slices; aux/image_pre_processing.py:42-56
writes image row 0 first, and the reader reverses the lines of each slice, so
the last line of a slice is y = 0.  Anything but 0/1 is an error
(src/io.rs:88-96).
"""
import os

import numpy as np
import pytest

from lbflow_b200 import io
from lbflow_b200 import momentum as m


def write_like_image_pre_processing(path, slices):
    """One slice per image, as write_bounce_back_map_file writes it (each row
    ends with a newline, tokens separated by one space); slices are joined by a
    blank line.  slices[z][r][x] is image row r (row 0 at the top)."""
    with open(path, "w") as fh:
        for z, img in enumerate(slices):
            if z:
                fh.write("\n")
            for row in img:
                fh.write(" ".join(str(int(v)) for v in row) + "\n")


def test_map_xyz_reference_layout_2d(tmp_path, monkeypatch):
    rng = np.random.default_rng(5)
    img = (rng.random((7, 11)) < 0.3).astype(np.uint8)       # 7 image rows, 11 columns
    os.makedirs(tmp_path / "pre_processing")
    write_like_image_pre_processing(tmp_path / "pre_processing" / "map.xyz", [img])
    monkeypatch.chdir(tmp_path)
    mask = m.NodeTypes.FromBounceBackMapFile.generate([11, 7])
    # node (x, y) = image row ny - 1 - y, column x
    want = img[::-1].ravel()
    assert mask.dtype == np.uint8 and np.array_equal(mask, want)


def test_map_xyz_reference_layout_3d(tmp_path, monkeypatch):
    rng = np.random.default_rng(6)
    nx, ny, nz = 9, 5, 4
    slices = [(rng.random((ny, nx)) < 0.4).astype(np.uint8) for _ in range(nz)]
    os.makedirs(tmp_path / "pre_processing")
    write_like_image_pre_processing(tmp_path / "pre_processing" / "map.xyz", slices)
    monkeypatch.chdir(tmp_path)
    mask = m.NodeTypes.FromBounceBackMapFile.generate([nx, ny, nz])
    want = np.stack([s[::-1] for s in slices]).ravel()      # z slowest, then y, then x
    assert np.array_equal(mask, want)
    # the writer is the reader's inverse
    assert np.array_equal(io.parse_bounce_back_map(io.format_bounce_back_map(want, [nx, ny, nz])), want)


def test_map_xyz_tolerates_extra_whitespace(tmp_path):
    text = "  0 1\t1\n1 0 0  \n\n\n0 0 1\n1 1 1\n\n"
    got = io.parse_bounce_back_map(text)
    assert got.tolist() == [1, 0, 0, 0, 1, 1, 1, 1, 1, 0, 0, 1]


def test_map_xyz_rejects_bad_tokens():
    with pytest.raises(ValueError, match="Invalid node type"):
        io.parse_bounce_back_map("0 1\n2 0\n")


def test_map_xyz_size_mismatch(tmp_path, monkeypatch):
    os.makedirs(tmp_path / "pre_processing")
    write_like_image_pre_processing(tmp_path / "pre_processing" / "map.xyz", [np.zeros((3, 3), np.uint8)])
    monkeypatch.chdir(tmp_path)
    with pytest.raises(ValueError, match="does not match"):
        m.NodeTypes.FromBounceBackMapFile.generate([4, 3])


def test_from_time_step_reads_data_dir(tmp_path, monkeypatch):
    """InitialDensity/InitialVelocity::FromTimeStep(t) read data/<t>/density.csv and
    velocity.csv (src/momentum/io.rs:358-394, src/io.rs:145-175)."""
    rng = np.random.default_rng(1)
    rho = 1.0 + 1e-3 * rng.standard_normal(12)
    u = 1e-2 * rng.standard_normal((12, 2))
    io.write_step_data(40, rho, u, root=str(tmp_path / "data"))
    monkeypatch.chdir(tmp_path)
    got_r = m.InitialDensity.FromTimeStep(40).generate([4, 3])
    got_u = m.InitialVelocity.FromTimeStep(40).generate([4, 3])
    # {:.8e} text keeps 9 significant digits
    assert np.allclose(got_r, rho, rtol=1e-8, atol=0) and np.allclose(got_u, u, rtol=1e-8, atol=1e-12)
