"""Input readers (magma_input.h) and the synthetic workload generators."""
import os
import struct

import numpy as np
import pytest

from conftest import load_pkg


def test_bin_round_trip(tmp_path):
    pkg = load_pkg()
    x = np.random.default_rng(1).normal(size=(123, 5)).astype(np.float32)
    p = str(tmp_path / "a.bin")
    pkg.inputs.write_bin(p, x)
    raw = open(p, "rb").read()
    assert struct.unpack("<ii", raw[:8]) == (123, 5)  # magma_input.h:115-116
    assert len(raw) == 8 + 123 * 5 * 4
    np.testing.assert_array_equal(pkg.inputs.read_input(p), x)


def test_bin_truncated(tmp_path):
    pkg = load_pkg()
    p = str(tmp_path / "t.bin")
    with open(p, "wb") as f:
        f.write(struct.pack("<ii", 10, 3))
        f.write(b"\0" * 16)
    with pytest.raises(ValueError):
        pkg.inputs.read_bin(p)
    with open(p, "wb") as f:
        f.write(b"\1\2")
    with pytest.raises(ValueError):
        pkg.inputs.read_bin(p)


def test_csv_matches_atof_then_float(tmp_path):
    pkg = load_pkg()
    p = str(tmp_path / "a.csv")
    vals = [["0.1", "1e-3", "-2.5"], ["3.14159265358979", "7", "1e30"]]
    with open(p, "w") as f:
        for row in vals:
            f.write(" ".join(row) + "\n")
    x = pkg.inputs.read_input(p)
    assert x.dtype == np.float32 and x.shape == (2, 3)
    np.testing.assert_array_equal(x, np.array([[float(v) for v in r] for r in vals], np.float64).astype(np.float32))


def test_hdf5_unsupported(tmp_path):
    pkg = load_pkg()
    with pytest.raises(RuntimeError):
        pkg.inputs.read_input(str(tmp_path / "x.h5"))


def test_generators_are_seeded_and_shaped():
    pkg = load_pkg()
    a = pkg.synthetic.config1(n=5000)
    b = pkg.synthetic.config1(n=5000)
    np.testing.assert_array_equal(a.coords, b.coords)
    assert a.coords.dtype == np.float32 and a.coords.shape == (5000, 2)
    assert (a.eps, a.min_pts) == (0.8, 5)
    c = pkg.synthetic.config2(n=20000)
    assert c.coords.shape == (20000, 3) and (c.eps, c.min_pts) == (1.5, 10)
    d = pkg.synthetic.config3(n=20000)
    assert d.coords.shape == (20000, 8) and (d.eps, d.min_pts) == (1.2, 8)
    e = pkg.synthetic.config5(n=50000)
    assert e.coords.shape == (50000, 2) and (e.eps, e.min_pts) == (0.5, 4)
    assert np.isfinite(e.coords).all()
