"""MATLAB v7.3 (HDF5) .mat files, read without h5py (utils/io.py:25-69).

The reader (h5mat.read_mat73) is pinned to a file MATLAB wrote: scipy's
test data holds `testdouble` saved by MATLAB 7.4 as v7.3 (HDF5) and the same
variable in the v4 - v7 formats that scipy's loadmat reads; both must agree
exactly.  Files from the test writer (tests/h5write.py, the subset MATLAB
uses: symbol-table groups, contiguous and chunked layouts with shuffle +
deflate, compound {real, imag}) cover 3-D stacks, complex arrays, groups and
the ptychography loader's v7.3 branch, with the reference's transposition
and gap decimation (utils/io.py:115-120).
"""
import glob
import importlib
import os

import numpy as np
import pytest

from conftest import load_pkg
from h5write import write_mat73

def _recovery():
    return importlib.import_module(load_pkg().__name__ + ".recovery")


SCIPY_DATA = os.path.join(os.path.dirname(__import__("scipy.io.matlab").io.matlab.__file__), "tests", "data")


def test_reads_a_file_matlab_wrote():
    h5 = load_pkg().h5mat
    v73 = os.path.join(SCIPY_DATA, "testhdf5_7.4_GLNX86.mat")
    if not os.path.exists(v73):
        pytest.skip("scipy's MATLAB test files are not installed")
    from scipy.io import loadmat
    assert h5.is_hdf5(v73)
    got = h5.read_mat73(v73)
    assert list(got) == ["testdouble"]
    twins = sorted(glob.glob(os.path.join(SCIPY_DATA, "testdouble_*.mat")))
    assert twins
    for f in twins:
        want = loadmat(f)["testdouble"]
        assert got["testdouble"].shape == want.shape == (1, 9)
        assert np.array_equal(got["testdouble"], want), f
    # and through the loader's read_data, which falls back from loadmat to it
    rd = _recovery().read_data(v73)
    assert np.array_equal(rd["testdouble"], got["testdouble"])


@pytest.mark.parametrize("chunked", [False, True])
def test_round_trip_arrays_and_groups(tmp_path, chunked):
    h5 = load_pkg().h5mat
    rng = np.random.default_rng(1)
    v = {
        "d2": rng.standard_normal((5, 7)),
        "s3": rng.standard_normal((6, 4, 9)).astype(np.float32),
        "z2": (rng.standard_normal((8, 3)) + 1j * rng.standard_normal((8, 3))),
        "c3": (rng.standard_normal((4, 4, 5)) + 1j * rng.standard_normal((4, 4, 5))).astype(np.complex64),
        "row": np.arange(11.0)[None, :],
        "grp": {"a": rng.standard_normal((3, 2)), "#refs#": np.zeros((1, 1))},
        "cplx": {"real": rng.standard_normal((2, 5)), "imag": rng.standard_normal((2, 5))},
    }
    chunks = {"d2": (2, 3), "s3": (4, 3, 2), "z2": (8, 3), "c3": (3, 2, 5), "row": (1, 4)} if chunked else None
    p = str(tmp_path / "v.mat")
    write_mat73(p, v, chunks=chunks)
    got = h5.read_mat73(p)
    assert set(got) == set(v)
    for k in ("d2", "s3", "z2", "c3", "row"):
        assert got[k].shape == v[k].shape and np.array_equal(got[k], v[k]), k
        assert got[k].dtype.kind == v[k].dtype.kind
    assert set(got["grp"]) == {"a"} and np.array_equal(got["grp"]["a"], v["grp"]["a"])
    assert np.array_equal(got["cplx"], v["cplx"]["real"] + 1j * v["cplx"]["imag"])
    assert set(h5.read_mat73(p, "z2")) == {"z2"}


def test_ptychography_loader_reads_v73(tmp_path):
    """A bundle saved with -v7.3: locations, complex probe and object, a raw
    stack [M, M, F] stored chunked per frame with deflate; gap 2."""
    rec = _recovery()
    rng = np.random.default_rng(2)
    M, F = 16, 10
    bundle = {
        "xlocation": rng.uniform(-5, 5, (1, F)),
        "ylocation": rng.uniform(-5, 5, (1, F)),
        "probe": (rng.standard_normal((M, M)) + 1j * rng.standard_normal((M, M))),
        "imRaw": rng.poisson(20.0, (M, M, F)).astype(np.float64),
        "obj": (rng.standard_normal((40, 40)) + 1j * rng.standard_normal((40, 40))),
    }
    write_mat73(str(tmp_path / "bundle.mat"), bundle, chunks={"imRaw": (M, M, 1), "obj": (20, 20)})
    d = rec.load_ptychography_data(str(tmp_path), bundle_file="bundle.mat", gap=2)
    assert np.array_equal(d["xlocation"], bundle["xlocation"].squeeze()[::2])
    assert np.array_equal(d["ylocation"], bundle["ylocation"].squeeze()[::2])
    assert np.array_equal(d["probe"], bundle["probe"])
    assert np.array_equal(d["imRaw"], bundle["imRaw"][:, :, ::2])
    assert np.array_equal(d["obj"], bundle["obj"])


def test_not_hdf5_and_unsupported(tmp_path):
    h5 = load_pkg().h5mat
    p = tmp_path / "x.bin"
    p.write_bytes(b"\x00" * 2048)
    assert not h5.is_hdf5(str(p))
    with pytest.raises(h5.H5Error):
        h5.read_mat73(str(p))
