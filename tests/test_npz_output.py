"""Reusable output (pmx_write_npz, the CLI's -npz 1): the NumPy container
stands in for the reference's planned HDF5 export (src/pmx_io.cpp:744-807).
The writer is host code: its tests run on the CPU; the CLI test needs a GPU."""
import os
import subprocess
import zipfile

import numpy as np
import pytest

import picomax_b200 as pm
from conftest import golden_args, load_golden


def test_npz_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    arrays = {"block": rng.standard_normal((3, 3, 2, 6, 7)), "scalar": np.array(-1.25),
              "empty": np.zeros((0, 4)), "vec": rng.standard_normal(2049),
              "transposed": rng.standard_normal((5, 9)).T, "ints": np.arange(12).reshape(3, 4)}
    path = str(tmp_path / "r.npz")
    pm.write_npz(path, arrays)
    with zipfile.ZipFile(path) as zf:
        assert zf.testzip() is None  # every CRC-32 checks
        assert {i.compress_type for i in zf.infolist()} == {zipfile.ZIP_STORED}
    z = np.load(path)
    assert sorted(z.files) == sorted(arrays)
    for k, v in arrays.items():
        assert z[k].dtype == np.float64 and z[k].shape == v.shape
        assert np.array_equal(z[k], np.asarray(v, np.float64))


def test_npz_errors(tmp_path):
    with pytest.raises(pm.PicomaxError) as e:
        pm.write_npz(str(tmp_path / "missing_dir" / "x.npz"), {"a": np.ones(3)})
    assert e.value.status == pm.PMX_ERR_IO
    lib = pm.load()
    assert lib.pmx_write_npz(None, 0, None, None, None, None) == pm.PMX_ERR_INVALID
    # an empty archive is valid
    pm.write_npz(str(tmp_path / "empty.npz"), {})
    assert np.load(str(tmp_path / "empty.npz")).files == []


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["si_band", "si_epsLL"])
def test_cli_npz_matches_dat(name, tmp_path):
    g = load_golden(name)
    args = golden_args(g, tmp_path)
    r = subprocess.run([pm.CLI_PATH] + args + ["-wdir", str(tmp_path), "-outputfile", "out", "-npz", "1"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:]
    dat = np.fromfile(os.path.join(tmp_path, "out.dat"), np.float64)
    z = np.load(os.path.join(tmp_path, "out.npz"))
    p = pm.Problem(args)
    info = p.info
    if name.endswith("band"):
        assert z["eband"].shape == (info.nq, info.nband)
        assert np.array_equal(z["eband"].ravel(), dat)
        assert np.array_equal(z["qpoints"], p.qpoints())
    else:
        npair = info.neps * (info.neps + 1) // 2
        shape = (3, 3, info.nq, npair, info.nfreq)
        assert z["ReXij"].shape == shape and z["ImXij"].shape == shape
        n = z["ReXij"].size
        assert np.array_equal(z["ReXij"].ravel(), dat[:n]) and np.array_equal(z["ImXij"].ravel(), dat[n:])
        k = 0
        for m in range(info.neps):
            for nn in range(m + 1):
                assert tuple(z["pairs"][k]) == (m, nn)
                k += 1
        assert np.allclose(z["freq"], info.dfreq * np.arange(info.nfreq), rtol=0, atol=0)
        G, _ = p.gvectors()
        assert np.array_equal(z["gvec"], G[:info.neps])
        assert np.array_equal(z["qvec"], p.qpoints())
    p.close()
