"""PDEP database files: layout of WEST's pdep_merge_and_write_G / pdep_db_write
(IO_kernel/pdep_io.f90:35-150, IO_kernel/pdep_db.f90:56-200), read back by an
independent NumPy reader and by wb_pdep_db_read.  Host-only, no GPU."""
import json
import os

import numpy as np
import pytest

from west_b200.pdep import cubic_cell, pdep_db_read, pdep_db_write


def _data(npw=97, n=5, seed=3):
    rng = np.random.default_rng(seed)
    vec = rng.standard_normal((npw, n)) + 1j * rng.standard_normal((npw, n))
    ev = -np.sort(rng.random(n))[::-1] * 3.0
    return ev, np.asfortranarray(vec)


def test_files_follow_west_layout(tmp_path):
    ev, vec = _data()
    pdep_db_write(str(tmp_path), ev, vec, cubic_cell(20.0))
    names = sorted(os.listdir(tmp_path))
    assert names == [f"Q{1:09d}E{j:09d}.dat" for j in range(1, 6)] + ["summary.json"]
    for j in range(5):
        raw = np.fromfile(tmp_path / f"Q000000001E{j + 1:09d}.dat", dtype=np.uint8)
        hdr = raw[:128].view(np.int32)
        assert hdr[0] == 210405 and hdr[1] == 1 and hdr[2] == 97 and not hdr[3:].any()
        assert raw.size == 128 + 97 * 16
        np.testing.assert_array_equal(raw[128:].view(np.complex128), vec[:, j])
    sm = json.load(open(tmp_path / "summary.json"))["dielectric_matrix"]
    assert sm["domain"]["a1"] == [20.0, 0.0, 0.0]
    assert abs(sm["domain"]["b1"][0] - 2 * np.pi / 20.0) < 1e-15
    entry = sm["pdep"][0]
    assert entry["iq"] == 1 and entry["q"] == [0.0, 0.0, 0.0]
    assert entry["eigenval"] == ev.tolist()
    assert entry["eigenvec"] == [f"Q000000001E{j:09d}.dat" for j in range(1, 6)]


def test_roundtrip(tmp_path):
    ev, vec = _data()
    pdep_db_write(str(tmp_path), ev, vec, cubic_cell(15.0))
    rev, rvec = pdep_db_read(str(tmp_path), 5, 97)
    np.testing.assert_array_equal(rev, ev)
    np.testing.assert_array_equal(rvec, vec)
    rev3, rvec3 = pdep_db_read(str(tmp_path), 3, 97)        # n_pdep_read_from_file < n_pdep_eigen
    np.testing.assert_array_equal(rvec3, vec[:, :3])


def test_read_rejects_mismatches(tmp_path):
    from west_b200.lib import WestB200Error
    ev, vec = _data()
    pdep_db_write(str(tmp_path), ev, vec, cubic_cell(15.0))
    with pytest.raises(WestB200Error, match="dimension"):
        pdep_db_read(str(tmp_path), 5, 96)
    with pytest.raises(WestB200Error, match="fewer than the requested"):
        pdep_db_read(str(tmp_path), 6, 97)
    os.remove(tmp_path / "Q000000001E000000005.dat")
    with pytest.raises(WestB200Error, match="cannot open"):
        pdep_db_read(str(tmp_path), 5, 97)
    bad = tmp_path / "Q000000001E000000002.dat"
    raw = np.fromfile(bad, dtype=np.uint8)
    raw[:4].view(np.int32)[0] = 1
    raw.tofile(bad)
    with pytest.raises(WestB200Error, match="version"):
        pdep_db_read(str(tmp_path), 5, 97)
