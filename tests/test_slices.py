"""Slice files of save/resultsHandler.m (MAT-file Level 5) and their reader, against SciPy's
independent MAT-file implementation (no GPU: the host-level img_slice_write / img_slice_read).

The writer must produce what MATLAB's save(fileName, sliceName) of resultsHandler's struct holds: one
variable sx_<label>_<suffix> with the fields in resultsHandler's order and SaveManager.getSaveSlice
cuts; the reader must take what Initializer.loadDataFromFile takes, from files written with or
without compression and with narrowed numeric types.
"""
import numpy as np
import pytest
import scipy.io

from imogen_b200 import ImogenError
from imogen_b200.run import read_slice, write_slice
from tests.parity import smooth_state

FIELDS = ["gamma", "time", "about", "ver", "iter", "mass", "momX", "momY", "momZ", "ener", "magX", "magY", "magZ",
          "grav", "dGrid", "dim"]


def _load(path):
    d = scipy.io.loadmat(str(path), squeeze_me=False, struct_as_record=True)
    names = [k for k in d if not k.startswith("__")]
    assert len(names) == 1, names
    return names[0], d[names[0]][0, 0]


def test_xyz_slice_matches_resultshandler_struct(tmp_path):
    grid = (12, 10, 6)
    st = smooth_state(grid, seed=3, mhd=True)
    p = tmp_path / "3D_XYZ_FINAL.mat"
    write_slice(p, st, grid, dgrid=(0.1, 0.2, 0.3), gamma=1.4, time=0.25, iteration=7, iter_max=100, time_max=1.0,
                dt_history=[0.01 * k for k in range(1, 8)], about="kh test", version=0.6, wall_max=12.0,
                started="04-Dec-2026 10:00:00")
    name, s = _load(p)
    assert name == "sx_XYZ_FINAL"
    assert list(s.dtype.names) == FIELDS
    assert s["gamma"][0, 0] == 1.4 and s["ver"][0, 0] == 0.6 and s["iter"][0, 0] == 7
    assert s["about"][0] == "kh test" and s["dim"][0] == "3D"
    t = s["time"][0, 0]
    assert list(t.dtype.names) == ["time", "history", "iterMax", "timeMax", "wallMax", "started", "iteration"]
    assert t["time"][0, 0] == 0.25 and t["iterMax"][0, 0] == 100 and t["wallMax"][0, 0] == 12.0
    assert t["history"].shape == (7, 1) and np.allclose(t["history"][:, 0], [0.01 * k for k in range(1, 8)], rtol=0)
    assert t["started"][0] == "04-Dec-2026 10:00:00" and t["iteration"][0, 0] == 7
    rho, mom, ener, mag = st
    assert np.array_equal(s["mass"], rho) and np.array_equal(s["ener"], ener)
    for c, f in enumerate("XYZ"):
        assert np.array_equal(s["mom" + f], mom[c]) and np.array_equal(s["mag" + f], mag[c])
    assert s["grav"].shape == (0, 0)
    assert [s["dGrid"][0, k][0, 0] for k in range(3)] == [0.1, 0.2, 0.3]


@pytest.mark.parametrize("slice,label,cut", [
    ("X", "X", lambda a: a[:, 2, 4][:, None]), ("Y", "Y", lambda a: a[1, :, 4][None, :]),
    ("Z", "Z", lambda a: a[1, 2, :][:, None]), ("XY", "XY", lambda a: a[:, :, 4]),
    ("XZ", "XZ", lambda a: a[:, 2, :]), ("YZ", "YZ", lambda a: a[1, :, :])])
def test_cuts_follow_getsaveslice_and_squeeze(tmp_path, slice, label, cut):
    grid = (8, 7, 6)
    st = smooth_state(grid, seed=4, mhd=True)
    p = tmp_path / "cut.mat"
    write_slice(p, st, grid, slice=slice, index=(2, 3, 5), suffix="00010")
    name, s = _load(p)
    assert name == f"sx_{label}_00010"
    assert s["dim"][0] == ("1D" if len(label) == 1 else "2D")
    assert np.array_equal(s["mass"], cut(st[0])) and np.array_equal(s["momY"], cut(st[1][1]))


def test_two_dimensional_grid_and_no_magnet(tmp_path):
    grid = (9, 5, 1)
    st = smooth_state(grid, seed=5, mhd=False)
    p = tmp_path / "2d.mat"
    write_slice(p, st, grid, magnet=False, treadmill=1, treadmill_history=[0, 1, -1], slice="SP-XYZ", suffix="START")
    name, s = _load(p)
    assert name == "sx_SP0x2DXYZ_START"                # genvarname's hex code for '-'
    assert "tread" in s.dtype.names and list(s.dtype.names).index("tread") == 5
    tr = s["tread"][0, 0]
    assert tr["direction"][0, 0] == 1 and tr["history"][:, 0].tolist() == [0, 1, -1]
    assert s["mass"].shape == (9, 5) and s["magX"].shape == (0, 0) and s["dim"][0] == "Cust"
    (rho, mom, ener, mag), has_mag = read_slice(p)
    assert not has_mag and np.array_equal(rho, st[0]) and not mag.any()


@pytest.mark.parametrize("compress", [False, True])
def test_reader_takes_matlab_style_files(tmp_path, compress):
    """A struct saved by another MAT writer, compressed (MATLAB 7's default) or not, with integer-typed
    arrays (MATLAB narrows integer-valued doubles when it saves)."""
    grid = (6, 5, 4)
    rho, mom, ener, mag = smooth_state(grid, seed=6, mhd=True)
    rho_int = np.arange(np.prod(grid), dtype=np.int16).reshape(grid) + 1
    sl = {"gamma": 5 / 3, "time": {"time": 0.0, "history": np.zeros((0, 1))}, "about": "", "ver": 0.0, "iter": 0,
          "mass": rho_int, "momX": mom[0], "momY": mom[1], "momZ": mom[2], "ener": ener, "magX": mag[0],
          "magY": mag[1], "magZ": mag[2], "grav": np.zeros((0, 0)), "dGrid": np.array([[0.1, 0.1, 0.1]], dtype=object),
          "dim": "3D"}
    p = tmp_path / "other.mat"
    scipy.io.savemat(str(p), {"sx_XYZ_FINAL": sl}, do_compression=compress)
    (r, m, e, b), has_mag = read_slice(p)
    assert has_mag
    assert np.array_equal(r, rho_int.astype(float)) and np.array_equal(e, ener)
    assert np.array_equal(m, mom) and np.array_equal(b, mag)


def test_round_trip_through_our_own_reader(tmp_path):
    grid = (7, 6, 5)
    st = smooth_state(grid, seed=8, mhd=True)
    p = tmp_path / "rt.mat"
    write_slice(p, st, grid)
    (r, m, e, b), has_mag = read_slice(p)
    assert has_mag
    for x, y in zip((r, m, e, b), st):
        assert np.array_equal(x, y)


def test_reader_rejects_what_it_cannot_resume_from(tmp_path):
    p = tmp_path / "bad.mat"
    p.write_bytes(b"not a mat file" * 20)
    with pytest.raises(ImogenError):
        read_slice(p)
    q = tmp_path / "nostruct.mat"
    scipy.io.savemat(str(q), {"x": np.ones((3, 3))})
    with pytest.raises(ImogenError):
        read_slice(q)
    with pytest.raises(ImogenError):
        read_slice(tmp_path / "missing.mat")
