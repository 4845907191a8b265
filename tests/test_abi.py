"""The C ABI library: loads, exports every symbol include/imogen_b200.h declares, and rejects
invalid settings before touching a GPU (CPU only)."""
import ctypes
import os
import re

import pytest

import imogen_b200
from imogen_b200 import _lib
from imogen_b200.run import bc_table, make_config

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "imogen_b200.h")).read()
    return sorted(set(re.findall(r"\b(img_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    syms = header_symbols()
    assert len(syms) >= 18
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(_lib.SYMBOLS)


def test_sweep_order_table_matches_the_oracle():
    """img_sweep_order (host only) returns the same directVec rows as both oracles (flux.m:17-27)."""
    from oracle import np_oracle
    L = _lib.lib()
    out = (ctypes.c_int * 3)()
    for it in range(1, 14):
        for order, table in ((1, np_oracle.FORWARD_ORDER), (-1, np_oracle.BACKWARD_ORDER)):
            assert L.img_sweep_order(order, it, out) == 0
            assert tuple(out) == table[(it - 1) % 6]
    assert L.img_sweep_order(0, 1, out) == -1


def test_create_rejects_settings_the_reference_cannot_run():
    L = _lib.lib()
    for kw, code in [(dict(grid=(32, 1, 1), bc="mirror"), -4), (dict(grid=(19, 32, 1), bc="fade"), -4)]:
        c = make_config(**kw)
        h = ctypes.c_void_p()
        assert L.img_create(ctypes.byref(h), ctypes.byref(c)) == code
        assert b"BC" in L.img_last_error(None)
    c = make_config(grid=(32, 32, 1), precision=7)
    h = ctypes.c_void_p()
    assert L.img_create(ctypes.byref(h), ctypes.byref(c)) == -1


def test_bytes_required_counts_state_scratch_and_edges():
    n = 64 * 48
    b64 = imogen_b200.bytes_required(grid=(64, 48, 1), magnet=True, precision="fp64")
    b32 = imogen_b200.bytes_required(grid=(64, 48, 1), magnet=True, precision="mixed")
    # 11 state arrays + 2 magnet scratch arrays; the mixed form adds an FP64 transfer stage
    assert b64 >= 13 * n * 8 and b32 >= 13 * n * 4 + n * 8 and b64 > b32
    bt = imogen_b200.bytes_required(grid=(64, 48, 1), magnet=True, bc="trans")
    assert bt > b64          # stored edges of the trans objects


def test_bc_table_forms():
    assert bc_table("trans") == [[[4] * 3, [4] * 3]] * 4
    t = bc_table({"x": ("const", "wall"), "y": "circ", "z": "circ"})
    assert t[0] == [[1, 0, 0], [5, 0, 0]]


def test_null_context_is_an_error_not_a_crash():
    L = _lib.lib()
    assert L.img_step(None) == -1
    assert L.img_sync(None) == -1


def test_mex_gateway_compiles_against_the_abi():
    """The MEX gateway (imogen_b200/mex) compiles with the C ABI header and a declarations-only
    mex.h, and every img_* function it calls is exported by the library."""
    import re
    import shutil
    import subprocess
    import tempfile
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = os.path.join(root, "imogen_b200", "mex", "imogen_b200_mex.c")
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-c", src, "-I", os.path.join(root, "tests", "mexstub"),
                            "-I", os.path.join(root, "include"), "-o", os.path.join(d, "mex.o")],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
    called = set(re.findall(r"\b(img_[a-z_]+)\(", open(src).read()))
    assert called <= set(_lib.SYMBOLS), called - set(_lib.SYMBOLS)


def test_create_rejects_viscosity_the_segment_kernel_cannot_take():
    """Artificial viscosity runs in the one-block segment kernel: circ or const ends shared by all
    classes, and a segment tiling for every swept pencil length (checked before any device call)."""
    L = _lib.lib()
    cases = [dict(grid=(64, 32, 1), bc="trans"), dict(grid=(64, 32, 1), bc="mirror"),
             dict(grid=(64, 32, 1), bc={"mass": "circ", "mom": "const", "ener": "circ", "mag": "circ"}),
             dict(grid=(100, 32, 1), bc="circ"),        # x: 100 / C threads is no power of two up to 32
             dict(grid=(64, 4096, 1), bc="circ")]       # y: N / C > 512 threads
    for kw in cases:
        c = make_config(viscosity="neumann_richtmyer", **kw)
        h = ctypes.c_void_p()
        assert L.img_create(ctypes.byref(h), ctypes.byref(c)) == -4, kw
        assert b"viscosity" in L.img_last_error(None), kw
    for bad in (dict(viscosity=3), dict(radiation=2)):
        c = make_config(grid=(64, 32, 1), **bad)
        h = ctypes.c_void_p()
        assert L.img_create(ctypes.byref(h), ctypes.byref(c)) == -1, bad


def test_config_defaults_match_the_reference_constructors():
    """ArtificialViscosity() (ArtificialViscosity.m:31-37) and Radiation() (Radiation.m:32-37)."""
    c = _lib.ImgConfig()
    _lib.lib().img_config_default(ctypes.byref(c))
    assert (c.viscosity_type, c.visc_linear, c.visc_quadratic) == (0, 0.0, 0.0)
    assert (c.radiation_type, c.rad_exponent, c.rad_initial_maximum) == (0, 0.5, 0.0)


def test_create_rejects_the_boundaries_the_reference_cannot_run():
    """linear_shift.m uses an undefined variable; wormhole_shift.m needs a third dimension; a lower
    wormhole side couples pencils across the grid and is not on this path."""
    L = _lib.lib()
    for kw, word in [(dict(grid=(32, 16, 1), bc="linear"), b"linear"),
                     (dict(grid=(32, 16, 1), bc={"x": ("wormhole", "const"), "y": "circ"}), b"wormhole"),
                     (dict(grid=(16, 16, 16), bc={"x": "circ", "y": ("wormhole", "const"), "z": "circ"}), b"wormhole")]:
        c = make_config(**kw)
        h = ctypes.c_void_p()
        assert L.img_create(ctypes.byref(h), ctypes.byref(c)) == -4, kw
        assert word in L.img_last_error(None), kw


def test_create_checks_the_treadmill_setting():
    L = _lib.lib()
    for kw, code in [(dict(grid=(32, 16, 1), treadmill=4), -1),
                     (dict(grid=(40000, 2, 1), treadmill=1), -4)]:   # 2 x 40000 FP64 values exceed one block
        c = make_config(**kw)
        h = ctypes.c_void_p()
        assert L.img_create(ctypes.byref(h), ctypes.byref(c)) == code, kw
        assert b"treadmill" in L.img_last_error(None), kw


def test_create_checks_the_point_fade_setting():
    L = _lib.lib()
    for kw in (dict(fade_location=(3, 3, 1), fade_size=2.0, fade_active=("mass",)),):
        for bad in (dict(fade_location=(0, 3, 1)), dict(fade_location=(3, 40, 1)), dict(fade_size=0.0)):
            c = make_config(grid=(32, 16, 1), **dict(kw, **bad))
            h = ctypes.c_void_p()
            assert L.img_create(ctypes.byref(h), ctypes.byref(c)) == -1, bad
            assert b"fade" in L.img_last_error(None), bad
    c = make_config(grid=(32, 16, 1))
    c.fade_active = 64
    h = ctypes.c_void_p()
    assert L.img_create(ctypes.byref(h), ctypes.byref(c)) == -1
