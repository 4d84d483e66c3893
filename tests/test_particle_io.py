"""The reference's particle files (loadd.f90:147-670, main.f90:455-476) written
and read back: Fortran Ew.d formatting against hand-worked values, the
allpartdata record layout (type particle_restart, loadd.f90:149-160), and
round trips of every file.
"""
import os

import numpy as np
import pytest

from suguru_b200 import particle_io as P
from suguru_b200 import workloads as W


@pytest.mark.parametrize("x,w,d,out", [
    (-12.5, 15, 7, " -0.1250000E+02"),
    (0.0, 15, 7, "  0.0000000E+00"),
    (0.5, 15, 7, "  0.5000000E+00"),
    (0.99999999, 15, 7, "  0.1000000E+01"),
    (1e100, 15, 7, "  0.1000000+101"),
    (6.02214076e23, 16, 8, "  0.60221408E+24"),
    (-1e-5, 16, 8, " -0.10000000E-04"),
    (1.0 / 3.0, 16, 8, "  0.33333333E+00"),
])
def test_fortran_e(x, w, d, out):
    assert P.fortran_e(x, w, d) == out
    assert len(out) == w


def test_fortran_e_round_trip():
    rng = np.random.default_rng(3)
    x = rng.normal(size=200) * 10.0 ** rng.integers(-30, 30, size=200)
    back = np.array([P.parse_fortran_e(P.fortran_e(v, 15, 7)) for v in x])
    assert np.all(np.abs(back - x) <= 5e-7 * np.abs(x))  # half a unit of the 7th digit, mantissa >= 0.1


def test_allpartdata_layout_and_round_trip(tmp_path):
    rng = np.random.default_rng(4)
    npart, nl = 3, 50
    scal = rng.normal(size=(npart, 6))
    arr = rng.normal(size=(npart, 22, nl))
    path = os.path.join(tmp_path, P.allpartdata_name(1200))
    P.write_allpartdata(path, scal, arr)
    assert os.path.basename(path) == "allpartdata0001200"
    raw = np.fromfile(path, dtype=np.float64)
    assert raw.size == npart * (6 + 22 * nl)  # recl = np * skip reals, skip = 6 + 22 nl
    # particle 2: x, y, z, integralv, volume, volume0, then xfp(1:nl), yfp(1:nl), ...
    rec = raw[(6 + 22 * nl):2 * (6 + 22 * nl)]
    assert np.array_equal(rec[:6], scal[1])
    assert np.array_equal(rec[6:6 + nl], arr[1, P.PARTICLE_ARRAYS.index("xfp")])
    assert np.array_equal(rec[6 + 21 * nl:], arr[1, P.PARTICLE_ARRAYS.index("area")])
    s2, a2 = P.read_allpartdata(path, npart, nl)
    assert np.array_equal(s2, scal) and np.array_equal(a2, arr)
    with pytest.raises(ValueError):
        P.read_allpartdata(path, npart, nl + 1)


def test_capsule_txt_round_trip(tmp_path):
    wl = W.small_config(ncap=1, degrees=(7,))
    path = os.path.join(tmp_path, P.capsule_txt_name(1, 100))
    assert os.path.basename(path) == "Capsule001step0000100.txt"
    P.write_capsule_txt(path, wl.x, wl.y, wl.z)
    lines = open(path).read().splitlines()
    assert len(lines) == wl.npts and all(len(s) == 45 for s in lines)
    assert lines[0] == "".join(P.fortran_e(v, 15, 7) for v in (wl.y[0], wl.z[0], wl.x[0]))  # y, z, x
    x, y, z = P.read_capsule_txt(path)
    for a, b in ((x, wl.x), (y, wl.y), (z, wl.z)):
        assert np.all(np.abs(a - b) <= 5e-7 * np.abs(b))


def test_step_outputs_and_state(tmp_path):
    wl = W.small_config(ncap=3, degrees=(7,))
    off = wl.offsets
    pos = (wl.x, wl.y, wl.z)
    vel = tuple(np.full(wl.npts, v) for v in (0.1, -0.2, 0.3))
    P.write_step_outputs(str(tmp_path), 100, 0.25, off, pos, vel, 0.01, 0.02)
    for p in range(1, 4):
        assert os.path.exists(os.path.join(tmp_path, P.capsule_txt_name(p, 100)))
    cv = open(os.path.join(tmp_path, "center_velocity.txt")).read().splitlines()
    ep = open(os.path.join(tmp_path, "epsilonxy.txt")).read().splitlines()
    assert len(cv) == 3 and len(ep) == 3  # one line per capsule, as the reference's loop writes them
    f = [P.parse_fortran_e(cv[0][16 * q:16 * (q + 1)]) for q in range(7)]
    assert f[0] == 0.25 and abs(f[1] - wl.x[off[0]:off[1]].mean()) <= 1e-8 and abs(f[4] - 0.1) <= 1e-9
    scal, arr = P.particle_state(off, pos, velocity=vel, volume=np.ones(3))
    assert scal.shape == (3, 6) and arr.shape == (3, 22, off[1])
    assert np.array_equal(arr[1, P.PARTICLE_ARRAYS.index("yfp")], wl.y[off[1]:off[2]])
    assert np.array_equal(arr[2, P.PARTICLE_ARRAYS.index("ul")], vel[0][off[2]:off[3]])
