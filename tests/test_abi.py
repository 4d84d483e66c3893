"""CPU tests of the C ABI library: it loads, exports every symbol declared in
include/sg_coupling.h, its host tables agree with the oracle, and invalid
configurations are rejected with SG_ERR_CONFIG before any device work."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle as O
from suguru_b200 import build, coupling

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return coupling.lib()


def header_symbols(name="sg_coupling.h"):
    text = open(os.path.join(ROOT, "include", name)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sg_[a-z_]+)\s*\(", text)))


def test_exports_every_declared_symbol(lib):
    syms = header_symbols()
    assert len(syms) >= 10
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(coupling.EXPORTS) == syms


def test_every_header_is_covered(lib):
    headers = sorted(f for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h"))
    assert headers == ["sg_coupling.h", "sg_testing.h", "sg_workload.h"]
    syms = header_symbols("sg_testing.h")
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(coupling.TEST_EXPORTS) == syms
    syms = header_symbols("sg_workload.h")
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(coupling.WORKLOAD_EXPORTS) == syms


def test_build_flags_target_sm100a():
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


def test_host_gauss_matches_oracle(lib):
    for n in (15, 32, 48, 63):
        th, w = coupling.gauss(n)
        th2, w2 = O.gaqd(n)
        assert np.abs(th - th2).max() < 1e-15
        assert np.abs(w - w2).max() < 1e-15


def test_host_legendre_matches_oracle(lib):
    for t in (0.07, 1.3, 2.9):
        a = coupling.legendre(t, 16, 16)
        b = O.legendre(t, 16, 16)
        for x, y in zip(a, b):
            assert np.abs(x - y).max() < 1e-13 * max(1.0, np.abs(y).max())


def _cfg(**kw):
    deg = np.array(kw.pop("degree", [15]), np.int32)
    rad = np.array(kw.pop("radius", [0.25]), np.float64)
    c = coupling.sg_config()
    c.itot, c.jtot, c.ktot = 64, 32, 32
    c.lx, c.ly, c.lz = 2.0, 1.0, 1.0
    c.ncap = deg.size
    c.degree = deg.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    c.radius = rad.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    c.gs, c.csk = 1.0, 1.0
    c.precision, c.mem, c.device, c.surrogate = 0, 0, 0, 0
    for k, v in kw.items():
        setattr(c, k, v)
    return c, deg, rad


@pytest.mark.parametrize("bad", [dict(degree=[1]), dict(degree=[40]), dict(radius=[-1.0]), dict(precision=7),
                                 dict(mem=3), dict(lx=0.0), dict(surrogate=1)])
def test_invalid_config_rejected(lib, bad):
    cfg, deg, rad = _cfg(**bad)
    h = ctypes.c_void_p()
    rc = lib.sg_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == 1  # SG_ERR_CONFIG
    assert lib.sg_last_error(h)
    lib.sg_destroy(h)


def test_null_arguments(lib):
    assert lib.sg_create(None, None) == 5  # SG_ERR_ARG
    assert lib.sg_interp(None, *([None] * 9)) == 5


def test_spread_noalloc_refuses_before_any_device_work(lib):
    """sg_spread_noalloc checks the grid and the sizes on the host before it
    looks up its scratch array or queues anything, so on a machine without a
    GPU these refusals still come back as their own codes (not SG_ERR_CUDA).
    The field pointers are never dereferenced on these paths."""
    buf = (ctypes.c_double * 4)()
    p = ctypes.cast(buf, ctypes.c_void_p)
    dx = 1.0 / 16
    f = lib.sg_spread_noalloc
    # jtot = 25 = 1 mod 8: neither FP64 tile shape (32x8x4, 8x8x4) fits
    assert f(64, 25, 16, 64 * dx, 25 * dx, 16 * dx, 0, None, None, None, None, None, None, None,
             p, p, p, None) == 5  # SG_ERR_ARG
    # 512 x 256 x 256 on 32x8x4 tiles: 16 * 32 * 64 = 32768 tiles > SG_NOALLOC_MAX_TILES
    assert f(512, 256, 256, 512 * dx, 256 * dx, 256 * dx, 0, None, None, None, None, None, None, None,
             p, p, p, None) == 7  # SG_ERR_TOO_LARGE
    # 65,537 points > SG_NOALLOC_MAX_POINTS
    assert f(64, 48, 40, 4.0, 3.0, 2.5, 65537, p, p, p, p, p, p, p, p, p, p, None) == 7

