"""CPU tests of the FP64 oracle: pinned against the reference's recorded
outputs (SPHEREPACK test logs, kernel partition of unity), the reference's own
membmodel.c compiled from its sources, independent libraries (scipy, mpmath),
and analytic known-answer cases."""
import math

import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W
from util import rel_l2


# spherepack3.2_impi-15/output/darwin.dp:699-701 (tsha.f, nlat=15), printed to 4 digits
DARWIN_THTG15 = [0.1551, 0.3561, 0.5582, 0.7606, 0.9631, 1.166, 1.368, 1.571, 1.773, 1.976, 2.178, 2.381,
                 2.583, 2.786, 2.986]


def test_gaqd_nodes_match_darwin_log():
    th, w = O.gaqd(15)
    assert np.allclose(th, DARWIN_THTG15, atol=5.01e-4)
    assert abs(w.sum() - 2.0) < 1e-14


def test_gaqd_nlat63_against_mpmath():
    # darwin.dp:434-436: nlat=63 node error 7.1e-17, weight error 6.6e-15 (relative max)
    mp = pytest.importorskip("mpmath")
    mp.mp.dps = 40
    th, w = O.gaqd(63)
    xs = sorted((mp.mpf(r) for r in mp.polyroots(mp.taylor(lambda t: mp.legendre(63, t), 0, 63)[::-1],
                                                   maxsteps=200, extraprec=200)), reverse=True)
    th_ref = np.array([float(mp.acos(x)) for x in xs])
    assert np.abs(th - th_ref).max() / np.abs(th_ref).max() < 2e-16 * 10
    dP = [mp.diff(lambda t: mp.legendre(63, t), x) for x in xs]
    w_ref = np.array([float(2 / ((1 - x * x) * d * d)) for x, d in zip(xs, dP)])
    assert np.abs(w - w_ref).max() / np.abs(w_ref).max() < 6.6e-15 * 2
    assert abs(w.sum() - 2.0) < 1e-14


def test_kernel_partition_of_unity_matches_log():
    # out.log:1  "Integral over kernel = 0.99999999999996703"
    assert abs(O.kerneltest() - 0.99999999999996703) < 1e-15
    # and the discrete partition of unity per dimension
    for c in np.linspace(0, 1, 7):
        s = sum(O.kernel(i - c) for i in range(-3, 4))
        assert abs(s - 1.0) < 1e-14


def test_kernel_values():
    # kernel.f90:7-25
    assert O.kernel(0.0) == pytest.approx(2.0 / 3.0, abs=1e-16)
    assert O.kernel(0.5) == pytest.approx(0.5, abs=1e-16)
    assert O.kernel(1.5) == 0.0 and O.kernel(-1.6) == 0.0
    assert O.kernel(1.0) == pytest.approx((5 - 3 - math.sqrt(1)) / 6, abs=1e-16)


def test_legendre_against_scipy():
    from scipy.special import lpmv
    for t in (0.05, 0.7, 1.9, 3.1):
        P, D, D2 = O.legendre(t, 12, 20)
        for m in range(12):
            for n in range(m, 20):
                ref = math.sqrt((2 * n + 1) / 2 * math.factorial(n - m) / math.factorial(n + m)) * \
                    lpmv(m, n, math.cos(t)) * (-1) ** m
                assert P[m, n] == pytest.approx(ref, rel=1e-12, abs=1e-13)


def test_legendre_derivatives_fd():
    h = 1e-5
    for t in (0.3, 1.2, 2.5):
        P, D, D2 = O.legendre(t, 10, 16)
        Pp, Dp, _ = O.legendre(t + h, 10, 16)
        Pm, Dm, _ = O.legendre(t - h, 10, 16)
        assert np.abs((Pp - Pm) / (2 * h) - D).max() < 1e-6
        assert np.abs((Dp - Dm) / (2 * h) - D2).max() < 1e-5


def test_legendre_ode():
    # theta-form Legendre ODE: P'' + cot P' + (n(n+1) - m^2/sin^2) P = 0
    t = 0.83
    P, D, D2 = O.legendre(t, 12, 18)
    for m in range(12):
        for n in range(m, 18):
            r = D2[m, n] + math.cos(t) / math.sin(t) * D[m, n] + (n * (n + 1) - m * m / math.sin(t) ** 2) * P[m, n]
            assert abs(r) < 1e-11 * max(1, n * n)


def _tsha_field(th, nlon, k):
    ph = np.arange(nlon) * 2 * np.pi / nlon
    T, Pp = np.meshgrid(th, ph, indexing="ij")
    return (np.sin(T) * (np.sin(T) * np.cos(T) * np.sin(Pp) * np.cos(Pp))) ** k


def test_tsha_roundtrip_gaussian():
    # tsha.f icase=3 (shagc/shsgc, nlat=15, nlon=18, nt=3): err2 = 0.17708E-15 (darwin.dp:740)
    th, _ = O.gaqd(15)
    s = np.stack([_tsha_field(th, 18, k) for k in (1, 2, 3)])
    a, b = O.shagc(s)
    g = O.shsgc(a, b, 18)
    err2 = np.sqrt(((g - s) ** 2).sum() / s.size)
    assert err2 < 1e-15


def test_trssph_gauss_to_gauss():
    # testrssph.f data exp(sin t (sin t cos t sin p cos p)) transferred between
    # Gaussian grids (92 x 194 -> 19 x 36 and back); darwin.dp:372,386 report
    # 7.6e-12 / 5.5e-12 for the equally spaced variant.
    def f(nlat, nlon):
        th, _ = O.gaqd(nlat)
        return np.exp(_tsha_field(th, nlon, 1))
    big, small = f(92, 194), f(19, 36)
    out_small = O.trssph(big, 19, 36)
    assert np.sqrt(((out_small - small) ** 2).mean()) < 1e-6
    out_big = O.trssph(small, 92, 194)
    assert np.sqrt(((out_big - big) ** 2).mean()) < 1e-6
    # band-limited data transfers exactly
    th, _ = O.gaqd(24)
    g = _tsha_field(th, 48, 2)
    back = O.trssph(O.trssph(g, 40, 80), 24, 48)
    assert np.abs(back - g).max() < 1e-14


def test_skalak_matches_reference_membmodel():
    """The restated Skalak law against the reference's own membmodel.c (oracle/_ref)."""
    ref = O.ref_membmodel("skalak")
    if ref is None:
        pytest.skip("oracle/_ref not built (reference tree absent)")
    import ctypes
    dp = ctypes.POINTER(ctypes.c_double)
    rng = np.random.default_rng(0)
    for _ in range(50):
        gs, csk = rng.uniform(0.2, 3), rng.uniform(0.5, 50)
        I1, I2 = rng.normal(0, 0.3), rng.normal(0, 0.3)
        I1de, I2de = rng.normal(size=2), rng.normal(size=2)
        ref.ref_set_hf_gscell(0.5 * gs)  # sph.f90:35
        w1, w2 = np.zeros(1), np.zeros(1)
        w1d, w2d = np.zeros(2), np.zeros(2)
        args = [np.array([gs]), np.array([csk]), np.array([I1]), np.array([I2]), I1de.copy(), I2de.copy()]
        ref.calpwspi_deri_(w1.ctypes.data_as(dp), w2.ctypes.data_as(dp), w1d.ctypes.data_as(dp),
                           w2d.ctypes.data_as(dp), *[a.ctypes.data_as(dp) for a in args])
        mine = O.skalak(I1, I2, I1de, I2de, gs, csk)
        assert np.allclose(mine, [w1[0], w2[0], w1d[0], w1d[1], w2d[0], w2d[1]], rtol=1e-15, atol=0)


def test_neo_hookean_matches_reference_membmodel():
    """The restated neo-Hookean law against the reference's own membmodel.c
    compiled with -DNONHOOK (its default build; oracle/_ref)."""
    ref = O.ref_membmodel("nh")
    if ref is None:
        pytest.skip("oracle/_ref not built (reference tree absent)")
    import ctypes
    dp = ctypes.POINTER(ctypes.c_double)
    rng = np.random.default_rng(1)
    for _ in range(50):
        gs, csk = rng.uniform(0.2, 3), rng.uniform(0.5, 50)
        I1, I2 = rng.normal(0, 0.3), rng.uniform(-0.5, 0.8)
        I1de, I2de = rng.normal(size=2), rng.normal(size=2)
        ref.ref_set_hf_gscell(0.5 * gs)  # sph.f90:35
        w1, w2 = np.zeros(1), np.zeros(1)
        w1d, w2d = np.zeros(2), np.zeros(2)
        args = [np.array([gs]), np.array([csk]), np.array([I1]), np.array([I2]), I1de.copy(), I2de.copy()]
        ref.calpwspi_deri_(w1.ctypes.data_as(dp), w2.ctypes.data_as(dp), w1d.ctypes.data_as(dp),
                           w2d.ctypes.data_as(dp), *[a.ctypes.data_as(dp) for a in args])
        mine = O.membrane_law(1, I1, I2, I1de, I2de, gs, csk)
        assert np.allclose(mine, [w1[0], w2[0], w1d[0], w1d[1], w2d[0], w2d[1]], rtol=1e-15, atol=0)
        # law 0 through the same entry point is the Skalak law
        assert np.array_equal(O.membrane_law(0, I1, I2, I1de, I2de, gs, csk),
                              O.skalak(I1, I2, I1de, I2de, gs, csk))


L15 = 15


def test_sphere_has_zero_force_and_exact_area_normals():
    R = 0.25
    x, y, z = W.capsule_points(L15, R, (2.0, 1.0, 1.0))
    f, n, a = O.complagrforces(L15, R, x, y, z)
    assert np.abs(f).max() < 1e-9
    xh = np.stack([x - 2, y - 1, z - 1]) / R
    assert np.abs(n + xh).max() < 1e-10  # normal a1 x a2 points inward for this parametrisation
    # area carries the reference's truncation of sin(theta)-weighted metric; within 0.5%
    assert abs(a.sum() / (4 * np.pi * R * R) - 1) < 5e-3


@pytest.mark.parametrize("lam,csk", [(1.05, 1.0), (0.97, 1.0), (1.02, 5.0)])
def test_uniform_dilation_laplace_law(lam, csk):
    """Skalak isotropic stretch: tau = Gs[(l^2-1) + C l^2 (l^4-1)], f = 2 tau / r (inward)."""
    R, gs = 0.25, 1.3
    x, y, z = W.capsule_points(L15, lam * R, (1.0, 1.0, 1.0))
    f, n, a = O.complagrforces(L15, R, x, y, z, gs=gs, csk=csk)
    tau = gs * ((lam ** 2 - 1) + csk * lam ** 2 * (lam ** 4 - 1))
    r = lam * R
    xh = np.stack([x - 1, y - 1, z - 1]) / r
    assert np.abs(f + (2 * tau / r) * xh).max() < 1e-8 * abs(2 * tau / r) + 1e-8


@pytest.mark.parametrize("lam", [0.9, 1.05, 1.2])
def test_uniform_dilation_neo_hookean(lam):
    """Neo-Hookean isotropic stretch: W1 = Gs/2, W2 = -Gs/2 (I2+1)^-2 with I2 = l^4 - 1,
    so T = Gs (l^-2 - l^-8) A, tau = T:a / 2 = Gs (1 - l^-6) and f = 2 tau / r (inward);
    a sphere at the reference radius carries no force."""
    R, gs = 0.25, 1.3
    x, y, z = W.capsule_points(L15, lam * R, (1.0, 1.0, 1.0))
    f, n, a = O.complagrforces(L15, R, x, y, z, gs=gs, csk=7.0, law=1)  # C plays no part
    tau = gs * (1 - lam ** -6)
    r = lam * R
    xh = np.stack([x - 1, y - 1, z - 1]) / r
    assert np.abs(f + (2 * tau / r) * xh).max() < 1e-8 * abs(2 * tau / r) + 1e-8
    x0, y0, z0 = W.capsule_points(L15, R, (1.0, 1.0, 1.0))
    f0, _, _ = O.complagrforces(L15, R, x0, y0, z0, gs=gs, law=1)
    assert np.abs(f0).max() < 1e-9


def test_translation_noise_floor():
    """The reference-structured computation (no centring, 'faithful') differs from
    the centred one only by roundoff amplified near the poles: below 1e-9."""
    wl = W.config0()
    f0, n0, a0 = O.complagrforces(L15, float(wl.radius[0]), wl.x, wl.y, wl.z)
    f1, n1, a1 = O.complagrforces(L15, float(wl.radius[0]), wl.x, wl.y, wl.z, faithful=True)
    for c in range(3):
        assert rel_l2(f1[c], f0[c]) < 1e-9
        assert rel_l2(n1[c], n0[c]) < 1e-12
    assert rel_l2(a1, a0) < 1e-12


def test_net_force_is_small():
    # internal membrane forces carry no net force: sum f * area ~ 0
    wl = W.config0()
    f, n, a = O.complagrforces(L15, float(wl.radius[0]), wl.x, wl.y, wl.z)
    net = (f * a).sum(axis=1)
    assert np.abs(net).max() < 1e-3 * (np.abs(f) * a).sum()


def test_interp_spread_adjoint_and_conservation():
    wl = W.small_config()
    u, v, w = wl.velocity()
    itot, jtot, ktot, dx, dy, dz = wl.grid
    ul, vl, wlv = O.interp(wl.grid, u, v, w, wl.x, wl.y, wl.z)
    rng = np.random.default_rng(0)
    f = rng.normal(size=(3, wl.npts))
    a = rng.uniform(0.5, 1.5, wl.npts)
    g = O.spread(wl.grid, wl.x, wl.y, wl.z, f[0], f[1], f[2], a)
    inner = lambda A, B: (A[1:-1, 1:-1, 1:-1] * B[1:-1, 1:-1, 1:-1]).sum()
    lhs = (inner(u, g[0]) + inner(v, g[1]) + inner(w, g[2])) * dx * dy * dz
    rhs = (ul * f[0] * a + vl * f[1] * a + wlv * f[2] * a).sum()
    assert abs(lhs - rhs) < 1e-12 * abs(rhs)
    for c in range(3):  # total force is conserved by the partition of unity
        assert abs(g[c][1:-1, 1:-1, 1:-1].sum() * dx * dy * dz - (f[c] * a).sum()) < 1e-11 * np.abs(f[c] * a).sum()
    # halos are copies (bound.f90:141-190)
    assert np.array_equal(g[0][:, :, 0], g[0][:, :, -2]) and np.array_equal(g[0][:, 0, :], g[0][:, -2, :])


def test_faithful_windows_equal_fast():
    wl = W.small_config()
    u, v, w = wl.velocity()
    a = O.interp(wl.grid, u, v, w, wl.x, wl.y, wl.z)
    b = O.interp(wl.grid, u, v, w, wl.x, wl.y, wl.z, faithful=True)
    for p, q in zip(a, b):
        assert np.abs(p - q).max() < 1e-13


def test_surf_vol_sphere():
    R = 0.25
    x, y, z = W.capsule_points(L15, R, (1.0, 1.0, 1.0))
    f, n, a = O.complagrforces(L15, R, x, y, z)
    out = O.surf_vol(x, y, z, n[0], n[1], n[2], a)
    # 1000-layer quadrature: sum_{l} ((l-1)/1000)^2 / 1000 = 0.3328335 instead of 1/3
    vol_expected = 0.3328335 * (a * R).sum()
    assert out[0] == pytest.approx(vol_expected, rel=1e-12)
    assert out[3] < 1e-12  # exy2 of a sphere
    assert np.allclose(out[4:7], [1, 1, 1], atol=1e-14)


def test_update_pos_clamps_walls():
    x = np.array([0.1, 0.2]); y = np.array([0.3, 0.4]); z = np.array([0.01, 1.99])
    u = np.array([1.0, 1.0]); v = np.array([0.0, 0.0]); w = np.array([-2.0, 2.0])
    x2, y2, z2 = O.update_pos(0.01, 2.0, x, y, z, u, v, w)
    assert np.allclose(x2, [0.11, 0.21]) and z2[0] == 0.0 and z2[1] == 2.0
