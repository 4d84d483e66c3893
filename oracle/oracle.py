"""ctypes wrapper of the CPU FP64 oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py -- never by the product package.  The oracle is a
restatement of the reference's coupling step; see sg_oracle.h for the reference
file:line each entry point follows.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build():
    """Compile liboracle.so (and oracle/_ref when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        i, d, l = ctypes.c_int, ctypes.c_double, ctypes.c_long
        L.or_gaqd.argtypes = [i, _dp, _dp]
        L.or_legendre.argtypes = [d, i, i, _dp, _dp, _dp]
        L.or_legendre.restype = None
        L.or_shagc.argtypes = [i, i, i, _dp, _dp, _dp]
        L.or_shsgc.argtypes = [i, i, i, _dp, _dp, _dp]
        L.or_trssph.argtypes = [i, i, i, _dp, i, i, _dp]
        L.or_kernel.argtypes = [d]
        L.or_kernel.restype = d
        L.or_kerneltest.argtypes = []
        L.or_kerneltest.restype = d
        L.or_complagrforces.argtypes = [i, d, d, d, i] + [_dp] * 10
        L.or_capsule_spectra.argtypes = [i, d, d, d] + [_dp] * 7
        L.or_interp.argtypes = [i, i, i, d, d, d, i, _dp, _dp, _dp, l, _dp, _dp, _dp, _dp, _dp, _dp]
        L.or_spread.argtypes = [i, i, i, d, d, d, i, l] + [_dp] * 10
        L.or_spread_ind.argtypes = [i, i, i, d, d, d, i, l] + [_dp] * 10
        L.or_update_pos.argtypes = [l, d, d] + [_dp] * 6
        L.or_update_pos.restype = None
        L.or_update_pos_capsules.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_long), d, d, d, d] + [_dp] * 6
        L.or_update_pos_capsules.restype = None
        L.or_surf_vol.argtypes = [l] + [_dp] * 7 + [d, _dp]
        L.or_surf_vol.restype = None
        L.or_collisions.argtypes = [l, _dp, _dp, d, d, d, d, d, d, _dp]
        L.or_collisions.restype = None
        L.or_skalak.argtypes = [d, d, _dp, _dp, d, d, _dp]
        L.or_skalak.restype = None
        L.or_membrane_law.argtypes = [i, d, d, _dp, _dp, d, d, _dp]
        L.or_membrane_law.restype = None
        L.or_complagrforces_law.argtypes = [i, d, d, d, i, i] + [_dp] * 10
        L.or_complagrforces_bend.argtypes = [i, d, d, d, i, d, i] + [_dp] * 10
        L.or_coupling_step.argtypes = ([i, i, i, d, d, d, i, _ip, _dp, d, d, i, i] + [_dp] * 20)
        _LIB = L
    return _LIB


def _p(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def gaqd(nlat):
    th, w = np.zeros(nlat), np.zeros(nlat)
    assert lib().or_gaqd(nlat, _p(th), _p(w)) == 0
    return th, w


def legendre(theta, mm, nn):
    """P, dP/dtheta, d2P/dtheta2 as [m, n] arrays (SPHEREPACK normalisation)."""
    P, D, D2 = (np.zeros((mm, nn)) for _ in range(3))
    lib().or_legendre(float(theta), mm, nn, _p(P), _p(D), _p(D2))
    return P, D, D2


def trunc_l(nlat, nlon):
    l = (nlon + 2) // 2 if nlon % 2 == 0 else (nlon + 1) // 2
    return min(l, nlat)


def shagc(g):
    """Analysis of g[nf, nlat, nlon] (or [nlat, nlon]) -> a, b [nf, l, nlat]."""
    g = _f64(g)
    squeeze = g.ndim == 2
    if squeeze:
        g = g[None]
    nf, nlat, nlon = g.shape
    l = trunc_l(nlat, nlon)
    a, b = np.zeros((nf, l, nlat)), np.zeros((nf, l, nlat))
    assert lib().or_shagc(nlat, nlon, nf, _p(g), _p(a), _p(b)) == 0
    return (a[0], b[0]) if squeeze else (a, b)


def shsgc(a, b, nlon):
    a, b = _f64(a), _f64(b)
    squeeze = a.ndim == 2
    if squeeze:
        a, b = a[None], b[None]
    nf, l, nlat = a.shape
    assert l == trunc_l(nlat, nlon)
    g = np.zeros((nf, nlat, nlon))
    assert lib().or_shsgc(nlat, nlon, nf, _p(a), _p(b), _p(g)) == 0
    return g[0] if squeeze else g


def trssph(da, nlatb, nlonb):
    da = _f64(da)
    squeeze = da.ndim == 2
    if squeeze:
        da = da[None]
    nf, nlata, nlona = da.shape
    db = np.zeros((nf, nlatb, nlonb))
    assert lib().or_trssph(nlata, nlona, nf, _p(da), nlatb, nlonb, _p(db)) == 0
    return db[0] if squeeze else db


def kernel(r):
    return lib().or_kernel(float(r))


def kerneltest():
    return lib().or_kerneltest()


def complagrforces(L, radius, x, y, z, gs=1.0, csk=1.0, faithful=False, law=0, eb=0.0):
    """One capsule: flat force-grid positions -> (f[3,nl], n[3,nl], area[nl]).

    law: 0 Skalak (membmodel.c:81-99), 1 neo-Hookean (membmodel.c:60-79).
    eb: bending modulus; nonzero adds the bending terms of ibend = 1
    (sph.f90:1705-1709), 0 is the reference with ibend = 0."""
    nl = 8 * (L + 1) ** 2
    x, y, z = _f64(x), _f64(y), _f64(z)
    assert x.size == nl
    out = [np.zeros(nl) for _ in range(7)]
    rc = lib().or_complagrforces_bend(L, radius, gs, csk, int(law), float(eb), int(faithful), _p(x), _p(y),
                                      _p(z), *[_p(o) for o in out])
    assert rc == 0, rc
    return np.stack(out[0:3]), np.stack(out[3:6]), out[6]


def capsule_spectra(L, radius, x, y, z, gs=1.0, csk=1.0):
    """Shape and filtered-force SH coefficients (degree < L+1), [3, N, N] each (a, b)."""
    N = L + 1
    outs = [np.zeros((3, N, N)) for _ in range(4)]
    rc = lib().or_capsule_spectra(L, radius, gs, csk, _p(_f64(x)), _p(_f64(y)), _p(_f64(z)), *[_p(o) for o in outs])
    assert rc == 0
    return outs


def interp(grid, u, v, w, x, y, z, faithful=False):
    itot, jtot, ktot, dx, dy, dz = grid
    n = x.size
    ul, vl, wl = np.zeros(n), np.zeros(n), np.zeros(n)
    lib().or_interp(itot, jtot, ktot, dx, dy, dz, int(faithful), _p(_f64(u)), _p(_f64(v)), _p(_f64(w)), n,
                    _p(_f64(x)), _p(_f64(y)), _p(_f64(z)), _p(ul), _p(vl), _p(wl))
    return ul, vl, wl


def spread(grid, x, y, z, fx, fy, fz, area, faithful=False):
    itot, jtot, ktot, dx, dy, dz = grid
    shape = (ktot + 2, jtot + 2, itot + 2)  # C view of Fortran (0:i1,0:j1,0:k1)
    gx, gy, gz = np.zeros(shape), np.zeros(shape), np.zeros(shape)
    lib().or_spread(itot, jtot, ktot, dx, dy, dz, int(faithful), x.size, _p(_f64(x)), _p(_f64(y)), _p(_f64(z)),
                    _p(_f64(fx)), _p(_f64(fy)), _p(_f64(fz)), _p(_f64(area)), _p(gx), _p(gy), _p(gz))
    return gx, gy, gz


def spread_ind(grid, x, y, z, nx, ny, nz, area, faithful=False):
    """lagr2eulrind (interp_spread.f90:978-1387): gx, gy, gz on (0:i1,0:j1,0:k1)."""
    itot, jtot, ktot, dx, dy, dz = grid
    shape = (ktot + 2, jtot + 2, itot + 2)
    gx, gy, gz = np.zeros(shape), np.zeros(shape), np.zeros(shape)
    lib().or_spread_ind(itot, jtot, ktot, dx, dy, dz, int(faithful), x.size, _p(_f64(x)), _p(_f64(y)), _p(_f64(z)),
                        _p(_f64(nx)), _p(_f64(ny)), _p(_f64(nz)), _p(_f64(area)), _p(gx), _p(gy), _p(gz))
    return gx, gy, gz


def overlap_lid(grid, nf, nr, u, v, w, p, indic):
    """interpolation (interpolation.f90:10-69) on one rank: the lid of the overlap mesh.

    grid = (itot, jtot, ktot, dx, dy, dz) with lx = itot dx as the library's
    context takes it; fields [k][j][i] with halos (the reference's (0:i1,0:j1,0:k1)).
    Returns ub, vb, wb, pb, indb [jtot nr + 2][itot nr + 2] (the (0:i1c,0:j1c)
    arrays).  dx = 1/(itot/lx) and dxc = 1/(itotc/lx) as param.f90:25-26,40-41
    evaluate them; every expression in the reference's order (numpy: no fused
    multiply-adds)."""
    itot, jtot = grid[0], grid[1]
    lx, ly = itot * grid[3], jtot * grid[4]
    dx, dy = 1.0 / (itot / lx), 1.0 / (jtot / ly)
    dxc, dyc = 1.0 / ((itot * nr) / lx), 1.0 / ((jtot * nr) / ly)
    i = np.arange(itot * nr + 2, dtype=np.float64)[None, :]
    j = np.arange(jtot * nr + 2, dtype=np.float64)[:, None]
    xp = (i * dxc) + ((0.5 * (1.0 - (1.0 / nr))) * dx)
    yp = (j * dyc) + ((0.5 * (1.0 - (1.0 / nr))) * dy)
    fx, fy = np.floor(xp / dx), np.floor(yp / dy)
    x1, x2 = fx * dx, (fx + 1.0) * dx
    y1, y2 = fy * dy, (fy + 1.0) * dy
    den = (x2 - x1) * (y2 - y1)
    c11 = ((x2 - xp) * (y2 - yp)) / den
    c12 = ((x2 - xp) * (yp - y1)) / den
    c21 = ((xp - x1) * (y2 - yp)) / den
    c22 = ((xp - x1) * (yp - y1)) / den
    im = np.broadcast_to(fx.astype(np.int64), c11.shape)
    jm = np.broadcast_to(fy.astype(np.int64), c11.shape)
    out = []
    for q, f in enumerate((u, v, w, p, indic)):
        lo, hi = f[nf], f[nf + 1]
        if q == 2:  # w at the face nf + 1
            g = lambda jj, ii: hi[jj, ii]
        else:
            g = lambda jj, ii: 0.5 * (lo[jj, ii] + hi[jj, ii])
        q11, q12, q21, q22 = g(jm, im), g(jm + 1, im), g(jm, im + 1), g(jm + 1, im + 1)
        out.append((((c11 * q11) + (c12 * q12)) + (c21 * q21)) + (c22 * q22))
    return out


def boundp(f):
    """boundp / boundind (bound.f90:88-139): Neumann z halos, then periodic x, y halo copies."""
    f[0] = f[1]
    f[-1] = f[-2]
    f[:, :, -1] = f[:, :, 1]
    f[:, :, 0] = f[:, :, -2]
    f[:, -1, :] = f[:, 1, :]
    f[:, 0, :] = f[:, -2, :]
    return f


def solver_rows(kmax, dz, e, shift=0.0):
    """initsolver(e) rows a, b, c (initsolver.f90:20-100): e = 0, 1 Neumann at both walls;
    e = 2 the no-slip ghost rows of u, v and b -= Rep/dt; e = 3 the w rows (w = 0 at the top
    face: an identity last row) and b -= Rep/dt.  shift = Rep/dt."""
    dzi = 1.0 / dz
    a = np.full(kmax, dzi * dzi)
    c = np.full(kmax, dzi * dzi)
    b = -(a + c)
    if e in (0, 1):
        b[0] = b[0] + a[0]
        b[-1] = b[-1] + c[-1]
        a[0] = 0.0
        c[-1] = 0.0
    else:
        if e == 2:
            b[0] = b[0] - a[0]
            b[-1] = b[-1] - c[-1]
            a[0] = 0.0
            c[-1] = 0.0
        else:
            b[-1] = 1.0
            a[0] = 0.0
            a[-1] = 0.0
            c[-1] = 0.0
        b = b - shift
        if e == 3:
            b[-1] = 1.0
    return a, b, c


def poisson_solver1d(rhs, dx, dy, dz, e=0, shift=0.0):
    """solver1d after initsolver(e) (solver.f90:43-157, initsolver.f90:11-130): the
    second-order Laplacian (minus shift = Rep/dt for e = 2, 3), periodic in x and y (real
    FFTs; eigenvalues -4/dx^2 sin^2(pi m / itot) and the same in y, initsolver.f90:111-130)
    and the rows of solver_rows in z, solved per mode by the reference's tridiagonal
    elimination: for e = 0, 1 its last pivot is exactly zero for the mean mode, which is then
    set to zero; for e = 3 the last row takes no eigenvalue.  rhs: [kmax, jtot, itot]."""
    kmax, jtot, itot = rhs.shape
    a, b, c = solver_rows(kmax, dz, e, shift)
    # xrt(2m) = -4 dxi^2 sin(2m pi / (2 itot))^2 (initsolver.f90:111-116), likewise yrt
    dxi, dyi = 1.0 / dx, 1.0 / dy
    lx = -4.0 * dxi * dxi * np.sin((2 * np.arange(itot // 2 + 1)) * np.pi / (2.0 * itot)) ** 2
    jm = np.minimum(np.arange(jtot), jtot - np.arange(jtot))  # complex y modes j and jtot - j share yrt
    ly = -4.0 * dyi * dyi * np.sin((2 * jm) * np.pi / (2.0 * jtot)) ** 2
    lam = ly[:, None] + lx[None, :]
    p = np.fft.rfft2(rhs, axes=(1, 2))
    d = np.zeros(p.shape)
    z = 1.0 / (b[0] + lam)
    d[0] = c[0] * z
    p[0] = p[0] * z
    for k in range(1, kmax - 1):
        z = 1.0 / ((b[k] + lam) - a[k] * d[k - 1])
        d[k] = c[k] * z
        p[k] = (p[k] - a[k] * p[k - 1]) * z
    z = ((b[-1] + lam) if e != 3 else b[-1]) - a[-1] * d[-2]
    nz = z != 0.0
    p[-1] = np.where(nz, (p[-1] - a[-1] * p[-2]) / np.where(nz, z, 1.0), 0.0)
    for k in range(kmax - 2, -1, -1):
        p[k] = p[k] - d[k] * p[k + 1]
    return np.fft.irfft2(p, s=(jtot, itot), axes=(1, 2))


def bounduvw(u, v, w, vb2=0.0, vt2=0.0):
    """bounduvw (bound.f90:7-86): walls u(0) = -u(1), v(0) = vb2 - v(1), w(0) = 0,
    u(k1) = -u(kmax), v(k1) = vt2 - v(kmax), w(kmax) = 0, w(k1) = w(kmax-1) (vb2 = vt2 = 0
    for iniu 'zer', 'poi', 'log' with no-slip walls; 2 bulk_v_sup both for free slip;
    lz shear and -lz shear for 'cou'); then the periodic x, y halo copies."""
    u[0] = -u[1]
    v[0] = vb2 - v[1]
    w[0] = 0.0
    u[-1] = -u[-2]
    v[-1] = vt2 - v[-2]
    w[-2] = 0.0
    w[-1] = w[-3]
    for f in (u, v, w):
        f[:, :, -1] = f[:, :, 1]
        f[:, :, 0] = f[:, :, -2]
        f[:, -1, :] = f[:, 1, :]
        f[:, 0, :] = f[:, -2, :]


def _sh(f, dk, dj, di):
    """f at (i + di, j + dj, k + dk) over the interior, f of shape (k1+1, j1+1, i1+1)."""
    K, J, I = f.shape
    return f[1 + dk:K - 1 + dk, 1 + dj:J - 1 + dj, 1 + di:I - 1 + di]


def _adv(U, V, W, comp, dxi, dyi, dzi):
    """The convective flux differences of momxad / momyad / momzad (mom.f90:9-54, 136-181,
    266-311) at one time level: returns the three (p, m) pairs of the x, y and z faces."""
    S = _sh
    if comp == 0:
        xp = 0.25 * (S(U, 0, 0, 1) + S(U, 0, 0, 0)) * (S(U, 0, 0, 1) + S(U, 0, 0, 0))
        xm = 0.25 * (S(U, 0, 0, -1) + S(U, 0, 0, 0)) * (S(U, 0, 0, -1) + S(U, 0, 0, 0))
        yp = 0.25 * (S(U, 0, 1, 0) + S(U, 0, 0, 0)) * (S(V, 0, 0, 1) + S(V, 0, 0, 0))
        ym = 0.25 * (S(U, 0, -1, 0) + S(U, 0, 0, 0)) * (S(V, 0, -1, 1) + S(V, 0, -1, 0))
        zp = 0.25 * (S(U, 1, 0, 0) + S(U, 0, 0, 0)) * (S(W, 0, 0, 1) + S(W, 0, 0, 0))
        zm = 0.25 * (S(U, -1, 0, 0) + S(U, 0, 0, 0)) * (S(W, -1, 0, 1) + S(W, -1, 0, 0))
    elif comp == 1:
        xp = 0.25 * (S(U, 0, 0, 0) + S(U, 0, 1, 0)) * (S(V, 0, 0, 0) + S(V, 0, 0, 1))
        xm = 0.25 * (S(U, 0, 0, -1) + S(U, 0, 1, -1)) * (S(V, 0, 0, 0) + S(V, 0, 0, -1))
        yp = 0.25 * (S(V, 0, 0, 0) + S(V, 0, 1, 0)) * (S(V, 0, 0, 0) + S(V, 0, 1, 0))
        ym = 0.25 * (S(V, 0, 0, 0) + S(V, 0, -1, 0)) * (S(V, 0, 0, 0) + S(V, 0, -1, 0))
        zp = 0.25 * (S(W, 0, 0, 0) + S(W, 0, 1, 0)) * (S(V, 1, 0, 0) + S(V, 0, 0, 0))
        zm = 0.25 * (S(W, -1, 0, 0) + S(W, -1, 1, 0)) * (S(V, -1, 0, 0) + S(V, 0, 0, 0))
    else:
        xp = 0.25 * (S(W, 0, 0, 0) + S(W, 0, 0, 1)) * (S(U, 0, 0, 0) + S(U, 1, 0, 0))
        xm = 0.25 * (S(W, 0, 0, 0) + S(W, 0, 0, -1)) * (S(U, 0, 0, -1) + S(U, 1, 0, -1))
        yp = 0.25 * (S(W, 0, 0, 0) + S(W, 0, 1, 0)) * (S(V, 0, 0, 0) + S(V, 1, 0, 0))
        ym = 0.25 * (S(W, 0, 0, 0) + S(W, 0, -1, 0)) * (S(V, 0, -1, 0) + S(V, 1, -1, 0))
        zp = 0.25 * (S(W, 0, 0, 0) + S(W, 1, 0, 0)) * (S(W, 0, 0, 0) + S(W, 1, 0, 0))
        zm = 0.25 * (S(W, 0, 0, 0) + S(W, -1, 0, 0)) * (S(W, 0, 0, 0) + S(W, -1, 0, 0))
    return (xp, xm), (yp, ym), (zp, zm)


def momad(comp, uo, vo, wo, uoo, voo, woo, dxi, dyi, dzi):
    """momxad / momyad / momzad: Adams-Bashforth convection, 1.5 (level n) - 0.5 (level n-1)."""
    (xp, xm), (yp, ym), (zp, zm) = _adv(uo, vo, wo, comp, dxi, dyi, dzi)
    (xpo, xmo), (ypo, ymo), (zpo, zmo) = _adv(uoo, voo, woo, comp, dxi, dyi, dzi)
    return (dxi * ((1.5 * (-xp + xm)) - (.5 * (-xpo + xmo)))
            + dyi * ((1.5 * (-yp + ym)) - (.5 * (-ypo + ymo)))
            + dzi * ((1.5 * (-zp + zm)) - (.5 * (-zpo + zmo))))


def flow_step(grid, dt, rep, uo, vo, wo, uoo, voo, woo, pnew, fx, fy, fz, vb2=0.0, vt2=0.0):
    """One step of the reference's FFT flow solver (fsolver = 'f', main.f90:333-347):
    fftuvw (fftuvw.f90:13-127: pressure gradient and IB force, momxp..momzp; Adams-Bashforth
    convection, momxad..momzad; the implicit Helmholtz solves of w with initsolver(3) and of
    u, v with initsolver(2)), bounduvw, fillps, solver1d after initsolver(1), boundp, correc,
    bounduvw, pnew += p, boundp.  Fields (0:i1,0:j1,0:k1) as [k][j][i]; uo.. is the velocity
    at the start of the step (the reference's unew = uo), uoo the one before.  Returns
    (u, v, w, pnew) at the end of the step."""
    itot, jtot, ktot, dx, dy, dz = grid
    dxi, dyi, dzi = 1.0 / dx, 1.0 / dy, 1.0 / dz
    I = (slice(1, -1),) * 3
    S = _sh
    rhs = []
    for comp, (f, dq) in enumerate(((fx, (0, 0, 1)), (fy, (0, 1, 0)), (fz, (1, 0, 0)))):
        dxyz = (dxi, dyi, dzi)[comp]
        durk = (-dxyz * ((S(pnew, *dq) - S(pnew, 0, 0, 0)))) + f[I]
        d = -durk
        d = d - momad(comp, uo, vo, wo, uoo, voo, woo, dxi, dyi, dzi)
        d = d - ((uo, vo, wo)[comp][I] / dt)
        rhs.append(d * rep)
    shift = rep / dt
    rhs[2][-1] = 0.0
    u, v, w = (np.zeros_like(uo) for _ in range(3))
    w[I] = poisson_solver1d(rhs[2], dx, dy, dz, e=3, shift=shift)
    u[I] = poisson_solver1d(rhs[0], dx, dy, dz, e=2, shift=shift)
    v[I] = poisson_solver1d(rhs[1], dx, dy, dz, e=2, shift=shift)
    bounduvw(u, v, w, vb2, vt2)
    dti = 1.0 / dt
    ps = ((S(w, 0, 0, 0) - S(w, -1, 0, 0)) * (dti * dzi) + (S(v, 0, 0, 0) - S(v, 0, -1, 0)) * (dti * dyi)
          + (S(u, 0, 0, 0) - S(u, 0, 0, -1)) * (dti * dxi))
    p = np.zeros_like(uo)
    p[I] = poisson_solver1d(ps, dx, dy, dz, e=1)
    boundp(p)
    u[I] = u[I] - (dt * dxi) * (S(p, 0, 0, 1) - S(p, 0, 0, 0))
    v[I] = v[I] - (dt * dyi) * (S(p, 0, 1, 0) - S(p, 0, 0, 0))
    w[I] = w[I] - (dt * dzi) * (S(p, 1, 0, 0) - S(p, 0, 0, 0))
    bounduvw(u, v, w, vb2, vt2)
    pn = _f64(pnew) + p
    boundp(pn)
    return u, v, w, pn


def indicator(grid, x, y, z, nx, ny, nz, area, visc0=1.0 / 0.0016, lam=1.0, thetainc=70.0 * np.pi / 180.0,
              ta=1160000.0, rep=0.0016, fy=None, fz=None):
    """indicator.f90:19-182 without the overlap mesh: the capsules raised by ktot/4 dz, G by
    lagr2eulrind, its central-difference divergence, the Poisson solve, boundind, the shift
    back, the 0.01 / 0.9 thresholds on the interior, the viscosity visc0 (1 + (lambda - 1) I)
    with boundp, and the centrifugal terms added to fy, fz (interior cells).
    Returns dict(g=(gx, gy, gz), indi=..., indic=..., visc=..., fy=..., fz=...)."""
    itot, jtot, ktot, dx, dy, dz = grid
    q = ktot // 4
    gx, gy, gz = spread_ind(grid, x, y, _f64(z) + q * dz, nx, ny, nz, area)
    shape = gx.shape
    dg = ((gx[1:-1, 1:-1, 2:] - gx[1:-1, 1:-1, :-2]) * 0.5 * (1.0 / dx)
          + (gy[1:-1, 2:, 1:-1] - gy[1:-1, :-2, 1:-1]) * 0.5 * (1.0 / dy)
          + (gz[2:, 1:-1, 1:-1] - gz[:-2, 1:-1, 1:-1]) * 0.5 * (1.0 / dz))
    indi = np.zeros(shape)
    indi[1:-1, 1:-1, 1:-1] = poisson_solver1d(dg, dx, dy, dz)
    boundp(indi)
    indic = np.zeros(shape)
    indic[1:ktot - q + 1, 1:-1, 1:-1] = indi[1 + q:ktot + 1, 1:-1, 1:-1]
    boundp(indic)
    inner = indic[1:-1, 1:-1, 1:-1]
    inner[inner < 0.01] = 0.0
    inner[inner >= 0.9] = 1.0
    visc = np.zeros(shape)
    visc[1:-1, 1:-1, 1:-1] = visc0 * (1.0 + (lam - 1.0) * indic[1:-1, 1:-1, 1:-1])
    boundp(visc)
    fy = np.zeros(shape) if fy is None else _f64(fy).copy()
    fz = np.zeros(shape) if fz is None else _f64(fz).copy()
    amp = (ta / rep ** 2) ** 0.25
    fy[1:-1, 1:-1, 1:-1] += 0.5 * (indic[1:-1, 1:-1, 1:-1] + indic[1:-1, 2:, 1:-1]) * np.sin(thetainc) * amp
    fz[1:-1, 1:-1, 1:-1] += 0.5 * (indic[1:-1, 1:-1, 1:-1] + indic[2:, 1:-1, 1:-1]) * (-np.cos(thetainc)) * amp
    return dict(g=(gx, gy, gz), dg=dg, indi=indi, indic=indic, visc=visc, fy=fy, fz=fz)


def update_pos(dt, lz, x, y, z, u, v, w):
    x, y, z = _f64(x).copy(), _f64(y).copy(), _f64(z).copy()
    lib().or_update_pos(x.size, dt, lz, _p(x), _p(y), _p(z), _p(_f64(u)), _p(_f64(v)), _p(_f64(w)))
    return x, y, z


def collisions(z, area, fz, dx, dy, col=5.68533e-2, betacol=15.36, rep=0.0016, rad0=None, dz=None):
    """collisions.f90:10-32: returns fz + the wall force (rad0 defaults to 2.5 dz)."""
    if rad0 is None:
        rad0 = 2.5 * dz
    out = _f64(fz).copy()
    lib().or_collisions(z.size, _p(_f64(z)), _p(_f64(area)), dx, dy, col, betacol, rep, rad0, _p(out))
    return out


def update_pos_capsules(offsets, dt, lx, ly, lz, x, y, z, u, v, w):
    """Update_Pos.f90:95-180 with the periodic shift of capsules whose centroid left the box."""
    x, y, z = _f64(x).copy(), _f64(y).copy(), _f64(z).copy()
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    lib().or_update_pos_capsules(off.size - 1, off.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), dt, lx, ly, lz,
                                 _p(x), _p(y), _p(z), _p(_f64(u)), _p(_f64(v)), _p(_f64(w)))
    return x, y, z


def surf_vol(x, y, z, nx, ny, nz, area, exy1_prev=0.0):
    out = np.zeros(7)
    lib().or_surf_vol(x.size, *[_p(_f64(a)) for a in (x, y, z, nx, ny, nz, area)], float(exy1_prev), _p(out))
    return out


def coupling_step(grid, degree, radius, u, v, w, x, y, z, gs=1.0, csk=1.0, faithful=False, nthreads=1):
    """Whole step over all capsules; returns dict of outputs and per-stage seconds."""
    itot, jtot, ktot, dx, dy, dz = grid
    degree = np.ascontiguousarray(degree, dtype=np.int32)
    radius = _f64(radius)
    n = x.size
    shape = (ktot + 2, jtot + 2, itot + 2)
    lag = [np.zeros(n) for _ in range(10)]
    eul = [np.zeros(shape) for _ in range(3)]
    t = np.zeros(3)
    rc = lib().or_coupling_step(itot, jtot, ktot, dx, dy, dz, degree.size, degree.ctypes.data_as(_ip), _p(radius),
                                gs, csk, int(faithful), int(nthreads), _p(_f64(u)), _p(_f64(v)), _p(_f64(w)),
                                _p(_f64(x)), _p(_f64(y)), _p(_f64(z)), *[_p(a) for a in lag], *[_p(a) for a in eul],
                                _p(t))
    assert rc == 0
    return dict(u=np.stack(lag[0:3]), f=np.stack(lag[3:6]), n=np.stack(lag[6:9]), area=lag[9],
                fgrid=np.stack(eul), seconds=t)


def skalak(I1, I2, I1de, I2de, gs=1.0, csk=1.0):
    out = np.zeros(6)
    lib().or_skalak(float(I1), float(I2), _p(_f64(I1de)), _p(_f64(I2de)), gs, csk, _p(out))
    return out


def membrane_law(law, I1, I2, I1de, I2de, gs=1.0, csk=1.0):
    """W1, W2, dW1[2], dW2[2] of law 0 (Skalak) or 1 (neo-Hookean)."""
    out = np.zeros(6)
    lib().or_membrane_law(int(law), float(I1), float(I2), _p(_f64(I1de)), _p(_f64(I2de)), gs, csk, _p(out))
    return out


def ref_membmodel(law="skalak"):
    """The reference's own membmodel.c, compiled into oracle/_ref (None if absent)."""
    path = os.path.join(_HERE, "_ref", "libmembmodel_%s.so" % law)
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    L.calpwspi_deri_.argtypes = [_dp] * 10
    L.calpwspi_deri_.restype = None
    L.ref_set_hf_gscell.argtypes = [ctypes.c_double]
    L.ref_set_hf_gscell.restype = None
    return L
