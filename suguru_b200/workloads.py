"""Seeded synthetic inputs for the coupling-step workloads.

The reference publishes no fixtures for this path, so every workload is built
here from seeds: capsule centres, SH degrees, membrane shapes and the
prescribed Eulerian velocity.  Point order per capsule is the reference's flat
order cap = i*m_capf + j on the 2N x 4N force grid (Gauss colatitude i north to
south, longitude j), N = L+1 (forcing.f90:37-44, sph.f90:75-88); capsules are
concatenated.  Coordinates follow the reference orientation
x = c_x + r sin(t) sin(p), y = c_y + r sin(t) cos(p), z = c_z + r cos(t)
(sph.f90:84-86).

Eulerian arrays are numpy C arrays of shape (ktot+2, jtot+2, itot+2): the
Fortran (0:i1, 0:j1, 0:k1) layout of common.f90:6, x fastest.
"""
from dataclasses import dataclass, field

import numpy as np


# ------------------------------------------------------------------ SH basics
def gauss_colat(nlat):
    """Gauss-Legendre colatitudes (0, pi), north to south, and weights."""
    x, w = np.polynomial.legendre.leggauss(nlat)
    return np.arccos(x)[::-1].copy(), w[::-1].copy()


def pbar(theta, L):
    """SPHEREPACK-normalised P^m_n(cos theta) as P[m, n, i] for m, n <= L."""
    theta = np.atleast_1d(np.asarray(theta, dtype=np.float64))
    x, s = np.cos(theta), np.sin(theta)
    P = np.zeros((L + 1, L + 1, theta.size))
    pmm = np.full(theta.size, np.sqrt(0.5))
    for m in range(L + 1):
        if m > 0:
            pmm = pmm * np.sqrt((2.0 * m + 1.0) / (2.0 * m)) * s
        P[m, m] = pmm
        if m + 1 <= L:
            P[m, m + 1] = np.sqrt(2.0 * m + 3.0) * x * pmm
        for n in range(m + 2, L + 1):
            a = np.sqrt((4.0 * n * n - 1.0) / (n * n - m * m))
            b = np.sqrt(((n - 1.0) ** 2 - m * m) / (4.0 * (n - 1.0) ** 2 - 1.0))
            P[m, n] = a * (x * P[m, n - 1] - b * P[m, n - 2])
    return P


def npts_of(L):
    return 8 * (L + 1) ** 2


def force_grid(L):
    N = L + 1
    th, w = gauss_colat(2 * N)
    ph = np.arange(4 * N) * (2.0 * np.pi / (4 * N))
    return th, w, ph


def shape_radius(L, R, ca, cb):
    """r(theta, phi) on the force grid from perturbation coefficients ca, cb [m, n]."""
    th, _, ph = force_grid(L)
    P = pbar(th, L)  # [m, n, i]
    r = np.full((th.size, ph.size), float(R))
    for m in range(L + 1):
        Gm_a = np.einsum("n,ni->i", ca[m], P[m])
        Gm_b = np.einsum("n,ni->i", cb[m], P[m])
        r += np.outer(Gm_a, np.cos(m * ph)) + np.outer(Gm_b, np.sin(m * ph))
    return r


def capsule_points(L, R, centre, ca=None, cb=None):
    """Flat (x, y, z) force points of one capsule."""
    th, _, ph = force_grid(L)
    if ca is None:
        r = np.full((th.size, ph.size), float(R))
    else:
        r = shape_radius(L, R, ca, cb)
    T, P = np.meshgrid(th, ph, indexing="ij")
    x = centre[0] + r * np.sin(T) * np.sin(P)
    y = centre[1] + r * np.sin(T) * np.cos(P)
    z = centre[2] + r * np.cos(T)
    return x.ravel(), y.ravel(), z.ravel()


def random_shape(rng, L, amp):
    """Perturbation coefficients ~ N(0, amp^2) * l^-2 for 1 <= l <= L (l=0 zero)."""
    ca = np.zeros((L + 1, L + 1))
    cb = np.zeros((L + 1, L + 1))
    for n in range(1, L + 1):
        for m in range(0, n + 1):
            ca[m, n] = rng.normal(0.0, amp) / n**2
            if m > 0:
                cb[m, n] = rng.normal(0.0, amp) / n**2
    return ca, cb


# ------------------------------------------------------------------ velocity
def velocity_modes(rng, nmodes=16, kmax=4):
    nx = rng.integers(-kmax, kmax + 1, size=nmodes)
    ny = rng.integers(-kmax, kmax + 1, size=nmodes)
    ph = rng.uniform(0.0, 2.0 * np.pi, size=nmodes)
    A = rng.normal(0.0, 1.0, size=(nmodes, 3))
    return dict(nx=nx, ny=ny, phase=ph, amp=A)


def velocity_field(grid, modes, shear=0.0, t=0.0, omega=None, dtype=np.float64):
    """u, v, w on the staggered MAC grid including the halo (0..i1 etc.).

    u_c = sum_q A_qc cos(2 pi nx x/Lx + 2 pi ny y/Ly + phase_q + omega_q t) sin(pi z/Lz),
    sampled at each component's own location; u additionally gets shear*z.
    """
    itot, jtot, ktot, dx, dy, dz = grid
    Lx, Ly, Lz = itot * dx, jtot * dy, ktot * dz
    i = np.arange(itot + 2, dtype=np.float64)
    j = np.arange(jtot + 2, dtype=np.float64)
    k = np.arange(ktot + 2, dtype=np.float64)
    face = dict(x=i * dx, y=j * dy, z=k * dz)
    cent = dict(x=(i - 0.5) * dx, y=(j - 0.5) * dy, z=(k - 0.5) * dz)
    out = []
    ph = modes["phase"] + (0.0 if omega is None else omega * t)
    for c in range(3):
        xs = face["x"] if c == 0 else cent["x"]
        ys = face["y"] if c == 1 else cent["y"]
        zs = face["z"] if c == 2 else cent["z"]
        F = np.zeros((jtot + 2, itot + 2))
        for q in range(len(ph)):
            ex = np.exp(1j * 2.0 * np.pi * modes["nx"][q] * xs / Lx)
            ey = np.exp(1j * (2.0 * np.pi * modes["ny"][q] * ys / Ly + ph[q]))
            F += modes["amp"][q, c] * np.real(np.outer(ey, ex))
        S = np.sin(np.pi * zs / Lz)
        U = S[:, None, None] * F[None, :, :]
        if c == 0 and shear:
            U = U + (shear * zs)[:, None, None]
        out.append(np.ascontiguousarray(U, dtype=dtype))
    return out


# ------------------------------------------------------------------ configs
@dataclass
class Workload:
    name: str
    grid: tuple               # (itot, jtot, ktot, dx, dy, dz)
    degree: np.ndarray        # int32 [ncap]
    radius: np.ndarray        # float64 [ncap]
    centre: np.ndarray        # [ncap, 3]
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    modes: dict
    shear: float
    gs: float = 1.0
    csk: float = 1.0
    shapes: list = field(default_factory=list)

    @property
    def ncap(self):
        return int(self.degree.size)

    @property
    def npts(self):
        return int(self.x.size)

    @property
    def offsets(self):
        return np.concatenate([[0], np.cumsum([npts_of(int(L)) for L in self.degree])]).astype(np.int64)

    def velocity(self, dtype=np.float64, t=0.0, omega=None):
        return velocity_field(self.grid, self.modes, self.shear, t=t, omega=omega, dtype=dtype)


def _place(rng, ncap, radii, box, gap, zmargin, rmax_factor=1.25, max_tries=200000):
    Lx, Ly, Lz = box
    cen = np.zeros((ncap, 3))
    placed = 0
    tries = 0
    while placed < ncap:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place capsules")
        r = radii[placed] * rmax_factor
        c = np.array([rng.uniform(0, Lx), rng.uniform(0, Ly), rng.uniform(r + zmargin, Lz - r - zmargin)])
        ok = True
        if placed:
            d = cen[:placed] - c
            d[:, 0] -= Lx * np.round(d[:, 0] / Lx)
            d[:, 1] -= Ly * np.round(d[:, 1] / Ly)
            dist = np.sqrt((d**2).sum(1))
            ok = np.all(dist >= radii[:placed] * rmax_factor + r + gap)
        if ok:
            cen[placed] = c
            placed += 1
    return cen


def _build(name, grid, degree, radius, centre, amps, shape_rng, modes, shear):
    xs, ys, zs, shapes = [], [], [], []
    for c in range(len(degree)):
        L = int(degree[c])
        ca, cb = random_shape(shape_rng, L, amps[c])
        shapes.append((ca, cb))
        x, y, z = capsule_points(L, radius[c], centre[c], ca, cb)
        xs.append(x)
        ys.append(y)
        zs.append(z)
    return Workload(name, grid, np.asarray(degree, np.int32), np.asarray(radius, np.float64), centre,
                    np.concatenate(xs), np.concatenate(ys), np.concatenate(zs), modes, shear, shapes=shapes)


def config0():
    """Single capsule, L=15, R=8dx at the box centre, grid 128x64x64, dx=1/32."""
    dx = 1.0 / 32
    grid = (128, 64, 64, dx, dx, dx)
    R = 8 * dx
    modes = velocity_modes(np.random.default_rng(1))
    return _build("c0_single_L15", grid, [15], [R], np.array([[2.0, 1.0, 1.0]]), [0.05 * R],
                  np.random.default_rng(0), modes, 0.0)


def config1(ncap=256):
    """Dense suspension: 256 capsules, L=15, R=8dx, grid 256x256x128."""
    dx = 1.0 / 32
    grid = (256, 256, 128, dx, dx, dx)
    R = 8 * dx
    radius = np.full(ncap, R)
    centre = _place(np.random.default_rng(2), ncap, radius, (256 * dx, 256 * dx, 128 * dx), 2 * dx, 2 * dx)
    modes = velocity_modes(np.random.default_rng(1))
    return _build("c1_dense_256x_L15", grid, np.full(ncap, 15), radius, centre, np.full(ncap, 0.05 * R),
                  np.random.default_rng(3), modes, 1.0)


def config2_degrees(rng, ncap, dx):
    radius = rng.uniform(4.0, 12.0, size=ncap) * dx
    degree = np.clip(np.round(1.5 * radius / dx), 7, 23).astype(np.int32)
    return radius, degree


def config2(ncap=1024):
    """Uneven batch: 1024 capsules, R~U[4,12]dx, L=clamp(round(1.5R/dx),7,23), grid 512x256x256."""
    dx = 1.0 / 32
    grid = (512, 256, 256, dx, dx, dx)
    rng = np.random.default_rng(4)
    radius, degree = config2_degrees(rng, ncap, dx)
    amp = rng.uniform(0.01, 0.1, size=ncap) * radius
    centre = _place(np.random.default_rng(5), ncap, radius, (512 * dx, 256 * dx, 256 * dx), 2 * dx, 2 * dx)
    modes = velocity_modes(np.random.default_rng(1))
    return _build("c2_uneven_1024x", grid, degree, radius, centre, amp, np.random.default_rng(6), modes, 1.0)


def small_config(ncap=3, seed=7, grid=(64, 48, 40), degrees=(7, 11, 15)):
    """A few capsules on a small grid, some straddling the periodic x/y faces."""
    dx = 1.0 / 16
    g = (grid[0], grid[1], grid[2], dx, dx, dx)
    rng = np.random.default_rng(seed)
    degree = np.array([degrees[c % len(degrees)] for c in range(ncap)], np.int32)
    radius = np.array([(4.0 + 1.5 * (c % 3)) * dx for c in range(ncap)])
    Lx, Ly, Lz = grid[0] * dx, grid[1] * dx, grid[2] * dx
    centre = np.zeros((ncap, 3))
    for c in range(ncap):
        centre[c] = [(0.02 + 0.37 * c) * Lx % Lx, (0.97 - 0.31 * c) * Ly % Ly, 0.5 * Lz + (c - 1) * 0.1 * Lz]
    modes = velocity_modes(rng)
    return _build("small", g, degree, radius, centre, 0.05 * radius, rng, modes, 0.5)
