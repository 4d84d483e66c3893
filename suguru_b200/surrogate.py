"""Training data, exact linear response and training of the membrane-force surrogate.

The surrogate (suguru_b200/csrc/sg_surrogate*.cu) replaces the plain Skalak
force of capsules of SH degree 15 in the mixed-precision step:
  y = (L0 + C L1) x + a^2 MLP(x / a, C, log a),  a = |x|
with x the 768 displacement coefficients divided by R (slot 0 carrying C) and
y the force coefficients after the reference's force filter times R / Gs.
This module only drives the library through its C ABI:

  * `sample_shapes` draws capsule shapes: radial perturbations
    r = R (1 + sum q_lm Y_lm) and general vector displacements, with
    q ~ N(0, amp^2) l^-2 and amp log-uniform in [amp_lo, amp_hi] (the
    training distribution: 1e-3 to 0.2 R, C uniform in [0.5, 2]);
  * `make_dataset` labels them with the plain FP64 model on the GPU
    (sg_capsule_spectra);
  * `linear_response` differentiates the plain FP64 model at the sphere by
    central differences, column by column, for C = 0 and C = 1 (the force is
    affine in C), giving L0 and L1;
  * `train` runs the library's own training kernels (sg_surrogate_train);
  * `calibrate_trust` picks the residual-check limits on held-out data.
"""
import numpy as np

from . import workloads as W
from .coupling import CouplingStep

L_SUR = 15
N_SUR = L_SUR + 1
NN = N_SUR * N_SUR
DIN = 3 * NN


# ------------------------------------------------------------------ slots
def slot_table(N=N_SUR):
    """(ab, m, n) per slot of one component: a(m,n) m-major for m <= n, then b(m,n) for m >= 1."""
    out = []
    for m in range(N):
        for n in range(m, N):
            out.append((0, m, n))
    for m in range(1, N):
        for n in range(m, N):
            out.append((1, m, n))
    return np.array(out, dtype=np.int64)


def slots_from_ab(a, b):
    """[3][N][N] a, b (SPHEREPACK coefficients) -> flat slot vector [3 N^2]."""
    N = a.shape[-1]
    t = slot_table(N)
    out = np.zeros(3 * N * N)
    for c in range(3):
        src = np.where(t[:, 0] == 0, a[c][t[:, 1], t[:, 2]], b[c][t[:, 1], t[:, 2]])
        out[c * N * N:(c + 1) * N * N] = src
    return out


def synthesis_basis(L=L_SUR):
    """B[s, p]: the field at force-grid point p of a unit coefficient in slot s,
    SPHEREPACK synthesis (shsgc.f: a cos(m phi) - b sin(m phi), half weight on m = 0)."""
    N = L + 1
    th, _, ph = W.force_grid(L)
    P = W.pbar(th, L)  # [m, n, i]
    t = slot_table(N)
    Bm = np.zeros((t.shape[0], th.size, ph.size))
    for s, (ab, m, n) in enumerate(t):
        h = 0.5 if m == 0 else 1.0
        ang = np.cos(m * ph) if ab == 0 else -np.sin(m * ph)
        Bm[s] = h * np.outer(P[m, n], ang)
    return Bm.reshape(t.shape[0], -1)


def _sphere_dirs(L=L_SUR):
    th, _, ph = W.force_grid(L)
    T, Pp = np.meshgrid(th, ph, indexing="ij")
    return np.stack([np.sin(T) * np.sin(Pp), np.sin(T) * np.cos(Pp), np.cos(T)]).reshape(3, -1)


def _degree_of_slot(N=N_SUR):
    return slot_table(N)[:, 2]


# ------------------------------------------------------------------ shapes
def _draw(rng, ncap, nslot, decay, amp_lo, amp_hi, general_frac):
    amp = np.exp(rng.uniform(np.log(amp_lo), np.log(amp_hi), size=ncap))
    general = rng.uniform(size=ncap) < general_frac
    q = rng.normal(size=(ncap, nslot)) * decay * amp[:, None]
    qg = rng.normal(size=(3, ncap, nslot)) * decay * amp[None, :, None]
    return amp, general, q, qg


def sample_shapes(rng, ncap, R=1.0, amp_lo=1e-3, amp_hi=0.2, general_frac=0.5, L=L_SUR, basis=None):
    """Point coordinates [3][ncap * npts] of ncap capsules centred at the origin, and their amplitudes.

    Radial family: r = R (1 + sum q Y); general family: an independent
    displacement R sum q_c Y per component; q ~ N(0, amp^2) l^-2 for l >= 1."""
    basis = synthesis_basis(L) if basis is None else basis
    S = _sphere_dirs(L)
    deg = _degree_of_slot(L + 1).astype(np.float64)
    decay = np.where(deg >= 1, 1.0 / np.maximum(deg, 1.0) ** 2, 0.0)
    amp, general, q, qg = _draw(rng, ncap, basis.shape[0], decay, amp_lo, amp_hi, general_frac)
    dr = q @ basis  # [ncap, npts]
    dg = qg @ basis  # [3, ncap, npts]
    g = general[:, None]
    pos = R * S[:, None, :] * (1.0 + np.where(g, 0.0, dr))[None] + R * np.where(g[None], dg, 0.0)
    return pos.reshape(3, -1), amp, general


def _sample_shapes_device(rng, ncap, basis_t, S_t, decay, R, amp_lo=1e-3, amp_hi=0.2, general_frac=0.5):
    """sample_shapes with the synthesis on the GPU (same random draws, torch for the products)."""
    import torch
    amp, general, q, qg = _draw(rng, ncap, basis_t.shape[0], decay, amp_lo, amp_hi, general_frac)
    dev = basis_t.device
    dr = torch.from_numpy(q).to(dev) @ basis_t
    dg = torch.from_numpy(qg).to(dev) @ basis_t
    g = torch.from_numpy(general).to(dev)[:, None]
    pos = R * S_t[:, None, :] * (1.0 + torch.where(g, torch.zeros_like(dr), dr))[None] + R * torch.where(
        g[None], dg, torch.zeros_like(dg))
    pos = pos.reshape(3, -1)
    return [pos[c].contiguous() for c in range(3)], amp


def _context(ncap, precision="fp64", mem="host"):
    grid = (16, 16, 16, 0.25, 0.25, 0.25)
    return CouplingStep(grid, np.full(ncap, L_SUR), np.full(ncap, 1.0), precision=precision, mem=mem)


def make_dataset(n, seed, batch=1024, R=1.0, csk_range=(0.5, 2.0), device=True, **shape_kw):
    """n labelled samples: X [n][768] (slot 0 = C), Y [n][768], and the amplitudes.

    Labels come from the plain FP64 model on the GPU; with device=True the
    shapes are also synthesised there (torch products, numpy random draws)."""
    rng = np.random.default_rng(seed)
    basis = synthesis_basis()
    X = np.zeros((n, DIN), np.float32)
    Y = np.zeros((n, DIN), np.float32)
    A = np.zeros(n)
    cs = None
    if device:
        import torch
        basis_t = torch.from_numpy(basis).cuda()
        S_t = torch.from_numpy(_sphere_dirs()).cuda()
        deg = _degree_of_slot().astype(np.float64)
        decay = np.where(deg >= 1, 1.0 / np.maximum(deg, 1.0) ** 2, 0.0)
    for k0 in range(0, n, batch):
        k1 = min(n, k0 + batch)
        nc = k1 - k0
        if cs is None or cs.degree.size != nc:
            cs = _context(nc, mem="device" if device else "host")
        if device:
            pos, amp = _sample_shapes_device(rng, nc, basis_t, S_t, decay, R, **shape_kw)
            torch.cuda.synchronize()
        else:
            pos, amp, _ = sample_shapes(rng, nc, R=R, basis=basis, **shape_kw)
        C = rng.uniform(*csk_range, size=nc)
        cs.set_capsule_membrane(gs=1.0, csk=C)
        d, f = cs.capsule_spectra(pos[0], pos[1], pos[2])
        if device:
            d, f = d.cpu().numpy(), f.cpu().numpy()
        d = d.reshape(nc, DIN) / R
        f = f.reshape(nc, DIN) * R  # Gs = 1
        d[:, 0] = C
        d[:, NN] = 0.0
        d[:, 2 * NN] = 0.0
        X[k0:k1] = d
        Y[k0:k1] = f
        A[k0:k1] = amp
    return X, Y, A


def linear_response(eps=1e-4, R=1.0):
    """L0, L1 [768][768]: d(force coefficients * R)/d(displacement coefficients / R) at the sphere."""
    basis = synthesis_basis()
    S = _sphere_dirs()
    nslot = basis.shape[0]
    cols = [(c, s) for c in range(3) for s in range(nslot)]
    ncap = 2 * len(cols)
    cs = _context(ncap)
    pos = np.repeat(R * S[:, None, :], ncap, axis=1)  # [3][ncap][npts]
    for k, (c, s) in enumerate(cols):
        pos[c, 2 * k] += eps * R * basis[s]
        pos[c, 2 * k + 1] -= eps * R * basis[s]
    pos = pos.reshape(3, -1)
    J = []
    for C in (0.0, 1.0):
        cs.set_capsule_membrane(gs=1.0, csk=C)
        _, f = cs.capsule_spectra(pos[0], pos[1], pos[2])
        f = f.reshape(ncap, DIN) * R
        J.append(((f[0::2] - f[1::2]) / (2 * eps)).T)  # [out][in]
    L0, L1 = J[0], J[1] - J[0]
    for Lm in (L0, L1):  # translations carry no force; slot 0 holds C, not a displacement
        Lm[:, [0, NN, 2 * NN]] = 0.0
    cs.close()
    return L0.astype(np.float32), L1.astype(np.float32)


def train(cs, X, Y, L0, L1, epochs=30, batch=1024, lr=1e-3, seed=0):
    """Set the linear response and train the network of a surrogate context."""
    cs.surrogate_set_linear(L0, L1)
    return cs.surrogate_train(X, Y, epochs=epochs, batch=batch, lr=lr, seed=seed)


def rel_err_rows(Yp, Y):
    return np.linalg.norm(Yp - Y, axis=1) / np.maximum(np.linalg.norm(Y, axis=1), 1e-30)


def calibrate_trust(cs, Xv, Yv, tol, c_range=(0.5, 2.0)):
    """Residual-check limits from held-out data: the largest displacement
    amplitude and MLP/linear ratio below which every validation sample's
    relative force-coefficient error stays within tol."""
    Yp = cs.surrogate_predict(Xv, parts=3)
    Ylin = cs.surrogate_predict(Xv, parts=1)
    err = rel_err_rows(Yp, Yv)
    amp = np.linalg.norm(Xv[:, 1:], axis=1)
    ratio = np.linalg.norm(Yp - Ylin, axis=1) / np.maximum(np.linalg.norm(Ylin, axis=1), 1e-30)
    order = np.argsort(amp)
    bad = np.where(err[order] > tol)[0]
    amp_max = float(amp[order][bad[0] - 1]) if bad.size and bad[0] > 0 else (
        float(amp.max()) if not bad.size else 0.0)
    ok = amp <= amp_max
    ratio_max = float(ratio[ok].max()) if ok.any() else 0.0
    cs.surrogate_set_trust(amp_max, ratio_max, *c_range)
    return dict(amp_max=amp_max, ratio_max=ratio_max, err=err, amp=amp, ratio=ratio)
