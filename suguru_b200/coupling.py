"""Host-side mirror of the reference's coupling-step subroutines over the C ABI.

The reference (Fortran, WhiteTshirtXI/Suguru) calls per time step
(main.f90:225-241) ``eulr2lagr``, ``complagrforces``, ``lagr2eulr``,
``Update_Pos`` and ``surf_vol`` on module globals.  ``CouplingStep`` keeps
those names; each method calls the matching ``sg_*`` entry point of
``libsuguru_b200.so`` (include/sg_coupling.h).

Arrays are either numpy host arrays (``mem="host"``: the library copies them
in and out) or torch CUDA tensors (``mem="device"``).  Eulerian arrays have the
Fortran (0:i1, 0:j1, 0:k1) layout, i.e. numpy shape (ktot+2, jtot+2, itot+2)
C-contiguous; Lagrangian arrays are flat, capsules concatenated, each in the
reference order cap = i*m_capf + j.

There is no CPU fallback: constructing a ``CouplingStep`` without the built
library or without a CUDA device raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBPATH = os.path.join(_HERE, "libsuguru_b200.so")
_LIB = None

SG_PREC_FP64, SG_PREC_MIXED = 0, 1
SG_MEM_HOST, SG_MEM_DEVICE = 0, 1
ERRORS = {0: "SG_OK", 1: "SG_ERR_CONFIG", 2: "SG_ERR_CUDA", 3: "SG_ERR_TIMEOUT", 4: "SG_ERR_FALLBACK",
          5: "SG_ERR_ARG", 6: "SG_ERR_STATE", 7: "SG_ERR_TOO_LARGE"}

# every symbol declared in include/sg_coupling.h
EXPORTS = ["sg_create", "sg_destroy", "sg_last_error", "sg_synchronize", "sg_interp", "sg_membrane_force",
           "sg_spread", "sg_step", "sg_update_pos", "sg_surf_vol", "sg_gauss", "sg_legendre",
           "sg_last_launch_count", "sg_set_profiling", "sg_stage_times", "sg_spread_noalloc",
           "sg_set_tile_shape", "sg_get_tile_shape", "sg_autotune", "sg_graph_capture", "sg_graph_launch",
           "sg_graph_release", "sg_set_capsule_membrane", "sg_capsule_spectra", "sg_surrogate_param_count",
           "sg_surrogate_params", "sg_surrogate_set_linear", "sg_surrogate_train", "sg_surrogate_predict",
           "sg_surrogate_set_trust", "sg_surrogate_last_counts", "sg_set_point_split", "sg_get_point_split",
           "sg_set_tensor_cores", "sg_set_legendre_terms", "sg_get_legendre_terms", "sg_set_capsule_law",
           "sg_set_legendre_tile_rows", "sg_get_legendre_tile_rows", "sg_set_wall_collisions", "sg_collisions",
           "sg_set_indicator_params", "sg_indicator", "sg_set_flow_params", "sg_flow_step",
           "sg_contraction_work", "sg_set_capsule_bending", "sg_overlap_lid", "sg_set_fused_force",
           "sg_get_fused_force"]
# test hooks declared in include/sg_testing.h
TEST_EXPORTS = ["sg_test_legendre", "sg_test_gemm", "sg_test_mlp_grad"]
WORKLOAD_EXPORTS = ["sg_prescribed_flow"]  # include/sg_workload.h
# spreading tile shapes (cells); 0 in x: whole x rows (FP32 only)
TILE_SHAPES = ((32, 8, 4), (16, 16, 8), (32, 8, 8), (8, 8, 4), (0, 4, 4), (0, 8, 4), (32, 16, 4))
STAGES = ("bin", "interp", "membrane", "spread", "contract")


class SgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (ERRORS.get(code, code), msg))
        self.code = code


class sg_config(ctypes.Structure):
    _fields_ = [("itot", ctypes.c_int), ("jtot", ctypes.c_int), ("ktot", ctypes.c_int),
                ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
                ("ncap", ctypes.c_int), ("degree", ctypes.POINTER(ctypes.c_int)),
                ("radius", ctypes.POINTER(ctypes.c_double)), ("gs", ctypes.c_double), ("csk", ctypes.c_double),
                ("precision", ctypes.c_int), ("surrogate", ctypes.c_int), ("mem", ctypes.c_int),
                ("device", ctypes.c_int), ("async_", ctypes.c_int), ("stream", ctypes.c_void_p)]


def library_path():
    return _LIBPATH


def lib():
    """Load libsuguru_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(_LIBPATH):
        raise RuntimeError("libsuguru_b200.so is not built; run suguru_b200/build.py (no CPU fallback exists)")
    L = ctypes.CDLL(_LIBPATH)
    vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
    L.sg_create.argtypes = [ctypes.POINTER(sg_config), ctypes.POINTER(ctypes.c_void_p)]
    L.sg_destroy.argtypes = [vp]
    L.sg_destroy.restype = None
    L.sg_last_error.argtypes = [vp]
    L.sg_last_error.restype = ctypes.c_char_p
    L.sg_synchronize.argtypes = [vp]
    L.sg_interp.argtypes = [vp] * 10
    L.sg_membrane_force.argtypes = [vp] * 11
    L.sg_spread.argtypes = [vp] * 11
    L.sg_step.argtypes = [vp] * 20
    L.sg_update_pos.argtypes = [vp, ctypes.c_double] + [vp] * 6
    L.sg_surf_vol.argtypes = [vp] * 10
    L.sg_set_wall_collisions.argtypes = [vp, ctypes.c_int] + [ctypes.c_double] * 4
    L.sg_collisions.argtypes = [vp] * 4
    L.sg_set_indicator_params.argtypes = [vp] + [ctypes.c_double] * 5
    L.sg_indicator.argtypes = [vp] * 12
    L.sg_set_flow_params.argtypes = [vp] + [ctypes.c_double] * 3
    L.sg_flow_step.argtypes = [vp, ctypes.c_double] + [vp] * 13
    L.sg_gauss.argtypes = [ctypes.c_int, dp, dp]
    L.sg_legendre.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, dp, dp, dp]
    L.sg_last_launch_count.argtypes = [vp]
    L.sg_set_profiling.argtypes = [vp, ctypes.c_int]
    L.sg_stage_times.argtypes = [vp, ctypes.POINTER(ctypes.c_float), ctypes.c_int]
    L.sg_contraction_work.argtypes = [vp, dp]
    ip = ctypes.POINTER(ctypes.c_int)
    L.sg_set_tile_shape.argtypes = [vp, ctypes.c_int]
    L.sg_set_point_split.argtypes = [vp, ctypes.c_int]
    L.sg_set_tensor_cores.argtypes = [vp, ctypes.c_int]
    L.sg_set_capsule_law.argtypes = [vp, vp]
    L.sg_set_capsule_bending.argtypes = [vp, vp]
    L.sg_set_fused_force.argtypes = [vp, ctypes.c_int]
    L.sg_get_fused_force.argtypes = [vp]
    L.sg_overlap_lid.argtypes = [vp, ctypes.c_int, ctypes.c_int] + [vp] * 10
    L.sg_set_legendre_tile_rows.argtypes = [vp, ctypes.c_int]
    L.sg_get_legendre_tile_rows.argtypes = [vp]
    L.sg_set_legendre_terms.argtypes = [vp, ctypes.c_int]
    L.sg_get_legendre_terms.argtypes = [vp, ctypes.c_int]
    L.sg_get_point_split.argtypes = [vp]
    L.sg_get_tile_shape.argtypes = [vp, ip, ip, ip, ip]
    L.sg_autotune.argtypes = [vp] * 20 + [ctypes.c_int, ip, ctypes.POINTER(ctypes.c_float)]
    L.sg_graph_capture.argtypes = [vp] * 20
    L.sg_graph_launch.argtypes = [vp]
    L.sg_graph_release.argtypes = [vp]
    L.sg_prescribed_flow.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [ctypes.c_int] + [vp] * 5 + \
        [ctypes.c_double, vp, ctypes.c_int] + [vp] * 5
    L.sg_test_legendre.argtypes = [ctypes.c_int] * 6 + [vp] * 3
    L.sg_test_mlp_grad.argtypes = [ctypes.c_int] * 4 + [vp] * 5
    L.sg_set_capsule_membrane.argtypes = [vp] * 3
    L.sg_capsule_spectra.argtypes = [vp] * 6
    L.sg_surrogate_param_count.argtypes = []
    L.sg_surrogate_param_count.restype = ctypes.c_long
    L.sg_surrogate_params.argtypes = [vp, ctypes.c_int, vp, ctypes.c_long]
    L.sg_surrogate_set_linear.argtypes = [vp] * 3
    L.sg_surrogate_train.argtypes = [vp, vp, vp, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                     ctypes.c_ulonglong, vp]
    L.sg_surrogate_predict.argtypes = [vp, vp, ctypes.c_long, ctypes.c_int, vp]
    L.sg_surrogate_set_trust.argtypes = [vp] + [ctypes.c_float] * 4
    L.sg_surrogate_last_counts.argtypes = [vp, ip, ip]
    L.sg_test_gemm.argtypes = [ctypes.c_int] * 4 + [vp] * 3 + [ctypes.c_int, ctypes.c_float] + [vp] * 4 + [
        ctypes.c_int]
    d = ctypes.c_double
    L.sg_spread_noalloc.argtypes = ([ctypes.c_int] * 3 + [d] * 3 + [ctypes.c_long] + [vp] * 11)
    _LIB = L
    return L


def test_legendre(A, B, tensor_cores=True, tri=False, terms=3, tile_rows=128):
    """D[m,q,j] = sum_k A[m,q,k] B[m,j,k] through one Legendre kernel (test hook).

    tensor_cores: the tcgen05 kernel with `terms` split products (3: BF16x3,
    6: BF16x6) on tiles of `tile_rows` (64 or 128) data rows; otherwise the
    FP32 CUDA-core kernel.
    """
    A = np.ascontiguousarray(A, dtype=np.float32)
    B = np.ascontiguousarray(B, dtype=np.float64)
    M, Q, K = A.shape
    J = B.shape[1]
    assert B.shape == (M, J, K)
    D = np.zeros((M, Q, J), dtype=np.float32)
    mode = (int(terms) + (100 if tile_rows == 64 else 0)) if tensor_cores else 0
    rc = lib().sg_test_legendre(mode, M, Q, J, K, int(bool(tri)), _ptr(B), _ptr(A), _ptr(D))
    if rc:
        raise SgError(rc, "sg_test_legendre")
    return D


def to_bf16_bits(x):
    """Round-to-nearest-even FP32 -> bf16 bit patterns (uint16)."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return r


def from_bf16_bits(b):
    return (np.asarray(b, dtype=np.uint32) << 16).view(np.float32)


def test_gemm(A, B, split=False, bias=None, gelu=False, alpha=1.0, splitk=False):
    """C = alpha A B^T (+ bias) (GELU) on the tensor cores (test hook).

    split=False: A, B are rounded to bf16 first; split=True: FP32 in, BF16x3.
    Returns (C, Cpre, Cb, CbT) with the bf16 outputs as FP32 values."""
    A = np.ascontiguousarray(A, dtype=np.float32)
    B = np.ascontiguousarray(B, dtype=np.float32)
    M, K = A.shape
    N = B.shape[0]
    a = A if split else to_bf16_bits(A)
    b = B if split else to_bf16_bits(B)
    C = np.zeros((M, N), np.float32)
    P = np.zeros((M, N), np.float32)
    Cb = np.zeros((M, N), np.uint16)
    CbT = np.zeros((N, M), np.uint16)
    bi = None if bias is None else np.ascontiguousarray(bias, dtype=np.float32)
    rc = lib().sg_test_gemm(int(split), M, N, K, _ptr(a), _ptr(b), _ptr(bi), int(gelu), ctypes.c_float(alpha),
                            _ptr(C), _ptr(P), _ptr(Cb), _ptr(CbT), int(splitk))
    if rc:
        raise SgError(rc, "sg_test_gemm")
    return C, P, from_bf16_bits(Cb), from_bf16_bits(CbT)


def test_mlp_grad(params, X, T, din, dh, dout):
    """Loss and parameter gradients of one forward/backward pass (test hook)."""
    params = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    T = np.ascontiguousarray(T, dtype=np.float32)
    B = X.shape[0]
    loss = np.zeros(1, np.float32)
    grads = np.zeros_like(params)
    rc = lib().sg_test_mlp_grad(din, dh, dout, B, _ptr(params), _ptr(X), _ptr(T), _ptr(loss), _ptr(grads))
    if rc:
        raise SgError(rc, "sg_test_mlp_grad")
    return float(loss[0]), grads


def gauss(nlat):
    th, w = np.zeros(nlat), np.zeros(nlat)
    dp = ctypes.POINTER(ctypes.c_double)
    rc = lib().sg_gauss(nlat, th.ctypes.data_as(dp), w.ctypes.data_as(dp))
    if rc:
        raise SgError(rc, "sg_gauss")
    return th, w


def legendre(theta, mm, nn):
    P, D, D2 = (np.zeros((mm, nn)) for _ in range(3))
    dp = ctypes.POINTER(ctypes.c_double)
    rc = lib().sg_legendre(float(theta), mm, nn, P.ctypes.data_as(dp), D.ctypes.data_as(dp), D2.ctypes.data_as(dp))
    if rc:
        raise SgError(rc, "sg_legendre")
    return P, D, D2


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):  # torch tensor
        assert a.is_contiguous()
        return ctypes.c_void_p(a.data_ptr())
    assert a.flags.c_contiguous
    return ctypes.c_void_p(a.ctypes.data)


class CouplingStep:
    """One coupling-step context (sg_create) over a fixed set of capsules."""

    def __init__(self, grid, degree, radius, gs=1.0, csk=1.0, precision="fp64", mem="host", device=0,
                 surrogate=False, stream=None, async_=False):
        self.grid = tuple(grid)
        itot, jtot, ktot, dx, dy, dz = self.grid
        self.degree = np.ascontiguousarray(degree, dtype=np.int32)
        self.radius = np.ascontiguousarray(radius, dtype=np.float64)
        self.precision = precision
        self.mem = mem
        self.rdtype = np.float64 if precision == "fp64" else np.float32
        self.npts = int(sum(8 * (int(L) + 1) ** 2 for L in self.degree))
        self.field_shape = (ktot + 2, jtot + 2, itot + 2)
        cfg = sg_config()
        cfg.itot, cfg.jtot, cfg.ktot = itot, jtot, ktot
        cfg.lx, cfg.ly, cfg.lz = itot * dx, jtot * dy, ktot * dz
        cfg.ncap = int(self.degree.size)
        cfg.degree = self.degree.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        cfg.radius = self.radius.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        cfg.gs, cfg.csk = float(gs), float(csk)
        cfg.precision = SG_PREC_FP64 if precision == "fp64" else SG_PREC_MIXED
        cfg.surrogate = int(bool(surrogate))
        cfg.mem = SG_MEM_HOST if mem == "host" else SG_MEM_DEVICE
        cfg.device = int(device)
        cfg.async_ = int(bool(async_))
        cfg.stream = stream
        self._cfg = cfg
        h = ctypes.c_void_p()
        rc = lib().sg_create(ctypes.byref(cfg), ctypes.byref(h))
        self._h = h
        if rc:
            msg = lib().sg_last_error(h).decode() if h else ""
            if h:
                lib().sg_destroy(h)
            self._h = None
            raise SgError(rc, "sg_create: " + msg)

    def close(self):
        if getattr(self, "_h", None):
            lib().sg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, where):
        if rc:
            raise SgError(rc, "%s: %s" % (where, lib().sg_last_error(self._h).decode()))

    # ---- allocation helpers (host numpy or device torch)
    def _lag(self, n=1):
        if self.mem == "host":
            return [np.zeros(self.npts, self.rdtype) for _ in range(n)]
        import torch
        dt = torch.float64 if self.rdtype == np.float64 else torch.float32
        return [torch.zeros(self.npts, dtype=dt, device="cuda") for _ in range(n)]

    def _eul(self, n=1):
        if self.mem == "host":
            return [np.zeros(self.field_shape, self.rdtype) for _ in range(n)]
        import torch
        dt = torch.float64 if self.rdtype == np.float64 else torch.float32
        return [torch.empty(self.field_shape, dtype=dt, device="cuda") for _ in range(n)]

    # ---- the reference's subroutines
    def eulr2lagr(self, u, v, w, X, Y, Z, out=None):
        """interp_spread.f90:12 -- velocity at the force points."""
        U, V, W = out if out is not None else self._lag(3)
        self._check(lib().sg_interp(self._h, *map(_ptr, (u, v, w, X, Y, Z, U, V, W))), "sg_interp")
        return U, V, W

    def complagrforces(self, X, Y, Z, out=None):
        """forcing.f90:11 -- membrane force, unit normals and area."""
        o = out if out is not None else self._lag(7)
        self._check(lib().sg_membrane_force(self._h, *map(_ptr, (X, Y, Z, *o))), "sg_membrane_force")
        return (o[0], o[1], o[2]), (o[3], o[4], o[5]), o[6]

    def lagr2eulr(self, X, Y, Z, FX, FY, FZ, AREA, out=None):
        """interp_spread.f90:510 -- spread force * area onto the Eulerian grid."""
        fx, fy, fz = out if out is not None else self._eul(3)
        self._check(lib().sg_spread(self._h, *map(_ptr, (X, Y, Z, FX, FY, FZ, AREA, fx, fy, fz))), "sg_spread")
        return fx, fy, fz

    def step(self, u, v, w, X, Y, Z, lag_out=None, eul_out=None):
        """eulr2lagr + complagrforces + lagr2eulr with one binning of the points."""
        L = lag_out if lag_out is not None else self._lag(10)
        E = eul_out if eul_out is not None else self._eul(3)
        self._check(lib().sg_step(self._h, *map(_ptr, (u, v, w, X, Y, Z, *L, *E))), "sg_step")
        return dict(u=L[0:3], f=L[3:6], n=L[6:9], area=L[9], fgrid=E)

    def set_tile_shape(self, shape):
        """Spreading tile shape: index into TILE_SHAPES, or -1 for the default."""
        self._check(lib().sg_set_tile_shape(self._h, int(shape)), "sg_set_tile_shape")

    def set_point_split(self, split):
        """Work items per capsule of the persistent pointwise kernels (1..8)."""
        self._check(lib().sg_set_point_split(self._h, int(split)), "sg_set_point_split")

    def set_capsule_law(self, law):
        """Membrane law per capsule: 0 Skalak, 1 neo-Hookean (membmodel.c:60-99)."""
        law = np.ascontiguousarray(law, dtype=np.int32)
        assert law.size == self.degree.size
        self._check(lib().sg_set_capsule_law(self._h, law.ctypes.data_as(ctypes.c_void_p)), "sg_set_capsule_law")

    def set_fused_force(self, on=True):
        """Mixed path: the whole force stage in one kernel per capsule (FP32 contractions) or staged."""
        self._check(lib().sg_set_fused_force(self._h, int(bool(on))), "sg_set_fused_force")

    def fused_force(self):
        return bool(lib().sg_get_fused_force(self._h))

    def set_capsule_bending(self, eb):
        """Bending modulus per capsule (0 = the ibend = 0 force; sph.f90:1705-1709)."""
        eb = np.ascontiguousarray(np.broadcast_to(np.asarray(eb, dtype=np.float64), self.degree.shape))
        self._check(lib().sg_set_capsule_bending(self._h, eb.ctypes.data_as(ctypes.c_void_p)),
                    "sg_set_capsule_bending")

    def overlap_lid(self, nf, nr, u, v, w, p, indic, out=None):
        """interpolation.f90:10-69: ub, vb, wb, pb, indb on the (itot nr + 2) x (jtot nr + 2) lid nodes."""
        itot, jtot = self.grid[0], self.grid[1]
        shape = (jtot * nr + 2, itot * nr + 2)
        for a in (u, v, w, p, indic):
            assert str(a.dtype) in ("float64", "torch.float64"), "the lid takes FP64 fields"
        if out is None:
            if self.mem == "host":
                out = [np.zeros(shape) for _ in range(5)]
            else:
                import torch
                out = [torch.zeros(shape, dtype=torch.float64, device=u.device) for _ in range(5)]
        self._check(lib().sg_overlap_lid(self._h, int(nf), int(nr), *map(_ptr, (u, v, w, p, indic)),
                                         *map(_ptr, out)), "sg_overlap_lid")
        return out

    def set_legendre_tile_rows(self, rows):
        """Data rows per tensor-core Legendre tile: 128 or 64 (results do not depend on it)."""
        self._check(lib().sg_set_legendre_tile_rows(self._h, int(rows)), "sg_set_legendre_tile_rows")

    def legendre_tile_rows(self):
        return int(lib().sg_get_legendre_tile_rows(self._h))

    def set_legendre_terms(self, terms=0):
        """Split mode of the tensor-core Legendre products: 3 (BF16x3), 6 (BF16x6), 0 automatic by degree."""
        self._check(lib().sg_set_legendre_terms(self._h, int(terms)), "sg_set_legendre_terms")

    def legendre_terms(self, degree):
        """Split products (3 or 6) that capsules of this SH degree run with."""
        return int(lib().sg_get_legendre_terms(self._h, int(degree)))

    def set_tensor_cores(self, on=True):
        """Mixed path: Legendre contractions on the tensor cores (BF16x3) or on CUDA cores (FP32)."""
        self._check(lib().sg_set_tensor_cores(self._h, int(bool(on))), "sg_set_tensor_cores")

    def point_split(self):
        return lib().sg_get_point_split(self._h)

    def tile_shape(self):
        v = [ctypes.c_int() for _ in range(4)]
        self._check(lib().sg_get_tile_shape(self._h, *[ctypes.byref(x) for x in v]), "sg_get_tile_shape")
        return v[0].value, (v[1].value, v[2].value, v[3].value)

    def autotune(self, u, v, w, X, Y, Z, lag_out=None, eul_out=None, reps=3):
        """Time `reps` steps per valid tile shape and keep the fastest; returns (shape, ms per step)."""
        L = lag_out if lag_out is not None else self._lag(10)
        E = eul_out if eul_out is not None else self._eul(3)
        best, ms = ctypes.c_int(), ctypes.c_float()
        self._check(lib().sg_autotune(self._h, *map(_ptr, (u, v, w, X, Y, Z, *L, *E)), int(reps),
                                      ctypes.byref(best), ctypes.byref(ms)), "sg_autotune")
        return best.value, ms.value

    def graph_capture(self, u, v, w, X, Y, Z, lag_out, eul_out):
        """Capture one step on fixed device arrays into a CUDA graph."""
        self._check(lib().sg_graph_capture(self._h, *map(_ptr, (u, v, w, X, Y, Z, *lag_out, *eul_out))),
                    "sg_graph_capture")

    def graph_launch(self):
        self._check(lib().sg_graph_launch(self._h), "sg_graph_launch")

    def graph_release(self):
        self._check(lib().sg_graph_release(self._h), "sg_graph_release")

    # ---------------------------------------------------------- surrogate
    def set_capsule_membrane(self, gs=None, csk=None):
        """Per-capsule Skalak Gs and C (None keeps the current values)."""
        n = self.degree.size
        g = None if gs is None else np.ascontiguousarray(np.broadcast_to(gs, n), dtype=np.float64)
        c = None if csk is None else np.ascontiguousarray(np.broadcast_to(csk, n), dtype=np.float64)
        self._check(lib().sg_set_capsule_membrane(self._h, _ptr(g), _ptr(c)), "sg_set_capsule_membrane")

    def capsule_spectra(self, X, Y, Z):
        """Plain-model displacement and filtered-force coefficients, [sum 3(L+1)^2] each (host mode)."""
        n = int(sum(3 * (int(L) + 1) ** 2 for L in self.degree))
        if self.mem == "host":
            d, f = np.zeros(n), np.zeros(n)
        else:
            import torch
            d = torch.zeros(n, dtype=torch.float64, device="cuda")
            f = torch.zeros(n, dtype=torch.float64, device="cuda")
        self._check(lib().sg_capsule_spectra(self._h, *map(_ptr, (X, Y, Z, d, f))), "sg_capsule_spectra")
        return d, f

    def surrogate_params(self, values=None):
        """Get (values=None) or set the surrogate's parameters as one float32 vector."""
        n = lib().sg_surrogate_param_count()
        if values is None:
            buf = np.zeros(n, np.float32)
            self._check(lib().sg_surrogate_params(self._h, 0, _ptr(buf), n), "sg_surrogate_params")
            return buf
        buf = np.ascontiguousarray(values, dtype=np.float32)
        self._check(lib().sg_surrogate_params(self._h, 1, _ptr(buf), buf.size), "sg_surrogate_params")
        return buf

    def surrogate_set_linear(self, L0, L1):
        a = np.ascontiguousarray(L0, dtype=np.float32)
        b = np.ascontiguousarray(L1, dtype=np.float32)
        self._check(lib().sg_surrogate_set_linear(self._h, _ptr(a), _ptr(b)), "sg_surrogate_set_linear")

    def surrogate_train(self, X, Y, epochs, batch=1024, lr=1e-3, seed=0):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        hist = np.zeros(epochs, np.float32)
        self._check(lib().sg_surrogate_train(self._h, _ptr(X), _ptr(Y), X.shape[0], int(epochs), int(batch),
                                             ctypes.c_float(lr), ctypes.c_ulonglong(seed), _ptr(hist)),
                    "sg_surrogate_train")
        return hist

    def surrogate_predict(self, X, parts=3):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.zeros_like(X)
        self._check(lib().sg_surrogate_predict(self._h, _ptr(X), X.shape[0], int(parts), _ptr(Y)),
                    "sg_surrogate_predict")
        return Y

    def surrogate_set_trust(self, amp_max, ratio_max, c_min=0.0, c_max=1e30):
        self._check(lib().sg_surrogate_set_trust(self._h, ctypes.c_float(amp_max), ctypes.c_float(ratio_max),
                                                 ctypes.c_float(c_min), ctypes.c_float(c_max)),
                    "sg_surrogate_set_trust")

    def surrogate_counts(self):
        a, b = ctypes.c_int(), ctypes.c_int()
        self._check(lib().sg_surrogate_last_counts(self._h, ctypes.byref(a), ctypes.byref(b)),
                    "sg_surrogate_last_counts")
        return a.value, b.value

    def update_pos(self, dt, X, Y, Z, U, V, W):
        """Update_Pos.f90:95-126 -- in place on X, Y, Z."""
        self._check(lib().sg_update_pos(self._h, ctypes.c_double(dt), *map(_ptr, (X, Y, Z, U, V, W))),
                    "sg_update_pos")

    def set_wall_collisions(self, in_step=True, col=5.68533e-2, betacol=15.36, rad0=None, rep=0.0016):
        """Constants of collisions.f90 (param.f90:57,64; rad0 defaults to 2.5 dz).
        in_step: sg_step applies the wall force between the membrane force and
        the spreading, as main.f90:229-233 does."""
        if rad0 is None:
            rad0 = 2.5 * self.grid[5]
        self._check(lib().sg_set_wall_collisions(self._h, int(bool(in_step)), float(col), float(betacol),
                                                 float(rad0), float(rep)), "sg_set_wall_collisions")

    def collisions(self, Z, AREA, FZ):
        """collisions.f90:10-32 -- FZ += wall force, in place."""
        self._check(lib().sg_collisions(self._h, *map(_ptr, (Z, AREA, FZ))), "sg_collisions")
        return FZ

    def set_indicator_params(self, visc0=1.0 / 0.0016, lam=1.0, thetainc=70.0 * np.pi / 180.0, ta=1160000.0,
                             rep=0.0016):
        """Constants of indicator.f90 (param.f90:52,57); allocates the indicator's workspace."""
        self._check(lib().sg_set_indicator_params(self._h, float(visc0), float(lam), float(thetainc), float(ta),
                                                  float(rep)), "sg_set_indicator_params")

    def indicator(self, X, Y, Z, NX, NY, NZ, AREA, fy=None, fz=None, out=None):
        """indicator.f90:19-182 -- (indic, visc); fy, fz (optional) get the centrifugal terms in place."""
        indic, visc = out if out is not None else self._eul(2)
        self._check(lib().sg_indicator(self._h, *map(_ptr, (X, Y, Z, NX, NY, NZ, AREA, indic, visc, fy, fz))),
                    "sg_indicator")
        return indic, visc

    def set_flow_params(self, rep=0.0016, vb2=0.0, vt2=0.0):
        """Rep and the wall values of v of the FFT flow solver (FP64 contexts)."""
        self._check(lib().sg_set_flow_params(self._h, float(rep), float(vb2), float(vt2)), "sg_set_flow_params")

    def flow_step(self, dt, uo, vo, wo, uoo, voo, woo, p, fx, fy, fz, out=None):
        """fsolver = 'f' (main.f90:333-347): returns (u, v, w) after one step; p is updated in place."""
        u, v, w = out if out is not None else self._eul(3)
        self._check(lib().sg_flow_step(self._h, ctypes.c_double(dt),
                                       *map(_ptr, (uo, vo, wo, uoo, voo, woo, p, fx, fy, fz, u, v, w))),
                    "sg_flow_step")
        return u, v, w

    def surf_vol(self, X, Y, Z, NX, NY, NZ, AREA, exy1_prev=None):
        """surf_vol.f90:12 -- [ncap, 7]: volume, area, exy1, exy2, centroid."""
        ncap = self.degree.size
        if self.mem == "host":
            out = np.zeros((ncap, 7))
        else:
            import torch
            out = torch.zeros((ncap, 7), dtype=torch.float64, device="cuda")
        self._check(lib().sg_surf_vol(self._h, *map(_ptr, (X, Y, Z, NX, NY, NZ, AREA, exy1_prev, out))),
                    "sg_surf_vol")
        return out

    def synchronize(self):
        self._check(lib().sg_synchronize(self._h), "sg_synchronize")

    def last_launch_count(self):
        return lib().sg_last_launch_count(self._h)

    def set_profiling(self, on=True):
        self._check(lib().sg_set_profiling(self._h, int(bool(on))), "sg_set_profiling")

    def contraction_work(self):
        """Flops of one step's Legendre contractions: algorithmic, issued on the
        tensor cores (0 on the CUDA-core path), and the number of launches."""
        out = (ctypes.c_double * 3)()
        self._check(lib().sg_contraction_work(self._h, out), "sg_contraction_work")
        return {"flops": out[0], "issued_flops": out[1], "launches": int(out[2])}

    def stage_times(self):
        """Milliseconds of the last step's stages (CUDA events on the context
        stream); "contract" is the Legendre contraction launches inside the
        membrane stage."""
        ms = (ctypes.c_float * len(STAGES))()
        self._check(lib().sg_stage_times(self._h, ms, len(STAGES)), "sg_stage_times")
        return dict(zip(STAGES, list(ms)))
