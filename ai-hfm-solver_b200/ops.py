"""Stateless operators on CUDA tensors, mirroring the reference's frozen Keras layers.

The reference builds one ``keras.models.Sequential`` per stencil and grid size
(``CNN3D_A_<n>``, ``CNN3D_res_<n>``, ``CNN3D_prol_<n>``, ``CNN3D_central_2nd_*``,
``CNN3D_{Su,Sv,Sw,pu,pv,pw}``) and calls it on ``(1, Z, Y, X, 1)`` float32 tensors.  Here
one object per stencil serves every size (Keras does not enforce ``InputLayer`` shapes in
eager calls either, ``Anisotropic_3d_Multigrid_7point_BC_Rec.ipynb`` cell 8), and inputs may
be ``(1, Z, Y, X, 1)``, ``(Z, Y, X)`` or a batch ``(B, Z, Y, X)``.  Every call launches an
sm_100a kernel from ``libhfm.so`` on the current torch stream; tensors are only the I/O
container.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib as L


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _grid(x):
    """Return (B, Z, Y, X) for a reference-shaped or batched tensor."""
    s = tuple(x.shape)
    if len(s) == 5:
        if s[-1] != 1:
            raise ValueError("expected a single channel (..., 1)")
        return s[0], s[1], s[2], s[3]
    if len(s) == 4:
        return s
    if len(s) == 3:
        return (1,) + s
    raise ValueError("expected (1,Z,Y,X,1), (B,Z,Y,X) or (Z,Y,X), got %s" % (s,))


def _check_field(x, name="x"):
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise TypeError("%s must be a CUDA tensor" % name)
    if x.dtype != torch.float32:
        raise TypeError("%s must be float32" % name)
    if not x.is_contiguous():
        raise ValueError("%s must be contiguous" % name)


def _ptr(x):
    return C.c_void_p(x.data_ptr()) if x is not None else C.c_void_p(0)


def _w27(K):
    a = np.ascontiguousarray(np.asarray(K, dtype=np.float32).reshape(27))
    return a, a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------------------- operators
class Operator:
    """A discretised operator A as passed to the library (``hfm_operator``)."""

    kind = None

    def struct(self):
        raise NotImplementedError

    def _keep(self):
        return ()


class Const7(Operator):
    """Constant-coefficient anisotropic 7-point operator (``w2`` of
    ``Anisotropic_3d_Multigrid_7point.ipynb:75-90``) with kz = Dz/dz^2, ky = Dy/dy^2,
    kx = Dx/dx^2."""
    kind = L.OP_CONST7

    def __init__(self, kz, ky, kx, scale=1.0):
        self.k = (float(kz), float(ky), float(kx))
        self.scale = float(scale)

    @property
    def diag(self):
        return 2.0 * sum(self.k) * self.scale

    def struct(self):
        s = L.HfmOperator()
        s.kind, s.coef_dtype, s.scale = self.kind, L.F32, self.scale
        for i, v in enumerate(self.k):
            s.k[i] = v
        return s


class Stencil27(Operator):
    """An arbitrary frozen 3x3x3 kernel used as a matrix (``CNN3D_A_<n>`` with ``w5``,
    ``naiver_stokes_3D.py:239-307``); Jacobi diagonal = centre weight."""
    kind = L.OP_K27

    def __init__(self, K, scale=1.0):
        self.K = np.asarray(K, dtype=np.float32).reshape(3, 3, 3)
        self.scale = float(scale)

    @property
    def diag(self):
        return float(self.K[1, 1, 1]) * self.scale

    def struct(self):
        s = L.HfmOperator()
        s.kind, s.coef_dtype, s.scale = self.kind, L.F32, self.scale
        for i, v in enumerate(self.K.reshape(27)):
            s.k[i] = float(v)
        return s


class Sigma7(Operator):
    """Variable-coefficient 7-point operator from per-cell conductivities (sx, sy, sz)
    (``BGS_multigrid_v1.ipynb`` cell 40 operator form, README face means
    ``Anisotropic Resistivity Tomography/README:14-26``).  ``c = (cz, cy, cx)`` = 1/h^2."""
    kind = L.OP_SIGMA7

    def __init__(self, sx, sy, sz, c=(1.0, 1.0, 1.0), scale=1.0):
        for name, a in (("sx", sx), ("sy", sy), ("sz", sz)):
            _check_field(a, name)
        self.s = (sx, sy, sz)
        self.c = tuple(float(v) for v in c)
        self.scale = float(scale)

    def struct(self):
        s = L.HfmOperator()
        s.kind, s.coef_dtype, s.scale = self.kind, L.F32, self.scale
        for i, v in enumerate(self.c):
            s.c[i] = v
        for i, a in enumerate(self.s):
            s.coef[i] = a.data_ptr()
        return s


class Dir7(Operator):
    """The reference's six directional coefficient arrays ``A_MAT_{xm1,xp1,ym1,yp1,zm1,zp1}``
    and ``A_MAT_TOT`` (``BGS_multigrid_v1.ipynb`` cells 38 and 40)."""
    kind = L.OP_DIR7
    ORDER = ("xm", "xp", "ym", "yp", "zm", "zp", "tot")

    def __init__(self, coeffs, scale=1.0):
        self.A = [coeffs[k] for k in self.ORDER]
        for k, a in zip(self.ORDER, self.A):
            _check_field(a, k)
        self.scale = float(scale)

    def struct(self):
        s = L.HfmOperator()
        s.kind, s.coef_dtype, s.scale = self.kind, L.F32, self.scale
        for i, a in enumerate(self.A):
            s.coef[i] = a.data_ptr()
        return s


def bgs_mesh(shape, ax=0.02, ay=0.4, az=0.02):
    """Non-uniform cell sizes of ``BGS_multigrid_v1.ipynb`` cell 34 on a (Z, Y, X) grid:
    dx = 1 + ax k and dy = 1 + ay k with k the distance in cells from the centre plane (the
    same on both halves), dz = 1 + az z.  Returns (mesh_x, mesh_y, mesh_z) float64 arrays of
    the grid's shape."""
    Z, Y, X = shape

    def sym(n, a):
        i = np.arange(n)
        return 1.0 + a * np.where(i >= n // 2, i - n // 2, n // 2 - 1 - i)

    mx = np.broadcast_to(sym(X, ax)[None, None, :], shape).copy()
    my = np.broadcast_to(sym(Y, ay)[None, :, None], shape).copy()
    mz = np.broadcast_to((1.0 + az * np.arange(Z))[:, None, None], shape).copy()
    return mx, my, mz


def bgs_mesh_p1(mesh, axis):
    """The shifted sizes of ``BGS_multigrid_v1.ipynb`` cell 36: interior cells take the size
    of the next cell along ``axis`` (axis 0 = z, 1 = y, 2 = x); the two boundary cells keep
    their own."""
    out = np.array(mesh, copy=True)
    sl = lambda a, b: tuple(slice(a, b) if d == axis else slice(None) for d in range(3))
    out[sl(1, -1)] = mesh[sl(2, None)]
    return out


def dir7_from_mesh(D, mesh_x, mesh_y, mesh_z, device="cuda"):
    """``Dir7`` coefficients of ``BGS_multigrid_v1.ipynb`` cell 38: A_{x-} = D / mesh_x^2,
    A_{x+} = D / mesh_x_p1^2 (likewise y, z), A_TOT their sum in the cell's order; computed in
    float64 on the host as the reference does with NumPy, stored float32 on the device.
    ``D`` is a scalar or an array of the grid's shape."""
    p1 = [bgs_mesh_p1(m, ax) for m, ax in ((mesh_x, 2), (mesh_y, 1), (mesh_z, 0))]
    D = np.asarray(D, np.float64)
    a = {"xm": D / mesh_x ** 2, "ym": D / mesh_y ** 2, "zm": D / mesh_z ** 2,
         "xp": D / p1[0] ** 2, "yp": D / p1[1] ** 2, "zp": D / p1[2] ** 2}
    a["tot"] = a["xm"] + a["ym"] + a["zm"] + a["xp"] + a["yp"] + a["zp"]
    shape = np.broadcast_shapes(np.shape(mesh_x), np.shape(D))
    return Dir7({k: torch.from_numpy(np.ascontiguousarray(np.broadcast_to(v, shape), np.float32)).to(device)
                 for k, v in a.items()})


# ---------------------------------------------------------------------------- functions
def conv3d_same(x, K, out=None):
    """``Conv3D(1, kernel_size=3, strides=1, padding='SAME')`` with frozen kernel ``K``."""
    _check_field(x)
    B, Z, Y, X = _grid(x)
    out = torch.empty_like(x) if out is None else out
    keep, wp = _w27(K)
    L.call("hfm_conv3d_k3", _ptr(x), _ptr(out), B, Z, Y, X, wp, _stream())
    return out


def restrict_avg(x):
    """``CNN3D_res_<n>``: 2x2x2 average, stride 2, VALID (odd trailing cells dropped)."""
    _check_field(x)
    B, Z, Y, X = _grid(x)
    shp = list(x.shape)
    if len(shp) == 5:
        shp[1:4] = [Z // 2, Y // 2, X // 2]
    else:
        shp[-3:] = [Z // 2, Y // 2, X // 2]
    out = torch.empty(shp, dtype=x.dtype, device=x.device)
    L.call("hfm_restrict_avg", _ptr(x), _ptr(out), B, Z, Y, X, _stream())
    return out


def prolong_nearest(x):
    """``CNN3D_prol_<n>``: ``UpSampling3D(size=(2, 2, 2))``."""
    _check_field(x)
    B, Z, Y, X = _grid(x)
    shp = list(x.shape)
    if len(shp) == 5:
        shp[1:4] = [2 * Z, 2 * Y, 2 * X]
    else:
        shp[-3:] = [2 * Z, 2 * Y, 2 * X]
    out = torch.empty(shp, dtype=x.dtype, device=x.device)
    L.call("hfm_prolong_nearest", _ptr(x), _ptr(out), B, Z, Y, X, _stream())
    return out


def apply(op, phi, out=None):
    """``A phi`` (``CNN3D_A_<n>(phi)``, ``A_operator_<n>(phi)``)."""
    _check_field(phi, "phi")
    B, Z, Y, X = _grid(phi)
    out = torch.empty_like(phi) if out is None else out
    s = op.struct()
    L.call("hfm_op_apply", C.byref(s), _ptr(phi), _ptr(out), B, Z, Y, X, _stream())
    return out


def residual(op, phi, b, flags=0, out=None):
    """``r = A phi - b`` (``Anisotropic_3d_Multigrid_7point.ipynb:409``)."""
    _check_field(phi, "phi")
    _check_field(b, "b")
    B, Z, Y, X = _grid(phi)
    out = torch.empty_like(phi) if out is None else out
    s = op.struct()
    L.call("hfm_op_residual", C.byref(s), _ptr(phi), _ptr(b), _ptr(out), B, Z, Y, X,
           flags, _stream())
    return out


def jacobi(op, phi, rhs, omega=1.0, sweeps=1, flags=0):
    """``sweeps`` weighted-Jacobi sweeps; omega = 1 is the reference's
    ``w - A(w)/d + r/d`` (``Anisotropic_3d_Multigrid_7point.ipynb:424``)."""
    _check_field(rhs, "rhs")
    if phi is not None:
        _check_field(phi, "phi")
    else:
        flags |= L.FLAG_ZERO_GUESS
    B, Z, Y, X = _grid(rhs)
    out = torch.empty_like(rhs)
    tmp = torch.empty_like(rhs) if sweeps > 1 else None
    s = op.struct()
    L.call("hfm_op_jacobi", C.byref(s), _ptr(phi), _ptr(rhs), _ptr(out), _ptr(tmp), B, Z, Y, X,
           float(omega), int(sweeps), flags, _stream())
    return out


def residual_restrict(op, phi, b, flags=0, want_fine=False):
    """Fused ``R (A phi - b)``; also returns the fine residual when ``want_fine``."""
    _check_field(phi, "phi")
    _check_field(b, "b")
    B, Z, Y, X = _grid(phi)
    rc = torch.empty((B, Z // 2, Y // 2, X // 2), dtype=phi.dtype, device=phi.device)
    rf = torch.empty_like(phi) if want_fine else None
    s = op.struct()
    L.call("hfm_residual_restrict", C.byref(s), _ptr(phi), _ptr(b), _ptr(rf), _ptr(rc),
           B, Z, Y, X, flags, _stream())
    return (rc, rf) if want_fine else rc


def prolong_correct_smooth(op, phi, w_coarse, rhs, omega=1.0, flags=0):
    """Fused ``J(phi - P w)`` against ``rhs``; ``phi=None`` gives ``J(P w)``."""
    _check_field(rhs, "rhs")
    B, Z, Y, X = _grid(rhs)
    out = torch.empty_like(rhs)
    s = op.struct()
    L.call("hfm_prolong_correct_smooth", C.byref(s), _ptr(phi), _ptr(w_coarse), _ptr(rhs),
           _ptr(out), B, Z, Y, X, float(omega), flags, _stream())
    return out


def norm2(x, batch=None):
    """Per-instance ``||x||_2`` accumulated in float64 (deterministic order)."""
    _check_field(x)
    B = x.shape[0] if batch is None else batch
    n = x.numel() // B
    out = torch.empty(B, dtype=torch.float64, device=x.device)
    scratch = torch.empty(max(1, L.lib().hfm_reduce_scratch_bytes(n, B)), dtype=torch.uint8,
                          device=x.device)
    L.call("hfm_norm2_f64", _ptr(x), n, B, _ptr(out), _ptr(scratch), _stream())
    return out


def max_abs(x, batch=None):
    """Per-instance ``max |x|`` (the reference's ``np.max`` diagnostics)."""
    _check_field(x)
    B = x.shape[0] if batch is None else batch
    n = x.numel() // B
    out = torch.empty(B, dtype=torch.float32, device=x.device)
    scratch = torch.empty(max(1, L.lib().hfm_reduce_scratch_bytes(n, B)), dtype=torch.uint8,
                          device=x.device)
    L.call("hfm_max_abs", _ptr(x), n, B, _ptr(out), _ptr(scratch), _stream())
    return out


# ------------------------------------------------------------- Keras-style layer objects
class Conv3DSame:
    """Callable with the reference's layer semantics: ``Conv3DSame(w)(x)``."""

    def __init__(self, K):
        self.K = np.asarray(K, dtype=np.float32).reshape(3, 3, 3)

    def __call__(self, x):
        return conv3d_same(x, self.K)

    def count_params(self):
        return 28  # 27 weights + 1 bias, as Keras reports (7point_BC_Rec.ipynb:196)


class Restriction:
    def __call__(self, x):
        return restrict_avg(x)

    def count_params(self):
        return 9  # 8 weights + 1 bias (7point_BC_Rec.ipynb:279)


class Prolongation:
    def __call__(self, x):
        return prolong_nearest(x)
