"""Frozen stencil weights of the reference, as 27-entry float32 tables indexed (dz, dy, dx).

These are the operator surface the reference fixes at layer construction time; each
function cites where the reference builds the same kernel.  A kernel ``K`` (3,3,3) applies
as ``y[z,y,x] = sum K[a,b,c] phi[z+a-1, y+b-1, x+c-1]`` with zero padding.
"""
import numpy as np

_OUTER = np.array([[2, 3, 2], [3, 6, 3], [2, 3, 2]], dtype=np.float64) / 26.0
_CENTRE = np.array([[3, 6, 3], [6, -88, 6], [3, 6, 3]], dtype=np.float64) / 26.0
_DX1 = np.array([[-0.014, 0.0, 0.014], [-0.056, 0.0, 0.056], [-0.014, 0.0, 0.014]])
_DX2 = np.array([[-0.056, 0.0, 0.056], [-0.22, 0.0, 0.22], [-0.056, 0.0, 0.056]])
_DY1 = np.array([[0.014, 0.056, 0.014], [0.0, 0.0, 0.0], [-0.014, -0.056, -0.014]])
_DY2 = np.array([[0.056, 0.22, 0.056], [0.0, 0.0, 0.0], [-0.056, -0.22, -0.056]])
_DZ1 = np.array([[0.014, 0.056, 0.014], [0.056, 0.22, 0.056], [0.014, 0.056, 0.014]])


def anisotropic7(Dx=200.0, Dy=100.0, Dz=50.0, dx=1.0, dy=1.0, dz=1.0, dt=1.0):
    """The 7-point operator ``w2`` of
    ``Anisotropic Resistivity Tomography/Anisotropic_3d_Multigrid_7point.ipynb:75-90``
    (``dt`` scaling as in ``notebooks/Multigrid_3d_7point_source.ipynb`` cell 3): centre
    ``2(Dx/dx^2 + Dy/dy^2 + Dz/dz^2)``, neighbours ``-D/d^2``."""
    kz, ky, kx = dt * Dz / dz ** 2, dt * Dy / dy ** 2, dt * Dx / dx ** 2
    K = np.zeros((3, 3, 3))
    K[1, 1, 1] = 2 * (kx + ky + kz)
    K[0, 1, 1] = K[2, 1, 1] = -kz
    K[1, 0, 1] = K[1, 2, 1] = -ky
    K[1, 1, 0] = K[1, 1, 2] = -kx
    return K.astype(np.float32)


def diffusion27(dt, Re, dx=1.0):
    """``w1`` of ``scripts/naiver_stokes_3D.py:36-49`` (27-point Laplacian x dt*Re/dx^2)."""
    return (np.stack([_OUTER, _CENTRE, _OUTER]) * (dt * Re / dx ** 2)).astype(np.float32)


def pressure27(dx=1.0):
    """``w5`` of ``scripts/naiver_stokes_3D.py:96-108``: ``-L27/dx^2``, diagonal 88/26."""
    return (-np.stack([_OUTER, _CENTRE, _OUTER]) / dx ** 2).astype(np.float32)


def advection(dt, dx=1.0, factor=1.0):
    """``w2, w3, w4`` of ``scripts/naiver_stokes_3D.py:51-94`` (smoothed central x/y/z
    differences x dt/dx; ``factor`` 0.5 for ``Urban Modelling/AI_HFM_v3.ipynb`` cell 8).
    The y and z kernels put ``+`` on the low-index side, as the reference does."""
    s = dt / dx * factor
    kx = np.stack([_DX1, _DX2, _DX1]) * s
    ky = np.stack([_DY1, _DY2, _DY1]) * s
    kz = np.stack([_DZ1, np.zeros((3, 3)), -_DZ1]) * s
    return kx.astype(np.float32), ky.astype(np.float32), kz.astype(np.float32)


def divergence(dt, dx=1.0, factor=1.0):
    """``w6, w7, w8`` of ``scripts/naiver_stokes_3D.py:110-152``: the same kernels divided
    by ``dx*dt`` (``factor`` 0.5 for ``AI_HFM_v3.ipynb`` cell 10)."""
    kx, ky, kz = advection(1.0, 1.0, 1.0)
    s = factor / (dx * dt)
    return (kx * s).astype(np.float32), (ky * s).astype(np.float32), (kz * s).astype(np.float32)


def advection_diffusion_2d(dt=10.0, dx=1.0, dy=1.0, Dx=0.1, Dy=0.1, ub=1.0):
    """3x3 implicit advection-diffusion operator of ``Unstructured Mesh/Multigrid_2D.ipynb``
    cell 3 (``w2[0][a][b][0]`` as ``[a, b]``), for the 2D reference cycle."""
    cx, cy, cu = Dx * dt / dx ** 2, Dy * dt / dy ** 2, ub * dt / dx
    return np.array([[0.0, -cy, 0.0],
                     [-cx - cu, 1.0 + 2.0 * (cx + cy) + 2.0 * cu, -cx],
                     [0.0, -cy - cu, 0.0]])
