"""The reference's frozen Conv3D kernels, built exactly as the reference builds them.

Every kernel is returned as a ``(3, 3, 3)`` float64 array indexed ``(dz, dy, dx)``; the
reference stores it as ``w[0, a, b, c, 0]`` of a ``(1, 3, 3, 3, 1)`` array.
"""
import numpy as np


def w2_7point(Dx=200.0, Dy=100.0, Dz=50.0, dx=1.0, dy=1.0, dz=1.0, dt=1.0):
    """Constant-coefficient anisotropic 7-point operator ``A`` (the ``w2`` of
    ``Anisotropic Resistivity Tomography/Anisotropic_3d_Multigrid_7point.ipynb:75-90``).

    ``w2 = -[pd1, pd2, pd3]`` with ``pd1 = pd3`` holding ``Dz/dz**2`` at the centre and
    ``pd2`` the in-plane 5-point star ``Dy/dy**2`` (rows), ``Dx/dx**2`` (columns) and
    ``-(2Dx/dx**2 + 2Dy/dy**2 + 2Dz/dz**2)`` at the centre.  ``dt`` multiplies every entry,
    as in ``notebooks/Multigrid_3d_7point_source.ipynb`` cell 3.
    """
    w = np.zeros((3, 3, 3))
    cz, cy, cx = dt * Dz / dz ** 2, dt * Dy / dy ** 2, dt * Dx / dx ** 2
    pd1 = np.array([[0, 0, 0], [0, cz, 0], [0, 0, 0]], dtype=np.float64)
    pd2 = np.array([[0, cy, 0], [cx, -(2 * cx + 2 * cy + 2 * cz), cx], [0, cy, 0]],
                   dtype=np.float64)
    w[0] = -pd1
    w[1] = -pd2
    w[2] = -pd1
    return w


_LAP27_OUTER = np.array([[2, 3, 2], [3, 6, 3], [2, 3, 2]], dtype=np.float64) / 26.0
_LAP27_CENTRE = np.array([[3, 6, 3], [6, -88, 6], [3, 6, 3]], dtype=np.float64) / 26.0


def w1_diffusion27(dt, Re, dx=1.0):
    """27-point diffusion increment ``w1`` (``scripts/naiver_stokes_3D.py:36-49``;
    ``Urban Modelling/AI_HFM_v3.ipynb`` cell 7): planes z+-1 = [[2,3,2],[3,6,3],[2,3,2]]/26,
    centre plane [[3,6,3],[6,-88,6],[3,6,3]]/26, all times ``dt*Re/dx**2``."""
    s = dt * Re / dx ** 2
    return np.stack([_LAP27_OUTER, _LAP27_CENTRE, _LAP27_OUTER]) * s


def w5_pressure27(dx=1.0):
    """27-point pressure operator ``w5 = -L27/dx**2`` (``scripts/naiver_stokes_3D.py:96-108``),
    diagonal ``w5[1,1,1] = 88/26``."""
    return -np.stack([_LAP27_OUTER, _LAP27_CENTRE, _LAP27_OUTER]) / dx ** 2


_X1 = np.array([[-0.014, 0.0, 0.014], [-0.056, 0.0, 0.056], [-0.014, 0.0, 0.014]])
_X2 = np.array([[-0.056, 0.0, 0.056], [-0.22, 0.0, 0.22], [-0.056, 0.0, 0.056]])
_Y1 = np.array([[0.014, 0.056, 0.014], [0.0, 0.0, 0.0], [-0.014, -0.056, -0.014]])
_Y2 = np.array([[0.056, 0.22, 0.056], [0.0, 0.0, 0.0], [-0.056, -0.22, -0.056]])
_Z1 = np.array([[0.014, 0.056, 0.014], [0.056, 0.22, 0.056], [0.014, 0.056, 0.014]])


def central_x():
    """Unscaled smoothed central x-derivative kernel (``p_div_x1..3``,
    ``scripts/naiver_stokes_3D.py:51-59``)."""
    return np.stack([_X1, _X2, _X1])


def central_y():
    """Unscaled y kernel (``p_div_y1..3``, ``naiver_stokes_3D.py:61-69``).  The ``+`` entries
    sit on the low-y side, so it evaluates ``-d/dy`` relative to ``central_x``; kept
    literally."""
    return np.stack([_Y1, _Y2, _Y1])


def central_z():
    """Unscaled z kernel (``p_div_z1..3``, ``naiver_stokes_3D.py:71-79``): ``+`` plane at
    z-1, zero centre plane, ``-`` plane at z+1."""
    return np.stack([_Z1, np.zeros((3, 3)), -_Z1])


def advection_kernels(dt, dx=1.0, factor=1.0):
    """``w2, w3, w4`` = central x/y/z kernels times ``dt/dx`` (times 0.5 in
    ``AI_HFM_v3.ipynb`` cell 8): used for ``CNN3D_central_2nd_{x,y,z}adv`` and
    ``CNN3D_{pu,pv,pw}`` (``naiver_stokes_3D.py:81-94``)."""
    s = dt / dx * factor
    return central_x() * s, central_y() * s, central_z() * s


def divergence_kernels(dt, dx=1.0, factor=1.0):
    """``w6, w7, w8`` = the same kernels divided by ``dx*dt`` (``naiver_stokes_3D.py:110-152``;
    times 0.5 in ``AI_HFM_v3.ipynb`` cell 10) for ``CNN3D_Su/Sv/Sw``."""
    s = factor / (dx * dt)
    return central_x() * s, central_y() * s, central_z() * s


def directional_kernels():
    """The six one-sided difference kernels of
    ``Anisotropic Resistivity Tomography/BGS_multigrid_v1.ipynb`` cell 11.  Each computes
    ``phi_c - phi_nb`` for one neighbour; returned in the order xm, xp, ym, yp, zm, zp."""
    ks = []
    for axis, off in ((2, -1), (2, 1), (1, -1), (1, 1), (0, -1), (0, 1)):
        k = np.zeros((3, 3, 3))
        k[1, 1, 1] = 1.0
        idx = [1, 1, 1]
        idx[axis] += off
        k[tuple(idx)] = -1.0
        ks.append(k)
    return ks


def w2_2d_advection_diffusion(dt=10.0, dx=1.0, dy=1.0, Dx=0.1, Dy=0.1, ub=1.0):
    """The 3x3 operator of ``Unstructured Mesh/Multigrid_2D.ipynb`` cell 3 (implicit
    advection-diffusion, upwind in both directions), as ``w2[0][a][b][0]`` -> ``[a, b]``:
    north / south ``-Dy dt/dy^2`` (south also ``-ub dt/dx``), west ``-Dx dt/dx^2 - ub dt/dx``,
    east ``-Dx dt/dx^2``, centre ``1 + 2(Dx dt/dx^2 + Dy dt/dy^2) + 2 ub dt/dx``."""
    w = np.zeros((3, 3))
    w[0, 1] = -Dy * dt / dy ** 2
    w[1, 0] = -Dx * dt / dx ** 2 - ub * dt / dx
    w[1, 1] = 1 + 2 * (Dx * dt / dx ** 2 + Dy * dt / dy ** 2) + 2 * ub * dt / dx
    w[1, 2] = -Dx * dt / dx ** 2
    w[2, 1] = -Dy * dt / dy ** 2 - ub * dt / dx
    return w
