"""TensorFlow 2.0 layer semantics used by the reference, restated in NumPy.

All functions accept arrays shaped ``(..., Z, Y, X)``: the reference tensors are
``(1, Z, Y, X, 1)`` (batch and channel of size one), and the oracle drops those two axes.
Memory order is ``[z][y][x]`` with X fastest, as in the reference
(``Anisotropic Resistivity Tomography/Anisotropic_3d_Multigrid_7point_BC_Rec.ipynb`` builds
``(1, nz, ny, nx, 1)`` with the z conductivity on axis 1).
"""
import numpy as np


def conv3d_same(x, K, dtype=np.float32):
    """``tf.keras.layers.Conv3D(1, kernel_size=3, strides=1, padding='SAME')`` with frozen
    kernel ``K`` and zero bias.

    TF convolutions are cross-correlations: ``y[z,y,x] = sum K[a,b,c] * x[z+a-1, y+b-1,
    x+c-1]`` with out-of-range samples equal to zero (SAME padding of one cell on each side
    for k=3, s=1).  ``K`` is indexed ``(dz, dy, dx)``; the reference builds it as
    ``w[0, a, b, c, 0]`` and ``tf.keras.initializers.constant`` reshapes ``(1,3,3,3,1)`` to
    the layer's ``(3,3,3,1,1)`` row-major (printed kernel:
    ``Anisotropic Resistivity Tomography/notebooks/Multigrid_3d_7point_source.ipynb`` cell 10
    output).  Call sites: ``Anisotropic_3d_Multigrid_7point.ipynb`` cell 7 (lines 124-183),
    ``scripts/naiver_stokes_3D.py:166-307``.
    """
    x = np.asarray(x, dtype=dtype)
    K = np.asarray(K, dtype=dtype).reshape(3, 3, 3)
    Z, Y, X = x.shape[-3:]
    pad = [(0, 0)] * (x.ndim - 3) + [(1, 1)] * 3
    xp = np.pad(x, pad)
    out = np.zeros_like(x)
    for a in range(3):
        for b in range(3):
            for c in range(3):
                k = K[a, b, c]
                if k != 0:
                    out += k * xp[..., a:a + Z, b:b + Y, c:c + X]
    return out


def restrict_avg(x, dtype=np.float32):
    """``Conv3D(1, kernel_size=2, strides=2, padding='VALID')`` with all weights 0.125
    (``Anisotropic_3d_Multigrid_7point.ipynb:78`` and cell 9, lines 194-240).

    ``out[i,j,k] = sum_{a,b,c in {0,1}} 0.125 * x[2i+a, 2j+b, 2k+c]``; VALID padding floors
    odd extents, so a trailing odd plane, row or column is dropped.
    """
    x = np.asarray(x, dtype=dtype)
    Z, Y, X = x.shape[-3:]
    Zc, Yc, Xc = Z // 2, Y // 2, X // 2
    w = dtype(0.125)
    out = np.zeros(x.shape[:-3] + (Zc, Yc, Xc), dtype=dtype)
    for a in range(2):
        for b in range(2):
            for c in range(2):
                out += w * x[..., a:2 * Zc:2, b:2 * Yc:2, c:2 * Xc:2]
    return out


def prolong_nearest(x, dtype=np.float32):
    """``tf.keras.layers.UpSampling3D(size=(2, 2, 2))``
    (``Anisotropic_3d_Multigrid_7point.ipynb`` cell 11, lines 251-289): every coarse value is
    repeated into its 2x2x2 block, ``out[2i+a, 2j+b, 2k+c] = x[i, j, k]``."""
    x = np.asarray(x, dtype=dtype)
    for ax in (-3, -2, -1):
        x = np.repeat(x, 2, axis=ax)
    return x
