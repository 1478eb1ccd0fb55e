"""Generate the golden fixtures in this directory.

Run from the repository root: ``python tests/golden/make_golden.py``.

Two kinds of fixture are written:

* ``reference_pins.json`` - numbers the reference itself printed, typed in from its saved
  notebook outputs (``Anisotropic Resistivity Tomography/notebooks/
  Multigrid_3d_7point_source.ipynb`` cells 4, 5, 6 and 10: the 7-point kernel at
  dt=0.1, Dx=200, Dy=100, Dz=50, dx=1; ``Anisotropic_3d_Multigrid_7point_BC_Rec.ipynb``
  lines 196 and 279: parameter counts).  These pin the oracle's kernel layout.
* ``oracle_small.npz`` - seeded small-grid inputs and the oracle's outputs for every
  operator and for a few reference cycles.  TensorFlow 2.0 (the reference's pinned
  dependency) is not installable here, so these are the oracle's values, cross-checked at
  generation time against an independent ``torch.nn.functional.conv3d`` evaluation of the
  same layers; the GPU parity tests compare the CUDA library against them.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import mg, tfops, weights as W  # noqa: E402


def torch_conv_same(x, K):
    import torch
    t = torch.from_numpy(np.asarray(x, np.float64))[None, None]
    k = torch.from_numpy(np.asarray(K, np.float64).reshape(1, 1, 3, 3, 3))
    return torch.nn.functional.conv3d(t, k, padding=1)[0, 0].numpy()


def main():
    pins = {
        "source": "notebooks/Multigrid_3d_7point_source.ipynb cells 4-6, 10 (dt=0.1, Dx=200, Dy=100, Dz=50, dx=1)",
        "sum_w2": 0.0,
        "centre_plane": [[-0.0, -10.0, -0.0], [-20.0, 70.0, -20.0], [-0.0, -10.0, -0.0]],
        "centre_weight": 70.0,
        "kernel_3x3x3": [
            [[-0.0, -0.0, -0.0], [-0.0, -5.0, -0.0], [-0.0, -0.0, -0.0]],
            [[-0.0, -10.0, -0.0], [-20.0, 70.0, -20.0], [-0.0, -10.0, -0.0]],
            [[-0.0, -0.0, -0.0], [-0.0, -5.0, -0.0], [-0.0, -0.0, -0.0]],
        ],
        "params_conv3x3x3": 28,
        "params_restrict2x2x2": 9,
    }
    with open(os.path.join(HERE, "reference_pins.json"), "w") as f:
        json.dump(pins, f, indent=1)

    rng = np.random.default_rng(20240601)
    out = {}
    shapes = [(1, 1, 1), (2, 2, 2), (3, 5, 4), (4, 4, 4), (5, 7, 6), (8, 6, 10)]
    K7 = W.w2_7point()
    K27 = W.w5_pressure27()
    Kr = rng.standard_normal((3, 3, 3))
    for i, s in enumerate(shapes):
        x = rng.standard_normal(s).astype(np.float32)
        b = rng.standard_normal(s).astype(np.float32)
        sig = np.exp(rng.standard_normal((3,) + s)).astype(np.float32)
        out["x_%d" % i] = x
        out["b_%d" % i] = b
        out["sig_%d" % i] = sig
        for name, K in (("k7", K7), ("k27", K27), ("kr", Kr)):
            y = tfops.conv3d_same(x, K, np.float64)
            ref = torch_conv_same(x, K)
            assert np.allclose(y, ref, rtol=1e-12, atol=1e-12), "conv semantics disagree"
            out["conv_%s_%d" % (name, i)] = tfops.conv3d_same(x, K, np.float32)
        op = mg.Sigma7(sig[0], sig[1], sig[2], dtype=np.float32)
        out["sigma_apply_%d" % i] = op.apply(x)
        out["sigma_jacobi_%d" % i] = mg.jacobi(op, x, b, 2.0 / 3.0)
        out["k7_jacobi_ref_%d" % i] = mg.jacobi_ref(mg.Stencil27(K7), x, b)
        if min(s) >= 2:
            out["restrict_%d" % i] = tfops.restrict_avg(x)
        out["prolong_%d" % i] = tfops.prolong_nearest(x)
    out["kr"] = Kr.astype(np.float32)

    # reference sawtooth cycles on 16^3 (7-point, box source = initial guess, 5 levels)
    n = 16
    b = np.zeros((n, n, n), np.float32)
    b[5:10, 5:10, 5:10] = 1.0
    ops = mg.hierarchy(mg.Stencil27(K7), 5)
    phi = b.copy()
    for c in range(3):
        phi = mg.sawtooth_cycle(ops, phi, b)
        out["saw7_after_%d" % (c + 1)] = phi
    out["saw7_b"] = b
    # NS pressure form (27-point w5, no fine Jacobi, r/p zero at x end) on 16^3, 4 levels
    pb = rng.standard_normal((n, n, n)).astype(np.float32)
    ops27 = mg.hierarchy(mg.Stencil27(K27), 4)
    p = np.zeros_like(pb)
    for c in range(2):
        p = mg.sawtooth_cycle(ops27, p, pb, fine_smooth=False, zero_xend=True)
        out["sawns_after_%d" % (c + 1)] = p
    out["sawns_b"] = pb
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
