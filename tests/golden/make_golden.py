"""Generate the golden fixtures in this directory.

Run from the repository root with the reference checkout named by ``HFM_REFERENCE_ROOT``:
``HFM_REFERENCE_ROOT=<checkout> python tests/golden/make_golden.py``.

Two kinds of fixture are written:

* ``reference_pins.json`` - numbers the reference itself printed in its saved notebook
  outputs.  Typed in: ``Anisotropic Resistivity Tomography/notebooks/
  Multigrid_3d_7point_source.ipynb`` cells 4, 5, 6 and 10 (the 7-point kernel at dt=0.1,
  Dx=200, Dy=100, Dz=50, dx=1) and ``Anisotropic_3d_Multigrid_7point_BC_Rec.ipynb`` lines 196
  and 279 (parameter counts): these pin the oracle's kernel layout.  Read from the notebook
  files (the reference checkout must be present, ``HFM_REFERENCE_ROOT``): the corrections
  ``w_2`` (2x2) and ``w_4`` (4x4) of one serial 2D sawtooth cycle
  (``notebooks/Parallel_multigrid_2D.ipynb`` cell 20, printed by cells 50 and 52), and the
  norm of the serial 3D solution after 100 sawtooth cycles
  (``notebooks/parallel_multigrid_advection_diffusion_3D.ipynb`` cell 15, printed by cell
  72).  These pin solution values.
* ``oracle_small.npz`` - seeded small-grid inputs and the oracle's outputs for every
  operator and for a few reference cycles.  TensorFlow 2.0 (the reference's pinned
  dependency) is not installable here, so these are the oracle's values, cross-checked at
  generation time against an independent ``torch.nn.functional.conv3d`` evaluation of the
  same layers; the GPU parity tests compare the CUDA library against them.
"""
import json
import os
import re
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


def _notebooks():
    """The reference checkout's notebook folder: HFM_REFERENCE_ROOT must name the checkout."""
    root = os.environ.get("HFM_REFERENCE_ROOT")
    if not root:
        raise SystemExit("set HFM_REFERENCE_ROOT to the bc1chen/AI-HFM-Solver checkout")
    return os.path.join(root, "Anisotropic Resistivity Tomography", "notebooks")


def _cell_text(notebook, cell):
    with open(os.path.join(_notebooks(), notebook)) as f:
        nb = json.load(f)
    out = []
    for o in nb["cells"][cell].get("outputs", []):
        out.append("".join(o.get("text", [])) if "text" in o
                   else "".join(o.get("data", {}).get("text/plain", [])))
    return "".join(out)


def _first_tensor(text):
    """Numbers of the first printed ``tf.Tensor(...)`` in ``text``, with its shape."""
    m = re.search(r"tf\.Tensor\((.*?), shape=\(([0-9, ]+)\)", text, re.S)
    vals = [float(v) for v in re.findall(r"-?\d+\.\d*(?:e-?\d+)?", m.group(1))]
    shape = tuple(int(v) for v in m.group(2).replace(" ", "").split(",") if v)
    return np.array(vals).reshape(shape).tolist()


def printed_solution_values():
    w2 = _first_tensor(_cell_text("Parallel_multigrid_2D.ipynb", 50))
    w4 = _first_tensor(_cell_text("Parallel_multigrid_2D.ipynb", 52))
    lines = _cell_text("parallel_multigrid_advection_diffusion_3D.ipynb", 72).splitlines()
    serial_norm = float(lines[1])     # print(serial_l1), after "ABE of subdomains"
    return {
        "mg2d_source": "notebooks/Parallel_multigrid_2D.ipynb cell 20 (128^2, dt=10, Dx=Dy=0.1, "
                       "ub=1, 40x40 box at 43 as source and initial guess, levels 128..2, "
                       "one cycle); values printed by cells 50 and 52",
        "mg2d_w2": w2,
        "mg2d_w4": w4,
        "mg3d_source": "notebooks/parallel_multigrid_advection_diffusion_3D.ipynb cell 15 "
                       "(128^3, 7-point Dx=Dy=Dz=100, 40^3 box at 43 as source and initial "
                       "guess, levels 128..2 with two Jacobi sweeps at 2^3, 100 cycles); "
                       "np.linalg.norm of the float32 result printed by cell 72",
        "mg3d_norm_after_100": serial_norm,
    }


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
    pins.update(printed_solution_values())
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
