"""CPU oracle for the stencil + multigrid hot path (TEST INFRASTRUCTURE ONLY).

This package restates, in NumPy, the arithmetic that the reference (bc1chen/AI-HFM-Solver,
"AI4CFD") performs with frozen TensorFlow 2.0 Keras layers:

* ``tfops``    - Conv3D(k=3, s=1, 'SAME') as cross-correlation with zero padding, the
                 stride-2 VALID averaging restriction and UpSampling3D(2) prolongation.
* ``weights``  - the reference's hand-set kernels (7-point anisotropic, 27-point diffusion
                 and pressure, smoothed central advection / gradient / divergence).
* ``mg``       - the reference "sawtooth" multigrid cycles (7-point, variable-coefficient
                 six-direction form, NS pressure form), plus the textbook V / F cycles with
                 weighted Jacobi used by the solver configurations.
* ``ns``       - velocity / pressure / source boundary rules, the sigma-mask immersed body
                 and the two-stage momentum update of the NS scripts.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may
import this package, and only as the checker or as the timed CPU stand-in for the
reference.  The product path (``ai-hfm-solver_b200``) never calls into it.

Pinning.  TensorFlow 2.0.0 (the reference's pinned dependency, ``environment.yml:31``) is
not installable here, so the oracle cannot be compared with the reference's own outputs.
What *is* pinned:

* the kernel layout / axis order / cross-correlation convention, by the weights the
  reference printed (``Anisotropic Resistivity Tomography/notebooks/
  Multigrid_3d_7point_source.ipynb`` cells 4, 5 and 10: ``sum(w2) == 0``, the centre plane
  ``[[-0,-10,-0],[-20,70,-20],[-0,-10,-0]]`` and the full ``(3,3,3,1,1)`` kernel);
* the parameter counts of the Keras models (28 for a 3x3x3 conv + bias, 9 for 2x2x2);
* the convolution semantics, by an independent second implementation
  (``torch.nn.functional.conv3d`` on the CPU) in the tests.

Numeric *solution* values of the reference are **parity unpinned**: the reference saved no
arrays and its mesh inputs are missing, so no golden solution vector exists.
"""
