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
not installable here, so the oracle cannot be run beside the reference.  It is pinned to
numbers the reference printed in its saved notebook outputs (``tests/golden/
reference_pins.json``, extracted by ``tests/golden/make_golden.py``):

* the kernel layout / axis order / cross-correlation convention, by the weights the
  reference printed (``Anisotropic Resistivity Tomography/notebooks/
  Multigrid_3d_7point_source.ipynb`` cells 4, 5 and 10: ``sum(w2) == 0``, the centre plane
  ``[[-0,-10,-0],[-20,70,-20],[-0,-10,-0]]`` and the full ``(3,3,3,1,1)`` kernel);
* the parameter counts of the Keras models (28 for a 3x3x3 conv + bias, 9 for 2x2x2);
* solution values of the 2D reference cycle: the 2x2 and 4x4 corrections of one serial cycle
  of ``notebooks/Parallel_multigrid_2D.ipynb`` (cell 20, printed by cells 50 and 52), equal
  to the printed 8 decimals;
* solution values of the 3D reference cycle: the norm of the serial solution after 100
  cycles of ``notebooks/parallel_multigrid_advection_diffusion_3D.ipynb`` (cell 15, printed by
  cell 72: 288.47165), equal when the norm is summed as a float32 BLAS dot and within 1e-4
  of the exact norm;
* the convolution semantics, by an independent second implementation
  (``torch.nn.functional.conv3d`` on the CPU) in the tests.

Not pinned: values of the variable-coefficient and time-stepping paths, whose reference runs
read mesh files that are missing from the reference.
"""
