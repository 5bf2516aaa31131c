"""CPU oracle for the Diff-FVR hot path -- TEST INFRASTRUCTURE ONLY.

This package is the checker, never the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it.
The product path (``diff-fvr_b200/fvr``) never imports, links or executes
anything from here and fails loudly when its CUDA library is missing.

Contents (each function cites the reference ``file:line`` it restates):

* ``torch_convention`` -- float64 NumPy restatement of the parallel-beam
  ``TorchDiffFVREngine`` (``src/fvr/torch_engine.py``) and of the trilinear
  slice gather ``fourier_slice_3d`` (``src/fvr/triton_slice.py``), with a
  hand-derived per-sample adjoint for the pose gradient.
* ``pou`` -- float64 restatement of the PoU-FVR cone-beam renderer
  (``src/fvr/cone_beam_fvr.py``) and the pinhole warp-sum, with its adjoint.
* ``numpy_convention`` -- restatement of ``DifferentiableFourierVolumeRenderer``
  (``src/fvr/diff_fvr.py``) and ``SpectralGradientEngine``
  (``src/fvr/gradients.py``).
* ``fvr_oracle.c`` -- plain-C (OpenMP) restatement of the batched spectral-NCC
  loss + pose gradient, used as the timed CPU baseline and for full-size
  checks.

Parity of the oracle is pinned against golden vectors produced by running the
reference itself (``tests/golden/make_golden.py``; fixtures in
``tests/golden/*.npz``).
"""
