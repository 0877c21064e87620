"""CPU oracle for the FlowPM particle-mesh path -- TEST INFRASTRUCTURE ONLY.

This package is a restatement of the reference's algorithm for the PM hot
path, written for checking results, never for producing them.  Only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it.  The product package ``flowpm_b200`` does not, and
fails loudly when its CUDA library is missing instead of falling back here.

Modules (each function cites the reference file:line it restates):

* ``background`` -- ``flowpm/tfbackground.py`` (E(a), the growth ODE solved by
  RK4 on 256 log-spaced steps of a in [1e-2, 1], linear interpolation in ln a,
  the FastPM factors Gf/gf), NumPy, in float32 (what the reference computes)
  or float64 (the same method in double precision).
* ``power`` -- ``flowpm/tfpower.py`` + ``flowpm/scipy/integrate.py``
  (Eisenstein & Hu 1998 transfer function, sigma8 normalisation by Simpson's
  rule).
* ``pm`` -- ``flowpm/kernels.py``, ``flowpm/utils.py``, ``flowpm/tfpm.py`` and
  ``flowpm/pk.py`` in torch on the CPU (float32 or float64; autograd through
  it stands in for TensorFlow's tape gradient).

Parity pin: the oracle is checked against golden fixtures produced by running
the reference's own Python source (``tests/golden/make_golden.py``; TensorFlow
2.5 ops emulated in NumPy by ``tests/golden/tfshim.py`` because TensorFlow is
not installable here) and against the reference's FP64 background oracle
``flowpm/legacy_background.py`` -- see ``tests/test_oracle_golden.py``.
"""
