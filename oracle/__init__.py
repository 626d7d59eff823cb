"""CPU oracle for the DiffCP cloth-MPM hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker.  The product
(``diffcp_b200``) never imports it: the CUDA path fails loudly when its
extension is missing instead of falling back here.

Contents
--------
``sim64``      torch restatement (FP64 by default) of ``src/simulation.py`` and
               ``compute_loss`` of ``src/parameter_fitting_functions.py``;
               gradients come from ``torch.autograd`` over the restatement,
               with the reference's hand-written clamped 2x2 SVD backward
               (``simulation.py:44-50,71-94``) available as a custom Function.
``scene_ref``  restatement of the scene constants and normalisation of
               ``src/initialization.py``.

Parity pin
----------
The forward restatement is pinned by golden vectors that were produced by
executing the reference's own source files (``src/initialization.py``,
``src/taichi_variable_definition.py``, ``src/simulation.py``,
``src/parameter_fitting_functions.py``) under a NumPy stand-in for the Taichi
runtime (``tests/golden/make_golden.py``).  Gradients are pinned against
central finite differences of that same reference-source execution run in
FP64.  Taichi's own reverse-mode AD could not be executed (the ``taichi``
package is not installed and is not vendored by the reference), so gradient
parity with Taichi AD specifically is unpinned.
"""
