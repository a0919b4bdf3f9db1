"""CPU oracle for the TensorSPH particle pass -- TEST INFRASTRUCTURE ONLY.

This package is a numpy restatement of the reference algorithms (TensorSPH,
``src/tensorsph/...``) for the neighbour search and the pair pass.  It exists
to check the CUDA path and to time a CPU baseline:

* only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
  ``--impl reference`` legs of ``bench.py`` may import it;
* nothing under ``tensorsph_b200`` imports it, and the product path never falls
  back to it (the CUDA library is mandatory there).

Parity pin: ``tests/golden/make_golden.py`` runs the reference itself (PyTorch
eager, CPU) on seeded inputs and stores inputs and outputs as ``.npz``
fixtures; ``tests/test_oracle_golden.py`` checks every oracle function against
them (bit-exact for pairs and cell order, tolerance for floating point).
"""
