"""CPU oracle for the TorchSim classical-potential hot path (TEST INFRASTRUCTURE ONLY).

This package is a plain-numpy FP64 restatement of the reference algorithms
(TorchSim ``torch-sim-atomistic`` 0.6.1).  It exists to check the CUDA product
path; it is never the product.  Only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` may import it.

Parity pin: every function here is checked against golden vectors produced by
running the reference itself (``tests/golden/make_golden.py``, committed with
its ``.npz`` outputs) in ``tests/test_oracle_golden.py``.

Modules
-------
neighbors   periodic neighbour list (pair set, wrap, half list)
pair        LJ / Morse / soft-sphere / species-matrix pair energy, force, virial
md          velocity-Verlet, BAOAB Langevin, momenta initialisation, kT
fire        ASE-/VV-FIRE and the Frechet cell filter
linalg3     3x3 expm + Frechet derivative (Pade-13), matrix log
"""
