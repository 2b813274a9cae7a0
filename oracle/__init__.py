"""CPU oracle for the MaoMi optical stage (TEST INFRASTRUCTURE ONLY).

This package is a NumPy/SciPy restatement of the reference's CPU algorithm for
the optical stage and the local-PSF renderer.  It exists to check the CUDA
product path: only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline leg may import it.  The product package ``maomi_b200`` never
imports or calls anything here, and it has no CPU fallback.

Pinning: ``tests/golden/make_golden.py`` runs the reference implementation
itself (MaoMi 0.8.0b1, imported read-only) on seeded inputs and stores its
outputs as fixtures; ``tests/test_oracle_golden.py`` checks this restatement
against every fixture (FP64 to ~1e-12, FP32 to the reference's own FP32
rounding level).
"""
