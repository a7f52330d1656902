"""CPU oracle for PyExner's explicit finite-volume step (test infrastructure only).

This package is the CHECKER, not the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm may import
or execute it.  The product path (``pyexner_b200``) never calls into it and fails
loudly when its CUDA library is missing.

Contents (NumPy, float64, vectorised, literal operation order of the reference):
  * ``roe_exner``  – Roe-Exner face flux, wave speeds / CFL, MPM grass factor, Exner
    update, momentum corrections, the stage and init of the "Roe Exner" bundle
    (PyExner src/PyExner/solvers/kernels/roe_exner.py, solvers/roe_exner_solver.py);
  * ``roe``        – plain Roe SWE step and CFL (solvers/kernels/roe.py, solvers/roe_solver.py);
  * ``boundaries`` – polygon masks, boundary/interior index maps and the ghost-cell
    handlers on the hot path (domain/boundary_registry.py, domain/boundaries/*.py);
  * ``integrators``– fixed-step Forward Euler and SSPRK2 loops.

Parity pin: ``tests/golden/*.npz`` were produced by executing PyExner's own modules
(unmodified) on float64 numpy through ``tests/golden/jaxshim.py``; the script that made
them is ``tests/golden/make_golden.py``.  ``tests/test_oracle_golden.py`` checks this
oracle against every one of those vectors.  The shim replaces XLA's arithmetic by
numpy's, so the pin is "the reference's code with numpy float64 arithmetic" (XLA and
numpy can differ in the last ulp of transcendental functions).
"""
