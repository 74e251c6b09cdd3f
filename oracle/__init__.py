"""CPU oracle for the phaseless-AFQMC walker step (test infrastructure only).

This package is a numpy/scipy restatement of ipie's CPU algorithm for the
single-determinant, real-Cholesky walker step.  It is the checker: only the
tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may
import it.  The product (``ipie_b200``) never calls into it.
"""
