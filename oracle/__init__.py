"""CPU oracle for the tiled LU / Cholesky task-graph path (test infrastructure).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
import this package, and only to check or to time a CPU reference.  The product
path (``mustard_b200``) never imports it.

Contents
--------
gen      -- the reference's ``srand(420)`` generator (include/gen.h:23-38) and the
            seeded uniform / SPD generators the benchmark configurations name.
tiled    -- the reference's task lists (cholesky_mustard.cu:224-395,
            lu_mustard.cu:345-533), its last-writer dependency inference
            (mustard/mustard.h:279-296) and a sequential executor of the task list
            with LAPACK/BLAS tile operations.
verify   -- the reference's ``--verify`` criterion (include/verify.h:17-129) plus
            normwise residuals.
"""
