"""CPU oracle for the MPS/MPO RK4 hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, in NumPy (OpenBLAS zgemm + LAPACK zgeqrf/zungqr), the
algorithms of jdnz/MatrixProductStates.jl that the RK4 time step runs through:

* ``mps_ref``  -- src/mps_base.jl, src/orthonormalisation.jl, src/compression.jl,
                  src/timeevolution.jl, src/constructors.jl, src/MatrixProductStates.jl
* ``models``   -- the spin-model MPO builders of examples/spin_model_quantum_trajectory_rk4.jl
                  and examples/spin_model_density_matrix.jl
* ``drivers``  -- the trajectory / density-matrix time loops of those examples
* ``dense``    -- exact dense state-vector / density-matrix RK4, used to pin the
                  restatement where the single-site sweep is exact (full bond dim)

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker / the timed CPU
baseline.  The GPU product never routes through it.

PARITY UNPINNED: the reference ships no tests, fixtures or golden vectors
(test/runtests.jl:1-2 only loads the module) and cannot run here (it needs
Julia 0.6.4, which is absent).  The restatement is instead pinned against exact
dense evolution at full bond dimension (``dense``), against the RK4 algebra, and
against conservation laws (trace, hermiticity, jump-probability sums).
"""
