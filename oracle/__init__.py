"""CPU FP64 oracle for the PWDFT Hamiltonian / eigensolver hot path.

TEST INFRASTRUCTURE ONLY.  This package restates, in NumPy, the algorithms
of the reference plane-wave DFT code (xmqin/pwdft_develop) that the CUDA
library in ``pwdft_develop_b200`` replaces.  Each function cites the
reference file:line it follows.  Only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg may import it, and only as the checker or
the timed CPU baseline -- never as the thing measured or shipped.

Parity status: the reference needs MPI, FFTW, MKL, libxc and yaml-cpp, none
of which exist on this machine, so the reference binary cannot be run.  The
oracle is pinned (a) against reference functions that compile standalone
(``IP_c2f``/``IP_f2c`` and ``spline``/``seval`` from ``src/utility.cpp``,
built by ``oracle/build_ref.sh`` into ``oracle/_ref/``), and (b) by
known-answer tests (free-electron spectrum, single plane waves, Parseval,
Hermiticity, Teter closed form, projector normalisation, charge
neutrality).  Everything else is "parity partially pinned".
"""
