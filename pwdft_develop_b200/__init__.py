"""pwdft_develop_b200 -- B200-native (sm_100a) plane-wave DFT Hamiltonian
application and block eigensolver, a drop-in for the reference's
Hamiltonian::MultSpinor / Spinor / Fourier / EigenSolver path.

The compute path is the native library ``libpwdft_b200.so`` (CUDA kernels +
C++ host code behind the C ABI in ``include/pwdft_b200.h``); this package is
a thin Python host mirror used by tests and benchmarks.
"""
from ._lib import PwError, lib  # noqa: F401  (fails loudly if the library is missing)
from .core import CellBatch, Context, HpsiGraph  # noqa: F401
