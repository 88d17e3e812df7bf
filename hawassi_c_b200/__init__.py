"""B200-native engine for HAWASSI's 1D pseudo-spectral Hamiltonian RHS and its
RKF45 time stepping.

The compute path is the CUDA library ``lib/libhawassi_b200.so`` (sm_100a), driven
through its C ABI (``include/hawassi_b200.h``).  This package is the host-side
mirror of the reference's call surface:

* :class:`Engine` -- one deck or a ragged ensemble of decks; ``rhs`` replaces
  ``rhs_HsF1/2/3`` (1d/rhs.c), ``evolve_apply`` replaces ``gsl_odeiv_evolve_apply``
  (1d/functions.c:550) and ``run`` replaces the time loop of ``ode_solver_Ham``.
* :mod:`hawassi_c_b200.decks` -- writes seeded synthetic decks in the reference's
  ``input.txt`` / ``influx.dat`` / ``bath.dat`` format.

There is no CPU fallback: without the built library or a CUDA device every
entry point raises.
"""
from .engine import Engine, EngineError, fp64_peak_tflops, library_path, load_library  # noqa: F401

__all__ = ["Engine", "EngineError", "fp64_peak_tflops", "library_path", "load_library"]
