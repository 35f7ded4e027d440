"""B200-native eight-band k.p eigensolve: matrix-free H.X and LOBPCG on sm_100a.

Drop-in for qd3Dsolver's hot path: `kp_pryor.confined_hamiltonian` returns a device-resident
operator, and `eigensolvers.solve_interior` / `solve_lowest` run LOBPCG on the GPU with the
reference's signatures and return conventions. Host-side input producers live in `workloads`.
"""
from . import _lib  # noqa: F401

__all__ = ['kp_pryor', 'eigensolvers', 'workloads']
