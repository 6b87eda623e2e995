"""B200-native CCSD for NuLattice's lattice Hamiltonians.

Public entry points:

* :func:`ccsd_solver` -- drop-in for ``NuLattice.CCM.soa.coupled_cluster.ccsd_solver``
* :func:`get_norm_ordered_ham` -- lattice Hamiltonian builder in the reference's conventions
"""
from .ccsd import ccsd_solver  # noqa: F401
from .hamiltonian import (normal_ordered_hamiltonian, phys_unit, closed_shell_holes,  # noqa: F401
                          contact_couplings)

__all__ = ["ccsd_solver", "normal_ordered_hamiltonian", "phys_unit", "closed_shell_holes",
           "contact_couplings"]
