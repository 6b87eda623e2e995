"""B200-native CCSD for NuLattice's lattice Hamiltonians.

Public entry points:

* :func:`ccsd_solver` -- drop-in for ``NuLattice.CCM.soa.coupled_cluster.ccsd_solver``
  (and its NumPy twin ``NuLattice.CCM.coupled_cluster.ccsd_solver``)
* :func:`normal_ordered_hamiltonian` -- the lattice Hamiltonian (hopping, SU(4)
  contact, three-body contact) normal-ordered to a closed-site reference, as the
  blocks ``ccsd_solver`` takes; the counterpart of the reference's
  ``get_norm_ordered_ham``
* :func:`closed_shell_holes`, :func:`contact_couplings`, :func:`phys_unit` --
  hole lists, coupling-unit conversion and the physical energy unit
"""
from .ccsd import ccsd_solver  # noqa: F401
from .hamiltonian import (normal_ordered_hamiltonian, phys_unit, closed_shell_holes,  # noqa: F401
                          contact_couplings)

__all__ = ["ccsd_solver", "normal_ordered_hamiltonian", "phys_unit", "closed_shell_holes",
           "contact_couplings"]
