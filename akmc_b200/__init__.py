"""akmc_b200: B200-native force/energy path of adaptive kinetic Monte Carlo (AKMC).

EAM density/embedding/force passes and Buckingham + Ewald (real-space erfc and
reciprocal structure-factor) sums as hand-written sm_100a CUDA kernels behind a C ABI
(include/akmc.h, ``libakmc_b200.so``), with this package as the host-side mirror of the
reference's ``Field`` / ``Species`` / ``Energy`` interface, and batched FIRE relaxation
and Dimer saddle-search walkers on top of it (:class:`Walkers`).
"""
from ._lib import AkmcError, Energy, STATUS, STATUS_NAMES, load  # noqa: F401
from .field import Batch, Element, Field, Species, PREC_FP64, PREC_MIXED, FAMILY_EAM, FAMILY_IONIC  # noqa: F401
from .walkers import Walkers, dimer_params, fire_params  # noqa: F401

__all__ = ["AkmcError", "Energy", "Field", "Batch", "Species", "Element", "load", "Walkers",
           "fire_params", "dimer_params",
           "PREC_FP64", "PREC_MIXED", "FAMILY_EAM", "FAMILY_IONIC", "STATUS", "STATUS_NAMES"]
