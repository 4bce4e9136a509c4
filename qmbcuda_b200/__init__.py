"""B200-native XXZ/Heisenberg exact diagonalization (Lanczos ground states
with Abelian symmetries) behind a C ABI (include/qmb_b200.h).

The compute path is libqmb_b200.so (hand-written sm_100a CUDA + C++ host
code); this package binds it with ctypes.  Importing it loads the library and
fails if it has not been built (`python qmbcuda_b200/build.py`).
"""
from . import _capi
from ._capi import QMBError, check, lib
from .engine import (Batch, Hamiltonian, Sector, TermTable, chain_bonds, export_nosym,
                     export_ref, fourier_terms, geometry, load_ref_ell, multiply_terms, operator_terms,
                     reciprocal_basis, save_ref_ell, square_bonds, translation_group,
                     with_spin_flip, xxz_terms)

lib()

__all__ = ["Batch", "Hamiltonian", "QMBError", "Sector", "TermTable", "chain_bonds", "check",
           "export_nosym", "export_ref", "fourier_terms", "geometry", "lib", "load_ref_ell", "multiply_terms",
           "operator_terms", "reciprocal_basis", "save_ref_ell", "square_bonds", "translation_group",
           "with_spin_flip", "xxz_terms"]
