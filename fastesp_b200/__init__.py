"""fastesp_b200 -- exact electrostatic potential of a Gaussian-basis density on B200.

Drop-in for fastesp's public API (fastesp/__init__.py:27-42)::

    from fastesp_b200 import read_molden, Basis, build_table

    wfn = read_molden("mol.molden.input")
    basis = Basis(wfn)
    density = basis.density_matrix_cartesian()
    table = build_table(wfn, basis, density, points_bohr)   # built on the GPU
    esp = table.esp()                                        # (n_points,) Hartree/e

The pair table is built and evaluated by CUDA kernels for sm_100a
(csrc/, C ABI in include/fastesp_b200.h) called through ctypes; the MOLDEN
reader and Cartesian basis are host-side NumPy.
"""
from __future__ import annotations

from .basis import Basis, cart_order, overlap_matrix
from .ints import boys, primitive_pair_integral
from .molden import Wavefunction, read_molden
from .table import PairTable, basis_payload, build_table, write_basis_payload

__version__ = "0.1.0"

__all__ = [
    "Wavefunction", "read_molden",
    "Basis", "cart_order", "overlap_matrix",
    "boys", "primitive_pair_integral",
    "PairTable", "build_table",
    "basis_payload", "write_basis_payload",
    "__version__",
]
