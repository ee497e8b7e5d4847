"""MOLDEN wavefunction reader (host side).

Same contract as fastesp's ``read_molden`` (fastesp/molden.py:65-169):

* ``[Atoms] AU`` only -- coordinates are taken as Bohr (fastesp/molden.py:86-90);
* ``[GTO]``: per atom a ``<atom> 0`` line, then shells ``<l-letter> <nprim> <scale>``
  followed by ``nprim`` lines ``exponent coefficient`` (fastesp/molden.py:93-117);
* ``[5D]``/``[7F]``/``[9G]`` style flags mark spherical shells
  (fastesp/molden.py:119);
* ``[MO]``: blocks of ``Sym=/Ene=/Spin=/Occup=`` headers followed by
  ``index value`` rows; the coefficient is the last field of a row, the AO count
  is the largest index seen (fastesp/molden.py:121-162).

Nothing here runs on the GPU: the reader produces the shells and MO
coefficients that :class:`fastesp_b200.basis.Basis` turns into the Cartesian
density consumed by the table-build kernels.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

BOHR = 0.529177210903  # Angstrom per Bohr (CODATA 2018)

_L_LETTERS = "spdfghijkl"

# Nuclear charges by element symbol (the set fastesp's table builder knows,
# fastesp/table.py:262-265).
Z_OF = {"H": 1.0, "He": 2.0, "Li": 3.0, "Be": 4.0, "B": 5.0, "C": 6.0, "N": 7.0,
        "O": 8.0, "F": 9.0, "Ne": 10.0, "Na": 11.0, "Mg": 12.0, "Al": 13.0,
        "Si": 14.0, "P": 15.0, "S": 16.0, "Cl": 17.0, "Ar": 18.0, "Br": 35.0,
        "I": 53.0}
_SECTION = re.compile(r"^\[([^\]]+)\]\s*(.*)$")
_ATOM_LINE = re.compile(
    r"^\s*(\S+)\s+(\d+)\s+(\d+)\s+([-+\d.eEdD]+)\s+([-+\d.eEdD]+)\s+([-+\d.eEdD]+)")


@dataclass
class Shell:
    """One contracted Cartesian/spherical Gaussian shell on an atom."""
    atom: int            # 0-based atom index
    l: int               # angular momentum
    exps: np.ndarray     # (nprim,) primitive exponents
    coeffs: np.ndarray   # (nprim,) contraction coefficients as written in the file


@dataclass
class Wavefunction:
    symbols: list
    coords: np.ndarray      # (natom, 3) Bohr
    shells: list
    mo_energy: np.ndarray   # (nmo,)
    mo_occ: np.ndarray      # (nmo,)
    mo_coeff: np.ndarray    # (nao, nmo) in the stored (spherical) AO order
    spherical: dict = field(default_factory=dict)

    @property
    def natom(self) -> int:
        return len(self.symbols)

    @property
    def nao(self) -> int:
        return int(self.mo_coeff.shape[0])

    @property
    def nelec(self) -> float:
        return float(np.sum(self.mo_occ))


def _float(tok: str) -> float:
    return float(tok.replace("D", "E").replace("d", "e"))


def _coefficient_block(block: list):
    """(indices, values) of one MO's "index value" lines.  The common layout
    (two numbers on every non-empty line) is converted in one NumPy call; any
    other layout line by line, taking the first and the last field of a row as
    the reference does."""
    rows = len(block) - block.count("")
    text = " ".join(block).replace("D", "E").replace("d", "e")
    try:
        arr = np.array(text.split(), dtype=np.float64)
    except ValueError:
        arr = None
    if arr is not None and arr.size == 2 * rows:
        pairs = arr.reshape(-1, 2)
        return pairs[:, 0].astype(np.int64), pairs[:, 1].copy()
    idx, val = [], []
    for ln in block:
        f = ln.split()
        if len(f) >= 2:
            idx.append(int(f[0]))
            val.append(_float(f[-1]))
    return np.asarray(idx, dtype=np.int64), np.asarray(val, dtype=np.float64)


_HEADER_LINE = re.compile(r"^[ \t]*\[.*$", re.M)
_SYM_LINE = re.compile(r"^[ \t]*Sym=", re.M)


def _section_text(text: str) -> dict:
    """Map section name -> its body text: from the end of its header line to the
    next line that starts with ``[`` (first occurrence of a name wins)."""
    heads = list(_HEADER_LINE.finditer(text))
    out = {}
    for k, m in enumerate(heads):
        h = _SECTION.match(m.group(0).strip())
        if not h or h.group(1).strip() in out:
            continue
        end = heads[k + 1].start() if k + 1 < len(heads) else len(text)
        out[h.group(1).strip()] = text[m.end():end]
    return out


def read_molden(path) -> Wavefunction:
    """Parse a MOLDEN file into a :class:`Wavefunction` (atomic units).

    Works on the file text: section headers are found with one multiline
    search, each section is sliced out by offset, and every MO's coefficient
    rows are converted in one NumPy call (the bulk of a large file)."""
    text = Path(path).read_text(errors="ignore")
    sec = _section_text(text)
    for need in ("Atoms", "GTO", "MO"):
        if need not in sec:
            raise ValueError(f"{path}: MOLDEN section [{need}] missing")

    symbols, coords = [], []
    for raw in sec["Atoms"].splitlines():
        m = _ATOM_LINE.match(raw)
        if m:
            symbols.append(m.group(1))
            coords.append([_float(m.group(k)) for k in (4, 5, 6)])
    coords_arr = np.asarray(coords, dtype=np.float64).reshape(-1, 3)

    shells = []
    gto = sec["GTO"].splitlines()
    atom = -1
    i = 0
    while i < len(gto):
        f = gto[i].split()
        if not f:
            i += 1
            continue
        if len(f) == 2 and f[0].lstrip("-").isdigit():
            atom = int(f[0]) - 1
            i += 1
            continue
        l = _L_LETTERS.index(f[0].lower())
        nprim = int(f[1])
        rows = [gto[i + 1 + k].split() for k in range(nprim)]
        shells.append(Shell(atom=atom, l=l,
                            exps=np.array([_float(r[0]) for r in rows]),
                            coeffs=np.array([_float(r[1]) for r in rows])))
        i += 1 + nprim

    spherical = {l: f"{2 * l + 1}{'SPDFGH'[l]}" in sec for l in range(5)}

    energies, occs, cols = [], [], []
    mo = sec["MO"]
    starts = [m.start() for m in _SYM_LINE.finditer(mo)]
    for k, a in enumerate(starts):
        lines = mo[a:starts[k + 1] if k + 1 < len(starts) else len(mo)].splitlines()
        ene = occ = 0.0
        j = 1                                  # lines[0] is the Sym= line
        while j < len(lines):
            t = lines[j].strip()
            if t.startswith("Ene="):
                ene = _float(t.split("=", 1)[1])
            elif t.startswith("Occup="):
                occ = _float(t.split("=", 1)[1])
            elif not (t.startswith("Spin=") or not t):
                break
            j += 1
        energies.append(ene)
        occs.append(occ)
        cols.append(_coefficient_block(lines[j:]))

    if not cols:
        raise ValueError(f"{path}: no molecular orbitals in [MO]")
    nao = max(int(ix.max()) for ix, _ in cols if ix.size)
    coeff = np.zeros((nao, len(cols)))
    for j, (ix, v) in enumerate(cols):
        coeff[ix - 1, j] = v
    return Wavefunction(symbols=symbols, coords=coords_arr, shells=shells,
                        mo_energy=np.asarray(energies), mo_occ=np.asarray(occs),
                        mo_coeff=coeff, spherical=spherical)


def write_molden(path, symbols, coords, shells, mo_coeff, mo_occ,
                 mo_energy=None) -> Path:
    """Write a MOLDEN file in the layout :func:`read_molden` accepts.

    ``shells`` is a list of :class:`Shell`; ``mo_coeff`` is (nao_spherical, nmo)
    in the spherical ordering (real solid harmonics, m = 0, +1, -1, ...).
    Coefficients are written with 12 decimals, exponents and contraction
    coefficients with 10, as the reference's synthetic-wavefunction writer does
    (tests/test_pipeline.py:34-54).
    """
    path = Path(path)
    out = ["[Molden Format]", "[Atoms] AU"]
    for i, (s, (x, y, z)) in enumerate(zip(symbols, np.asarray(coords))):
        out.append(f"{s} {i + 1} {int(Z_OF[s])} {x:.10f} {y:.10f} {z:.10f}")
    out.append("[GTO]")
    for a in range(len(symbols)):
        out.append(f" {a + 1} 0")
        for sh in shells:
            if sh.atom != a:
                continue
            out.append(f"{_L_LETTERS[sh.l]}   {len(sh.exps)} 1.0 ")
            for e, c in zip(sh.exps, sh.coeffs):
                out.append(f"   {e:20.10f} {c:20.10f}")
        out.append("")
    out += ["[5D]", "[7F]", "[9G]", "[MO]"]
    mo_coeff = np.asarray(mo_coeff)
    ene = np.full(mo_coeff.shape[1], -0.5) if mo_energy is None else mo_energy
    for k in range(mo_coeff.shape[1]):
        out.append(f" Sym=     {k + 1}a")
        out.append(f" Ene= {ene[k]: .14E}")
        out.append(" Spin= Alpha")
        out.append(f" Occup=  {mo_occ[k]:.6f}")
        col = mo_coeff[:, k]
        out.extend(f"{i + 1:5d} {v:20.12f}" for i, v in enumerate(col))
    path.write_text("\n".join(out) + "\n")
    return path
