"""Seeded synthetic ESP workloads.

The reference benchmarks a 54-atom protein fragment whose MOLDEN file and point
sets are not distributed, so the workloads here are generated from a seed with
the shapes of the reference's benchmark system:

* ``small``   : 6 atoms (Z in {1,6,7,8}), heavy atoms 3s2p1d, H 2s1p, 1-6
  primitives per shell, exponents log-uniform in [0.1, 1e4], ~60 Cartesian
  functions, 300 points on the 1.4 x Bondi surface.
* ``frag54``  : 54 atoms (30 C / 8 N / 8 O / 8 H) in a packed chain with
  1.0-1.6 A bonds, triple-zeta-plus-diffuse-like basis up to f (diffuse
  exponents down to 0.02): ~1650 Cartesian functions, ~2090 primitives.
* ``tz``      : ``natom`` atoms (default 6) of the frag54 recipe (all classes L=0..6).
* ``adjoint20``: 20 atoms of the same recipe with an l<=2 basis (~270 functions).
* ``batch``   : molecules of 5-60 atoms with l<=2 bases.
* ``qz``      : a few atoms whose heavy atoms also carry a g shell (classes up
  to L = 8, the g-shell kernel instances).

Contraction coefficients are drawn uniform in [0.1, 1] and multiplied by the
radial factor N_s(a, l) that MOLDEN coefficients carry (the convention
:class:`fastesp_b200.basis.Basis` reads).  Occupied orbitals are random and
orthonormal in the basis metric (C^T S C = 1, canonical orthogonalisation that
drops overlap eigenvalues below ``lindep``), n_occ = sum(Z)/2, so the density
satisfies Tr(P S) = N_elec.  Points lie on the union of 1.4 x Bondi vdW spheres
(Fibonacci sphere per atom, exposed points only), or on a cubic grid.
"""
from __future__ import annotations

import hashlib
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from .basis import Basis, overlap_matrix, primitive_norm
from .molden import BOHR, Shell, Wavefunction, read_molden, write_molden

BONDI = {"H": 1.20, "C": 1.70, "N": 1.55, "O": 1.52, "S": 1.80, "P": 1.80}
Z_OF_SYM = {"H": 1, "C": 6, "N": 7, "O": 8}

# (l, nprim, log10 exponent range) per shell.  Exponent ranges loosely follow a
# triple-zeta basis with diffuse functions; the exact values are drawn per atom.
_TZ_HEAVY = [(0, 4, (1.0, 3.7)), (0, 1, (-0.1, 0.5)), (0, 1, (-0.8, -0.3)),
             (0, 1, (-1.7, -1.1)),
             (1, 3, (0.0, 1.6)), (1, 1, (-0.8, -0.3)), (1, 1, (-1.7, -1.1)),
             (2, 1, (-0.1, 0.3)), (2, 1, (-0.8, -0.4)),
             (3, 1, (-0.4, 0.1))]
_TZ_H = [(0, 3, (-0.5, 1.6)), (0, 1, (-1.0, -0.5)), (0, 1, (-1.7, -1.2)),
         (1, 1, (-0.5, 0.1))]
_QZ_HEAVY = _TZ_HEAVY + [(4, 1, (-0.3, 0.2))]     # adds a g shell (classes up to L = 8)
_DZ_HEAVY = [(0, 4, (0.5, 3.5)), (0, 1, (-0.3, 0.3)), (0, 1, (-1.0, -0.5)),
             (1, 3, (-0.3, 1.5)), (1, 1, (-1.0, -0.5)),
             (2, 1, (-0.4, 0.1))]
_DZ_H = [(0, 3, (-0.7, 1.4)), (0, 1, (-1.2, -0.7)), (1, 1, (-0.5, 0.0))]


@dataclass
class System:
    """A synthetic molecule: geometry, basis shells and occupied orbitals."""
    name: str
    symbols: list
    coords: np.ndarray      # (natom, 3) Bohr
    shells: list            # list[Shell]
    mo_coeff: np.ndarray    # (nsph, nmo)
    mo_occ: np.ndarray

    def wavefunction(self) -> Wavefunction:
        return Wavefunction(symbols=list(self.symbols), coords=self.coords,
                            shells=self.shells, mo_energy=np.full(len(self.mo_occ), -0.5),
                            mo_occ=self.mo_occ, mo_coeff=self.mo_coeff,
                            spherical={0: False, 1: False, 2: True, 3: True, 4: True})

    def write(self, path) -> Path:
        return write_molden(path, self.symbols, self.coords, self.shells,
                            self.mo_coeff, self.mo_occ)


def _chain_geometry(rng, symbols, bond=(1.0, 1.6), min_sep=1.0, pack=True):
    """Packed chain: each atom bonded to the previous one at a random length (A)."""
    pts = [np.zeros(3)]
    for _ in range(1, len(symbols)):
        prev = pts[-1]
        allp = np.array(pts)
        best = None
        for _try in range(200):
            d = rng.uniform(*bond)
            dirs = rng.normal(size=(64, 3))
            dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
            cand = prev + d * dirs
            sep = np.linalg.norm(cand[:, None, :] - allp[None, :, :], axis=2)
            sep[:, -1] = np.inf
            ok = (sep >= min_sep).all(axis=1)
            if not ok.any():
                continue
            cand = cand[ok]
            if pack:
                cen = allp.mean(axis=0)
                best = cand[np.argmin(np.linalg.norm(cand - cen, axis=1))]
            else:
                best = cand[0]
            break
        if best is None:
            raise RuntimeError("could not place atom")
        pts.append(best)
    xyz = np.array(pts)
    return np.round((xyz - xyz.mean(axis=0)) / BOHR, 10)


def _draw_shells(rng, symbols, recipe_heavy, recipe_h):
    shells = []
    for a, s in enumerate(symbols):
        for (l, nprim, (lo, hi)) in (recipe_h if s == "H" else recipe_heavy):
            ex = np.sort(10.0 ** rng.uniform(lo, hi, size=nprim))[::-1]
            d = rng.uniform(0.1, 1.0, size=nprim)
            shells.append(_shell(a, l, ex, d))
    return shells


def _shell(atom, l, ex, d):
    """Shell with values rounded to the precision the MOLDEN writer keeps."""
    ex = np.round(ex, 10)
    return Shell(atom=atom, l=l, exps=ex, coeffs=np.round(d * primitive_norm(ex, l, 0, 0), 10))


def _small_shells(rng, symbols):
    shells = []
    for a, s in enumerate(symbols):
        spec = [(0, 2), (0, 1), (1, 1)] if s == "H" else \
            [(0, 1), (0, 1), (0, 1), (1, 1), (1, 1), (2, 1)]
        for l, _ in spec:
            nprim = int(rng.integers(1, 7))
            ex = np.sort(10.0 ** rng.uniform(-1.0, 4.0, size=nprim))[::-1]
            d = rng.uniform(0.1, 1.0, size=nprim)
            shells.append(_shell(a, l, ex, d))
    return shells


def _occupied_orbitals(rng, symbols, coords, shells, lindep=1e-4):
    """Random occupied orbitals, orthonormal in the spherical-basis overlap metric."""
    wfn = Wavefunction(symbols=list(symbols), coords=coords, shells=shells,
                       mo_energy=np.zeros(1), mo_occ=np.zeros(1),
                       mo_coeff=np.zeros((1, 1)))
    b = Basis(wfn)
    t = b.block_transform()
    s_sph = t.T @ overlap_matrix(b) @ t
    w, v = np.linalg.eigh(s_sph)
    keep = w > lindep * w.max()
    x = v[:, keep] / np.sqrt(w[keep])[None, :]
    nz = sum(Z_OF_SYM[s] for s in symbols)
    ndocc, nsocc = nz // 2, nz % 2
    nocc = ndocc + nsocc
    q, _ = np.linalg.qr(rng.normal(size=(x.shape[1], nocc)))
    c = np.round(x @ q, 12)
    occ = np.array([2.0] * ndocc + [1.0] * nsocc)
    return c, occ


def make_system(name: str, seed: int = 0, natom: int | None = None) -> System:
    """Generate one of the named synthetic systems (deterministic in ``seed``)."""
    rng = np.random.default_rng([seed, sum(name.encode())])
    if name == "small":
        symbols = [str(x) for x in rng.choice(["H", "C", "N", "O"], size=6,
                                               p=[0.25, 0.35, 0.2, 0.2])]
        if all(s == "H" for s in symbols):
            symbols[0] = "C"
        coords = _chain_geometry(rng, symbols, bond=(1.0, 1.5))
        shells = _small_shells(rng, symbols)
    elif name == "frag54":
        symbols = ["C"] * 30 + ["N"] * 8 + ["O"] * 8 + ["H"] * 8
        rng.shuffle(symbols)
        coords = _chain_geometry(rng, symbols, bond=(1.0, 1.6))
        shells = _draw_shells(rng, symbols, _TZ_HEAVY, _TZ_H)
    elif name == "tz":
        n = natom if natom is not None else 6
        comp = np.array(["C"] * 30 + ["N"] * 8 + ["O"] * 8 + ["H"] * 8)
        symbols = [str(x) for x in rng.choice(comp, size=n, replace=n > len(comp))]
        coords = _chain_geometry(rng, symbols, bond=(1.0, 1.6))
        shells = _draw_shells(rng, symbols, _TZ_HEAVY, _TZ_H)
    elif name == "qz":
        n = natom if natom is not None else 4
        comp = np.array(["C"] * 30 + ["N"] * 8 + ["O"] * 8 + ["H"] * 8)
        symbols = [str(x) for x in rng.choice(comp, size=n, replace=n > len(comp))]
        if all(s == "H" for s in symbols):
            symbols[0] = "C"
        coords = _chain_geometry(rng, symbols, bond=(1.0, 1.6))
        shells = _draw_shells(rng, symbols, _QZ_HEAVY, _TZ_H)
    elif name in ("adjoint20", "batch"):
        n = natom if natom is not None else 20
        comp = np.array(["C"] * 30 + ["N"] * 8 + ["O"] * 8 + ["H"] * 8)
        symbols = [str(x) for x in rng.choice(comp, size=n, replace=n > len(comp))]
        coords = _chain_geometry(rng, symbols, bond=(1.0, 1.6))
        shells = _draw_shells(rng, symbols, _DZ_HEAVY, _DZ_H)
    else:
        raise ValueError(f"unknown system {name!r}")
    c, occ = _occupied_orbitals(rng, symbols, coords, shells)
    return System(name=name, symbols=symbols, coords=coords, shells=shells,
                  mo_coeff=c, mo_occ=occ)


def fibonacci_sphere(n: int) -> np.ndarray:
    i = np.arange(n) + 0.5
    phi = np.arccos(1.0 - 2.0 * i / n)
    th = np.pi * (1.0 + 5.0 ** 0.5) * i
    return np.stack([np.sin(phi) * np.cos(th), np.sin(phi) * np.sin(th), np.cos(phi)], axis=1)


def vdw_surface_points(symbols, coords, n_points: int, seed: int = 0,
                       scale: float = 1.4, mode: str = "retry") -> np.ndarray:
    """~uniform points on the exposed union of ``scale`` x Bondi spheres (Bohr).

    Per atom, ceil(3 n_points share) + 50 Fibonacci-sphere candidates (share:
    the atom's fraction of the total sphere area), kept when no other sphere
    covers them.  ``mode="reference"`` is the reference's point scripts
    exactly (examples/vdw_surface_esp.py:38-52, benchmarks/make_points.py:
    40-58, which use scale 1.0): one candidate pass, then ``n_points`` of them
    drawn by the seeded generator in its (unsorted) order, or all of them if
    there are fewer.  ``mode="retry"`` (the benchmark workloads) doubles the
    oversampling until there are enough candidates and keeps the drawn ones in
    candidate order.
    """
    if mode not in ("retry", "reference"):
        raise ValueError(f"mode must be 'retry' or 'reference', got {mode!r}")
    rad = np.array([scale * BONDI[s] / BOHR for s in symbols])
    share = rad ** 2 / (rad ** 2).sum()
    rng = np.random.default_rng(seed)
    over = 3.0
    while True:
        cand = []
        for a in range(len(symbols)):
            n = int(np.ceil(n_points * share[a] * over)) + 50
            p = coords[a] + rad[a] * fibonacci_sphere(n)
            d = np.linalg.norm(p[:, None, :] - coords[None, :, :], axis=2)
            cand.append(p[(d >= rad[None, :] - 1e-9).all(axis=1)])
        cand = np.concatenate(cand)
        if len(cand) >= n_points or mode == "reference":
            break
        over *= 2.0
    if mode == "reference":
        if len(cand) > n_points:
            cand = cand[rng.choice(len(cand), size=n_points, replace=False)]
        return np.ascontiguousarray(cand)
    sel = np.sort(rng.choice(len(cand), n_points, replace=False))
    return np.ascontiguousarray(cand[sel])


def cubic_grid_points(coords, n_points: int, spacing: float = 0.2, margin: float = 4.0,
                      exclude: float = 0.3, seed: int = 0) -> np.ndarray:
    """``n_points`` drawn from a cubic grid enclosing the molecule (Bohr).

    Grid spacing ``spacing``, ``margin`` Bohr around the atoms, points closer
    than ``exclude`` to a nucleus removed; a seeded subset of the grid is taken.
    """
    lo = coords.min(axis=0) - margin
    hi = coords.max(axis=0) + margin
    axes = [np.arange(lo[k], hi[k] + 0.5 * spacing, spacing) for k in range(3)]
    n_tot = int(np.prod([len(a) for a in axes]))
    rng = np.random.default_rng(seed)
    take = rng.choice(n_tot, size=min(n_tot, int(n_points * 1.2) + 64), replace=False)
    take.sort()
    nx, ny, nz = (len(a) for a in axes)
    ix, rem = np.divmod(take, ny * nz)
    iy, iz = np.divmod(rem, nz)
    pts = np.stack([axes[0][ix], axes[1][iy], axes[2][iz]], axis=1)
    d = np.linalg.norm(pts[:, None, :] - coords[None, :, :], axis=2).min(axis=1)
    pts = pts[d >= exclude]
    return np.ascontiguousarray(pts[:n_points])


def cache_dir() -> Path:
    d = Path(os.environ.get("FASTESP_B200_CACHE", Path.home() / ".cache" / "fastesp_b200"))
    d.mkdir(parents=True, exist_ok=True)
    return d


def molden_for(name: str, seed: int = 0, natom: int | None = None) -> Path:
    """Path of the MOLDEN file of a synthetic system, generated once and cached."""
    tag = f"{name}-s{seed}" + (f"-n{natom}" if natom is not None else "")
    path = cache_dir() / f"{tag}.molden.input"
    if not path.exists():
        tmp = path.with_suffix(f".tmp{os.getpid()}")
        make_system(name, seed, natom).write(tmp)
        os.replace(tmp, path)
    return path


def load_workload(name: str, n_points: int, seed: int = 0, points_seed: int = 1,
                  grid: bool = False, natom: int | None = None):
    """(wfn, basis, density, points) of a synthetic workload, via the MOLDEN reader.

    ``seed`` picks the molecule, ``points_seed`` the point sample.
    """
    wfn = read_molden(molden_for(name, seed, natom))
    basis = Basis(wfn)
    dens = basis.density_matrix_cartesian()
    if grid:
        pts = cubic_grid_points(wfn.coords, n_points, seed=points_seed)
    else:
        pts = vdw_surface_points(wfn.symbols, wfn.coords, n_points, seed=points_seed)
    return wfn, basis, dens, pts


def batch_workload(n_mol: int = 64, seed: int = 0):
    """The uneven batch: ``n_mol`` molecules with atom counts uniform in [5, 60],
    l<=2 bases, and 200-5000 surface points each (log-uniform).  Returns a list
    of (wfn, basis, density, points)."""
    rng = np.random.default_rng([seed, 4242])
    out = []
    for i in range(n_mol):
        natom = int(rng.integers(5, 61))
        npts = int(round(np.exp(rng.uniform(np.log(200.0), np.log(5000.0)))))
        out.append(load_workload("batch", npts, seed=1000 * seed + i, points_seed=i + 1,
                                 natom=natom))
    return out


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()[:16]
