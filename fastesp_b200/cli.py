"""Command line interface, mirroring ``fastesp`` (fastesp/cli.py:292-320).

    python -m fastesp_b200 esp WF.molden --points pts_bohr.txt -o esp.txt
    python -m fastesp_b200 build-native     # compile libfastesp_b200.so for sm_100a
    python -m fastesp_b200 selftest         # analytic integrals vs an independent quadrature

``esp`` keeps the reference's flags and its output file format (a count line,
then `` x y z V`` rows written with %20.12f x3 and %22.14e, fastesp/cli.py:193-199).
Its only backend is the CUDA path of this package: ``--backend auto`` and
``--backend cuda`` select it, and ``cpp`` / ``numpy`` (the reference's CPU
paths) are refused with a message rather than emulated.  ``--precision mixed``
selects the FP32/FP64 evaluator.
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

from . import __version__

BOHR_PER_ANGSTROM = 1.0 / 0.529177210903
HARTREE_EV = 27.211386245988


def read_points(path, angstrom: bool = False) -> np.ndarray:
    """Rows of at least three numbers; other lines are skipped (fastesp/cli.py:211-226)."""
    rows = []
    for line in Path(path).read_text().splitlines():
        f = line.split()
        if len(f) < 3:
            continue
        try:
            rows.append([float(x) for x in f[:3]])
        except ValueError:
            continue
    pts = np.asarray(rows, float).reshape(-1, 3)
    if len(pts) == 0:
        raise SystemExit(f"fastesp_b200: no points in {path}")
    return pts * BOHR_PER_ANGSTROM if angstrom else pts


def write_esp(path, pts, esp) -> None:
    with Path(path).open("w") as f:
        f.write(f"{len(pts)}\n")
        for (x, y, z), v in zip(pts, esp):
            f.write(f" {x:20.12f} {y:20.12f} {z:20.12f} {v:22.14e}\n")


def run_esp(molden, points_file, out_file=None, backend="auto", tol=1e-12, angstrom=False,
            precision="fp64", verbose=True) -> np.ndarray:
    if backend in ("cpp", "numpy"):
        raise SystemExit(f"fastesp_b200: backend {backend!r} is the reference's CPU path and is "
                         "not part of this package; use --backend cuda (or auto)")
    import torch
    from .basis import Basis
    from .molden import read_molden
    from .table import build_table
    if not torch.cuda.is_available():
        raise SystemExit("fastesp_b200: no CUDA device; this package runs on the GPU only")
    t0 = time.perf_counter()
    wfn = read_molden(molden)
    basis = Basis(wfn)
    density = basis.density_matrix_cartesian()
    t_load = time.perf_counter() - t0
    pts = read_points(points_file, angstrom)
    dev = torch.device("cuda", torch.cuda.current_device())
    pts_d = torch.as_tensor(pts, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    t0 = time.perf_counter()
    ev[0].record()
    table = build_table(wfn, basis, density, pts_d, tol=tol)
    ev[1].record()
    esp_d = table.esp(pts_d, precision=precision)
    ev[2].record()
    esp = esp_d.cpu().numpy()
    t_wall = time.perf_counter() - t0
    t_build = ev[0].elapsed_time(ev[1]) * 1e-3
    t_solve = ev[1].elapsed_time(ev[2]) * 1e-3
    if verbose:
        print(f"  backend      : cuda ({precision})")
        print(f"  basis        : {basis.n} Cartesian functions, "
              f"{sum(len(e) for e in basis.exps)} primitives")
        print(f"  load         : {t_load:8.3f} s")
        print(f"  pair table   : {t_build:8.4f} s  ({table.n_pairs} primitive pairs kept)")
        print(f"  ESP kernel   : {t_solve:8.4f} s")
        tot = t_build + t_solve
        print(f"  total (excl. load): {tot:.4f} s for {len(pts)} points "
              f"({1e3 * tot / len(pts):.4f} ms/point); wall incl. transfers {t_wall:.4f} s")
        print(f"  ESP range    : {esp.min() * HARTREE_EV:+.4f} .. {esp.max() * HARTREE_EV:+.4f} V")
    if out_file:
        write_esp(out_file, pts, esp)
        if verbose:
            print(f"  wrote        : {out_file}")
    return esp


def selftest(verbose: bool = True) -> int:
    """Primitive integrals <a|1/|r-C||b> of the CUDA path against an independent
    evaluation: 1/r = (2/sqrt(pi)) int_0^inf exp(-u^2 r^2) du turns the integral
    into a u-integral of a three-Gaussian product, whose x, y, z factors are
    polynomial x Gaussian and are integrated exactly by Gauss-Hermite; the
    u-integral uses Gauss-Legendre on u = s/(1-s)."""
    from .ints import primitive_pair_integral
    worst = 0.0
    A = np.array([0.3, -0.4, 0.2])
    B = A + np.array([1.1, 0.5, -0.6])
    C = np.array([0.1, 1.6, 1.1])
    al, be = 0.45, 0.72
    for la, lb in [((0, 0, 0), (0, 0, 0)), ((1, 0, 0), (0, 0, 0)), ((2, 0, 0), (0, 1, 0)),
                   ((1, 1, 0), (0, 0, 1)), ((2, 1, 1), (1, 2, 0)), ((2, 2, 0), (0, 2, 2))]:
        ana = primitive_pair_integral(al, A, la, be, B, lb, C)
        ref = u_quadrature(al, A, la, be, B, lb, C)
        rel = abs(ana - ref) / max(abs(ref), 1e-300)
        worst = max(worst, rel)
        if verbose:
            print(f"  <{la}|1/r|{lb}>  analytic {ana:+.12e}  quadrature {ref:+.12e}  rel {rel:.1e}")
    ok = worst < 1e-10
    print(f"  worst rel {worst:.1e}")
    print("  SELFTEST", "PASS" if ok else "FAIL")
    return 0 if ok else 1


def u_quadrature(al, A, la, be, B, lb, C, nu=400):
    """<a|1/|r-C||b> by the u-integral described in selftest()."""
    A, B, C = (np.asarray(v, float) for v in (A, B, C))
    s, ws = np.polynomial.legendre.leggauss(nu)
    s = 0.5 * (s + 1.0)
    ws = 0.5 * ws
    u = s / (1.0 - s)
    wu = ws / (1.0 - s) ** 2
    nh = (max(la) + max(lb)) // 2 + 2
    xh, wh = np.polynomial.hermite.hermgauss(nh)
    total = 0.0
    for uk, wk in zip(u, wu):
        u2 = uk * uk
        q = al + be + u2
        S = (al * A + be * B + u2 * C) / q
        pre = np.exp(-(al * be * np.sum((A - B) ** 2) + al * u2 * np.sum((A - C) ** 2)
                       + be * u2 * np.sum((B - C) ** 2)) / q)
        val = pre
        for ax in range(3):
            x = S[ax] + xh / np.sqrt(q)
            f = (x - A[ax]) ** la[ax] * (x - B[ax]) ** lb[ax]
            val = val * np.sum(wh * f) / np.sqrt(q)
        total += wk * val
    return 2.0 / np.sqrt(np.pi) * total


def main(argv=None) -> int:
    ap = argparse.ArgumentParser("fastesp_b200", description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--version", action="version", version=f"fastesp_b200 {__version__}")
    sub = ap.add_subparsers(dest="cmd", required=True)
    e = sub.add_parser("esp", help="electrostatic potential at a set of points")
    e.add_argument("wavefunction", type=Path, help="MOLDEN file")
    e.add_argument("--points", type=Path, required=True,
                   help="text file, one 'x y z' per line (Bohr unless --angstrom)")
    e.add_argument("-o", "--out", type=Path, default=None)
    e.add_argument("--backend", choices=["auto", "cuda", "cpp", "numpy"], default="auto")
    e.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    e.add_argument("--tol", type=float, default=1e-12,
                   help="primitive pair screening threshold in Hartree/e")
    e.add_argument("--angstrom", action="store_true", help="input points in Angstrom")
    e.add_argument("-q", "--quiet", action="store_true")
    b = sub.add_parser("build-native", help="compile libfastesp_b200.so for sm_100a")
    b.add_argument("--force", action="store_true")
    s = sub.add_parser("selftest", help="validate the analytic integrals")
    s.add_argument("-q", "--quiet", action="store_true")
    a = ap.parse_args(argv)
    if a.cmd == "esp":
        run_esp(a.wavefunction, a.points, a.out, backend=a.backend, tol=a.tol,
                angstrom=a.angstrom, precision=a.precision, verbose=not a.quiet)
        return 0
    if a.cmd == "build-native":
        from .build import build
        print(f"  library: {build(force=a.force)}")
        return 0
    return selftest(verbose=not a.quiet)


if __name__ == "__main__":
    sys.exit(main())
