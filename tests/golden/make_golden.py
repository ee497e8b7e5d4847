"""Generate the golden fixtures by running the reference (ZidongS/fastesp) itself.

    python tests/golden/make_golden.py [--reference DIR] [--quick]

DIR defaults to $FASTESP_REFERENCE, else a checkout named ``reference`` beside
this repository.

The reference's Python package is imported read-only from its checkout, and its
C++ table builder is run from ``oracle/_ref/build_pairs`` (built from the
reference sources by ``make -C oracle``).  Outputs (small .npz/.molden files)
go to this directory and are committed; the tests compare the NumPy oracle,
the host-side reader/basis and the CUDA kernels against them.  Nothing reads
the reference at test time.

Fixtures
  boys.npz            reference ``boys(m, T)`` on a (m, T) grid
  pair_types.npz      reference ``_pair_type(L)`` / ``a_table`` for L = 0..8
  prim_integrals.npz  reference ``primitive_pair_integral`` at the geometry of
                      its own quadrature test, plus s-s closed-form cases
  <sys>.molden        the synthetic MOLDEN file (small systems only)
  <sys>.npz           reference density, pair table (tol 1e-12), ESP /
                      electron / nuclear at tol 1e-12 and tol 0, and the C++
                      builder's kept-pair count and ESP (its screening rule)
  frag54_300.npz      54-atom system at 300 vdW points (the MOLDEN file is
                      regenerated from its seed; ESP at tol 1e-12 and 0)
  ref_points.npz      the reference's vdW-surface sampler
                      (examples/vdw_surface_esp.py: vdw_surface_points) on the
                      small system and the 54-atom system, several seeds
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("FASTESP_REFERENCE")
                    or str(ROOT.parent / "reference"))
    ap.add_argument("--quick", action="store_true", help="skip the 54-atom fixture")
    ap.add_argument("--only", default="",
                    help="comma list: boys,pair_types,prim,systems,frag54,points")
    a = ap.parse_args()
    sys.path.insert(0, a.reference)
    sys.path.insert(0, str(ROOT))
    import fastesp as R                              # the reference package
    from fastesp import esp as Resp, ints as Rints
    from fastesp_b200 import synth

    only = set(filter(None, a.only.split(",")))
    want = (lambda k: not only or k in only)
    build_pairs = ROOT / "oracle" / "_ref" / "build_pairs"
    if not build_pairs.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "_ref/build_pairs",
                        f"REF={a.reference}"], check=True)

    # ---- Boys (reference values, plus 40-digit values of the same function) --
    if want("boys"):
        import mpmath as mp
        mp.mp.dps = 40
        T = np.concatenate([[0.0, 1e-14, 1e-12, 1e-10, 1e-8], np.logspace(-6, 5, 221),
                            np.linspace(0.0, 60.0, 241)[1:], [0.1, 1.0, 5.0, 30.0, 1e4]])
        ms = np.arange(17)
        F = np.array([[Rints.boys(int(m), t) for t in T] for m in ms])

        def exact(m, t):
            if t == 0.0:
                return 1.0 / (2 * m + 1)
            a_ = mp.mpf(m) + mp.mpf(1) / 2
            return float(mp.gammainc(a_, 0, mp.mpf(t)) / (2 * mp.power(mp.mpf(t), a_)))
        F_exact = np.array([[exact(int(m), float(t)) for t in T] for m in ms[:10]])
        np.savez_compressed(HERE / "boys.npz", T=T, m=ms, F=F, F_exact=F_exact)
    # ---- the reference's vdW-surface sampler ---------------------------------
    if want("points"):
        import importlib.util
        spec = importlib.util.spec_from_file_location(
            "ref_vdw_surface_esp", Path(a.reference) / "examples" / "vdw_surface_esp.py")
        ex = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(ex)
        out = {}
        with tempfile.TemporaryDirectory() as td:
            cases = (("small", synth.make_system("small", 0), ((300, 0), (300, 5))),
                     ("frag54", synth.make_system("frag54", 0), ((3000, 0), (2000, 20260909))))
            for tag, sysm, runs in cases:
                wfn = R.read_molden(sysm.write(Path(td) / f"{tag}.molden"))
                for n, seed in runs:
                    out[f"{tag}_{n}_{seed}"] = ex.vdw_surface_points(wfn, n, seed=seed)
        np.savez_compressed(HERE / "ref_points.npz", **out)
        print("ref_points:", {k: v.shape for k, v in out.items()})
    if not any(want(k) for k in ("pair_types", "prim", "systems", "frag54")):
        return 0

    # ---- per-L contraction tables -------------------------------------------
    d = {"a8": Rints.a_table(8)}
    for L in range(9):
        M0, w, abs_t, mono, mvals, npow = Resp._pair_type(L)
        d.update({f"M0_{L}": M0, f"w_{L}": w, f"abst_{L}": abs_t, f"mono_{L}": mono,
                  f"m_{L}": mvals})
    np.savez_compressed(HERE / "pair_types.npz", **d)

    # ---- single-pair integrals ----------------------------------------------
    A = np.array([0.3, -0.4, 0.2])
    B = A + np.array([1.1, 0.5, -0.6])
    C = np.array([0.1, 1.6, 1.1])
    cases = [((0, 0, 0), (0, 0, 0)), ((1, 0, 0), (0, 0, 0)), ((0, 1, 0), (1, 0, 0)),
             ((1, 1, 0), (0, 0, 1)), ((2, 0, 0), (0, 1, 0)), ((1, 0, 0), (0, 0, 2)),
             ((2, 1, 0), (1, 0, 0)), ((2, 0, 0), (2, 0, 0)), ((3, 0, 0), (1, 1, 0)),
             ((2, 1, 0), (2, 1, 0)), ((3, 2, 0), (2, 1, 0)), ((3, 3, 3), (3, 3, 3))]
    vals = [Rints.primitive_pair_integral(0.45, A, la, 0.72, B, lb, C) for la, lb in cases]
    rng = np.random.default_rng(0)
    ss = []
    for _ in range(8):
        A2 = rng.normal(0, 1, 3)
        B2 = A2 + rng.normal(0, 1, 3)
        C2 = rng.normal(0, 3, 3)
        al = float(np.exp(rng.uniform(-2, 2.5)))
        be = float(np.exp(rng.uniform(-2, 2.5)))
        ss.append(np.concatenate([A2, B2, C2, [al, be,
                                  Rints.primitive_pair_integral(al, A2, (0, 0, 0), be, B2,
                                                                (0, 0, 0), C2)]]))
    np.savez(HERE / "prim_integrals.npz", A=A, B=B, C=C, alpha=0.45, beta=0.72,
             la=np.array([c[0] for c in cases]), lb=np.array([c[1] for c in cases]),
             value=np.array(vals), ss=np.array(ss))

    # ---- whole-pipeline fixtures ----------------------------------------------
    def pipeline(tag, wfn_path, npts, seed, keep_table):
        t0 = time.time()
        wfn = R.read_molden(wfn_path)
        basis = R.Basis(wfn)
        P = basis.density_matrix_cartesian()
        S = R.overlap_matrix(basis) if basis.n <= 400 else None
        pts = synth.vdw_surface_points(wfn.symbols, wfn.coords, npts, seed=seed)
        out = {"points": pts, "nelec": wfn.nelec}
        if keep_table:
            out["density"] = P
            out["overlap"] = S
        for tol, key in ((1e-12, "t12"), (0.0, "t0")):
            tab = R.build_table(wfn, basis, P, pts, tol=tol)
            out[f"npairs_{key}"] = tab.n_pairs
            out[f"electron_{key}"] = tab.electron()
            out[f"nuclear_{key}"] = tab.nuclear()
            out[f"esp_{key}"] = tab.esp()
            if keep_table and key == "t12":
                for k in ("pp_exp", "pp_cx", "pp_cy", "pp_cz", "pp_K", "pp_nt", "pp_off",
                          "pp_nmono", "pp_monooff", "mo_parent", "mo_axis", "tm_aidx",
                          "tm_m", "tm_g"):
                    out[f"tab_{k}"] = getattr(tab, k)
        # the reference C++ builder (its own screening rule), evaluated by the
        # reference NumPy evaluator: what ``fastesp esp --backend cpp`` does
        with tempfile.TemporaryDirectory() as td:
            bb, pb = Path(td) / "basis.bin", Path(td) / "pairs.bin"
            R.write_basis_payload(bb, R.basis_payload(wfn, basis, P, pts))
            r = subprocess.run([str(build_pairs), str(bb), str(pb), "1e-12"],
                               capture_output=True, text=True, check=True)
            ct = R.PairTable.read(pb)
            out["native_npairs_t12"] = ct.n_pairs
            out["native_esp_t12"] = ct.esp()
            out["native_sumrule"] = float(r.stderr.split("Tr(P S) =")[1].split()[0])
        np.savez_compressed(HERE / f"{tag}.npz", **{k: v for k, v in out.items()
                                                    if v is not None})
        print(f"{tag}: {out['npairs_t12']} pairs (native {out['native_npairs_t12']}), "
              f"{time.time() - t0:.1f} s")

    for tag, name, nat, npts in (("small", "small", None, 300), ("tz6", "tz", 6, 200)):
        path = HERE / f"{tag}.molden"
        synth.make_system(name, 0, nat).write(path)
        pipeline(tag, path, npts, seed=1, keep_table=True)
    if not a.quick:
        with tempfile.TemporaryDirectory() as td:
            path = synth.make_system("frag54", 0).write(Path(td) / "frag54.molden")
            pipeline("frag54_300", path, 300, seed=1, keep_table=False)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
