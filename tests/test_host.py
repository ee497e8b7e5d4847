"""Host-side pieces: MOLDEN reader, basis/density, Hermite tables, C ABI loading, planning."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from fastesp_b200 import Basis, basis_payload, cart_order, overlap_matrix, read_molden
from fastesp_b200 import _lib, hermite as H, synth
from fastesp_b200.basis import cartesian_overlap_block, pure_to_cartesian

ROOT = Path(__file__).resolve().parents[1]


def test_spherical_transform_is_orthonormal():
    """T S T^T = 1 for l <= 4 (reference tests/test_pipeline.py:82-86)."""
    for l in range(5):
        T = pure_to_cartesian(l)
        S = cartesian_overlap_block(l)
        assert np.abs(T @ S @ T.T - np.eye(2 * l + 1)).max() < 1e-14


@pytest.mark.parametrize("tag", ["small", "tz6"])
def test_density_and_overlap_match_reference(tag, request):
    wfn, basis, P, g = request.getfixturevalue(f"{tag}_system")
    np.testing.assert_allclose(P, g["density"], rtol=0, atol=1e-13 * np.abs(g["density"]).max())
    S = overlap_matrix(basis)
    np.testing.assert_allclose(S, g["overlap"], rtol=0, atol=1e-13)
    # Tr(P S) = N_elec (reference tests/test_pipeline.py:102-111)
    assert float((P * S).sum()) == pytest.approx(float(g["nelec"]), abs=1e-8)


def test_mos_orthonormal_in_basis_metric():
    sysm = synth.make_system("small", 3)
    b = Basis(sysm.wavefunction())
    t = b.block_transform()
    s = t.T @ overlap_matrix(b) @ t
    c = sysm.mo_coeff
    assert np.abs(c.T @ s @ c - np.eye(c.shape[1])).max() < 1e-9


def test_hermite_tables_match_reference(golden):
    g = golden("pair_types")
    np.testing.assert_array_equal(H.a_table(8), g["a8"])
    for L in range(9):
        keys, rows = H.class_terms(L)
        T = L + 1
        M0 = np.zeros((len(keys), T ** 3))
        for k, row in enumerate(rows):
            for (tx, ty, tz), c in row:
                M0[k, (tx * T + ty) * T + tz] = c
        np.testing.assert_array_equal(M0, g[f"M0_{L}"])
        np.testing.assert_array_equal(np.array([k[:3] for k in keys]), g[f"mono_{L}"])


def test_reader_parses_flags_and_counts(small_system):
    wfn, basis, P, g = small_system
    assert wfn.spherical[2] and wfn.spherical[3]
    assert wfn.nelec == pytest.approx(float(g["nelec"]))
    assert basis.n == sum(len(cart_order(sh.l)) for sh in wfn.shells)


def _header_functions():
    txt = (ROOT / "include" / "fastesp_b200.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(fe_[a-z0-9_]+)\s*\(", txt)))


def test_library_loads_and_exports_header_symbols():
    lib = _lib.lib()
    names = _header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(_lib.exported_symbols())
    assert lib.fe_version() >= 100


def test_plan_sizes_without_gpu():
    wfn, basis, P, pts = synth.load_workload("small", 50, seed=1)
    pl = basis_payload(wfn, basis, P, pts)
    keep = {k: np.ascontiguousarray(pl[k], np.int32)
            for k in ("fn_atom", "fn_nprim", "fn_off", "fn_lx", "fn_ly", "fn_lz", "fn_shell")}
    keep.update({k: np.ascontiguousarray(pl[k], np.float64) for k in ("fc", "pexp", "pcoef", "Z", "xyz")})
    b = _lib.FeBasis(pl["n_func"], pl["n_prim"], pl["n_atoms"],
                     *(keep[k].ctypes.data for k in ("fn_atom", "fn_nprim", "fn_off", "fn_lx", "fn_ly",
                                                     "fn_lz", "fn_shell", "fc", "pexp", "pcoef", "Z", "xyz")))
    h = C.c_void_p()
    _lib.check(_lib.lib().fe_plan_create(C.byref(b), C.byref(h)))
    s = _lib.FeSizes()
    _lib.check(_lib.lib().fe_plan_sizes(h, C.byref(s)))
    ns = len(wfn.shells)
    assert s.n_shell == ns and s.n_shell_pair == ns * (ns + 1) // 2
    nprim = [len(sh.exps) for sh in wfn.shells]
    tot = sum(nprim[i] * nprim[j] for i in range(ns) for j in range(i, ns))
    assert s.n_work == tot == sum(s.cap)
    _lib.lib().fe_plan_destroy(h)


def test_plan_rejects_bad_basis():
    wfn, basis, P, pts = synth.load_workload("small", 10, seed=1)
    pl = basis_payload(wfn, basis, P, pts)
    pl["fn_shell"] = np.arange(basis.n, dtype=np.int32)      # every function its own shell
    keep = {k: np.ascontiguousarray(pl[k], np.int32)
            for k in ("fn_atom", "fn_nprim", "fn_off", "fn_lx", "fn_ly", "fn_lz", "fn_shell")}
    keep.update({k: np.ascontiguousarray(pl[k], np.float64) for k in ("fc", "pexp", "pcoef", "Z", "xyz")})
    b = _lib.FeBasis(pl["n_func"], pl["n_prim"], pl["n_atoms"],
                     *(keep[k].ctypes.data for k in ("fn_atom", "fn_nprim", "fn_off", "fn_lx", "fn_ly",
                                                     "fn_lz", "fn_shell", "fc", "pexp", "pcoef", "Z", "xyz")))
    h = C.c_void_p()
    rc = _lib.lib().fe_plan_create(C.byref(b), C.byref(h))
    assert rc == 1
    assert b"functions" in _lib.lib().fe_last_error()


def test_table_layout_is_aligned():
    cap = (C.c_int * 9)(*[7, 0, 3, 1, 0, 0, 2, 0, 0])
    o64 = (C.c_size_t * 9)()
    o32 = (C.c_size_t * 9)()
    oa = C.c_size_t()
    _lib.check(_lib.lib().fe_table_offsets(cap, 5, o64, o32, C.byref(oa)))
    assert all(v % 256 == 0 for v in list(o64) + list(o32) + [oa.value])
    assert _lib.lib().fe_table_bytes(cap, 5) >= oa.value + 5 * 32


def test_basis_payload_file(tmp_path, small_system):
    from fastesp_b200 import write_basis_payload
    wfn, basis, P, g = small_system
    pl = basis_payload(wfn, basis, P, g["points"])
    write_basis_payload(tmp_path / "basis.bin", pl)
    raw = (tmp_path / "basis.bin").read_bytes()
    n = pl["n_func"]
    expect = 32 + 7 * 4 * n + 8 * (3 * n + 2 * pl["n_prim"] + n * n + 3 * len(g["points"])
                                  + 4 * pl["n_atoms"])
    assert len(raw) == expect


def test_synthetic_workload_shapes():
    s = synth.make_system("frag54", 0)
    b = Basis(s.wavefunction())
    assert len(s.symbols) == 54 and sorted(set(s.symbols)) == ["C", "H", "N", "O"]
    assert 1550 <= b.n <= 1750
    assert 1950 <= sum(len(e) for e in b.exps) <= 2200
    assert max(sh.l for sh in s.shells) == 3
    pts = synth.vdw_surface_points(s.symbols, s.coords, 500, seed=2)
    rad = np.array([1.4 * synth.BONDI[x] / 0.529177210903 for x in s.symbols])
    d = np.linalg.norm(pts[:, None, :] - s.coords[None], axis=2)
    assert (d >= rad[None, :] - 1e-9).all()
    assert np.isclose(d / rad[None, :], 1.0, atol=1e-9).any(axis=1).all()


def test_generated_adjoint_chunks_partition_terms():
    """The adjoint moment chunks cover every term once, in order, never split a
    monomial's terms, and keep at most MOM_CHUNK accumulators."""
    import importlib.util
    from pathlib import Path
    from fastesp_b200 import hermite as H
    spec = importlib.util.spec_from_file_location(
        "gen_classes", Path(__file__).resolve().parents[1] / "fastesp_b200" / "csrc" / "gen_classes.py")
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    for L in range(9):
        keys, _ = H.class_terms(L)
        spans = gen.mom_chunks(L)
        assert spans[0][0] == 0 and spans[-1][1] == len(keys)
        for (a0, b0), (a1, b1) in zip(spans, spans[1:]):
            assert b0 == a1
        for a, b in spans:
            assert 0 < b - a <= gen.MOM_CHUNK
            if a > 0:
                assert keys[a][:3] != keys[a - 1][:3]


def test_record_strides_are_16_byte_multiples():
    from fastesp_b200 import hermite as H
    for L in range(9):
        nt = H.n_terms(L)
        assert H.record_stride(L) * 8 % 16 == 0 and H.record_stride(L) >= 6 + nt
        assert H.record_stride_f32(L) * 4 % 16 == 0 and H.record_stride_f32(L) >= 12 + 2 * nt + L + 1


def _gen_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "gen_classes", Path(__file__).resolve().parents[1] / "fastesp_b200" / "csrc" / "gen_classes.py")
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    return gen


def test_mixed_routing_bound_holds(tz6_system):
    """The mixed path's routing bound sum_n b_n / |R|^(n+1) (constants from the
    generator, b_n as the table build forms them) is never below the exact
    K sum_k |G_k R^a F_m(p R^2)| of a pair, near or far, on every class."""
    import oracle.esp_oracle as O
    gen = _gen_module()
    wfn, basis, P, g = tz6_system
    pp = O.primitive_pairs(wfn.shells, wfn.coords, g["density"])
    rng = np.random.default_rng(3)
    pts = np.asarray(g["points"], float)
    worst = 0.0
    for L in sorted(set(int(v) for v in pp["L"])):
        keys, _ = H.class_terms(L)
        _, _, _, mono, mvals, _ = O.pair_type(L)
        assert [tuple(k) for k in keys] == [(*map(int, a), int(m)) for a, m in zip(mono, mvals)]
        rc = gen.route_constants(L)
        order = gen.consumption_order(L)
        idx = np.nonzero(pp["L"] == L)[0]
        for i in rng.choice(idx, min(len(idx), 200), replace=False):
            p, K, G = pp["p"][i], pp["K"][i], np.asarray(pp["G"][i])
            b = np.zeros(L + 1)
            for j, k in enumerate(order):
                n, m, c = rc[j]
                b[n] += abs(G[k]) * c * p ** -(m + 0.5)
            b *= K
            for s in (1.0, 0.3, 0.05):
                R = (pts[rng.integers(len(pts))] - pp["P"][i]) * s
                r = float(np.linalg.norm(R))
                F = [O.boys(int(m), np.array([p * r * r]))[0] for m in mvals]
                exact = K * np.sum(np.abs(G) * np.abs(np.prod(R[None, :] ** mono, 1)) * F)
                bound = np.sum(b * r ** -(np.arange(L + 1) + 1.0))
                worst = max(worst, exact / bound)
    assert 0.0 < worst <= 1.0 + 1e-12, worst


def test_molden_reader_fast_and_fallback_paths_agree(tmp_path):
    """Fortran D exponents, an extra field on a row and whitespace-only lines
    (the line-by-line path) give the same wavefunction as the plain file."""
    import numpy as np
    from pathlib import Path
    from fastesp_b200 import read_molden
    src = Path(__file__).resolve().parent / "golden" / "small.molden"
    w0 = read_molden(src)
    lines = src.read_text().splitlines()
    out, in_mo = [], False
    for ln in lines:
        if ln.strip().startswith("[MO]"):
            in_mo = True
        f = ln.split()
        if in_mo and len(f) == 2 and f[0].isdigit():
            ln = f"{f[0]} {float(f[1]):.12E}".replace("E", "D")
        out.append(ln)
    # one row with three fields (first and last are used) and a blank-with-spaces line
    for k, ln in enumerate(out):
        f = ln.split()
        if len(f) == 2 and "D" in f[1]:
            out[k] = f"{f[0]} x {f[1]}"
            out.insert(k + 1, "    ")
            break
    p = tmp_path / "variant.molden"
    p.write_text("\n".join(out) + "\n")
    w1 = read_molden(p)
    np.testing.assert_array_equal(w1.mo_occ, w0.mo_occ)
    np.testing.assert_allclose(w1.mo_coeff, w0.mo_coeff, rtol=1e-12, atol=0)


def _ref_sampler_cases(golden, tmp_path):
    from fastesp_b200 import read_molden
    g = golden("ref_points")
    for key in g.files:
        tag, n, seed = key.split("_")
        wfn = read_molden(synth.make_system(tag, 0).write(tmp_path / f"{tag}.molden"))
        yield wfn, int(n), int(seed), g[key]


def test_host_sampler_reproduces_reference_sampler(golden, tmp_path):
    """mode="reference" at 1.0x radii draws the reference sampler's points
    (examples/vdw_surface_esp.py:38-52) for the same seed, in its order."""
    for wfn, n, seed, want in _ref_sampler_cases(golden, tmp_path):
        got = synth.vdw_surface_points(wfn.symbols, wfn.coords, n, seed=seed, scale=1.0,
                                       mode="reference")
        assert got.shape == want.shape
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)
