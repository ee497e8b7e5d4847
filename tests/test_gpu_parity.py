"""CUDA path vs the reference: golden fixtures, the oracle, and size-independent properties.

Tolerances (FP64 path): 1e-12 a.u. on the small fixtures, 1e-10 a.u. on the
54-atom system (the parity bar), exact equality where the arithmetic is the
same (kept-pair sets, determinism, point permutations).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle.esp_oracle as O
from fastesp_b200 import _lib, build_table, primitive_pair_integral
from fastesp_b200 import hermite as H
from fastesp_b200 import synth
from fastesp_b200.ints import boys
from fastesp_b200.molden import Z_OF
from fastesp_b200.table import PairTable

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _device_status_clean():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    _lib.status(clear=True)
    yield
    assert _lib.status(clear=True) == 0, "a kernel reported a device-side failure"


def test_boys_gpu_matches_reference(golden):
    """Against 40-digit values: 4e-15 relative.  Against the reference's own
    hypergeometric values: within that function's own error plus 4e-15."""
    g = golden("boys")
    for m in range(10):
        got = boys(m, g["T"])
        ex = g["F_exact"][m]
        rel = np.abs(got - ex) / np.abs(ex)
        assert rel.max() < 4e-15, (m, g["T"][np.argmax(rel)], rel.max())
        ref = g["F"][m]
        assert (np.abs(got - ref) <= np.abs(ref - ex) + 4e-15 * np.abs(ex)).all()


def _asym_thresholds():
    import re
    from pathlib import Path
    hdr = (Path(__file__).resolve().parents[1] / "fastesp_b200" / "csrc" / "classes_gen.cuh").read_text()
    m = re.search(r"fe_boys_asym_T\[FE_MMAX \+ 1\] = \{([^}]*)\}", hdr)
    return [float(v) for v in m.group(1).split(",")]


def test_boys_gpu_regime_edges():
    """Continuity across the tabulated / upward / asymptotic switches."""
    th = _asym_thresholds()
    for M in range(10):
        for e in (12.0, th[M]):
            T = np.array([np.nextafter(e, 0.0), e, np.nextafter(e, 1e9)])
            got = np.stack([boys(m, T) for m in range(M + 1)])
            ref = np.stack([O.boys(m, T) for m in range(M + 1)])
            assert (np.abs(got - ref) / ref).max() < 4e-15 * (1 + M), (M, e)


def _class_order(tab_arrays):
    """Reference-order flat table -> per class the row indices (within-class order kept)."""
    nt = tab_arrays["pp_nt"]
    by_nt = {H.n_terms(L): L for L in range(9)}
    cls = np.array([by_nt[int(t)] for t in nt])
    return cls


@pytest.mark.parametrize("tag", ["small", "tz6"])
def test_build_matches_reference_table(tag, request):
    wfn, basis, P, g = request.getfixturevalue(f"{tag}_system")
    tab = build_table(wfn, basis, g["density"], g["points"], tol=1e-12)
    assert tab.n_pairs == int(g["npairs_t12"])
    cls = _class_order({"pp_nt": g["tab_pp_nt"]})
    gmax = np.abs(g["tab_tm_g"]).max()
    for L in range(9):
        rows = np.nonzero(cls == L)[0]
        assert tab.counts[L] == len(rows)
        if not len(rows):
            continue
        rec = tab.records(L)
        np.testing.assert_allclose(rec[:, 0], g["tab_pp_exp"][rows], rtol=1e-15)
        np.testing.assert_allclose(rec[:, 1], g["tab_pp_cx"][rows], rtol=1e-14, atol=1e-15)
        np.testing.assert_allclose(rec[:, 2], g["tab_pp_cy"][rows], rtol=1e-14, atol=1e-15)
        np.testing.assert_allclose(rec[:, 3], g["tab_pp_cz"][rows], rtol=1e-14, atol=1e-15)
        np.testing.assert_allclose(rec[:, 4], g["tab_pp_K"][rows], rtol=1e-13)
        nt = H.n_terms(L)
        off = g["tab_pp_off"][rows][:, None] + np.arange(nt)[None, :]
        np.testing.assert_allclose(tab.coefficients(L), g["tab_tm_g"][off], rtol=0, atol=1e-13 * gmax)


@pytest.mark.parametrize("tag", ["small", "tz6"])
@pytest.mark.parametrize("tol,key", [(1e-12, "t12"), (0.0, "t0")])
def test_esp_matches_reference_small(tag, tol, key, request):
    wfn, basis, P, g = request.getfixturevalue(f"{tag}_system")
    tab = build_table(wfn, basis, g["density"], g["points"], tol=tol)
    assert tab.n_pairs == int(g[f"npairs_{key}"])
    np.testing.assert_allclose(tab.esp(), g[f"esp_{key}"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(tab.electron(), g[f"electron_{key}"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(tab.nuclear(), g[f"nuclear_{key}"], rtol=1e-15, atol=0)


@pytest.mark.parametrize("tag", ["small", "tz6"])
def test_native_rule_matches_reference_builder(tag, request):
    wfn, basis, P, g = request.getfixturevalue(f"{tag}_system")
    tab = build_table(wfn, basis, g["density"], g["points"], tol=1e-12, rule="native")
    assert tab.n_pairs == int(g["native_npairs_t12"])
    np.testing.assert_allclose(tab.esp(), g["native_esp_t12"], rtol=0, atol=1e-12)
    assert tab.sum_rule == pytest.approx(float(g["native_sumrule"]), rel=1e-9)


@pytest.mark.parametrize("tol,key", [(1e-12, "t12"), (0.0, "t0")])
def test_frag54_300_matches_reference(frag54, golden, tol, key):
    """54-atom l<=3 system at the reference's own 300 points: parity bar 1e-10 a.u."""
    wfn, basis, P = frag54
    g = golden("frag54_300")
    tab = build_table(wfn, basis, P, g["points"], tol=tol)
    assert tab.n_pairs == int(g[f"npairs_{key}"])
    err = np.abs(tab.esp() - g[f"esp_{key}"]).max()
    assert err <= 1e-10, err


def test_frag54_native_rule(frag54, golden):
    wfn, basis, P = frag54
    g = golden("frag54_300")
    tab = build_table(wfn, basis, P, g["points"], tol=1e-12, rule="native")
    assert tab.n_pairs == int(g["native_npairs_t12"])
    assert np.abs(tab.esp() - g["native_esp_t12"]).max() <= 1e-10
    assert tab.sum_rule == pytest.approx(float(g["native_sumrule"]), rel=1e-9)


def test_evaluate_reference_format_table(tmp_path, tz6_system):
    """A table in the reference's pairs.bin layout, built by the oracle, evaluated on the GPU."""
    wfn, basis, P, g = tz6_system
    Z = np.array([Z_OF[s] for s in wfn.symbols])
    ot = O.build_table(wfn.shells, wfn.coords, Z, g["density"], g["points"], tol=0.0)
    ot.write(tmp_path / "pairs.bin")
    gt = PairTable.read(tmp_path / "pairs.bin")
    assert gt.n_pairs == ot.n_pairs
    np.testing.assert_allclose(gt.esp(), ot.esp(), rtol=0, atol=1e-12)
    pts2 = g["points"][::7] + 0.37
    np.testing.assert_allclose(gt.esp(pts2), ot.esp(pts2), rtol=0, atol=1e-12)
    # the imported table's FP32 records are derived on the device (fe_table_make_f32)
    np.testing.assert_allclose(gt.esp(precision="mixed"), ot.esp(), rtol=0, atol=1e-6)


def test_export_reference_format_table(tmp_path, small_system):
    wfn, basis, P, g = small_system
    tab = build_table(wfn, basis, g["density"], g["points"], tol=1e-12)
    tab.write(tmp_path / "pairs.bin")
    ot = O.OracleTable.read(tmp_path / "pairs.bin")
    assert ot.n_pairs == tab.n_pairs
    np.testing.assert_allclose(ot.esp(), g["esp_t12"], rtol=0, atol=1e-12)


def test_primitive_pair_integrals(golden):
    """The reference's quadrature-pinned cases (its tests/test_integrals.py:72-85);
    shells above g (l > 4) are outside this library's classes and must be refused."""
    g = golden("prim_integrals")
    checked = 0
    for la, lb, v in zip(g["la"], g["lb"], g["value"]):
        args = (float(g["alpha"]), g["A"], tuple(la), float(g["beta"]), g["B"], tuple(lb), g["C"])
        if max(sum(la), sum(lb)) > 4:
            with pytest.raises(_lib.FeError, match=r"l=\d+ > 4"):
                primitive_pair_integral(*args)
            continue
        assert primitive_pair_integral(*args) == pytest.approx(v, rel=1e-12, abs=1e-15)
        checked += 1
    assert checked == 10
    for row in g["ss"]:
        A, B, C, al, be, v = row[:3], row[3:6], row[6:9], row[9], row[10], row[11]
        assert primitive_pair_integral(al, A, (0, 0, 0), be, B, (0, 0, 0), C) == \
            pytest.approx(v, rel=1e-13)


def test_edge_cases(small_system):
    import torch
    wfn, basis, P, g = small_system
    tab = build_table(wfn, basis, g["density"], g["points"], tol=1e-12)
    assert tab.esp(np.zeros((0, 3))).shape == (0,)
    one = tab.esp(g["points"][:1])
    assert one.shape == (1,) and one[0] == pytest.approx(g["esp_t12"][0], abs=1e-12)
    # a device tensor stays on the device
    d = torch.as_tensor(g["points"], device="cuda")
    out = tab.esp(d)
    assert isinstance(out, torch.Tensor) and out.is_cuda
    np.testing.assert_allclose(out.cpu().numpy(), g["esp_t12"], rtol=0, atol=1e-12)
    # far field: V -> (sum Z - N_elec) / r, and the electron part -> N_elec / r
    far = np.array([[1e5, 0.0, 0.0], [0.0, -2e5, 0.0], [0.0, 0.0, 3e5]])
    tab0 = build_table(wfn, basis, g["density"], far, tol=0.0)
    r = np.linalg.norm(far - wfn.coords.mean(0), axis=1)
    nel = float(g["nelec"])
    np.testing.assert_allclose(tab0.electron(), nel / r, rtol=1e-3)
    # points with no table rows: an empty density gives the bare nuclear potential
    tz = build_table(wfn, basis, np.zeros_like(g["density"]), g["points"], tol=1e-12)
    assert tz.n_pairs == 0
    np.testing.assert_allclose(tz.esp(), g["nuclear_t12"], rtol=1e-15)


def test_zero_points_build(small_system):
    wfn, basis, P, g = small_system
    tab = build_table(wfn, basis, g["density"], np.zeros((0, 3)), tol=1e-12)
    # with nothing to screen against every pair is kept
    assert tab.n_pairs == int(g["npairs_t0"])
    np.testing.assert_allclose(tab.esp(g["points"]), g["esp_t0"], rtol=0, atol=1e-12)


# ---------------------------------------------------------------------------
# full size (the 30000-point workload): size-independent properties
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def frag54_30k(frag54):
    wfn, basis, P = frag54
    pts = synth.vdw_surface_points(wfn.symbols, wfn.coords, 30000, seed=1)
    return wfn, basis, P, pts


def test_full_size_unscreened_matches_reference_points(frag54, golden):
    """The unscreened table evaluated at the reference's 300 points reproduces its values."""
    wfn, basis, P = frag54
    g = golden("frag54_300")
    pts = synth.vdw_surface_points(wfn.symbols, wfn.coords, 30000, seed=3)
    tab = build_table(wfn, basis, P, pts, tol=0.0)
    assert np.abs(tab.esp(g["points"]) - g["esp_t0"]).max() <= 1e-10


def test_full_size_deterministic_and_permutation_invariant(frag54_30k):
    wfn, basis, P, pts = frag54_30k
    tab = build_table(wfn, basis, P, pts, tol=1e-12)
    a = tab.esp()
    b = tab.esp()
    np.testing.assert_array_equal(a, b)
    perm = np.random.default_rng(0).permutation(len(pts))
    np.testing.assert_array_equal(tab.esp(pts[perm]), a[perm])
    # a subset evaluated alone differs only by the order of its split sums
    np.testing.assert_allclose(tab.esp(pts[:300]), a[:300], rtol=0, atol=1e-11)


def test_full_size_linear_in_density(frag54_30k):
    wfn, basis, P, pts = frag54_30k
    rng = np.random.default_rng(5)
    Q = rng.normal(size=P.shape) * 1e-3
    Q = Q + Q.T
    e1 = build_table(wfn, basis, P, pts, tol=0.0).electron()
    e2 = build_table(wfn, basis, Q, pts, tol=0.0).electron()
    e12 = build_table(wfn, basis, P + Q, pts, tol=0.0).electron()
    assert np.abs(e12 - e1 - e2).max() <= 1e-10


def test_full_size_screening_changes_little(frag54_30k):
    """Screening at 1e-12 moves the answer by far less than the parity bar
    (reference tests/test_pipeline.py:167-178 at full size)."""
    wfn, basis, P, pts = frag54_30k
    full = build_table(wfn, basis, P, pts, tol=0.0).esp()
    scr = build_table(wfn, basis, P, pts, tol=1e-12).esp()
    assert np.abs(full - scr).max() < 1e-9


def test_full_size_translation_invariant(frag54_30k):
    """Shifting nuclei, basis and points together leaves V unchanged."""
    from fastesp_b200 import Basis
    from fastesp_b200.molden import Wavefunction
    wfn, basis, P, pts = frag54_30k
    shift = np.array([1.25, -0.5, 0.75])
    w2 = Wavefunction(symbols=wfn.symbols, coords=wfn.coords + shift, shells=wfn.shells,
                      mo_energy=wfn.mo_energy, mo_occ=wfn.mo_occ, mo_coeff=wfn.mo_coeff,
                      spherical=wfn.spherical)
    b2 = Basis(w2)
    sub = pts[::10]
    v1 = build_table(wfn, basis, P, sub, tol=0.0).esp()
    v2 = build_table(w2, b2, P, sub + shift, tol=0.0).esp()
    assert np.abs(v1 - v2).max() < 1e-9


# ---------------------------------------------------------------------------
# mixed precision: FP32 Boys/polynomial with FP64 routing, <= 1e-6 a.u.
# ---------------------------------------------------------------------------
MIXED_TOL = 1e-6


@pytest.mark.parametrize("tag", ["small", "tz6"])
def test_mixed_small_systems(tag, request):
    wfn, basis, P, g = request.getfixturevalue(f"{tag}_system")
    tab = build_table(wfn, basis, g["density"], g["points"], tol=1e-12)
    assert np.abs(tab.esp(precision="mixed") - g["esp_t12"]).max() <= MIXED_TOL
    assert np.abs(tab.electron(precision="mixed") - g["electron_t12"]).max() <= MIXED_TOL


def test_mixed_frag54_reference_points(frag54, golden):
    wfn, basis, P = frag54
    g = golden("frag54_300")
    tab = build_table(wfn, basis, P, g["points"], tol=1e-12)
    assert np.abs(tab.esp(precision="mixed") - g["esp_t12"]).max() <= MIXED_TOL


def test_mixed_full_size_vs_fp64(frag54_30k):
    """The 30000-point workload: max and RMS error of the mixed path against FP64."""
    wfn, basis, P, pts = frag54_30k
    tab = build_table(wfn, basis, P, pts, tol=1e-12)
    v64 = tab.esp()
    vmx, n64 = tab.esp_stats()
    err = np.abs(vmx - v64)
    print(f"mixed vs fp64: max {err.max():.3e} rms {np.sqrt((err ** 2).mean()):.3e}, "
          f"FP64-routed (pair, warp) evaluations {n64}")
    assert err.max() <= MIXED_TOL
    np.testing.assert_array_equal(tab.esp(precision="mixed"), vmx)     # deterministic


def test_mixed_routing_extremes(tz6_system):
    """tau -> 0 routes every pair to FP64 (FP64 result); a huge tau is pure FP32."""
    wfn, basis, P, g = tz6_system
    tab = build_table(wfn, basis, g["density"], g["points"], tol=1e-12)
    v64 = tab.esp()
    all64, n_all = tab.esp_stats(tau=1e-300)
    assert n_all > 0
    assert np.abs(all64 - v64).max() <= 1e-11
    none64, n_none = tab.esp_stats(tau=1e300)
    assert n_none == 0
    assert np.abs(none64 - v64).max() < 1e-3


def test_mixed_imported_table_routes_like_built(tmp_path, small_system):
    """pairs.bin carries no screening bound, but the routing bound of the mixed
    path comes from each pair's G, p and K alone: an imported table routes and
    evaluates exactly as the table it was written from."""
    wfn, basis, P, g = small_system
    tab = build_table(wfn, basis, g["density"], g["points"], tol=1e-12)
    tab.write(tmp_path / "pairs.bin")
    back = PairTable.read(tmp_path / "pairs.bin")
    vm, n_built = tab.esp_stats()
    vb, n_back = back.esp_stats()
    assert n_back == n_built
    np.testing.assert_array_equal(vb, vm)
    assert np.abs(vb - g["esp_t12"]).max() <= MIXED_TOL


@pytest.mark.parametrize("npts", [300, 30000])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_every_workspace_row_is_written(frag54, npts, prec):
    """Evaluate through the C ABI with the workspace filled with NaN: every
    partial-sum row the reduction reads must have been written by a kernel."""
    import torch
    wfn, basis, P = frag54
    pts = synth.vdw_surface_points(wfn.symbols, wfn.coords, npts, seed=7)
    pd = torch.as_tensor(pts, device="cuda")
    tab = build_table(wfn, basis, P, pts, tol=1e-12)
    L = _lib.lib()
    mode = 0 if prec == "fp64" else 1
    nb = tab.ws_bytes(npts, prec)
    ws = torch.full((nb // 8,), float("nan"), dtype=torch.float64, device="cuda")
    out = torch.full((npts,), float("nan"), dtype=torch.float64, device="cuda")
    if prec == "fp64":
        _lib.check(L.fe_esp_fp64(_lib.ptr(tab._buf), _lib.ptr(pd), npts, _lib.ptr(out),
                                 _lib.ptr(ws), nb, _lib.stream_ptr()))
    else:
        _lib.check(L.fe_esp_mixed(_lib.ptr(tab._buf), _lib.ptr(pd), npts, _lib.ptr(out),
                                  _lib.ptr(ws), nb, 0.0, None, _lib.stream_ptr()))
    got = out.cpu().numpy()
    assert np.isfinite(got).all()
    ref = tab.esp(pts, precision=prec)
    np.testing.assert_array_equal(got, ref)


def test_point_order_keeps_rows_and_fp64_bits(frag54, golden):
    """The evaluators' spatial point order (fe_point_order_bytes): the FP64 values
    are the same bit for bit with and without the order's workspace, every value
    lands in its caller's row (a permuted point set gives the permuted values,
    bit for bit in FP64), and the mixed path stays within its bound."""
    import torch
    wfn, basis, P = frag54
    g = golden("frag54_300")
    tab = build_table(wfn, basis, P, g["points"], tol=1e-12)
    n = len(g["points"])
    L = _lib.lib()
    pd = torch.as_tensor(g["points"], device="cuda")
    perm = np.random.default_rng(5).permutation(n)
    pp = torch.as_tensor(g["points"][perm], device="cuda")
    bare = int(L.fe_eval_ws_bytes(n))
    full = bare + int(L.fe_point_order_bytes(n))
    assert full > bare

    def fp64(points, nbytes):
        ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        out = torch.empty(n, dtype=torch.float64, device="cuda")
        _lib.check(L.fe_esp_fp64(_lib.ptr(tab._buf), _lib.ptr(points), n, _lib.ptr(out),
                                 _lib.ptr(ws), nbytes, _lib.stream_ptr()))
        return out.cpu().numpy()
    caller_order = fp64(pd, bare)
    spatial = fp64(pd, full)
    np.testing.assert_array_equal(spatial, caller_order)
    np.testing.assert_array_equal(fp64(pp, full), spatial[perm])
    assert np.abs(spatial - g["esp_t12"]).max() <= 1e-10
    vm = tab.esp(pp, precision="mixed").cpu().numpy()
    assert np.abs(vm - spatial[perm]).max() <= MIXED_TOL
