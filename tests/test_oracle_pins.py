"""Pin the NumPy oracle against fixtures generated by running the reference.

The fixtures (tests/golden/) come from tests/golden/make_golden.py, which runs
ZidongS/fastesp itself; these tests check that the oracle -- the checker of
every GPU parity test -- reproduces the reference before it is trusted.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle.esp_oracle as O
from fastesp_b200.molden import Z_OF


def test_boys_matches_reference(golden):
    g = golden("boys")
    for m in g["m"]:
        np.testing.assert_array_equal(O.boys(int(m), g["T"]), g["F"][m])


def test_boys_known_values():
    """F_m(0) = 1/(2m+1); F_0 closed form; dF_m/dT = -F_(m+1) (test_integrals.py:13-27)."""
    import math
    for m in range(6):
        assert O.boys(m, 1e-14) == pytest.approx(1.0 / (2 * m + 1), rel=1e-12)
    for T in (0.1, 1.0, 5.0, 30.0):
        assert O.boys(0, T) == pytest.approx(0.5 * math.sqrt(math.pi / T) * math.erf(math.sqrt(T)),
                                             rel=1e-13)
    h = 1e-6
    num = (O.boys(1, 2.7 + h) - O.boys(1, 2.7 - h)) / (2 * h)
    assert num == pytest.approx(-O.boys(2, 2.7), rel=1e-6)


def test_pair_types_match_reference(golden):
    g = golden("pair_types")
    np.testing.assert_array_equal(O.a_table(8), g["a8"])
    for L in range(9):
        M0, w, abs_t, mono, mvals, _ = O.pair_type(L)
        np.testing.assert_array_equal(M0, g[f"M0_{L}"])
        np.testing.assert_array_equal(w, g[f"w_{L}"])
        np.testing.assert_array_equal(abs_t, g[f"abst_{L}"])
        np.testing.assert_array_equal(mono, g[f"mono_{L}"])
        np.testing.assert_array_equal(mvals, g[f"m_{L}"])


def test_primitive_integrals_match_reference(golden):
    g = golden("prim_integrals")
    for la, lb, v in zip(g["la"], g["lb"], g["value"]):
        got = O.primitive_pair_integral(float(g["alpha"]), g["A"], tuple(la), float(g["beta"]),
                                        g["B"], tuple(lb), g["C"])
        assert got == pytest.approx(v, rel=1e-13, abs=1e-16)
    for row in g["ss"]:
        A, B, C, al, be, v = row[:3], row[3:6], row[6:9], row[9], row[10], row[11]
        assert O.primitive_pair_integral(al, A, (0, 0, 0), be, B, (0, 0, 0), C) == \
            pytest.approx(v, rel=1e-13)


@pytest.mark.parametrize("tag", ["small", "tz6"])
def test_oracle_table_and_esp_match_reference(tag, request):
    wfn, basis, P, g = request.getfixturevalue(f"{tag}_system")
    np.testing.assert_allclose(P, g["density"], rtol=0, atol=1e-13 * np.abs(g["density"]).max())
    Z = np.array([Z_OF[s] for s in wfn.symbols])
    pts = g["points"]
    tab = O.build_table(wfn.shells, wfn.coords, Z, g["density"], pts, tol=1e-12)
    assert tab.n_pairs == int(g["npairs_t12"])
    for k in ("pp_nt", "pp_off", "pp_nmono", "pp_monooff", "mo_parent", "mo_axis",
              "tm_aidx", "tm_m"):
        np.testing.assert_array_equal(getattr(tab, k), g[f"tab_{k}"])
    for k in ("pp_exp", "pp_cx", "pp_cy", "pp_cz"):
        np.testing.assert_allclose(getattr(tab, k), g[f"tab_{k}"], rtol=1e-15, atol=0)
    # exp() of a batched array may take another SIMD path than the reference's
    np.testing.assert_allclose(tab.pp_K, g["tab_pp_K"], rtol=1e-14, atol=0)
    gmax = np.abs(g["tab_tm_g"]).max()
    np.testing.assert_allclose(tab.tm_g, g["tab_tm_g"], rtol=0, atol=1e-14 * gmax)
    esp = tab.esp()
    np.testing.assert_allclose(esp, g["esp_t12"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(tab.nuclear(), g["nuclear_t12"], rtol=1e-15, atol=0)
    tab0 = O.build_table(wfn.shells, wfn.coords, Z, g["density"], pts, tol=0.0)
    assert tab0.n_pairs == int(g["npairs_t0"])
    np.testing.assert_allclose(tab0.esp(), g["esp_t0"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("tag", ["small", "tz6"])
def test_oracle_native_rule_matches_reference_builder(tag, request):
    """The C++ builder's screening rule (build_pairs.cpp:311-328) as restated."""
    wfn, basis, P, g = request.getfixturevalue(f"{tag}_system")
    Z = np.array([Z_OF[s] for s in wfn.symbols])
    pp = O.primitive_pairs(wfn.shells, wfn.coords, g["density"])
    keep = O.screen_mask(pp, g["points"], 1e-12, rule="native")
    # the C++ builder also drops pairs whose G vector is all zero (none here)
    assert int(keep.sum()) == int(g["native_npairs_t12"])
    tab = O.table_from_pairs(pp, keep, g["points"], Z, wfn.coords)
    np.testing.assert_allclose(tab.esp(), g["native_esp_t12"], rtol=0, atol=1e-12)
    assert O.sum_rule(pp) == pytest.approx(float(g["native_sumrule"]), rel=1e-8)


def test_oracle_pairs_bin_roundtrip(tmp_path, small_system):
    wfn, basis, P, g = small_system
    Z = np.array([Z_OF[s] for s in wfn.symbols])
    tab = O.build_table(wfn.shells, wfn.coords, Z, P, g["points"], tol=1e-12)
    tab.write(tmp_path / "pairs.bin")
    back = O.OracleTable.read(tmp_path / "pairs.bin")
    for k in ("pp_exp", "pp_K", "tm_g", "tm_aidx", "mo_parent", "pts", "Z", "xyz"):
        np.testing.assert_array_equal(getattr(back, k), getattr(tab, k))


def test_oracle_gradient_matches_central_differences(small_system):
    """The oracle's term-by-term field formula against central differences of
    its own potential (the pin for the GPU field and adjoint tests)."""
    wfn, basis, P, g = small_system
    Z = np.array([Z_OF[s] for s in wfn.symbols])
    pts = g["points"][:12]
    tab = O.build_table(wfn.shells, wfn.coords, Z, g["density"], pts, tol=1e-12)
    an = tab.esp_gradient(pts)
    h = 1e-5
    fd = np.zeros_like(an)
    for c in range(3):
        d = np.zeros_like(pts)
        d[:, c] = h
        fd[:, c] = (tab.esp(pts + d) - tab.esp(pts - d)) / (2 * h)
    scale = np.maximum(np.abs(an), 1e-3 * np.abs(an).max())
    assert (np.abs(fd - an) / scale).max() < 1e-6
