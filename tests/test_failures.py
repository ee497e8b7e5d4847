"""Failure paths, made without a GPU fault.

The reference's tools exit the process on bad input (fastesp/native/esp_gpu.cu:
23-31, 77-84; build_pairs.cpp:44-51).  Here every failure comes back as an
error code or a raised FeError, and the device context stays usable:

* host side (CPU): a truncated or malformed pairs.bin is refused before any
  device work;
* device side (GPU): points with NaN coordinates give NaN potentials for
  those points only, with a clean status word; a bounded wait that nothing
  completes (the library's self-test: an mbarrier with no arrivals and no
  copy in flight) gives up after a short limit, reports FE_ST_TIMEOUT and
  FE_ERR_DEVICE, and the next evaluation is correct.
"""
from __future__ import annotations

import struct

import numpy as np
import pytest

from fastesp_b200 import _lib, build_table
from fastesp_b200.table import PairTable


def _pairs_bin_from_golden(small_system, tmp_path):
    """A valid pairs.bin written from the small system's reference table."""
    from fastesp_b200.molden import Z_OF
    wfn, _, _, g = small_system
    a = {k[4:]: g[k] for k in g.files if k.startswith("tab_")}
    pts = g["points"]
    Z = np.array([Z_OF[s_] for s_ in wfn.symbols], np.float64)
    n, nt = len(a["pp_exp"]), len(a["tm_g"])
    path = tmp_path / "pairs.bin"
    with path.open("wb") as f:
        f.write(struct.pack("<8i", n, nt, len(pts), len(Z), 0, 0, 0, 0))
        for k in ("pp_exp", "pp_cx", "pp_cy", "pp_cz", "pp_K"):
            f.write(np.ascontiguousarray(a[k], np.float64).tobytes())
        for k in ("pp_nt", "pp_off", "pp_nmono", "pp_monooff", "mo_parent", "mo_axis",
                  "tm_aidx", "tm_m"):
            f.write(np.ascontiguousarray(a[k], np.int32).tobytes())
        f.write(np.ascontiguousarray(a["tm_g"], np.float64).tobytes())
        f.write(np.ascontiguousarray(pts, np.float64).tobytes())
        f.write(np.ascontiguousarray(Z, np.float64).tobytes())
        f.write(np.ascontiguousarray(wfn.coords, np.float64).tobytes())
    return path


@pytest.mark.parametrize("keep", [0, 20, 0.5, -8])
def test_truncated_pairs_bin_is_refused(small_system, tmp_path, keep):
    path = _pairs_bin_from_golden(small_system, tmp_path)
    data = path.read_bytes()
    cut = int(len(data) * keep) if isinstance(keep, float) else (keep if keep >= 0 else len(data) + keep)
    bad = tmp_path / "cut.bin"
    bad.write_bytes(data[:cut])
    with pytest.raises(_lib.FeError) as e:
        PairTable.read(bad)
    assert e.value.code == 3 and ("truncated" in str(e.value) or "shorter" in str(e.value))


def test_negative_header_count_is_refused(small_system, tmp_path):
    path = _pairs_bin_from_golden(small_system, tmp_path)
    data = bytearray(path.read_bytes())
    data[0:4] = struct.pack("<i", -5)
    bad = tmp_path / "neg.bin"
    bad.write_bytes(bytes(data))
    with pytest.raises(_lib.FeError) as e:
        PairTable.read(bad)
    assert e.value.code == 1


def test_uncut_pairs_bin_parses(small_system, tmp_path):
    """The file the truncation tests cut is complete: its host-side parse (the
    step before any device work) reads every section."""
    path = _pairs_bin_from_golden(small_system, tmp_path)
    seen = {}

    def fake_from_arrays(a, pts, Z, xyz, device=None):
        seen.update(n=len(a["pp_exp"]), nt=len(a["tm_g"]), npt=len(pts), nat=len(Z))
        return None
    orig = PairTable.from_arrays
    PairTable.from_arrays = staticmethod(fake_from_arrays)
    try:
        PairTable.read(path)
    finally:
        PairTable.from_arrays = orig
    g = small_system[3]
    assert seen == dict(n=len(g["tab_pp_exp"]), nt=len(g["tab_tm_g"]), npt=len(g["points"]),
                        nat=len(small_system[0].symbols))


@pytest.mark.gpu
def test_nan_points_give_nan_values_and_clean_status(small_system):
    import torch
    wfn, basis, P, g = small_system
    pts = np.array(g["points"], np.float64)
    tab = build_table(wfn, basis, P, pts, tol=1e-12)
    want = tab.esp(pts)
    bad = pts.copy()
    rows = [0, 7, len(pts) - 1]
    bad[rows[0], 0] = np.nan
    bad[rows[1], :] = np.nan
    bad[rows[2], 2] = np.nan
    _lib.status(clear=True)
    for precision in ("fp64", "mixed"):
        got = tab.esp(torch.as_tensor(bad, device="cuda"), precision=precision).cpu().numpy()
        assert np.isnan(got[rows]).all(), precision
        ok = np.setdiff1d(np.arange(len(pts)), rows)
        tol = 1e-12 if precision == "fp64" else 1e-6
        assert np.abs(got[ok] - want[ok]).max() <= tol, precision
    assert _lib.status(clear=True) == 0


@pytest.mark.gpu
def test_bounded_wait_gives_up_and_context_survives(small_system):
    import torch
    L = _lib.lib()
    _lib.status(clear=True)
    done = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.fe_wait_selftest(2_000_000, _lib.ptr(done), _lib.stream_ptr())   # ~1 ms of SM clock
    assert rc == 5, L.fe_last_error()                                        # FE_ERR_DEVICE
    assert b"gave up" in L.fe_last_error()
    assert int(done.item()) == 2
    assert _lib.status(clear=True) & 1                                       # FE_ST_TIMEOUT
    assert _lib.status(clear=True) == 0
    # the context is intact: a normal evaluation still gives the reference values
    wfn, basis, P, g = small_system
    tab = build_table(wfn, basis, P, g["points"], tol=1e-12)
    np.testing.assert_allclose(tab.esp(), g["esp_t12"], rtol=0, atol=1e-12)
    assert _lib.status(clear=True) == 0
