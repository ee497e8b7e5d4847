"""The allocation-free evaluator (fe_esp_fp64_noalloc).

It exists for callers that cannot allocate device memory -- a host framework
that owns the device-memory budget and lends only input and output buffers, or
a binding of the reference's table-and-points-in / potentials-out interface.
Its scratch is a static 16 MiB device array shared by all calls, so the test
checks two calls in a row against the workspace-taking fe_esp_fp64, and that a
point count whose scratch would not fit is refused.  Collected last on purpose.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from fastesp_b200 import _lib, build_table, synth

pytestmark = pytest.mark.gpu

TOL = 1e-12      # the FP64 parity tolerance of the small-system tests


@pytest.mark.parametrize("npts", [300, 30000])
def test_noalloc_matches_workspace_entry_point(npts):
    import torch
    assert torch.cuda.is_available()
    wfn, basis, P, _ = synth.load_workload("frag54", 10, seed=0)
    pts = synth.vdw_surface_points(wfn.symbols, wfn.coords, npts, seed=11)
    tab = build_table(wfn, basis, P, pts, tol=1e-12)
    L = _lib.lib()
    pd = torch.as_tensor(pts, device="cuda")
    ref = torch.empty(npts, dtype=torch.float64, device="cuda")
    ws = torch.empty(L.fe_eval_ws_bytes(npts), dtype=torch.uint8, device="cuda")
    _lib.check(L.fe_esp_fp64(_lib.ptr(tab._buf), _lib.ptr(pd), npts, _lib.ptr(ref),
                             _lib.ptr(ws), ws.numel(), _lib.stream_ptr()))
    want = ref.cpu().numpy()
    for _ in range(2):                       # the static scratch keeps the last call's data
        out = torch.full((npts,), float("nan"), dtype=torch.float64, device="cuda")
        _lib.check(L.fe_esp_fp64_noalloc(_lib.ptr(tab._buf), _lib.ptr(pd), npts, _lib.ptr(out),
                                         _lib.stream_ptr()))
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        np.testing.assert_allclose(got, want, rtol=0, atol=TOL)
    assert _lib.status(clear=True) == 0


def test_noalloc_refuses_oversized_point_counts():
    import torch
    L = _lib.lib()
    cap = L.fe_noalloc_scratch_bytes()
    n = 1
    while L.fe_eval_ws_bytes(n) <= cap:
        n *= 2
    wfn, basis, P, pts = synth.load_workload("small", 10, seed=0)
    tab = build_table(wfn, basis, P, pts, tol=1e-12)
    dummy = torch.empty(8, dtype=torch.float64, device="cuda")
    rc = L.fe_esp_fp64_noalloc(_lib.ptr(tab._buf), _lib.ptr(dummy), n, _lib.ptr(dummy),
                               _lib.stream_ptr())
    assert rc == 3                           # FE_ERR_SIZE, refused before any launch
    assert b"static array" in L.fe_last_error()
