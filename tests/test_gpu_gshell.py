"""g shells (classes L = 7, 8: the separately compiled g-class kernel
instances) through every path: FP64 against the oracle, mixed, field,
adjoint and batch."""
from __future__ import annotations

import numpy as np
import pytest

import oracle.esp_oracle as O
from fastesp_b200 import _lib, build_table, synth
from fastesp_b200.molden import Z_OF

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _device_status_clean():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    _lib.status(clear=True)
    yield
    assert _lib.status(clear=True) == 0, "a kernel reported a device-side failure"


@pytest.fixture(scope="module")
def qz():
    wfn, basis, P, pts = synth.load_workload("qz", 200, seed=0)
    assert max(s.l for s in wfn.shells) == 4
    Z = np.array([Z_OF[s] for s in wfn.symbols])
    otab = O.build_table(wfn.shells, wfn.coords, Z, P, pts, tol=1e-12)
    return wfn, basis, P, pts, otab


def test_gshell_classes_present_and_fp64_matches_oracle(qz):
    wfn, basis, P, pts, otab = qz
    tab = build_table(wfn, basis, P, pts)
    assert tab.counts[7] > 0 and tab.counts[8] > 0
    assert tab.n_pairs == otab.n_pairs
    np.testing.assert_allclose(tab.esp(pts), otab.esp(pts), rtol=0, atol=1e-10)


def test_gshell_mixed_and_field(qz):
    wfn, basis, P, pts, otab = qz
    tab = build_table(wfn, basis, P, pts)
    v64 = tab.esp(pts)
    # default routing: the mixed bar; nothing routed: plain FP32 everywhere (FP32
    # accuracy, which the routing exists to improve); everything routed: FP64
    for tau, tol in ((0.0, 1e-6), (1e9, 1e-4), (1e-9, 1e-10)):
        vm = tab.esp(pts, precision="mixed", tau=tau)
        assert np.abs(vm - v64).max() < tol, (tau, np.abs(vm - v64).max())
    _, g = tab.esp_gradient(pts)
    assert np.abs(g - otab.esp_gradient(pts)).max() < 1e-9


def test_gshell_adjoint_directional(qz):
    import torch
    wfn, basis, P, pts, _ = qz
    Pd = torch.as_tensor(P, device="cuda")
    ptd = torch.as_tensor(pts, device="cuda")
    rng = np.random.default_rng(4)
    w = torch.as_tensor(rng.normal(size=len(pts)), device="cuda")
    dP, _ = build_table(wfn, basis, Pd, ptd).adjoint(ptd, w, coords=False)
    D = rng.normal(size=P.shape)
    D = torch.as_tensor(0.5 * (D + D.T), device="cuda")
    h = 1e-5

    def lin(Q):
        return float((build_table(wfn, basis, Q, ptd).esp(ptd) * w).sum())

    fd = (lin(Pd + h * D) - lin(Pd - h * D)) / (2 * h)
    an = float((dP * D).sum())
    assert abs(fd - an) <= 1e-6 * abs(an), (fd, an)


def test_gshell_batch(qz, small_system):
    import torch
    from fastesp_b200.batch import BatchESP
    wfn, basis, P, pts, _ = qz
    t1 = build_table(wfn, basis, P, pts)
    ws, bs, Ps, g = small_system
    t2 = build_table(ws, bs, Ps, g["points"])
    pl = [torch.as_tensor(pts, device="cuda"), torch.as_tensor(g["points"], device="cuda")]
    out = BatchESP([t1, t2], pl, shape=(2, 4)).run()
    np.testing.assert_allclose(out[0].cpu().numpy(), t1.esp(pts), rtol=0, atol=1e-11)
    np.testing.assert_allclose(out[1].cpu().numpy(), g["esp_t12"], rtol=0, atol=1e-12)
