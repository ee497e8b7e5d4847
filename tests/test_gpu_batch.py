"""Batched persistent launch: same values as the per-molecule FP64 path, for
uneven molecules and point counts, every tile shape, with and without the
CUDA graph."""
from __future__ import annotations

import numpy as np
import pytest

from fastesp_b200 import _lib, build_table, synth
from fastesp_b200.batch import SHAPES, BatchESP, separate_launches

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _device_status_clean():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    _lib.status(clear=True)
    yield
    assert _lib.status(clear=True) == 0, "a kernel reported a device-side failure"


@pytest.fixture(scope="module")
def batch12():
    import torch
    mols = synth.batch_workload(12, seed=1)
    tabs, pts = [], []
    for wfn, basis, P, p in mols:
        pd = torch.as_tensor(p, device="cuda")
        tabs.append(build_table(wfn, basis, torch.as_tensor(P, device="cuda"), pd))
        pts.append(pd)
    return tabs, pts


def _check(vals, tabs, pts):
    for v, t, p in zip(vals, tabs, pts):
        ref = t.esp(p)
        assert float((v - ref).abs().max()) < 1e-11


@pytest.mark.parametrize("shape", SHAPES)
def test_batch_matches_per_molecule(batch12, shape):
    tabs, pts = batch12
    b = BatchESP(tabs, pts, shape=shape, graph=False)
    _check(b.run(), tabs, pts)


def test_batch_graph_autotuned_and_deterministic(batch12):
    import torch
    tabs, pts = batch12
    b = BatchESP(tabs, pts)                       # autotuned, captured in a graph
    assert b.shape in SHAPES and b.tuning is not None
    first = [v.clone() for v in b.run()]
    _check(first, tabs, pts)
    for v, w in zip(first, b.run()):
        assert torch.equal(v, w)
    b2 = BatchESP(tabs, pts)                      # tuned shape reused
    assert b2.shape == b.shape and b2.tuning is None
    outs, run = separate_launches(tabs, pts)
    run()
    for v, w in zip(first, outs):
        assert float((v - w).abs().max()) < 1e-11


def test_batch_with_empty_and_tiny_members(batch12, small_system):
    """A molecule without points and one with fewer points than a warp."""
    import torch
    tabs, pts = batch12
    wfn, basis, P, g = small_system
    ts = build_table(wfn, basis, P, g["points"])
    extra_pts = [torch.zeros((0, 3), dtype=torch.float64, device="cuda"),
                 torch.as_tensor(g["points"][:5], device="cuda")]
    b = BatchESP(tabs[:3] + [ts, ts], pts[:3] + extra_pts, shape=(2, 4), graph=True)
    vals = b.run()
    assert vals[3].numel() == 0
    np.testing.assert_allclose(vals[4].cpu().numpy(), g["esp_t12"][:5], rtol=0, atol=1e-12)
    _check(vals[:3], tabs[:3], pts[:3])


def test_batch_rejects_unknown_pair_tile(batch12):
    tabs, pts = batch12
    with pytest.raises(_lib.FeError) as e:
        BatchESP(tabs[:2], pts[:2], shape=(2, 4, 12288), graph=False)
    assert "stage_bytes" in str(e.value)
