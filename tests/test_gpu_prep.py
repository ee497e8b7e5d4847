"""The steps before the evaluation on the GPU: density matrix and evaluation
points, against the host (NumPy) versions."""
from __future__ import annotations

import numpy as np
import pytest

from fastesp_b200 import build_table, synth
from fastesp_b200.points import grid_points, surface_points

pytestmark = pytest.mark.gpu


def test_density_on_gpu(frag54, small_system):
    for wfn, basis in ((small_system[0], small_system[1]), (frag54[0], frag54[1])):
        host = basis.density_matrix_cartesian()
        dev = basis.density_matrix_cartesian(device="cuda")
        scale = np.abs(host).max()
        assert float(np.abs(dev.cpu().numpy() - host).max()) <= 1e-13 * scale


@pytest.mark.parametrize("n,seed", [(300, 1), (30000, 1), (5000, 7)])
def test_surface_points_match_host(frag54, n, seed):
    wfn = frag54[0]
    host = synth.vdw_surface_points(wfn.symbols, wfn.coords, n, seed=seed)
    dev = surface_points(wfn.symbols, wfn.coords, n, seed=seed).cpu().numpy()
    assert dev.shape == host.shape
    assert np.abs(dev - host).max() < 1e-12


def test_grid_points_match_host(frag54):
    wfn = frag54[0]
    for n in (1000, 100000):
        host = synth.cubic_grid_points(wfn.coords, n, seed=2)
        dev = grid_points(wfn.coords, n, seed=2).cpu().numpy()
        np.testing.assert_array_equal(dev, host)


def test_gpu_prepared_inputs_give_reference_values(small_system):
    """Density and points prepared on the GPU, then build + evaluate: the
    reference's values at its own points."""
    import torch
    wfn, basis, P, g = small_system
    Pd = basis.density_matrix_cartesian(device="cuda")
    pts = torch.as_tensor(g["points"], device="cuda")
    v = build_table(wfn, basis, Pd, pts).esp(pts).cpu().numpy()
    np.testing.assert_allclose(v, g["esp_t12"], rtol=0, atol=1e-12)


def test_surface_points_match_reference_sampler(golden, tmp_path):
    """The GPU sampler in mode="reference" at 1.0x radii against the points the
    reference's own sampler (examples/vdw_surface_esp.py:38-52) drew for the
    same molecules and seeds (tests/golden/ref_points.npz)."""
    from fastesp_b200 import read_molden
    g = golden("ref_points")
    for key in g.files:
        tag, n, seed = key.split("_")
        wfn = read_molden(synth.make_system(tag, 0).write(tmp_path / f"{tag}.molden"))
        got = surface_points(wfn.symbols, wfn.coords, int(n), seed=int(seed), scale=1.0,
                             mode="reference").cpu().numpy()
        want = g[key]
        assert got.shape == want.shape, key
        assert np.abs(got - want).max() < 1e-12, key
