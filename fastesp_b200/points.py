"""Evaluation points generated on the GPU.

``surface_points`` samples the exposed union of scaled Bondi spheres the way
the reference's point scripts do (benchmarks/make_points.py:22-58,
examples/vdw_surface_esp.py:38-52): per atom a share of Fibonacci-sphere
candidates proportional to its sphere area, oversampled, kept when outside
every other sphere, then a seeded subset (``mode="reference"`` draws exactly
as those scripts do; the default, used for the benchmark workloads at 1.4x
radii, retries with more candidates when too few survive and keeps the drawn
points in candidate order).  ``grid_points`` takes a seeded
subset of a cubic grid around the molecule and drops points near nuclei.

The O(N_candidates x N_atoms) candidate generation and exposure test run as
CUDA kernels (csrc/points.cuh); the seeded subset choice is NumPy on the host
(only the candidate count crosses to the host), so for a given seed the points
are those of the host generators in ``synth`` (up to the last bit of the
trigonometric functions).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .synth import BOHR, BONDI


def _dev(device):
    import torch
    return torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())


def _compact(run, ncand, device):
    import torch
    L = _lib.lib()
    ws = torch.empty(max(256, int(L.fe_points_ws_bytes(int(ncand)))), dtype=torch.uint8, device=device)
    out = torch.empty((max(int(ncand), 1), 3), dtype=torch.float64, device=device)
    cnt = torch.zeros(1, dtype=torch.int32, device=device)
    _lib.check(run(out, cnt, ws))
    return out[: int(cnt.item())]


def surface_candidates(symbols, coords, counts, slack=1e-9, scale=1.4, device=None):
    """Kept candidates (device, candidate order) of ``counts[a]`` Fibonacci
    points on the ``scale`` x Bondi sphere of each atom."""
    import torch
    dev = _dev(device)
    rad = np.array([scale * BONDI[s] / BOHR for s in symbols], np.float64)
    off = np.concatenate([[0], np.cumsum(np.asarray(counts, np.int64))]).astype(np.int64)
    xyz_d = torch.as_tensor(np.ascontiguousarray(coords, np.float64), device=dev)
    rad_d = torch.as_tensor(rad, device=dev)
    off_d = torch.as_tensor(off, device=dev)
    n = int(off[-1])
    L = _lib.lib()
    return _compact(lambda out, cnt, ws: L.fe_surface_points(
        _lib.ptr(xyz_d), _lib.ptr(rad_d), len(symbols), _lib.ptr(off_d), n, float(slack),
        _lib.ptr(out), out.shape[0], _lib.ptr(cnt), _lib.ptr(ws), ws.numel(), _lib.stream_ptr()),
        n, dev)


def surface_points(symbols, coords, n_points: int, seed: int = 0, scale: float = 1.4,
                   mode: str = "retry", device=None):
    """(n_points, 3) Bohr on the exposed ``scale`` x Bondi surface, as a CUDA tensor.

    ``mode`` as in :func:`fastesp_b200.synth.vdw_surface_points`: "reference"
    draws exactly as the reference's point scripts (one candidate pass, seeded
    draw in the generator's order, all candidates if fewer; they use scale
    1.0), "retry" as the benchmark workloads."""
    import torch
    if mode not in ("retry", "reference"):
        raise ValueError(f"mode must be 'retry' or 'reference', got {mode!r}")
    rad = np.array([scale * BONDI[s] / BOHR for s in symbols])
    share = rad ** 2 / (rad ** 2).sum()
    rng = np.random.default_rng(seed)
    over = 3.0
    while True:
        counts = [int(np.ceil(n_points * share[a] * over)) + 50 for a in range(len(symbols))]
        cand = surface_candidates(symbols, coords, counts, scale=scale, device=device)
        if cand.shape[0] >= n_points or mode == "reference":
            break
        over *= 2.0
    if mode == "reference":
        if cand.shape[0] <= n_points:
            return cand.contiguous()
        sel = rng.choice(cand.shape[0], size=n_points, replace=False)
    else:
        sel = np.sort(rng.choice(cand.shape[0], n_points, replace=False))
    return cand[torch.as_tensor(sel, device=cand.device)].contiguous()


def grid_points(coords, n_points: int, spacing: float = 0.2, margin: float = 4.0,
                exclude: float = 0.3, seed: int = 0, device=None):
    """(<= n_points, 3) Bohr: a seeded subset of the cubic grid around the
    molecule with points closer than ``exclude`` to a nucleus removed."""
    import torch
    dev = _dev(device)
    coords = np.ascontiguousarray(coords, np.float64)
    lo = coords.min(axis=0) - margin
    hi = coords.max(axis=0) + margin
    axes = [np.arange(lo[k], hi[k] + 0.5 * spacing, spacing) for k in range(3)]
    n_tot = int(np.prod([len(a) for a in axes]))
    rng = np.random.default_rng(seed)
    take = np.sort(rng.choice(n_tot, size=min(n_tot, int(n_points * 1.2) + 64), replace=False))
    xyz_d = torch.as_tensor(coords, device=dev)
    idx_d = torch.as_tensor(take.astype(np.int64), device=dev)
    ax_d = torch.as_tensor(np.concatenate(axes), device=dev)
    L = _lib.lib()
    pts = _compact(lambda out, cnt, ws: L.fe_grid_points(
        _lib.ptr(xyz_d), len(coords), float(exclude), _lib.ptr(idx_d), len(take), _lib.ptr(ax_d),
        len(axes[0]), len(axes[1]), len(axes[2]), _lib.ptr(out), out.shape[0], _lib.ptr(cnt),
        _lib.ptr(ws), ws.numel(), _lib.stream_ptr()), len(take), dev)
    return pts[:n_points].contiguous()
