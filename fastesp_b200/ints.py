"""Integral primitives on the GPU (fastesp/ints.py).

* :func:`boys` -- F_m(T) from the CUDA Boys kernel (the evaluator's own code),
  same values as the reference's hypergeometric form (fastesp/ints.py:35-40).
* :func:`a_table` -- the Hermite-derivative recurrence table (ints.py:46-59).
* :func:`primitive_pair_integral` -- <g_A^a|1/|r-C||g_B^b> for bare primitives
  (ints.py:138-158), computed by building a one-pair table on the GPU and
  evaluating it: the same code path as every ESP.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .hermite import a_table  # noqa: F401  (re-exported)


def boys(m, T):
    """F_m(T) = int_0^1 t^(2m) exp(-T t^2) dt for scalar m in 0..9, array T."""
    import torch
    m = int(m)
    is_t = isinstance(T, torch.Tensor)
    dev = T.device if is_t and T.is_cuda else torch.device("cuda", torch.cuda.current_device())
    t = (T if is_t else torch.as_tensor(np.asarray(T, np.float64))).to(dev, torch.float64)
    flat = t.reshape(-1).contiguous()
    out = torch.empty((flat.numel(), m + 1), dtype=torch.float64, device=dev)
    _lib.check(_lib.lib().fe_boys_fp64(_lib.ptr(flat), flat.numel(), m, _lib.ptr(out),
                                       _lib.stream_ptr()))
    res = out[:, m].reshape(t.shape)
    if is_t:
        return res
    r = res.cpu().numpy()
    return r if r.ndim else float(r)


def boys_all(mmax, T):
    """(N, mmax+1) array of F_0..F_mmax at the N arguments T (device tensor in, out)."""
    import torch
    flat = T.reshape(-1).contiguous().to(torch.float64)
    out = torch.empty((flat.numel(), mmax + 1), dtype=torch.float64, device=flat.device)
    _lib.check(_lib.lib().fe_boys_fp64(_lib.ptr(flat), flat.numel(), int(mmax), _lib.ptr(out),
                                       _lib.stream_ptr()))
    return out


def primitive_pair_integral(alpha, A, la, beta, B, lb, C_, a_tab=None, E=None):
    """<g_A^a | 1/|r-C| | g_B^b> for bare (unnormalised) Cartesian primitives."""
    from .basis import Basis, cart_order
    from .molden import Shell, Wavefunction
    from .table import build_table
    la, lb = tuple(int(v) for v in la), tuple(int(v) for v in lb)
    lA, lB = sum(la), sum(lb)
    wfn = Wavefunction(symbols=["H", "H"], coords=np.array([A, B], np.float64),
                       shells=[Shell(0, lA, np.array([float(alpha)]), np.array([1.0])),
                               Shell(1, lB, np.array([float(beta)]), np.array([1.0]))],
                       mo_energy=np.zeros(1), mo_occ=np.zeros(1), mo_coeff=np.zeros((1, 1)))
    basis = Basis(wfn)
    dens = np.zeros((basis.n, basis.n))
    i = cart_order(lA).index(la)
    j = len(cart_order(lA)) + cart_order(lB).index(lb)
    dens[i, j] = 1.0
    C_ = np.asarray(C_, np.float64).reshape(1, 3)
    return float(build_table(wfn, basis, dens, C_, tol=0.0).electron(C_)[0])
