"""Pair table on the GPU: build, evaluation, and the reference's file formats.

Drop-in for fastesp's ``fastesp.table`` (fastesp/table.py):

* :func:`build_table` (fastesp/table.py:176-259) -- same signature; the table is
  built by the CUDA kernels and stays in device memory.  ``rule`` picks the
  screening test: ``"numpy"`` reproduces ``build_table``'s (table.py:193),
  ``"native"`` the C++ builder's (build_pairs.cpp:326-328) that
  ``fastesp esp --backend cpp/cuda`` uses.
* :class:`PairTable` -- ``esp`` / ``electron`` / ``nuclear`` (table.py:73-104)
  evaluate on the GPU; ``write`` / ``read`` speak the ``pairs.bin`` layout
  (table.py:11-23, 119-170), so tables built by the reference's C++ builder can
  be evaluated here and vice versa.
* :func:`basis_payload` / :func:`write_basis_payload` (table.py:268-316): the
  ``basis.bin`` payload, which is also exactly the C ABI's ``fe_basis``.

Arrays may be NumPy (results come back as NumPy) or CUDA torch tensors
(results stay on the device).
"""
from __future__ import annotations

import ctypes as C
import struct
from pathlib import Path

import numpy as np

from . import _lib
from . import hermite as H
from .basis import Basis, cart_order
from .molden import Z_OF, Wavefunction

HEADER_FIELDS = 8
NCLASS = _lib.NCLASS


def _torch():
    import torch
    return torch


def _device(device=None):
    torch = _torch()
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() \
            else torch.device("cuda")
    return torch.device(device)


def _to_dev(a, device, dtype=None):
    """Contiguous FP64 tensor on ``device`` (no copy if already there)."""
    torch = _torch()
    dtype = dtype or torch.float64
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(device=device,
                                                                           dtype=dtype)


def _is_torch(a) -> bool:
    try:
        import torch
        return isinstance(a, torch.Tensor)
    except ImportError:
        return False


def _gpos(L: int) -> np.ndarray:
    """Record position of every class-L term (the order the kernels read them)."""
    from .csrc.gen_classes import consumption_order
    order = consumption_order(L)
    pos = np.empty(len(order), np.int64)
    pos[np.array(order)] = np.arange(len(order))
    return pos


def _empty_bytes(n, device):
    torch = _torch()
    return torch.empty(max(int(n), 256), dtype=torch.uint8, device=device)


# ---------------------------------------------------------------------------
# basis payload (fastesp/table.py:268-316)
# ---------------------------------------------------------------------------
def _shell_ids(wfn: Wavefunction) -> np.ndarray:
    ids = []
    for sid, sh in enumerate(wfn.shells):
        ids += [sid] * len(cart_order(sh.l))
    return np.asarray(ids, np.int32)


def basis_payload(wfn: Wavefunction, basis: Basis, density, points) -> dict:
    """Flat basis/density/points arrays (fastesp/table.py:268-293)."""
    fn_nprim = np.array([len(e) for e in basis.exps], np.int32)
    return dict(
        n_func=basis.n, n_prim=int(fn_nprim.sum()), n_points=len(points),
        n_atoms=wfn.natom, max_prim=int(fn_nprim.max()) if len(fn_nprim) else 0,
        fn_atom=np.asarray(basis.atoms, np.int32), fn_nprim=fn_nprim,
        fn_off=np.concatenate([[0], np.cumsum(fn_nprim)[:-1]]).astype(np.int32),
        fn_lx=np.asarray(basis.ang_arr[:, 0], np.int32),
        fn_ly=np.asarray(basis.ang_arr[:, 1], np.int32),
        fn_lz=np.asarray(basis.ang_arr[:, 2], np.int32),
        fn_shell=_shell_ids(wfn),
        fc=np.asarray(basis.centers, np.float64).ravel(),
        pexp=np.concatenate(basis.exps).astype(np.float64) if basis.n else np.zeros(0),
        pcoef=np.concatenate(basis.coefs).astype(np.float64) if basis.n else np.zeros(0),
        dens=density, pts=points,
        Z=np.array([Z_OF[s] for s in wfn.symbols], np.float64),
        xyz=np.ascontiguousarray(wfn.coords, np.float64))


def write_basis_payload(path, payload: dict) -> None:
    """basis.bin: 8 int32 header, int32 function arrays, FP64 arrays (table.py:307-316)."""
    with Path(path).open("wb") as f:
        f.write(struct.pack("<8i", payload["n_func"], payload["n_prim"], payload["n_points"],
                            payload["n_atoms"], payload["max_prim"], 0, 0, 0))
        for k in ("fn_atom", "fn_nprim", "fn_off", "fn_lx", "fn_ly", "fn_lz", "fn_shell"):
            f.write(np.ascontiguousarray(payload[k], np.int32).tobytes())
        for k in ("fc", "pexp", "pcoef", "dens", "pts", "Z", "xyz"):
            v = payload[k]
            if _is_torch(v):
                v = v.detach().cpu().numpy()
            f.write(np.ascontiguousarray(v, np.float64).tobytes())


# ---------------------------------------------------------------------------
# Plan: basis-dependent, density- and point-independent
# ---------------------------------------------------------------------------
class Plan:
    """Shell grouping, shell-pair/primitive-pair enumeration and work lists of a
    basis, uploaded once to the device and reused by every table build."""

    def __init__(self, payload: dict, device=None):
        L = _lib.lib()
        self.device = _device(device)
        keep = {k: np.ascontiguousarray(payload[k], np.int32)
                for k in ("fn_atom", "fn_nprim", "fn_off", "fn_lx", "fn_ly", "fn_lz", "fn_shell")}
        keep.update({k: np.ascontiguousarray(payload[k], np.float64)
                     for k in ("fc", "pexp", "pcoef", "Z", "xyz")})
        self._host = keep
        b = _lib.FeBasis(payload["n_func"], payload["n_prim"], payload["n_atoms"],
                         *(keep[k].ctypes.data for k in ("fn_atom", "fn_nprim", "fn_off", "fn_lx",
                                                         "fn_ly", "fn_lz", "fn_shell", "fc",
                                                         "pexp", "pcoef", "Z", "xyz")))
        h = C.c_void_p()
        _lib.check(L.fe_plan_create(C.byref(b), C.byref(h)))
        self._h = h
        self.sizes = _lib.FeSizes()
        _lib.check(L.fe_plan_sizes(h, C.byref(self.sizes)))
        self.n_func = payload["n_func"]
        self.n_atoms = payload["n_atoms"]
        self.Z = keep["Z"]
        self.xyz = keep["xyz"].reshape(-1, 3)
        self.d_plan = _empty_bytes(self.sizes.plan_bytes, self.device)
        _lib.check(L.fe_plan_upload(h, _lib.ptr(self.d_plan), _lib.stream_ptr()))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().fe_plan_destroy(h)
            except Exception:       # interpreter shutdown: module globals already gone
                pass
            self._h = None


def plan_for(wfn: Wavefunction, basis: Basis, device=None) -> Plan:
    """The (cached) device plan of ``basis``."""
    dev = _device(device)
    cache = basis.__dict__.setdefault("_fe_plans", {})
    key = str(dev)
    if key not in cache:
        pl = basis_payload(wfn, basis, np.zeros((0, 0)), np.zeros((0, 3)))
        cache[key] = Plan(pl, dev)
    return cache[key]


# ---------------------------------------------------------------------------
# table
# ---------------------------------------------------------------------------
class PairTable:
    """Device-resident contracted pair table (layout in csrc/table.cuh).

    ``pts``, ``Z`` and ``xyz`` mirror the reference's fields: the points the
    table was screened against (the default evaluation points) and the nuclei.
    """

    def __init__(self, buf, pts, Z, xyz, device, plan=None):
        self._buf = buf
        self.pts = pts
        self.Z = np.asarray(Z, np.float64)
        self.xyz = np.asarray(xyz, np.float64).reshape(-1, 3)
        self.device = device
        self.plan = plan
        self._info = None
        self.meta = {}

    # -- header --------------------------------------------------------
    @property
    def info(self) -> _lib.FeTableInfo:
        if self._info is None:
            inf = _lib.FeTableInfo()
            _lib.check(_lib.lib().fe_table_info_get(_lib.ptr(self._buf), C.byref(inf),
                                                    _lib.stream_ptr()))
            self._info = inf
        return self._info

    @property
    def counts(self) -> list:
        return list(self.info.count)

    @property
    def n_pairs(self) -> int:
        return int(self.info.n_pairs)

    @property
    def n_terms(self) -> int:
        return int(sum(c * H.n_terms(L) for L, c in enumerate(self.counts)))

    @property
    def max_mono(self) -> int:
        return max((len(H.mono_schedule(L)[0]) for L, c in enumerate(self.counts) if c), default=0)

    @property
    def sum_rule(self) -> float:
        """Tr(P S) of the density the table was built from (build_pairs.cpp:294-296)."""
        return float(self.info.sum_rule)

    # -- evaluation ----------------------------------------------------
    def _points(self, points):
        pts = self.pts if points is None else points
        as_numpy = not _is_torch(pts)
        d = _to_dev(pts, self.device).reshape(-1, 3)
        return d, as_numpy

    def esp(self, points=None, precision: str = "fp64", tau: float = 0.0):
        """nuclear - electron in Hartree/e (fastesp/table.py:102-104).

        ``precision="mixed"`` uses the FP32/FP64 evaluator (``tau``: its FP64
        routing threshold in a.u., 0 for the default).
        """
        return self._eval(points, precision, mode=0, tau=tau)

    def electron(self, points=None, precision: str = "fp64", tau: float = 0.0):
        """int rho(r)/|r-C| dr (fastesp/table.py:73-93)."""
        return self._eval(points, precision, mode=1, tau=tau)

    def nuclear(self, points=None):
        """sum_A Z_A/|C-R_A| (fastesp/table.py:95-100)."""
        return self._eval(points, "fp64", mode=2)

    def _eval(self, points, precision, mode, tau=0.0, n64=None):
        torch = _torch()
        if precision not in ("fp64", "mixed"):
            raise ValueError(f"unknown precision {precision!r}")
        d, as_numpy = self._points(points)
        n = int(d.shape[0])
        out = torch.empty(n, dtype=torch.float64, device=self.device)
        L = _lib.lib()
        s = _lib.stream_ptr()
        if mode == 2:
            _lib.check(L.fe_nuclear_fp64(_lib.ptr(self._buf), _lib.ptr(d), n, _lib.ptr(out),
                                         None, 0, s))
        elif precision == "fp64":
            ws = _empty_bytes(_lib.ws_bytes(n, "fp64"), self.device)
            fn = L.fe_esp_fp64 if mode == 0 else L.fe_electron_fp64
            _lib.check(fn(_lib.ptr(self._buf), _lib.ptr(d), n, _lib.ptr(out), _lib.ptr(ws),
                          ws.numel(), s))
        else:
            ws = _empty_bytes(self.ws_bytes(n, "mixed"), self.device)
            fn = L.fe_esp_mixed if mode == 0 else L.fe_electron_mixed
            _lib.check(fn(_lib.ptr(self._buf), _lib.ptr(d), n, _lib.ptr(out), _lib.ptr(ws),
                          ws.numel(), float(tau), _lib.ptr(n64), s))
        return out.cpu().numpy() if as_numpy else out

    def ws_bytes(self, n_points: int, precision: str = "fp64") -> int:
        """Workspace bytes of an evaluation of ``n_points`` points with this table."""
        return _lib.ws_bytes(n_points, precision, self.info_caps())

    def esp_stats(self, points=None, tau: float = 0.0):
        """Mixed-precision ESP and the number of (pair, warp) evaluations routed to FP64."""
        torch = _torch()
        n64 = torch.zeros(1, dtype=torch.int64, device=self.device)
        v = self._eval(points, "mixed", 0, tau=tau, n64=n64)
        return v, int(n64.item())

    # -- derivatives ---------------------------------------------------
    def esp_gradient(self, points=None, weights=None):
        """(V, dV/dC) in FP64: the potential and its gradient with respect to
        the points, (n,) and (n, 3); dV/dC is minus the electric field.  With
        ``weights`` w (n,), the gradient rows are scaled by w (dL/dC for
        dL/dV = w)."""
        torch = _torch()
        d, as_numpy = self._points(points)
        n = int(d.shape[0])
        v = torch.empty(n, dtype=torch.float64, device=self.device)
        g = torch.empty((n, 3), dtype=torch.float64, device=self.device)
        w = None if weights is None else _to_dev(weights, self.device).reshape(-1)
        if w is not None and w.numel() != n:
            raise ValueError(f"weights must have {n} entries, got {w.numel()}")
        L = _lib.lib()
        ws = _empty_bytes(int(L.fe_field_ws_bytes(n)), self.device)
        _lib.check(L.fe_esp_field_fp64(_lib.ptr(self._buf), _lib.ptr(d), n, _lib.ptr(w),
                                       _lib.ptr(v), _lib.ptr(g), _lib.ptr(ws), ws.numel(),
                                       _lib.stream_ptr()))
        if as_numpy:
            return v.cpu().numpy(), g.cpu().numpy()
        return v, g

    def field(self, points=None):
        """Electric field -dV/dC (n, 3), Hartree/(e Bohr)."""
        v, g = self.esp_gradient(points)
        return -g

    def adjoint(self, points, dLdV, density: bool = True, coords: bool = True):
        """Gradients of a loss L(V) with V = esp(points) and dL/dV given:
        (dL/dP (n_func, n_func) or None, dL/dC (n, 3) or None), FP64, for the
        Cartesian density P this table was built from; the kept pair set is held
        fixed.  dL/dP needs a table built by build_table."""
        torch = _torch()
        if density and self.plan is None:
            raise ValueError("dL/dP needs a table built by build_table (imported tables "
                             "carry no pair sources)")
        d, as_numpy = self._points(points)
        n = int(d.shape[0])
        w = _to_dev(dLdV, self.device).reshape(-1)
        if w.numel() != n:
            raise ValueError(f"dL/dV must have {n} entries, got {w.numel()}")
        plan = self.plan
        L = _lib.lib()
        dP = (torch.empty((plan.n_func, plan.n_func), dtype=torch.float64, device=self.device)
              if density else None)
        dC = torch.empty((n, 3), dtype=torch.float64, device=self.device) if coords else None
        if plan is not None:
            nbytes = int(L.fe_adjoint_ws_bytes(plan._h, n))
            ws = _empty_bytes(nbytes, self.device)
            _lib.check(L.fe_esp_adjoint(plan._h, _lib.ptr(plan.d_plan), _lib.ptr(self._buf),
                                        _lib.ptr(d), n, _lib.ptr(w), _lib.ptr(dC), _lib.ptr(dP),
                                        _lib.ptr(ws), ws.numel(), _lib.stream_ptr()))
        elif coords:
            ws = _empty_bytes(int(L.fe_field_ws_bytes(n)), self.device)
            _lib.check(L.fe_esp_field_fp64(_lib.ptr(self._buf), _lib.ptr(d), n, _lib.ptr(w),
                                           None, _lib.ptr(dC), _lib.ptr(ws), ws.numel(),
                                           _lib.stream_ptr()))
        if as_numpy:
            return (None if dP is None else dP.cpu().numpy(),
                    None if dC is None else dC.cpu().numpy())
        return dP, dC

    # -- export / import (pairs.bin) -----------------------------------
    def coefficients(self, L: int) -> np.ndarray:
        """(count, nt) G coefficients of class L in the reference's term order."""
        r = self.records(L)
        pos = _gpos(L)
        return r[:, 6 + pos]

    def records(self, L: int) -> np.ndarray:
        """(count, rec64) FP64 records of class L copied to the host."""
        n = self.counts[L]
        rec = H.record_stride(L)
        off = self._offsets()[0][L]
        raw = self._buf[off:off + n * rec * 8]
        return raw.view(_torch().float64).reshape(n, rec).cpu().numpy()

    def _offsets(self):
        cap = (C.c_int * NCLASS)(*self.info_caps())
        o64 = (C.c_size_t * NCLASS)()
        o32 = (C.c_size_t * NCLASS)()
        oa = C.c_size_t()
        _lib.check(_lib.lib().fe_table_offsets(cap, len(self.Z), o64, o32, C.byref(oa)))
        return list(o64), list(o32), oa.value

    def info_caps(self) -> list:
        if self.plan is not None:
            return list(self.plan.sizes.cap)
        return self.counts

    def to_arrays(self) -> dict:
        """The table in the reference's flat layout (fastesp/table.py:40-62), class by class."""
        pp = {k: [] for k in ("pp_exp", "pp_cx", "pp_cy", "pp_cz", "pp_K", "pp_nt", "pp_off",
                              "pp_nmono", "pp_monooff", "mo_parent", "mo_axis", "tm_aidx",
                              "tm_m", "tm_g")}
        toff = moff = 0
        for L in range(NCLASS):
            n = self.counts[L]
            if n == 0:
                continue
            r = self.records(L)
            nt = H.n_terms(L)
            parent, axis, aidx = H.mono_schedule(L)
            nm = len(parent)
            pp["pp_exp"].append(r[:, 0])
            pp["pp_cx"].append(r[:, 1])
            pp["pp_cy"].append(r[:, 2])
            pp["pp_cz"].append(r[:, 3])
            pp["pp_K"].append(r[:, 4])
            pp["pp_nt"].append(np.full(n, nt, np.int32))
            pp["pp_off"].append((toff + nt * np.arange(n)).astype(np.int32))
            pp["pp_nmono"].append(np.full(n, nm, np.int32))
            pp["pp_monooff"].append((moff + nm * np.arange(n)).astype(np.int32))
            pp["mo_parent"].append(np.tile(parent, n))
            pp["mo_axis"].append(np.tile(axis, n))
            pp["tm_aidx"].append(np.tile(aidx, n))
            pp["tm_m"].append(np.tile(H.term_m(L), n))
            pp["tm_g"].append(r[:, 6 + _gpos(L)].ravel())
            toff += nt * n
            moff += nm * n
        out = {}
        for k, v in pp.items():
            dt = np.float64 if k in ("pp_exp", "pp_cx", "pp_cy", "pp_cz", "pp_K", "tm_g") else np.int32
            out[k] = np.concatenate(v).astype(dt) if v else np.zeros(0, dt)
        return out

    def write(self, path) -> None:
        """Write the table in the pairs.bin layout (fastesp/table.py:119-141)."""
        a = self.to_arrays()
        pts = self.pts.detach().cpu().numpy() if _is_torch(self.pts) else np.asarray(self.pts)
        with Path(path).open("wb") as f:
            f.write(struct.pack("<8i", len(a["pp_exp"]), len(a["tm_g"]), len(pts), len(self.Z),
                                self.max_mono, 0, 0, 0))
            for k in ("pp_exp", "pp_cx", "pp_cy", "pp_cz", "pp_K"):
                f.write(np.ascontiguousarray(a[k], np.float64).tobytes())
            for k in ("pp_nt", "pp_off", "pp_nmono", "pp_monooff", "mo_parent", "mo_axis",
                      "tm_aidx", "tm_m"):
                f.write(np.ascontiguousarray(a[k], np.int32).tobytes())
            f.write(np.ascontiguousarray(a["tm_g"], np.float64).tobytes())
            f.write(np.ascontiguousarray(pts, np.float64).tobytes())
            f.write(np.ascontiguousarray(self.Z, np.float64).tobytes())
            f.write(np.ascontiguousarray(self.xyz, np.float64).tobytes())

    @classmethod
    def read(cls, path, device=None) -> "PairTable":
        """Load a pairs.bin table (fastesp/table.py:143-170) into device memory.

        Every pair must have the term layout of its angular class (what both
        reference builders write); the class is identified by the term count.
        """
        d = Path(path).read_bytes()
        if len(d) < 4 * HEADER_FIELDS:
            raise _lib.FeError(3, f"{path}: {len(d)} bytes, shorter than the pairs.bin header")
        n, nt, npt, nat, _ = struct.unpack_from("<8i", d, 0)[:5]
        if min(n, nt, npt, nat) < 0:
            raise _lib.FeError(1, f"{path}: negative count in the pairs.bin header")
        o = 4 * HEADER_FIELDS

        def rd(dt, count):
            nonlocal o
            nb = np.dtype(dt).itemsize * count
            if o + nb > len(d):
                raise _lib.FeError(3, f"{path}: truncated pairs.bin ({len(d)} bytes; the header's "
                                      f"counts need more than {o + nb})")
            a = np.frombuffer(d, dtype=dt, count=count, offset=o)
            o += nb
            return a

        f = {k: rd(np.float64, n) for k in ("pp_exp", "pp_cx", "pp_cy", "pp_cz", "pp_K")}
        f.update({k: rd(np.int32, n) for k in ("pp_nt", "pp_off", "pp_nmono", "pp_monooff")})
        n_mono = int(f["pp_monooff"][-1]) + int(f["pp_nmono"][-1]) if n else 0
        mo_parent, mo_axis = rd(np.int32, n_mono), rd(np.int32, n_mono)
        tm_aidx, tm_m, tm_g = rd(np.int32, nt), rd(np.int32, nt), rd(np.float64, nt)
        pts = rd(np.float64, 3 * npt).reshape(npt, 3)
        Z = rd(np.float64, nat)
        xyz = rd(np.float64, 3 * nat).reshape(nat, 3)
        return cls.from_arrays(dict(f, mo_parent=mo_parent, mo_axis=mo_axis, tm_aidx=tm_aidx,
                                    tm_m=tm_m, tm_g=tm_g), pts, Z, xyz, device)

    @classmethod
    def from_arrays(cls, a: dict, pts, Z, xyz, device=None) -> "PairTable":
        torch = _torch()
        dev = _device(device)
        by_nt = {H.n_terms(L): L for L in range(NCLASS)}
        cls_of = np.array([by_nt.get(int(t), -1) for t in a["pp_nt"]], np.int64)
        if (cls_of < 0).any():
            raise ValueError("pairs.bin holds a pair whose term count matches no class")
        counts = [int((cls_of == L).sum()) for L in range(NCLASS)]
        recs = []
        for L in range(NCLASS):
            sel = np.nonzero(cls_of == L)[0]
            ntL = H.n_terms(L)
            parent, axis, aidx = H.mono_schedule(L)
            rec = np.zeros((len(sel), H.record_stride(L)))
            if len(sel):
                toff = a["pp_off"][sel][:, None] + np.arange(ntL)[None, :]
                moff = a["pp_monooff"][sel][:, None] + np.arange(len(parent))[None, :]
                if not (np.array_equal(a["tm_m"][toff], np.broadcast_to(H.term_m(L), toff.shape))
                        and np.array_equal(a["tm_aidx"][toff], np.broadcast_to(aidx, toff.shape))
                        and np.array_equal(a["mo_parent"][moff], np.broadcast_to(parent, moff.shape))
                        and np.array_equal(a["mo_axis"][moff], np.broadcast_to(axis, moff.shape))):
                    raise ValueError(f"pairs.bin class {L}: term layout differs from the class's")
                rec[:, 0] = a["pp_exp"][sel]
                rec[:, 1] = a["pp_cx"][sel]
                rec[:, 2] = a["pp_cy"][sel]
                rec[:, 3] = a["pp_cz"][sel]
                rec[:, 4] = a["pp_K"][sel]
                rec[:, 5] = np.inf          # no screening bound in pairs.bin
                rec[:, 6 + _gpos(L)] = a["tm_g"][toff]
            recs.append(rec)
        L_ = _lib.lib()
        cap = (C.c_int * NCLASS)(*counts)
        nbytes = L_.fe_table_bytes(cap, len(Z))
        buf = _empty_bytes(nbytes, dev)
        Zc = np.ascontiguousarray(Z, np.float64)
        xc = np.ascontiguousarray(xyz, np.float64)
        _lib.check(L_.fe_table_init(_lib.ptr(buf), cap, len(Zc), Zc.ctypes.data, xc.ctypes.data,
                                    _lib.stream_ptr()))
        o64 = (C.c_size_t * NCLASS)()
        _lib.check(L_.fe_table_offsets(cap, len(Zc), o64, None, None))
        for L in range(NCLASS):
            if counts[L]:
                src = torch.from_numpy(recs[L].ravel()).view(torch.uint8)
                buf[o64[L]:o64[L] + src.numel()].copy_(src)
        _lib.check(L_.fe_table_make_f32(_lib.ptr(buf), _lib.stream_ptr()))
        return cls(buf, np.asarray(pts, np.float64), Zc, xc, dev)


def build_table(wfn: Wavefunction, basis: Basis, density, points, tol: float = 1e-12,
                progress: bool = False, rule: str = "numpy", device=None) -> PairTable:
    """Build the contracted pair table on the GPU (fastesp/table.py:176-259).

    ``density``: (n_func, n_func) Cartesian density (NumPy or torch);
    ``points``: (N, 3) Bohr, used by the screen and as default evaluation points.
    """
    if rule not in _lib.RULES:
        raise ValueError(f"rule must be one of {sorted(_lib.RULES)}")
    plan = plan_for(wfn, basis, device)
    dev = plan.device
    dens = _to_dev(density, dev)
    if tuple(dens.shape) != (basis.n, basis.n):
        raise ValueError(f"density must be ({basis.n}, {basis.n}), got {tuple(dens.shape)}")
    pts_d = _to_dev(points, dev).reshape(-1, 3)
    buf = _empty_bytes(plan.sizes.table_bytes, dev)
    ws = _empty_bytes(_lib.lib().fe_build_ws_bytes(plan._h, int(pts_d.shape[0])), dev)
    _lib.check(_lib.lib().fe_table_build(plan._h, _lib.ptr(plan.d_plan), _lib.ptr(dens),
                                         _lib.ptr(pts_d), int(pts_d.shape[0]), float(tol),
                                         _lib.RULES[rule], _lib.ptr(buf), _lib.ptr(ws),
                                         ws.numel(), _lib.stream_ptr()))
    pts_keep = points if _is_torch(points) else np.asarray(points, np.float64)
    t = PairTable(buf, pts_keep, plan.Z, plan.xyz, dev, plan)
    if progress:
        print(f"  pairs kept {t.n_pairs}")
    return t


__all__ = ["PairTable", "build_table", "basis_payload", "write_basis_payload", "Plan",
           "plan_for", "Z_OF"]
