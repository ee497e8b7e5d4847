"""Field and adjoint kernels: against the oracle's analytic field and against
central finite differences (h = 1e-5, FP64) of the CUDA forward path.

Bars: the field agrees with the oracle's term-by-term derivative to 1e-9 a.u.
absolute; gradients agree with central differences to 1e-6 relative.  The loss
is quadratic in the density for a fixed kept pair set, so the central
difference in P has no truncation error and each density entry is compared on
its own.  In the points the difference quotient carries the rounding of V
(about 1e-12 a.u. on nuclear and electron parts of size 1e2) divided by 2h,
about 5e-8 at h = 1e-5, so point gradients are compared norm-wise: the largest
deviation over the sample relative to the largest gradient component.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle.esp_oracle as O
from fastesp_b200 import _lib, build_table, synth
from fastesp_b200.molden import Z_OF
from fastesp_b200.table import PairTable

pytestmark = pytest.mark.gpu

H_FD = 1e-5
REL = 1e-6


@pytest.fixture(scope="module", autouse=True)
def _device_status_clean():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    _lib.status(clear=True)
    yield
    assert _lib.status(clear=True) == 0, "a kernel reported a device-side failure"


@pytest.fixture(scope="module")
def adjoint20():
    """The 20-atom l<=2 system with 500 surface points and the loss target
    V_target = V(P + E), E symmetric Gaussian noise of sigma 1e-3."""
    import torch
    wfn, basis, P, pts = synth.load_workload("adjoint20", 500, seed=0)
    rng = np.random.default_rng(7)
    E = rng.normal(0.0, 1e-3, P.shape)
    E = 0.5 * (E + E.T)
    dev = torch.device("cuda", 0)
    Pd = torch.as_tensor(P, device=dev)
    ptd = torch.as_tensor(pts, device=dev)
    vt = build_table(wfn, basis, Pd + torch.as_tensor(E, device=dev), ptd).esp(ptd)
    return wfn, basis, Pd, ptd, vt


def _loss(wfn, basis, P, pts, vt):
    v = build_table(wfn, basis, P, pts).esp(pts)
    return 0.5 * float(((v - vt) ** 2).sum())


def _norm_rel_err(fd, an):
    fd, an = np.asarray(fd, float), np.asarray(an, float)
    return float(np.abs(fd - an).max() / np.abs(an).max())


def _rel_err(fd, an):
    fd, an = np.asarray(fd, float), np.asarray(an, float)
    scale = np.maximum(np.abs(an), 1e-3 * np.abs(an).max())
    return float((np.abs(fd - an) / scale).max())


@pytest.mark.parametrize("tag", ["small", "tz6"])
def test_field_matches_oracle(tag, request):
    wfn, basis, P, g = request.getfixturevalue(f"{tag}_system")
    Z = np.array([Z_OF[s] for s in wfn.symbols])
    pts = g["points"]
    otab = O.build_table(wfn.shells, wfn.coords, Z, g["density"], pts, tol=1e-12)
    tab = build_table(wfn, basis, g["density"], pts)
    v, dvdc = tab.esp_gradient(pts)
    np.testing.assert_allclose(v, g["esp_t12"], rtol=0, atol=1e-12)
    ref = otab.esp_gradient(pts)
    assert np.abs(dvdc - ref).max() < 1e-9, np.abs(dvdc - ref).max()
    np.testing.assert_allclose(tab.field(pts), -dvdc, rtol=0, atol=0)


def test_field_matches_central_differences(frag54, golden):
    wfn, basis, P = frag54
    pts = golden("frag54_300")["points"][:64]
    tab = build_table(wfn, basis, P, pts)
    _, g = tab.esp_gradient(pts)
    # fourth-order five-point stencil at h = 1e-3: truncation ~1e-12 h^4 f^(5),
    # rounding ~1e-9
    h = 1e-3
    fd = np.zeros_like(g)
    for c in range(3):
        d = np.zeros_like(pts)
        d[:, c] = h
        fd[:, c] = (8 * (tab.esp(pts + d) - tab.esp(pts - d))
                    - (tab.esp(pts + 2 * d) - tab.esp(pts - 2 * d))) / (12 * h)
    assert _norm_rel_err(fd, g) < REL
    assert _rel_err(fd, g) < 1e-5


def test_adjoint_points_is_weighted_field(adjoint20):
    import torch
    wfn, basis, P, pts, vt = adjoint20
    tab = build_table(wfn, basis, P, pts)
    w = torch.linspace(-1.0, 2.0, pts.shape[0], dtype=torch.float64, device=pts.device)
    _, g = tab.esp_gradient(pts)
    dP, dC = tab.adjoint(pts, w, density=False)
    assert dP is None
    torch.testing.assert_close(dC, w[:, None] * g, rtol=0, atol=0)
    _, gw = tab.esp_gradient(pts, weights=w)
    torch.testing.assert_close(gw, dC, rtol=0, atol=0)


def test_autograd_density_gradient_matches_central_differences(adjoint20):
    """dL/dP of L = 0.5 ||V - V_target||^2 through the autograd op, against
    central differences of single density entries and of a random symmetric
    direction."""
    import torch
    from fastesp_b200.autograd import esp
    wfn, basis, P, pts, vt = adjoint20
    Pg = P.clone().requires_grad_(True)
    v = esp(Pg, pts, wfn, basis)
    loss = 0.5 * ((v - vt) ** 2).sum()
    loss.backward()
    dP = Pg.grad.cpu().numpy()
    assert np.isfinite(dP).all() and np.abs(dP).max() > 0
    # entries: the largest gradients, and a seeded random sample
    rng = np.random.default_rng(3)
    n = P.shape[0]
    big = np.argsort(-np.abs(dP).ravel())[:6]
    rnd = rng.choice(n * n, size=6, replace=False)
    fd, an = [], []
    for flat in np.concatenate([big, rnd]):
        i, j = divmod(int(flat), n)
        e = torch.zeros_like(P)
        e[i, j] = H_FD
        fd.append((_loss(wfn, basis, P + e, pts, vt) - _loss(wfn, basis, P - e, pts, vt))
                  / (2 * H_FD))
        an.append(dP[i, j])
    assert _rel_err(fd, an) < REL, (fd, an)
    D = rng.normal(size=(n, n))
    D = torch.as_tensor(0.5 * (D + D.T), device=P.device)
    fdd = (_loss(wfn, basis, P + H_FD * D, pts, vt) - _loss(wfn, basis, P - H_FD * D, pts, vt)) \
        / (2 * H_FD)
    and_ = float((torch.as_tensor(dP, device=P.device) * D).sum())
    assert abs(fdd - and_) <= REL * abs(and_), (fdd, and_)


def test_autograd_points_gradient_matches_central_differences(adjoint20):
    import torch
    from fastesp_b200.autograd import esp
    wfn, basis, P, pts, vt = adjoint20
    pg = pts.clone().requires_grad_(True)
    v = esp(P, pg, wfn, basis)
    (0.5 * ((v - vt) ** 2).sum()).backward()
    an = pg.grad.cpu().numpy()
    tab = build_table(wfn, basis, P, pts)

    def loss_at(q):
        return 0.5 * float(((tab.esp(q) - vt) ** 2).sum())

    rng = np.random.default_rng(5)
    fd, ref = [], []
    for i in rng.choice(pts.shape[0], size=8, replace=False):
        for c in range(3):
            d = torch.zeros_like(pts)
            d[i, c] = H_FD
            fd.append((loss_at(pts + d) - loss_at(pts - d)) / (2 * H_FD))
            ref.append(an[i, c])
    assert _norm_rel_err(fd, ref) < REL


def test_density_gradient_l3_classes(frag54, golden):
    """Directional derivative on the 54-atom l<=3 system (classes up to L = 6,
    whose moments run in 2 and 3 term chunks)."""
    import torch
    wfn, basis, P = frag54
    pts = torch.as_tensor(golden("frag54_300")["points"], device="cuda")
    Pd = torch.as_tensor(P, device="cuda")
    rng = np.random.default_rng(11)
    w = torch.as_tensor(rng.normal(size=pts.shape[0]), device="cuda")
    tab = build_table(wfn, basis, Pd, pts)
    dP, _ = tab.adjoint(pts, w, coords=False)
    D = rng.normal(size=P.shape)
    D = torch.as_tensor(0.5 * (D + D.T), device="cuda")

    def lin(Q):
        return float((build_table(wfn, basis, Q, pts).esp(pts) * w).sum())

    fd = (lin(Pd + H_FD * D) - lin(Pd - H_FD * D)) / (2 * H_FD)
    an = float((dP * D).sum())
    assert abs(fd - an) <= REL * abs(an), (fd, an)


def test_adjoint_is_deterministic(adjoint20):
    import torch
    wfn, basis, P, pts, vt = adjoint20
    tab = build_table(wfn, basis, P, pts)
    w = tab.esp(pts) - vt
    a = tab.adjoint(pts, w)
    b = tab.adjoint(pts, w)
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
    # the gradient of a symmetric perturbation is symmetric where both
    # orderings of a shell pair share one weight
    assert torch.isfinite(a[0]).all()


def test_imported_table_gives_points_gradient_only(tmp_path, small_system):
    wfn, basis, P, g = small_system
    tab = build_table(wfn, basis, P, g["points"])
    tab.write(tmp_path / "pairs.bin")
    imp = PairTable.read(tmp_path / "pairs.bin")
    w = np.linspace(0.5, 1.5, len(g["points"]))
    with pytest.raises(ValueError):
        imp.adjoint(g["points"], w)
    _, dc = imp.adjoint(g["points"], w, density=False)
    _, dc0 = tab.adjoint(g["points"], w, density=False)
    np.testing.assert_allclose(dc, dc0, rtol=0, atol=1e-12)
