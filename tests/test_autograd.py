"""Adjoint FMM (exafmm.autograd.FmmFunction): gradients with respect to charges and coordinates.

Checked three ways: against the adjoint computed by FP64 direct summation on the GPU (the transposed
sums, tolerance 1e-6 relative: the FMM error at p = 8), against central finite differences of the
FMM itself (h = 1e-4; charges enter linearly, coordinates through the kernel), and against the
reference's own gradient output on the golden Yukawa fixture (dL/dy = w * grad phi).
"""
import numpy as np
import pytest

from golden_cases import load

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _sphere(n, seed):
    v = np.random.default_rng(seed).standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _rel(a, b):
    a, b = np.asarray(a, float).ravel(), np.asarray(b, float).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _direct_adjoint(kernel, wavek, x, q, y, w):
    """dL/dq, dL/dx (source part) and dL/dy for L = sum_i w_i phi(y_i), by FP64 direct sums."""
    from exafmm import _core
    psi = _core.gradient_p2p(kernel, y, w, x, wavek)    # sources at y with charges w, targets at x
    g = _core.gradient_p2p(kernel, x, q, y, wavek)      # forward gradient at y
    return psi[:, 0], q[:, None] * psi[:, 1:4], w[:, None] * g[:, 1:4]


def test_adjoint_same_points_yukawa_matches_direct_sums():
    _need_gpu()
    import exafmm.modified_helmholtz as mh
    from exafmm.autograd import fmm_apply
    n, k = 3000, 10.0
    x = _sphere(n, 0)
    rng = np.random.default_rng(1)
    q, w = rng.uniform(-1, 1, n), rng.standard_normal(n)
    X = torch.tensor(x, device="cuda", requires_grad=True)
    Q = torch.tensor(q, device="cuda", requires_grad=True)
    fmm = mh.ModifiedHelmholtzFmm(8, 64, k)
    out = fmm_apply(Q, X, X, fmm)
    (out[:, 0] * torch.tensor(w, device="cuda")).sum().backward()
    dq, dx_src, dy = _direct_adjoint("modified_helmholtz", k, x, q, x, w)
    assert _rel(Q.grad.cpu(), dq) < 1e-6
    assert _rel(X.grad.cpu(), dx_src + dy) < 1e-6


def test_adjoint_distinct_points_laplace_matches_direct_sums():
    _need_gpu()
    import exafmm.laplace as lap
    from exafmm.autograd import fmm_apply
    rng = np.random.default_rng(2)
    x, y = rng.random((2000, 3)), rng.random((1500, 3))
    q, w = rng.uniform(-1, 1, 2000), rng.standard_normal(1500)
    X = torch.tensor(x, device="cuda", requires_grad=True)
    Y = torch.tensor(y, device="cuda", requires_grad=True)
    Q = torch.tensor(q, device="cuda", requires_grad=True)
    out = fmm_apply(Q, X, Y, lap.LaplaceFmm(8, 64))
    (out[:, 0] * torch.tensor(w, device="cuda")).sum().backward()
    dq, dx, dy = _direct_adjoint("laplace", 0.0, x, q, y, w)
    assert _rel(Q.grad.cpu(), dq) < 1e-6
    assert _rel(X.grad.cpu(), dx) < 1e-6
    assert _rel(Y.grad.cpu(), dy) < 1e-6


def test_adjoint_matches_central_differences():
    _need_gpu()
    import exafmm.modified_helmholtz as mh
    from exafmm.autograd import fmm_apply
    n, k, h = 2000, 10.0, 1e-4
    x = _sphere(n, 3)
    rng = np.random.default_rng(4)
    q, w = rng.uniform(-1, 1, n), rng.standard_normal(n)
    W = torch.tensor(w, device="cuda")
    fmm = mh.ModifiedHelmholtzFmm(8, 64, k)

    def loss(xa, qa):
        X = torch.tensor(xa, device="cuda")
        return float((fmm_apply(torch.tensor(qa, device="cuda"), X, X, fmm)[:, 0] * W).sum())

    X = torch.tensor(x, device="cuda", requires_grad=True)
    Q = torch.tensor(q, device="cuda", requires_grad=True)
    (fmm_apply(Q, X, X, fmm)[:, 0] * W).sum().backward()
    gq, gx = Q.grad.cpu().numpy(), X.grad.cpu().numpy()
    # interior points only, so that no perturbation moves the bounding box
    inner = np.where(np.all(np.abs(x) < 0.9 * np.abs(x).max(axis=0), axis=1))[0]
    idx = rng.choice(inner, 8, replace=False)
    fq, fx, aq, ax = [], [], [], []
    for j in idx:
        e = np.zeros(n); e[j] = h
        fq.append((loss(x, q + e) - loss(x, q - e)) / (2 * h)); aq.append(gq[j])
        d = int(rng.integers(3))
        xp, xm = x.copy(), x.copy()
        xp[j, d] += h; xm[j, d] -= h
        fx.append((loss(xp, q) - loss(xm, q)) / (2 * h)); ax.append(gx[j, d])
    assert _rel(aq, fq) < 1e-6
    assert _rel(ax, fx) < 1e-4


def test_adjoint_target_gradient_matches_reference_fixture():
    """dL/dy = w * grad phi, with grad phi the reference's own output (golden fixture)."""
    _need_gpu()
    import exafmm.modified_helmholtz as mh
    from exafmm.autograd import fmm_apply
    g = load("yukawa_sphere_p4")
    x, y, q = g["src"], g["trg"], g["q"]
    w = np.random.default_rng(5).standard_normal(len(y))
    Y = torch.tensor(y, device="cuda", requires_grad=True)
    fmm = mh.ModifiedHelmholtzFmm(int(g["p"]), int(g["ncrit"]), complex(g["wavek"]).real)
    out = fmm_apply(torch.tensor(q, device="cuda"), torch.tensor(x, device="cuda"), Y, fmm)
    (out[:, 0] * torch.tensor(w, device="cuda")).sum().backward()
    assert _rel(Y.grad.cpu(), w[:, None] * g["out"][:, 1:4]) < 1e-9


def test_adjoint_rejects_gradient_cotangents():
    _need_gpu()
    import exafmm.laplace as lap
    from exafmm.autograd import fmm_apply
    x = torch.rand((500, 3), dtype=torch.float64, device="cuda")
    q = torch.rand(500, dtype=torch.float64, device="cuda", requires_grad=True)
    out = fmm_apply(q, x, x, lap.LaplaceFmm(4, 64))
    with pytest.raises(NotImplementedError):
        out[:, 1].sum().backward()
