"""xfmm_gradient_p2p_noalloc against xfmm_gradient_p2p, both through the C ABI.

The no-alloc entry point runs the same packing and P2P kernels as xfmm_gradient_p2p, only with its
scratch in a static device array, so the two agree to rounding: tolerance 1e-14 (relative L2).
Collected last (file name) so that it also runs after every other test in one process; it passes
alone in a fresh process as well.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TOL = 1e-14
SCRATCH = 16 << 20
CASES = [("laplace", 0.0, 0.0), ("modified_helmholtz", 10.0, 0.0), ("helmholtz", 5.0, 0.0)]


def _lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from exafmm import _lib
    return _lib


def _bodies(seed, nsrc, ntrg, cplx):
    rng = np.random.default_rng(seed)
    src = torch.tensor(rng.random((nsrc, 3)), dtype=torch.float64, device="cuda")
    trg = torch.tensor(rng.random((ntrg, 3)), dtype=torch.float64, device="cuda")
    qn = rng.uniform(-1, 1, (nsrc, 2) if cplx else nsrc)
    q = torch.tensor(qn, dtype=torch.float64, device="cuda")
    return src, q, trg


def _call(L, name, fn, kid, wk, prec, src, q, trg, out, stream):
    P = ctypes.c_void_p
    args = [kid, wk, 0.0, prec, P(src.data_ptr()), src.shape[0], P(q.data_ptr()), P(trg.data_ptr()),
            trg.shape[0], P(out.data_ptr())]
    if name == "existing":
        code = fn(*args, 1, P(stream))
    else:
        code = fn(*args, P(stream))
    L.check(code)


def _rel(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("kernel,wk,_", CASES)
def test_noalloc_matches_existing_on_two_consecutive_calls(kernel, wk, _, precision):
    L = _lib()
    lib = L.lib()
    kid, prec = L.KERNEL_IDS[kernel], L.PRECISIONS[precision]
    cplx = kernel == "helmholtz"
    width = 8 if cplx else 4
    stream = torch.cuda.current_stream().cuda_stream
    for call, (ns, nt) in enumerate([(3000, 2000), (1777, 2531)]):
        src, q, trg = _bodies(100 + call, ns, nt, cplx)
        ref = torch.zeros((nt, width), dtype=torch.float64, device="cuda")
        _call(L, "existing", lib.xfmm_gradient_p2p, kid, wk, prec, src, q, trg, ref, stream)
        got = torch.zeros((nt, width), dtype=torch.float64, device="cuda")
        _call(L, "noalloc", lib.xfmm_gradient_p2p_noalloc, kid, wk, prec, src, q, trg, got, stream)
        torch.cuda.synchronize()
        assert torch.isfinite(got).all()
        err = _rel(got, ref)
        assert err <= TOL, (call, err)


def test_noalloc_accumulates_into_out():
    L = _lib()
    lib = L.lib()
    stream = torch.cuda.current_stream().cuda_stream
    src, q, trg = _bodies(7, 500, 300, False)
    base = torch.full((300, 4), 0.25, dtype=torch.float64, device="cuda")
    ref = torch.zeros_like(base)
    _call(L, "existing", lib.xfmm_gradient_p2p, 0, 0.0, 0, src, q, trg, ref, stream)
    got = base.clone()
    _call(L, "noalloc", lib.xfmm_gradient_p2p_noalloc, 0, 0.0, 0, src, q, trg, got, stream)
    torch.cuda.synchronize()
    assert _rel(got - base, ref) <= TOL


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = _lib()
    lib = L.lib()
    stream = torch.cuda.current_stream().cuda_stream
    ns = SCRATCH // 40 + 1  # sources alone overflow the scratch
    src = torch.zeros((ns, 3), dtype=torch.float64, device="cuda")
    q = torch.zeros(ns, dtype=torch.float64, device="cuda")
    trg = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    out = torch.full((4, 4), 3.0, dtype=torch.float64, device="cuda")
    with pytest.raises(L.FmmError) as e:
        _call(L, "noalloc", lib.xfmm_gradient_p2p_noalloc, 0, 0.0, 0, src, q, trg, out, stream)
    assert e.value.code == 1 and "scratch" in str(e.value)
    torch.cuda.synchronize()
    assert bool((out == 3.0).all())  # nothing was launched


def test_noalloc_rejects_host_pointers():
    L = _lib()
    lib = L.lib()
    src = np.zeros((8, 3))
    q = np.zeros(8)
    trg = np.zeros((4, 3))
    out = np.zeros((4, 4))
    P = ctypes.c_void_p
    code = lib.xfmm_gradient_p2p_noalloc(0, 0.0, 0.0, 0, src.ctypes.data_as(P), 8, q.ctypes.data_as(P),
                                         trg.ctypes.data_as(P), 4, out.ctypes.data_as(P), None)
    assert code == 1
    assert b"device memory" in lib.xfmm_last_error()
