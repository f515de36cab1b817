"""ctypes driver for liborc.so, the oracle's C restatement (test infrastructure only).

``build`` restates the reference's tree, balance and list construction
(build_tree.h, build_non_adaptive_tree.h, build_list.h) and returns the same flat
dump format as ``oracle.ref.RefFmm.dump``; ``gradient_p2p``/``potential_p2p``
restate the scalar direct kernels (laplace.h, modified_helmholtz.h, helmholtz.h);
``direct`` is the FP64 direct-summation accuracy oracle on sampled targets.
Only tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of ``bench.py``
may import this module.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
KERNELS = {"laplace": 0, "modified_helmholtz": 1, "helmholtz": 2}
_L = None


def nsurf_of(p):
    """fmm_base.h:30: number of surface points."""
    return 6 * (p - 1) * (p - 1) + 2


def lib():
    global _L
    if _L is not None:
        return _L
    path = os.path.join(HERE, "liborc.so")
    if not os.path.exists(path):
        subprocess.run(["make", "-C", HERE, "orc"], check=True, capture_output=True)
    L = ctypes.CDLL(path)
    vp, i32 = ctypes.c_void_p, ctypes.c_int
    L.orc_build.restype = vp
    L.orc_build.argtypes = [i32, vp, i32, vp, i32, i32, i32]
    L.orc_free.argtypes = [vp]
    L.orc_sizes.argtypes = [vp, vp]
    L.orc_dump.argtypes = [vp] * 17
    for f in (L.orc_gradient_p2p, L.orc_potential_p2p):
        f.argtypes = [i32, ctypes.c_double, ctypes.c_double, i32, vp, vp, i32, vp, vp]
    _L = L
    return L


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def build(src, trg, ncrit, depth=None, nsurf=296):
    """Tree + lists; ``depth=None`` -> adaptive + 2:1 balance, else uniform to ``depth``."""
    L = lib()
    src = np.ascontiguousarray(src, dtype=np.float64)
    trg = np.ascontiguousarray(trg, dtype=np.float64)
    h = L.orc_build(len(src), _p(src), len(trg), _p(trg), int(ncrit), -1 if depth is None else int(depth),
                    int(nsurf))
    if not h:
        raise MemoryError("orc_build failed")
    try:
        s = np.zeros(8, dtype=np.int64)
        L.orc_sizes(h, _p(s))
        nn, nl, nnl, dep, np2p, nm2p, np2l = s[:7].tolist()
        d = dict(
            geo=np.zeros(6), key=np.zeros(nn, np.uint64), ni=np.zeros((nn, 8), np.int32), nx=np.zeros((nn, 4)),
            leafs=np.zeros(nl, np.int32), nonleafs=np.zeros(nnl, np.int32),
            src_perm=np.zeros(len(src), np.int32), trg_perm=np.zeros(len(trg), np.int32),
            colleagues=np.zeros((nn, 27), np.int32), m2l=np.zeros((nn, 26), np.int32),
            p2p_off=np.zeros(nn + 1, np.int64), p2p=np.zeros(max(np2p, 1), np.int32),
            m2p_off=np.zeros(nn + 1, np.int64), m2p=np.zeros(max(nm2p, 1), np.int32),
            p2l_off=np.zeros(nn + 1, np.int64), p2l=np.zeros(max(np2l, 1), np.int32))
        order = ["geo", "key", "ni", "nx", "leafs", "nonleafs", "src_perm", "trg_perm", "colleagues", "m2l",
                 "p2p_off", "p2p", "m2p_off", "m2p", "p2l_off", "p2l"]
        L.orc_dump(h, *[_p(d[k]) for k in order])
    finally:
        L.orc_free(h)
    d["p2p"], d["m2p"], d["p2l"] = d["p2p"][:np2p], d["m2p"][:nm2p], d["p2l"][:np2l]
    d["depth"] = dep
    d["x0"] = d["geo"][:3].copy()
    d["r0"] = float(d["geo"][3])
    return d


def _kernel_call(fn, kernel, src, q, trg, wavek, width):
    L = lib()
    kid = KERNELS[kernel]
    src = np.ascontiguousarray(src, dtype=np.float64).reshape(-1, 3)
    trg = np.ascontiguousarray(trg, dtype=np.float64).reshape(-1, 3)
    cplx = kid == 2
    qq = np.ascontiguousarray(q, dtype=np.complex128 if cplx else np.float64)
    shape = (len(trg), width) if width > 1 else (len(trg),)
    out = np.zeros(shape, dtype=np.complex128 if cplx else np.float64)
    k = complex(wavek)
    getattr(L, fn)(kid, k.real, k.imag, len(src), _p(src), _p(qq), len(trg), _p(trg), _p(out))
    return out


def gradient_p2p(kernel, src, q, trg, wavek=0.0):
    """(ntrg, 4) potential + gradient, FP64 scalar restatement."""
    return _kernel_call("orc_gradient_p2p", kernel, src, q, trg, wavek, 4)


def potential_p2p(kernel, src, q, trg, wavek=0.0):
    """(ntrg,) potential, FP64 scalar restatement."""
    return _kernel_call("orc_potential_p2p", kernel, src, q, trg, wavek, 1)


def direct(kernel, src, q, trg_sample, wavek=0.0):
    """FP64 direct summation over ALL sources at the sampled targets (the accuracy oracle)."""
    return gradient_p2p(kernel, src, q, trg_sample, wavek)


def rel_l2(approx, exact):
    """Relative L2 errors of potential (column 0) and gradient (columns 1-3), as fmm_base.h:251-265."""
    approx = np.asarray(approx)
    exact = np.asarray(exact)
    pe = np.sqrt(np.sum(np.abs(approx[:, 0] - exact[:, 0]) ** 2) / np.sum(np.abs(exact[:, 0]) ** 2))
    ge = np.sqrt(np.sum(np.abs(approx[:, 1:] - exact[:, 1:]) ** 2) / np.sum(np.abs(exact[:, 1:]) ** 2))
    return float(pe), float(ge)
