"""ctypes driver for the reference build in oracle/_ref (test infrastructure only).

Drives the UNMODIFIED exafmm-t headers through oracle/ref_capi.cpp:
``RefFmm.setup`` follows python/exafmm.cpp:155-180 (tree, balance, lists,
M2L_setup, precompute) and ``RefFmm.evaluate`` follows python/exafmm.cpp:190-267
(upward_pass + downward_pass of include/fmm_base.h:162-200, then the scatter to
the original target order).  Only tests, ``__graft_entry__.smoke`` and the
CPU-baseline leg of ``bench.py`` may import this module.
"""
import ctypes
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
KERNELS = {"laplace": 0, "modified_helmholtz": 1, "helmholtz": 2}


def _isa():
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
    except OSError:
        flags = ""
    return "avx512" if " avx512f" in flags and " avx512dq" in flags else "avx2"


_LIBS = {}


def _name(nonadaptive, fp32):
    # fp32: the reference's single-precision (-DFLOAT) build, adaptive only
    return "libxfmm_ref_%s%s.so" % ("f32_" if fp32 else ("na_" if nonadaptive else ""), _isa())


def available(nonadaptive=False, fp32=False):
    return os.path.exists(os.path.join(REF_DIR, _name(nonadaptive, fp32)))


def lib(nonadaptive=False, fp32=False):
    key = (bool(nonadaptive), bool(fp32))
    if key in _LIBS:
        return _LIBS[key]
    # the reference calls BLAS from inside OpenMP regions; keep OpenBLAS single-threaded
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    name = _name(nonadaptive, fp32)
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        raise RuntimeError("reference oracle library missing: %s (run make -C oracle)" % path)
    L = ctypes.CDLL(path)
    vp, i32, f64p = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
    L.ref_create.restype = vp
    L.ref_create.argtypes = [i32, i32, i32, ctypes.c_double, ctypes.c_double, ctypes.c_char_p]
    L.ref_setup.argtypes = [vp, i32, vp, vp, i32, vp, i32]
    L.ref_evaluate.argtypes = [vp, vp, vp]
    L.ref_clear_values.argtypes = [vp]
    L.ref_update_charges.argtypes = [vp, vp]
    L.ref_sizes.argtypes = [vp, vp]
    L.ref_dump.argtypes = [vp] * 17
    L.ref_verify.argtypes = [vp, i32, vp]
    L.ref_free.argtypes = [vp]
    L.ref_gradient_p2p.argtypes = [i32, ctypes.c_double, ctypes.c_double, i32, vp, vp, i32, vp, vp]
    L.ref_num_threads.restype = i32
    _LIBS[key] = L
    return L


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class RefFmm:
    """One reference FMM instance plus its tree (the state python/exafmm.cpp keeps in Tree)."""

    def __init__(self, kernel, p, ncrit, wavek=0.0, nonadaptive_depth=None, datdir=None, fp32=False):
        self.kernel = kernel
        self.kid = KERNELS[kernel]
        self.p, self.ncrit = p, ncrit
        self.wavek = complex(wavek)
        self.nonadaptive = nonadaptive_depth is not None
        self.depth_arg = -1 if nonadaptive_depth is None else int(nonadaptive_depth)
        if fp32 and self.nonadaptive:
            raise ValueError("the single-precision reference build is adaptive only")
        self.L = lib(self.nonadaptive, fp32)
        self._tmp = None
        if datdir is None:
            self._tmp = tempfile.TemporaryDirectory(prefix="xfmm_ref_")
            datdir = self._tmp.name
        # precompute cache keyed on everything the operators depend on (the reference's own
        # name omits the wavenumber: laplace.h:18-21, modified_helmholtz.h:21-24)
        fn = "%s_p%d_k%.6g_%.6g_%s.dat" % (kernel, p, self.wavek.real, self.wavek.imag,
                                          "na%d" % self.depth_arg if self.nonadaptive else "ad")
        self.datfile = os.path.join(datdir, fn).encode()
        self.h = self.L.ref_create(self.kid, p, ncrit, self.wavek.real, self.wavek.imag, self.datfile)
        self.nsrc = self.ntrg = 0

    def setup(self, src, q, trg):
        src = np.ascontiguousarray(src, dtype=np.float64)
        trg = np.ascontiguousarray(trg, dtype=np.float64)
        qq = np.ascontiguousarray(q, dtype=np.complex128 if self.kid == 2 else np.float64)
        self._keep = (src, trg, qq)
        self.nsrc, self.ntrg = len(src), len(trg)
        self.L.ref_setup(self.h, self.nsrc, _p(src), _p(qq), self.ntrg, _p(trg), self.depth_arg)
        return self

    def evaluate(self, stage_times=False):
        out = np.zeros((self.ntrg, 4), dtype=np.complex128 if self.kid == 2 else np.float64)
        t = np.zeros(8)
        self.L.ref_evaluate(self.h, _p(out), _p(t))
        if stage_times:
            return out, dict(zip(["P2M", "M2M", "P2L", "M2P", "P2P", "M2L", "L2L", "L2P"], t))
        return out

    def clear_values(self):
        self.L.ref_clear_values(self.h)

    def update_charges(self, q):
        qq = np.ascontiguousarray(q, dtype=np.complex128 if self.kid == 2 else np.float64)
        self.L.ref_update_charges(self.h, _p(qq))

    def verify(self, sample=True):
        e = np.zeros(2)
        self.L.ref_verify(self.h, int(sample), _p(e))
        return e

    def sizes(self):
        s = np.zeros(8, dtype=np.int64)
        self.L.ref_sizes(self.h, _p(s))
        return dict(zip(["nnodes", "nleafs", "nnonleafs", "depth", "np2p", "nm2p", "np2l", "nsurf"], s.tolist()))

    def dump(self):
        """Tree + lists in flat arrays (node order = the reference's node idx order)."""
        s = self.sizes()
        nn = s["nnodes"]
        d = dict(
            geo=np.zeros(6), key=np.zeros(nn, np.uint64), ni=np.zeros((nn, 8), np.int32),
            nx=np.zeros((nn, 4)), leafs=np.zeros(s["nleafs"], np.int32),
            nonleafs=np.zeros(s["nnonleafs"], np.int32), src_perm=np.zeros(self.nsrc, np.int32),
            trg_perm=np.zeros(self.ntrg, np.int32), colleagues=np.zeros((nn, 27), np.int32),
            m2l=np.zeros((nn, 26), np.int32), p2p_off=np.zeros(nn + 1, np.int64),
            p2p=np.zeros(max(s["np2p"], 1), np.int32), m2p_off=np.zeros(nn + 1, np.int64),
            m2p=np.zeros(max(s["nm2p"], 1), np.int32), p2l_off=np.zeros(nn + 1, np.int64),
            p2l=np.zeros(max(s["np2l"], 1), np.int32))
        order = ["geo", "key", "ni", "nx", "leafs", "nonleafs", "src_perm", "trg_perm", "colleagues", "m2l",
                 "p2p_off", "p2p", "m2p_off", "m2p", "p2l_off", "p2l"]
        self.L.ref_dump(self.h, *[_p(d[k]) for k in order])
        d["depth"] = s["depth"]
        d["x0"] = d["geo"][:3].copy()
        d["r0"] = float(d["geo"][3])
        for k in ("p2p", "m2p", "p2l"):
            d[k] = d[k][: s["n" + k]]
        return d

    def close(self):
        if self.h:
            self.L.ref_free(self.h)
            self.h = None
        if self._tmp is not None:
            self._tmp.cleanup()
            self._tmp = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gradient_p2p(kernel, src, q, trg, wavek=0.0):
    """The reference SIMD gradient_P2P over raw arrays (accumulated into zeros)."""
    L = lib(False)
    kid = KERNELS[kernel]
    src = np.ascontiguousarray(src, dtype=np.float64)
    trg = np.ascontiguousarray(trg, dtype=np.float64)
    cplx = kid == 2
    qq = np.ascontiguousarray(q, dtype=np.complex128 if cplx else np.float64)
    out = np.zeros((len(trg), 4), dtype=np.complex128 if cplx else np.float64)
    k = complex(wavek)
    L.ref_gradient_p2p(kid, k.real, k.imag, len(src), _p(src), _p(qq), len(trg), _p(trg), _p(out))
    return out
