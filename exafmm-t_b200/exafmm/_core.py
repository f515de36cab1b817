"""Python surface of exafmm-t's pybind11 module (python/exafmm.cpp:325-563) over the C ABI.

Names, argument names and return shapes follow the reference:
  init_sources(coords (n,3), charges (n,)) -> Bodies      python/exafmm.cpp:35-82
  init_targets(coords (n,3)) -> Bodies                    python/exafmm.cpp:90-106
  <Kernel>Fmm(p, ncrit[, wavek], filename="")             python/exafmm.cpp:441-476
  setup(sources, targets, fmm) -> Tree                    python/exafmm.cpp:155-180
  evaluate(tree, fmm, verbose=False) -> (ntrg, 4)         python/exafmm.cpp:190-267
  update_charges(tree, charges), clear_values(tree)       python/exafmm.cpp:275-323
  fmm.verify(leafs, sample=True) -> [err_p, err_grad]     include/fmm_base.h:208-267
Additions: a ``precision`` keyword ("fp64" as the reference, or "mixed"), a
``nonadaptive_depth`` keyword on setup (the reference's -DNON_ADAPTIVE build), and
torch CUDA tensors accepted wherever arrays are (device pointers, no copy).
"""
import ctypes

import numpy as np

from . import _lib

_DTYPE = {"laplace": np.float64, "modified_helmholtz": np.float64, "helmholtz": np.complex128}


def _current_stream():
    return ctypes.c_void_p(0)


class Bodies:
    """Sources or targets (the reference's std::vector<Body>): coordinates and charges."""

    def __init__(self, coords, charges=None, dtype=np.float64):
        if hasattr(coords, "is_cuda"):
            if coords.dim() != 2 or coords.shape[1] != 3:
                raise RuntimeError("coords should have a shape of (n, 3)")
            self.coords = coords.contiguous()
        else:
            c = np.asarray(coords)
            if c.ndim != 2 or c.shape[1] != 3:
                raise RuntimeError("coords should have a shape of (n, 3), charges should have a shape of (n,)"
                                   if charges is not None else "coords should have a shape of (n, 3)")
            self.coords = np.ascontiguousarray(c, dtype=np.float64)
        self.charges = None
        if charges is not None:
            if hasattr(charges, "is_cuda"):
                q = charges.contiguous()
                if q.dim() != 1:
                    raise RuntimeError("coords should have a shape of (n, 3), charges should have a shape of (n,)")
            else:
                q = np.asarray(charges)
                if q.ndim != 1:
                    raise RuntimeError("coords should have a shape of (n, 3), charges should have a shape of (n,)")
                q = np.ascontiguousarray(q, dtype=dtype)
            if q.shape[0] != self.coords.shape[0]:
                raise RuntimeError("Number of coords and charges must match")
            self.charges = q

    def __len__(self):
        return int(self.coords.shape[0])


class FmmBase:
    kernel = "laplace"

    def __init__(self, p=4, ncrit=64, filename="", wavek=0.0, precision="fp64"):
        if precision not in _lib.PRECISIONS:
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.p, self.ncrit, self.filename = int(p), int(ncrit), filename
        self.wavek = wavek
        self.precision = precision
        k = complex(wavek)
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().xfmm_fmm_create(_lib.KERNEL_IDS[self.kernel], self.p, self.ncrit, k.real, k.imag,
                                              _lib.PRECISIONS[precision], ctypes.byref(h)))
        self._h = h
        if filename:
            # operators read from / written to this file in the reference's .dat layout at setup
            _lib.check(_lib.lib().xfmm_fmm_set_operator_file(h, str(filename).encode()))
        self.nsurf = 6 * (self.p - 1) ** 2 + 2
        n1 = 2 * self.p
        self.nconv = n1 ** 3
        self.nfreq = self.nconv if self.kernel == "helmholtz" else n1 * n1 * (n1 // 2 + 1)

    @property
    def depth(self):
        return self._info()[0][5]

    @property
    def r0(self):
        return self._info()[1][3]

    @property
    def x0(self):
        return self._info()[1][:3].copy()

    def _info(self):
        i6 = np.zeros(6, np.int64)
        d4 = np.zeros(4)
        _lib.check(_lib.lib().xfmm_fmm_info(self._h, i6.ctypes.data, d4.ctypes.data))
        return i6, d4

    def verify(self, leafs, sample=True):
        """Relative L2 error of potential and gradient vs FP64 direct summation (fmm_base.h:208-267)."""
        tree = leafs.tree
        e = np.zeros(2)
        _lib.check(_lib.lib().xfmm_verify(self._h, tree._h, int(bool(sample)), e.ctypes.data, _current_stream()))
        return [float(e[0]), float(e[1])]

    def stage_times(self, tree):
        """Device ms of the last evaluate on ``tree``: P2M, M2M, P2L, M2L, L2L, L2P(check->equiv),
        P2P+M2P+L2P, total, the M2L forward-transform / Hadamard / backward-transform sub-stages, the
        number of this library's kernel launches, and the near (P2P) / far (M2P+L2P) split."""
        t = np.zeros(14)
        _lib.check(_lib.lib().xfmm_stage_times(self._h, tree._h, t.ctypes.data))
        names = ["P2M", "M2M", "P2L", "M2L", "L2L", "L2P_dc2e", "P2P_M2P_L2P", "total", "M2L_fft", "M2L_hadamard",
                 "M2L_ifft", "launches", "P2P", "M2P_L2P"]
        return dict(zip(names, t.tolist()))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().xfmm_fmm_free(h)
            except Exception:
                pass
            self._h = None


class LaplaceFmm(FmmBase):
    """LaplaceFmm(p, ncrit, filename="") -- include/laplace.h:15-22."""
    kernel = "laplace"

    def __init__(self, p=4, ncrit=64, filename="", precision="fp64"):
        super().__init__(p, ncrit, filename, 0.0, precision)


class ModifiedHelmholtzFmm(FmmBase):
    """ModifiedHelmholtzFmm(p, ncrit, wavek, filename="") -- include/modified_helmholtz.h:17-25."""
    kernel = "modified_helmholtz"

    def __init__(self, p=4, ncrit=64, wavek=1.0, filename="", precision="fp64"):
        super().__init__(p, ncrit, filename, float(wavek), precision)


class HelmholtzFmm(FmmBase):
    """HelmholtzFmm(p, ncrit, wavek, filename="") -- include/helmholtz.h:16-24."""
    kernel = "helmholtz"

    def __init__(self, p=4, ncrit=64, wavek=1.0 + 0.0j, filename="", precision="fp64"):
        super().__init__(p, ncrit, filename, complex(wavek), precision)


class Node:
    """Read-only view of one tree node (python/exafmm.cpp:393-421 fields)."""

    __slots__ = ("idx", "level", "is_leaf", "nsrcs", "ntrgs", "parent", "octant", "x", "r", "key", "isrcs", "itrgs")

    def __repr__(self):
        return "Node(idx=%d, level=%d, leaf=%s, nsrcs=%d, ntrgs=%d)" % (self.idx, self.level, self.is_leaf,
                                                                       self.nsrcs, self.ntrgs)


class _NodeList:
    def __init__(self, tree, indices):
        self.tree = tree
        self.indices = indices

    def __len__(self):
        return len(self.indices)

    def __getitem__(self, i):
        return self.tree._node(int(self.indices[i]))

    def __iter__(self):
        for i in range(len(self)):
            yield self[i]


class Tree:
    """Device-resident tree of one setup() (python/exafmm.cpp:113-118)."""

    def __init__(self, h, fmm, nsrc, ntrg):
        self._h, self.fmm, self.nsrc, self.ntrg = h, fmm, nsrc, ntrg
        self._dump = None

    TUNING = {"sparse_hadamard_tiles_per_cta": 1}  # include/xfmm.h XFMM_TUNE_*

    def set_tuning(self, name, value):
        """Tile option for later evaluates of this tree (no reference counterpart); 0 restores the default."""
        _lib.check(_lib.lib().xfmm_set_tuning(self._h, self.TUNING[name], int(value)))

    def info(self):
        v = np.zeros(12, np.int64)
        _lib.check(_lib.lib().xfmm_tree_info(self._h, v.ctypes.data))
        keys = ["nnodes", "nleafs", "nnonleafs", "depth", "np2p", "nm2p", "np2l", "n_m2l_src", "p2p_pairs",
                "m2p_pairs", "l2p_pairs", "m2l_pairs"]
        return dict(zip(keys, v.tolist()))

    def dump(self):
        """Flat arrays of the tree and lists in the reference's node order."""
        if self._dump is not None:
            return self._dump
        s = self.info()
        nn = s["nnodes"]
        d = dict(
            geo=np.zeros(6), key=np.zeros(nn, np.uint64), ni=np.zeros((nn, 8), np.int32), nx=np.zeros((nn, 4)),
            leafs=np.zeros(s["nleafs"], np.int32), nonleafs=np.zeros(s["nnonleafs"], np.int32),
            src_perm=np.zeros(self.nsrc, np.int32), trg_perm=np.zeros(self.ntrg, np.int32),
            colleagues=np.zeros((nn, 27), np.int32), m2l=np.zeros((nn, 26), np.int32),
            p2p_off=np.zeros(nn + 1, np.int64), p2p=np.zeros(max(s["np2p"], 1), np.int32),
            m2p_off=np.zeros(nn + 1, np.int64), m2p=np.zeros(max(s["nm2p"], 1), np.int32),
            p2l_off=np.zeros(nn + 1, np.int64), p2l=np.zeros(max(s["np2l"], 1), np.int32))
        order = ["geo", "key", "ni", "nx", "leafs", "nonleafs", "src_perm", "trg_perm", "colleagues", "m2l",
                 "p2p_off", "p2p", "m2p_off", "m2p", "p2l_off", "p2l"]
        _lib.check(_lib.lib().xfmm_tree_dump(self._h, *[d[k].ctypes.data for k in order]))
        for k in ("p2p", "m2p", "p2l"):
            d[k] = d[k][: s["n" + k]]
        d["depth"] = s["depth"]
        d["x0"] = d["geo"][:3].copy()
        d["r0"] = float(d["geo"][3])
        self._dump = d
        return d

    def _node(self, i):
        d = self.dump()
        n = Node()
        row = d["ni"][i]
        n.idx, n.level, n.is_leaf, n.nsrcs, n.ntrgs, n.parent, n.octant = (int(row[0]), int(row[1]), bool(row[2]),
                                                                           int(row[3]), int(row[4]), int(row[5]),
                                                                           int(row[6]))
        n.x = d["nx"][i, :3].copy()
        n.r = float(d["nx"][i, 3])
        n.key = int(d["key"][i])
        if n.is_leaf:
            # body ranges of the leaf in tree order
            if not hasattr(self, "_ranges"):
                self._ranges = {}
                so = to = 0
                for li in d["leafs"]:
                    self._ranges[int(li)] = (so, to)
                    so += int(d["ni"][li, 3])
                    to += int(d["ni"][li, 4])
            so, to = self._ranges.get(i, (0, 0))
            n.isrcs = d["src_perm"][so:so + n.nsrcs].tolist()
            n.itrgs = d["trg_perm"][to:to + n.ntrgs].tolist()
        else:
            n.isrcs, n.itrgs = [], []
        return n

    @property
    def nodes(self):
        return _NodeList(self, np.arange(self.info()["nnodes"]))

    @property
    def leafs(self):
        return _NodeList(self, self.dump()["leafs"])

    @property
    def nonleafs(self):
        return _NodeList(self, self.dump()["nonleafs"])

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.lib().xfmm_tree_free(h)
            except Exception:
                pass
            self._h = None


def _kernel_of(fmm):
    return fmm.kernel


def init_sources(coords, charges, kernel="laplace"):
    return Bodies(coords, charges, _DTYPE[kernel])


def init_targets(coords):
    return Bodies(coords)


def setup(sources, targets, fmm, nonadaptive_depth=None):
    """Tree + balance, lists, M2L setup and precomputation (python/exafmm.cpp:155-180)."""
    if sources.charges is None:
        raise RuntimeError("sources need charges")
    L = _lib.lib()
    st = _current_stream()
    sp, sdev = _lib.ptr(sources.coords)
    tp, tdev = _lib.ptr(targets.coords)
    if sdev != tdev:
        raise RuntimeError("sources and targets must both be host arrays or both be CUDA tensors")
    h = ctypes.c_void_p()
    depth = -1 if nonadaptive_depth is None else int(nonadaptive_depth)
    _lib.check(L.xfmm_build_tree(fmm._h, sp, len(sources), tp, len(targets), depth, sdev, st, ctypes.byref(h)))
    tree = Tree(h, fmm, len(sources), len(targets))
    _lib.check(L.xfmm_build_list(fmm._h, h, st))
    _lib.check(L.xfmm_m2l_setup(fmm._h, h, st))
    _lib.check(L.xfmm_precompute(fmm._h, h, st))
    update_charges(tree, sources.charges)
    tree._sources, tree._targets = sources, targets
    return tree


def update_charges(tree, charges):
    """Rewrite the source charges in the caller's original order (python/exafmm.cpp:275-305)."""
    fmm = tree.fmm
    if not hasattr(charges, "is_cuda"):
        charges = np.ascontiguousarray(charges, dtype=_DTYPE[fmm.kernel])
        if charges.shape != (tree.nsrc,):
            raise RuntimeError("charges should have a shape of (nsrc,)")
    elif charges.is_complex():
        import torch
        charges = torch.view_as_real(charges.contiguous()).reshape(-1)
    qp, qdev = _lib.ptr(charges)
    _lib.check(_lib.lib().xfmm_set_charges(fmm._h, tree._h, qp, qdev, _current_stream()))


def clear_values(tree):
    """Zero equivalent densities and check potentials (python/exafmm.cpp:313-323)."""
    _lib.check(_lib.lib().xfmm_clear_values(tree.fmm._h, tree._h, _current_stream()))


def evaluate(tree, fmm, verbose=False, out=None):
    """Potential and gradient at every target, (ntrg, 4) in the original target order."""
    L = _lib.lib()
    if out is None:
        out = np.zeros((tree.ntrg, 4), dtype=_DTYPE[fmm.kernel])
    op, odev = _lib.ptr(out)
    _lib.check(L.xfmm_evaluate(fmm._h, tree._h, op, odev, _current_stream()))
    if verbose:
        for k, v in fmm.stage_times(tree).items():
            print("%-20s : %.7e ms" % (k, v))
    return out


def gradient_p2p(kernel, src, q, trg, wavek=0.0, precision="fp64"):
    """Direct potential + gradient (the kernels' gradient_P2P) on the GPU, (ntrg, 4)."""
    src = np.ascontiguousarray(src, np.float64)
    trg = np.ascontiguousarray(trg, np.float64)
    q = np.ascontiguousarray(q, _DTYPE[kernel])
    out = np.zeros((len(trg), 4), dtype=_DTYPE[kernel])
    k = complex(wavek)
    _lib.check(_lib.lib().xfmm_gradient_p2p(_lib.KERNEL_IDS[kernel], k.real, k.imag, _lib.PRECISIONS[precision],
                                            src.ctypes.data, len(src), q.ctypes.data, trg.ctypes.data, len(trg),
                                            out.ctypes.data, 0, _current_stream()))
    return out
