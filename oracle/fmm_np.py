"""numpy restatement of exafmm-t's KIFMM evaluate path (test infrastructure only).

The oracle for the GPU far field: it consumes the tree and lists of the C
restatement (``orc.build``) and recomputes every operator and pass in FP64:

  geometry       surface                geometry.h:21-63
                 convolution_grid       geometry.h:75-92
                 surf2conv up/dn maps   geometry.h:101-134
                 relative positions     geometry.h:156-215
  precompute     check2equiv (SVD pinv) fmm_scale_invariant.h:446-514, fmm.h:451-521
                 M2M / L2L              fmm_scale_invariant.h:51-77,  fmm.h:47-74
                 M2L kernel FFT tables  fmm_scale_invariant.h:517-558, fmm.h:524-629
  evaluate       P2M                    fmm_scale_invariant.h:163-195, fmm.h:156-185
                 M2M                    fmm_scale_invariant.h:233-253, fmm.h:221-241
                 P2L / M2P / P2P        fmm_base.h:82-154
                 M2L (FFT, Hadamard,    fmm_scale_invariant.h:343-440, 560-646;
                      iFFT)             fmm.h:335-446, 631-788; intrinsics.h (matmult_8x8x2)
                 L2L                    fmm_scale_invariant.h:256-275, fmm.h:244-263
                 L2P                    fmm_scale_invariant.h:198-230, fmm.h:188-218

Laplace uses the scale-invariant level-0 operators (P2M/L2P scaled by 0.5^level,
M2L by 2^(level+1)); modified Helmholtz and Helmholtz use per-level operators.
Surface-to-grid maps use round-to-nearest where the reference truncates
(identical for every p <= 20: the values are within rounding of integers).
An optional ``emulate`` hook lets tests round intermediate quantities to FP32 to
study the error of mixed precision.
"""
import numpy as np


FOUR_PI = 4.0 * np.pi
KERNELS = ("laplace", "modified_helmholtz", "helmholtz")


# ----------------------------------------------------------------------------- geometry
def nsurf_of(p):
    return 6 * (p - 1) * (p - 1) + 2


def surface(p, r0, level, c, alpha):
    """geometry.h:21-63."""
    n = nsurf_of(p)
    coord = np.zeros((n, 3))
    coord[0] = -1.0
    cnt = 1
    for i in range(p - 1):
        for j in range(p - 1):
            coord[cnt] = (-1.0, (2.0 * (i + 1) - p + 1) / (p - 1), (2.0 * j - p + 1) / (p - 1))
            cnt += 1
    for i in range(p - 1):
        for j in range(p - 1):
            coord[cnt] = ((2.0 * i - p + 1) / (p - 1), -1.0, (2.0 * (j + 1) - p + 1) / (p - 1))
            cnt += 1
    for i in range(p - 1):
        for j in range(p - 1):
            coord[cnt] = ((2.0 * (i + 1) - p + 1) / (p - 1), (2.0 * j - p + 1) / (p - 1), -1.0)
            cnt += 1
    coord[cnt:] = -coord[: n // 2]
    r = r0 * 0.5 ** level
    b = alpha * r
    return coord * b + np.asarray(c, dtype=np.float64)


def convolution_grid(p, r0, level, c):
    """geometry.h:75-92; row g = i + n1*j + n1^2*k."""
    d = 2 * r0 * 0.5 ** level
    a = d * 1.05
    n1 = 2 * p
    k, j, i = np.meshgrid(np.arange(n1), np.arange(n1), np.arange(n1), indexing="ij")
    g = np.stack([(i - p) * a / (p - 1) + c[0], (j - p) * a / (p - 1) + c[1], (k - p) * a / (p - 1) + c[2]], -1)
    return g.reshape(-1, 3)


def surf2conv(p, up):
    """geometry.h:101-134: surface point -> flat conv-grid index (up: reversed, dn: shifted)."""
    n1 = 2 * p
    c = [0.5 * (p - 1)] * 3
    s = surface(p, 0.5, 0, c, float(p - 1))
    off = (p - 1) if up else (2 * p - 1)
    ix = np.rint(off - s).astype(np.int64)
    return ix[:, 0] + ix[:, 1] * n1 + ix[:, 2] * n1 * n1


def rel_coords(max_r, min_r, step):
    """geometry.h:156-173 enumeration order (k outer, j, i inner)."""
    out = []
    for k in range(-max_r, max_r + 1, step):
        for j in range(-max_r, max_r + 1, step):
            for i in range(-max_r, max_r + 1, step):
                if abs(i) >= min_r or abs(j) >= min_r or abs(k) >= min_r:
                    out.append((i, j, k))
    return np.array(out, dtype=np.int64)


M2M_REL = rel_coords(1, 1, 2)      # 8, index == octant
M2L_REL = rel_coords(1, 1, 1)      # 26 parent offsets
M2LH_REL = rel_coords(3, 2, 1)     # 316 child offsets


def m2l_index_map():
    """geometry.h:176-195: [26][64] -> helper index, j = src_octant*8 + trg_octant; -1 if adjacent."""
    lut = {tuple(c): n for n, c in enumerate(M2LH_REL)}
    m = -np.ones((len(M2L_REL), 64), dtype=np.int64)
    for i, pr in enumerate(M2L_REL):
        for j1 in range(8):
            for j2 in range(8):
                cr = (pr[0] * 2 - (j1 & 1) + (j2 & 1), pr[1] * 2 - ((j1 >> 1) & 1) + ((j2 >> 1) & 1),
                      pr[2] * 2 - ((j1 >> 2) & 1) + ((j2 >> 2) & 1))
                m[i, j2 * 8 + j1] = lut.get(cr, -1)
    return m


# ----------------------------------------------------------------------------- kernels
def potential(kernel, wavek, src, q, trg):
    """Potential at trg (m,3) from charges q at src (n,3); r == 0 pairs skipped."""
    dx = trg[:, None, :] - src[None, :, :]
    r2 = np.einsum("ijk,ijk->ij", dx, dx)
    nz = r2 != 0
    r = np.sqrt(np.where(nz, r2, 1.0))
    if kernel == "laplace":
        g = 1.0 / r
    elif kernel == "modified_helmholtz":
        g = np.exp(-wavek.real * r) / r
    else:
        g = np.exp(1j * wavek * r) / r
    g = np.where(nz, g, 0.0)
    return (g @ q) / FOUR_PI


def gradient(kernel, wavek, src, q, trg):
    """(m,4): potential and gradient w.r.t. the target position."""
    with np.errstate(divide="ignore", invalid="ignore"):
        return _gradient(kernel, wavek, src, q, trg)


def _gradient(kernel, wavek, src, q, trg):
    dx = trg[:, None, :] - src[None, :, :]
    r2 = np.einsum("ijk,ijk->ij", dx, dx)
    nz = r2 != 0
    r = np.sqrt(np.where(nz, r2, 1.0))
    if kernel == "laplace":
        g = 1.0 / r
        dg = -1.0 / (r2 * r)
    elif kernel == "modified_helmholtz":
        k = wavek.real
        g = np.exp(-k * r) / r
        dg = -g * (k * r + 1) / r2
    else:
        k = wavek
        g = np.exp(1j * k * r) / r
        dg = (1j * k / r - 1 / r2) * g
    g = np.where(nz, g, 0.0)
    dg = np.where(nz, dg, 0.0)
    out = np.empty((len(trg), 4), dtype=np.result_type(g, q))
    out[:, 0] = g @ q
    for d in range(3):
        out[:, 1 + d] = (dg * dx[:, :, d]) @ q
    return out / FOUR_PI


def kernel_matrix(kernel, wavek, src, trg):
    """fmm_base.h:65-76: M[i, j] = potential at trg j from unit charge at src i."""
    return potential_matrix(kernel, wavek, src, trg).T


def potential_matrix(kernel, wavek, src, trg):
    dx = trg[:, None, :] - src[None, :, :]
    r2 = np.einsum("ijk,ijk->ij", dx, dx)
    nz = r2 != 0
    r = np.sqrt(np.where(nz, r2, 1.0))
    if kernel == "laplace":
        g = 1.0 / r
    elif kernel == "modified_helmholtz":
        g = np.exp(-wavek.real * r) / r
    else:
        g = np.exp(1j * wavek * r) / r
    return np.where(nz, g, 0.0) / FOUR_PI


# ----------------------------------------------------------------------------- precompute
class Operators:
    """Check-to-equivalent pinv factors, M2M/L2L and M2L tables for one level (FP64)."""

    def __init__(self, kernel, wavek, p, r0, level, m2l_level=None, eps=1e-16):
        self.kernel, self.wavek, self.p = kernel, wavek, p
        n = nsurf_of(p)
        cplx = kernel == "helmholtz"
        c = np.zeros(3)
        up_check = surface(p, r0, level, c, 2.95)
        up_equiv = surface(p, r0, level, c, 1.05)
        M = kernel_matrix(kernel, wavek, up_check, up_equiv)
        U, s, VH = np.linalg.svd(M)
        smax = np.max(np.abs(s))
        sinv = np.where(s > eps * smax * 4, 1.0 / np.where(s > 0, s, 1.0), 0.0)
        if not cplx:
            V = VH.T
            self.UC2E_U = U.T
            self.UC2E_V = V * sinv[None, :]
            self.DC2E_U = VH
            self.DC2E_V = U * sinv[None, :]
        else:
            V = VH.conj().T
            UH = U.conj().T
            self.UC2E_U = UH
            self.UC2E_V = V * sinv[None, :]
            self.DC2E_U = V.T
            self.DC2E_V = UH.T * sinv[None, :]
        # M2M / L2L (fmm_scale_invariant.h:51-77)
        sc = r0 * 0.5 ** (level + 1)
        self.M2M = np.zeros((8, n, n), dtype=M.dtype)
        self.L2L = np.zeros((8, n, n), dtype=M.dtype)
        for i, rc in enumerate(M2M_REL):
            child = surface(p, r0, level + 1, rc * sc, 1.05)
            pc2ce = kernel_matrix(kernel, wavek, up_check, child)
            self.M2M[i] = self.UC2E_V @ (self.UC2E_U @ pc2ce)
            self.L2L[i] = (pc2ce.T @ self.DC2E_V) @ self.DC2E_U
        # M2L tables for children at `m2l_level` (fmm_scale_invariant.h:517-558 / fmm.h:524-629)
        self.M2L = None
        if m2l_level is not None:
            self.M2L = m2l_tables(kernel, wavek, p, r0, m2l_level)


def m2l_tables(kernel, wavek, p, r0, l):
    """[26, nfreq, 64] complex; entry j = src_octant*8 + trg_octant, already divided by nconv.

    Laplace (scale invariant) uses l == 0 with offsets rel*2*r0; the per-level
    kernels use l = 1..depth with offsets rel*r0*0.5^(l-1)."""
    n1 = 2 * p
    nconv = n1 ** 3
    cplx = kernel == "helmholtz"
    helper = []
    for rel in M2LH_REL:
        coord = rel * (r0 / 0.5) if l == 0 else rel * r0 * 0.5 ** (l - 1)
        grid = convolution_grid(p, r0, l, coord)
        vals = kernel_matrix(kernel, wavek, grid, np.zeros((1, 3)))[:, 0]
        vals = vals.reshape(n1, n1, n1)
        helper.append((np.fft.fftn(vals) if cplx else np.fft.rfftn(vals)).reshape(-1))
    helper = np.array(helper)
    imap = m2l_index_map()
    nfreq = helper.shape[1]
    T = np.zeros((26, nfreq, 64), dtype=np.complex128)
    for i in range(26):
        for j in range(64):
            if imap[i, j] >= 0:
                T[i, :, j] = helper[imap[i, j]] / nconv
    return T


# ----------------------------------------------------------------------------- evaluate
class NpFmm:
    """Reference-semantics FMM on the oracle tree.  ``evaluate`` returns (ntrg, 4) in input order."""

    def __init__(self, kernel, p, ncrit, wavek=0.0, nonadaptive_depth=None, emulate=None, pinv_eps=1e-16):
        self.pinv_eps = pinv_eps
        assert kernel in KERNELS
        self.kernel, self.p, self.ncrit = kernel, p, ncrit
        self.wavek = complex(wavek)
        self.nonadaptive_depth = nonadaptive_depth
        self.nsurf = nsurf_of(p)
        self.emulate = emulate or (lambda stage, x: x)

    def setup(self, src, q, trg):
        from . import orc
        self.src = np.ascontiguousarray(src, np.float64)
        self.trg = np.ascontiguousarray(trg, np.float64)
        self.q = np.asarray(q, dtype=np.complex128 if self.kernel == "helmholtz" else np.float64)
        self.t = orc.build(self.src, self.trg, self.ncrit, self.nonadaptive_depth, self.nsurf)
        t = self.t
        self.depth = t["depth"]
        self.r0 = t["r0"]
        ni = t["ni"]
        self.level = ni[:, 1]
        self.is_leaf = ni[:, 2].astype(bool)
        self.nsrcs, self.ntrgs = ni[:, 3], ni[:, 4]
        self.child0 = ni[:, 7]
        self.center = t["nx"][:, :3]
        # body ranges of leaves in tree order
        nn = len(ni)
        self.sbeg = np.zeros(nn, np.int64)
        self.tbeg = np.zeros(nn, np.int64)
        so = to = 0
        for li in t["leafs"]:
            self.sbeg[li], self.tbeg[li] = so, to
            so += self.nsrcs[li]
            to += self.ntrgs[li]
        self.sx = self.src[t["src_perm"]]
        self.tx = self.trg[t["trg_perm"]]
        self.sq = self.q[t["src_perm"]]
        wk = self.wavek
        if self.kernel == "laplace":
            self.ops = {0: Operators(self.kernel, wk, self.p, self.r0, 0, m2l_level=0, eps=self.pinv_eps)}
        else:
            self.ops = {l: Operators(self.kernel, wk, self.p, self.r0, l,
                                     m2l_level=l if l >= 1 else None, eps=self.pinv_eps)
                        for l in range(self.depth + 1)}
        return self

    def _op(self, level):
        return self.ops[0] if self.kernel == "laplace" else self.ops[level]

    def leaf_src(self, i):
        return self.sx[self.sbeg[i]:self.sbeg[i] + self.nsrcs[i]], self.sq[self.sbeg[i]:self.sbeg[i] + self.nsrcs[i]]

    def leaf_trg(self, i):
        return self.tx[self.tbeg[i]:self.tbeg[i] + self.ntrgs[i]]

    def evaluate(self, charges=None):
        t, p, n = self.t, self.p, self.nsurf
        if charges is not None:
            self.q = np.asarray(charges, dtype=self.q.dtype)
            self.sq = self.q[t["src_perm"]]
        kern, wk, r0 = self.kernel, self.wavek, self.r0
        cplx = kern == "helmholtz"
        dt = np.complex128 if cplx else np.float64
        nn = len(self.level)
        up = np.zeros((nn, n), dt)
        dn = np.zeros((nn, n), dt)
        trg_val = np.zeros((len(self.trg), 4), dt)
        E = self.emulate
        c0 = np.zeros(3)
        leafs = t["leafs"]
        # ---- P2M
        for i in leafs:
            lv = self.level[i]
            chk = surface(p, r0, lv, c0, 2.95) + self.center[i]
            xs, qs = self.leaf_src(i)
            cp = potential(kern, wk, xs, qs, chk) if len(xs) else np.zeros(n, dt)
            cp = E("p2m_check", cp)
            op = self._op(lv)
            e = op.UC2E_V @ (op.UC2E_U @ cp)
            up[i] = (0.5 ** lv) * e if kern == "laplace" else e
            up[i] = E("p2m_equiv", up[i])
        # ---- M2M (post-order == deepest level first)
        for lv in range(self.depth - 1, -1, -1):
            for i in np.nonzero((self.level == lv) & ~self.is_leaf)[0]:
                op = self._op(lv)
                for oc in range(8):
                    up[i] += op.M2M[oc] @ up[self.child0[i] + oc]
                up[i] = E("m2m", up[i])
        # ---- P2L
        for i in range(nn):
            a, b = t["p2l_off"][i], t["p2l_off"][i + 1]
            if a == b:
                continue
            chk = surface(p, r0, self.level[i], c0, 1.05) + self.center[i]
            for s in t["p2l"][a:b]:
                xs, qs = self.leaf_src(s)
                dn[i] += potential(kern, wk, xs, qs, chk)
        # ---- M2P
        for i in leafs:
            a, b = t["m2p_off"][i], t["m2p_off"][i + 1]
            xt = self.leaf_trg(i)
            for s in t["m2p"][a:b]:
                eq = surface(p, r0, self.level[s], c0, 1.05) + self.center[s]
                trg_val[self.tbeg[i]:self.tbeg[i] + len(xt)] += gradient(kern, wk, eq, up[s], xt)
        # ---- P2P
        for i in leafs:
            a, b = t["p2p_off"][i], t["p2p_off"][i + 1]
            xt = self.leaf_trg(i)
            if not len(xt):
                continue
            srcs = t["p2p"][a:b]
            xs = np.concatenate([self.leaf_src(s)[0] for s in srcs]) if len(srcs) else np.zeros((0, 3))
            qs = np.concatenate([self.leaf_src(s)[1] for s in srcs]) if len(srcs) else np.zeros(0, dt)
            if len(xs):
                trg_val[self.tbeg[i]:self.tbeg[i] + len(xt)] += E("p2p", gradient(kern, wk, xs, qs, xt))
        # ---- M2L
        self._m2l(up, dn)
        # ---- L2L (pre-order == shallowest level first)
        for lv in range(0, self.depth):
            for i in np.nonzero((self.level == lv) & ~self.is_leaf)[0]:
                op = self._op(lv)
                for oc in range(8):
                    dn[self.child0[i] + oc] += E("l2l", op.L2L[oc] @ dn[i])
        # ---- L2P
        for i in leafs:
            lv = self.level[i]
            op = self._op(lv)
            e = op.DC2E_V @ (op.DC2E_U @ dn[i])
            e = (0.5 ** lv) * e if kern == "laplace" else e
            e = E("l2p_equiv", e)
            xt = self.leaf_trg(i)
            if len(xt):
                eq = surface(p, r0, lv, c0, 2.95) + self.center[i]
                trg_val[self.tbeg[i]:self.tbeg[i] + len(xt)] += gradient(kern, wk, eq, e, xt)
        self.up, self.dn = up, dn
        out = np.zeros_like(trg_val)
        out[t["trg_perm"]] = trg_val
        return out

    def _m2l(self, up, dn):
        t, p, n = self.t, self.p, self.nsurf
        n1 = 2 * p
        cplx = self.kernel == "helmholtz"
        mup, mdn = surf2conv(p, True), surf2conv(p, False)
        E = self.emulate
        nonleafs = t["nonleafs"]
        m2l = t["m2l"]
        lv_groups = [None] if self.kernel == "laplace" else list(range(self.depth))
        for lv in lv_groups:
            trgs = nonleafs if lv is None else nonleafs[self.level[nonleafs] == lv]
            if len(trgs) == 0:
                continue
            srcs = np.unique(m2l[trgs][m2l[trgs] >= 0])
            table = self.ops[0].M2L if lv is None else self.ops[lv + 1].M2L
            # fft_up_equiv
            spec = {}
            for s in srcs:
                grid = np.zeros((8, n1 ** 3), dtype=up.dtype)
                grid[:, mup] = up[self.child0[s]:self.child0[s] + 8]
                g = grid.reshape(8, n1, n1, n1)
                f = np.fft.fftn(g, axes=(1, 2, 3)) if cplx else np.fft.rfftn(g, axes=(1, 2, 3))
                spec[s] = E("m2l_in", f.reshape(8, -1).T)  # [freq, child]
            # hadamard + ifft_dn_check
            for tnode in trgs:
                acc = None
                for ipos in range(26):
                    s = m2l[tnode, ipos]
                    if s < 0:
                        continue
                    M = table[ipos].reshape(-1, 8, 8)  # [k, s_oct, t_oct]
                    contrib = np.einsum("kst,ks->kt", M, spec[s])
                    acc = contrib if acc is None else acc + contrib
                if acc is None:
                    continue
                acc = E("m2l_out", acc)
                f = acc.T.reshape(8, n1, n1, -1)
                if cplx:
                    g = np.fft.ifftn(f, axes=(1, 2, 3)) * n1 ** 3
                else:
                    g = np.fft.irfftn(f, s=(n1, n1, n1), axes=(1, 2, 3)) * n1 ** 3
                g = g.reshape(8, -1)[:, mdn]
                scale = 2.0 ** (self.level[tnode] + 1) if self.kernel == "laplace" else 1.0
                dn[self.child0[tnode]:self.child0[tnode] + 8] += g * scale
