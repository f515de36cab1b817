"""Many independent particle systems evaluated as one captured CUDA graph (no counterpart in the
reference, which evaluates one system per call).

Each system gets its own tree, lists and device buffers for its charges and results.  Laplace systems
share one Fmm object: its scale-invariant operators, precomputed once for the first system's root radius,
serve every other radius (the evaluate scales the body-to-check potentials by the ratio of the radii);
the other kernels' operators depend on the radius, so each of those systems gets its own Fmm object.
With one shared operator table (mixed Laplace) the work that shares it is one launch over all systems:
the pseudo-inverse factors of P2M and L2P, the M2M and L2L of each level, the sparse M2L Hadamard between
the systems' forward and backward M2L transforms, and the far field.  The systems are held by one native batch (xfmm_batch_*):
one evaluate of every system runs each system's stages before and after its near field on concurrent
streams forked from the batch stream (largest systems first, each to the least-loaded stream), and the
near field of all systems as one persistent kernel that drains a work queue of (system, target leaf)
items, largest first, followed by one launch of the close-pair corrections of all systems.  That
evaluate is captured once into a CUDA graph and replayed with a single launch; ``evaluate_each`` runs
the per-system evaluates one after another without the graph or the batch.  Charges are read from
``charges[i]`` (device tensors) at every replay, so new values are picked up by writing into those
tensors in place.  The work runs on the batch's own stream, ordered after the caller's current stream,
which in turn waits for it: results may be read on the current stream.

``autotune()`` captures the graph for each candidate stream count and each candidate tile shape of the
persistent near-field kernel (CTAs per SM; targets per lane, the height of a warp's target tile), times
replays on the device and keeps the fastest; then, with those, it does the same for the sparse M2L
Hadamard's target tiles per CTA (set on every tree through xfmm_set_tuning).
"""
import ctypes

import numpy as np
import torch

from . import _core, _lib

NEAR_CTAS_PER_SM, NEAR_TARGETS_PER_LANE, HADAMARD_TILES_PER_CTA = 1, 2, 3  # include/xfmm.h XFMM_BATCH_*


class BatchedFmm:
    """systems: list of (coords (n, 3) array, charges (n,) array); fmm_factory() -> a new Fmm object."""

    def __init__(self, systems, fmm_factory, nonadaptive_depth=None, share_operators=True):
        self.fmms, self.trees, self.charges, self.outs = [], [], [], []
        shared = None
        for coords, q in systems:
            # the scale-invariant Laplace operators serve every system of the batch (one precompute)
            fmm = shared if shared is not None else fmm_factory()
            if share_operators and fmm.kernel == "laplace":
                shared = fmm
            dtype = np.complex128 if fmm.kernel == "helmholtz" else np.float64
            src = _core.init_sources(coords, np.asarray(q, dtype), fmm.kernel)
            tree = _core.setup(src, _core.init_targets(coords), fmm, nonadaptive_depth)
            qt = torch.tensor(np.asarray(q, dtype), device="cuda")
            if qt.is_complex():
                qt = torch.view_as_real(qt).reshape(-1)
            width = 8 if fmm.kernel == "helmholtz" else 4
            self.fmms.append(fmm)
            self.trees.append(tree)
            self.charges.append(qt)
            self.outs.append(torch.zeros((len(coords), width), dtype=torch.float64, device="cuda"))
        self.n = [len(c) for c, _ in systems]
        self.stream = torch.cuda.Stream()
        k = len(self.n)
        fa = (ctypes.c_void_p * k)(*[f._h.value for f in self.fmms])
        ta = (ctypes.c_void_p * k)(*[t._h.value for t in self.trees])
        self._qp = (ctypes.c_void_p * k)(*[q.data_ptr() for q in self.charges])
        self._op = (ctypes.c_void_p * k)(*[o.data_ptr() for o in self.outs])
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().xfmm_batch_create(fa, ta, k, ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h)))
        self._b = h
        self.graph = None
        self.nstreams = 1
        self.near_ctas_per_sm, self.near_tpl = 0, 2  # persistent near field (0: as many CTAs as fit)
        self.tuning = {}        # (streams, CTAs per SM, targets per lane) -> ms per replay
        self.tiles_per_cta = 0  # sparse Hadamard tiles per CTA on every tree (0: the library default)
        self.tile_tuning = {}   # tiles per CTA -> ms per replay, with the chosen shape

    @property
    def n_operator_sets(self):
        """Distinct Fmm objects (operator sets) the systems use."""
        return len({id(f) for f in self.fmms})

    def __del__(self):
        b = getattr(self, "_b", None)
        if b is None or not b.value:
            return
        self.graph = None
        self._b = None
        try:
            _lib.lib().xfmm_batch_free(b)
        except (AttributeError, TypeError):  # interpreter shutdown: the library module is already gone
            pass

    def set_near_shape(self, ctas_per_sm, targets_per_lane):
        """Tile shape of the persistent near-field kernel; recapture after."""
        L = _lib.lib()
        _lib.check(L.xfmm_batch_set_tuning(self._b, NEAR_CTAS_PER_SM, int(ctas_per_sm)))
        _lib.check(L.xfmm_batch_set_tuning(self._b, NEAR_TARGETS_PER_LANE, int(targets_per_lane)))
        self.near_ctas_per_sm, self.near_tpl = int(ctas_per_sm), int(targets_per_lane)

    def _batch(self, nstreams):
        _lib.check(_lib.lib().xfmm_batch_evaluate(self._b, self._qp, self._op, int(nstreams),
                                                  ctypes.c_void_p(self.stream.cuda_stream)))

    def _enqueue(self, stream_handle):
        L = _lib.lib()
        st = ctypes.c_void_p(stream_handle)
        for i in range(len(self.n)):
            fmm, tree, q, out = self.fmms[i], self.trees[i], self.charges[i], self.outs[i]
            _lib.check(L.xfmm_set_charges(fmm._h, tree._h, ctypes.c_void_p(q.data_ptr()), 1, st))
            _lib.check(L.xfmm_evaluate(fmm._h, tree._h, ctypes.c_void_p(out.data_ptr()), 1, st))

    def evaluate_each(self):
        """One evaluate per system, launched one after another on the batch stream (no graph, no batch)."""
        self.stream.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(self.stream):
            self._enqueue(self.stream.cuda_stream)
        torch.cuda.current_stream().wait_stream(self.stream)
        return self.outs

    def evaluate_batch(self, nstreams=None):
        """One batched evaluate of every system (no graph)."""
        self.stream.wait_stream(torch.cuda.current_stream())
        self._batch(self.nstreams if nstreams is None else nstreams)
        torch.cuda.current_stream().wait_stream(self.stream)
        return self.outs

    def capture(self, nstreams=1):
        """Capture one batched evaluate of every system into a CUDA graph, the per-system stages spread
        over nstreams concurrent streams.  One evaluate runs here first, outside the capture."""
        self.evaluate_batch(nstreams)
        self.stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.stream):
            self._batch(int(nstreams))
        self.graph = g
        self.nstreams = int(nstreams)
        return g

    def _time_graph(self, g, reps):
        self.replay()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        for _ in range(reps):
            with torch.cuda.stream(self.stream):
                g.replay()
        e1.record(self.stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    def set_tiles_per_cta(self, value):
        """Sparse M2L Hadamard tiles per CTA (0: the library default) of the batch's one-launch Hadamard
        (systems sharing one operator set) and of every tree's own; recapture after."""
        for tree in self.trees:
            tree.set_tuning("sparse_hadamard_tiles_per_cta", value)
        _lib.check(_lib.lib().xfmm_batch_set_tuning(self._b, HADAMARD_TILES_PER_CTA, int(value)))
        self.tiles_per_cta = int(value)

    def autotune(self, candidates=(4, 8, 16, 32), near_shapes=((0, 2), (4, 2), (0, 1), (2, 2)), reps=3,
                 tile_candidates=(1, 2, 4, 8)):
        """Capture the graph for each stream count in candidates and each persistent near-field shape
        (CTAs per SM, targets per lane) in near_shapes, time `reps` replays of each on the device (after
        one untimed replay) and keep the fastest; then, with those, the same for each sparse-Hadamard
        tiles-per-CTA value in tile_candidates.  self.tuning maps each (streams, CTAs per SM, targets per
        lane), self.tile_tuning each tile value, to its milliseconds per replay."""
        best = None
        for ns in candidates:
            ns = max(1, min(int(ns), len(self.n)))
            for cps, tpl in near_shapes:
                key = (ns, int(cps), int(tpl))
                if key in self.tuning:
                    continue
                self.set_near_shape(cps, tpl)
                g = self.capture(ns)
                self.tuning[key] = self._time_graph(g, reps)
                if best is None or self.tuning[key] < self.tuning[best]:
                    best = key
                del g
                self.graph = None
        if best is None:
            best = min(self.tuning, key=self.tuning.get)
        self.set_near_shape(best[1], best[2])
        self.capture(best[0])
        if tile_candidates:
            best_ms, best_tiles = None, self.tiles_per_cta
            for tiles in tile_candidates:
                self.set_tiles_per_cta(tiles)
                g = self.capture(self.nstreams)
                self.tile_tuning[int(tiles)] = self._time_graph(g, reps)
                if best_ms is None or self.tile_tuning[int(tiles)] < best_ms:
                    best_ms, best_tiles = self.tile_tuning[int(tiles)], int(tiles)
            self.set_tiles_per_cta(best_tiles)
            self.capture(self.nstreams)
        return self.nstreams

    def replay(self):
        """All systems in one graph launch (capture() first)."""
        if self.graph is None:
            raise RuntimeError("capture() before replay()")
        self.stream.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(self.stream):
            self.graph.replay()
        torch.cuda.current_stream().wait_stream(self.stream)
        return self.outs


def plummer(n, rng, a=1.0, rmax=10.0):
    """n points of a Plummer sphere with scale radius a, truncated at radius rmax."""
    r = np.empty(0)
    while r.size < n:
        u = rng.random(2 * n)
        rr = a / np.sqrt(np.maximum(u, 1e-300) ** (-2.0 / 3.0) - 1.0)
        r = np.concatenate([r, rr[rr <= rmax]])
    r = r[:n]
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True) * r[:, None]


def batched_workload(nsys=256, nmin=2000, nmax=200000, seed=0):
    """The batched configuration: sizes log-uniform in [nmin, nmax], half uniform-cube and half
    Plummer systems, charges U[-1, 1)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(nmin), np.log(nmax), nsys)).astype(np.int64)
    systems = []
    for i, n in enumerate(sizes):
        x = rng.random((n, 3)) if i % 2 == 0 else plummer(int(n), rng)
        systems.append((x, rng.uniform(-1.0, 1.0, n)))
    return systems
