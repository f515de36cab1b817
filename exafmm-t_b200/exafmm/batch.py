"""Many independent particle systems evaluated as one captured CUDA graph (no counterpart in the
reference, which evaluates one system per call).

Each system gets its own Fmm object (operators depend on the system's bounding box), tree, lists and
device buffers for its charges and results.  One evaluate of every system (charges in, potentials
and gradients out, all device-resident) is captured once into a CUDA graph and then replayed with a
single launch; ``evaluate_each`` runs the same calls one system after another without the graph.
Charges are read from ``charges[i]`` (device tensors) at every replay, so new values are picked up
by writing into those tensors in place.  The work runs on the batch's own stream, ordered after the
caller's current stream, which in turn waits for it: results may be read on the current stream.

Inside the graph the systems may run concurrently: ``capture(nstreams)`` forks the batch stream into
``nstreams`` streams (each system's calls stay in order on one of them; systems are dealt, largest
first, to the stream with the fewest bodies so far) and joins them again, so the small grids of small
systems share the GPU instead of running one after another.  Every system owns its operators, tree,
work buffers and library handles (cuBLAS with a fixed workspace), so nothing is shared between the
streams.  ``autotune()`` captures the graph for each candidate stream count, times replays on the
device and keeps the fastest; then, at that stream count, it does the same for each candidate tile
shape of the sparse M2L Hadamard (target tiles per CTA, set on every tree through xfmm_set_tuning).
"""
import ctypes

import numpy as np
import torch

from . import _core, _lib


class BatchedFmm:
    """systems: list of (coords (n, 3) array, charges (n,) array); fmm_factory() -> a new Fmm object."""

    def __init__(self, systems, fmm_factory, nonadaptive_depth=None):
        self.fmms, self.trees, self.charges, self.outs = [], [], [], []
        for coords, q in systems:
            fmm = fmm_factory()
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
        self._side = []
        self.graph = None
        self.nstreams = 1
        self.tuning = {}        # stream count -> ms per replay
        self.tiles_per_cta = 0  # sparse Hadamard tiles per CTA on every tree (0: the library default)
        self.tile_tuning = {}   # tiles per CTA -> ms per replay, at the chosen stream count

    def _enqueue(self, stream_handle, order=None):
        L = _lib.lib()
        st = ctypes.c_void_p(stream_handle)
        for i in (range(len(self.n)) if order is None else order):
            fmm, tree, q, out = self.fmms[i], self.trees[i], self.charges[i], self.outs[i]
            _lib.check(L.xfmm_set_charges(fmm._h, tree._h, ctypes.c_void_p(q.data_ptr()), 1, st))
            _lib.check(L.xfmm_evaluate(fmm._h, tree._h, ctypes.c_void_p(out.data_ptr()), 1, st))

    def _deal(self, nstreams):
        """Systems per stream: largest first, each to the stream with the fewest bodies so far."""
        load, lists = [0] * nstreams, [[] for _ in range(nstreams)]
        for i in sorted(range(len(self.n)), key=lambda i: -self.n[i]):
            k = min(range(nstreams), key=lambda k: load[k])
            lists[k].append(i)
            load[k] += self.n[i]
        return [l for l in lists if l]

    def _enqueue_forked(self, nstreams):
        """All systems on nstreams streams forked from and joined back into the batch stream."""
        if nstreams <= 1:
            self._enqueue(self.stream.cuda_stream)
            return
        while len(self._side) < nstreams:
            self._side.append(torch.cuda.Stream())
        fork = torch.cuda.Event()
        fork.record(self.stream)
        for k, order in enumerate(self._deal(nstreams)):
            side = self._side[k]
            side.wait_event(fork)
            self._enqueue(side.cuda_stream, order)
            join = torch.cuda.Event()
            join.record(side)
            self.stream.wait_event(join)

    def evaluate_each(self):
        """One evaluate per system, launched one after another on the batch stream (no graph)."""
        self.stream.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(self.stream):
            self._enqueue(self.stream.cuda_stream)
        torch.cuda.current_stream().wait_stream(self.stream)
        return self.outs

    def capture(self, nstreams=1):
        """Capture one evaluate of every system into a CUDA graph, the systems spread over nstreams
        concurrent streams.  The first evaluate of each system (which sizes its work buffers) runs
        here, before the capture begins."""
        self.evaluate_each()
        self.stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.stream):
            self._enqueue_forked(int(nstreams))
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
        """Sparse M2L Hadamard tiles per CTA on every tree (0: the library default); recapture after."""
        for tree in self.trees:
            tree.set_tuning("sparse_hadamard_tiles_per_cta", value)
        self.tiles_per_cta = int(value)

    def autotune(self, candidates=(1, 2, 4, 8, 16, 32), reps=3, tile_candidates=(1, 2, 4, 8)):
        """Capture the graph for each stream count in candidates, time `reps` replays of each on the
        device (after one untimed replay) and keep the fastest graph; then, at that stream count, the
        same for each sparse-Hadamard tiles-per-CTA value in tile_candidates.  self.tuning maps each
        stream count, self.tile_tuning each tile value, to its milliseconds per replay."""
        self._autotune_streams(candidates, reps)
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

    def _autotune_streams(self, candidates, reps):
        best = None
        for ns in candidates:
            ns = max(1, min(int(ns), len(self.n)))
            if ns in self.tuning:
                continue
            g = self.capture(ns)
            self.tuning[ns] = self._time_graph(g, reps)
            if best is None or self.tuning[ns] < self.tuning[best[0]]:
                best = (ns, g)
            else:
                del g
        if best is not None:
            self.nstreams, self.graph = best
        else:  # every candidate timed before: recapture the fastest
            self.capture(min(self.tuning, key=self.tuning.get))
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
