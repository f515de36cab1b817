// capi.cpp -- the extern "C" boundary of libexafmm_b200.so (declared in include/xfmm.h).
// Every entry point catches all C++ exceptions and returns an xfmm_status; the message
// of the last failure on the calling thread is available from xfmm_last_error().
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "xfmm_internal.h"

struct xfmm_fmm {
  xfmm::Fmm f;
};
struct xfmm_tree {
  xfmm::Tree t;
};

namespace {
thread_local std::string g_err;

template <class F>
xfmm_status guarded(F&& fn) {
  try {
    fn();
    return XFMM_OK;
  } catch (const xfmm::Error& e) {
    g_err = e.msg;
    return (xfmm_status)e.code;
  } catch (const std::bad_alloc&) {
    g_err = "host allocation failed";
    return XFMM_ERR_OOM;
  } catch (const std::exception& e) {
    g_err = e.what();
    return XFMM_ERR_CUDA;
  } catch (...) {
    g_err = "unknown error";
    return XFMM_ERR_CUDA;
  }
}

inline cudaStream_t S(void* s) { return (cudaStream_t)s; }

// copy a host array to a temporary device buffer, or pass a device pointer through
struct DevIn {
  xfmm::DBuf<double> buf;
  const double* p = nullptr;
  DevIn(const double* src, size_t n, int on_device, cudaStream_t s) {
    if (on_device) {
      p = src;
    } else {
      buf.upload(src, n, s);
      p = buf.p;
    }
  }
};

void check_finite_host(const double* a, size_t n, const char* what) {
  for (size_t i = 0; i < n; i++)
    if (!std::isfinite(a[i])) throw xfmm::Error(XFMM_ERR_NUMERIC, std::string("non-finite value in ") + what);
}
}  // namespace

void xfmm::set_last_error(const char* msg) { g_err = msg; }

extern "C" {

const char* xfmm_last_error(void) { return g_err.c_str(); }
const char* xfmm_version(void) { return "exafmm-t_b200 0.1 (sm_100a)"; }

xfmm_status xfmm_fmm_create(int kernel, int p, int ncrit, double k_re, double k_im, int precision,
                            xfmm_fmm** out) {
  return guarded([&] {
    XREQUIRE(out, XFMM_ERR_ARG, "null output handle");
    XREQUIRE(kernel >= 0 && kernel <= 2, XFMM_ERR_ARG, "unknown kernel");
    XREQUIRE(p >= 2 && p <= 16, XFMM_ERR_UNSUPPORTED, "expansion order p must be in [2, 16]");
    XREQUIRE(ncrit >= 1, XFMM_ERR_ARG, "ncrit must be positive");
    XREQUIRE(precision == XFMM_FP64 || precision == XFMM_MIXED, XFMM_ERR_ARG, "unknown precision");
    XREQUIRE(std::isfinite(k_re) && std::isfinite(k_im), XFMM_ERR_ARG, "non-finite wavenumber");
    auto* h = new xfmm_fmm();
    xfmm::Fmm& f = h->f;
    f.kernel = kernel;
    f.p = p;
    f.ncrit = ncrit;
    f.k_re = k_re;
    f.k_im = kernel == XFMM_HELMHOLTZ ? k_im : 0.0;
    f.precision = precision;
    f.nsurf = xfmm::nsurf_of(p);  // fmm_base.h:30-35
    f.n1 = 2 * p;
    f.nconv = f.n1 * f.n1 * f.n1;
    f.nfreq = kernel == XFMM_HELMHOLTZ ? f.nconv : f.n1 * f.n1 * (f.n1 / 2 + 1);
    *out = h;
  });
}

xfmm_status xfmm_fmm_set_operator_file(xfmm_fmm* fmm, const char* filename) {
  return guarded([&] {
    XREQUIRE(fmm, XFMM_ERR_ARG, "null argument");
    fmm->f.filename = filename ? filename : "";
    fmm->f.precomputed = false;  // the next precompute reads (or writes) the file
  });
}

xfmm_status xfmm_fmm_free(xfmm_fmm* fmm) {
  return guarded([&] { delete fmm; });
}

xfmm_status xfmm_fmm_info(const xfmm_fmm* fmm, int64_t* i6, double* d4) {
  return guarded([&] {
    XREQUIRE(fmm && i6 && d4, XFMM_ERR_ARG, "null argument");
    const xfmm::Fmm& f = fmm->f;
    i6[0] = f.p;
    i6[1] = f.nsurf;
    i6[2] = f.nconv;
    i6[3] = f.nfreq;
    i6[4] = f.ncrit;
    i6[5] = f.depth;
    for (int d = 0; d < 3; d++) d4[d] = f.x0[d];
    d4[3] = f.r0;
  });
}

xfmm_status xfmm_build_tree(xfmm_fmm* fmm, const double* src_xyz, int64_t nsrc, const double* trg_xyz, int64_t ntrg,
                            int nonadaptive_depth, int on_device, void* stream, xfmm_tree** out) {
  return guarded([&] {
    XREQUIRE(fmm && out && src_xyz && trg_xyz, XFMM_ERR_ARG, "null argument");
    XREQUIRE(nsrc > 0 && ntrg > 0, XFMM_ERR_ARG, "need at least one source and one target");
    if (!on_device) {
      check_finite_host(src_xyz, 3 * (size_t)nsrc, "source coordinates");
      check_finite_host(trg_xyz, 3 * (size_t)ntrg, "target coordinates");
    }
    auto* h = new xfmm_tree();
    try {
      h->t.nsrc = nsrc;
      h->t.ntrg = ntrg;
      DevIn s(src_xyz, 3 * (size_t)nsrc, on_device, S(stream)), t(trg_xyz, 3 * (size_t)ntrg, on_device, S(stream));
      xfmm::build_tree(fmm->f, h->t, s.p, t.p, nonadaptive_depth, S(stream));
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

xfmm_status xfmm_tree_free(xfmm_tree* tree) {
  return guarded([&] { delete tree; });
}

xfmm_status xfmm_build_list(xfmm_fmm* fmm, xfmm_tree* tree, void* stream) {
  return guarded([&] {
    XREQUIRE(fmm && tree, XFMM_ERR_ARG, "null argument");
    xfmm::build_lists(fmm->f, tree->t, S(stream));
  });
}

xfmm_status xfmm_m2l_setup(xfmm_fmm* fmm, xfmm_tree* tree, void* stream) {
  return guarded([&] {
    XREQUIRE(fmm && tree, XFMM_ERR_ARG, "null argument");
    xfmm::m2l_setup(fmm->f, tree->t, S(stream));
  });
}

xfmm_status xfmm_precompute(xfmm_fmm* fmm, xfmm_tree* tree, void* stream) {
  return guarded([&] {
    XREQUIRE(fmm && tree, XFMM_ERR_ARG, "null argument");
    xfmm::Fmm& f = fmm->f;
    XREQUIRE(tree->t.r0 > 0, XFMM_ERR_STATE, "precompute before build_tree");
    f.r0 = tree->t.r0;
    f.depth = tree->t.depth;
    // cached operators are reused when r0 (and depth, for the per-level kernels) match (the load_matrix
    // check of fmm_scale_invariant.h:113-148, keyed on everything here); the scale-invariant Laplace
    // operators serve any r0 (the evaluate applies the ratio of the radii, op_scale in evaluate.cu)
    const bool same = f.precomputed && (f.kernel == XFMM_LAPLACE ? f.pre_r0 > 0 : f.pre_r0 == f.r0) &&
                      (f.kernel == XFMM_LAPLACE || f.pre_depth >= tree->t.depth);
    if (!same) xfmm::precompute(f, tree->t.depth, S(stream));
  });
}

xfmm_status xfmm_set_charges(xfmm_fmm* fmm, xfmm_tree* tree, const double* q, int on_device, void* stream) {
  return guarded([&] {
    XREQUIRE(fmm && tree && q, XFMM_ERR_ARG, "null argument");
    xfmm::set_charges(fmm->f, tree->t, q, on_device != 0, S(stream));
  });
}

xfmm_status xfmm_clear_values(xfmm_fmm* fmm, xfmm_tree* tree, void* stream) {
  return guarded([&] {
    XREQUIRE(fmm && tree, XFMM_ERR_ARG, "null argument");
    xfmm::clear_values(fmm->f, tree->t, S(stream));
  });
}

xfmm_status xfmm_upward_pass(xfmm_fmm* fmm, xfmm_tree* tree, void* stream) {
  return guarded([&] {
    XREQUIRE(fmm && tree, XFMM_ERR_ARG, "null argument");
    xfmm::upward_pass(fmm->f, tree->t, S(stream));
  });
}

xfmm_status xfmm_downward_pass(xfmm_fmm* fmm, xfmm_tree* tree, void* stream) {
  return guarded([&] {
    XREQUIRE(fmm && tree, XFMM_ERR_ARG, "null argument");
    xfmm::downward_pass(fmm->f, tree->t, S(stream));
  });
}

xfmm_status xfmm_get_values(xfmm_fmm* fmm, xfmm_tree* tree, double* out, int on_device, void* stream) {
  return guarded([&] {
    XREQUIRE(fmm && tree && out, XFMM_ERR_ARG, "null argument");
    const size_t n = (size_t)tree->t.ntrg * 4 * (fmm->f.is_complex() ? 2 : 1);
    if (on_device) {
      xfmm::get_values(fmm->f, tree->t, out, S(stream));
    } else {
      tree->t.stage_out.reserve(n);
      xfmm::get_values(fmm->f, tree->t, tree->t.stage_out.p, S(stream));
      XCUDA(cudaMemcpyAsync(out, tree->t.stage_out.p, n * sizeof(double), cudaMemcpyDeviceToHost, S(stream)));
      XCUDA(cudaStreamSynchronize(S(stream)));
      xfmm::check_device_status(fmm->f, tree->t);
    }
  });
}

xfmm_status xfmm_evaluate(xfmm_fmm* fmm, xfmm_tree* tree, double* out, int on_device, void* stream) {
  return guarded([&] {
    XREQUIRE(fmm && tree && out, XFMM_ERR_ARG, "null argument");
    xfmm::clear_values(fmm->f, tree->t, S(stream));
    xfmm::upward_pass(fmm->f, tree->t, S(stream));
    xfmm::downward_pass(fmm->f, tree->t, S(stream));
    const size_t n = (size_t)tree->t.ntrg * 4 * (fmm->f.is_complex() ? 2 : 1);
    if (on_device) {
      xfmm::get_values(fmm->f, tree->t, out, S(stream));
    } else {
      tree->t.stage_out.reserve(n);
      xfmm::get_values(fmm->f, tree->t, tree->t.stage_out.p, S(stream));
      XCUDA(cudaMemcpyAsync(out, tree->t.stage_out.p, n * sizeof(double), cudaMemcpyDeviceToHost, S(stream)));
      XCUDA(cudaStreamSynchronize(S(stream)));
      xfmm::check_device_status(fmm->f, tree->t);
    }
  });
}

xfmm_status xfmm_tree_info(const xfmm_tree* tree, int64_t* v) {
  return guarded([&] {
    XREQUIRE(tree && v, XFMM_ERR_ARG, "null argument");
    const xfmm::Tree& t = tree->t;
    v[0] = t.nnodes;
    v[1] = t.nleafs;
    v[2] = t.nnonleafs;
    v[3] = t.depth;
    v[4] = t.np2p;
    v[5] = t.nm2p;
    v[6] = t.np2l;
    v[7] = t.n_m2l_src;
    v[8] = t.p2p_pairs;
    v[9] = t.m2p_pairs;
    v[10] = t.l2p_pairs;
    v[11] = t.m2l_pairs;
  });
}

xfmm_status xfmm_tree_dump(const xfmm_tree* tree, double* geo, uint64_t* key, int32_t* ni, double* nx, int32_t* leafs,
                           int32_t* nonleafs, int32_t* src_perm, int32_t* trg_perm, int32_t* colleagues,
                           int32_t* m2l, int64_t* p2p_off, int32_t* p2p, int64_t* m2p_off, int32_t* m2p,
                           int64_t* p2l_off, int32_t* p2l) {
  return guarded([&] {
    XREQUIRE(tree, XFMM_ERR_ARG, "null argument");
    const xfmm::Tree& t = tree->t;
    XREQUIRE(t.lists_built, XFMM_ERR_STATE, "tree_dump before build_list");
    cudaStream_t s = 0;
    const int nn = t.nnodes;
    for (int d = 0; d < 3; d++) geo[d] = t.x0[d];
    geo[3] = t.r0;
    auto k = t.key.download(s);
    std::copy(k.begin(), k.end(), key);
    auto lv = t.level.download(s), il = t.is_leaf.download(s), ns = t.nsrcs.download(s), nt = t.ntrgs.download(s),
         pa = t.parent.download(s), oc = t.octant.download(s), c0 = t.child0.download(s);
    auto ct = t.center.download(s);
    for (int i = 0; i < nn; i++) {
      int32_t v[8] = {i, lv[i], il[i], ns[i], nt[i], pa[i], oc[i], il[i] ? -1 : c0[i]};
      for (int j = 0; j < 8; j++) ni[8 * (size_t)i + j] = v[j];
      nx[4 * (size_t)i] = ct[i].x;
      nx[4 * (size_t)i + 1] = ct[i].y;
      nx[4 * (size_t)i + 2] = ct[i].z;
      nx[4 * (size_t)i + 3] = ct[i].w;
    }
    std::copy(t.h_leafs.begin(), t.h_leafs.end(), leafs);
    std::copy(t.h_nonleafs.begin(), t.h_nonleafs.end(), nonleafs);
    auto sp = t.src_perm.download(s), tp = t.trg_perm.download(s), co = t.colleagues.download(s),
         ml = t.m2l.download(s);
    std::copy(sp.begin(), sp.end(), src_perm);
    std::copy(tp.begin(), tp.end(), trg_perm);
    std::copy(co.begin(), co.end(), colleagues);
    std::copy(ml.begin(), ml.end(), m2l);
    auto po = t.p2p_off.download(s), mo = t.m2p_off.download(s), xo = t.p2l_off.download(s);
    std::copy(po.begin(), po.end(), p2p_off);
    std::copy(mo.begin(), mo.end(), m2p_off);
    std::copy(xo.begin(), xo.end(), p2l_off);
    auto pl = t.p2p.download(s, t.np2p), mp = t.m2p.download(s, t.nm2p), xl = t.p2l.download(s, t.np2l);
    std::copy(pl.begin(), pl.end(), p2p);
    std::copy(mp.begin(), mp.end(), m2p);
    std::copy(xl.begin(), xl.end(), p2l);
  });
}

xfmm_status xfmm_selftest_bounded_wait(int64_t limit_cycles) {
  return guarded([&] { xfmm::selftest_bounded_wait(limit_cycles); });
}

xfmm_status xfmm_stage_times(xfmm_fmm* fmm, xfmm_tree* tree, double* ms14) {
  return guarded([&] {
    XREQUIRE(fmm && tree && ms14, XFMM_ERR_ARG, "null argument");
    xfmm::stage_times(fmm->f, tree->t, ms14);
  });
}

xfmm_status xfmm_set_tuning(xfmm_tree* tree, int option, int value) {
  return guarded([&] {
    XREQUIRE(tree, XFMM_ERR_ARG, "null argument");
    XREQUIRE(option == XFMM_TUNE_SPARSE_HADAMARD_TILES_PER_CTA, XFMM_ERR_ARG, "unknown tuning option");
    XREQUIRE(value >= 0 && value <= 64, XFMM_ERR_ARG, "sparse Hadamard tiles per CTA must be 0..64");
    tree->t.hadr_tpc = value;
  });
}

xfmm_status xfmm_batch_create(xfmm_fmm* const* fmms, xfmm_tree* const* trees, int n, void* stream, xfmm_batch** out) {
  return guarded([&] {
    XREQUIRE(fmms && trees && out && n > 0, XFMM_ERR_ARG, "null argument");
    std::vector<xfmm::Fmm*> f(n);
    std::vector<xfmm::Tree*> t(n);
    for (int k = 0; k < n; k++) {
      XREQUIRE(fmms[k] && trees[k], XFMM_ERR_ARG, "null system handle");
      f[k] = &fmms[k]->f;
      t[k] = &trees[k]->t;
    }
    *out = reinterpret_cast<xfmm_batch*>(xfmm::batch_create(f.data(), t.data(), n, S(stream)));
  });
}

xfmm_status xfmm_batch_evaluate(xfmm_batch* b, const double* const* charges, double* const* outs, int nstreams,
                                void* stream) {
  return guarded([&] {
    XREQUIRE(b && outs, XFMM_ERR_ARG, "null argument");
    xfmm::batch_evaluate(reinterpret_cast<xfmm::Batch*>(b), charges, outs, nstreams, S(stream));
  });
}

xfmm_status xfmm_batch_set_tuning(xfmm_batch* b, int option, int value) {
  return guarded([&] {
    XREQUIRE(b, XFMM_ERR_ARG, "null argument");
    xfmm::batch_set_tuning(reinterpret_cast<xfmm::Batch*>(b), option, value);
  });
}

xfmm_status xfmm_batch_free(xfmm_batch* b) {
  return guarded([&] { xfmm::batch_free(reinterpret_cast<xfmm::Batch*>(b)); });
}

xfmm_status xfmm_batch_schedule(const int64_t* sizes, int n, int nstreams, int* stream_of) {
  return guarded([&] {
    XREQUIRE((sizes && stream_of) || n == 0, XFMM_ERR_ARG, "null argument");
    xfmm::batch_schedule(sizes, n, nstreams, stream_of);
  });
}

xfmm_status xfmm_gradient_p2p(int kernel, double k_re, double k_im, int precision, const double* src_xyz,
                              int64_t nsrc, const double* q, const double* trg_xyz, int64_t ntrg, double* out,
                              int on_device, void* stream) {
  return guarded([&] {
    XREQUIRE(kernel >= 0 && kernel <= 2, XFMM_ERR_ARG, "unknown kernel");
    XREQUIRE(nsrc >= 0 && ntrg >= 0, XFMM_ERR_ARG, "negative size");
    XREQUIRE(precision == XFMM_FP64 || precision == XFMM_MIXED, XFMM_ERR_ARG, "unknown precision");
    if (ntrg == 0) return;
    XREQUIRE(src_xyz && q && trg_xyz && out, XFMM_ERR_ARG, "null argument");
    const int vs = kernel == XFMM_HELMHOLTZ ? 2 : 1;
    cudaStream_t s = S(stream);
    DevIn sx(src_xyz, 3 * (size_t)nsrc, on_device, s), tx(trg_xyz, 3 * (size_t)ntrg, on_device, s),
        qq(q, (size_t)nsrc * vs, on_device, s);
    xfmm::DBuf<double> tmp;
    double* o = out;
    const size_t nout = (size_t)ntrg * 4 * vs;
    if (!on_device) {
      tmp.upload(out, nout, s);
      o = tmp.p;
    }
    xfmm::gradient_p2p_raw(kernel, k_re, k_im, precision, sx.p, nsrc, qq.p, tx.p, ntrg, o, s);
    if (!on_device) {
      XCUDA(cudaMemcpyAsync(out, o, nout * sizeof(double), cudaMemcpyDeviceToHost, s));
      XCUDA(cudaStreamSynchronize(s));
    }
  });
}

xfmm_status xfmm_verify(xfmm_fmm* fmm, xfmm_tree* tree, int sample, double* err2, void* stream) {
  return guarded([&] {
    XREQUIRE(fmm && tree && err2, XFMM_ERR_ARG, "null argument");
    xfmm::verify(fmm->f, tree->t, sample, err2, S(stream));
  });
}

}  // extern "C"
