// ref_capi.cpp -- C ABI over the UNMODIFIED exafmm-t reference headers.
//
// Test infrastructure only.  Compiled by oracle/Makefile against the reference's
// own include/ directory into oracle/_ref/libxfmm_ref{,_na}.so, it lets the tests
// and the CPU-baseline leg of bench.py drive the reference's stock code path:
//   setup    = python/exafmm.cpp:129-180 (get_bounds, build_tree [+balance_tree],
//              init_rel_coord, set_colleagues, build_list, M2L_setup, precompute)
//   evaluate = fmm_base.h:162-200 (upward_pass + downward_pass), stage by stage so
//              that each stage can be timed, then the scatter of
//              python/exafmm.cpp:190-267 back to the original target order.
// Built twice: adaptive (build_tree.h) and -DNON_ADAPTIVE (build_non_adaptive_tree.h).
#include <omp.h>

#include <cstdint>
#include <cstring>
#include <string>

#include "exafmm_t.h"
#if NON_ADAPTIVE
#include "build_non_adaptive_tree.h"
#else
#include "build_tree.h"
#endif
#include "build_list.h"
#include "helmholtz.h"
#include "laplace.h"
#include "modified_helmholtz.h"

using namespace exafmm_t;

namespace {

struct Base {
  int kernel = 0;
  virtual ~Base() {}
};

template <typename T, typename F>
struct Handle : Base {
  F fmm;
  Bodies<T> sources, targets;
  Nodes<T> nodes;
  NodePtrs<T> leafs, nonleafs;
  int nsrc = 0, ntrg = 0;
  explicit Handle(const F& f) : fmm(f) {}
};

template <typename T>
inline T make_value(const double* q, int i);
template <>
inline real_t make_value<real_t>(const double* q, int i) { return q[i]; }
template <>
inline complex_t make_value<complex_t>(const double* q, int i) { return complex_t(q[2 * i], q[2 * i + 1]); }

template <typename T>
inline void put_value(double* out, size_t i, const T& v);
template <>
inline void put_value<real_t>(double* out, size_t i, const real_t& v) { out[i] = v; }
template <>
inline void put_value<complex_t>(double* out, size_t i, const complex_t& v) {
  out[2 * i] = v.real();
  out[2 * i + 1] = v.imag();
}

template <typename T, typename F>
int setup(Handle<T, F>* h, int nsrc, const double* sxyz, const double* sq, int ntrg, const double* txyz,
          int nonadaptive_depth) {
  h->nsrc = nsrc;
  h->ntrg = ntrg;
  h->sources.resize(nsrc);
  h->targets.resize(ntrg);
  for (int i = 0; i < nsrc; i++) {
    for (int d = 0; d < 3; d++) h->sources[i].X[d] = sxyz[3 * i + d];
    h->sources[i].q = make_value<T>(sq, i);
    h->sources[i].ibody = i;
  }
  for (int i = 0; i < ntrg; i++) {
    for (int d = 0; d < 3; d++) h->targets[i].X[d] = txyz[3 * i + d];
    h->targets[i].ibody = i;
  }
  F& fmm = h->fmm;
  get_bounds<T>(h->sources, h->targets, fmm.x0, fmm.r0);
#if NON_ADAPTIVE
  fmm.depth = nonadaptive_depth;
  h->nodes = build_tree<T>(h->sources, h->targets, h->leafs, h->nonleafs, fmm);
#else
  (void)nonadaptive_depth;
  h->nodes = build_tree<T>(h->sources, h->targets, h->leafs, h->nonleafs, fmm);
  balance_tree(h->nodes, h->sources, h->targets, h->leafs, h->nonleafs, fmm);
#endif
  init_rel_coord();
  set_colleagues<T>(h->nodes);
  build_list<T>(h->nodes, fmm);
  fmm.M2L_setup(h->nonleafs);
  fmm.precompute();
  return 0;
}

template <typename T, typename F>
int evaluate(Handle<T, F>* h, double* out, double* t) {
  F& fmm = h->fmm;
  double s[9];
  s[0] = omp_get_wtime();
  fmm.P2M(h->leafs);
  s[1] = omp_get_wtime();
#pragma omp parallel
#pragma omp single nowait
  fmm.M2M(&h->nodes[0]);
  s[2] = omp_get_wtime();
  fmm.P2L(h->nodes);
  s[3] = omp_get_wtime();
  fmm.M2P(h->leafs);
  s[4] = omp_get_wtime();
  fmm.P2P(h->leafs);
  s[5] = omp_get_wtime();
  fmm.M2L(h->nodes);
  s[6] = omp_get_wtime();
#pragma omp parallel
#pragma omp single nowait
  fmm.L2L(&h->nodes[0]);
  s[7] = omp_get_wtime();
  fmm.L2P(h->leafs);
  s[8] = omp_get_wtime();
  if (t)
    for (int i = 0; i < 8; i++) t[i] = s[i + 1] - s[i];
  if (out) {
    for (size_t i = 0; i < h->leafs.size(); ++i) {
      Node<T>* leaf = h->leafs[i];
      for (size_t j = 0; j < leaf->itrgs.size(); ++j)
        for (int c = 0; c < 4; c++) put_value<T>(out, (size_t)leaf->itrgs[j] * 4 + c, leaf->trg_value[4 * j + c]);
    }
  }
  return 0;
}

template <typename T, typename F>
void clear_values(Handle<T, F>* h) {
  for (auto& node : h->nodes) {
    std::fill(node.up_equiv.begin(), node.up_equiv.end(), T(0.));
    std::fill(node.dn_equiv.begin(), node.dn_equiv.end(), T(0.));
    if (node.is_leaf) std::fill(node.trg_value.begin(), node.trg_value.end(), T(0.));
  }
}

template <typename T, typename F>
void update_charges(Handle<T, F>* h, const double* q) {
  for (auto leaf : h->leafs)
    for (size_t j = 0; j < leaf->isrcs.size(); ++j) leaf->src_value[j] = make_value<T>(q, leaf->isrcs[j]);
}

template <typename T, typename F>
void sizes(Handle<T, F>* h, int64_t* s) {
  int64_t np2p = 0, nm2p = 0, np2l = 0;
  for (auto& n : h->nodes) {
    np2p += n.P2P_list.size();
    nm2p += n.M2P_list.size();
    np2l += n.P2L_list.size();
  }
  s[0] = h->nodes.size();
  s[1] = h->leafs.size();
  s[2] = h->nonleafs.size();
  s[3] = h->fmm.depth;
  s[4] = np2p;
  s[5] = nm2p;
  s[6] = np2l;
  s[7] = h->fmm.nsurf;
}

template <typename T, typename F>
void dump(Handle<T, F>* h, double* geo /* 6: x0[3], r0, 0, 0 */, uint64_t* key, int32_t* ni /* nnodes*8 */,
          double* nx /* nnodes*4 */, int32_t* leafs, int32_t* nonleafs, int32_t* src_perm, int32_t* trg_perm,
          int32_t* colleagues /* nnodes*27 */, int32_t* m2l /* nnodes*26 */, int64_t* p2p_off, int32_t* p2p,
          int64_t* m2p_off, int32_t* m2p, int64_t* p2l_off, int32_t* p2l) {
  const size_t nn = h->nodes.size();
  Node<T>* base = &h->nodes[0];
  for (int d = 0; d < 3; d++) geo[d] = h->fmm.x0[d];
  geo[3] = h->fmm.r0;
  int64_t o1 = 0, o2 = 0, o3 = 0;
  for (size_t i = 0; i < nn; i++) {
    Node<T>& n = h->nodes[i];
    key[i] = n.key;
    ni[8 * i + 0] = (int32_t)n.idx;
    ni[8 * i + 1] = n.level;
    ni[8 * i + 2] = n.is_leaf ? 1 : 0;
    ni[8 * i + 3] = n.nsrcs;
    ni[8 * i + 4] = n.ntrgs;
    ni[8 * i + 5] = n.parent ? (int32_t)(n.parent - base) : -1;
    ni[8 * i + 6] = n.octant;
    ni[8 * i + 7] = (!n.is_leaf && !n.children.empty()) ? (int32_t)(n.children[0] - base) : -1;
    for (int d = 0; d < 3; d++) nx[4 * i + d] = n.x[d];
    nx[4 * i + 3] = n.r;
    for (int c = 0; c < 27; c++)
      colleagues[27 * i + c] = (c < (int)n.colleagues.size() && n.colleagues[c]) ? (int32_t)(n.colleagues[c] - base) : -1;
    for (int c = 0; c < 26; c++)
      m2l[26 * i + c] = (c < (int)n.M2L_list.size() && n.M2L_list[c]) ? (int32_t)(n.M2L_list[c] - base) : -1;
    p2p_off[i] = o1;
    for (auto s : n.P2P_list) p2p[o1++] = (int32_t)(s - base);
    m2p_off[i] = o2;
    for (auto s : n.M2P_list) m2p[o2++] = (int32_t)(s - base);
    p2l_off[i] = o3;
    for (auto s : n.P2L_list) p2l[o3++] = (int32_t)(s - base);
  }
  p2p_off[nn] = o1;
  m2p_off[nn] = o2;
  p2l_off[nn] = o3;
  for (size_t i = 0; i < h->leafs.size(); i++) leafs[i] = (int32_t)(h->leafs[i] - base);
  for (size_t i = 0; i < h->nonleafs.size(); i++) nonleafs[i] = (int32_t)(h->nonleafs[i] - base);
  size_t a = 0, b = 0;
  for (auto leaf : h->leafs) {
    for (int s : leaf->isrcs) src_perm[a++] = s;
    for (int t : leaf->itrgs) trg_perm[b++] = t;
  }
}

typedef Handle<real_t, LaplaceFmm> HL;
typedef Handle<real_t, ModifiedHelmholtzFmm> HY;
typedef Handle<complex_t, HelmholtzFmm> HH;

}  // namespace

#define DISPATCH(h, call)                      \
  switch (((Base*)(h))->kernel) {              \
    case 0: { HL* x = (HL*)(h); call; break; } \
    case 1: { HY* x = (HY*)(h); call; break; } \
    default: { HH* x = (HH*)(h); call; break; } \
  }

extern "C" {

// kernel: 0 = Laplace, 1 = modified Helmholtz (k_re), 2 = Helmholtz (k_re + i k_im)
void* ref_create(int kernel, int p, int ncrit, double k_re, double k_im, const char* datfile) {
  std::string fn = datfile ? std::string(datfile) : std::string();
  Base* b = nullptr;
  if (kernel == 0) b = new HL(LaplaceFmm(p, ncrit, fn));
  else if (kernel == 1) b = new HY(ModifiedHelmholtzFmm(p, ncrit, (real_t)k_re, fn));
  else b = new HH(HelmholtzFmm(p, ncrit, complex_t(k_re, k_im), fn));
  b->kernel = kernel;
  return b;
}

int ref_setup(void* h, int nsrc, const double* sxyz, const double* sq, int ntrg, const double* txyz, int depth) {
  DISPATCH(h, setup(x, nsrc, sxyz, sq, ntrg, txyz, depth));
  return 0;
}

int ref_evaluate(void* h, double* out, double* stage_times) {
  DISPATCH(h, evaluate(x, out, stage_times));
  return 0;
}

void ref_clear_values(void* h) { DISPATCH(h, clear_values(x)); }
void ref_update_charges(void* h, const double* q) { DISPATCH(h, update_charges(x, q)); }
void ref_sizes(void* h, int64_t* s) { DISPATCH(h, sizes(x, s)); }

void ref_dump(void* h, double* geo, uint64_t* key, int32_t* ni, double* nx, int32_t* leafs, int32_t* nonleafs,
              int32_t* src_perm, int32_t* trg_perm, int32_t* colleagues, int32_t* m2l, int64_t* p2p_off,
              int32_t* p2p, int64_t* m2p_off, int32_t* m2p, int64_t* p2l_off, int32_t* p2l) {
  DISPATCH(h, dump(x, geo, key, ni, nx, leafs, nonleafs, src_perm, trg_perm, colleagues, m2l, p2p_off, p2p,
                   m2p_off, m2p, p2l_off, p2l));
}

int ref_verify(void* h, int sample, double* err2) {
  RealVec e;
  DISPATCH(h, e = x->fmm.verify(x->leafs, sample != 0));
  err2[0] = e[0];
  err2[1] = e[1];
  return 0;
}

void ref_free(void* h) {
  switch (((Base*)h)->kernel) {
    case 0: delete (HL*)h; break;
    case 1: delete (HY*)h; break;
    default: delete (HH*)h; break;
  }
}

// gradient_P2P of the reference kernels (laplace.h:91-164, modified_helmholtz.h:94-172, helmholtz.h:106-208)
// over raw arrays; out is accumulated into (ntrg*4 reals, or ntrg*4 interleaved complex).
int ref_gradient_p2p(int kernel, double k_re, double k_im, int ns, const double* sxyz, const double* sq, int nt,
                     const double* txyz, double* out) {
  RealVec sc(sxyz, sxyz + 3 * ns), tc(txyz, txyz + 3 * nt);
  if (kernel == 2) {
    HelmholtzFmm f(4, 64, complex_t(k_re, k_im), "unused.dat");
    ComplexVec sv(ns), tv(4 * nt, complex_t(0., 0.));
    for (int i = 0; i < ns; i++) sv[i] = complex_t(sq[2 * i], sq[2 * i + 1]);
    f.gradient_P2P(sc, sv, tc, tv);
    for (int i = 0; i < 4 * nt; i++) {
      out[2 * i] += tv[i].real();
      out[2 * i + 1] += tv[i].imag();
    }
    return 0;
  }
  RealVec sv(sq, sq + ns), tv(4 * nt, 0.);
  if (kernel == 0) {
    LaplaceFmm f(4, 64, "unused.dat");
    f.gradient_P2P(sc, sv, tc, tv);
  } else {
    ModifiedHelmholtzFmm f(4, 64, (real_t)k_re, "unused.dat");
    f.gradient_P2P(sc, sv, tc, tv);
  }
  for (int i = 0; i < 4 * nt; i++) out[i] += tv[i];
  return 0;
}

int ref_num_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
