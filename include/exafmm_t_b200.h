/*
 * exafmm_t_b200.h -- the exafmm-t C++ API for the FMM evaluate path, over the C ABI of
 * libexafmm_b200.so (xfmm.h).  Header-only, C++14, host code only (no CUDA headers needed):
 * a caller written against the reference's headers compiles against this one and runs the
 * B200 path.  Link with -lexafmm_b200.
 *
 * Names, signatures and field names follow the reference (namespace exafmm_t):
 *   Body, Bodies, Node, Nodes, NodePtrs, vec3, real_t, complex_t, RealVec  include/exafmm_t.h:60-135
 *   FmmBase: p, nsurf, nconv, nfreq, ncrit, depth, r0, x0, filename       include/fmm_base.h:13-35
 *            upward_pass, downward_pass, verify                          include/fmm_base.h:162-267
 *            precompute, M2L_setup                                       include/fmm_scale_invariant.h:151-160,
 *                                                                        277-341; include/fmm.h:141-153, 265-333
 *   LaplaceFmm(p, ncrit, filename)                                       include/laplace.h:15
 *   ModifiedHelmholtzFmm(p, ncrit, wavek, filename)                      include/modified_helmholtz.h:17
 *   HelmholtzFmm(p, ncrit, wavek, filename)                              include/helmholtz.h:16
 *   get_bounds, build_tree, balance_tree                                 include/build_tree.h:21-35, 182-199, 337-359
 *                                                                        include/build_non_adaptive_tree.h:18-32, 181-194
 *   init_rel_coord                                                       include/geometry.h:198-215
 *   set_colleagues, build_list                                           include/build_list.h:124-197
 *
 * How the calls map onto the device path:
 *   - build_tree uploads the bodies, builds the tree on the GPU (xfmm_build_tree) and returns host
 *     views of its nodes.  The adaptive tree comes back already 2:1 balanced (the GPU build does
 *     both steps), so balance_tree only checks its arguments.  With NON_ADAPTIVE defined to 1, as for
 *     the reference's uniform build, the tree is uniform to fmm.depth (set it before the call).
 *   - init_rel_coord and set_colleagues have no work of their own (the relative-position tables are
 *     compile-time constants; the colleagues and the U, V, W and X lists are built on the GPU with the
 *     tree); build_list fills every node's colleague and list pointers.
 *   - precompute and M2L_setup run on the GPU for the last tree built with this Fmm.
 *   - upward_pass uploads the source charges held in the Bodies given to build_tree, zeroes the
 *     equivalent densities and runs the upward pass; downward_pass runs the downward pass and copies
 *     the potentials and gradients back into the leaves' trg_value (tree order inside each leaf,
 *     4 values per target: potential, d/dx, d/dy, d/dz), as the reference leaves them.
 *   - verify computes the relative L2 errors of potential and gradient against FP64 direct sums
 *     on the GPU, over all targets or the targets of 10 leaves (sample = true).
 * The precision of the evaluate path is a constructor argument beyond the reference's: XFMM_FP64
 * (default, the reference's arithmetic) or XFMM_MIXED.  Errors are reported as std::runtime_error
 * carrying the library's message.  A non-empty filename names the operator file in the reference's .dat
 * layout: precompute reads it when it matches the tree (size and r0) and otherwise computes the
 * operators on the device and writes it, as the reference does.
 */
#ifndef EXAFMM_T_B200_H
#define EXAFMM_T_B200_H

#include <algorithm>
#include <array>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "xfmm.h"

#ifndef NON_ADAPTIVE
#define NON_ADAPTIVE 0
#endif

namespace exafmm_t {

using real_t = double;
using complex_t = std::complex<real_t>;
using RealVec = std::vector<real_t>;
using ComplexVec = std::vector<complex_t>;

struct vec3 {
  real_t v[3] = {0, 0, 0};
  real_t& operator[](int i) { return v[i]; }
  const real_t& operator[](int i) const { return v[i]; }
};

template <typename T>
struct Body {
  int ibody = 0;           // position in the caller's input
  vec3 X;                  // coordinates
  T q = T();               // charge
  T p = T();               // potential
  std::array<T, 3> F{};    // gradient
};
template <typename T>
using Bodies = std::vector<Body<T>>;

template <typename T>
struct Node {
  size_t idx = 0;          // index in the tree (the reference's node numbering)
  bool is_leaf = false;
  int ntrgs = 0, nsrcs = 0;
  vec3 x;                  // centre
  real_t r = 0;            // half side length
  uint64_t key = 0;        // Morton key with level offset
  int level = 0, octant = 0;
  Node* parent = nullptr;
  std::vector<Node*> children, colleagues, P2L_list, M2P_list, P2P_list, M2L_list;
  std::vector<int> isrcs, itrgs;     // callers' indices of the leaf's sources and targets
  std::vector<T> trg_value;          // 4 values per target after downward_pass
};

namespace detail {
inline void check(xfmm_status s) {
  if (s != XFMM_OK) throw std::runtime_error(std::string("exafmm_t_b200: ") + xfmm_last_error());
}
struct TreeFree {
  void operator()(xfmm_tree* t) const { xfmm_tree_free(t); }
};
struct FmmFree {
  void operator()(xfmm_fmm* f) const { xfmm_fmm_free(f); }
};
template <typename T> inline void put_charge(std::vector<double>& out, size_t i, const T& q);
template <> inline void put_charge<real_t>(std::vector<double>& out, size_t i, const real_t& q) { out[i] = q; }
template <> inline void put_charge<complex_t>(std::vector<double>& out, size_t i, const complex_t& q) {
  out[2 * i] = q.real();
  out[2 * i + 1] = q.imag();
}
template <typename T> inline T get_value(const std::vector<double>& in, size_t i);
template <> inline real_t get_value<real_t>(const std::vector<double>& in, size_t i) { return in[i]; }
template <> inline complex_t get_value<complex_t>(const std::vector<double>& in, size_t i) {
  return complex_t(in[2 * i], in[2 * i + 1]);
}
}  // namespace detail

// Node storage plus the device tree it describes.  A std::vector of nodes, as in the reference; it also
// owns the device tree, which the Fmm of build_tree uses for the later calls.
template <typename T>
class Nodes : public std::vector<Node<T>> {
 public:
  using std::vector<Node<T>>::vector;
  std::shared_ptr<xfmm_tree> tree;
  int64_t nsrc = 0, ntrg = 0;
  std::vector<int> src_perm, trg_perm;  // tree order -> callers' order
};
template <typename T>
using NodePtrs = std::vector<Node<T>*>;

template <typename T>
class FmmBase {
 public:
  int p = 0, nsurf = 0, nconv = 0, nfreq = 0, ncrit = 0, depth = 0;
  real_t r0 = 0;
  vec3 x0;
  bool is_precomputed = false, is_real = std::is_same<T, real_t>::value;
  std::string filename;

  FmmBase(int kernel, int p_, int ncrit_, complex_t wavek, std::string filename_, xfmm_precision precision)
      : p(p_), ncrit(ncrit_), filename(std::move(filename_)) {
    xfmm_fmm* h = nullptr;
    detail::check(xfmm_fmm_create(kernel, p_, ncrit_, wavek.real(), wavek.imag(), precision, &h));
    fmm_.reset(h, detail::FmmFree());
    if (!filename.empty()) detail::check(xfmm_fmm_set_operator_file(h, filename.c_str()));
    int64_t i6[6];
    double d4[4];
    detail::check(xfmm_fmm_info(h, i6, d4));
    nsurf = (int)i6[1];
    nconv = (int)i6[2];
    nfreq = (int)i6[3];
  }
  virtual ~FmmBase() {}

  xfmm_fmm* handle() const { return fmm_.get(); }
  xfmm_tree* tree_handle() const {
    if (!tree_) throw std::runtime_error("exafmm_t_b200: build_tree has not been called with this Fmm");
    return tree_.get();
  }

  // Operators for the current tree (r0, depth), read from or written to `filename` when one is named.
  void precompute() {
    detail::check(xfmm_precompute(handle(), tree_handle(), nullptr));
    is_precomputed = true;
  }
  void M2L_setup(NodePtrs<T>& /*nonleafs*/) { detail::check(xfmm_m2l_setup(handle(), tree_handle(), nullptr)); }

  void upward_pass(Nodes<T>& /*nodes*/, NodePtrs<T>& /*leafs*/, bool /*verbose*/ = true) {
    detail::check(xfmm_set_charges(handle(), tree_handle(), charges_.data(), 0, nullptr));
    detail::check(xfmm_clear_values(handle(), tree_handle(), nullptr));
    detail::check(xfmm_upward_pass(handle(), tree_handle(), nullptr));
  }

  void downward_pass(Nodes<T>& nodes, NodePtrs<T>& leafs, bool /*verbose*/ = true) {
    detail::check(xfmm_downward_pass(handle(), tree_handle(), nullptr));
    const size_t w = is_real ? 1 : 2;
    std::vector<double> out((size_t)ntrg_ * 4 * w);
    detail::check(xfmm_get_values(handle(), tree_handle(), out.data(), 0, nullptr));
    for (Node<T>* leaf : leafs) {
      leaf->trg_value.assign(4 * (size_t)leaf->ntrgs, T());
      for (int k = 0; k < leaf->ntrgs; k++) {
        const size_t orig = (size_t)leaf->itrgs[k];
        for (int c = 0; c < 4; c++) leaf->trg_value[4 * k + c] = detail::get_value<T>(out, 4 * orig + c);
      }
    }
    (void)nodes;
  }

  RealVec verify(NodePtrs<T>& /*leafs*/, bool sample = false) {
    double e[2] = {0, 0};
    detail::check(xfmm_verify(handle(), tree_handle(), sample ? 1 : 0, e, nullptr));
    return RealVec{e[0], e[1]};
  }

  // used by build_tree
  void attach(const std::shared_ptr<xfmm_tree>& t, std::vector<double> charges, int64_t ntrg) {
    tree_ = t;
    charges_ = std::move(charges);
    ntrg_ = ntrg;
    int64_t i6[6];
    double d4[4];
    detail::check(xfmm_fmm_info(handle(), i6, d4));
    depth = (int)i6[5];
    for (int d = 0; d < 3; d++) x0[d] = d4[d];
    r0 = d4[3];
  }

 private:
  std::shared_ptr<xfmm_fmm> fmm_;
  std::shared_ptr<xfmm_tree> tree_;
  std::vector<double> charges_;
  int64_t ntrg_ = 0;
};

class LaplaceFmm : public FmmBase<real_t> {
 public:
  LaplaceFmm(int p_, int ncrit_, std::string filename_ = std::string(), xfmm_precision precision = XFMM_FP64)
      : FmmBase<real_t>(XFMM_LAPLACE, p_, ncrit_, 0.0, std::move(filename_), precision) {}
};

class ModifiedHelmholtzFmm : public FmmBase<real_t> {
 public:
  real_t wavek;
  ModifiedHelmholtzFmm(int p_, int ncrit_, real_t wavek_, std::string filename_ = std::string(),
                       xfmm_precision precision = XFMM_FP64)
      : FmmBase<real_t>(XFMM_MODIFIED_HELMHOLTZ, p_, ncrit_, wavek_, std::move(filename_), precision),
        wavek(wavek_) {}
};

class HelmholtzFmm : public FmmBase<complex_t> {
 public:
  complex_t wavek;
  HelmholtzFmm(int p_, int ncrit_, complex_t wavek_, std::string filename_ = std::string(),
               xfmm_precision precision = XFMM_FP64)
      : FmmBase<complex_t>(XFMM_HELMHOLTZ, p_, ncrit_, wavek_, std::move(filename_), precision), wavek(wavek_) {}
};

// Bounding cube of sources and targets: centre and half side length x 1.00001 (the reference's rule).
template <typename T>
void get_bounds(const Bodies<T>& sources, const Bodies<T>& targets, vec3& x0, real_t& r0) {
  vec3 lo, hi;
  for (int d = 0; d < 3; d++) {
    lo[d] = sources.empty() ? 0 : sources[0].X[d];
    hi[d] = lo[d];
  }
  auto grow = [&](const Bodies<T>& b) {
    for (const Body<T>& v : b)
      for (int d = 0; d < 3; d++) {
        lo[d] = std::min(lo[d], v.X[d]);
        hi[d] = std::max(hi[d], v.X[d]);
      }
  };
  grow(sources);
  grow(targets);
  r0 = 0;
  for (int d = 0; d < 3; d++) {
    x0[d] = (hi[d] + lo[d]) / 2;
    r0 = std::max(r0, std::max(x0[d] - lo[d], hi[d] - x0[d]));
  }
  r0 *= 1.00001;
}

namespace detail {
// Host views of the device tree from xfmm_tree_dump: node fields, children, leaf body ranges and, when
// `lists` is set, the colleagues and the P2P, M2P, P2L and M2L lists.  The nodes are written in place
// when the storage already has the tree's size, so pointers taken earlier stay valid.
template <typename T>
void materialise(Nodes<T>& nodes, NodePtrs<T>& leafs, NodePtrs<T>& nonleafs, bool lists) {
  xfmm_tree* t = nodes.tree.get();
  int64_t info[12];
  check(xfmm_tree_info(t, info));
  const int64_t nn = info[0], nl = info[1], nnl = info[2];
  const int64_t np2p = info[4], nm2p = info[5], np2l = info[6];
  std::vector<double> geo(6), nx(4 * nn);
  std::vector<uint64_t> key(nn);
  std::vector<int32_t> ni(8 * nn), lf(nl), nlf(nnl), coll(27 * nn), m2l(26 * nn);
  std::vector<int32_t> p2p(std::max<int64_t>(np2p, 1)), m2p(std::max<int64_t>(nm2p, 1)),
      p2l(std::max<int64_t>(np2l, 1));
  std::vector<int64_t> p2p_off(nn + 1), m2p_off(nn + 1), p2l_off(nn + 1);
  nodes.src_perm.resize(nodes.nsrc);
  nodes.trg_perm.resize(nodes.ntrg);
  check(xfmm_tree_dump(t, geo.data(), key.data(), ni.data(), nx.data(), lf.data(), nlf.data(), nodes.src_perm.data(),
                       nodes.trg_perm.data(), coll.data(), m2l.data(), p2p_off.data(), p2p.data(), m2p_off.data(),
                       m2p.data(), p2l_off.data(), p2l.data()));
  if ((int64_t)nodes.size() != nn) nodes.assign((size_t)nn, Node<T>());
  Node<T>* base = nodes.data();
  auto at = [&](int32_t i) { return i >= 0 ? base + i : nullptr; };
  for (int64_t i = 0; i < nn; i++) {
    Node<T>& n = nodes[i];
    const int32_t* r = &ni[8 * i];
    n.idx = (size_t)r[0];
    n.level = r[1];
    n.is_leaf = r[2] != 0;
    n.nsrcs = r[3];
    n.ntrgs = r[4];
    n.parent = at(r[5]);
    n.octant = r[6];
    n.children.clear();
    if (!n.is_leaf && r[7] >= 0)
      for (int c = 0; c < 8; c++) n.children.push_back(base + r[7] + c);
    for (int d = 0; d < 3; d++) n.x[d] = nx[4 * i + d];
    n.r = nx[4 * i + 3];
    n.key = key[i];
    n.colleagues.clear();
    n.M2L_list.clear();
    n.P2P_list.clear();
    n.M2P_list.clear();
    n.P2L_list.clear();
    if (!lists) continue;
    for (int c = 0; c < 27; c++) n.colleagues.push_back(at(coll[27 * i + c]));  // null: no colleague there
    for (int c = 0; c < 26; c++) n.M2L_list.push_back(at(m2l[26 * i + c]));     // null: no interaction
    for (int64_t e = p2p_off[i]; e < p2p_off[i + 1]; e++) n.P2P_list.push_back(base + p2p[e]);
    for (int64_t e = m2p_off[i]; e < m2p_off[i + 1]; e++) n.M2P_list.push_back(base + m2p[e]);
    for (int64_t e = p2l_off[i]; e < p2l_off[i + 1]; e++) n.P2L_list.push_back(base + p2l[e]);
  }
  leafs.clear();
  nonleafs.clear();
  int64_t so = 0, to = 0;
  for (int32_t li : lf) {
    Node<T>& n = nodes[li];
    n.isrcs.assign(nodes.src_perm.begin() + so, nodes.src_perm.begin() + so + n.nsrcs);
    n.itrgs.assign(nodes.trg_perm.begin() + to, nodes.trg_perm.begin() + to + n.ntrgs);
    so += n.nsrcs;
    to += n.ntrgs;
    leafs.push_back(&n);
  }
  for (int32_t k : nlf) nonleafs.push_back(&nodes[k]);
}
}  // namespace detail

// Tree over sources and targets, built on the GPU with its interaction lists.  Adaptive (ncrit bodies per
// leaf) and 2:1 balanced; uniform to fmm.depth when NON_ADAPTIVE is 1.  Sets fmm.x0, fmm.r0 and fmm.depth.
template <typename T>
Nodes<T> build_tree(Bodies<T>& sources, Bodies<T>& targets, NodePtrs<T>& leafs, NodePtrs<T>& nonleafs,
                    FmmBase<T>& fmm) {
  const size_t ns = sources.size(), nt = targets.size();
  std::vector<double> sx(3 * ns), tx(3 * nt), q(ns * (std::is_same<T, real_t>::value ? 1 : 2));
  for (size_t i = 0; i < ns; i++) {
    for (int d = 0; d < 3; d++) sx[3 * i + d] = sources[i].X[d];
    detail::put_charge<T>(q, i, sources[i].q);
  }
  for (size_t i = 0; i < nt; i++)
    for (int d = 0; d < 3; d++) tx[3 * i + d] = targets[i].X[d];
  xfmm_tree* h = nullptr;
  detail::check(xfmm_build_tree(fmm.handle(), sx.data(), (int64_t)ns, tx.data(), (int64_t)nt,
                                NON_ADAPTIVE ? fmm.depth : -1, 0, nullptr, &h));
  Nodes<T> nodes;
  nodes.tree.reset(h, detail::TreeFree());
  nodes.nsrc = (int64_t)ns;
  nodes.ntrg = (int64_t)nt;
  // the device lists are built with the tree (the host views read both); the nodes' list pointers are
  // filled in by build_list, as in the reference
  detail::check(xfmm_build_list(fmm.handle(), h, nullptr));
  fmm.attach(nodes.tree, std::move(q), (int64_t)nt);
  detail::materialise(nodes, leafs, nonleafs, false);
  return nodes;
}

// The tree of build_tree is balanced already; kept for callers written against the reference.
template <typename T>
void balance_tree(Nodes<T>& nodes, Bodies<T>& /*sources*/, Bodies<T>& /*targets*/, NodePtrs<T>& /*leafs*/,
                  NodePtrs<T>& /*nonleafs*/, FmmBase<T>& /*fmm*/) {
  if (!nodes.tree) throw std::runtime_error("exafmm_t_b200: balance_tree before build_tree");
}

inline void init_rel_coord() {}

template <typename T>
void set_colleagues(Nodes<T>& /*nodes*/) {}

// U, V, W, X lists and colleagues (built on the GPU with the tree): every node's list pointers are filled in.
template <typename T>
void build_list(Nodes<T>& nodes, FmmBase<T>& /*fmm*/) {
  if (!nodes.tree) throw std::runtime_error("exafmm_t_b200: build_list before build_tree");
  NodePtrs<T> leafs, nonleafs;
  detail::materialise(nodes, leafs, nonleafs, true);
}

}  // namespace exafmm_t
#endif
