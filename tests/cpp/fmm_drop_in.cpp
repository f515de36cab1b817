// A caller written against the exafmm-t C++ API (the call sequence of the reference's tests/fmm_*.cpp
// drivers: bounds, tree, balance, relative coordinates, colleagues, lists, precompute, M2L setup, upward
// and downward pass, verify), compiled against include/exafmm_t_b200.h and linked with libexafmm_b200.so.
//
//   fmm_drop_in <input.bin> <output.bin>
//
// input : int32 kernel (0 Laplace, 1 modified Helmholtz, 2 Helmholtz), p, ncrit, depth (uniform tree,
//         NON_ADAPTIVE builds), precision; int64 nsrc, ntrg; float64 wavek (re, im);
//         float64 src[nsrc][3], q[nsrc] (complex: [nsrc][2]), trg[ntrg][3]
// output: int32 depth, nleafs, nnonleafs; float64 x0[3], r0; float64 err[2] (verify, all targets);
//         uint64 key of every leaf in leaf order; float64 values[ntrg][4] in the caller's target order
//         (complex: [ntrg][4][2]) assembled from the leaves' trg_value
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "exafmm_t_b200.h"

using namespace exafmm_t;

namespace {

struct Input {
  int kernel, p, ncrit, depth, precision;
  int64_t nsrc, ntrg;
  double wk[2];
  std::vector<double> src, q, trg;
};

template <typename T> T charge(const Input& in, int64_t i);
template <> real_t charge<real_t>(const Input& in, int64_t i) { return in.q[i]; }
template <> complex_t charge<complex_t>(const Input& in, int64_t i) { return complex_t(in.q[2 * i], in.q[2 * i + 1]); }
void put(std::vector<double>& v, size_t i, real_t x) { v[i] = x; }
void put(std::vector<double>& v, size_t i, complex_t x) {
  v[2 * i] = x.real();
  v[2 * i + 1] = x.imag();
}

template <typename T, typename F>
void run(const Input& in, F& fmm, FILE* out) {
  Bodies<T> sources(in.nsrc), targets(in.ntrg);
  for (int64_t i = 0; i < in.nsrc; i++) {
    sources[i].ibody = (int)i;
    for (int d = 0; d < 3; d++) sources[i].X[d] = in.src[3 * i + d];
    sources[i].q = charge<T>(in, i);
  }
  for (int64_t i = 0; i < in.ntrg; i++) {
    targets[i].ibody = (int)i;
    for (int d = 0; d < 3; d++) targets[i].X[d] = in.trg[3 * i + d];
  }
#if NON_ADAPTIVE
  fmm.depth = in.depth;
#endif
  get_bounds(sources, targets, fmm.x0, fmm.r0);
  NodePtrs<T> leafs, nonleafs;
  Nodes<T> nodes = build_tree(sources, targets, leafs, nonleafs, fmm);
#if !NON_ADAPTIVE
  balance_tree(nodes, sources, targets, leafs, nonleafs, fmm);
#endif
  init_rel_coord();
  set_colleagues(nodes);
  build_list(nodes, fmm);
  fmm.precompute();
  fmm.M2L_setup(nonleafs);
  fmm.upward_pass(nodes, leafs, false);
  fmm.downward_pass(nodes, leafs, false);
  RealVec err = fmm.verify(leafs, false);

  const int hdr[3] = {fmm.depth, (int)leafs.size(), (int)nonleafs.size()};
  const double geo[6] = {fmm.x0[0], fmm.x0[1], fmm.x0[2], fmm.r0, err[0], err[1]};
  fwrite(hdr, sizeof(int), 3, out);
  fwrite(geo, sizeof(double), 6, out);
  for (Node<T>* leaf : leafs) fwrite(&leaf->key, sizeof(uint64_t), 1, out);
  const size_t w = std::is_same<T, real_t>::value ? 1 : 2;
  std::vector<double> vals((size_t)in.ntrg * 4 * w);
  for (Node<T>* leaf : leafs)
    for (int k = 0; k < leaf->ntrgs; k++)
      for (int c = 0; c < 4; c++) put(vals, 4 * (size_t)leaf->itrgs[k] + c, leaf->trg_value[4 * k + c]);
  fwrite(vals.data(), sizeof(double), vals.size(), out);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
    return 2;
  }
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 2;
  Input in;
  int32_t h[5];
  int64_t n[2];
  if (fread(h, sizeof(int32_t), 5, f) != 5 || fread(n, sizeof(int64_t), 2, f) != 2 || fread(in.wk, 8, 2, f) != 2)
    return 2;
  in.kernel = h[0];
  in.p = h[1];
  in.ncrit = h[2];
  in.depth = h[3];
  in.precision = h[4];
  in.nsrc = n[0];
  in.ntrg = n[1];
  const size_t qw = in.kernel == 2 ? 2 : 1;
  in.src.resize(3 * in.nsrc);
  in.q.resize(qw * in.nsrc);
  in.trg.resize(3 * in.ntrg);
  if (fread(in.src.data(), 8, in.src.size(), f) != in.src.size() || fread(in.q.data(), 8, in.q.size(), f) != in.q.size() ||
      fread(in.trg.data(), 8, in.trg.size(), f) != in.trg.size())
    return 2;
  fclose(f);
  FILE* out = fopen(argv[2], "wb");
  if (!out) return 2;
  const xfmm_precision prec = in.precision ? XFMM_MIXED : XFMM_FP64;
  try {
    if (in.kernel == 0) {
      LaplaceFmm fmm(in.p, in.ncrit, "", prec);
      run<real_t>(in, fmm, out);
    } else if (in.kernel == 1) {
      ModifiedHelmholtzFmm fmm(in.p, in.ncrit, in.wk[0], "", prec);
      run<real_t>(in, fmm, out);
    } else {
      HelmholtzFmm fmm(in.p, in.ncrit, complex_t(in.wk[0], in.wk[1]), "", prec);
      run<complex_t>(in, fmm, out);
    }
  } catch (const std::exception& e) {
    fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  fclose(out);
  return 0;
}
