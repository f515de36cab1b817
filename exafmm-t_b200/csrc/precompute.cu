// precompute.cu -- FP64 precomputation of the translation operators (Fmm::precompute).
//
//   check-to-equivalent pinv  fmm_scale_invariant.h:446-514, fmm.h:451-521 (LAPACK gesvd there,
//                             cuSOLVER gesvd here); P = pinv(K(check 2.95, equiv 1.05)) with the
//                             reference's truncation s_i > 4*eps*s_max (eps = 1e-16 for FP64,
//                             1e-10 for the mixed path so FP32 equivalent densities stay exact
//                             enough); applied in the reference's two factors (see LevelOps)
//   M2M / L2L                 fmm_scale_invariant.h:51-77, fmm.h:47-74: M2M[c] = (V S+)(U^H K(parent check,
//                             child equiv)); L2L[c] == M2M[c]^T (pinv(K^T) = pinv(K)^T)
//   M2L kernel FFT tables     fmm_scale_invariant.h:517-558, fmm.h:524-629: 316 convolution grids ->
//                             3-D FFT (cuFFT, FP64) -> 26 tables [nfreq][8 src x 8 trg] / nconv
// Laplace is scale invariant: one set of level-0 operators.  The other kernels get
// operators for every level 0..depth and M2L tables for child levels 1..depth.
#include <cublas_v2.h>
#include <cufft.h>
#include <cusolverDn.h>

#include <array>
#include <cmath>
#include <map>
#include <tuple>

#include "xfmm_internal.h"

namespace xfmm {

#define XCUBLAS(call)                                                                               \
  do {                                                                                              \
    cublasStatus_t st_ = (call);                                                                    \
    if (st_ != CUBLAS_STATUS_SUCCESS)                                                               \
      throw Error(XFMM_ERR_CUDA, std::string("cuBLAS ") + #call + " failed: " + std::to_string((int)st_)); \
  } while (0)
#define XCUSOLVER(call)                                                                                 \
  do {                                                                                                  \
    cusolverStatus_t st_ = (call);                                                                      \
    if (st_ != CUSOLVER_STATUS_SUCCESS)                                                                 \
      throw Error(XFMM_ERR_CUDA, std::string("cuSOLVER ") + #call + " failed: " + std::to_string((int)st_)); \
  } while (0)
#define XCUFFT(call)                                                                                 \
  do {                                                                                               \
    cufftResult st_ = (call);                                                                        \
    if (st_ != CUFFT_SUCCESS)                                                                        \
      throw Error(XFMM_ERR_CUDA, std::string("cuFFT ") + #call + " failed: " + std::to_string((int)st_)); \
  } while (0)

// geometry.h:21-54: unit surface points before the alpha*r scaling
void host_surface_base(int p, std::vector<double>& c) {
  const int n = nsurf_of(p);
  c.assign(3 * n, 0.0);
  c[0] = c[1] = c[2] = -1.0;
  int cnt = 1;
  for (int i = 0; i < p - 1; i++)
    for (int j = 0; j < p - 1; j++, cnt++) {
      c[3 * cnt] = -1.0;
      c[3 * cnt + 1] = (2.0 * (i + 1) - p + 1) / (p - 1);
      c[3 * cnt + 2] = (2.0 * j - p + 1) / (p - 1);
    }
  for (int i = 0; i < p - 1; i++)
    for (int j = 0; j < p - 1; j++, cnt++) {
      c[3 * cnt] = (2.0 * i - p + 1) / (p - 1);
      c[3 * cnt + 1] = -1.0;
      c[3 * cnt + 2] = (2.0 * (j + 1) - p + 1) / (p - 1);
    }
  for (int i = 0; i < p - 1; i++)
    for (int j = 0; j < p - 1; j++, cnt++) {
      c[3 * cnt] = (2.0 * (i + 1) - p + 1) / (p - 1);
      c[3 * cnt + 1] = (2.0 * j - p + 1) / (p - 1);
      c[3 * cnt + 2] = -1.0;
    }
  for (int i = 0; i < (n / 2) * 3; i++) c[3 * cnt + i] = -c[i];
}

namespace {

// geometry.h:55-62
std::vector<double> host_surface(int p, double r0, int level, const double* ctr, double alpha) {
  std::vector<double> c;
  host_surface_base(p, c);
  const double r = r0 * std::pow(0.5, level);
  const double b = alpha * r;
  for (size_t i = 0; i < c.size() / 3; i++)
    for (int d = 0; d < 3; d++) c[3 * i + d] = c[3 * i + d] * b + ctr[d];
  return c;
}

// geometry.h:101-134 (rounded; identical to the reference's truncation for p <= 20)
std::vector<int> host_surf2conv(int p, bool up) {
  const int n1 = 2 * p;
  const double ctr[3] = {0.5 * (p - 1), 0.5 * (p - 1), 0.5 * (p - 1)};
  std::vector<double> s = host_surface(p, 0.5, 0, ctr, double(p - 1));
  const double off = up ? (p - 1) : (2 * p - 1);
  std::vector<int> m(s.size() / 3);
  for (size_t i = 0; i < m.size(); i++) {
    const int a = (int)std::lround(off - s[3 * i]), b = (int)std::lround(off - s[3 * i + 1]),
              c = (int)std::lround(off - s[3 * i + 2]);
    m[i] = a + b * n1 + c * n1 * n1;
  }
  return m;
}

// geometry.h:156-195
std::vector<std::array<int, 3>> rel_coords(int max_r, int min_r, int step) {
  std::vector<std::array<int, 3>> out;
  for (int k = -max_r; k <= max_r; k += step)
    for (int j = -max_r; j <= max_r; j += step)
      for (int i = -max_r; i <= max_r; i += step)
        if (std::abs(i) >= min_r || std::abs(j) >= min_r || std::abs(k) >= min_r) out.push_back({i, j, k});
  return out;
}
std::vector<int> m2l_index_map() {
  auto m2l = rel_coords(1, 1, 1), helper = rel_coords(3, 2, 1);
  std::map<std::tuple<int, int, int>, int> lut;
  for (size_t i = 0; i < helper.size(); i++) lut[{helper[i][0], helper[i][1], helper[i][2]}] = (int)i;
  std::vector<int> m(26 * 64, -1);
  for (int i = 0; i < 26; i++)
    for (int j1 = 0; j1 < 8; j1++)
      for (int j2 = 0; j2 < 8; j2++) {
        const int a = m2l[i][0] * 2 - (j1 & 1) + (j2 & 1), b = m2l[i][1] * 2 - ((j1 >> 1) & 1) + ((j2 >> 1) & 1),
                  c = m2l[i][2] * 2 - ((j1 >> 2) & 1) + ((j2 >> 2) & 1);
        auto it = lut.find({a, b, c});
        m[i * 64 + j2 * 8 + j1] = it == lut.end() ? -1 : it->second;
      }
  return m;
}

constexpr double FOURPI = 4.0 * 3.14159265358979323846;

// potential of a unit charge (the kernels' scalar formulas, laplace.h:269-274 etc.), complex form
__device__ __forceinline__ double2 green64(int kernel, double k_re, double k_im, double r2) {
  if (r2 == 0) return make_double2(0, 0);
  const double r = sqrt(r2);
  if (kernel == XFMM_LAPLACE) return make_double2(1.0 / r / FOURPI, 0);
  if (kernel == XFMM_MODIFIED_HELMHOLTZ) return make_double2(exp(-k_re * r) / r / FOURPI, 0);
  const double e = exp(-k_im * r) / r / FOURPI;
  double sn, cs;
  sincos(k_re * r, &sn, &cs);
  return make_double2(e * cs, e * sn);
}

// M[i*nt + j] = G(trg_j - src_i)   (fmm_base.h:65-76), real or interleaved complex output
__global__ void k_kernel_matrix(int kernel, double k_re, double k_im, const double* src, int ns, const double* trg,
                                int nt, double* out, int cplx) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)ns * nt) return;
  const int i = (int)(e / nt), j = (int)(e % nt);
  const double dx = trg[3 * j] - src[3 * i], dy = trg[3 * j + 1] - src[3 * i + 1], dz = trg[3 * j + 2] - src[3 * i + 2];
  const double2 g = green64(kernel, k_re, k_im, dx * dx + dy * dy + dz * dz);
  if (cplx) {
    out[2 * e] = g.x;
    out[2 * e + 1] = g.y;
  } else {
    out[e] = g.x;
  }
}

// conv grids of all 316 helper offsets: value at g = potential at origin of a unit charge at grid point g
__global__ void k_conv_values(int kernel, double k_re, double k_im, int p, double a, const double* offs, int nh,
                              double* out, int cplx) {
  const int n1 = 2 * p, nconv = n1 * n1 * n1;
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)nh * nconv) return;
  const int h = (int)(e / nconv), g = (int)(e % nconv);
  const int i = g % n1, j = (g / n1) % n1, k = g / (n1 * n1);
  // geometry.h:85-87
  const double x = (i - p) * a / (p - 1) + offs[3 * h], y = (j - p) * a / (p - 1) + offs[3 * h + 1],
               z = (k - p) * a / (p - 1) + offs[3 * h + 2];
  const double2 gv = green64(kernel, k_re, k_im, x * x + y * y + z * z);
  if (cplx) {
    out[2 * e] = gv.x;
    out[2 * e + 1] = gv.y;
  } else {
    out[e] = gv.x;
  }
}

__global__ void k_sinv(const double* s, int n, double thr, double* sinv) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) sinv[i] = s[i] > thr ? 1.0 / s[i] : 0.0;
}

// Row-major factors of M = U_M S VH_M from cuSOLVER's column-major SVD of A = M^T = U_c S V_c^H:
// M = conj(V_c) S U_c^T, and read as row-major arrays the memory of cuSOLVER's U is U_c^T = VH_M
// and the memory of its VT (= V_c^H, column-major) is conj(V_c) = U_M.
// Writes the GEMM operands of P2M / L2P and the two factors used to form M2M.
__global__ void k_svd_factors(const double* Uc, const double* Vc, const double* sinv, int n, int cplx, double* p2m1,
                              double* p2m2, double* l2p1, double* l2p2, double* Uh, double* Vs) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * n) return;
  const int k = (int)(e / n), j = (int)(e % n);
  const int64_t kj = (int64_t)k * n + j, jk = (int64_t)j * n + k;
  // U_M[k][j] = Vc[k][j], VH_M[k][j] = Uc[k][j]
  if (cplx) {
    const double2* U2 = (const double2*)Uc;
    const double2* V2 = (const double2*)Vc;
    const double2 vkj = V2[kj], vjk = V2[jk], ukj = U2[kj], ujk = U2[jk];
    ((double2*)p2m1)[kj] = make_double2(vkj.x, -vkj.y);                      // conj(U_M[k][j])
    ((double2*)p2m2)[kj] = make_double2(ukj.x * sinv[k], -ukj.y * sinv[k]);  // conj(VH_M[k][j]) / s_k
    ((double2*)l2p1)[kj] = make_double2(ujk.x, -ujk.y);                      // conj(VH_M[j][k])
    ((double2*)l2p2)[kj] = make_double2(vjk.x * sinv[k], -vjk.y * sinv[k]);  // conj(U_M[j][k]) / s_k
    ((double2*)Uh)[kj] = make_double2(vjk.x, -vjk.y);                        // (U_M^H)[k][j] = conj(U_M[j][k])
    ((double2*)Vs)[kj] = make_double2(ujk.x * sinv[j], -ujk.y * sinv[j]);   // (V_M S+)[k][j]
  } else {
    p2m1[kj] = Vc[kj];
    p2m2[kj] = Uc[kj] * sinv[k];
    l2p1[kj] = Uc[jk];
    l2p2[kj] = Vc[jk] * sinv[k];
    Uh[kj] = Vc[jk];
    Vs[kj] = Uc[jk] * sinv[j];
  }
}

// T[ipos][f][j] = helper[imap[ipos][j]][f] / nconv
__global__ void k_m2l_tables(const double2* helper, int nfreq, const int* imap, double nconv, double2* T) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= 26ll * nfreq * 64) return;
  const int j = (int)(e % 64), f = (int)((e / 64) % nfreq), ipos = (int)(e / (64ll * nfreq));
  const int h = imap[ipos * 64 + j];
  double2 v = make_double2(0, 0);
  if (h >= 0) {
    const double2 x = helper[(int64_t)h * nfreq + f];
    v = make_double2(x.x / nconv, x.y / nconv);
  }
  T[e] = v;
}

// out[k][j] = (transpose ? A[j][k] : A[k][j]) for an n x n block, written into a wider row layout
__global__ void k_place(const double* A, int n, int transpose, int cplx, int out_ld, int out_row0, int out_col0,
                        void* out, int out_single) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * n) return;
  const int k = (int)(e / n), j = (int)(e % n);
  const int64_t src = transpose ? (int64_t)j * n + k : (int64_t)k * n + j;
  const int64_t dst = (int64_t)(out_row0 + k) * out_ld + out_col0 + j;
  if (cplx) {
    const double re = A[2 * src], im = A[2 * src + 1];
    if (out_single) ((float2*)out)[dst] = make_float2((float)re, (float)im);
    else ((double2*)out)[dst] = make_double2(re, im);
  } else {
    if (out_single) ((float*)out)[dst] = (float)A[src];
    else ((double*)out)[dst] = A[src];
  }
}
__global__ void k_to_single(const double* in, float* out, int64_t n) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e < n) out[e] = (float)in[e];
}

inline int nb(int64_t n) { return (int)std::max<int64_t>(1, (n + 255) / 256); }

struct Handles {
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t sol = nullptr;
  ~Handles() {
    if (blas) cublasDestroy(blas);
    if (sol) cusolverDnDestroy(sol);
  }
};

}  // namespace

void precompute(Fmm& f, int depth, cudaStream_t s) {
  const int p = f.p, n = f.nsurf, n1 = f.n1, nconv = f.nconv, nfreq = f.nfreq;
  const bool cplx = f.is_complex();
  const int vs = cplx ? 2 : 1;        // doubles per value
  const bool single = f.mixed();
  const size_t wsz = (single ? sizeof(float) : sizeof(double)) * vs;  // bytes per working value
#ifndef XFMM_PINV_EPS_MIXED
#define XFMM_PINV_EPS_MIXED 1e-10
#endif
  const double eps = single ? XFMM_PINV_EPS_MIXED : 1e-16;
  const double r0 = f.r0;
  Handles H;
  XCUBLAS(cublasCreate(&H.blas));
  XCUBLAS(cublasSetStream(H.blas, s));
  XCUSOLVER(cusolverDnCreate(&H.sol));
  XCUSOLVER(cusolverDnSetStream(H.sol, s));

  // geometry tables shared by all levels
  host_surface_base(p, f.h_surf_base);
  f.surf_base.upload(f.h_surf_base, s);
  std::vector<int> mup = host_surf2conv(p, true), mdn = host_surf2conv(p, false);
  f.map_up.upload(mup, s);
  f.map_dn.upload(mdn, s);
  std::vector<int> inv(nconv, -1);
  for (int k = 0; k < n; k++) inv[mup[k]] = k;
  f.conv_to_surf_up.upload(inv, s);
  {
    // e^{2 pi i m / n1} for m < n1, as (cos, sin) pairs: the DFT factors of the M2L transforms
    const int n1 = 2 * p;
    std::vector<double> tw(2 * n1);
    for (int m = 0; m < n1; m++) {
      const double a = 2.0 * 3.14159265358979323846 * m / n1;
      tw[2 * m] = std::cos(a);
      tw[2 * m + 1] = std::sin(a);
    }
    f.dft_tw.upload(tw, s);
  }
  std::vector<int> imap = m2l_index_map();
  DBuf<int> d_imap;
  d_imap.upload(imap, s);
  auto helper_rel = rel_coords(3, 2, 1);
  auto m2m_rel = rel_coords(1, 1, 2);

  const int nlev = f.kernel == XFMM_LAPLACE ? 1 : depth + 1;
  f.ops.clear();
  f.ops.resize(nlev);
  const double zero[3] = {0, 0, 0};
  DBuf<double> d_chk, d_eqv, M(n * (size_t)n * vs), Mcopy(n * (size_t)n * vs), S(n), U(n * (size_t)n * vs),
      VT(n * (size_t)n * vs), K(n * (size_t)n * vs), M2M(8 * (size_t)n * n * vs), Uh(n * (size_t)n * vs),
      Vs(n * (size_t)n * vs), Tmp(n * (size_t)n * vs), sinv(n);
  DBuf<double> F[4];
  for (auto& b : F) b.alloc(n * (size_t)n * vs);
  DBuf<int> info(1);
  for (int lev = 0; lev < nlev; lev++) {
    LevelOps& op = f.ops[lev];
    // ---- K(check, equiv) and its regularised pinv
    std::vector<double> chk = host_surface(p, r0, lev, zero, 2.95), eqv = host_surface(p, r0, lev, zero, 1.05);
    d_chk.upload(chk, s);
    d_eqv.upload(eqv, s);
    k_kernel_matrix<<<nb((int64_t)n * n), 256, 0, s>>>(f.kernel, f.k_re, f.k_im, d_chk.p, n, d_eqv.p, n, M.p, cplx);
    XLAUNCH();
    XCUDA(cudaMemcpyAsync(Mcopy.p, M.p, M.bytes(), cudaMemcpyDeviceToDevice, s));
    int lwork = 0;
    if (cplx) XCUSOLVER(cusolverDnZgesvd_bufferSize(H.sol, n, n, &lwork));
    else XCUSOLVER(cusolverDnDgesvd_bufferSize(H.sol, n, n, &lwork));
    DBuf<double> work((size_t)std::max(lwork, 1) * vs), rwork(5 * (size_t)n);
    if (cplx)
      XCUSOLVER(cusolverDnZgesvd(H.sol, 'A', 'A', n, n, (cuDoubleComplex*)Mcopy.p, n, S.p, (cuDoubleComplex*)U.p, n,
                                 (cuDoubleComplex*)VT.p, n, (cuDoubleComplex*)work.p, lwork, rwork.p, info.p));
    else
      XCUSOLVER(cusolverDnDgesvd(H.sol, 'A', 'A', n, n, Mcopy.p, n, S.p, U.p, n, VT.p, n, work.p, lwork, rwork.p,
                                 info.p));
    int hinfo = 0;
    XCUDA(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    std::vector<double> hs = S.download(s);
    XREQUIRE(hinfo == 0, XFMM_ERR_NUMERIC, "check-to-equivalent SVD did not converge");
    double smax = 0;
    for (double v : hs) smax = std::max(smax, std::fabs(v));
    // singular values come in descending order: the factors' first `rank` rows/columns carry everything
    int rank = 0;
    for (double v : hs) rank += v > eps * smax * 4;
    op.rank = std::max(rank, 1);
    k_sinv<<<nb(n), 256, 0, s>>>(S.p, n, eps * smax * 4, sinv.p);
    k_svd_factors<<<nb((int64_t)n * n), 256, 0, s>>>(U.p, VT.p, sinv.p, n, cplx, F[0].p, F[1].p, F[2].p, F[3].p,
                                                      Uh.p, Vs.p);
    XLAUNCH();
    // ---- M2M[c] = (V S+) (U^H K(parent check, child equiv)), row-major, in the reference's factored
    //      order (fmm_scale_invariant.h:67-71); cuBLAS is column-major, so row-major X*Y = gemm(Y, X)
    const double sc = r0 * std::pow(0.5, lev + 1);
    for (int c = 0; c < 8; c++) {
      const double cc[3] = {m2m_rel[c][0] * sc, m2m_rel[c][1] * sc, m2m_rel[c][2] * sc};
      std::vector<double> ceq = host_surface(p, r0, lev + 1, cc, 1.05);
      d_eqv.upload(ceq, s);
      k_kernel_matrix<<<nb((int64_t)n * n), 256, 0, s>>>(f.kernel, f.k_re, f.k_im, d_chk.p, n, d_eqv.p, n, K.p, cplx);
      XLAUNCH();
      double* out = M2M.p + (size_t)c * n * n * vs;
      if (cplx) {
        const cuDoubleComplex one = make_cuDoubleComplex(1, 0), z = make_cuDoubleComplex(0, 0);
        XCUBLAS(cublasZgemm(H.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, (cuDoubleComplex*)K.p, n,
                            (cuDoubleComplex*)Uh.p, n, &z, (cuDoubleComplex*)Tmp.p, n));
        XCUBLAS(cublasZgemm(H.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, (cuDoubleComplex*)Tmp.p, n,
                            (cuDoubleComplex*)Vs.p, n, &z, (cuDoubleComplex*)out, n));
      } else {
        const double one = 1, z = 0;
        XCUBLAS(cublasDgemm(H.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, K.p, n, Uh.p, n, &z, Tmp.p, n));
        XCUBLAS(cublasDgemm(H.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, Tmp.p, n, Vs.p, n, &z, out, n));
      }
    }
    // ---- GEMM operands in the working precision
    // the check-to-equivalent factors stay FP64 in both precisions
    DBuf<char>* dst[4] = {&op.p2m_B1, &op.p2m_B2, &op.l2p_B1, &op.l2p_B2};
    for (int i = 0; i < 4; i++) {
      dst[i]->alloc((size_t)n * n * vs * sizeof(double));
      XCUDA(cudaMemcpyAsync(dst[i]->p, F[i].p, (size_t)n * n * vs * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    // the mixed path's L2P first factor (an orthogonal rotation of FP32 check values) runs in FP32
    if (single && !cplx) {
      op.l2p_B1f.alloc((size_t)n * n * sizeof(float));
      k_to_single<<<nb((int64_t)n * n), 256, 0, s>>>(F[2].p, (float*)op.l2p_B1f.p, (int64_t)n * n);
      XLAUNCH();
    }
    op.m2m_B.alloc((size_t)8 * n * n * wsz);
    op.l2l_B.alloc((size_t)8 * n * n * wsz);
    for (int c = 0; c < 8; c++) {
      const double* Mc = M2M.p + (size_t)c * n * n * vs;
      k_place<<<nb((int64_t)n * n), 256, 0, s>>>(Mc, n, 1, cplx, n, c * n, 0, op.m2m_B.p, single);
      k_place<<<nb((int64_t)n * n), 256, 0, s>>>(Mc, n, 0, cplx, 8 * n, 0, c * n, op.l2l_B.p, single);
    }
    XLAUNCH();
  }

  // ---- M2L tables
  const int nh = (int)helper_rel.size();
  const std::vector<int> tab_levels = f.kernel == XFMM_LAPLACE ? std::vector<int>{0} : [&] {
    std::vector<int> v;
    for (int l = 1; l <= depth; l++) v.push_back(l);
    return v;
  }();
  if (!tab_levels.empty()) {
    DBuf<double> grid((size_t)nh * nconv * vs), spec((size_t)nh * nfreq * 2), T64((size_t)26 * nfreq * 64 * 2);
    DBuf<double> offs(3 * (size_t)nh);
    cufftHandle plan;
    int dims[3] = {n1, n1, n1};
    XCUFFT(cufftPlanMany(&plan, 3, dims, nullptr, 1, nconv, nullptr, 1, nfreq, cplx ? CUFFT_Z2Z : CUFFT_D2Z, nh));
    XCUFFT(cufftSetStream(plan, s));
    for (int l : tab_levels) {
      std::vector<double> ho(3 * nh);
      for (int h = 0; h < nh; h++)
        for (int d = 0; d < 3; d++)
          ho[3 * h + d] = l == 0 ? helper_rel[h][d] * (r0 / 0.5) : helper_rel[h][d] * r0 * std::pow(0.5, l - 1);
      offs.upload(ho, s);
      const double a = 2 * r0 * std::pow(0.5, l) * 1.05;
      k_conv_values<<<nb((int64_t)nh * nconv), 256, 0, s>>>(f.kernel, f.k_re, f.k_im, p, a, offs.p, nh, grid.p,
                                                             cplx);
      XLAUNCH();
      if (cplx)
        XCUFFT(cufftExecZ2Z(plan, (cufftDoubleComplex*)grid.p, (cufftDoubleComplex*)spec.p, CUFFT_FORWARD));
      else
        XCUFFT(cufftExecD2Z(plan, grid.p, (cufftDoubleComplex*)spec.p));
      k_m2l_tables<<<nb(26ll * nfreq * 64), 256, 0, s>>>((double2*)spec.p, nfreq, d_imap.p, (double)nconv,
                                                          (double2*)T64.p);
      XLAUNCH();
      LevelOps& op = f.ops[l];
      const int64_t cnt = 26ll * nfreq * 64 * 2;
      if (single) {
        op.m2l_T.alloc(cnt * sizeof(float));
        k_to_single<<<nb(cnt), 256, 0, s>>>(T64.p, (float*)op.m2l_T.p, cnt);
        XLAUNCH();
      } else {
        op.m2l_T.alloc(cnt * sizeof(double));
        XCUDA(cudaMemcpyAsync(op.m2l_T.p, T64.p, cnt * sizeof(double), cudaMemcpyDeviceToDevice, s));
      }
    }
    XCUDA(cudaStreamSynchronize(s));
    cufftDestroy(plan);
  }
  XCUDA(cudaStreamSynchronize(s));
  f.precomputed = true;
  f.pre_r0 = r0;
  f.pre_depth = depth;
}

}  // namespace xfmm
