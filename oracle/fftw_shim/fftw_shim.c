/*
 * fftw_shim.c -- implementation of the FFTW3-API subset declared in fftw3.h.
 *
 * Test infrastructure: linked only into the oracle build of the reference
 * (oracle/_ref).  It restates the discrete Fourier transform
 *     X[k] = sum_j x[j] * exp(sign * 2*pi*i * j*k / n)          (unnormalised)
 * per dimension of a row-major array, with a mixed-radix Cooley-Tukey
 * decimation-in-time recursion (radix 4, 2, 3, 5, then any prime by direct
 * summation).  No FFTW source is used; only FFTW's documented array and sign
 * conventions are followed (see fftw3.h).  Plans are read-only after creation,
 * so one plan may be executed concurrently from several OpenMP threads, as the
 * reference does (fmm_scale_invariant.h:577-602).
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct {
  double re, im;
} cplx;

enum { KIND_C2C = 0, KIND_R2C = 1, KIND_C2R = 2 };

typedef struct {
  int n;
  int nfac;
  int fac[64];     /* pairs (radix, remaining length) */
  cplx* tw_fwd;    /* exp(-2 pi i k / n) */
  cplx* tw_bwd;    /* exp(+2 pi i k / n) */
} fft1d;

struct xfmm_fft_plan_s {
  int kind, rank, howmany, istride, idist, ostride, odist, sign;
  int n[8];
  int total;
  fft1d ax[8];
};

static void fft1d_init(fft1d* f, int n) {
  f->n = n;
  int m = n, k = 0;
  while (m > 1) {
    int p = 0;
    if (m % 4 == 0) p = 4;
    else if (m % 2 == 0) p = 2;
    else if (m % 3 == 0) p = 3;
    else if (m % 5 == 0) p = 5;
    else {
      for (int q = 7; q * q <= m; q += 2)
        if (m % q == 0) { p = q; break; }
      if (!p) p = m;
    }
    m /= p;
    f->fac[2 * k] = p;
    f->fac[2 * k + 1] = m;
    k++;
  }
  f->nfac = k;
  f->tw_fwd = (cplx*)malloc(sizeof(cplx) * (n > 0 ? n : 1));
  f->tw_bwd = (cplx*)malloc(sizeof(cplx) * (n > 0 ? n : 1));
  for (int j = 0; j < n; j++) {
    double a = 2.0 * M_PI * (double)j / (double)n;
    f->tw_fwd[j].re = cos(a);
    f->tw_fwd[j].im = -sin(a);
    f->tw_bwd[j].re = cos(a);
    f->tw_bwd[j].im = sin(a);
  }
}

static inline cplx cmul(cplx a, cplx b) {
  cplx c;
  c.re = a.re * b.re - a.im * b.im;
  c.im = a.re * b.im + a.im * b.re;
  return c;
}

/* Recursive DIT step: out[0..p*m) <- DFT of in[0], in[fstride], ... */
static void dit(cplx* out, const cplx* in, int fstride, const int* fac, const fft1d* f, const cplx* tw, int sign) {
  const int p = fac[0], m = fac[1];
  if (m == 1) {
    for (int q = 0; q < p; q++) out[q] = in[(size_t)q * fstride];
  } else {
    for (int q = 0; q < p; q++) dit(out + q * m, in + (size_t)q * fstride, fstride * p, fac + 2, f, tw, sign);
  }
  const int n = f->n;
  if (p == 2) {
    for (int u = 0; u < m; u++) {
      cplx a = out[u];
      cplx b = cmul(out[u + m], tw[(size_t)u * fstride]);
      out[u].re = a.re + b.re;
      out[u].im = a.im + b.im;
      out[u + m].re = a.re - b.re;
      out[u + m].im = a.im - b.im;
    }
  } else if (p == 4) {
    for (int u = 0; u < m; u++) {
      cplx a0 = out[u];
      cplx a1 = cmul(out[u + m], tw[(size_t)u * fstride]);
      cplx a2 = cmul(out[u + 2 * m], tw[(size_t)2 * u * fstride]);
      cplx a3 = cmul(out[u + 3 * m], tw[(size_t)3 * u * fstride]);
      cplx s02 = {a0.re + a2.re, a0.im + a2.im}, d02 = {a0.re - a2.re, a0.im - a2.im};
      cplx s13 = {a1.re + a3.re, a1.im + a3.im}, d13 = {a1.re - a3.re, a1.im - a3.im};
      /* multiply d13 by sign*i: forward (sign=-1) -> -i */
      cplx rd13;
      if (sign < 0) { rd13.re = d13.im; rd13.im = -d13.re; }
      else { rd13.re = -d13.im; rd13.im = d13.re; }
      out[u].re = s02.re + s13.re;          out[u].im = s02.im + s13.im;
      out[u + 2 * m].re = s02.re - s13.re;  out[u + 2 * m].im = s02.im - s13.im;
      out[u + m].re = d02.re + rd13.re;     out[u + m].im = d02.im + rd13.im;
      out[u + 3 * m].re = d02.re - rd13.re; out[u + 3 * m].im = d02.im - rd13.im;
    }
  } else {
    cplx scratch[64];
    cplx* s = p <= 64 ? scratch : (cplx*)malloc(sizeof(cplx) * p);
    for (int u = 0; u < m; u++) {
      for (int q = 0; q < p; q++) s[q] = cmul(out[u + q * m], tw[((size_t)q * u * fstride) % n]);
      for (int q1 = 0; q1 < p; q1++) {
        const int k = u + q1 * m;
        cplx acc = {0.0, 0.0};
        for (int q = 0; q < p; q++) {
          cplx t = cmul(s[q], tw[((size_t)q * q1 * m * fstride) % n]);
          acc.re += t.re;
          acc.im += t.im;
        }
        out[k] = acc;
      }
    }
    if (s != scratch) free(s);
  }
}

static void fft1d_exec(const fft1d* f, const cplx* in, cplx* out, int sign) {
  if (f->n == 1) { out[0] = in[0]; return; }
  dit(out, in, 1, f->fac, f, sign < 0 ? f->tw_fwd : f->tw_bwd, sign);
}

/* In-place complex n-D transform of a contiguous row-major array. */
static void cnd_exec(const struct xfmm_fft_plan_s* p, cplx* a, int sign) {
  int maxn = 1;
  for (int d = 0; d < p->rank; d++) if (p->n[d] > maxn) maxn = p->n[d];
  cplx* lin = (cplx*)malloc(sizeof(cplx) * maxn);
  cplx* lout = (cplx*)malloc(sizeof(cplx) * maxn);
  for (int d = 0; d < p->rank; d++) {
    const int L = p->n[d];
    size_t inner = 1;
    for (int e = d + 1; e < p->rank; e++) inner *= (size_t)p->n[e];
    size_t outer = (size_t)p->total / ((size_t)L * inner);
    for (size_t o = 0; o < outer; o++) {
      for (size_t i = 0; i < inner; i++) {
        cplx* base = a + o * (size_t)L * inner + i;
        for (int j = 0; j < L; j++) lin[j] = base[(size_t)j * inner];
        fft1d_exec(&p->ax[d], lin, lout, sign);
        for (int j = 0; j < L; j++) base[(size_t)j * inner] = lout[j];
      }
    }
  }
  free(lin);
  free(lout);
}

static struct xfmm_fft_plan_s* make_plan(int kind, int rank, const int* n, int howmany, int istride, int idist,
                                         int ostride, int odist, int sign) {
  struct xfmm_fft_plan_s* p = (struct xfmm_fft_plan_s*)calloc(1, sizeof(*p));
  p->kind = kind;
  p->rank = rank;
  p->howmany = howmany;
  p->istride = istride;
  p->idist = idist;
  p->ostride = ostride;
  p->odist = odist;
  p->sign = sign;
  p->total = 1;
  for (int d = 0; d < rank; d++) {
    p->n[d] = n[d];
    p->total *= n[d];
    fft1d_init(&p->ax[d], n[d]);
  }
  return p;
}

static int half_total(const struct xfmm_fft_plan_s* p) {
  return p->total / p->n[p->rank - 1] * (p->n[p->rank - 1] / 2 + 1);
}

/* index helpers: full row-major index -> (prefix, last) */
static void exec_c2c(const struct xfmm_fft_plan_s* p, const double* in, double* out) {
  cplx* a = (cplx*)malloc(sizeof(cplx) * p->total);
  for (int b = 0; b < p->howmany; b++) {
    const double* ib = in + 2 * (size_t)b * p->idist;
    double* ob = out + 2 * (size_t)b * p->odist;
    for (int j = 0; j < p->total; j++) {
      a[j].re = ib[2 * (size_t)j * p->istride];
      a[j].im = ib[2 * (size_t)j * p->istride + 1];
    }
    cnd_exec(p, a, p->sign);
    for (int j = 0; j < p->total; j++) {
      ob[2 * (size_t)j * p->ostride] = a[j].re;
      ob[2 * (size_t)j * p->ostride + 1] = a[j].im;
    }
  }
  free(a);
}

static void exec_r2c(const struct xfmm_fft_plan_s* p, const double* in, double* out) {
  cplx* a = (cplx*)malloc(sizeof(cplx) * p->total);
  const int nl = p->n[p->rank - 1], nh = nl / 2 + 1;
  const int rows = p->total / nl;
  for (int b = 0; b < p->howmany; b++) {
    const double* ib = in + (size_t)b * p->idist;
    double* ob = out + 2 * (size_t)b * p->odist;
    for (int j = 0; j < p->total; j++) {
      a[j].re = ib[(size_t)j * p->istride];
      a[j].im = 0.0;
    }
    cnd_exec(p, a, FFTW_FORWARD);
    for (int r = 0; r < rows; r++)
      for (int k = 0; k < nh; k++) {
        size_t o = (size_t)(r * nh + k) * p->ostride;
        ob[2 * o] = a[r * nl + k].re;
        ob[2 * o + 1] = a[r * nl + k].im;
      }
  }
  free(a);
}

static void exec_c2r(const struct xfmm_fft_plan_s* p, const double* in, double* out) {
  cplx* a = (cplx*)malloc(sizeof(cplx) * p->total);
  const int rank = p->rank;
  const int nl = p->n[rank - 1], nh = nl / 2 + 1;
  const int rows = p->total / nl;
  for (int b = 0; b < p->howmany; b++) {
    const double* ib = in + 2 * (size_t)b * p->idist;
    double* ob = out + (size_t)b * p->odist;
    for (int r = 0; r < rows; r++) {
      /* multi-index of the row, and of its mirror (-r mod n) */
      int idx[8], rem = r, mr = 0;
      for (int d = rank - 2; d >= 0; d--) {
        idx[d] = rem % p->n[d];
        rem /= p->n[d];
      }
      for (int d = 0; d < rank - 1; d++) mr = mr * p->n[d] + ((p->n[d] - idx[d]) % p->n[d]);
      for (int k = 0; k < nl; k++) {
        if (k < nh) {
          size_t o = (size_t)(r * nh + k) * p->istride;
          a[r * nl + k].re = ib[2 * o];
          a[r * nl + k].im = ib[2 * o + 1];
        } else {
          size_t o = (size_t)(mr * nh + (nl - k)) * p->istride;
          a[r * nl + k].re = ib[2 * o];
          a[r * nl + k].im = -ib[2 * o + 1];
        }
      }
    }
    cnd_exec(p, a, FFTW_BACKWARD);
    for (int j = 0; j < p->total; j++) ob[(size_t)j * p->ostride] = a[j].re;
  }
  free(a);
}

/* Thread-seconds spent inside the transforms, summed over every calling thread, so that a caller can
 * state how much of the reference's M2L stage this stand-in for FFTW accounts for. */
static unsigned long long g_exec_ns = 0;

static unsigned long long now_ns(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (unsigned long long)t.tv_sec * 1000000000ull + (unsigned long long)t.tv_nsec;
}

double xfmm_shim_exec_seconds(void) { return 1e-9 * (double)__atomic_load_n(&g_exec_ns, __ATOMIC_RELAXED); }
void xfmm_shim_reset(void) { __atomic_store_n(&g_exec_ns, 0ull, __ATOMIC_RELAXED); }

static void dispatch(const struct xfmm_fft_plan_s* p, const double* in, double* out) {
  const unsigned long long t0 = now_ns();
  if (p->kind == KIND_C2C) exec_c2c(p, in, out);
  else if (p->kind == KIND_R2C) exec_r2c(p, in, out);
  else exec_c2r(p, in, out);
  __atomic_fetch_add(&g_exec_ns, now_ns() - t0, __ATOMIC_RELAXED);
}

/* float entry points run the double transform on converted copies */
static void dispatch_f(const struct xfmm_fft_plan_s* p, const float* in, float* out) {
  size_t nin, nout;
  const size_t cnt = (size_t)p->howmany;
  if (p->kind == KIND_C2C) {
    nin = 2 * ((cnt - 1) * p->idist + (size_t)(p->total - 1) * p->istride + 1);
    nout = 2 * ((cnt - 1) * p->odist + (size_t)(p->total - 1) * p->ostride + 1);
  } else if (p->kind == KIND_R2C) {
    nin = (cnt - 1) * p->idist + (size_t)(p->total - 1) * p->istride + 1;
    nout = 2 * ((cnt - 1) * p->odist + (size_t)(half_total(p) - 1) * p->ostride + 1);
  } else {
    nin = 2 * ((cnt - 1) * p->idist + (size_t)(half_total(p) - 1) * p->istride + 1);
    nout = (cnt - 1) * p->odist + (size_t)(p->total - 1) * p->ostride + 1;
  }
  double* di = (double*)malloc(sizeof(double) * nin);
  double* dout = (double*)malloc(sizeof(double) * nout);
  for (size_t i = 0; i < nin; i++) di[i] = in[i];
  for (size_t i = 0; i < nout; i++) dout[i] = out[i];
  dispatch(p, di, dout);
  for (size_t i = 0; i < nout; i++) out[i] = (float)dout[i];
  free(di);
  free(dout);
}

static void destroy(struct xfmm_fft_plan_s* p) {
  if (!p) return;
  for (int d = 0; d < p->rank; d++) {
    free(p->ax[d].tw_fwd);
    free(p->ax[d].tw_bwd);
  }
  free(p);
}

static void flops(const struct xfmm_fft_plan_s* p, double* add, double* mul, double* fma) {
  double n = (double)p->total, lg = log2(n > 1 ? n : 2);
  *add = 3.0 * n * lg * p->howmany;
  *mul = 2.0 * n * lg * p->howmany;
  *fma = 0.0;
}

/* ---- double API ---- */
fftw_plan fftw_plan_dft(int rank, const int* n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags) {
  (void)in; (void)out; (void)flags;
  return make_plan(KIND_C2C, rank, n, 1, 1, 0, 1, 0, sign);
}
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed, int istride,
                             int idist, fftw_complex* out, const int* onembed, int ostride, int odist, int sign,
                             unsigned flags) {
  (void)in; (void)out; (void)flags; (void)inembed; (void)onembed;
  return make_plan(KIND_C2C, rank, n, howmany, istride, idist, ostride, odist, sign);
}
fftw_plan fftw_plan_dft_r2c(int rank, const int* n, double* in, fftw_complex* out, unsigned flags) {
  (void)in; (void)out; (void)flags;
  return make_plan(KIND_R2C, rank, n, 1, 1, 0, 1, 0, FFTW_FORWARD);
}
fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany, double* in, const int* inembed, int istride,
                                 int idist, fftw_complex* out, const int* onembed, int ostride, int odist,
                                 unsigned flags) {
  (void)in; (void)out; (void)flags; (void)inembed; (void)onembed;
  return make_plan(KIND_R2C, rank, n, howmany, istride, idist, ostride, odist, FFTW_FORWARD);
}
fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed,
                                 int istride, int idist, double* out, const int* onembed, int ostride, int odist,
                                 unsigned flags) {
  (void)in; (void)out; (void)flags; (void)inembed; (void)onembed;
  return make_plan(KIND_C2R, rank, n, howmany, istride, idist, ostride, odist, FFTW_BACKWARD);
}
void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out) { dispatch(p, (double*)in, (double*)out); }
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out) { dispatch(p, in, (double*)out); }
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out) { dispatch(p, (double*)in, out); }
void fftw_destroy_plan(fftw_plan p) { destroy(p); }
void fftw_flops(const fftw_plan p, double* add, double* mul, double* fma) { flops(p, add, mul, fma); }

/* ---- float API ---- */
fftwf_plan fftwf_plan_dft(int rank, const int* n, fftwf_complex* in, fftwf_complex* out, int sign, unsigned flags) {
  (void)in; (void)out; (void)flags;
  return make_plan(KIND_C2C, rank, n, 1, 1, 0, 1, 0, sign);
}
fftwf_plan fftwf_plan_many_dft(int rank, const int* n, int howmany, fftwf_complex* in, const int* inembed,
                               int istride, int idist, fftwf_complex* out, const int* onembed, int ostride,
                               int odist, int sign, unsigned flags) {
  (void)in; (void)out; (void)flags; (void)inembed; (void)onembed;
  return make_plan(KIND_C2C, rank, n, howmany, istride, idist, ostride, odist, sign);
}
fftwf_plan fftwf_plan_dft_r2c(int rank, const int* n, float* in, fftwf_complex* out, unsigned flags) {
  (void)in; (void)out; (void)flags;
  return make_plan(KIND_R2C, rank, n, 1, 1, 0, 1, 0, FFTW_FORWARD);
}
fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int* n, int howmany, float* in, const int* inembed, int istride,
                                   int idist, fftwf_complex* out, const int* onembed, int ostride, int odist,
                                   unsigned flags) {
  (void)in; (void)out; (void)flags; (void)inembed; (void)onembed;
  return make_plan(KIND_R2C, rank, n, howmany, istride, idist, ostride, odist, FFTW_FORWARD);
}
fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int* n, int howmany, fftwf_complex* in, const int* inembed,
                                   int istride, int idist, float* out, const int* onembed, int ostride, int odist,
                                   unsigned flags) {
  (void)in; (void)out; (void)flags; (void)inembed; (void)onembed;
  return make_plan(KIND_C2R, rank, n, howmany, istride, idist, ostride, odist, FFTW_BACKWARD);
}
void fftwf_execute_dft(const fftwf_plan p, fftwf_complex* in, fftwf_complex* out) {
  dispatch_f(p, (float*)in, (float*)out);
}
void fftwf_execute_dft_r2c(const fftwf_plan p, float* in, fftwf_complex* out) { dispatch_f(p, in, (float*)out); }
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex* in, float* out) { dispatch_f(p, (float*)in, out); }
void fftwf_destroy_plan(fftwf_plan p) { destroy(p); }
void fftwf_flops(const fftwf_plan p, double* add, double* mul, double* fma) { flops(p, add, mul, fma); }
