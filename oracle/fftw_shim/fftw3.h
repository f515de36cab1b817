/*
 * fftw3.h -- FFTW3-API shim used ONLY to compile the reference's own headers
 * into the oracle library (oracle/_ref).  Test infrastructure, not product.
 *
 * FFTW3 itself (the reference's third-party dependency, version unpinned by
 * the reference: m4/ax_fftw.m4, setup.py:77 "-lfftw3 -lfftw3f") is absent from
 * this image.  This header declares the subset of the public FFTW3 interface
 * that the reference calls (include/exafmm_t.h:21-51, fmm_scale_invariant.h,
 * fmm.h) and fftw_shim.c implements it from the definition of the discrete
 * Fourier transform using FFTW's documented conventions:
 *   - transforms are unnormalised; FFTW_FORWARD = -1 is the exponent sign,
 *   - multi-dimensional arrays are row-major (last index fastest),
 *   - r2c output keeps n[rank-1]/2+1 entries along the last dimension,
 *   - "many" plans take howmany/stride/dist; embed arrays must be NULL.
 */
#ifndef XFMM_FFTW_SHIM_H
#define XFMM_FFTW_SHIM_H
#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef float fftwf_complex[2];
typedef struct xfmm_fft_plan_s* fftw_plan;
typedef struct xfmm_fft_plan_s* fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft(int rank, const int* n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed, int istride,
                             int idist, fftw_complex* out, const int* onembed, int ostride, int odist, int sign,
                             unsigned flags);
fftw_plan fftw_plan_dft_r2c(int rank, const int* n, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany, double* in, const int* inembed, int istride,
                                 int idist, fftw_complex* out, const int* onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed,
                                 int istride, int idist, double* out, const int* onembed, int ostride, int odist,
                                 unsigned flags);
void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out);
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out);
void fftw_destroy_plan(fftw_plan p);
void fftw_flops(const fftw_plan p, double* add, double* mul, double* fma);

fftwf_plan fftwf_plan_dft(int rank, const int* n, fftwf_complex* in, fftwf_complex* out, int sign, unsigned flags);
fftwf_plan fftwf_plan_many_dft(int rank, const int* n, int howmany, fftwf_complex* in, const int* inembed,
                               int istride, int idist, fftwf_complex* out, const int* onembed, int ostride,
                               int odist, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_r2c(int rank, const int* n, float* in, fftwf_complex* out, unsigned flags);
fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int* n, int howmany, float* in, const int* inembed, int istride,
                                   int idist, fftwf_complex* out, const int* onembed, int ostride, int odist,
                                   unsigned flags);
fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int* n, int howmany, fftwf_complex* in, const int* inembed,
                                   int istride, int idist, float* out, const int* onembed, int ostride, int odist,
                                   unsigned flags);
void fftwf_execute_dft(const fftwf_plan p, fftwf_complex* in, fftwf_complex* out);
void fftwf_execute_dft_r2c(const fftwf_plan p, float* in, fftwf_complex* out);
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex* in, float* out);
void fftwf_destroy_plan(fftwf_plan p);
void fftwf_flops(const fftwf_plan p, double* add, double* mul, double* fma);

#ifdef __cplusplus
}
#endif
#endif
