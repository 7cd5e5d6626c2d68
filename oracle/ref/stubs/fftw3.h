/* fftw3.h -- declarations of the FFTW 3 calls the reference's operator code
 * makes (fmm3d_mpi/matmgnt3d_mpi.cpp:302,341,408), for building it here
 * without FFTW (test infrastructure: oracle/_ref only).  The definitions in
 * ref_shims.cpp restate FFTW 3's documented semantics: row-major rank-n
 * transforms, r2c halving the last dimension to n/2+1, howmany interleaved
 * transforms addressed by stride and distance, forward sign -1, both
 * directions unnormalised. */
#ifndef FMMG_REF_STUB_FFTW3_H_
#define FMMG_REF_STUB_FFTW3_H_

typedef double fftw_complex[2];
typedef struct fmmg_ref_fftw_plan_s* fftw_plan;
#define FFTW_ESTIMATE (1U << 6)

#ifdef __cplusplus
extern "C" {
#endif
fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany, double* in, const int* inembed, int istride,
                                 int idist, fftw_complex* out, const int* onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed,
                                 int istride, int idist, double* out, const int* onembed, int ostride, int odist,
                                 unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
#ifdef __cplusplus
}
#endif

#endif
