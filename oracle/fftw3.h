/*
 * fftw3.h -- FFTW3 API subset used by the reference's CPU path.
 *
 * TEST INFRASTRUCTURE ONLY (oracle).  Nothing in the product links this.
 *
 * FFTW3 itself is a third-party dependency of the reference (unpinned version;
 * reference README.md:68, Makefile:71) and is not installed in this image.
 * This header declares only the ten entry points and two planner flags that the
 * reference's CPU sources call (src/fftw_wrapper.cpp:4-76,
 * src/random_field.cpp:52-56,76-80, src/fdm3d.cpp:133-187).  The behaviour behind
 * them (fftw_shim.c) restates FFTW3's published semantics:
 *   - r2c: unnormalised forward DFT, exponent -2*pi*i, real n0 x n1 x n2 row-major
 *     input, complex n0 x n1 x (n2/2+1) row-major output;
 *   - c2r: unnormalised backward DFT, exponent +2*pi*i, of Hermitian input in the
 *     same half-complex layout; when input and output alias, the real output rows
 *     are padded to 2*(n2/2+1) doubles ("in-place" layout).
 */
#ifndef CF_ORACLE_FFTW3_SHIM_H
#define CF_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct cf_fftw_plan_s *fftw_plan;

/* Planner flags; the shim plans identically for both. */
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_complex *fftw_alloc_complex(size_t n);
double *fftw_alloc_real(size_t n);

#ifdef __cplusplus
}
#endif

#endif
