/*
 * fftw3.h -- a project-written stand-in for the single-precision FFTW 3 API, oracle use only.
 *
 * TEST INFRASTRUCTURE. This header and fftw_shim.cpp exist so that the reference CPU backend
 * (slipcam cxx/cpu.cpp, which includes <fftw3.h>) compiles unchanged in a container without
 * FFTW. They declare exactly the nine names cpu.cpp uses (cpu.cpp:65-66, 70-71, 81-84, 99, 139,
 * 143) with FFTW's documented meaning:
 *   - fftwf_complex is float[2] (real, imaginary);
 *   - an r2c 2-D transform of n0 x n1 reals gives n0 x (n1/2 + 1) complex values, row-major,
 *     with the forward sign e^{-2 pi i j k / n};
 *   - a c2r 2-D transform is the unnormalized inverse (sign +1), reading the same half layout;
 *   - plans may be executed concurrently on other (aligned) arrays of the same shape.
 * The arithmetic is our own mixed-radix FFT in double precision (fftw_shim.cpp); results are
 * rounded to float once at the end, so they differ from real FFTW at the 1e-7 relative level.
 * Nothing outside oracle/ may include this header.
 */
#pragma once

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct fftwf_plan_s *fftwf_plan;

/* planner flags: accepted and ignored (the shim has a single algorithm) */
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

float *fftwf_alloc_real(size_t n);
fftwf_complex *fftwf_alloc_complex(size_t n);
void fftwf_free(void *p);

fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float *in, fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex *in, float *out, unsigned flags);
void fftwf_execute_dft_r2c(const fftwf_plan p, float *in, fftwf_complex *out);
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex *in, float *out);
void fftwf_destroy_plan(fftwf_plan p);

#ifdef __cplusplus
}
#endif
