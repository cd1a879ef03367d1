/*
 * Mixed-radix complex FFT in plain C99 (double precision).
 *
 * TEST INFRASTRUCTURE ONLY.  This file belongs to the CPU oracle: it is used
 * by the oracle restatement (oracle/npme_oracle.c) and by the project-written
 * replacement of the reference's MKL wrapper (oracle/ref/ext_library_shim.cpp)
 * that lets the reference's own sources be compiled here for parity checks.
 * Nothing in the GPU product links it.
 *
 * Conventions follow the reference's MKL usage (src/ExtLibrary.cpp:930-1090):
 * forward transform = sum_j x[j] exp(-2 pi i k j / n), no normalisation.
 * The backward transform uses exp(+2 pi i k j / n), also unnormalised.
 *
 * Algorithm: recursive decimation in time over the prime factorisation of n
 * (radix 4, 2, 3, 5 butterflies, generic O(p^2) butterfly for other primes).
 */
#ifndef NPME_ORACLE_FFT_H
#define NPME_ORACLE_FFT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_fft_plan orc_fft_plan;

/* Plans are cached per (n, sign); the cache is thread safe. */
const orc_fft_plan *orc_fft_plan_get(long n, int sign);

/* In-place 1-D transform of n complex doubles stored as (re, im) pairs.
 * work must hold n complex values (2n doubles). */
void orc_fft_exec(const orc_fft_plan *p, double *data, double *work);

/* Convenience: 1-D in place, allocates its own scratch. */
void orc_fft_1d(double *data, long n, int sign);

/* 3-D in place on data[n1][n2][n3] (row major, complex interleaved).
 * nthreads <= 1 runs serially; otherwise OpenMP over lines. */
void orc_fft_3d(double *data, long n1, long n2, long n3, int sign, int nthreads);

/* Batched 3-D: K consecutive n1*n2*n3 blocks. */
void orc_fft_3d_many(double *data, long K, long n1, long n2, long n3, int sign,
                     int nthreads);

#ifdef __cplusplus
}
#endif

#endif
