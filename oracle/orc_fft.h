/*
 * orc_fft.h -- CPU discrete Fourier transforms used by the oracle (test
 * infrastructure only; never linked into the product library).
 *
 * The reference computes its spatial and temporal transforms with Intel MKL
 * DFTI, complex-to-complex, double precision, forward sign -1, no scaling
 * (Codes_Folder/subrouts.cpp:8415-8417 and 12072-12108).  MKL is not part of
 * the reference tree and is not installed here, so the oracle uses this
 * mixed-radix Cooley-Tukey transform instead.  A DFT is fixed by its
 * definition, so results agree with MKL's to double rounding.
 */
#ifndef ORC_FFT_H
#define ORC_FFT_H

#ifdef __cplusplus
extern "C" {
#endif

/* In-place 1D complex DFT of length n on interleaved (re, im) doubles.
 * sign = -1 gives X[k] = sum_t x[t] exp(-2 pi i k t / n) (MKL forward). */
void orc_fft1d(double *data, long n, int sign);

/* In-place 2D complex DFT of a row-major [n0][n1] array. */
void orc_fft2d(double *data, long n0, long n1, int sign);

/* Naive O(n^2) DFT, used by the tests to check orc_fft1d. */
void orc_dft1d_naive(const double *in, double *out, long n, int sign);

#ifdef __cplusplus
}
#endif

#endif
