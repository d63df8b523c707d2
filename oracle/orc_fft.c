/*
 * orc_fft.c -- mixed-radix DFT for the oracle (test infrastructure only).
 *
 * Recursive decimation in time: a length-n transform with smallest prime
 * factor p is split into p sub-transforms of length n/p over the decimated
 * sequences, then combined with an O(p^2) butterfly per output column.
 * Twiddles come from one table of exp(sign 2 pi i j / n) for the top-level
 * n, built with cos/sin of reduced arguments, so every twiddle is accurate to
 * one double rounding.  Lengths with large prime factors fall back to O(n p),
 * which is acceptable at the sizes the oracle runs.
 */
#include "orc_fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static long smallest_factor(long n)
{
    if (n % 2 == 0) return 2;
    if (n % 3 == 0) return 3;
    if (n % 5 == 0) return 5;
    for (long p = 7; p * p <= n; p += 2)
        if (n % p == 0) return p;
    return n;
}

/* out[0..n) = DFT of in[0], in[stride], ...; tw = top-level table of size N,
 * step = N / n maps a length-n twiddle index onto it. */
static void fft_rec(const double *in, double *out, long n, long stride,
                    const double *tw, long N, long step, double *tmp)
{
    if (n == 1) {
        out[0] = in[0];
        out[1] = in[1];
        return;
    }
    long p = smallest_factor(n);
    long m = n / p;
    for (long r = 0; r < p; r++)
        fft_rec(in + 2 * r * stride, out + 2 * r * m, m, stride * p, tw, N,
                step * p, tmp);
    /* out[r*m + k] holds Y_r[k]; combine into X[k + m q]. */
    for (long k = 0; k < m; k++) {
        for (long q = 0; q < p; q++) {
            double re = 0.0, im = 0.0;
            long kk = k + m * q;
            for (long r = 0; r < p; r++) {
                long idx = ((r * kk) % n) * step;
                double wr = tw[2 * idx], wi = tw[2 * idx + 1];
                double yr = out[2 * (r * m + k)], yi = out[2 * (r * m + k) + 1];
                re += wr * yr - wi * yi;
                im += wr * yi + wi * yr;
            }
            tmp[2 * q] = re;
            tmp[2 * q + 1] = im;
        }
        for (long q = 0; q < p; q++) {
            out[2 * (k + m * q)] = tmp[2 * q];
            out[2 * (k + m * q) + 1] = tmp[2 * q + 1];
        }
    }
}

void orc_fft1d(double *data, long n, int sign)
{
    if (n <= 1) return;
    double *tw = (double *)malloc(sizeof(double) * 2 * n);
    double *out = (double *)malloc(sizeof(double) * 2 * n);
    double *tmp = (double *)malloc(sizeof(double) * 2 * n);
    const double two_pi = 2.0 * acos(-1.0);
    for (long j = 0; j < n; j++) {
        /* reduce to [-n/2, n/2] before taking the angle */
        long jj = (2 * j > n) ? j - n : j;
        double a = two_pi * (double)jj / (double)n;
        tw[2 * j] = cos(a);
        tw[2 * j + 1] = (double)sign * sin(a);
    }
    fft_rec(data, out, n, 1, tw, n, 1, tmp);
    memcpy(data, out, sizeof(double) * 2 * n);
    free(tw);
    free(out);
    free(tmp);
}

void orc_fft2d(double *data, long n0, long n1, int sign)
{
    for (long i = 0; i < n0; i++) orc_fft1d(data + 2 * i * n1, n1, sign);
    double *col = (double *)malloc(sizeof(double) * 2 * n0);
    for (long j = 0; j < n1; j++) {
        for (long i = 0; i < n0; i++) {
            col[2 * i] = data[2 * (i * n1 + j)];
            col[2 * i + 1] = data[2 * (i * n1 + j) + 1];
        }
        orc_fft1d(col, n0, sign);
        for (long i = 0; i < n0; i++) {
            data[2 * (i * n1 + j)] = col[2 * i];
            data[2 * (i * n1 + j) + 1] = col[2 * i + 1];
        }
    }
    free(col);
}

void orc_dft1d_naive(const double *in, double *out, long n, int sign)
{
    const double two_pi = 2.0 * acos(-1.0);
    for (long k = 0; k < n; k++) {
        double re = 0.0, im = 0.0;
        for (long t = 0; t < n; t++) {
            long idx = (k * t) % n;
            double a = two_pi * (double)idx / (double)n;
            double wr = cos(a), wi = sign * sin(a);
            re += wr * in[2 * t] - wi * in[2 * t + 1];
            im += wr * in[2 * t + 1] + wi * in[2 * t];
        }
        out[2 * k] = re;
        out[2 * k + 1] = im;
    }
}
