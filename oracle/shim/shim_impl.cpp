/*
 * shim_impl.cpp -- definitions behind the stand-in MKL DFTI, FFTW3 and GSL
 * headers in this folder.  Test infrastructure: it exists only so that the
 * reference's own Codes_Folder/subrouts.cpp can be compiled and run here as a
 * parity pin for the oracle.  Every transform runs on oracle/orc_fft.c.
 */
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <vector>

#include "mkl.h"
#include "fftw3.h"
#include "gsl/gsl_rng.h"
#include "gsl/gsl_statistics.h"

extern "C" {
#include "../orc_fft.h"
}

/* ---------------------------------------------------------------- DFTI */

struct orc_dfti_desc {
    int rank;
    long n[2];
    bool double_complex;
};

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE *handle,
                              enum DFTI_CONFIG_VALUE precision,
                              enum DFTI_CONFIG_VALUE domain,
                              MKL_LONG dimension, ...)
{
    if (!handle) return 1;
    orc_dfti_desc *d = new orc_dfti_desc();
    d->rank = (int)dimension;
    d->double_complex = (precision == DFTI_DOUBLE && domain == DFTI_COMPLEX);
    va_list ap;
    va_start(ap, dimension);
    if (dimension == 1) {
        d->n[0] = va_arg(ap, MKL_LONG);
        d->n[1] = 1;
    } else if (dimension == 2) {
        MKL_LONG *dims = va_arg(ap, MKL_LONG *);
        d->n[0] = dims[0];
        d->n[1] = dims[1];
    } else {
        va_end(ap);
        delete d;
        *handle = nullptr;
        return 2;
    }
    va_end(ap);
    *handle = d;
    return d->double_complex ? DFTI_NO_ERROR : 3;
}

MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE handle)
{
    return handle ? DFTI_NO_ERROR : 1;
}

MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE handle, void *data, ...)
{
    if (!handle || !data || !handle->double_complex) return 1;
    double *x = static_cast<double *>(data);
    if (handle->rank == 1)
        orc_fft1d(x, handle->n[0], -1);
    else
        orc_fft2d(x, handle->n[0], handle->n[1], -1);
    return DFTI_NO_ERROR;
}

MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE *handle)
{
    if (handle && *handle) {
        delete *handle;
        *handle = nullptr;
    }
    return DFTI_NO_ERROR;
}

/* --------------------------------------------------------------- CBLAS */

/* Row-major, no-transpose only: the forms the reference calls. */
void cblas_dgemv(enum CBLAS_LAYOUT, enum CBLAS_TRANSPOSE, int m, int n,
                 double alpha, const double *a, int lda, const double *x,
                 int incx, double beta, double *y, int incy)
{
    for (int i = 0; i < m; i++) {
        double s = 0.0;
        for (int j = 0; j < n; j++) s += a[i * lda + j] * x[j * incx];
        y[i * incy] = alpha * s + beta * y[i * incy];
    }
}

void cblas_dgemm(enum CBLAS_LAYOUT, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE,
                 int m, int n, int k, double alpha, const double *a, int lda,
                 const double *b, int ldb, double beta, double *c, int ldc)
{
    for (int i = 0; i < m; i++)
        for (int j = 0; j < n; j++) {
            double s = 0.0;
            for (int l = 0; l < k; l++) s += a[i * lda + l] * b[l * ldb + j];
            c[i * ldc + j] = alpha * s + beta * c[i * ldc + j];
        }
}

double cblas_ddot(int n, const double *x, int incx, const double *y, int incy)
{
    double s = 0.0;
    for (int i = 0; i < n; i++) s += x[i * incx] * y[i * incy];
    return s;
}

void cblas_daxpy(int n, double alpha, const double *x, int incx, double *y,
                 int incy)
{
    for (int i = 0; i < n; i++) y[i * incy] += alpha * x[i * incx];
}

/* ---------------------------------------------------------------- FFTW */

struct orc_fftw_plan_s {
    int rank;
    long n[3];
    int sign;
    fftw_complex *in;
    fftw_complex *out;
};

static fftw_plan make_plan(int rank, long n0, long n1, long n2,
                           fftw_complex *in, fftw_complex *out, int sign)
{
    fftw_plan p = new orc_fftw_plan_s();
    p->rank = rank;
    p->n[0] = n0;
    p->n[1] = n1;
    p->n[2] = n2;
    p->sign = sign;
    p->in = in;
    p->out = out;
    return p;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned)
{
    return make_plan(1, n, 1, 1, in, out, sign);
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in,
                           fftw_complex *out, int sign, unsigned)
{
    return make_plan(2, n0, n1, 1, in, out, sign);
}

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in,
                           fftw_complex *out, int sign, unsigned)
{
    return make_plan(3, n0, n1, n2, in, out, sign);
}

void fftw_execute(const fftw_plan p)
{
    if (!p) return;
    long total = p->n[0] * p->n[1] * p->n[2];
    std::vector<double> buf(2 * total);
    std::memcpy(buf.data(), p->in, sizeof(double) * 2 * total);
    if (p->rank == 1) {
        orc_fft1d(buf.data(), p->n[0], p->sign);
    } else if (p->rank == 2) {
        orc_fft2d(buf.data(), p->n[0], p->n[1], p->sign);
    } else {
        /* 3D: transform the trailing two axes, then the leading one. */
        long plane = p->n[1] * p->n[2];
        for (long a = 0; a < p->n[0]; a++)
            orc_fft2d(buf.data() + 2 * a * plane, p->n[1], p->n[2], p->sign);
        std::vector<double> col(2 * p->n[0]);
        for (long e = 0; e < plane; e++) {
            for (long a = 0; a < p->n[0]; a++) {
                col[2 * a] = buf[2 * (a * plane + e)];
                col[2 * a + 1] = buf[2 * (a * plane + e) + 1];
            }
            orc_fft1d(col.data(), p->n[0], p->sign);
            for (long a = 0; a < p->n[0]; a++) {
                buf[2 * (a * plane + e)] = col[2 * a];
                buf[2 * (a * plane + e) + 1] = col[2 * a + 1];
            }
        }
    }
    std::memcpy(p->out, buf.data(), sizeof(double) * 2 * total);
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

/* ----------------------------------------------------------------- GSL */

static const gsl_rng_type orc_default_type = {"orc-splitmix64"};
const gsl_rng_type *gsl_rng_default = &orc_default_type;

gsl_rng *gsl_rng_alloc(const gsl_rng_type *)
{
    gsl_rng *r = new gsl_rng();
    r->state = 0x9E3779B97F4A7C15ULL;
    return r;
}

void gsl_rng_set(gsl_rng *r, unsigned long seed) { r->state = seed; }

unsigned long gsl_rng_uniform_int(gsl_rng *r, unsigned long n)
{
    unsigned long long z = (r->state += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return n ? (unsigned long)(z % n) : 0UL;
}

void gsl_rng_free(gsl_rng *r) { delete r; }

double gsl_stats_mean(const double data[], size_t stride, size_t n)
{
    double s = 0.0;
    for (size_t i = 0; i < n; i++) s += data[i * stride];
    return n ? s / (double)n : 0.0;
}

double gsl_stats_sd(const double data[], size_t stride, size_t n)
{
    if (n < 2) return 0.0;
    double m = gsl_stats_mean(data, stride, n), s = 0.0;
    for (size_t i = 0; i < n; i++) {
        double d = data[i * stride] - m;
        s += d * d;
    }
    return std::sqrt(s / (double)(n - 1));
}
