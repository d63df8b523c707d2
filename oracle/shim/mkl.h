/*
 * Stand-in for the two pieces of Intel MKL the reference's SMD path calls:
 * the DFTI descriptor API for double-precision complex forward transforms
 * (Codes_Folder/smd_code.cpp:2174-2187, Codes_Folder/subrouts.cpp:8415-8417,
 * 12068-12108).  Written for the oracle build only; the transforms run on the
 * oracle's own mixed-radix FFT (oracle/orc_fft.c), not on MKL.
 */
#ifndef ORC_SHIM_MKL_H
#define ORC_SHIM_MKL_H

typedef long MKL_LONG;

enum DFTI_CONFIG_VALUE {
    DFTI_COMPLEX = 32,
    DFTI_REAL = 33,
    DFTI_SINGLE = 35,
    DFTI_DOUBLE = 36
};

#define DFTI_NO_ERROR 0L

/* CBLAS subset used by rotation helpers outside the SMD path
 * (Codes_Folder/aux_code.cpp:860, Codes_Folder/subrouts.cpp:5053-5085);
 * declared so the subroutine file compiles, implemented with plain loops. */
enum CBLAS_LAYOUT { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112 };

void cblas_dgemv(enum CBLAS_LAYOUT layout, enum CBLAS_TRANSPOSE trans,
                 int m, int n, double alpha, const double *a, int lda,
                 const double *x, int incx, double beta, double *y, int incy);
void cblas_dgemm(enum CBLAS_LAYOUT layout, enum CBLAS_TRANSPOSE ta,
                 enum CBLAS_TRANSPOSE tb, int m, int n, int k, double alpha,
                 const double *a, int lda, const double *b, int ldb,
                 double beta, double *c, int ldc);
double cblas_ddot(int n, const double *x, int incx, const double *y,
                  int incy);
void cblas_daxpy(int n, double alpha, const double *x, int incx, double *y,
                 int incy);

struct orc_dfti_desc;
typedef struct orc_dfti_desc *DFTI_DESCRIPTOR_HANDLE;

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE *handle,
                              enum DFTI_CONFIG_VALUE precision,
                              enum DFTI_CONFIG_VALUE domain,
                              MKL_LONG dimension, ...);
MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE handle);
MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE handle, void *data, ...);
MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE *handle);

#endif
