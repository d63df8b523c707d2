/*
 * Stand-in for the FFTW3 declarations the reference's subroutine file
 * needs to compile (Codes_Folder/subrouts.cpp:664-688, 7079-8075).  FFTW is
 * disabled on the reference's SMD path (FFTW_ON is rejected at
 * Codes_Folder/smd_code.cpp:357-363); the window-spectrum diagnostic is the
 * only caller that runs, and the oracle build never calls it.  Plans run on
 * the oracle's own FFT when they are executed.
 */
#ifndef ORC_SHIM_FFTW3_H
#define ORC_SHIM_FFTW3_H

typedef double fftw_complex[2];

struct orc_fftw_plan_s;
typedef struct orc_fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_PATIENT (1U << 5)

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in,
                           fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in,
                           fftw_complex *out, int sign, unsigned flags);
void fftw_execute(const fftw_plan plan);
void fftw_destroy_plan(fftw_plan plan);

#endif
