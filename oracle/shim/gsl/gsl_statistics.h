/*
 * Stand-in for the GSL statistics declarations used by the reference's MC
 * bootstrap statistics (Codes_Folder/aux_code.cpp:1084-1127).  Not on the
 * SMD path; present so the reference's subroutine file compiles for the
 * oracle build.
 */
#ifndef ORC_SHIM_GSL_STATISTICS_H
#define ORC_SHIM_GSL_STATISTICS_H

#include <stddef.h>

double gsl_stats_mean(const double data[], size_t stride, size_t n);
double gsl_stats_sd(const double data[], size_t stride, size_t n);

#endif
