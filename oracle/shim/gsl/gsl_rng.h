/*
 * Stand-in for the GSL random-number declarations used by the reference's
 * MC bootstrap statistics (Codes_Folder/aux_code.cpp:1050-1095).  Not on the
 * SMD path; present so the reference's subroutine file compiles for the
 * oracle build.
 */
#ifndef ORC_SHIM_GSL_RNG_H
#define ORC_SHIM_GSL_RNG_H

typedef struct orc_gsl_rng_type {
    const char *name;
} gsl_rng_type;

typedef struct orc_gsl_rng {
    unsigned long long state;
} gsl_rng;

extern const gsl_rng_type *gsl_rng_default;

gsl_rng *gsl_rng_alloc(const gsl_rng_type *type);
void gsl_rng_set(gsl_rng *r, unsigned long seed);
unsigned long gsl_rng_uniform_int(gsl_rng *r, unsigned long n);
void gsl_rng_free(gsl_rng *r);

#endif
