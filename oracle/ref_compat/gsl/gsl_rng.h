/* Stand-in declarations for the GSL RNG calls in the reference's main();
 * weak and undefined (main() is never called).  TEST INFRASTRUCTURE ONLY. */
#pragma once
typedef struct gsl_rng gsl_rng;
typedef struct gsl_rng_type gsl_rng_type;
__attribute__((weak)) extern const gsl_rng_type *gsl_rng_taus;
__attribute__((weak)) gsl_rng *gsl_rng_alloc(const gsl_rng_type *t);
__attribute__((weak)) void gsl_rng_set(const gsl_rng *r, unsigned long seed);
__attribute__((weak)) double gsl_rng_uniform(const gsl_rng *r);
