/* Test infrastructure: GSL API subset for linking the reference.
 * MT19937 per Matsumoto & Nishimura (1998), GSL-style default seed 4357;
 * gsl_rng_uniform = next 32-bit word / 2^32.  Gaussian: Box-Muller
 * (polar form, Marsaglia 1964).  I0: power series sum (x/2)^(2k)/(k!)^2. */
#include <math.h>
#include <stdlib.h>
#include "gsl/gsl_rng.h"
#include "gsl/gsl_randist.h"
#include "gsl/gsl_sf_bessel.h"

struct oracle_gsl_rng_s { unsigned long mt[624]; int mti; };
static const gsl_rng_type mt_type = {"mt19937"};
const gsl_rng_type *gsl_rng_default = &mt_type;

static void mt_seed(gsl_rng *r, unsigned long s) {
  if (s == 0) s = 4357;
  r->mt[0] = s & 0xffffffffUL;
  for (int i = 1; i < 624; i++)
    r->mt[i] = (1812433253UL * (r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) + (unsigned long)i) & 0xffffffffUL;
  r->mti = 624;
}

static unsigned long mt_next(gsl_rng *r) {
  static const unsigned long mag01[2] = {0x0UL, 0x9908b0dfUL};
  unsigned long y;
  if (r->mti >= 624) {
    int kk;
    for (kk = 0; kk < 624 - 397; kk++) {
      y = (r->mt[kk] & 0x80000000UL) | (r->mt[kk + 1] & 0x7fffffffUL);
      r->mt[kk] = r->mt[kk + 397] ^ (y >> 1) ^ mag01[y & 1UL];
    }
    for (; kk < 623; kk++) {
      y = (r->mt[kk] & 0x80000000UL) | (r->mt[kk + 1] & 0x7fffffffUL);
      r->mt[kk] = r->mt[kk + (397 - 624)] ^ (y >> 1) ^ mag01[y & 1UL];
    }
    y = (r->mt[623] & 0x80000000UL) | (r->mt[0] & 0x7fffffffUL);
    r->mt[623] = r->mt[396] ^ (y >> 1) ^ mag01[y & 1UL];
    r->mti = 0;
  }
  y = r->mt[r->mti++];
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9d2c5680UL;
  y ^= (y << 15) & 0xefc60000UL;
  y ^= (y >> 18);
  return y & 0xffffffffUL;
}

gsl_rng *gsl_rng_alloc(const gsl_rng_type *t) {
  (void)t;
  gsl_rng *r = (gsl_rng *)malloc(sizeof(gsl_rng));
  mt_seed(r, 0);
  return r;
}
void gsl_rng_free(gsl_rng *r) { free(r); }
double gsl_rng_uniform(const gsl_rng *r) { return mt_next((gsl_rng *)r) / 4294967296.0; }

static double uniform_pos(const gsl_rng *r) {
  double x;
  do x = gsl_rng_uniform(r);
  while (x == 0.0);
  return x;
}

/* GSL's gsl_ran_gaussian: polar Box-Muller on two gsl_rng_uniform_pos draws
 * (x, y) in the unit disc, returning the y-based variate. */
double gsl_ran_gaussian(const gsl_rng *r, double sigma) {
  double x, y, s;
  do {
    x = -1.0 + 2.0 * uniform_pos(r);
    y = -1.0 + 2.0 * uniform_pos(r);
    s = x * x + y * y;
  } while (s > 1.0 || s == 0.0);
  return sigma * y * sqrt(-2.0 * log(s) / s);
}

double gsl_sf_bessel_I0(double x) {
  double term = 1.0, sum = 1.0, q = 0.25 * x * x;
  for (int k = 1; k < 500 && term > 1e-17 * sum; k++) {
    term *= q / ((double)k * (double)k);
    sum += term;
  }
  return sum;
}
