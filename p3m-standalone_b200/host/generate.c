/* Generated test systems with the reference's six system types
 * (generate_system.c:29-224) and the same random stream: the reference draws
 * from GSL's default generator, MT19937 (Matsumoto & Nishimura 1998) seeded
 * with GSL's default seed 0 -> 4357 and the 1812433253 initialisation,
 * gsl_rng_uniform = 32-bit output / 2^32, and gsl_ran_gaussian = the polar
 * Box-Muller method on gsl_rng_uniform_pos.  Every system type allocates a
 * fresh generator, so each starts the stream from the seed.
 *
 * Charges: +-charge alternating (random and Gaussian), +-1 otherwise.  As in
 * the reference code (not its README), type 5 places y in [0.45 L, 0.55 L)
 * and the Gaussian type uses sigma = 0.5 around the box centre. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>

#include "p3m_host.h"

#define MT_N 624
#define MT_M 397

typedef struct {
  uint32_t mt[MT_N];
  int mti;
} mt_state;

static void mt_seed(mt_state *st, uint32_t seed) {
  if (seed == 0) seed = 4357; /* GSL's default seed */
  st->mt[0] = seed;
  for (int i = 1; i < MT_N; i++) st->mt[i] = 1812433253u * (st->mt[i - 1] ^ (st->mt[i - 1] >> 30)) + (uint32_t)i;
  st->mti = MT_N;
}

static uint32_t mt_next(mt_state *st) {
  static const uint32_t mag[2] = {0u, 0x9908b0dfu};
  if (st->mti >= MT_N) {
    int k;
    for (k = 0; k < MT_N - MT_M; k++) {
      const uint32_t y = (st->mt[k] & 0x80000000u) | (st->mt[k + 1] & 0x7fffffffu);
      st->mt[k] = st->mt[k + MT_M] ^ (y >> 1) ^ mag[y & 1u];
    }
    for (; k < MT_N - 1; k++) {
      const uint32_t y = (st->mt[k] & 0x80000000u) | (st->mt[k + 1] & 0x7fffffffu);
      st->mt[k] = st->mt[k + (MT_M - MT_N)] ^ (y >> 1) ^ mag[y & 1u];
    }
    const uint32_t y = (st->mt[MT_N - 1] & 0x80000000u) | (st->mt[0] & 0x7fffffffu);
    st->mt[MT_N - 1] = st->mt[MT_M - 1] ^ (y >> 1) ^ mag[y & 1u];
    st->mti = 0;
  }
  uint32_t y = st->mt[st->mti++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

static double uniform(mt_state *st) { return mt_next(st) / 4294967296.0; }

static double uniform_pos(mt_state *st) {
  double x;
  do x = uniform(st);
  while (x == 0.0);
  return x;
}

static double gaussian(mt_state *st, double sigma) {
  double x, y, r2;
  do {
    x = -1.0 + 2.0 * uniform_pos(st);
    y = -1.0 + 2.0 * uniform_pos(st);
    r2 = x * x + y * y;
  } while (r2 > 1.0 || r2 == 0.0);
  return sigma * y * sqrt(-2.0 * log(r2) / r2);
}

static system_t *new_system(int n, double box) {
  system_t *s = Init_system(n);
  s->length = box;
  s->q2 = 0.0;
  return s;
}

static system_t *random_system(int n, double box, double charge) {
  mt_state st;
  mt_seed(&st, 0);
  system_t *s = new_system(n, box);
  for (int i = 0; i < n; i++) {
    for (int d = 0; d < 3; d++) s->p->fields[d][i] = box * uniform(&st);
    s->q[i] = (1.0 - 2.0 * (i % 2)) * charge;
    s->q2 += s->q[i] * s->q[i];
  }
  return s;
}

static system_t *gaussian_system(int n, double box, double charge) {
  mt_state st;
  mt_seed(&st, 0);
  system_t *s = new_system(n, box);
  for (int i = 0; i < n; i++) {
    for (int d = 0; d < 3; d++) {
      double x;
      while (fabs(x = box / 2 + gaussian(&st, 0.5)) >= box) printf("%lf\n", x);
      s->p->fields[d][i] = x;
    }
    s->q[i] = (1.0 - 2.0 * (i % 2)) * charge;
    s->q2 += s->q[i] * s->q[i];
  }
  return s;
}

static system_t *inner_box(int n, double box) {
  puts("Generating inner box system.");
  mt_state st;
  mt_seed(&st, 0);
  system_t *s = new_system(n, box);
  for (int i = 0; i < n; i++) {
    for (int d = 0; d < 3; d++) s->p->fields[d][i] = 0.25 * box + 0.5 * box * uniform(&st);
    s->q[i] = 1.0 - 2.0 * (i % 2);
    s->q2 += s->q[i] * s->q[i];
  }
  return s;
}

static system_t *madelung(int n, double box) {
  const int per_row = (int)ceil(pow(n, 0.33333));
  const double a = box / per_row, off = 0.5 * a;
  n = per_row * per_row * per_row;
  printf("generate_madelung: box %lf, size %d, per_row %d, a %lf, off %lf\n", box, n, per_row, a, off);
  system_t *s = new_system(n, box);
  int id = 0;
  for (int i = 0; i < per_row; i++)
    for (int j = 0; j < per_row; j++)
      for (int k = 0; k < per_row; k++, id++) {
        s->p->x[id] = a * i + off;
        s->p->y[id] = a * j + off;
        s->p->z[id] = a * k + off;
        s->q[id] = 1.0 - 2.0 * ((i + j + k) % 2);
        s->q2 += s->q[id] * s->q[id];
      }
  return s;
}

static system_t *separated_dipoles(int n, double box) {
  const int ndip = n / 2;
  const double dist = 1.0, pi = 3.14159265358979323846264338328;
  mt_state st;
  mt_seed(&st, 0);
  system_t *s = new_system(2 * ndip, box);
  for (int i = 0, id = 0; i < ndip; i++, id += 2) {
    double x[3], dir[3];
    for (int d = 0; d < 3; d++) x[d] = box * uniform(&st);
    const double u = -1.0 + 2.0 * uniform(&st);
    const double theta = 2.0 * pi * uniform(&st);
    dir[0] = sqrt(1.0 - u * u) * cos(theta);
    dir[1] = sqrt(1.0 - u * u) * sin(theta);
    dir[2] = u;
    for (int d = 0; d < 3; d++) {
      double y = x[d] + dist * dir[d];
      while (y >= box) y -= box;
      while (y < 0.0) y += box;
      s->p->fields[d][id] = x[d];
      s->p->fields[d][id + 1] = y;
    }
    s->q[id] = 1.0;
    s->q[id + 1] = -1.0;
    s->q2 += 2.0;
  }
  return s;
}

static system_t *slab(int n, double box) {
  const double width = 0.1 * box, lower = 0.45 * box;
  printf("Generating slab system with %lf < x < %lf\n", lower, lower + width);
  mt_state st;
  mt_seed(&st, 0);
  system_t *s = new_system(n, box);
  for (int i = 0; i < n; i++) {
    s->p->y[i] = lower + width * uniform(&st);
    s->p->x[i] = box * uniform(&st);
    s->p->z[i] = box * uniform(&st);
    s->q[i] = 1.0 - 2.0 * (i % 2);
    s->q2 += s->q[i] * s->q[i];
  }
  return s;
}

system_t *generate_system(int type, int size, double box, double charge) {
  switch (type) {
    case SYSTEM_RANDOM: return random_system(size, box, charge);
    case SYSTEM_GAUSSIAN: return gaussian_system(size, box, charge);
    case SYSTEM_INNER_BOX: return inner_box(size, box);
    case SYSTEM_MADELUNG: return madelung(size, box);
    case SYSTEM_SEPARATED_DIPOLE: return separated_dipoles(size, box);
    case SYSTEM_SLAB: return slab(size, box);
    default: fprintf(stderr, "Warning, form factor not known.\n");
  }
  return NULL;
}
