/* Test infrastructure: thin C entry points around the REFERENCE's own code,
 * compiled from its unmodified sources (see build_ref.sh) into
 * oracle/_ref/libp3mref.so.  Tests use it to pin the oracle restatement and
 * bench.py uses it as the CPU reference arm.  Nothing here is shipped.
 *
 * Mirrors one alpha step of the reference driver (main.c:359-386):
 *   method.Init (alpha = 0 as at main.c:191) -> Influence_function(alpha)
 *   -> Calculate_forces (common.c:268-327).
 */
#define _POSIX_C_SOURCE 199309L
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "types.h"
#include "common.h"
#include "p3m-common.h"
#include "realpart.h"
#include "ewald.h"
#include "error.h"
#include "p3m-ik.h"
#include "p3m-ik-i.h"
#include "p3m-ad.h"
#include "p3m-ad-i.h"
#include "p3m-ik-real.h"
#include "p3m-ad-real.h"
#include "find_error.h"

static const method_t *method_by_id(int id) {
  switch (id) {
    case 0: return &method_p3m_ik;
    case 1: return &method_p3m_ik_i;
    case 2: return &method_p3m_ad;
    case 3: return &method_p3m_ad_i;
    case 4: return &method_ewald;
    case 6: return &method_p3m_ik_r;
    case 7: return &method_p3m_ad_r;
  }
  return NULL;
}

static system_t *make_system(int n, const double *x, const double *y, const double *z, const double *q, double L) {
  system_t *s = Init_system(n);
  s->length = L;
  s->q2 = 0.0;
  for (int i = 0; i < n; i++) {
    s->p->x[i] = x[i];
    s->p->y[i] = y[i];
    s->p->z[i] = z[i];
    s->q[i] = q[i];
    s->q2 += q[i] * q[i];
  }
  return s;
}

static void copy_out(const vector_array_t *v, int n, double *dst) {
  if (!dst) return;
  for (int d = 0; d < 3; d++) memcpy(dst + (size_t)d * n, v->fields[d], sizeof(double) * n);
}

/* Full force evaluation.  f, fk, fr: 3n doubles each (x block, y block,
 * z block) or NULL.  G: mesh^3 doubles or NULL.  tuning != 0 uses the
 * reference's timing mode (dummy G and weights, p3m-common.c:199-222) and
 * fills times[0..2] = t_c, t_g, t_f when times != NULL.  The number of
 * alphas > 1 runs an alpha sweep with the reference's own accumulation
 * (main.c:375) and returns the forces of the last alpha. */
int ref_forces(int method_id, int mesh, int cao, int mc, double alpha, double rcut, int n, const double *x,
               const double *y, const double *z, const double *q, double L, double *f, double *fk, double *fr,
               double *G, double *energy, int tuning, double *times) {
  const method_t *m = method_by_id(method_id);
  if (!m || method_id == 4) return -1;
  P3M_BRILLOUIN = mc;
  system_t *s = make_system(n, x, y, z, q, L);
  forces_t *fo = Init_forces(n);
  parameters_t p;
  memset(&p, 0, sizeof(p));
  p.rcut = rcut;
  p.mesh = mesh;
  p.cao = cao;
  p.cao3 = cao * cao * cao;
  p.ip = cao - 1;
  p.alpha = 0.0;
  p.tuning = tuning;
  data_t *d = m->Init(s, &p);
  p.alpha = alpha;
  if (!tuning) m->Influence_function(s, &p, d);
  s->energy = 0.0;
  Calculate_forces(m, s, &p, d, fo);
  copy_out(fo->f, n, f);
  copy_out(fo->f_k, n, fk);
  copy_out(fo->f_r, n, fr);
  if (G && !tuning) memcpy(G, d->G_hat, sizeof(double) * (size_t)mesh * mesh * mesh);
  if (energy) *energy = s->energy;
  if (times) {
    times[0] = d->runtime.t_c;
    times[1] = d->runtime.t_g;
    times[2] = d->runtime.t_f;
  }
  Free_data(d);
  Free_forces(fo);
  Free_system(s);
  return 0;
}

/* Self-force coefficients b(m') (81 doubles, m' in {-1,0,1}^3 row-major,
 * three directions each) after Influence_function of an ad method. */
int ref_self_force_coefficients(int method_id, int mesh, int cao, int mc, double alpha, int n, const double *x,
                                const double *y, const double *z, const double *q, double L, double *b81) {
  const method_t *m = method_by_id(method_id);
  if (!m || !(m->flags & METHOD_FLAG_self_force_correction)) return -1;
  P3M_BRILLOUIN = mc;
  system_t *s = make_system(n, x, y, z, q, L);
  parameters_t p;
  memset(&p, 0, sizeof(p));
  p.mesh = mesh;
  p.cao = cao;
  p.cao3 = cao * cao * cao;
  p.ip = cao - 1;
  p.alpha = 0.0;
  data_t *d = m->Init(s, &p);
  p.alpha = alpha;
  m->Influence_function(s, &p, d);
  memcpy(b81, d->self_force_corrections, sizeof(double) * 81);
  Free_data(d);
  Free_system(s);
  return 0;
}

/* Ewald reference forces exactly as the driver computes them
 * (Calculate_reference_forces, common.c:329-363).  Returns the error
 * estimate; alpha/kmax used are written to *alpha_out / *kmax_out. */
double ref_ewald(int n, const double *x, const double *y, const double *z, const double *q, double L, int mesh_param,
                 double *f, double *fk, double *fr, double *alpha_out, int *kmax_out) {
  system_t *s = make_system(n, x, y, z, q, L);
  parameters_t p;
  memset(&p, 0, sizeof(p));
  p.mesh = mesh_param;
  p.cao = 1;
  p.cao3 = 1;
  double err = Calculate_reference_forces(s, &p);
  copy_out(s->reference->f, n, f);
  copy_out(s->reference->f_k, n, fk);
  copy_out(s->reference->f_r, n, fr);
  if (alpha_out || kmax_out) {
    parameters_t op = p;
    op.rcut = 0.49 * s->length;
    op.mesh = mesh_param;
    op.alpha = Ewald_compute_optimal_alpha(s, &op);
    op.mesh = 2;
    while (method_ewald.Error(s, &op) > 1e-8) op.mesh += 2;
    if (alpha_out) *alpha_out = op.alpha;
    if (kmax_out) *kmax_out = op.mesh;
  }
  Free_system(s);
  return err;
}

/* Ewald k-space forces the way main.c's "error_k" column gets them
 * (main.c:190-196 copies the parameters with alpha = 0 before
 * method_ewald.Init; main.c:392-396 per alpha): Init with the P3M mesh, then
 * Influence_function and Kspace_force at alpha.  fk: 3n, overwritten. */
int ref_ewald_kspace_main(int n, const double *x, const double *y, const double *z, const double *q, double L,
                          int mesh, double alpha, double *fk) {
  system_t *s = make_system(n, x, y, z, q, L);
  forces_t *f = Init_forces(n);
  parameters_t p;
  memset(&p, 0, sizeof(p));
  p.mesh = mesh;
  p.cao = 1;
  p.cao3 = 1;
  p.alpha = 0.0;
  data_t *d = method_ewald.Init(s, &p);
  p.alpha = alpha;
  method_ewald.Influence_function(s, &p, d);
  method_ewald.Kspace_force(s, &p, d, f);
  copy_out(f->f_k, n, fk);
  Free_data(d);
  Free_forces(f);
  Free_system(s);
  return 0;
}

/* The method's error estimates (Error, Error_k) and Realspace_error. */
int ref_error_estimates(int method_id, int mesh, int cao, int mc, double alpha, double rcut, int n, const double *q,
                        double L, double *est3) {
  const method_t *m = method_by_id(method_id);
  if (!m || !m->Error) return -1;
  P3M_BRILLOUIN = mc;
  P3M_BRILLOUIN_TUNING = mc;
  double *zero = (double *)calloc((size_t)n, sizeof(double));
  system_t *s = make_system(n, zero, zero, zero, q, L);
  parameters_t p;
  memset(&p, 0, sizeof(p));
  p.rcut = rcut;
  p.mesh = mesh;
  p.cao = cao;
  p.cao3 = cao * cao * cao;
  p.ip = cao - 1;
  p.alpha = alpha;
  est3[0] = m->Error(s, &p);
  est3[1] = m->Error_k(s, &p);
  est3[2] = Realspace_error(s, &p);
  P3M_BRILLOUIN_TUNING = 1;
  Free_system(s);
  free(zero);
  return 0;
}

/* The reference's precomputed-table lookup (find_error.c:84-107): the
 * interpolated he_q for a tabulated (mesh, cao) or -1 on a miss. */
double ref_find_error(double alphaL, int mesh, int cao, int method_id) {
  return p3m_find_error(alphaL, mesh, cao, method_id);
}

/* Wall-clock seconds of the reference's timed region, one full
 * Calculate_forces (common.c:268-327: zeroing, Realteil when rcut != 0,
 * Kspace_force, f = f_k + f_r), as main.c:382-386 brackets it: Init and
 * Influence_function run once before the clock starts.  Returns the mean of
 * `reps` steps (<0 on an unknown method). */
double ref_step_seconds(int method_id, int mesh, int cao, int mc, double alpha, double rcut, int n, const double *x,
                        const double *y, const double *z, const double *q, double L, int reps) {
  const method_t *m = method_by_id(method_id);
  if (!m || method_id == 4 || reps < 1) return -1.0;
  P3M_BRILLOUIN = mc;
  system_t *s = make_system(n, x, y, z, q, L);
  forces_t *fo = Init_forces(n);
  parameters_t p;
  memset(&p, 0, sizeof(p));
  p.rcut = rcut;
  p.mesh = mesh;
  p.cao = cao;
  p.cao3 = cao * cao * cao;
  p.ip = cao - 1;
  p.alpha = 0.0;
  data_t *d = m->Init(s, &p);
  p.alpha = alpha;
  m->Influence_function(s, &p, d);
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (int r = 0; r < reps; r++) {
    s->energy = 0.0;
    Calculate_forces(m, s, &p, d, fo);
  }
  clock_gettime(CLOCK_MONOTONIC, &t1);
  Free_data(d);
  Free_forces(fo);
  Free_system(s);
  return ((double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec)) / reps;
}

/* The reference's real-space N^2 loop alone (realpart.c:124-167). */
int ref_realteil(int n, const double *x, const double *y, const double *z, const double *q, double L, double rcut,
                 double alpha, double *fr, double *energy) {
  system_t *s = make_system(n, x, y, z, q, L);
  forces_t *fo = Init_forces(n);
  parameters_t p;
  memset(&p, 0, sizeof(p));
  p.rcut = rcut;
  p.alpha = alpha;
  s->energy = 0.0;
  Realteil(s, &p, fo);
  copy_out(fo->f_r, n, fr);
  if (energy) *energy = s->energy;
  Free_forces(fo);
  Free_system(s);
  return 0;
}

/* The reference's inhomogeneous estimate (p3m-common.c:437-719) as main.c
 * calls it (main.c:436-440): `p` carries the force method's mesh, cao and
 * alpha; mesh/cao/mc are the estimator's own. */
double ref_inhomo_error(int n, const double *x, const double *y, const double *z, const double *q, double L,
                        int method_mesh, int method_cao, double alpha, int uniform, int mesh, int cao, int mc,
                        const char *out_file) {
  system_t *s = make_system(n, x, y, z, q, L);
  parameters_t p;
  memset(&p, 0, sizeof(p));
  p.mesh = method_mesh;
  p.cao = method_cao;
  p.cao3 = method_cao * method_cao * method_cao;
  p.ip = method_cao - 1;
  p.alpha = alpha;
  const double r = Generic_error_estimate_inhomo(s, &p, uniform, mesh, cao, mc, (char *)out_file, NULL);
  Free_system(s);
  return r;
}

/* The reference's Error_map (p3m-common.c:402-435): fk, fk_ref 3n each;
 * map receives the real parts of its mesh^3 complex mesh. */
int ref_error_map(int n, const double *x, const double *y, const double *z, double L, const double *fk,
                  const double *fk_ref, int mesh, int cao, double *map) {
  double *zero = (double *)calloc((size_t)n + 1, sizeof(double));
  system_t *s = make_system(n, x, y, z, zero, L);
  forces_t *f = Init_forces(n), *fr = Init_forces(n);
  for (int d = 0; d < 3; d++) {
    memcpy(f->f_k->fields[d], fk + (size_t)d * n, sizeof(double) * n);
    memcpy(fr->f_k->fields[d], fk_ref + (size_t)d * n, sizeof(double) * n);
  }
  double *em = Error_map(s, f, fr, mesh, cao);
  const size_t M = (size_t)mesh * mesh * mesh;
  for (size_t t = 0; t < M; t++) map[t] = em[2 * t];
  FFTW_FREE(em);
  Free_forces(f);
  Free_forces(fr);
  Free_system(s);
  free(zero);
  return 0;
}
