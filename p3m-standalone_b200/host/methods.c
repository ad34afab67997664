/* The method table (types.h:306-316) for the P3M methods 0, 1, 2, 3, 6 and
 * 7, each entry a thin adapter onto the p3mg C ABI, plus the step
 * orchestration of common.c:268-363 (Calculate_forces,
 * Calculate_reference_forces).  Names, short names, ids and flags are the
 * reference's (p3m-ik.c:46-49, p3m-ik-i.c:40-43, p3m-ad.c:39-41,
 * p3m-ad-i.c:39-41, p3m-ik-real.c:43-46, p3m-ad-real.c:39-41): they are
 * what the program prints and what callers select by.
 *
 * Library errors end the program with the library's message (the
 * reference's functions return void and exit on failure as well). */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "p3m_host.h"

void p3m_host_die(int status, const char *what) {
  const char *cuda = p3mg_last_cuda_error();
  fprintf(stderr, "%s failed: %s%s%s\n", what, p3mg_strerror(status), (cuda && *cuda) ? " / " : "",
          (cuda && *cuda) ? cuda : "");
  exit(1);
}

#define CHECK(call, what)             \
  do {                                \
    const int st_ = (call);           \
    if (st_ != P3MG_OK) p3m_host_die(st_, what); \
  } while (0)

static data_t *Init_gpu(int method_id, system_t *s, parameters_t *p) {
  data_t *d = (data_t *)calloc(1, sizeof(data_t));
  if (!d) {
    fputs("out of memory\n", stderr);
    exit(1);
  }
  d->method_id = method_id;
  d->system = s;
  CHECK(p3mg_create(&d->ctx, method_id, p->mesh, p->cao, p->mc, p->precision), "p3mg_create");
  CHECK(p3mg_set_system(d->ctx, s->nparticles, s->p->x, s->p->y, s->p->z, s->q, s->length), "p3mg_set_system");
  CHECK(p3mg_enable_timing(d->ctx, 1), "p3mg_enable_timing");
  return d;
}

void Free_data(data_t *d) {
  if (!d) return;
  p3mg_destroy(d->ctx);
  free(d);
}

static data_t *Init_ik(system_t *s, parameters_t *p) { return Init_gpu(0, s, p); }
static data_t *Init_ik_i(system_t *s, parameters_t *p) { return Init_gpu(1, s, p); }
static data_t *Init_ad(system_t *s, parameters_t *p) { return Init_gpu(2, s, p); }
static data_t *Init_ad_i(system_t *s, parameters_t *p) { return Init_gpu(3, s, p); }
static data_t *Init_ik_r(system_t *s, parameters_t *p) { return Init_gpu(6, s, p); }
static data_t *Init_ad_r(system_t *s, parameters_t *p) { return Init_gpu(7, s, p); }

/* G_opt for p->alpha (once per alpha, main.c:378). */
static void Influence_gpu(system_t *s, parameters_t *p, data_t *d) {
  (void)s;
  CHECK(p3mg_influence(d->ctx, p->alpha), "p3mg_influence");
}

/* Adds the k-space forces into f->f_k; the ad self-force correction of
 * methods 2 and 7 goes into f->f (p3m-ad-self-forces.c:114-139). */
static void Kspace_gpu(system_t *s, parameters_t *p, data_t *d, forces_t *f) {
  (void)s;
  (void)p;
  CHECK(p3mg_kspace_forces(d->ctx, f->f_k->x, f->f_k->y, f->f_k->z, f->f->x, f->f->y, f->f->z),
        "p3mg_kspace_forces");
}

static void estimates(int method_id, const system_t *s, const parameters_t *p, double est[3]) {
  CHECK(p3mg_estimate_errors(method_id, p->mesh, p->cao, p->mc_est, s->nparticles, s->q2, s->length, p->alpha,
                             p->rcut, est),
        "p3mg_estimate_errors");
}

#define ESTIMATE_FNS(tag, id)                                                                         \
  static double Error_##tag(system_t *s, parameters_t *p) {                                           \
    double e[3];                                                                                      \
    estimates(id, s, p, e);                                                                           \
    return e[0];                                                                                      \
  }                                                                                                   \
  static double Error_k_##tag(system_t *s, parameters_t *p) {                                         \
    double e[3];                                                                                      \
    estimates(id, s, p, e);                                                                           \
    return e[1];                                                                                      \
  }
ESTIMATE_FNS(ik, 0)
ESTIMATE_FNS(ik_i, 1)
ESTIMATE_FNS(ad, 2)
ESTIMATE_FNS(ad_i, 3)

const method_t method_p3m_ik = {0, "P3M with ik differentiation, not intelaced.", "p3m-ik",
                                METHOD_FLAG_P3M | METHOD_FLAG_ik, Init_ik, Influence_gpu, Kspace_gpu, Error_ik,
                                Error_k_ik};
const method_t method_p3m_ik_i = {1, "P3M with ik differentiation, interlaced.", "p3m-ik-i",
                                  METHOD_FLAG_P3M | METHOD_FLAG_ik | METHOD_FLAG_interlaced, Init_ik_i,
                                  Influence_gpu, Kspace_gpu, Error_ik_i, Error_k_ik_i};
const method_t method_p3m_ad = {2, "P3M with analytic differentiation, not intelaced.", "p3m-ad",
                                METHOD_FLAG_P3M | METHOD_FLAG_ad | METHOD_FLAG_self_force_correction, Init_ad,
                                Influence_gpu, Kspace_gpu, Error_ad, Error_k_ad};
const method_t method_p3m_ad_i = {3, "P3M with analytic differentiation, intelaced.", "p3m-ad-i",
                                  METHOD_FLAG_P3M | METHOD_FLAG_ad | METHOD_FLAG_interlaced, Init_ad_i,
                                  Influence_gpu, Kspace_gpu, Error_ad_i, Error_k_ad_i};
/* 6 and 7 use the estimates of 0 and 2 (p3m-ik-real.c:45, p3m-ad-real.c:41) */
const method_t method_p3m_ik_r = {6, "P3M with ik differentiation, not intelaced, real input.", "p3m-ik-r",
                                  METHOD_FLAG_P3M | METHOD_FLAG_ik, Init_ik_r, Influence_gpu, Kspace_gpu, Error_ik,
                                  Error_k_ik};
const method_t method_p3m_ad_r = {7, "P3M with analytic differentiation, not intelaced, real input.", "p3m-ad-r",
                                  METHOD_FLAG_P3M | METHOD_FLAG_ad | METHOD_FLAG_self_force_correction, Init_ad_r,
                                  Influence_gpu, Kspace_gpu, Error_ad, Error_k_ad};

const method_t *method_by_id(int id) {
  static const method_t *const all[] = {&method_p3m_ik,   &method_p3m_ik_i, &method_p3m_ad,
                                        &method_p3m_ad_i, &method_p3m_ik_r, &method_p3m_ad_r};
  for (size_t i = 0; i < sizeof all / sizeof all[0]; i++)
    if (all[i]->method_id == id) return all[i];
  return NULL;
}

/* One force evaluation (common.c:268-327): zero f, f_k, f_r; real space if
 * rcut != 0; k space; f += f_k + f_r.  The whole step runs on the GPU in
 * one call for the methods above; another method table entry goes through
 * its own Kspace_force. */
void Calculate_forces(const method_t *m, system_t *s, parameters_t *p, data_t *d, forces_t *f) {
  const size_t bytes = (size_t)s->nparticles * sizeof(double);
  if (d && d->ctx && m->Kspace_force == Kspace_gpu) {
    double e = 0.0;
    CHECK(p3mg_calculate_forces(d->ctx, p->rcut, f->f->x, f->f->y, f->f->z, f->f_k->x, f->f_k->y, f->f_k->z,
                                f->f_r->x, f->f_r->y, f->f_r->z, &e),
          "p3mg_calculate_forces");
    s->energy = e;
    double t[4];
    if (p3mg_stage_times(d->ctx, t) == P3MG_OK)
      for (int i = 0; i < 4; i++) d->runtime[i] = 1e-3 * t[i];
    return;
  }
  for (int i = 0; i < 3; i++) {
    memset(f->f->fields[i], 0, bytes);
    memset(f->f_k->fields[i], 0, bytes);
    memset(f->f_r->fields[i], 0, bytes);
  }
  m->Kspace_force(s, p, d, f);
  for (int j = 0; j < 3; j++)
    for (int i = 0; i < s->nparticles; i++) f->f->fields[j][i] += f->f_k->fields[j][i] + f->f_r->fields[j][i];
}

/* FP64 Ewald reference forces into s->reference (f and f_k), with the
 * reference's choice of alpha and kmax (common.c:329-363); returns the
 * Ewald error estimate. */
double Calculate_reference_forces(system_t *s, parameters_t *p) {
  p3mg_ctx *ctx = NULL;
  CHECK(p3mg_create(&ctx, 1, p->mesh, 1, 0, P3MG_FP64), "p3mg_create");
  CHECK(p3mg_set_system(ctx, s->nparticles, s->p->x, s->p->y, s->p->z, s->q, s->length), "p3mg_set_system");
  double alpha = 0.0, err = 0.0;
  int kmax = 0;
  forces_t *r = s->reference;
  CHECK(p3mg_ewald_reference(ctx, s->nparticles, NULL, r->f->x, r->f->y, r->f->z, r->f_k->x, r->f_k->y, r->f_k->z,
                             &alpha, &kmax, &err),
        "p3mg_ewald_reference");
  for (int j = 0; j < 3; j++)
    for (int i = 0; i < s->nparticles; i++) r->f_r->fields[j][i] = r->f->fields[j][i] - r->f_k->fields[j][i];
  printf("Reference Forces: alpha %lf, r_cut %lf, kmax %d, err %e\n", alpha, 0.49 * s->length, kmax, err);
  p3mg_destroy(ctx);
  return err;
}

/* Realspace_error (realpart.c:343-346) */
double Realspace_error(const system_t *s, const parameters_t *p) {
  return (2.0 * s->q2 * exp(-(p->rcut * p->alpha) * (p->rcut * p->alpha))) /
         sqrt((double)s->nparticles * p->rcut * s->length * s->length * s->length);
}
