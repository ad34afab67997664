/* p3mg-backed method tables for p3m-standalone (see p3m-gpu.h).
 *
 * Init creates one p3mg context per data_t (kept in data_t.method_data) for
 * the method's mesh, cao and the global aliasing order P3M_BRILLOUIN;
 * Influence_function computes G_opt for p->alpha on the GPU; Kspace_force
 * re-uploads the positions (they move between steps in a simulation) and
 * adds the k-space forces into f->f_k like the reference's P3M_* drivers,
 * subtracting the ad self-force from f->f for methods 2 and 7.  The
 * reference's Calculate_forces (common.c:268-327) calls these through the
 * table like any CPU method.  Library errors end the program the way the
 * reference reports a bad method (exit 126, main.c:346-349). */
#include <stdio.h>
#include <stdlib.h>

#include "common.h"
#include "p3m-common.h"
#include "p3m-ad-i.h"
#include "p3m-ad.h"
#include "p3m-ik-i.h"
#include "p3m-ik.h"
#include "p3m-gpu.h"
#include "p3mg.h"

static int gpu_precision = P3MG_FP64;

void p3m_gpu_set_precision(int precision) { gpu_precision = precision; }

static void check(int status, const char *what) {
  if (status != P3MG_OK) {
    fprintf(stderr, "%s: %s\n", what, p3mg_strerror(status));
    exit(126);
  }
}

static data_t *init_gpu(int id, system_t *s, parameters_t *p) {
  data_t *d = (data_t *)Init_array(1, sizeof(data_t));
  p3mg_ctx *ctx = NULL;
  check(p3mg_create(&ctx, id, p->mesh, p->cao, P3M_BRILLOUIN, gpu_precision), "p3mg_create");
  check(p3mg_set_system(ctx, s->nparticles, s->p->x, s->p->y, s->p->z, s->q, s->length), "p3mg_set_system");
  d->mesh = p->mesh;
  d->method_data = ctx;
  return d;
}

static data_t *init_ik(system_t *s, parameters_t *p) { return init_gpu(METHOD_P3M_ik, s, p); }
static data_t *init_ik_i(system_t *s, parameters_t *p) { return init_gpu(METHOD_P3M_ik_i, s, p); }
static data_t *init_ad(system_t *s, parameters_t *p) { return init_gpu(METHOD_P3M_ad, s, p); }
static data_t *init_ad_i(system_t *s, parameters_t *p) { return init_gpu(METHOD_P3M_ad_i, s, p); }
static data_t *init_ik_r(system_t *s, parameters_t *p) { return init_gpu(METHOD_P3M_ik_r, s, p); }
static data_t *init_ad_r(system_t *s, parameters_t *p) { return init_gpu(METHOD_P3M_ad_r, s, p); }

static void influence_gpu(system_t *s, parameters_t *p, data_t *d) {
  (void)s;
  check(p3mg_influence((p3mg_ctx *)d->method_data, p->alpha), "p3mg_influence");
}

static void kspace_gpu(system_t *s, parameters_t *p, data_t *d, forces_t *f) {
  p3mg_ctx *ctx = (p3mg_ctx *)d->method_data;
  (void)p;
  check(p3mg_set_system(ctx, s->nparticles, s->p->x, s->p->y, s->p->z, s->q, s->length), "p3mg_set_system");
  check(p3mg_kspace_forces(ctx, f->f_k->x, f->f_k->y, f->f_k->z, f->f->x, f->f->y, f->f->z), "p3mg_kspace_forces");
}

void p3m_gpu_free_data(data_t *d) {
  if (!d) return;
  if (d->method_data) p3mg_destroy((p3mg_ctx *)d->method_data);
  free(d);
}

const method_t method_p3m_ik_gpu = {METHOD_P3M_ik, "P3M with ik differentiation, not interlaced (B200).",
                                    "p3m-ik-gpu", METHOD_FLAG_P3M | METHOD_FLAG_ik,
                                    &init_ik, &influence_gpu, &kspace_gpu, &Error_ik, &Error_ik_k};
const method_t method_p3m_ik_i_gpu = {METHOD_P3M_ik_i, "P3M with ik differentiation, interlaced (B200).",
                                      "p3m-ik-i-gpu", METHOD_FLAG_P3M | METHOD_FLAG_ik | METHOD_FLAG_interlaced,
                                      &init_ik_i, &influence_gpu, &kspace_gpu, &Error_ik_i,
                                      &p3m_k_space_error_ik_i};
const method_t method_p3m_ad_gpu = {METHOD_P3M_ad, "P3M with analytic differentiation, not interlaced (B200).",
                                    "p3m-ad-gpu", METHOD_FLAG_P3M | METHOD_FLAG_ad |
                                    METHOD_FLAG_self_force_correction,
                                    &init_ad, &influence_gpu, &kspace_gpu, &Error_ad, &p3m_k_space_error_ad};
const method_t method_p3m_ad_i_gpu = {METHOD_P3M_ad_i, "P3M with analytic differentiation, interlaced (B200).",
                                      "p3m-ad-i-gpu", METHOD_FLAG_P3M | METHOD_FLAG_ad | METHOD_FLAG_interlaced,
                                      &init_ad_i, &influence_gpu, &kspace_gpu, &Error_ad_i,
                                      &p3m_k_space_error_ad_i};
const method_t method_p3m_ik_r_gpu = {METHOD_P3M_ik_r, "P3M with ik differentiation, real input (B200).",
                                      "p3m-ik-r-gpu", METHOD_FLAG_P3M | METHOD_FLAG_ik,
                                      &init_ik_r, &influence_gpu, &kspace_gpu, &Error_ik, &Error_ik_k};
const method_t method_p3m_ad_r_gpu = {METHOD_P3M_ad_r, "P3M with analytic differentiation, real input (B200).",
                                      "p3m-ad-r-gpu", METHOD_FLAG_P3M | METHOD_FLAG_ad |
                                      METHOD_FLAG_self_force_correction,
                                      &init_ad_r, &influence_gpu, &kspace_gpu, &Error_ad, &p3m_k_space_error_ad};
