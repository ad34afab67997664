/* Test infrastructure: the reference's own driver step (Init at alpha 0 as
 * main.c:191 does, Influence_function, Calculate_forces of common.c:268-327)
 * run through either its CPU method table or the p3mg-backed table of
 * p3m-standalone_b200/binding/p3m-gpu.c, so a test can show that the
 * reference program computes the same forces with the GPU plugin.  Built
 * by build_ref.sh into oracle/_ref/libp3mref_gpu.so, never shipped. */
#include <stdlib.h>
#include <string.h>

#include "types.h"
#include "common.h"
#include "p3m-common.h"
#include "p3m-ik.h"
#include "p3m-ik-i.h"
#include "p3m-ad.h"
#include "p3m-ad-i.h"
#include "p3m-ik-real.h"
#include "p3m-ad-real.h"
#include "p3m-gpu.h"

static const method_t *table(int gpu, int id) {
  switch (id) {
    case 0: return gpu ? &method_p3m_ik_gpu : &method_p3m_ik;
    case 1: return gpu ? &method_p3m_ik_i_gpu : &method_p3m_ik_i;
    case 2: return gpu ? &method_p3m_ad_gpu : &method_p3m_ad;
    case 3: return gpu ? &method_p3m_ad_i_gpu : &method_p3m_ad_i;
    case 6: return gpu ? &method_p3m_ik_r_gpu : &method_p3m_ik_r;
    case 7: return gpu ? &method_p3m_ad_r_gpu : &method_p3m_ad_r;
  }
  return NULL;
}

/* f, fk, fr: 3n doubles each (x block, y block, z block). */
int ref_binding_forces(int gpu, int precision, int method_id, int mesh, int cao, int mc, double alpha, double rcut,
                       int n, const double *x, const double *y, const double *z, const double *q, double L,
                       double *f, double *fk, double *fr, double *energy) {
  const method_t *m = table(gpu, method_id);
  if (!m) return -1;
  P3M_BRILLOUIN = mc;
  p3m_gpu_set_precision(precision);
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
  s->energy = 0.0;
  Calculate_forces(m, s, &p, d, fo);
  for (int c = 0; c < 3; c++) {
    memcpy(f + (size_t)c * n, fo->f->fields[c], sizeof(double) * n);
    memcpy(fk + (size_t)c * n, fo->f_k->fields[c], sizeof(double) * n);
    memcpy(fr + (size_t)c * n, fo->f_r->fields[c], sizeof(double) * n);
  }
  *energy = s->energy;
  if (gpu)
    p3m_gpu_free_data(d);
  else
    Free_data(d);
  Free_forces(fo);
  Free_system(s);
  return 0;
}
