/* Test infrastructure: FFTW3 API subset implemented with the oracle DFT.
 * In-place r2c/c2r plans use FFTW's padded real layout (last dimension
 * 2*(n2/2+1) doubles); out-of-place plans use the dense n2-wide rows. */
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"
#include "../dft.h"

enum { P_C2C_1D, P_C2C_3D, P_R2C_3D, P_C2R_3D };

struct oracle_fftw_plan_s {
  int kind;
  int n0, n1, n2;
  int sign;
  void *in;
  void *out;
};

void *fftw_malloc(size_t n) { return malloc(n ? n : 1); }
void fftw_free(void *p) { free(p); }

static fftw_plan mk(int kind, int n0, int n1, int n2, int sign, void *in, void *out) {
  fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
  p->kind = kind;
  p->n0 = n0;
  p->n1 = n1;
  p->n2 = n2;
  p->sign = sign;
  p->in = in;
  p->out = out;
  return p;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
  (void)flags;
  return mk(P_C2C_1D, n, 1, 1, sign, in, out);
}
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
  (void)flags;
  return mk(P_C2C_3D, n0, n1, n2, sign, in, out);
}
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags) {
  (void)flags;
  return mk(P_R2C_3D, n0, n1, n2, -1, in, out);
}
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags) {
  (void)flags;
  return mk(P_C2R_3D, n0, n1, n2, +1, in, out);
}

void fftw_execute(const fftw_plan p) {
  const long h = p->n2 / 2 + 1;
  switch (p->kind) {
    case P_C2C_1D:
    case P_C2C_3D: {
      long total = (long)p->n0 * p->n1 * p->n2;
      if (p->in != p->out) memcpy(p->out, p->in, sizeof(double) * 2 * total);
      if (p->kind == P_C2C_1D)
        oracle_dft_1d((double *)p->out, p->n0, 1, p->sign);
      else {
        int dims[3] = {p->n0, p->n1, p->n2};
        oracle_dft_nd((double *)p->out, 3, dims, p->sign);
      }
      break;
    }
    case P_R2C_3D: {
      long in_row = (p->in == p->out) ? 2 * h : p->n2;
      oracle_dft_r2c_3d((const double *)p->in, in_row, (double *)p->out, h, p->n0, p->n1, p->n2);
      break;
    }
    case P_C2R_3D: {
      long out_row = (p->in == p->out) ? 2 * h : p->n2;
      oracle_dft_c2r_3d((const double *)p->in, h, (double *)p->out, out_row, p->n0, p->n1, p->n2);
      break;
    }
  }
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
