/* Test infrastructure: CPU discrete Fourier transform used by the P3M oracle
 * and by the FFTW-API shim that lets the reference build here.
 *
 * FFTW3 (version unpinned: the reference links -lfftw3 from a private path,
 * Makefile:6) is not present in this image.  The reference only relies on the
 * published definition of the transforms it plans (types.h:61-69):
 *   forward  X[k] = sum_j x[j] exp(-2 pi i j.k / n)   (FFTW_FORWARD = -1)
 *   backward x[j] = sum_k X[k] exp(+2 pi i j.k / n)   (FFTW_BACKWARD = +1)
 * unnormalised, row-major, last index fastest, plus the real-input (r2c) and
 * Hermitian-input (c2r) forms with the last dimension halved to n/2+1.
 * This file restates that definition with a mixed-radix Cooley-Tukey
 * decomposition (radix = prime factors of n, generic DFT for any prime).
 * It is checked against numpy.fft in tests/test_oracle_dft.py.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use it.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "dft.h"

typedef struct {
  int n;
  int sign;
  int nfac;
  int fac[64];
  double *w; /* w[2e], w[2e+1] = cos, sin of sign*2*pi*e/n */
  double *tmp;
} line_plan;

static void factorize(int n, int *fac, int *nfac) {
  int k = 0;
  /* prefer larger radices first for fewer passes */
  const int pref[] = {4, 2, 3, 5, 7};
  int m = n;
  for (int pi = 0; pi < 5; pi++) {
    int p = pref[pi];
    while (m % p == 0 && m > 1) {
      fac[k++] = p;
      m /= p;
    }
  }
  for (int p = 11; m > 1; p += 2) {
    while (m % p == 0) {
      fac[k++] = p;
      m /= p;
    }
    if ((long)p * p > m && m > 1) {
      fac[k++] = m;
      m = 1;
    }
  }
  *nfac = k;
}

static line_plan *line_plan_new(int n, int sign) {
  line_plan *lp = (line_plan *)calloc(1, sizeof(line_plan));
  lp->n = n;
  lp->sign = sign;
  factorize(n, lp->fac, &lp->nfac);
  lp->w = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  for (int e = 0; e < n; e++) {
    /* angle reduced to [0, 2pi) exactly in integers before scaling */
    long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)e / (long double)n;
    lp->w[2 * e] = (double)cosl(a);
    lp->w[2 * e + 1] = (double)(sign * sinl(a));
  }
  lp->tmp = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  return lp;
}

static void line_plan_free(line_plan *lp) {
  if (!lp) return;
  free(lp->w);
  free(lp->tmp);
  free(lp);
}

/* out[0..n) = DFT of in[0], in[s], in[2s], ... ; n = product of fac[0..nf) */
static void rec(const line_plan *lp, const double *in, long s, double *out, int n, const int *fac, int nf,
                long wstep) {
  if (n == 1) {
    out[0] = in[0];
    out[1] = in[1];
    return;
  }
  const int p = fac[0];
  const int m = n / p;
  for (int r = 0; r < p; r++) rec(lp, in + 2 * r * s, s * p, out + 2 * (long)r * m, m, fac + 1, nf - 1, wstep * p);
  /* butterflies: X[k + q m] = sum_r W_n^{r(k+qm)} Y_r[k] ; W_n^e = w[e*wstep mod N] */
  const long N = lp->n;
  double t[2 * 64];
  double *tv = (p <= 64) ? t : (double *)malloc(sizeof(double) * 2 * p);
  for (int k = 0; k < m; k++) {
    for (int r = 0; r < p; r++) {
      const double *y = out + 2 * ((long)r * m + k);
      long e = ((long)r * k * wstep) % N;
      double c = lp->w[2 * e], sn = lp->w[2 * e + 1];
      tv[2 * r] = y[0] * c - y[1] * sn;
      tv[2 * r + 1] = y[0] * sn + y[1] * c;
    }
    for (int q = 0; q < p; q++) {
      double re = 0.0, im = 0.0;
      for (int r = 0; r < p; r++) {
        long e = ((long)r * q * m * wstep) % N;
        double c = lp->w[2 * e], sn = lp->w[2 * e + 1];
        re += tv[2 * r] * c - tv[2 * r + 1] * sn;
        im += tv[2 * r] * sn + tv[2 * r + 1] * c;
      }
      double *x = out + 2 * ((long)q * m + k);
      x[0] = re;
      x[1] = im;
    }
  }
  if (tv != t) free(tv);
}

static void line_exec(line_plan *lp, double *data, long stride) {
  /* gather, transform, scatter */
  const int n = lp->n;
  double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)n);
  for (int j = 0; j < n; j++) {
    buf[2 * j] = data[2 * j * stride];
    buf[2 * j + 1] = data[2 * j * stride + 1];
  }
  rec(lp, buf, 1, lp->tmp, n, lp->fac, lp->nfac, 1);
  for (int j = 0; j < n; j++) {
    data[2 * j * stride] = lp->tmp[2 * j];
    data[2 * j * stride + 1] = lp->tmp[2 * j + 1];
  }
  free(buf);
}

void oracle_dft_1d(double *data, int n, long stride, int sign) {
  line_plan *lp = line_plan_new(n, sign);
  line_exec(lp, data, stride);
  line_plan_free(lp);
}

/* In-place complex transform of an array with dims[0..rank), last fastest. */
void oracle_dft_nd(double *data, int rank, const int *dims, int sign) {
  long total = 1;
  for (int d = 0; d < rank; d++) total *= dims[d];
  for (int d = 0; d < rank; d++) {
    long stride = 1;
    for (int e = d + 1; e < rank; e++) stride *= dims[e];
    long outer = total / (stride * dims[d]);
    line_plan *lp = line_plan_new(dims[d], sign);
    for (long o = 0; o < outer; o++)
      for (long i = 0; i < stride; i++) line_exec(lp, data + 2 * (o * stride * dims[d] + i), stride);
    line_plan_free(lp);
  }
}

/* Real input (n0 x n1 x n2, row stride in_row doubles) -> half spectrum
 * (n0 x n1 x (n2/2+1) complex, row stride out_row complex). */
void oracle_dft_r2c_3d(const double *in, long in_row, double *out, long out_row, int n0, int n1, int n2) {
  const int h = n2 / 2 + 1;
  double *full = (double *)malloc(sizeof(double) * 2 * (size_t)n0 * n1 * n2);
  for (long a = 0; a < (long)n0 * n1; a++)
    for (int k = 0; k < n2; k++) {
      full[2 * (a * n2 + k)] = in[a * in_row + k];
      full[2 * (a * n2 + k) + 1] = 0.0;
    }
  int dims[3] = {n0, n1, n2};
  oracle_dft_nd(full, 3, dims, -1);
  /* copy via a temporary so in == out (in-place padded layout) is allowed */
  for (long a = 0; a < (long)n0 * n1; a++)
    for (int k = 0; k < h; k++) {
      out[2 * (a * out_row + k)] = full[2 * (a * n2 + k)];
      out[2 * (a * out_row + k) + 1] = full[2 * (a * n2 + k) + 1];
    }
  free(full);
}

/* Half spectrum -> real output.  The first two dimensions are transformed
 * as complex data; each last-dimension row is then treated as Hermitian:
 * the imaginary parts of its k=0 and k=n2/2 entries are ignored and the
 * remaining entries are mirrored, which is the documented c2r semantics. */
void oracle_dft_c2r_3d(const double *in, long in_row, double *out, long out_row, int n0, int n1, int n2) {
  const int h = n2 / 2 + 1;
  double *half = (double *)malloc(sizeof(double) * 2 * (size_t)n0 * n1 * h);
  for (long a = 0; a < (long)n0 * n1; a++)
    for (int k = 0; k < h; k++) {
      half[2 * (a * h + k)] = in[2 * (a * in_row + k)];
      half[2 * (a * h + k) + 1] = in[2 * (a * in_row + k) + 1];
    }
  /* complex backward transforms along dims 0 and 1 for every k2 */
  for (int d = 0; d < 2; d++) {
    int n = d == 0 ? n0 : n1;
    long stride = d == 0 ? (long)n1 * h : h;
    long outer = d == 0 ? 1 : n0;
    long inner = stride;
    line_plan *lp = line_plan_new(n, +1);
    for (long o = 0; o < outer; o++)
      for (long i = 0; i < inner; i++) line_exec(lp, half + 2 * (o * (long)n * stride + i), stride);
    line_plan_free(lp);
  }
  line_plan *lp = line_plan_new(n2, +1);
  double *row = (double *)malloc(sizeof(double) * 2 * (size_t)n2);
  for (long a = 0; a < (long)n0 * n1; a++) {
    const double *hr = half + 2 * a * h;
    for (int k = 0; k < h; k++) {
      row[2 * k] = hr[2 * k];
      row[2 * k + 1] = hr[2 * k + 1];
    }
    row[1] = 0.0;
    if (n2 % 2 == 0) row[2 * (n2 / 2) + 1] = 0.0;
    for (int k = 1; k < (n2 + 1) / 2; k++) {
      row[2 * (n2 - k)] = hr[2 * k];
      row[2 * (n2 - k) + 1] = -hr[2 * k + 1];
    }
    line_exec(lp, row, 1);
    for (int k = 0; k < n2; k++) out[a * out_row + k] = row[2 * k];
  }
  free(row);
  line_plan_free(lp);
  free(half);
}
