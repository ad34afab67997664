/* ORACLE — test infrastructure only.  A plain-C, single-threaded CPU
 * restatement of the reference's P3M force path, used as the checker by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg.  It is
 * never called by the product path.
 *
 * Pinned against the reference itself: tests/test_oracle_vs_ref.py runs the
 * reference compiled from its own sources (oracle/build_ref.sh) on the same
 * inputs and requires agreement to 1e-12 relative RMS, and the committed
 * golden fixtures under tests/golden/ hold reference outputs.
 *
 * Array convention: a "3n" force array holds the x block, then the y block,
 * then the z block (the reference's SoA vector_array_t, types.h:126-132).
 * Every force routine ACCUMULATES (+=) like the reference's Kspace_force.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "dft.h"
#include "p3m_oracle.h"

#define ORC_PI 3.1415926535897932384626433832795028841971693993751058209749445923078164062
#define SQ(a) ((a) * (a))

/* ---------------------------------------------------------------- helpers */

/* integer power by repeated multiplication (common.h:21-29 my_power) */
static double ipow(double b, int e) {
  double r = 1.0;
  while (e-- > 0) r *= b;
  return r;
}

/* sin(pi d)/(pi d) with the value 1 at d == 0 (p3m-common.c:71-75) */
static double sinc_pi(double d) {
  double a = ORC_PI * d;
  return d == 0.0 ? 1.0 : sin(a) / a;
}

/* wrap an index that is at most one period outside [0, m) (charge-assign.c:37-40) */
static int wrap1(int i, int m) { return i + (i < 0) * m - (i >= m) * m; }

/* signed frequency of index i: i - round(i/m) m, C round() = half away from
 * zero, so index m/2 maps to -m/2 (p3m-common.c:133-143) */
static double signed_freq(int i, int m) { return (double)i - round((double)i / (double)m) * (double)m; }

/* Cardinal B-spline weights of order cao at in-cell offset x in [-0.5, 0.5):
 * w[j] = W_j(x), dw[j] = dW_j/dx for stencil points j = 0..cao-1.
 * W_j(x) = M_cao(x + 1/2 + cao-1-j), M_n the uncentred cardinal B-spline on
 * [0, n], evaluated with the two-term recursion
 *   M_n(u) = [u M_{n-1}(u) + (n-u) M_{n-1}(u-1)] / (n-1)
 * and M_n'(u) = M_{n-1}(u) - M_{n-1}(u-1) (de Boor; Essmann et al. 1995).
 * These are the polynomials the reference tabulates (window-functions.c:
 * 46-183 caf_bspline / caf_bspline_d).  For cao = 1 the derivative is 0,
 * as in the reference's fall-through (window-functions.c:100-103). */
void oracle_bspline(int cao, double x, double *w, double *dw) {
  const double u = x + 0.5;
  double a[8] = {1.0, 0, 0, 0, 0, 0, 0, 0}, prev[8] = {0};
  for (int n = 2; n <= cao; n++) {
    memcpy(prev, a, sizeof(a));
    for (int k = 0; k < n; k++) {
      double lo = (k < n - 1) ? prev[k] : 0.0;
      double hi = (k > 0) ? prev[k - 1] : 0.0;
      a[k] = ((u + k) * lo + ((double)n - u - k) * hi) / (double)(n - 1);
    }
  }
  for (int j = 0; j < cao; j++) {
    int k = cao - 1 - j;
    w[j] = a[k];
    if (dw) dw[j] = (cao == 1) ? 0.0 : (prev[k] - (k > 0 ? prev[k - 1] : 0.0));
  }
}

/* Geometry of one coordinate (charge-assign.c:148-157):
 *   pos = x*Hi - shift + 0.5*ii, nmp = floor(pos + 0.5), base = wrap(nmp),
 *   arg = floor((pos - nmp + 0.5) * 131072) ; the weights are evaluated at the
 * tabulated offset (arg - 65536)/131072 (interpol.c:56-61, MaxInterpol 65536). */
static void geometry(double xc, double Hi, double shift, int ii, int m, int *base, double *xq) {
  double pos = xc * Hi - shift + 0.5 * ii;
  int nmp = (int)floor(pos + 0.5);
  *base = wrap1(nmp, m);
  int arg = (int)floor((pos - nmp + 0.5) * 131072.0);
  *xq = (double)(arg - 65536) / 131072.0;
}

static int is_interlaced(int method) { return method == 1 || method == 3; }
static int is_ad(int method) { return method == 2 || method == 3 || method == 7; }
static int is_r2c(int method) { return method == 6 || method == 7; }

/* ------------------------------------------------------ influence functions */

/* ik / ik-r: p3m-ik.c:93-173 */
static double G_ik(int NX, int NY, int NZ, int m, int cao, int mc, double alpha, double L) {
  const double Leni = 1.0 / L, fak1 = 1.0 / (double)m, fak2 = SQ(ORC_PI / alpha);
  const double nx = signed_freq(NX, m), ny = signed_freq(NY, m), nz = signed_freq(NZ, m);
  double Z[3] = {0, 0, 0}, N1 = 0.0;
  for (int MX = -mc; MX <= mc; MX++) {
    double NMX = nx + m * MX;
    double S1 = ipow(ipow(sinc_pi(fak1 * NMX), cao), 2);
    for (int MY = -mc; MY <= mc; MY++) {
      double NMY = ny + m * MY;
      double S2 = S1 * ipow(ipow(sinc_pi(fak1 * NMY), cao), 2);
      for (int MZ = -mc; MZ <= mc; MZ++) {
        double NMZ = nz + m * MZ;
        double S3 = S2 * ipow(ipow(sinc_pi(fak1 * NMZ), cao), 2);
        double NM2 = SQ(NMX * Leni) + SQ(NMY * Leni) + SQ(NMZ * Leni);
        N1 += S3;
        double zwi = S3 * exp(-fak2 * NM2) / NM2;
        Z[0] += NMX * zwi * Leni;
        Z[1] += NMY * zwi * Leni;
        Z[2] += NMZ * zwi * Leni;
      }
    }
  }
  /* the differential operator: signed frequency with the Nyquist entry 0 */
  double D[3] = {nx, ny, nz};
  int I[3] = {NX, NY, NZ};
  for (int d = 0; d < 3; d++)
    if (I[d] == m / 2) D[d] = 0.0; /* Dn[mesh/2] = 0 (p3m-common.c:130) */
  double num = D[0] * Z[0] * Leni + D[1] * Z[1] * Leni + D[2] * Z[2] * Leni;
  num /= (SQ(D[0] * Leni) + SQ(D[1] * Leni) + SQ(D[2] * Leni)) * SQ(N1);
  return 2.0 * num / ORC_PI;
}

/* ik interlaced: p3m-ik-i.c:78-166 */
static double G_ik_i(int NX, int NY, int NZ, int m, int cao, int mc, double alpha, double L) {
  const double Leni = 1.0 / L, fak1 = 1.0 / (double)m, fak2 = SQ(ORC_PI / alpha);
  const double nx = signed_freq(NX, m), ny = signed_freq(NY, m), nz = signed_freq(NZ, m);
  double Z[3] = {0, 0, 0}, N1 = 0.0, N2 = 0.0;
  for (int MX = -mc; MX <= mc; MX++) {
    double NMX = nx + m * MX;
    double S1 = ipow(sinc_pi(fak1 * NMX), 2 * cao);
    for (int MY = -mc; MY <= mc; MY++) {
      double NMY = ny + m * MY;
      double S2 = S1 * ipow(sinc_pi(fak1 * NMY), 2 * cao);
      for (int MZ = -mc; MZ <= mc; MZ++) {
        double NMZ = nz + m * MZ;
        double S3 = S2 * ipow(sinc_pi(fak1 * NMZ), 2 * cao);
        double NM2 = SQ(NMX * Leni) + SQ(NMY * Leni) + SQ(NMZ * Leni);
        N1 += S3;
        double zwi = S3 * exp(-fak2 * NM2) / NM2;
        Z[0] += NMX * zwi * Leni;
        Z[1] += NMY * zwi * Leni;
        Z[2] += NMZ * zwi * Leni;
        if (((MX + MY + MZ) % 2) == 0)
          N2 += S3;
        else
          N2 -= S3;
      }
    }
  }
  double D[3] = {nx, ny, nz};
  int I[3] = {NX, NY, NZ};
  for (int d = 0; d < 3; d++)
    if (I[d] == m / 2) D[d] = 0.0; /* Dn[mesh/2] = 0 (p3m-common.c:130) */
  double num = D[0] * Z[0] * Leni + D[1] * Z[1] * Leni + D[2] * Z[2] * Leni;
  num /= (SQ(D[0] * Leni) + SQ(D[1] * Leni) + SQ(D[2] * Leni));
  num /= 0.5 * (SQ(N1) + SQ(N2));
  return 2.0 * num / ORC_PI;
}

/* ad / ad-r: p3m-ad.c:69-158 ; ad interlaced: p3m-ad-i.c:70-150 */
static double G_ad(int NX, int NY, int NZ, int m, int cao, int mc, double alpha, double L, int interlaced) {
  const double Leni = 1.0 / L, fak1 = 1.0 / (double)m, fak2 = SQ(ORC_PI / alpha);
  const double nx = signed_freq(NX, m), ny = signed_freq(NY, m), nz = signed_freq(NZ, m);
  double Z = 0, N1 = 0, N2 = 0, N3 = 0, N4 = 0;
  for (int MX = -mc; MX <= mc; MX++) {
    double NMX = nx + m * MX;
    double S1 = ipow(sinc_pi(fak1 * NMX), 2 * cao);
    for (int MY = -mc; MY <= mc; MY++) {
      double NMY = ny + m * MY;
      double S2 = S1 * ipow(sinc_pi(fak1 * NMY), 2 * cao);
      for (int MZ = -mc; MZ <= mc; MZ++) {
        double NMZ = nz + m * MZ;
        double S3 = S2 * ipow(sinc_pi(fak1 * NMZ), 2 * cao);
        double NM2 = SQ(NMX * Leni) + SQ(NMY * Leni) + SQ(NMZ * Leni);
        N1 += S3;
        N2 += S3 * NM2;
        if (((MX + MY + MZ) % 2) == 0) {
          N3 += S3;
          N4 += S3 * NM2;
        } else {
          N3 -= S3;
          N4 -= S3 * NM2;
        }
        Z += S3 * exp(-fak2 * NM2);
      }
    }
  }
  if (interlaced) return Z / (0.5 * ORC_PI * (N1 * N2 + N3 * N4));
  return Z / (ORC_PI * N1 * N2);
}

int oracle_influence(int method, int m, int cao, int mc, double alpha, double L, double *G) {
  if (m < 2 || cao < 1 || cao > 7) return -1;
  const int half = m / 2;
  for (int NX = 0; NX < m; NX++)
    for (int NY = 0; NY < m; NY++)
      for (int NZ = 0; NZ < m; NZ++) {
        size_t ind = ((size_t)NX * m + NY) * m + NZ;
        double g;
        if (NX == 0 && NY == 0 && NZ == 0)
          g = 0.0;
        else if (is_ad(method)) {
          if (alpha == 0.0)
            g = 0.0; /* p3m-ad.c:120-123 (the ad-i path has no such guard) */
          else
            g = G_ad(NX, NY, NZ, m, cao, mc, alpha, L, method == 3);
        } else if (NX % half == 0 && NY % half == 0 && NZ % half == 0)
          g = 0.0; /* ik zeroes every k with all indices = 0 mod m/2 */
        else if (method == 1)
          g = G_ik_i(NX, NY, NZ, m, cao, mc, alpha, L);
        else
          g = G_ik(NX, NY, NZ, m, cao, mc, alpha, L);
        G[ind] = g;
      }
  return 0;
}

/* ad self-force coefficients b(m') for m' in {-1,0,1}^3 (81 doubles,
 * p3m-ad-self-forces.c:30-112): for direction d with m'_d != 0
 *   b_d(m') = pi m'_d mesh / L^4 * sum_{k: G(k)!=0} sum_{|a|<=1} G(k) U(k+a m) U(k+(a+m') m)
 * with U(k) = prod_d sinc(k_d/m)^cao.  The k-integers are the signed
 * frequencies (truncated to int like the reference). */
int oracle_self_force_coeffs(int m, int cao, double L, const double *G, double *b81) {
  const double mi = 1.0 / m;
  int ind = 0;
  for (int a0 = -1; a0 <= 1; a0++)
    for (int a1 = -1; a1 <= 1; a1++)
      for (int a2 = -1; a2 <= 1; a2++) {
        int mm[3] = {a0, a1, a2};
        for (int dir = 0; dir < 3; dir++) {
          if (mm[dir] == 0) {
            b81[ind++] = 0.0;
            continue;
          }
          double sum = 0.0;
          for (int nx = 0; nx < m; nx++)
            for (int ny = 0; ny < m; ny++)
              for (int nz = 0; nz < m; nz++) {
                double g = G[((size_t)nx * m + ny) * m + nz];
                if (g == 0.0) continue;
                int tx = (int)signed_freq(nx, m), ty = (int)signed_freq(ny, m), tz = (int)signed_freq(nz, m);
                for (int bx = -1; bx <= 1; bx++)
                  for (int by = -1; by <= 1; by++)
                    for (int bz = -1; bz <= 1; bz++) {
                      double U = pow(sinc_pi(mi * (tx + bx * m)) * sinc_pi(mi * (ty + by * m)) *
                                         sinc_pi(mi * (tz + bz * m)),
                                     cao);
                      double Us = pow(sinc_pi(mi * (tx + (bx + a0) * m)) * sinc_pi(mi * (ty + (by + a1) * m)) *
                                          sinc_pi(mi * (tz + (bz + a2) * m)),
                                      cao);
                      sum += g * U * Us;
                    }
              }
          b81[ind++] = (ORC_PI * mm[dir] * m) / SQ(SQ(L)) * sum;
        }
      }
  return 0;
}

/* ------------------------------------------------------------- k-space */

typedef struct {
  int base[3];
  double w[3][7];
  double dw[3][7];
} stencil_t;

static void make_stencil(const double *x, const double *y, const double *z, int i, double Hi, double shift, int ii,
                         int m, int cao, stencil_t *st) {
  const double c[3] = {x[i], y[i], z[i]};
  for (int d = 0; d < 3; d++) {
    double xq;
    geometry(c[d], Hi, shift, ii, m, &st->base[d], &xq);
    oracle_bspline(cao, xq, st->w[d], st->dw[d]);
  }
}

/* complex mesh index (interleaved re/im, p3m-common.h:26) */
static size_t cidx(int i, int j, int k, int m) { return 2 * (((size_t)i * m + j) * m + k); }

int oracle_kspace(int method, int m, int cao, int mc, double alpha, int n, const double *x, const double *y,
                  const double *z, const double *q, double L, const double *Gin, double *fk, double *ftot) {
  if (m < 2 || cao < 1 || cao > 7 || n < 0) return -1;
  if (!(method == 0 || method == 1 || method == 2 || method == 3 || method == 6 || method == 7)) return -2;
  const size_t M = (size_t)m * m * m;
  double *G = (double *)Gin;
  if (!G) {
    G = (double *)malloc(sizeof(double) * M);
    oracle_influence(method, m, cao, mc, alpha, L, G);
  }
  const double Hi = (double)m / L, Leni = 1.0 / L;
  const double shift = (double)((cao - 1) / 2);
  const int nmesh = is_interlaced(method) ? 2 : 1;
  double *Q = (double *)calloc(2 * M, sizeof(double));
  stencil_t st;

  /* charge assignment: mesh ii in the re (ii=0) or im (ii=1) slot */
  for (int ii = 0; ii < nmesh; ii++)
    for (int p = 0; p < n; p++) {
      make_stencil(x, y, z, p, Hi, shift, ii, m, cao, &st);
      for (int a = 0; a < cao; a++) {
        int I = wrap1(st.base[0] + a, m);
        for (int b = 0; b < cao; b++) {
          int J = wrap1(st.base[1] + b, m);
          for (int c = 0; c < cao; c++) {
            int K = wrap1(st.base[2] + c, m);
            Q[cidx(I, J, K, m) + ii] += q[p] * st.w[0][a] * st.w[1][b] * st.w[2][c];
          }
        }
      }
    }

  /* forward transform (sign -1).  r2c methods transform the real mesh with
   * the half-spectrum routine; that equals the c2c result on k_z <= m/2. */
  int dims[3] = {m, m, m};
  if (is_r2c(method)) {
    double *real = (double *)malloc(sizeof(double) * M);
    for (size_t t = 0; t < M; t++) real[t] = Q[2 * t];
    const int h = m / 2 + 1;
    double *half = (double *)malloc(sizeof(double) * 2 * (size_t)m * m * h);
    oracle_dft_r2c_3d(real, m, half, h, m, m, m);
    /* expand to the full spectrum by Hermitian symmetry for the shared code below */
    for (int i = 0; i < m; i++)
      for (int j = 0; j < m; j++)
        for (int k = 0; k < m; k++) {
          size_t o = cidx(i, j, k, m);
          if (k < h) {
            size_t s = 2 * (((size_t)i * m + j) * h + k);
            Q[o] = half[s];
            Q[o + 1] = half[s + 1];
          } else {
            int ci = (m - i) % m, cj = (m - j) % m, ck = m - k;
            size_t s = 2 * (((size_t)ci * m + cj) * h + ck);
            Q[o] = half[s];
            Q[o + 1] = -half[s + 1];
          }
        }
    free(real);
    free(half);
  } else
    oracle_dft_nd(Q, 3, dims, -1);

  if (!is_ad(method)) {
    /* ik: F_d(k) = i (2 pi / L) D(k_d) G(k) Q(k), three backward transforms */
    double *F[3];
    for (int d = 0; d < 3; d++) F[d] = (double *)malloc(sizeof(double) * 2 * M);
    for (int i = 0; i < m; i++)
      for (int j = 0; j < m; j++)
        for (int k = 0; k < m; k++) {
          size_t o = cidx(i, j, k, m);
          double g = G[((size_t)i * m + j) * m + k];
          double qr = Q[o] * g, qi = Q[o + 1] * g;
          int I3[3] = {i, j, k};
          for (int d = 0; d < 3; d++) {
            double D = (I3[d] == m / 2) ? 0.0 : signed_freq(I3[d], m);
            F[d][o] = -2.0 * ORC_PI * Leni * D * qi;
            F[d][o + 1] = 2.0 * ORC_PI * Leni * D * qr;
          }
        }
    for (int d = 0; d < 3; d++) oracle_dft_nd(F[d], 3, dims, +1);
    /* back-interpolation, prefactor 1/(2 L^3) (p3m-ik.c:242) ; interlaced
     * methods average the two meshes (charge-assign.c:646-725) */
    const double pref = 1.0 / (2.0 * L * L * L);
    for (int p = 0; p < n; p++) {
      double acc[3] = {0, 0, 0};
      for (int ii = 0; ii < nmesh; ii++) {
        make_stencil(x, y, z, p, Hi, shift, ii, m, cao, &st);
        double scale = (nmesh == 2) ? 0.5 * pref : pref;
        for (int a = 0; a < cao; a++) {
          int I = wrap1(st.base[0] + a, m);
          for (int b = 0; b < cao; b++) {
            int J = wrap1(st.base[1] + b, m);
            for (int c = 0; c < cao; c++) {
              int K = wrap1(st.base[2] + c, m);
              double B = scale * q[p] * st.w[0][a] * st.w[1][b] * st.w[2][c];
              size_t o = cidx(I, J, K, m) + ii;
              for (int d = 0; d < 3; d++) acc[d] -= F[d][o] * B;
            }
          }
        }
      }
      for (int d = 0; d < 3; d++) fk[(size_t)d * n + p] += acc[d];
    }
    for (int d = 0; d < 3; d++) free(F[d]);
  } else {
    /* ad: phi(k) = G(k) Q(k), one backward transform, gradient of the weights */
    for (size_t t = 0; t < M; t++) {
      Q[2 * t] *= G[t];
      Q[2 * t + 1] *= G[t];
    }
    oracle_dft_nd(Q, 3, dims, +1);
    const double pref = (double)m * Leni * Leni * Leni; /* p3m-ad.c:202 */
    for (int p = 0; p < n; p++) {
      double acc[3] = {0, 0, 0};
      for (int ii = 0; ii < nmesh; ii++) {
        make_stencil(x, y, z, p, Hi, shift, ii, m, cao, &st);
        double scale = (nmesh == 2) ? 0.5 * pref : pref;
        double qL = q[p] * Leni;
        for (int a = 0; a < cao; a++) {
          int I = wrap1(st.base[0] + a, m);
          for (int b = 0; b < cao; b++) {
            int J = wrap1(st.base[1] + b, m);
            for (int c = 0; c < cao; c++) {
              int K = wrap1(st.base[2] + c, m);
              double phi = Q[cidx(I, J, K, m) + ii];
              acc[0] -= scale * phi * st.dw[0][a] * st.w[1][b] * st.w[2][c] * qL;
              acc[1] -= scale * phi * st.w[0][a] * st.dw[1][b] * st.w[2][c] * qL;
              acc[2] -= scale * phi * st.w[0][a] * st.w[1][b] * st.dw[2][c] * qL;
            }
          }
        }
      }
      for (int d = 0; d < 3; d++) fk[(size_t)d * n + p] += acc[d];
    }
    /* self-force correction, methods 2 and 7 only, into the TOTAL force
     * (p3m-ad.c:204-206, p3m-ad-real.c:112-114, p3m-ad-self-forces.c:114-139) */
    if ((method == 2 || method == 7) && ftot) {
      double b[81];
      oracle_self_force_coeffs(m, cao, L, G, b);
      const double h = L / m;
      for (int p = 0; p < n; p++) {
        int t = 0;
        for (int a0 = -1; a0 <= 1; a0++)
          for (int a1 = -1; a1 <= 1; a1++)
            for (int a2 = -1; a2 <= 1; a2++) {
              double s = SQ(q[p]) * sin(2 * ORC_PI * (a0 * x[p] / h + a1 * y[p] / h + a2 * z[p] / h));
              for (int d = 0; d < 3; d++) ftot[(size_t)d * n + p] -= b[t++] * s;
            }
      }
    }
  }
  free(Q);
  if (G != Gin) free(G);
  return 0;
}

/* ---------------------------------------------------------- real space */

/* One ordered pair (realpart.c:137-165). */
static void pair_term(const double *x, const double *y, const double *z, const double *q, double L, double Li,
                      double rcut, double alpha, int t1, int t2, double *f3, double *energy) {
  const double wupi = 1.77245385090551602729816748334;
  double dx = x[t1] - x[t2];
  dx -= round(dx * Li) * L;
  double dy = y[t1] - y[t2];
  dy -= round(dy * Li) * L;
  double dz = z[t1] - z[t2];
  dz -= round(dz * Li) * L;
  double r = sqrt(dx * dx + dy * dy + dz * dz);
  if (r <= rcut) {
    double ar = alpha * r;
    double e = erfc(ar);
    double fak = q[t1] * q[t2] * (e / r + (2.0 * alpha / wupi) * exp(-ar * ar)) / SQ(r);
    f3[0] += fak * dx;
    f3[1] += fak * dy;
    f3[2] += fak * dz;
    *energy += 0.5 * q[t1] * q[t2] * e / r;
  }
}

/* Real-space erfc forces accumulated into fr (3n).  cells != 0 restricts the
 * candidate pairs with a cell list of side >= rcut (same pair set as the
 * reference's all-pairs loop when there are >= 3 cells per side; otherwise
 * the all-pairs loop runs). */
int oracle_realspace(int n, const double *x, const double *y, const double *z, const double *q, double L, double rcut,
                     double alpha, double *fr, double *energy, int cells) {
  const double Li = 1.0 / L;
  double en = 0.0;
  int nc = (int)floor(L / rcut);
  if (!cells || nc < 3 || rcut <= 0.0) {
    for (int t1 = 0; t1 < n; t1++) {
      double f3[3] = {0, 0, 0};
      for (int t2 = 0; t2 < n; t2++)
        if (t1 != t2) pair_term(x, y, z, q, L, Li, rcut, alpha, t1, t2, f3, &en);
      for (int d = 0; d < 3; d++) fr[(size_t)d * n + t1] += f3[d];
    }
  } else {
    if (nc > 512) nc = 512;
    const size_t ncell = (size_t)nc * nc * nc;
    int *head = (int *)malloc(sizeof(int) * ncell);
    int *next = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (size_t c = 0; c < ncell; c++) head[c] = -1;
    int *cid = (int *)malloc(sizeof(int) * 3 * (size_t)(n > 0 ? n : 1));
    for (int i = n - 1; i >= 0; i--) {
      int c3[3];
      const double cc[3] = {x[i], y[i], z[i]};
      for (int d = 0; d < 3; d++) {
        int v = (int)floor(cc[d] * Li * nc);
        v %= nc;
        if (v < 0) v += nc;
        c3[d] = v;
        cid[3 * i + d] = v;
      }
      size_t c = ((size_t)c3[0] * nc + c3[1]) * nc + c3[2];
      next[i] = head[c];
      head[c] = i;
    }
    for (int t1 = 0; t1 < n; t1++) {
      double f3[3] = {0, 0, 0};
      for (int dx = -1; dx <= 1; dx++)
        for (int dy = -1; dy <= 1; dy++)
          for (int dz = -1; dz <= 1; dz++) {
            int cx = (cid[3 * t1] + dx + nc) % nc, cy = (cid[3 * t1 + 1] + dy + nc) % nc,
                cz = (cid[3 * t1 + 2] + dz + nc) % nc;
            for (int t2 = head[((size_t)cx * nc + cy) * nc + cz]; t2 >= 0; t2 = next[t2])
              if (t2 != t1) pair_term(x, y, z, q, L, Li, rcut, alpha, t1, t2, f3, &en);
          }
      for (int d = 0; d < 3; d++) fr[(size_t)d * n + t1] += f3[d];
    }
    free(head);
    free(next);
    free(cid);
  }
  if (energy) *energy += en;
  return 0;
}

/* One force evaluation (Calculate_forces, common.c:268-327): zero, real
 * space when rcut != 0, k-space, f += f_k + f_r.  Arrays 3n; fk/fr may be
 * NULL (scratch used). */
int oracle_forces(int method, int m, int cao, int mc, double alpha, double rcut, int n, const double *x,
                  const double *y, const double *z, const double *q, double L, const double *G, double *f, double *fk,
                  double *fr, double *energy, int cells) {
  const size_t n3 = 3 * (size_t)n;
  double *fk_ = fk ? fk : (double *)malloc(sizeof(double) * n3);
  double *fr_ = fr ? fr : (double *)malloc(sizeof(double) * n3);
  memset(f, 0, sizeof(double) * n3);
  memset(fk_, 0, sizeof(double) * n3);
  memset(fr_, 0, sizeof(double) * n3);
  double en = 0.0;
  if (rcut != 0.0) oracle_realspace(n, x, y, z, q, L, rcut, alpha, fr_, &en, cells);
  int rc = oracle_kspace(method, m, cao, mc, alpha, n, x, y, z, q, L, G, fk_, f);
  for (size_t t = 0; t < n3; t++) f[t] += fk_[t] + fr_[t];
  if (energy) *energy = en;
  if (!fk) free(fk_);
  if (!fr) free(fr_);
  return rc;
}

/* ------------------------------------------------------------- Ewald */

static double ewald_err_r(double q2, double L, double rcut, double a) {
  /* Kolafa-Perram eq. 16 (ewald.c:175-181) */
  return q2 * sqrt(rcut / (2.0 * L * L * L)) * exp(-SQ(a) * rcut * rcut) / (SQ(a) * rcut * rcut);
}
static double ewald_err_k(double q2, int n, double L, int kmax, double a) {
  /* Petersen 1995 eq. 11 (ewald.c:183-196) */
  return 2.0 * q2 * a / L * sqrt(1.0 / (ORC_PI * kmax * n)) * exp(-SQ(ORC_PI * kmax / (a * L)));
}

/* alpha by bisection of err_r - err_k on [0.01, 10] to 1e-10 and kmax = 2,
 * 4, ... until the total estimate <= 1e-8 (common.c:337-344,
 * ewald.c:204-229).  The bisection's k-space term uses kmax = the caller's
 * P3M mesh parameter (the driver passes its own parameters_t there, so
 * op.mesh still holds the P3M mesh at common.c:339).  Returns -1 if the
 * bisection cannot start. */
int oracle_ewald_parameters(int n, double q2, double L, int mesh_param, double *alpha, int *kmax) {
  const double rcut = 0.49 * L;
  double lo = 0.01, hi = 10.0;
  double flo = ewald_err_r(q2, L, rcut, lo) - ewald_err_k(q2, n, L, mesh_param, lo);
  double fhi = ewald_err_r(q2, L, rcut, hi) - ewald_err_k(q2, n, L, mesh_param, hi);
  if (flo * fhi > 0.0) return -1;
  do {
    double g = 0.5 * (lo + hi);
    double fg = ewald_err_r(q2, L, rcut, g) - ewald_err_k(q2, n, L, mesh_param, g);
    if (flo * fg < 0.0)
      hi = g;
    else
      lo = g;
  } while (fabs(lo - hi) > 1.0e-10);
  double a = 0.5 * (lo + hi);
  int k = 2;
  while (sqrt(SQ(ewald_err_r(q2, L, rcut, a)) + SQ(ewald_err_k(q2, n, L, k, a))) > 1e-8) k += 2;
  *alpha = a;
  *kmax = k;
  return 0;
}

/* Ewald influence value for integer vector (|nx|,|ny|,|nz|) exactly as the
 * reference driver leaves its table: computed once with cutoff kmax^2
 * (Ewald_init -> Init_data, p3m-common.c:218) and again with cutoff
 * (kmax-1)^2 over indices < kmax (common.c:352), so entries with an index
 * equal to kmax keep the first cutoff. */
static double ewald_ghat(int ax, int ay, int az, int kmax, int shell, double alpha, double L) {
  int n2 = ax * ax + ay * ay + az * az;
  int cut = (!shell || ax == kmax || ay == kmax || az == kmax) ? kmax * kmax : (kmax - 1) * (kmax - 1);
  if (n2 == 0 || n2 > cut) return 0.0;
  return 2.0 / SQ(L) / n2 * exp(-SQ(ORC_PI / (alpha * L)) * n2);
}

/* k-space Ewald force on the targets tgt[0..nt) from all n sources
 * (ewald.c:122-166) accumulated into fk (3nt).  shell != 0: the influence
 * table of the reference-force driver (above); shell == 0: the plain
 * cutoff |n|^2 <= kmax^2. */
static int ewald_kspace(int n, const double *x, const double *y, const double *z, const double *q, double L,
                        double alpha, int kmax, int shell, int nt, const int *tgt, double *fk) {
  const double Leni = 1.0 / L;
  for (int nx = -kmax; nx <= kmax; nx++)
    for (int ny = -kmax; ny <= kmax; ny++)
      for (int nz = -kmax; nz <= kmax; nz++) {
        if (nx * nx + ny * ny + nz * nz > kmax * kmax) continue;
        double g = ewald_ghat(abs(nx), abs(ny), abs(nz), kmax, shell, alpha, L);
        double re = 0.0, im = 0.0;
        for (int i = 0; i < n; i++) {
          double kr = 2.0 * ORC_PI * Leni * (nx * x[i] + ny * y[i] + nz * z[i]);
          re += q[i] * cos(kr);
          im += q[i] * -sin(kr);
        }
        if (g == 0.0) continue;
        for (int t = 0; t < nt; t++) {
          int i = tgt ? tgt[t] : t;
          double kr = 2.0 * ORC_PI * Leni * (nx * x[i] + ny * y[i] + nz * z[i]);
          double ff = q[i] * g * (re * sin(kr) + im * cos(kr));
          fk[t] += nx * ff;
          fk[(size_t)nt + t] += ny * ff;
          fk[2 * (size_t)nt + t] += nz * ff;
        }
      }
  return 0;
}

int oracle_ewald_kspace(int n, const double *x, const double *y, const double *z, const double *q, double L, double alpha,
                        int kmax, int nt, const int *tgt, double *fk) {
  return ewald_kspace(n, x, y, z, q, L, alpha, kmax, 1, nt, tgt, fk);
}

/* The Ewald k-space forces of main.c's "error_k" column (main.c:392-396):
 * the influence table is first filled at alpha = 0 (all zero, main.c:190-196
 * before Ewald_init) and then at alpha with kmax = mesh - 1
 * (ewald.c:84-109), so the sum runs over 0 < |n|^2 <= (mesh-1)^2. */
int oracle_ewald_kspace_plain(int n, const double *x, const double *y, const double *z, const double *q, double L,
                              double alpha, int kmax, int nt, const int *tgt, double *fk) {
  return ewald_kspace(n, x, y, z, q, L, alpha, kmax, 0, nt, tgt, fk);
}

/* Reference forces (Calculate_reference_forces, common.c:329-363) on the
 * targets (all particles when tgt == NULL, nt == n): real space with
 * rcut = 0.49 L plus the Ewald k-space sum.  Arrays 3nt. */
int oracle_ewald(int n, const double *x, const double *y, const double *z, const double *q, double L, int mesh_param,
                 int nt, const int *tgt, double *f, double *fk, double *fr, double *alpha_out, int *kmax_out) {
  double q2 = 0.0;
  for (int i = 0; i < n; i++) q2 += q[i] * q[i];
  double alpha;
  int kmax;
  if (oracle_ewald_parameters(n, q2, L, mesh_param, &alpha, &kmax)) return -1;
  const size_t n3 = 3 * (size_t)nt;
  double *fk_ = fk ? fk : (double *)malloc(sizeof(double) * n3);
  double *fr_ = fr ? fr : (double *)malloc(sizeof(double) * n3);
  memset(fk_, 0, sizeof(double) * n3);
  memset(fr_, 0, sizeof(double) * n3);
  const double rcut = 0.49 * L, Li = 1.0 / L;
  double en = 0.0;
  for (int t = 0; t < nt; t++) {
    int i = tgt ? tgt[t] : t;
    double f3[3] = {0, 0, 0};
    for (int j = 0; j < n; j++)
      if (j != i) pair_term(x, y, z, q, L, Li, rcut, alpha, i, j, f3, &en);
    for (int d = 0; d < 3; d++) fr_[(size_t)d * nt + t] += f3[d];
  }
  oracle_ewald_kspace(n, x, y, z, q, L, alpha, kmax, nt, tgt, fk_);
  for (size_t t = 0; t < n3; t++) f[t] = fk_[t] + fr_[t];
  if (alpha_out) *alpha_out = alpha;
  if (kmax_out) *kmax_out = kmax;
  if (!fk) free(fk_);
  if (!fr) free(fr_);
  return 0;
}

/* RMS force error sqrt(sum |f - ref|^2 / n) (error.c:21-34, main.c:446). */
double oracle_rms_error(int n, const double *f, const double *ref) {
  double s = 0.0;
  for (size_t t = 0; t < 3 * (size_t)n; t++) s += SQ(f[t] - ref[t]);
  return sqrt(s) / sqrt((double)n);
}

/* ------------------------------------------------------ error estimates */

/* Realspace_error (realpart.c:343-346) */
double oracle_realspace_error(int n, double q2, double L, double rcut, double alpha) {
  return (2.0 * q2 * exp(-SQ(rcut * alpha))) / sqrt((double)n * rcut * L * L * L);
}

static double cot_sum(int nn, double mi, int cao) {
  /* closed form of sum_m sinc^(2cao)((n + m M)/M) (p3m-common.c:77-107) */
  double c = SQ(cos(ORC_PI * mi * (double)nn));
  switch (cao) {
    case 1: return 1.0;
    case 2: return (1.0 + c * 2.0) / 3.0;
    case 3: return (2.0 + c * (11.0 + c * 2.0)) / 15.0;
    case 4: return (17.0 + c * (180.0 + c * (114.0 + c * 4.0))) / 315.0;
    case 5: return (62.0 + c * (1072.0 + c * (1452.0 + c * (247.0 + c * 2.0)))) / 2835.0;
    case 6: return (1382.0 + c * (35396.0 + c * (83021.0 + c * (34096.0 + c * (2026.0 + c * 4.0))))) / 155925.0;
    case 7:
      return (21844.0 + c * (776661.0 + c * (2801040.0 + c * (2123860.0 + c * (349500.0 + c * (8166.0 + c * 4.0)))))) /
             6081075.0;
  }
  return 0.0;
}

/* Mesh-sum part of the analytic k-space error estimates:
 * ik p3m-ik.c:264-336, ik-i p3m-ik-i.c:249-318, ad p3m-ad.c:436-497,
 * ad-i p3m-ad-i.c:205-284.  mc_est = P3M_BRILLOUIN_TUNING.  Returns the
 * accumulated he_q starting from `he` (before the final fabs). */
static double kspace_he(int method, int m, int cao, int mc_est, double alpha, double L, double he) {
  const double mi = 1.0 / m, f1 = SQ(ORC_PI / (alpha * L));
  for (int nx = -m / 2; nx < m / 2; nx++)
    for (int ny = -m / 2; ny < m / 2; ny++)
      for (int nz = -m / 2; nz < m / 2; nz++) {
        int any = (nx != 0) || (ny != 0) || (nz != 0);
        int all = (nx != 0) && (ny != 0) && (nz != 0);
        if (is_ad(method) ? !all : !any) continue;
        double a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0;
        for (int mx = -mc_est; mx <= mc_est; mx++)
          for (int my = -mc_est; my <= mc_est; my++)
            for (int mz = -mc_est; mz <= mc_est; mz++) {
              double nmx = nx + mx * m, nmy = ny + my * m, nmz = nz + mz * m;
              double nm2 = SQ(nmx) + SQ(nmy) + SQ(nmz);
              double ex = exp(-f1 * nm2);
              double U2 = ipow(sinc_pi(mi * nmx) * sinc_pi(mi * nmy) * sinc_pi(mi * nmz), 2 * cao);
              int even = ((mx + my + mz) % 2) == 0;
              a1 += SQ(ex) / nm2;
              if (is_ad(method)) {
                a2 += U2 * ex;
                a3 += U2 * nm2;
                a4 += U2;
                a5 += even ? U2 * nm2 : -U2 * nm2;
                a6 += even ? U2 : -U2;
              } else {
                a2 += U2 * ex * (nx * nmx + ny * nmy + nz * nmz) / nm2;
                a3 += U2;
                a4 += even ? U2 : -U2;
              }
            }
        double n2 = (double)(nx * nx + ny * ny + nz * nz);
        if (method == 0 || method == 6) {
          double cs = cot_sum(nx, mi, cao) * cot_sum(ny, mi, cao) * cot_sum(nz, mi, cao);
          he += a1 - SQ(a2 / cs) / n2;
        } else if (method == 1) {
          he += a1 - SQ(a2) / (0.5 * n2 * (SQ(a3) + SQ(a4)));
        } else if (method == 3) {
          he += a1 - SQ(a2) / (0.5 * (a3 * a4 + a5 * a6));
        } else {
          if (a3 == 0.0 || a4 == 0.0) continue;
          he += a1 - SQ(a2) / (a3 * a4);
        }
      }
  return he;
}

/* Mesh sizes the reference ships precomputed k-space error tables for
 * (q.c:1, 83 sizes): the even 13-smooth sizes 4..300 except 286 = 2*11*13,
 * plus 360, 400, 480 and 512. */
int oracle_estimate_table_mesh(int m) {
  if (m == 360 || m == 400 || m == 480 || m == 512) return 1;
  if (m < 4 || m > 300 || (m % 2) || (m % 143) == 0) return 0;
  int r = m;
  static const int primes[6] = {2, 3, 5, 7, 11, 13};
  for (int i = 0; i < 6; i++)
    while (r % primes[i] == 0) r /= primes[i];
  return r == 1;
}

/* Analytic k-space error estimate (Error_k of the method table).
 *
 * ik (0, 6) and ik-i (1) first look alpha*L up in precomputed tables
 * (p3m-ik.c:267, p3m-ik-i.c:301, find_error.c:84-107): for a tabulated
 * mesh, cao 1..7 and alpha*L <= 100 the reference interpolates linearly
 * between the table's values at alpha*L = 0, 1, ..., 100.  Those table
 * values are the same mesh sum evaluated at the grid points (to the
 * table's 7 printed digits) with mc_est = 0 for ik and mc_est = 1 for ik-i,
 * so the table branch is restated by evaluating the sum at the two
 * bracketing grid points.  On a miss, ik
 * keeps the lookup's -1 as the start of its sum (p3m-ik.c:266-291); ik-i
 * resets to 0 (p3m-ik-i.c:303). */
double oracle_kspace_error(int method, int m, int cao, int mc_est, double alpha, int n, double q2, double L) {
  const double aL = alpha * L;
  double he;
  if ((method == 0 || method == 1 || method == 6) && oracle_estimate_table_mesh(m) && cao >= 1 && cao <= 7 &&
      aL <= 100.0) {
    const int l = (int)floor(aL);
    const double d = aL - l;
    const int mc_tab = (method == 1) ? 1 : 0;
    he = (1.0 - d) * fabs(kspace_he(method, m, cao, mc_tab, (double)l / L, L, 0.0));
    if (d != 0.0) he += d * fabs(kspace_he(method, m, cao, mc_tab, (double)(l + 1) / L, L, 0.0));
  } else {
    he = kspace_he(method, m, cao, mc_est, alpha, L, (method == 0 || method == 6) ? -1.0 : 0.0);
    if (method != 2 && method != 7) he = fabs(he);
  }
  return 2.0 * q2 * sqrt(he / (double)n) / SQ(L);
}

/* ------------------------------------- inhomogeneous estimate and error map */

/* signed index of a DFT bin: i - m for i >= m/2 (p3m-common.c:494-499) */
static int half_signed(int i, int m) { return (i >= m / 2) ? i - m : i; }

/* (sinc(a/m) sinc(b/m) sinc(c/m))^e (p3m-common.c:351-357, U and U2) */
static double window_hat(int a, int b, int c, int m, int e) {
  return pow(sinc_pi((double)a / m) * sinc_pi((double)b / m) * sinc_pi((double)c / m), e);
}

/* Influence function of the estimator: the B/A ratio of p3m-common.c:359-392
 * with no alias images (mc = 0), B = U2 Ghat k^2, A = U2 (k^2 U2), together
 * with Ghat = 4 pi/k^2 exp(-k^2/(4 alpha^2)) (p3m-common.c:310-313) and U2. */
static double inhomo_gopt(int a, int b, int c, int m, int cao, double alpha, double L, double *ghat, double *u2) {
  const double k2 = SQ(2.0 * ORC_PI / L) * (SQ((double)a) + SQ((double)b) + SQ((double)c));
  const double g = (4 * ORC_PI / k2) * exp(-k2 / (4 * alpha * alpha));
  const double w2 = window_hat(a, b, c, m, 2 * cao);
  *ghat = g;
  *u2 = w2;
  return (w2 * g * k2) / (w2 * (k2 * w2));
}

/* B-spline weights of order tab_cao at the tabulated offset of one
 * coordinate, read for `count` stencil points: entries past the table's
 * order are 0 here (the reference reads past its table rows there,
 * interpol.c:38-44). */
static void inhomo_stencil(double xc, double Hi, double shift, int m, int tab_cao, int count, int *base, double *w) {
  double pos = xc * Hi - shift;
  int nmp = (int)floor(pos + 0.5);
  int b = nmp % m;
  *base = b < 0 ? b + m : b;
  int arg = (int)floor((pos - nmp + 0.5) * 131072.0);
  double wt[8] = {0};
  oracle_bspline(tab_cao, (double)(arg - 65536) / 131072.0, wt, NULL);
  for (int j = 0; j < count; j++) w[j] = (j < tab_cao) ? wt[j] : 0.0;
}

/* Generic_error_estimate_inhomo (p3m-common.c:437-719).
 *
 * Mesh `mesh`, window order `cao`:
 *   rho2(r) = sum_i q_i^2 W(r - x_i)  (assign_charge_q2, charge-assign.c:1544-1590),
 *             or sum q^2 / mesh^3 everywhere with `uniform`;
 *   K_d(k) = -2 pi i k_d/L (U2 G_opt - Ghat)  (homogeneous part, :489-534);
 *   for each alias vector a in [-mc, mc]^3 without 0 (:558-625):
 *     K_d^a(k2) = -i (k2_d/L) 2 pi U(k2) U(-k2 - a m) G_opt(k2)
 *                 * sum_{k != 0} (k_d/L) 2 pi U(k) U(k + a m) G_opt(k)
 *     (the reference adds the product term by term over k for every k2; the
 *      sum over k factors out and is formed once here);
 *   K2(r) = sum_d Re(IDFT K_d)^2 + sum_a sum_d Re(IDFT K_d^a)^2;
 *   E = IDFT[DFT(rho2) * DFT(K2)], the product taken component by component
 *       (re*re, im*im) as at :664-672;
 *   rms_i = q_i^2 sum_stencil W E  (collect_rms_nocf, charge-assign.c:1650-1705)
 *           with the mesh spacing and stencil length of collect_mesh and
 *           collect_cao (the reference passes its force-method parameters
 *           there) and the window table of order cao;
 *   estimate = sqrt(sum_i rms_i / n).
 * DFTs unnormalised.  mesh_out (5 mesh^3 doubles, may be NULL) receives per
 * mesh point rho2, Re E, Im E, Re DFT(K2), Im DFT(K2) (the columns of the
 * reference's inhomo_output file, :688-692). */
int oracle_inhomo_error(int n, const double *x, const double *y, const double *z, const double *q, double L,
                        double alpha, int uniform, int mesh, int cao, int mc, int collect_mesh, int collect_cao,
                        double *estimate, double *mesh_out) {
  if (mesh < 2 || cao < 1 || cao > 7 || collect_cao < 1 || collect_cao > 7 || collect_mesh < 1 || mc < 0 || n < 0)
    return -1;
  const int m = mesh;
  const size_t M = (size_t)m * m * m;
  double *rho2 = (double *)calloc(2 * M, sizeof(double));
  double *E = (double *)calloc(2 * M, sizeof(double));
  double *K2 = (double *)calloc(2 * M, sizeof(double));
  double *Kd = (double *)calloc(6 * M, sizeof(double));
  double *gopt = (double *)malloc(M * sizeof(double));
  double *uw = (double *)malloc(M * sizeof(double));
  int dims[3] = {m, m, m};
  int base[3];
  double w[3][8];

  if (!uniform) {
    const double Hi = (double)m / L, shift = (double)((cao - 1) / 2);
    for (int i = 0; i < n; i++) {
      const double c[3] = {x[i], y[i], z[i]};
      for (int d = 0; d < 3; d++) inhomo_stencil(c[d], Hi, shift, m, cao, cao, &base[d], w[d]);
      const double q2 = SQ(q[i]);
      for (int a = 0; a < cao; a++) {
        const int I = (base[0] + a) % m;
        const double t0 = q2 * w[0][a];
        for (int b = 0; b < cao; b++) {
          const int J = (base[1] + b) % m;
          const double t1 = t0 * w[1][b];
          for (int cc = 0; cc < cao; cc++) rho2[cidx(I, J, (base[2] + cc) % m, m)] += t1 * w[2][cc];
        }
      }
    }
  } else {
    double q2 = 0.0;
    for (int i = 0; i < n; i++) q2 += SQ(q[i]);
    for (size_t t = 0; t < M; t++) rho2[2 * t] = q2 / (double)M;
  }

  /* homogeneous kernel, and G_opt / U per bin for the alias terms */
  for (int i = 0; i < m; i++)
    for (int j = 0; j < m; j++)
      for (int k = 0; k < m; k++) {
        const size_t t = ((size_t)i * m + j) * m + k;
        const int tn[3] = {half_signed(i, m), half_signed(j, m), half_signed(k, m)};
        gopt[t] = 0.0;
        uw[t] = window_hat(tn[0], tn[1], tn[2], m, cao);
        if (tn[0] == 0 && tn[1] == 0 && tn[2] == 0) continue;
        double ghat, u2;
        const double g = inhomo_gopt(tn[0], tn[1], tn[2], m, cao, alpha, L, &ghat, &u2);
        gopt[t] = g;
        const double kv = u2 * g - ghat;
        for (int d = 0; d < 3; d++) Kd[2 * (d * M + t) + 1] = -2 * ORC_PI * tn[d] / L * kv;
      }
  for (int d = 0; d < 3; d++) oracle_dft_nd(Kd + 2 * d * M, 3, dims, +1);
  for (size_t t = 0; t < M; t++) {
    double kr = 0.0;
    for (int d = 0; d < 3; d++) kr += SQ(Kd[2 * (d * M + t)]);
    K2[2 * t] = kr;
  }

  /* alias terms */
  for (int ax = -mc; ax <= mc; ax++)
    for (int ay = -mc; ay <= mc; ay++)
      for (int az = -mc; az <= mc; az++) {
        if (ax == 0 && ay == 0 && az == 0) continue;
        double S[3] = {0, 0, 0};
        for (int i = 0; i < m; i++)
          for (int j = 0; j < m; j++)
            for (int k = 0; k < m; k++) {
              const size_t t = ((size_t)i * m + j) * m + k;
              const int tn[3] = {half_signed(i, m), half_signed(j, m), half_signed(k, m)};
              if (tn[0] == 0 && tn[1] == 0 && tn[2] == 0) continue;
              const double k1 = 2 * ORC_PI * uw[t] *
                                window_hat(tn[0] + ax * m, tn[1] + ay * m, tn[2] + az * m, m, cao) * gopt[t];
              for (int d = 0; d < 3; d++) S[d] += (tn[d] / L) * k1;
            }
        memset(Kd, 0, 6 * M * sizeof(double));
        for (int i = 0; i < m; i++)
          for (int j = 0; j < m; j++)
            for (int k = 0; k < m; k++) {
              const size_t t = ((size_t)i * m + j) * m + k;
              const int tn[3] = {half_signed(i, m), half_signed(j, m), half_signed(k, m)};
              if (tn[0] == 0 && tn[1] == 0 && tn[2] == 0) continue;
              const double k2 = 2 * ORC_PI * uw[t] *
                                window_hat(-tn[0] - ax * m, -tn[1] - ay * m, -tn[2] - az * m, m, cao) * gopt[t];
              for (int d = 0; d < 3; d++) Kd[2 * (d * M + t) + 1] = -(tn[d] / L) * k2 * S[d];
            }
        for (int d = 0; d < 3; d++) oracle_dft_nd(Kd + 2 * d * M, 3, dims, +1);
        for (size_t t = 0; t < M; t++) {
          double kr = 0.0;
          for (int d = 0; d < 3; d++) kr += SQ(Kd[2 * (d * M + t)]);
          K2[2 * t] += kr;
        }
      }

  oracle_dft_nd(K2, 3, dims, -1);
  memcpy(E, rho2, 2 * M * sizeof(double));
  oracle_dft_nd(E, 3, dims, -1);
  for (size_t t = 0; t < 2 * M; t++) E[t] *= K2[t];
  oracle_dft_nd(E, 3, dims, +1);

  /* collect at the particles */
  double sum = 0.0;
  {
    const double Hi = (double)collect_mesh / L, shift = (double)((collect_cao - 1) / 2);
    for (int i = 0; i < n; i++) {
      const double c[3] = {x[i], y[i], z[i]};
      for (int d = 0; d < 3; d++) inhomo_stencil(c[d], Hi, shift, m, cao, collect_cao, &base[d], w[d]);
      const double q2 = SQ(q[i]);
      double r = 0.0;
      for (int a = 0; a < collect_cao; a++) {
        const int I = (base[0] + a) % m;
        const double t0 = q2 * w[0][a];
        for (int b = 0; b < collect_cao; b++) {
          const int J = (base[1] + b) % m;
          const double t1 = t0 * w[1][b];
          for (int cc = 0; cc < collect_cao; cc++) r += E[cidx(I, J, (base[2] + cc) % m, m)] * (t1 * w[2][cc]);
        }
      }
      sum += r;
    }
  }
  *estimate = sqrt(sum / n);
  if (mesh_out)
    for (size_t t = 0; t < M; t++) {
      mesh_out[5 * t + 0] = rho2[2 * t];
      mesh_out[5 * t + 1] = E[2 * t];
      mesh_out[5 * t + 2] = E[2 * t + 1];
      mesh_out[5 * t + 3] = K2[2 * t];
      mesh_out[5 * t + 4] = K2[2 * t + 1];
    }
  free(rho2);
  free(E);
  free(K2);
  free(Kd);
  free(gopt);
  free(uw);
  return 0;
}

/* Error_map (p3m-common.c:402-435): the squared k-space force error of
 * each particle, |fk_ref - fk|^2, assigned to a mesh of `mesh` points per
 * side with the window of order cao (assign_charge_nocf,
 * charge-assign.c:1592-1648).  fk and fk_ref are 3n arrays; map receives
 * mesh^3 doubles (the real parts of the reference's complex mesh). */
int oracle_error_map(int n, const double *x, const double *y, const double *z, double L, const double *fk,
                     const double *fk_ref, int mesh, int cao, double *map) {
  if (mesh < 1 || cao < 1 || cao > 7 || n < 0) return -1;
  const int m = mesh;
  const size_t M = (size_t)m * m * m;
  memset(map, 0, M * sizeof(double));
  const double Hi = (double)m / L, shift = (double)((cao - 1) / 2);
  int base[3];
  double w[3][8];
  for (int i = 0; i < n; i++) {
    double dF = 0.0;
    for (int d = 0; d < 3; d++) dF += SQ(fk_ref[(size_t)d * n + i] - fk[(size_t)d * n + i]);
    const double c[3] = {x[i], y[i], z[i]};
    for (int d = 0; d < 3; d++) inhomo_stencil(c[d], Hi, shift, m, cao, cao, &base[d], w[d]);
    for (int a = 0; a < cao; a++) {
      const int I = (base[0] + a) % m;
      const double t0 = dF * w[0][a];
      for (int b = 0; b < cao; b++) {
        const int J = (base[1] + b) % m;
        const double t1 = t0 * w[1][b];
        for (int cc = 0; cc < cao; cc++) map[((size_t)I * m + J) * m + (base[2] + cc) % m] += t1 * w[2][cc];
      }
    }
  }
  return 0;
}
