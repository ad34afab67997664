// Optimal influence function G_opt with its aliasing sums, and the ad
// self-force coefficients, in FP64 on the GPU (one thread per k-vector).
//
// Formulas (all per mesh index (NX,NY,NZ), signed frequencies
// n_d = i - round(i/m) m (p3m-common.c:133-143), aliases n_d + m M_d,
// |M_d| <= mc):
//   ik    p3m-ik.c:93-173     G = 2/pi * (D.Z/L) / (|D/L|^2 N1^2)
//   ik-i  p3m-ik-i.c:78-166   G = 2/pi * (D.Z/L) / (|D/L|^2 1/2 (N1^2 + N2^2))
//   ad    p3m-ad.c:69-158     G = Z / (pi N1 N2)
//   ad-i  p3m-ad-i.c:70-150   G = Z / (1/2 pi (N1 N2 + N3 N4))
// with the reference's zeroing: k = 0 always; for ik/ik-i every k whose
// three indices are 0 mod m/2; ad returns all zeros when alpha == 0.
// D is the differential operator Dn[i] = n_i with Dn[m/2] = 0
// (p3m-common.c:110-131).
#include <math.h>

#include "p3mg_internal.cuh"

namespace p3mg {

namespace {

__device__ __forceinline__ double ipow_d(double b, int e) {
  double r = 1.0;
  for (int i = 0; i < e; i++) r *= b;
  return r;
}

__device__ __forceinline__ double sinc_pi(double d) {
  const double a = P3MG_PI * d;
  return d == 0.0 ? 1.0 : sin(a) / a;
}

__device__ __forceinline__ double signed_freq(int i, int m) {
  return (double)i - round((double)i / (double)m) * (double)m;
}

// Per-axis alias factors of G_opt for an alias range mc (the three axes of
// the cubic box share them).  For mesh index i in [0, m) and alias r in
// [0, 2 mc + 1) -- the frequency n = n_i + m (r - mc), n_i the signed
// frequency of i --
//   A[3 (i NA + r)] = the sinc power ((sinc^cao)^2 or sinc^(2 cao)) at n / m,
//   A[3 (i NA + r) + 1] = n / L,   A[3 (i NA + r) + 2] = (n / L)^2,
//   E[(a m + i) NA + r] = exp(-(pi / alpha_a)^2 (n / L)^2) for alpha a of na
// (alphas on the device, or alpha_v when alphas is null).  The mesh-point
// kernels read these instead of evaluating 3 NA sines and 3 NA
// exponentials per point.
__global__ void influence_axis_kernel(double *__restrict__ A, double *__restrict__ E, int method, int m, int cao,
                                      int mc, double L, const double *__restrict__ alphas, double alpha_v, int na) {
  const int NA = 2 * mc + 1;
  const int nA = m * NA;
  const bool ik_sq = (method == 0 || method == 6);
  const double Leni = 1.0 / L, fak1 = 1.0 / (double)m;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nA * (na + 1); t += gridDim.x * blockDim.x) {
    const int a = t / nA - 1, e = t % nA;  // a = -1: the alpha-independent part
    const int i = e / NA, r = e % NA;
    const double n = signed_freq(i, m) + (double)(m * (r - mc));
    const double nl = n * Leni;
    if (a < 0) {
      const double sx = sinc_pi(fak1 * n);
      A[3 * e] = ik_sq ? ipow_d(ipow_d(sx, cao), 2) : ipow_d(sx, 2 * cao);
      A[3 * e + 1] = nl;
      A[3 * e + 2] = nl * nl;
    } else {
      const double pa = P3MG_PI / (alphas ? alphas[a] : alpha_v);
      E[(size_t)a * nA + e] = exp(-(pa * pa) * (nl * nl));
    }
  }
}

// G_opt at one mesh point (NX, NY, NZ) away from the zeroed ones, and with
// want_dg dG/dalpha (each exp(-(pi/alpha)^2 |n|^2) factor differentiated; the
// rest of the formula is linear in those sums).  MC >= 0: the alias range
// mc == MC fixed at compile time, so the per-axis sinc powers and Gaussian
// factors of the (2 MC + 1) aliases are tabulated once (3 (2MC+1) sin and
// exp instead of (2MC+1)^3; the Gaussian of an alias is the product of its
// three axis factors).  MC < 0: any mc, evaluated alias by alias.
template <int MC>
__device__ __forceinline__ void influence_point(int method, int m, int cao, int mc, double alpha, double L, int NX,
                                                int NY, int NZ, bool want_dg, double *g_out, double *dg_out,
                                                const double *__restrict__ A, const double *__restrict__ Ea) {
  const int half = m / 2;
  const bool ad = method_ad(method);
  const bool ik_sq = (method == 0 || method == 6);  // (sinc^cao)^2, else sinc^(2 cao)
  const double Leni = 1.0 / L, fak1 = 1.0 / (double)m;
  const double pa = P3MG_PI / alpha;
  const double fak2 = pa * pa;
  const double nx = signed_freq(NX, m), ny = signed_freq(NY, m), nz = signed_freq(NZ, m);
  double Zx = 0.0, Zy = 0.0, Zz = 0.0, Z = 0.0, N1 = 0.0, N2 = 0.0, N3 = 0.0, N4 = 0.0;
  double dZx = 0.0, dZy = 0.0, dZz = 0.0, dZ = 0.0;
  const double dfac = 2.0 * fak2 / alpha;  // d/dalpha of -fak2 NM2 is dfac NM2
  // one alias term: S3 the product of the sinc powers, NM* the shifted
  // frequencies, TE the Gaussian, par the parity of MX + MY + MZ
  // NLX..NLZ: the shifted frequencies over L
  auto term = [&](double S3, double NLX, double NLY, double NLZ, double NM2, double TE, bool even) {
    const double dTE = want_dg ? TE * NM2 * dfac : 0.0;
    N1 += S3;
    if (ad) {
      N2 += S3 * NM2;
      N3 += even ? S3 : -S3;
      N4 += even ? S3 * NM2 : -(S3 * NM2);
      Z += S3 * TE;
      dZ += S3 * dTE;
    } else {
      const double zwi = S3 * TE / NM2;
      Zx += NLX * zwi;
      Zy += NLY * zwi;
      Zz += NLZ * zwi;
      if (want_dg) {
        const double dzwi = S3 * dTE / NM2;
        dZx += NLX * dzwi;
        dZy += NLY * dzwi;
        dZz += NLZ * dzwi;
      }
      N2 += even ? S3 : -S3;
    }
  };
  if constexpr (MC >= 0) {
    // the per-axis factors from influence_axis_kernel's tables
    constexpr int NA = 2 * MC + 1;
    double Lx[NA], Ly[NA], Lz[NA], Qx[NA], Qy[NA], Qz[NA], Sx[NA], Sy[NA], Sz[NA], Ex[NA], Ey[NA], Ez[NA];
#pragma unroll
    for (int i = 0; i < NA; i++) {
      const double *ax = A + 3 * (NX * NA + i), *ay = A + 3 * (NY * NA + i), *az = A + 3 * (NZ * NA + i);
      Sx[i] = ax[0];
      Lx[i] = ax[1];
      Qx[i] = ax[2];
      Sy[i] = ay[0];
      Ly[i] = ay[1];
      Qy[i] = ay[2];
      Sz[i] = az[0];
      Lz[i] = az[1];
      Qz[i] = az[2];
      Ex[i] = Ea[NX * NA + i];
      Ey[i] = Ea[NY * NA + i];
      Ez[i] = Ea[NZ * NA + i];
    }
#pragma unroll
    for (int i = 0; i < NA; i++)
#pragma unroll
      for (int j = 0; j < NA; j++) {
        const double S2 = Sx[i] * Sy[j];
        const double Exy = Ex[i] * Ey[j];
        const double Q2 = Qx[i] + Qy[j];
#pragma unroll
        for (int k = 0; k < NA; k++)
          term(S2 * Sz[k], Lx[i], Ly[j], Lz[k], Q2 + Qz[k], Exy * Ez[k], ((i + j + k - 3 * MC) % 2) == 0);
      }
  } else {
    for (int MX = -mc; MX <= mc; MX++) {
      const double NMX = nx + (double)(m * MX);
      const double sx = sinc_pi(fak1 * NMX);
      const double S1 = ik_sq ? ipow_d(ipow_d(sx, cao), 2) : ipow_d(sx, 2 * cao);
      for (int MY = -mc; MY <= mc; MY++) {
        const double NMY = ny + (double)(m * MY);
        const double sy = sinc_pi(fak1 * NMY);
        const double S2 = S1 * (ik_sq ? ipow_d(ipow_d(sy, cao), 2) : ipow_d(sy, 2 * cao));
        for (int MZ = -mc; MZ <= mc; MZ++) {
          const double NMZ = nz + (double)(m * MZ);
          const double sz = sinc_pi(fak1 * NMZ);
          const double S3 = S2 * (ik_sq ? ipow_d(ipow_d(sz, cao), 2) : ipow_d(sz, 2 * cao));
          const double a = NMX * Leni, b = NMY * Leni, cc = NMZ * Leni;
          const double NM2 = a * a + b * b + cc * cc;
          term(S3, a, b, cc, NM2, exp(-fak2 * NM2), ((MX + MY + MZ) % 2) == 0);
        }
      }
    }
  }
  double g, dg = 0.0;
  if (ad) {
    const double den = (method == 3) ? (0.5 * P3MG_PI * (N1 * N2 + N3 * N4)) : (P3MG_PI * N1 * N2);
    g = Z / den;
    if (want_dg) dg = dZ / den;
  } else {
    const double Dx = (NX == half) ? 0.0 : nx, Dy = (NY == half) ? 0.0 : ny, Dz = (NZ == half) ? 0.0 : nz;
    double num = Dx * Zx * Leni + Dy * Zy * Leni + Dz * Zz * Leni;
    double dnum = Dx * dZx * Leni + Dy * dZy * Leni + Dz * dZz * Leni;
    const double dxl = Dx * Leni, dyl = Dy * Leni, dzl = Dz * Leni;
    const double d2 = dxl * dxl + dyl * dyl + dzl * dzl;
    if (method == 1) {
      num /= d2;
      num /= 0.5 * (N1 * N1 + N2 * N2);
      dnum /= d2;
      dnum /= 0.5 * (N1 * N1 + N2 * N2);
    } else {
      num /= d2 * (N1 * N1);
      dnum /= d2 * (N1 * N1);
    }
    g = 2.0 * num / P3MG_PI;
    dg = 2.0 * dnum / P3MG_PI;
  }
  *g_out = g;
  *dg_out = dg;
}

// G_opt is even along each axis, G(.., m - i, ..) = G(.., i, ..), for even
// meshes and for the ad methods (the alias set and the formulas are
// symmetric; for odd meshes the ik zeroing of the indices that are 0 mod
// m / 2 is not).  The kernels then evaluate only the folded points, indices
// 0 .. m / 2 on each axis, and write each value to its up to 8 mirror images.
__host__ __device__ inline bool influence_folds(int method, int m) { return (m % 2) == 0 || method_ad(method); }
__host__ __device__ inline int influence_extent(int method, int m) {
  return influence_folds(method, m) ? m / 2 + 1 : m;
}

// v to the mirror images (NX or m - NX, ...) of a folded point (one write
// without folding)
__device__ __forceinline__ void influence_put(double *__restrict__ G, int m, bool fold, int NX, int NY, int NZ,
                                              double v) {
  const int nx = (fold && NX != 0 && 2 * NX != m) ? 2 : 1;
  const int ny = (fold && NY != 0 && 2 * NY != m) ? 2 : 1;
  const int nz = (fold && NZ != 0 && 2 * NZ != m) ? 2 : 1;
  for (int sx = 0; sx < nx; sx++)
    for (int sy = 0; sy < ny; sy++)
      for (int sz = 0; sz < nz; sz++) {
        const int X = sx ? m - NX : NX, Y = sy ? m - NY : NY, Z = sz ? m - NZ : NZ;
        G[((size_t)X * m + Y) * m + Z] = v;
      }
}

// dG (may be NULL): dG/dalpha as well.  MC: see influence_point (launch
// through launch_influence, which picks it from mc).  Threads cover the
// points of influence_extent per axis.
template <int MC>
__global__ void influence_kernel(double *__restrict__ G, int method, int m, int cao, int mc, double alpha_v,
                                 const double *__restrict__ alphas, double L, double *__restrict__ dG,
                                 const double *__restrict__ A, const double *__restrict__ E) {
  const size_t M = (size_t)m * m * m;
  const bool fold = influence_folds(method, m);
  const int h = influence_extent(method, m);
  const size_t ind = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ind >= (size_t)h * h * h) return;
  // alpha batch: grid.y = alpha index (alphas on the device), G of entry y
  const double alpha = alphas ? alphas[blockIdx.y] : alpha_v;
  G += (size_t)blockIdx.y * M;
  const int NZ = (int)(ind % h);
  const int NY = (int)((ind / h) % h);
  const int NX = (int)(ind / ((size_t)h * h));
  const int half = m / 2;
  const bool ad = method_ad(method);
  double g = 0.0, dg = 0.0;
  const bool zero = ((NX | NY | NZ) == 0) || (ad && alpha == 0.0) ||
                    (!ad && (NX % half == 0) && (NY % half == 0) && (NZ % half == 0));
  if (!zero)
    influence_point<MC>(method, m, cao, mc, alpha, L, NX, NY, NZ, dG != nullptr, &g, &dg, A,
                        E ? E + (size_t)blockIdx.y * m * (2 * mc + 1) : nullptr);
  influence_put(G, m, fold, NX, NY, NZ, g);
  if (dG) influence_put(dG, m, fold, NX, NY, NZ, dg);
}

// G_opt for a group of AB alphas per thread (alpha batches, mc <= 2):
// everything but the Gaussian factors is independent of alpha, so the
// per-axis sinc powers, the alias sums N1..N4 and 1/|n_m|^2 are formed once
// per mesh point and only the per-axis Gaussians and their products are
// evaluated per alpha.  Same zeroing and final formula as influence_point.
template <int MC, int AB>
__global__ void influence_group_kernel(double *__restrict__ G, int method, int m, int cao,
                                       const double *__restrict__ alphas, int na, double L,
                                       const double *__restrict__ A, const double *__restrict__ E) {
  const size_t M = (size_t)m * m * m;
  const bool fold = influence_folds(method, m);
  const int h = influence_extent(method, m);
  const size_t ind = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (ind >= (size_t)h * h * h) return;
  const int a0 = blockIdx.y * AB;
  const int nag = min(AB, na - a0);
  const int NZ = (int)(ind % h);
  const int NY = (int)((ind / h) % h);
  const int NX = (int)(ind / ((size_t)h * h));
  const int half = m / 2;
  const bool ad = method_ad(method);
  const bool zero_all = ((NX | NY | NZ) == 0) || (!ad && (NX % half == 0) && (NY % half == 0) && (NZ % half == 0));
  if (zero_all) {
    for (int a = 0; a < nag; a++) influence_put(G + (size_t)(a0 + a) * M, m, fold, NX, NY, NZ, 0.0);
    return;
  }
  const double Leni = 1.0 / L;
  const double nx = signed_freq(NX, m), ny = signed_freq(NY, m), nz = signed_freq(NZ, m);
  constexpr int NA = 2 * MC + 1;
  // the per-axis factors from influence_axis_kernel's tables
  double Lx[NA], Ly[NA], Lz[NA], Qx[NA], Qy[NA], Qz[NA], Sx[NA], Sy[NA], Sz[NA];
#pragma unroll
  for (int i = 0; i < NA; i++) {
    const double *ax = A + 3 * (NX * NA + i), *ay = A + 3 * (NY * NA + i), *az = A + 3 * (NZ * NA + i);
    Sx[i] = ax[0];
    Lx[i] = ax[1];
    Qx[i] = ax[2];
    Sy[i] = ay[0];
    Ly[i] = ay[1];
    Qy[i] = ay[2];
    Sz[i] = az[0];
    Lz[i] = az[1];
    Qz[i] = az[2];
  }
  double Ex[AB][NA], Ey[AB][NA], Ez[AB][NA];
#pragma unroll
  for (int a = 0; a < AB; a++) {
    const double *Eg = E + (size_t)(a < nag ? a0 + a : a0) * m * NA;
#pragma unroll
    for (int i = 0; i < NA; i++) {
      Ex[a][i] = Eg[NX * NA + i];
      Ey[a][i] = Eg[NY * NA + i];
      Ez[a][i] = Eg[NZ * NA + i];
    }
  }
  double N1 = 0.0, N2 = 0.0, N3 = 0.0, N4 = 0.0;
  double Zx[AB], Zy[AB], Zz[AB], Z[AB];
#pragma unroll
  for (int a = 0; a < AB; a++) Zx[a] = Zy[a] = Zz[a] = Z[a] = 0.0;
#pragma unroll
  for (int i = 0; i < NA; i++)
#pragma unroll
    for (int j = 0; j < NA; j++) {
      const double S2 = Sx[i] * Sy[j];
#pragma unroll
      for (int k = 0; k < NA; k++) {
        const double S3 = S2 * Sz[k];
        const double NM2 = Qx[i] + Qy[j] + Qz[k];
        const bool even = ((i + j + k - 3 * MC) % 2) == 0;
        N1 += S3;
        if (ad) {
          N2 += S3 * NM2;
          N3 += even ? S3 : -S3;
          N4 += even ? S3 * NM2 : -(S3 * NM2);
#pragma unroll
          for (int a = 0; a < AB; a++) Z[a] += S3 * (Ex[a][i] * Ey[a][j] * Ez[a][k]);
        } else {
          N2 += even ? S3 : -S3;
          const double w = S3 / NM2;
#pragma unroll
          for (int a = 0; a < AB; a++) {
            const double zwi = w * (Ex[a][i] * Ey[a][j] * Ez[a][k]);
            Zx[a] += Lx[i] * zwi;
            Zy[a] += Ly[j] * zwi;
            Zz[a] += Lz[k] * zwi;
          }
        }
      }
    }
#pragma unroll
  for (int a = 0; a < AB; a++) {
    if (a >= nag) break;
    const double alpha = alphas[a0 + a];
    double g;
    if (ad) {
      if (alpha == 0.0) {
        g = 0.0;
      } else {
        const double den = (method == 3) ? (0.5 * P3MG_PI * (N1 * N2 + N3 * N4)) : (P3MG_PI * N1 * N2);
        g = Z[a] / den;
      }
    } else {
      const double Dx = (NX == half) ? 0.0 : nx, Dy = (NY == half) ? 0.0 : ny, Dz = (NZ == half) ? 0.0 : nz;
      double num = Dx * Zx[a] * Leni + Dy * Zy[a] * Leni + Dz * Zz[a] * Leni;
      const double dxl = Dx * Leni, dyl = Dy * Leni, dzl = Dz * Leni;
      const double d2 = dxl * dxl + dyl * dyl + dzl * dzl;
      if (method == 1) {
        num /= d2;
        num /= 0.5 * (N1 * N1 + N2 * N2);
      } else {
        num /= d2 * (N1 * N1);
      }
      g = 2.0 * num / P3MG_PI;
    }
    influence_put(G + (size_t)(a0 + a) * M, m, fold, NX, NY, NZ, g);
  }
}

// alphas per thread of influence_group_kernel (registers: 2 at mc = 2)
constexpr int influence_ab(int mc) { return mc >= 2 ? 2 : 4; }

// G (and dG) for grid (blocks, na) on the stream
void launch_influence(double *G, int method, int m, int cao, int mc, double alpha, const double *alphas, double L,
                      double *dG, unsigned blocks, int na, int threads, cudaStream_t st, const double *A,
                      const double *E) {
  const dim3 grid(blocks, na);
  switch (mc) {
    case 0: influence_kernel<0><<<grid, threads, 0, st>>>(G, method, m, cao, mc, alpha, alphas, L, dG, A, E); break;
    case 1: influence_kernel<1><<<grid, threads, 0, st>>>(G, method, m, cao, mc, alpha, alphas, L, dG, A, E); break;
    case 2: influence_kernel<2><<<grid, threads, 0, st>>>(G, method, m, cao, mc, alpha, alphas, L, dG, A, E); break;
    default:
      influence_kernel<-1><<<grid, threads, 0, st>>>(G, method, m, cao, mc, alpha, alphas, L, dG, nullptr, nullptr);
      break;
  }
}

// The per-axis tables of influence_axis_kernel for mc <= 2 and na alphas
// (alphas on the device, or the single alpha_v) in the context's table
// buffer; *A = *E = nullptr for larger mc (evaluated alias by alias).
int influence_tables(Ctx *c, const double *alphas, double alpha_v, int na, const double **A, const double **E) {
  *A = *E = nullptr;
  if (c->mc > 2) return P3MG_OK;
  const int m = c->mesh, NA = 2 * c->mc + 1;
  const size_t need = (size_t)m * NA * (3 + (size_t)na);
  if (need > c->infl_cap) {
    if (c->infl_tab) cudaFree(c->infl_tab);
    c->infl_tab = nullptr;
    c->infl_cap = 0;
    P3MG_CUDA_TRY(cudaMalloc(&c->infl_tab, need * sizeof(double)));
    c->infl_cap = need;
  }
  const int tot = m * NA * (na + 1);
  const int threads = 256;
  influence_axis_kernel<<<(tot + threads - 1) / threads, threads, 0, c->stream>>>(
      c->infl_tab, c->infl_tab + (size_t)3 * m * NA, c->method, m, c->cao, c->mc, c->L, alphas, alpha_v, na);
  c->launches++;
  P3MG_CUDA_TRY(cudaGetLastError());
  *A = c->infl_tab;
  *E = c->infl_tab + (size_t)3 * m * NA;
  return P3MG_OK;
}


// ad self-force sums S(m') for the 26 non-zero m' in {-1,0,1}^3
// (p3m-ad-self-forces.c:30-91):
//   S(m') = sum_{k: G(k) != 0} sum_{a in {-1,0,1}^3} G(k) U(k + a m) U(k + (a + m') m),
//   U(k) = (sinc(k_x/m) sinc(k_y/m) sinc(k_z/m))^cao, k the truncated signed frequency.
// U is a product over the axes, U(k + c m) = u_x[c_x] u_y[c_y] u_z[c_z], so
// the alias sum factorises:
//   sum_a U(k + a m) U(k + (a + m') m) = T_x(m'_x) T_y(m'_y) T_z(m'_z),
//   T_d(p) = sum_{a = -1..1} u_d[a] u_d[a + p],  p in {-1, 0, 1},
// nine products per axis and two per m' instead of 27 x 26 triple products.
// G is even along each axis (ad methods) and mirroring an index turns
// T(p) into T(-p), so the sum runs over the folded points (indices 0 .. m/2)
// with the per-axis factor R(p) = T(p) + T(-p) for an index with a distinct
// mirror image (T(p) otherwise): self_axis_kernel tabulates R per index.
__global__ void self_axis_kernel(double *__restrict__ R, int m, int cao) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > m / 2) return;
  // sinc(x + j) = (-1)^j sin(pi x) / (pi (x + j)), x = k / m: one sine for
  // the five alias offsets j = -2..2
  const double x = (double)(int)signed_freq(i, m) / (double)m;
  const double s0 = sin(P3MG_PI * x);
  double u[5];
#pragma unroll
  for (int c = 0; c < 5; c++) {
    const double dj = x + (double)(c - 2);
    const double sc = (dj == 0.0) ? 1.0 : ((c & 1) ? -s0 : s0) / (P3MG_PI * dj);
    u[c] = ipow_d(sc, cao);
  }
  double T[3];
#pragma unroll
  for (int p = -1; p <= 1; p++) T[p + 1] = u[1] * u[1 + p] + u[2] * u[2 + p] + u[3] * u[3 + p];
  const bool pair = (i != 0 && 2 * i != m);
#pragma unroll
  for (int p = 0; p < 3; p++) R[3 * i + p] = pair ? T[p] + T[2 - p] : T[p];
}

// Block reduction of the per-thread sums (each thread takes SELF_PTS folded
// points), then one FP64 atomic per sum.
constexpr int SELF_PTS = 8;

__global__ void self_force_sum_kernel(const double *__restrict__ G, const double *__restrict__ R, int m,
                                      double *__restrict__ S26) {
  __shared__ double red[26][8];
  const size_t M = (size_t)m * m * m;
  const int h = m / 2 + 1;
  const size_t H = (size_t)h * h * h;
  G += (size_t)blockIdx.y * M;  // alpha batch (grid.y)
  S26 += 26 * blockIdx.y;
  double acc[26];
#pragma unroll
  for (int t = 0; t < 26; t++) acc[t] = 0.0;
  const size_t first = ((size_t)blockIdx.x * SELF_PTS) * blockDim.x + threadIdx.x;
  for (int it = 0; it < SELF_PTS; it++) {
    const size_t ind = first + (size_t)it * blockDim.x;
    if (ind >= H) break;
    const int nz = (int)(ind % h), ny = (int)((ind / h) % h), nx = (int)(ind / ((size_t)h * h));
    const double g = G[((size_t)nx * m + ny) * m + nz];
    if (g == 0.0) continue;
    double Tx[3], Ty[3], Tz[3];
#pragma unroll
    for (int p = 0; p < 3; p++) {
      Tx[p] = R[3 * nx + p];
      Ty[p] = R[3 * ny + p];
      Tz[p] = R[3 * nz + p];
    }
    int t = 0;
#pragma unroll
    for (int px = 0; px < 3; px++)
#pragma unroll
      for (int py = 0; py < 3; py++) {
        const double gxy = g * (Tx[px] * Ty[py]);
#pragma unroll
        for (int pz = 0; pz < 3; pz++) {
          if (px == 1 && py == 1 && pz == 1) continue;
          acc[t++] += gxy * Tz[pz];
        }
      }
  }
  // warp reduce then across the (up to 8) warps of the block
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < 26; t++) {
    double v = acc[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[t][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 26) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[threadIdx.x][w];
    atomicAdd(&S26[threadIdx.x], v);
  }
}

// b_d(m') = pi m'_d mesh / L^4 * S(m'), zero where m'_d == 0 or alpha == 0
// (p3m-ad-self-forces.c:79-88, layout of Init_self_forces :98-106, and the
// early return of the ad influence function at alpha == 0,
// p3m-ad.c:120-123); one thread per coefficient, grid.y = alpha index.
__global__ void self_coeff_kernel(const double *__restrict__ S26, const double *__restrict__ alphas, int m, double L,
                                  double *__restrict__ b81) {
  const int t = threadIdx.x;
  if (t >= 81) return;
  const int y = blockIdx.y;
  const int ind = t / 3, d = t % 3;
  const int a0 = ind / 9 - 1, a1 = (ind / 3) % 3 - 1, a2 = ind % 3 - 1;
  const int mm[3] = {a0, a1, a2};
  const bool zero = (a0 == 0 && a1 == 0 && a2 == 0);
  const int slot = ind - (ind > 13 ? 1 : 0);  // the 26 sums skip m' = 0 (index 13)
  const double L4 = (L * L) * (L * L);
  double v = 0.0;
  if (!zero && mm[d] != 0 && alphas[y] != 0.0) v = (P3MG_PI * mm[d] * m) / L4 * S26[26 * y + slot];
  b81[81 * y + t] = v;
}

}  // namespace

// The self-force sums of na G meshes (G_all, M apart) into S26 (26 na
// doubles, zeroed here): per-axis factors (self_axis_kernel) into the
// context's small table, then the folded sum.
int self_force_sums(Ctx *c, const double *G_all, int na, double *S26) {
  const int m = c->mesh, h = m / 2 + 1;
  if (!c->self_R) P3MG_CUDA_TRY(cudaMalloc(&c->self_R, 3 * (P3MG_MAX_MESH / 2 + 1) * sizeof(double)));
  self_axis_kernel<<<(h + 127) / 128, 128, 0, c->stream>>>(c->self_R, m, c->cao);
  P3MG_CUDA_TRY(cudaMemsetAsync(S26, 0, 26 * (size_t)na * sizeof(double), c->stream));
  const int threads = 256;
  const size_t H = (size_t)h * h * h;
  const unsigned blocks = (unsigned)((H + (size_t)threads * SELF_PTS - 1) / ((size_t)threads * SELF_PTS));
  self_force_sum_kernel<<<dim3(blocks, na), threads, 0, c->stream>>>(G_all, c->self_R, m, S26);
  c->launches += 2;
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

// G_opt (and for methods 2 and 7 the self-force coefficients) for na alphas
// at once: G_all holds na meshes, b81_all 81 coefficients per alpha, S26
// is 26 na doubles of scratch.  For mc <= 2 groups of alphas share the
// alpha-independent alias sums (influence_group_kernel: each alpha's G
// equals a single call's to rounding); otherwise the single-alpha kernel
// over grid.y.
int influence_batch(Ctx *c, const double *d_alphas, int na, double *G_all, double *S26, double *b81_all) {
  const int m = c->mesh;
  const size_t M = c->M;
  const int threads = 256;
  const unsigned blocks = (unsigned)((M + threads - 1) / threads);
  const size_t h = (size_t)influence_extent(c->method, m);
  const unsigned gblocks = (unsigned)((h * h * h + threads - 1) / threads);
  const double *A = nullptr, *E = nullptr;
  P3MG_TRY(influence_tables(c, d_alphas, 0.0, na, &A, &E));
  if (na > 1 && c->mc <= 2) {
    const int ab = influence_ab(c->mc);
    const dim3 grid(gblocks, (na + ab - 1) / ab);
    if (c->mc == 0)
      influence_group_kernel<0, influence_ab(0)><<<grid, threads, 0, c->stream>>>(G_all, c->method, m, c->cao,
                                                                                 d_alphas, na, c->L, A, E);
    else if (c->mc == 1)
      influence_group_kernel<1, influence_ab(1)><<<grid, threads, 0, c->stream>>>(G_all, c->method, m, c->cao,
                                                                                 d_alphas, na, c->L, A, E);
    else
      influence_group_kernel<2, influence_ab(2)><<<grid, threads, 0, c->stream>>>(G_all, c->method, m, c->cao,
                                                                                 d_alphas, na, c->L, A, E);
  } else {
    launch_influence(G_all, c->method, m, c->cao, c->mc, 0.0, d_alphas, c->L, nullptr, gblocks, na, threads,
                     c->stream, A, E);
  }
  c->launches++;
  P3MG_CUDA_TRY(cudaGetLastError());
  if (method_self_force(c->method)) {
    P3MG_TRY(self_force_sums(c, G_all, na, S26));
    self_coeff_kernel<<<dim3(1, na), 96, 0, c->stream>>>(S26, d_alphas, m, c->L, b81_all);
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
  } else {
    P3MG_CUDA_TRY(cudaMemsetAsync(b81_all, 0, 81 * (size_t)na * sizeof(double), c->stream));
  }
  return P3MG_OK;
}

// G and dG/dalpha at the context's alpha into G_out / dG_out (M doubles each).
int influence_with_derivative(Ctx *c, double *G_out, double *dG_out) {
  const int threads = 256;
  const size_t h = (size_t)influence_extent(c->method, c->mesh);
  const unsigned gblocks = (unsigned)((h * h * h + threads - 1) / threads);
  const double *A = nullptr, *E = nullptr;
  P3MG_TRY(influence_tables(c, nullptr, c->alpha, 1, &A, &E));
  launch_influence(G_out, c->method, c->mesh, c->cao, c->mc, c->alpha, nullptr, c->L, dG_out, gblocks, 1, threads,
                   c->stream, A, E);
  c->launches++;
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

int influence_compute(Ctx *c, double alpha) {
  const int m = c->mesh;
  const size_t M = c->M;
  const int threads = 256;
  const unsigned blocks = (unsigned)((M + threads - 1) / threads);
  const double *A = nullptr, *E = nullptr;
  P3MG_TRY(influence_tables(c, nullptr, alpha, 1, &A, &E));
  const size_t h = (size_t)influence_extent(c->method, m);
  const unsigned gblocks = (unsigned)((h * h * h + threads - 1) / threads);
  launch_influence(c->G, c->method, m, c->cao, c->mc, alpha, nullptr, c->L, nullptr, gblocks, 1, threads, c->stream, A,
                   E);
  c->launches++;
  P3MG_CUDA_TRY(cudaGetLastError());
  if (c->precision != P3MG_FP64) {
    // FP32 copy of G for the mixed-precision convolution
    P3MG_TRY(g_to_f32(c));
  }
  memset(c->self_b_host, 0, sizeof(c->self_b_host));
  // the ad influence function with alpha == 0 returns before the
  // self-force initialisation (p3m-ad.c:120-123); keep zeros then
  if (method_self_force(c->method) && alpha != 0.0) {
    double *S26 = c->self_b;  // use the first 26 slots as the accumulator
    P3MG_TRY(self_force_sums(c, c->G, 1, S26));
    double S[26];
    P3MG_CUDA_TRY(cudaMemcpyAsync(S, S26, sizeof(S), cudaMemcpyDeviceToHost, c->stream));
    P3MG_CUDA_TRY(cudaStreamSynchronize(c->stream));
    // b_d(m') = pi m'_d mesh / L^4 * S(m'), zero where m'_d == 0
    // (p3m-ad-self-forces.c:79-88, layout of Init_self_forces :98-106)
    const double L4 = (c->L * c->L) * (c->L * c->L);
    int ind = 0, t = 0;
    for (int a0 = -1; a0 <= 1; a0++)
      for (int a1 = -1; a1 <= 1; a1++)
        for (int a2 = -1; a2 <= 1; a2++) {
          const int mm[3] = {a0, a1, a2};
          const bool zero = (a0 == 0 && a1 == 0 && a2 == 0);
          for (int d = 0; d < 3; d++)
            c->self_b_host[ind++] = (zero || mm[d] == 0) ? 0.0 : (P3MG_PI * mm[d] * m) / L4 * S[t];
          if (!zero) t++;
        }
  }
  c->alpha = alpha;
  P3MG_CUDA_TRY(cudaMemcpyAsync(c->self_b, c->self_b_host, 81 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  // the step's kernels read alpha from the device, so a captured step stays
  // valid when the influence function is recomputed for another alpha
  P3MG_CUDA_TRY(cudaMemcpyAsync(c->d_alpha, &c->alpha, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  P3MG_CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->have_G = true;
  return P3MG_OK;
}

}  // namespace p3mg

// ---------------------------------------------------------------------------
// Analytic error estimates (the reference's method.Error / method.Error_k):
//   k space  2 q2 sqrt(he / N) / L^2 with he a sum over the mesh vectors
//            n in [-m/2, m/2)^3 of aliasing sums over |m'| <= mc_est:
//     ik, ik-r  p3m-ik.c:264-336     he = |-1 + sum_{n!=0} a1 - (a2/cs)^2/n^2|
//     ik-i      p3m-ik-i.c:249-318   he = |sum_{n!=0} a1 - a2^2/(n^2/2 (a3^2 + a4^2))|
//     ad, ad-r  p3m-ad.c:436-497     he =  sum_{all n_d!=0} a1 - a2^2/(a3 a4)
//     ad-i      p3m-ad-i.c:205-284   he = |sum_{all n_d!=0} a1 - a2^2/(a3 a4/2 + a5 a6/2)|
//   (the ik estimate starts from the table-miss value -1, and the ad sums
//   skip every vector with a zero component, as the reference does);
//   real space  2 q2 exp(-(rcut alpha)^2) / sqrt(N rcut L^3)  (realpart.c:343-346).
// The reference substitutes interpolated tables (find_error.c:84-107) for
// ik/ik-i at tabulated (mesh, cao); these are the sums the tables hold.
// ---------------------------------------------------------------------------

namespace p3mg {
namespace {

__device__ __forceinline__ double cot_sum(int nn, double mi, int cao) {
  // closed form of sum over aliases of sinc^(2 cao) (p3m-common.c:77-107)
  const double c0 = cos(P3MG_PI * mi * (double)nn);
  const double c = c0 * c0;
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

__global__ void kspace_error_kernel(int method, int m, int cao, int mc, double alpha, double L, double *__restrict__ he) {
  __shared__ double red[8];
  const size_t M = (size_t)m * m * m;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double contrib = 0.0;
  if (t < M) {
    const int h = m / 2;
    const int nx = (int)(t / ((size_t)m * m)) - h, ny = (int)((t / m) % m) - h, nz = (int)(t % m) - h;
    const bool ad = method_ad(method);
    const bool any = (nx != 0) || (ny != 0) || (nz != 0);
    const bool all = (nx != 0) && (ny != 0) && (nz != 0);
    if (ad ? all : any) {
      const double mi = 1.0 / m;
      const double f1 = (P3MG_PI / (alpha * L)) * (P3MG_PI / (alpha * L));
      double a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0;
      for (int mx = -mc; mx <= mc; mx++)
        for (int my = -mc; my <= mc; my++)
          for (int mz = -mc; mz <= mc; mz++) {
            const double nmx = nx + mx * m, nmy = ny + my * m, nmz = nz + mz * m;
            const double nm2 = nmx * nmx + nmy * nmy + nmz * nmz;
            const double ex = exp(-f1 * nm2);
            const double sx = sinc_pi(mi * nmx), sy = sinc_pi(mi * nmy), sz = sinc_pi(mi * nmz);
            const double U2 = ipow_d(sx * sy * sz, 2 * cao);
            const bool even = ((mx + my + mz) % 2) == 0;
            a1 += ex * ex / nm2;
            if (ad) {
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
      const double n2 = (double)(nx * nx + ny * ny + nz * nz);
      if (method == 0 || method == 6) {
        const double cs = cot_sum(nx, mi, cao) * cot_sum(ny, mi, cao) * cot_sum(nz, mi, cao);
        contrib = a1 - (a2 / cs) * (a2 / cs) / n2;
      } else if (method == 1) {
        contrib = a1 - a2 * a2 / (0.5 * n2 * (a3 * a3 + a4 * a4));
      } else if (method == 3) {
        contrib = a1 - a2 * a2 / (0.5 * (a3 * a4 + a5 * a6));
      } else if (a3 != 0.0 && a4 != 0.0) {
        contrib = a1 - a2 * a2 / (a3 * a4);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) contrib += __shfl_xor_sync(0xffffffffu, contrib, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = contrib;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
    atomicAdd(he, s);
  }
}

}  // namespace

// Mesh sizes the reference ships precomputed k-space error tables for
// (q.c:1, 83 sizes): the even 13-smooth sizes 4..300 except 286 = 2*11*13,
// plus 360, 400, 480 and 512.
bool estimate_table_mesh(int m) {
  if (m == 360 || m == 400 || m == 480 || m == 512) return true;
  if (m < 4 || m > 300 || (m % 2) || (m % 143) == 0) return false;
  int r = m;
  for (int p : {2, 3, 5, 7, 11, 13})
    while (r % p == 0) r /= p;
  return r == 1;
}

// Analytic error estimates (Error / Error_k / Realspace_error of the method
// table).  ik (0, 6) and ik-i (1) first look alpha*L up in precomputed
// tables (p3m-ik.c:267, p3m-ik-i.c:301, find_error.c:84-107): for a
// tabulated mesh, cao 1..7 and alpha*L <= 100 the reference interpolates
// linearly between table values at alpha*L = 0, 1, ..., 100, which are the
// mesh sum at those points with mc_est = 0 (ik) or 1 (ik-i).  Here the sum
// is evaluated at the two bracketing grid points instead of reading a table.
// On a miss ik starts its sum from the lookup's -1 (p3m-ik.c:266-291).
int error_estimates(int method, int m, int cao, int n, double L, double q2, double alpha, double rcut, int mc_est,
                    cudaStream_t stream, long long *launches, double est[3]) {
  const size_t M = (size_t)m * m * m;
  const double aL = alpha * L;
  const bool ik = (method == 0 || method == 6);
  const bool table = (ik || method == 1) && estimate_table_mesh(m) && cao >= 1 && cao <= 7 && aL <= 100.0;
  const int l = table ? (int)floor(aL) : 0;
  const double d = table ? aL - l : 0.0;
  const int nsum = (table && d != 0.0) ? 2 : 1;
  double *d_he = nullptr;
  P3MG_CUDA_TRY(cudaMalloc(&d_he, 2 * sizeof(double)));
  cudaError_t e = cudaMemsetAsync(d_he, 0, 2 * sizeof(double), stream);
  for (int s = 0; s < nsum && e == cudaSuccess; s++) {
    const double a = table ? (double)(l + s) / L : alpha;
    const int mc = table ? (ik ? 0 : 1) : mc_est;
    kspace_error_kernel<<<(unsigned)((M + 255) / 256), 256, 0, stream>>>(method, m, cao, mc, a, L, d_he + s);
    if (launches) ++*launches;
    e = cudaGetLastError();
  }
  double he2[2] = {0.0, 0.0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(he2, d_he, sizeof(he2), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  cudaFree(d_he);
  if (e != cudaSuccess) {
    record_cuda_error(e);
    return P3MG_ERR_CUDA;
  }
  double he;
  if (table) {
    he = (1.0 - d) * fabs(he2[0]) + ((nsum == 2) ? d * fabs(he2[1]) : 0.0);
  } else {
    he = he2[0];
    if (ik) he -= 1.0;
    if (method != 2 && method != 7) he = fabs(he);
  }
  const double ek = (n > 0) ? 2.0 * q2 * sqrt(he / (double)n) / (L * L) : 0.0;
  const double er = (n > 0 && rcut > 0.0) ? (2.0 * q2 * exp(-(rcut * alpha) * (rcut * alpha))) /
                                                sqrt((double)n * rcut * L * L * L)
                                          : 0.0;
  est[0] = sqrt(er * er + ek * ek);
  est[1] = ek;
  est[2] = er;
  return P3MG_OK;
}

}  // namespace p3mg
