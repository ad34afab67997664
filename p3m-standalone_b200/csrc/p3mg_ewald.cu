// FP64 Ewald reference forces on the GPU -- the oracle every P3M result is
// measured against (Calculate_reference_forces, common.c:329-363):
//   real space: the erfc pair sum with rcut = 0.49 L over all sources;
//   k space:    F_i = q_i sum_{n != 0, |n| <= kmax} n g(n) Im(e^{i k.r_i} S(k)^*)
//               with S(k) = sum_j q_j e^{-i k.r_j}, k = 2 pi n / L,
//               g(n) = 2/L^2 exp(-(pi |n| / (alpha L))^2) / |n|^2
//   (Ewald_k_space, ewald.c:122-166; influence ewald.c:84-109).
// alpha comes from the reference's bisection of the real- and k-space
// error estimates (ewald.c:204-229, with the caller's P3M mesh as kmax, as
// the driver passes its own parameters, common.c:337-339) and kmax grows
// 2, 4, ... until the estimate is <= 1e-8 (common.c:341-344).  g keeps the
// reference's double initialisation: cutoff (kmax-1)^2 except for vectors
// with a component equal to kmax, which keep cutoff kmax^2
// (p3m-common.c:218, common.c:352).
//
// Forces are evaluated on a subset of target particles (all particles when
// the subset is the whole system).  Structure factors: one CTA per
// (k_x, k_y) column of the half space and chunk of k_z; each thread walks a
// slice of the sources, forms e^{-i(k_x x + k_y y)} and the k_z chain by
// repeated multiplication with e^{-i 2 pi z / L}, and the CTA reduces.  The
// k <-> -k symmetry (S(-k) = S(k)^*) gives the other half.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#include "p3mg_internal.cuh"

namespace p3mg {

namespace {

constexpr int EW_THREADS = 256;
constexpr int EW_KZC = 16;  // k_z values per CTA

// shell: the reference-force quirk above (cutoff (kmax-1)^2 except on the
// outer faces); otherwise the plain spherical cutoff kmax^2.
__device__ __forceinline__ double ewald_ghat(int ax, int ay, int az, int kmax, bool shell, double fak1, double fak2) {
  const int n2 = ax * ax + ay * ay + az * az;
  const int cut = (!shell || ax == kmax || ay == kmax || az == kmax) ? kmax * kmax : (kmax - 1) * (kmax - 1);
  if (n2 == 0 || n2 > cut) return 0.0;
  return fak1 / n2 * exp(-fak2 * n2);
}

// S(k) for the half-space columns: column c = (kx, ky), k_z chunk z0..z0+KZC.
// Output S[(c * nz + iz)] = (Re, Im) with iz = kz + kmax.
__global__ void __launch_bounds__(EW_THREADS) ewald_sk_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                                               const double *__restrict__ z, const double *__restrict__ q,
                                                               int n, double twopi_L, const int2 *__restrict__ cols,
                                                               int kmax, double2 *__restrict__ S) {
  __shared__ double2 red[EW_THREADS / 32][EW_KZC];
  const int c = blockIdx.x;
  const int2 col = cols[c];
  const int nz = 2 * kmax + 1;
  const int z0 = -kmax + blockIdx.y * EW_KZC;
  const int zc = min(EW_KZC, kmax + 1 - z0);  // k_z in [z0, z0 + zc)
  double re[EW_KZC], im[EW_KZC];
#pragma unroll
  for (int t = 0; t < EW_KZC; t++) re[t] = im[t] = 0.0;
  for (int j = threadIdx.x; j < n; j += EW_THREADS) {
    const double qj = q[j];
    double s, cxy, sz, cz;
    // e^{-i (kx x + ky y)}
    sincos(twopi_L * ((double)col.x * x[j] + (double)col.y * y[j]), &s, &cxy);
    double br = qj * cxy, bi = -qj * s;
    // e^{-i z0 kz' z} start and the step e^{-i 2 pi z / L}
    sincos(twopi_L * (double)z0 * z[j], &sz, &cz);
    double er = br * cz + bi * sz, ei = bi * cz - br * sz;
    sincos(twopi_L * z[j], &sz, &cz);
#pragma unroll
    for (int t = 0; t < EW_KZC; t++) {
      if (t < zc) {
        re[t] += er;
        im[t] += ei;
        const double nr = er * cz + ei * sz;
        ei = ei * cz - er * sz;
        er = nr;
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < EW_KZC; t++) {
    double a = re[t], b = im[t];
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if (lane == 0) red[warp][t] = make_double2(a, b);
  }
  __syncthreads();
  if (threadIdx.x < zc) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < EW_THREADS / 32; w++) {
      a += red[w][threadIdx.x].x;
      b += red[w][threadIdx.x].y;
    }
    S[(size_t)c * nz + (z0 + kmax + threadIdx.x)] = make_double2(a, b);
  }
}

// S(k) *= 2 g(k) in place: the influence weight of each k vector (0 where
// the cutoff drops it), doubled for the mirrored half space.  Applied once
// here instead of once per target.
__global__ void ewald_weight_kernel(const int2 *__restrict__ cols, int ncol, int kmax, bool shell, double fak1,
                                    double fak2, double2 *__restrict__ S) {
  const int nz = 2 * kmax + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ncol * nz) return;
  const int2 col = cols[t / nz];
  const int kz = t % nz - kmax;
  const double g = 2.0 * ewald_ghat(abs(col.x), abs(col.y), abs(kz), kmax, shell, fak1, fak2);
  const double2 s = S[t];
  S[t] = make_double2(g * s.x, g * s.y);
}

// k-space force on each target from the weighted half-space structure
// factors 2 g(k) S(k).  For k and -k the contributions are equal, so the
// half space counts twice (the k_x = 0, k_y = 0 column holds both k_z and
// -k_z already).
__global__ void ewald_kforce_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                    const double *__restrict__ z, const double *__restrict__ q,
                                    const int *__restrict__ tgt, int nt, double twopi_L, const int2 *__restrict__ cols,
                                    int ncol, int kmax, const double2 *__restrict__ S, double *__restrict__ fk) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int i = tgt ? tgt[t] : t;
  const double xi = x[i], yi = y[i], zi = z[i], qi = q[i];
  const int nz = 2 * kmax + 1;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  double sz1, cz1;
  sincos(twopi_L * zi, &sz1, &cz1);
  for (int c = 0; c < ncol; c++) {
    const int2 col = cols[c];
    const int kx = col.x, ky = col.y;
    const int kz_hi = (int)floor(sqrt((double)(kmax * kmax - kx * kx - ky * ky)) + 1e-9);
    const bool axis = (kx == 0 && ky == 0);
    const int kz_lo = axis ? 1 : -kz_hi;
    // e^{+i k.r} along the column by recurrence in kz
    double s, cxy, sz, cz;
    sincos(twopi_L * ((double)kx * xi + (double)ky * yi), &s, &cxy);
    sincos(twopi_L * (double)kz_lo * zi, &sz, &cz);
    double er = cxy * cz - s * sz, ei = s * cz + cxy * sz;
    for (int kz = kz_lo; kz <= kz_hi; kz++) {
      const double2 sk = S[(size_t)c * nz + (kz + kmax)];
      // q_i g (rhohat_re sin(k.r_i) + rhohat_im cos(k.r_i)), rhohat = S
      // (ewald.c:160-161), with 2 g already in sk
      const double ff = qi * (ei * sk.x + er * sk.y);
      fx += kx * ff;
      fy += ky * ff;
      fz += kz * ff;
      const double nr = er * cz1 - ei * sz1;
      ei = ei * cz1 + er * sz1;
      er = nr;
    }
  }
  fk[t] += fx;
  fk[(size_t)nt + t] += fy;
  fk[2 * (size_t)nt + t] += fz;
}

// Real-space erfc forces on the targets from all sources (rcut 0.49 L), the
// reference's pair formula and minimum-image rounding (realpart.c:137-165).
// grid.y splits the sources into slices; partial sums are added atomically.
__global__ void __launch_bounds__(256) ewald_real_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                                          const double *__restrict__ z, const double *__restrict__ q,
                                                          int n, const int *__restrict__ tgt, int nt, double L,
                                                          double rcut, double alpha, int slice,
                                                          double *__restrict__ fr) {
  __shared__ double4 sj[256];
  const int js = blockIdx.y * slice, je = min(n, js + slice);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = t < nt;
  const int i = act ? (tgt ? tgt[t] : t) : -1;
  const double Li = 1.0 / L;
  const double pref = 2.0 * alpha / 1.77245385090551602729816748334;
  double4 pi = act ? make_double4(x[i], y[i], z[i], q[i]) : make_double4(0, 0, 0, 0);
  double fx = 0, fy = 0, fz = 0;
  for (int jb = js; jb < je; jb += 256) {
    __syncthreads();
    const int jj = jb + threadIdx.x;
    if (jj < je) sj[threadIdx.x] = make_double4(x[jj], y[jj], z[jj], q[jj]);
    __syncthreads();
    const int cnt = min(256, je - jb);
    if (act)
      for (int u = 0; u < cnt; u++) {
        if (jb + u == i) continue;
        const double4 pj = sj[u];
        double dx = __dadd_rn(pi.x, -pj.x);
        dx = __dadd_rn(dx, -__dmul_rn(round(__dmul_rn(dx, Li)), L));
        double dy = __dadd_rn(pi.y, -pj.y);
        dy = __dadd_rn(dy, -__dmul_rn(round(__dmul_rn(dy, Li)), L));
        double dz = __dadd_rn(pi.z, -pj.z);
        dz = __dadd_rn(dz, -__dmul_rn(round(__dmul_rn(dz, Li)), L));
        const double r = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
        if (r <= rcut) {
          const double ar = alpha * r;
          const double fak = pi.w * pj.w * (erfc(ar) / r + pref * exp(-ar * ar)) / (r * r);
          fx += fak * dx;
          fy += fak * dy;
          fz += fak * dz;
        }
      }
  }
  if (act) {
    atomicAdd(&fr[t], fx);
    atomicAdd(&fr[(size_t)nt + t], fy);
    atomicAdd(&fr[2 * (size_t)nt + t], fz);
  }
}

// error estimates of the Ewald sum (ewald.c:175-202)
double err_r(double q2, double L, double rcut, double a) {
  return q2 * sqrt(rcut / (2.0 * L * L * L)) * exp(-a * a * rcut * rcut) / (a * a * rcut * rcut);
}
double err_k(double q2, int n, double L, int kmax, double a) {
  const double t = P3MG_PI * kmax / (a * L);
  return 2.0 * q2 * a / L * sqrt(1.0 / (P3MG_PI * kmax * n)) * exp(-t * t);
}

}  // namespace

// estimated RMS force error of the Ewald sum with real-space cutoff rcut
// (Ewald_estimate_error, ewald.c:199-201)
double ewald_error(int n, double q2, double L, double rcut, int kmax, double alpha) {
  const double r = err_r(q2, L, rcut, alpha), k = err_k(q2, n, L, kmax, alpha);
  return sqrt(r * r + k * k);
}

// alpha and kmax of the reference Ewald sum (see the file comment)
int ewald_parameters(int n, double q2, double L, int mesh_param, double *alpha, int *kmax) {
  const double rcut = 0.49 * L;
  double lo = 0.01, hi = 10.0;
  const double flo = err_r(q2, L, rcut, lo) - err_k(q2, n, L, mesh_param, lo);
  const double fhi = err_r(q2, L, rcut, hi) - err_k(q2, n, L, mesh_param, hi);
  if (flo * fhi > 0.0) return P3MG_ERR_ARG;
  do {
    const double g = 0.5 * (lo + hi);
    const double fg = err_r(q2, L, rcut, g) - err_k(q2, n, L, mesh_param, g);
    if (flo * fg < 0.0)
      hi = g;
    else
      lo = g;
  } while (fabs(lo - hi) > 1.0e-10);
  const double a = 0.5 * (lo + hi);
  int k = 2;
  while (sqrt(err_r(q2, L, rcut, a) * err_r(q2, L, rcut, a) + err_k(q2, n, L, k, a) * err_k(q2, n, L, k, a)) > 1e-8) {
    k += 2;
    if (k > 4096) return P3MG_ERR_ARG;  // the estimate cannot reach the precision (real-space term too large)
  }
  *alpha = a;
  *kmax = k;
  return P3MG_OK;
}

// Ewald forces on nt targets (device index array or NULL for all).
// d_fk (may be NULL): k-space forces, 3 nt doubles (x block, y block, z
// block), overwritten.  d_out (may be NULL): total forces, k space plus the
// real-space sum with cutoff rcut_real (none if rcut_real <= 0), overwritten.
int ewald_forces(Ctx *c, int nt, const int *d_tgt, double alpha, int kmax, bool shell, double rcut_real,
                 double *d_out, double *d_fk) {
  const int n = c->n;
  const double L = c->L;
  const double twopi_L = 2.0 * P3MG_PI / L;
  const double fak1 = 2.0 / (L * L);
  const double pa = P3MG_PI / (alpha * L);
  const double fak2 = pa * pa;
  // half-space columns (kx, ky): kx > 0, or kx == 0 and ky >= 0
  std::vector<int2> cols;
  for (int kx = 0; kx <= kmax; kx++)
    for (int ky = -kmax; ky <= kmax; ky++) {
      if (kx == 0 && ky < 0) continue;
      if (kx * kx + ky * ky > kmax * kmax) continue;
      cols.push_back(make_int2(kx, ky));
    }
  const int ncol = (int)cols.size();
  const int nz = 2 * kmax + 1;
  int2 *d_cols = nullptr;
  double2 *d_S = nullptr;
  P3MG_CUDA_TRY(cudaMalloc(&d_cols, sizeof(int2) * ncol));
  cudaError_t e = cudaMalloc(&d_S, sizeof(double2) * (size_t)ncol * nz);
  if (e != cudaSuccess) {
    cudaFree(d_cols);
    record_cuda_error(e);
    return P3MG_ERR_ALLOC;
  }
  int st = P3MG_OK;
  do {
    e = cudaMemcpyAsync(d_cols, cols.data(), sizeof(int2) * ncol, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_S, 0, sizeof(double2) * (size_t)ncol * nz, c->stream);
    double *kout = d_fk ? d_fk : d_out;
    const size_t bytes = sizeof(double) * 3 * (size_t)nt;
    if (e == cudaSuccess && d_fk) e = cudaMemsetAsync(d_fk, 0, bytes, c->stream);
    if (e == cudaSuccess && d_out) e = cudaMemsetAsync(d_out, 0, bytes, c->stream);
    if (e != cudaSuccess) break;
    if (n > 0 && kout) {
      dim3 grid(ncol, (nz + EW_KZC - 1) / EW_KZC);
      ewald_sk_kernel<<<grid, EW_THREADS, 0, c->stream>>>(c->x, c->y, c->z, c->q, n, twopi_L, d_cols, kmax, d_S);
      ewald_weight_kernel<<<(ncol * nz + 255) / 256, 256, 0, c->stream>>>(d_cols, ncol, kmax, shell, fak1, fak2, d_S);
      ewald_kforce_kernel<<<(nt + 127) / 128, 128, 0, c->stream>>>(c->x, c->y, c->z, c->q, d_tgt, nt, twopi_L, d_cols,
                                                                   ncol, kmax, d_S, kout);
      c->launches += 3;
      if (d_fk && d_out) e = cudaMemcpyAsync(d_out, d_fk, bytes, cudaMemcpyDeviceToDevice, c->stream);
      if (e == cudaSuccess) e = cudaGetLastError();
      if (e != cudaSuccess) break;
    }
    if (n > 0 && d_out && rcut_real > 0.0) {
      // enough CTAs for the whole GPU: split the sources into slices
      const int tb = (nt + 255) / 256;
      int nsplit = (4 * 148 + tb - 1) / tb;
      nsplit = nsplit < 1 ? 1 : nsplit;
      const int slice = (n + nsplit - 1) / nsplit;
      nsplit = (n + slice - 1) / slice;
      ewald_real_kernel<<<dim3(tb, nsplit), 256, 0, c->stream>>>(c->x, c->y, c->z, c->q, n, d_tgt, nt, L, rcut_real,
                                                                 alpha, slice, d_out);
      c->launches += 1;
      e = cudaGetLastError();
      if (e != cudaSuccess) break;
    }
    e = cudaStreamSynchronize(c->stream);
  } while (0);
  if (e != cudaSuccess) {
    record_cuda_error(e);
    st = P3MG_ERR_CUDA;
  }
  cudaFree(d_cols);
  cudaFree(d_S);
  return st;
}

}  // namespace p3mg
