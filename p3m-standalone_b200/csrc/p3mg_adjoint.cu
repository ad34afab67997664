// Electrostatic energy of the P3M approximation and its hand-written
// adjoint: dE/dx (the negative of the exact forces of this energy), dE/dq
// (the potentials), dE/dalpha and dE/dL.  The reference computes no P3M
// energy, so nothing here has a reference counterpart; the pieces follow
// the force pipeline (charge-assign.c, p3m-ad.c, realpart.c, ewald.c).
//
//   E      = E_k + E_r + E_self + E_neutral
//   E_k    = c/(2 L^3 nmesh) sum_s sum_m Q_s(m) phi_s(m)
//          = c/(2 L^3 nmesh) sum_s sum_k G(k) |Q^_s(k)|^2,
//            phi_s = IFFT(G FFT(Q_s)) (unnormalised transforms), nmesh = 2
//            for the interlaced methods: the unshifted and the half-cell-
//            shifted mesh, whose forces those methods average; c = 1 for
//            the ad influence functions and 1/2 for the ik ones, whose
//            forces carry 1/(2 L^3) (p3m-ik.c:242) where ad carries
//            mesh/L^3 on the derivative of the weights (p3m-ad.c:202)
//   E_r    = 1/2 sum_{i != j, r <= rcut} q_i q_j erfc(alpha r) / r
//   E_self = -alpha / sqrt(pi) sum q^2          (ewald.c:60-62)
//   E_neut = -pi Q^2 / (2 alpha^2 L^3), Q = sum q (zero for neutral systems)
//
// Q_s(m) = sum_i q_i W(x_i - m h) with the charge-assignment B-splines
// evaluated at the exact in-cell offset (not the reference's 2^-17 table
// bins), so E is a smooth function of the positions and
//   dE_k/dx_i = c/(L^3 nmesh) q_i sum_s sum_m phi_s(m) dW/dx_i,
//   dE_k/dq_i = c/(L^3 nmesh) sum_s sum_m phi_s(m) W,
//   dE_k/dalpha = c/(2 L^3 nmesh) sum_k dG/dalpha |Q^(k)|^2.
// For the ad methods dE/dx is minus the ad force (without the self-force
// correction of methods 2 and 7, which is not the gradient of an energy);
// for the ik methods it is the exact gradient of E, not the ik force.
// Every term has the form E(alpha, L) = F(alpha L) / L at fixed fractional
// coordinates, so dE/dL = (alpha dE/dalpha - E) / L (the isotropic virial
// is -L dE/dL).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "p3mg_internal.cuh"

namespace p3mg {

namespace {

constexpr int ADJ_THREADS = 256;

// sum_k G |P^|^2 and sum_k dG |P^|^2 (P^ the packed transform) into acc[0..1]
template <typename real>
__global__ void adj_energy_sums_kernel(const typename cplx<real>::type *__restrict__ P, const double *__restrict__ G,
                                       const double *__restrict__ dG, size_t M, double *__restrict__ acc) {
  __shared__ double red[2][ADJ_THREADS / 32];
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0, de = 0.0;
  if (t < M) {
    const typename cplx<real>::type v = P[t];
    const double p2 = (double)v.x * (double)v.x + (double)v.y * (double)v.y;
    e = G[t] * p2;
    de = dG[t] * p2;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_xor_sync(0xffffffffu, e, o);
    de += __shfl_xor_sync(0xffffffffu, de, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = e;
    red[1][threadIdx.x >> 5] = de;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double s = 0.0;
    for (int w = 0; w < ADJ_THREADS / 32; w++) s += red[threadIdx.x][w];
    atomicAdd(&acc[threadIdx.x], s);
  }
}

// Phi = G P^ (out of place)
template <typename real>
__global__ void adj_conv_kernel(const typename cplx<real>::type *__restrict__ P, const double *__restrict__ G, size_t M,
                                typename cplx<real>::type *__restrict__ Phi) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M) return;
  const real g = (real)G[t];
  typename cplx<real>::type v = P[t];
  v.x *= g;
  v.y *= g;
  Phi[t] = v;
}

__device__ __forceinline__ double adj_min_image(double d, double L) { return d - L * round(d / L); }

// Real space with fewer than 3 cells per side: one thread per particle over
// all particles (the cell-list case runs pairs_cell_kernel's adjoint form).  Accumulates
// gx += -ge f_i, gq += ge phi_i, and acc[0] += E_r, acc[1] += dE_r/dalpha.
template <typename real>
__global__ void __launch_bounds__(ADJ_THREADS) adj_pairs_kernel(const double *__restrict__ x,
                                                                 const double *__restrict__ y,
                                                                 const double *__restrict__ z,
                                                                 const double *__restrict__ q, int n, double L,
                                                                 double rcut, double alpha, int nc,
                                                                 const int *__restrict__ start,
                                                                 const int *__restrict__ cidx, double ge,
                                                                 double *__restrict__ gx, double *__restrict__ gq,
                                                                 double *__restrict__ acc) {
  __shared__ double red[2][ADJ_THREADS / 32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const real twopi = (real)1.12837916709551257389615890312;  // 2 / sqrt(pi)
  const real al = (real)alpha, rc2 = (real)(rcut * rcut);
  double e = 0.0, de = 0.0;
  if (i < n) {
    const double xi = x[i], yi = y[i], zi = z[i];
    const real qi = (real)q[i];
    real fx = 0, fy = 0, fz = 0, ph = 0;
    auto pair = [&](int j) {
      if (j == i) return;
      const real dx = (real)adj_min_image(xi - x[j], L);
      const real dy = (real)adj_min_image(yi - y[j], L);
      const real dz = (real)adj_min_image(zi - z[j], L);
      const real r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > rc2) return;
      const real r = sqrt(r2), ar = al * r;
      const real ec = erfc(ar), gs = exp(-ar * ar);
      const real qj = (real)q[j];
      const real fak = qi * qj * (ec / r + al * twopi * gs) / r2;
      fx += fak * dx;
      fy += fak * dy;
      fz += fak * dz;
      ph += qj * ec / r;
      e += 0.5 * (double)(qi * qj * ec / r);
      de += 0.5 * (double)(qi * qj * (-twopi * gs));
    };
    if (nc == 0) {
      for (int j = 0; j < n; j++) pair(j);
    } else {
      // i's cell as the binning computes it (bin_cells_kernel)
      const double hs = (double)(2 * nc) / L;
      const int c0 = wrap_full((int)floor(xi * hs), 2 * nc) >> 1, c1 = wrap_full((int)floor(yi * hs), 2 * nc) >> 1,
                c2 = wrap_full((int)floor(zi * hs), 2 * nc) >> 1;
      for (int d0 = -1; d0 <= 1; d0++)
        for (int d1 = -1; d1 <= 1; d1++)
          for (int d2 = -1; d2 <= 1; d2++) {
            const int cell = (wrap_full(c0 + d0, nc) * nc + wrap_full(c1 + d1, nc)) * nc + wrap_full(c2 + d2, nc);
            for (int s = start[cell * 8]; s < start[cell * 8 + 8]; s++) pair(cidx[s]);
          }
    }
    gx[i] -= ge * (double)fx;
    gx[(size_t)n + i] -= ge * (double)fy;
    gx[2 * (size_t)n + i] -= ge * (double)fz;
    gq[i] += ge * (double)ph;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_xor_sync(0xffffffffu, e, o);
    de += __shfl_xor_sync(0xffffffffu, de, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = e;
    red[1][threadIdx.x >> 5] = de;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double s = 0.0;
    for (int w = 0; w < ADJ_THREADS / 32; w++) s += red[threadIdx.x][w];
    atomicAdd(&acc[threadIdx.x], s);
  }
}

// sum q and sum q^2 into acc[0..1]
__global__ void charge_sums_kernel(const double *__restrict__ q, int n, double *__restrict__ acc) {
  __shared__ double red[2][ADJ_THREADS / 32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double a = 0.0, b = 0.0;
  if (i < n) {
    a = q[i];
    b = q[i] * q[i];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = a;
    red[1][threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double s = 0.0;
    for (int w = 0; w < ADJ_THREADS / 32; w++) s += red[threadIdx.x][w];
    atomicAdd(&acc[threadIdx.x], s);
  }
}

// self and neutralising terms of dE/dq: ge (-2 alpha/sqrt(pi) q_i - pi Q/(alpha^2 L^3)),
// Q = sum q read from the device sums (sums[4]) so the host need not wait for it
__global__ void adj_self_kernel(const double *__restrict__ q, int n, double c_self, double c_neut_per_Q,
                                const double *__restrict__ sums, double *__restrict__ gq) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) gq[i] += c_self * q[i] + c_neut_per_Q * sums[4];
}

// c of the k-space energy: 1 for ad, 1/2 for ik influence functions
double kspace_factor(const Ctx *c) { return method_ad(c->method) ? 1.0 : 0.5; }

template <typename real>
int adjoint_run(Ctx *c, double rcut, double ge, double *gx, double *gq, double *sums) {
  typedef typename cplx<real>::type C;
  const size_t M = c->M;
  const int nmesh = method_interlaced(c->method) ? 2 : 1;
  const double L = c->L, L3 = L * L * L;
  const unsigned mblocks = (unsigned)((M + ADJ_THREADS - 1) / ADJ_THREADS);
  C *P = reinterpret_cast<C *>(c->Q);
  C *Phi = reinterpret_cast<C *>(c->adj_phi);
  // mesh part: Q (exact weights) -> P^ -> sums of G |P^|^2 and dG |P^|^2
  // charge assignment with exact weights through the brick-tiled scatter
  // of the forces (particles brick-sorted first)
  P3MG_CUDA_TRY(cudaMemsetAsync(P, 0, M * sizeof(C), c->stream));
  if (c->n > 0) {
    P3MG_TRY(kspace_prepare(c));
    P3MG_TRY(adjoint_scatter(c));
  }
  P3MG_TRY(fft3d(c, P, 1, -1));
  // G and dG/dalpha depend only on alpha and L for a context (the mesh,
  // cao and aliasing range are fixed): computed once per (alpha, L), like
  // G_opt for the forces
  if (!(c->adj_key_alpha == c->alpha && c->adj_key_L == c->L)) {
    P3MG_TRY(influence_with_derivative(c, c->adj_G, c->adj_dG));
    c->adj_key_alpha = c->alpha;
    c->adj_key_L = c->L;
  }
  adj_energy_sums_kernel<real><<<mblocks, ADJ_THREADS, 0, c->stream>>>(P, c->adj_G, c->adj_dG, M, sums);
  adj_conv_kernel<real><<<mblocks, ADJ_THREADS, 0, c->stream>>>(P, c->adj_G, M, Phi);
  c->launches += 2;
  P3MG_CUDA_TRY(cudaGetLastError());
  P3MG_TRY(fft3d(c, Phi, 1, +1));
  if (c->n > 0) {
    const double s = kspace_factor(c) / (L3 * nmesh);
    P3MG_TRY(adjoint_gather(c, Phi, s, ge, gx, gq));
  }
  // real space
  if (rcut > 0.0 && c->n > 0) {
    int nc = 0;
    P3MG_TRY(pairs_bin(c, rcut, &nc));
    if (nc >= 3) {
      // the warp-cooperative cell kernel of the forces, with the potential
      // and dE_r/dalpha summed beside the force (pairs_cell_kernel, ADJ)
      P3MG_TRY(pairs_adjoint(c, rcut, nc, ge, gx, gq, sums + 2));
    } else {
      const int blocks = (c->n + ADJ_THREADS - 1) / ADJ_THREADS;
      adj_pairs_kernel<real><<<blocks, ADJ_THREADS, 0, c->stream>>>(c->x, c->y, c->z, c->q, c->n, L, rcut, c->alpha,
                                                                    0, c->cell_start, c->cell_idx, ge, gx, gq,
                                                                    sums + 2);
      c->launches++;
      P3MG_CUDA_TRY(cudaGetLastError());
    }
  }
  // charge sums for the self and neutralising terms
  if (c->n > 0) {
    charge_sums_kernel<<<(c->n + ADJ_THREADS - 1) / ADJ_THREADS, ADJ_THREADS, 0, c->stream>>>(c->q, c->n, sums + 4);
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
  }
  return P3MG_OK;
}

}  // namespace

// Energy parts [total, k-space, real space, self, neutralising] and, with
// ge != 0, ge times the gradients: gx (3 n, device, accumulated), gq (n,
// device, accumulated), dE/dalpha and dE/dL (host, overwritten).
int adjoint(Ctx *c, double rcut, double ge, double *gx, double *gq, double energy[5], double *dalpha, double *dL) {
  if (!c->adj_G) {
    P3MG_CUDA_TRY(cudaMalloc(&c->adj_G, c->M * sizeof(double)));
    P3MG_CUDA_TRY(cudaMalloc(&c->adj_dG, c->M * sizeof(double)));
    const size_t csz = (c->precision == P3MG_FP64) ? sizeof(double2) : sizeof(float2);
    P3MG_CUDA_TRY(cudaMalloc(&c->adj_phi, c->M * csz));
    P3MG_CUDA_TRY(cudaMalloc(&c->adj_sums, 8 * sizeof(double)));
  }
  P3MG_CUDA_TRY(cudaMemsetAsync(c->adj_sums, 0, 8 * sizeof(double), c->stream));
  if (c->precision == P3MG_FP64)
    P3MG_TRY(adjoint_run<double>(c, rcut, ge, gx, gq, c->adj_sums));
  else
    P3MG_TRY(adjoint_run<float>(c, rcut, ge, gx, gq, c->adj_sums));
  const double L = c->L, L3 = L * L * L, a = c->alpha;
  const double sqrtpi = 1.77245385090551602729816748334;
  if (gq && c->n > 0 && ge != 0.0) {
    const double c_self = ge * (-2.0 * a / sqrtpi);
    const double c_neut = (a > 0.0) ? ge * (-P3MG_PI / (a * a * L3)) : 0.0;
    adj_self_kernel<<<(c->n + ADJ_THREADS - 1) / ADJ_THREADS, ADJ_THREADS, 0, c->stream>>>(c->q, c->n, c_self, c_neut,
                                                                                           c->adj_sums, gq);
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
  }
  // the energy parts and dE/dalpha, dE/dL need the device sums: one small
  // copy at the end of the queued work
  double s[8];
  P3MG_CUDA_TRY(cudaMemcpyAsync(s, c->adj_sums, sizeof(s), cudaMemcpyDeviceToHost, c->stream));
  P3MG_CUDA_TRY(cudaStreamSynchronize(c->stream));
  const int nmesh = method_interlaced(c->method) ? 2 : 1;
  const double kf = kspace_factor(c);
  const double Ek = kf * s[0] / (2.0 * L3 * nmesh), dEk = kf * s[1] / (2.0 * L3 * nmesh);
  const double Er = s[2], dEr = s[3];
  const double Qn = s[4], q2 = s[5];
  const double Es = -a / sqrtpi * q2, dEs = -q2 / sqrtpi;
  const double En = (a > 0.0) ? -P3MG_PI * Qn * Qn / (2.0 * a * a * L3) : 0.0;
  const double dEn = (a > 0.0) ? P3MG_PI * Qn * Qn / (a * a * a * L3) : 0.0;
  const double E = Ek + Er + Es + En;
  energy[0] = E;
  energy[1] = Ek;
  energy[2] = Er;
  energy[3] = Es;
  energy[4] = En;
  const double dEa = dEk + dEr + dEs + dEn;
  if (dalpha) *dalpha = ge * dEa;
  if (dL) *dL = ge * (a * dEa - E) / L;
  return P3MG_OK;
}

}  // namespace p3mg
