// Templated kernels and launchers of the k-space pipeline (included by
// p3mg_assign_f64.cu and p3mg_assign_f32.cu, one precision each).
#pragma once
#include <math.h>

#include "p3mg_internal.cuh"

namespace p3mg {
namespace assign_impl {
namespace {

constexpr int ASSIGN_THREADS = 256;

__host__ __device__ inline int brick_tile(int B, int cao, int nmesh) { return B + cao - 1 + (nmesh == 2 ? 1 : 0); }

// ---------------------------------------------------------------- scatter

template <typename real, int CAO, int NMESH>
__global__ void __launch_bounds__(ASSIGN_THREADS) scatter_kernel(const double4 *__restrict__ sxyzq,
                                                                  const int *__restrict__ start, int m, int B, int nb,
                                                                  double Hi, double shift,
                                                                  typename cplx<real>::type *__restrict__ Q) {
  extern __shared__ unsigned char smem_raw[];
  real *tile0 = reinterpret_cast<real *>(smem_raw);
  const int T = brick_tile(B, CAO, NMESH);
  const int T3 = T * T * T;
  real *tile1 = tile0 + T3;
  const int bid = blockIdx.x;
  const int p0 = start[bid], p1 = start[bid + 1];
  if (p0 == p1) return;
  for (int t = threadIdx.x; t < NMESH * T3; t += blockDim.x) tile0[t] = (real)0;
  __syncthreads();
  const int bz = bid % nb, by = (bid / nb) % nb, bx = bid / (nb * nb);
  const int o0 = bx * B, o1 = by * B, o2 = bz * B;
  for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
    const double4 r = sxyzq[p];
    const real qp = (real)r.w;
#pragma unroll
    for (int ii = 0; ii < NMESH; ii++) {
      int base[3], arg[3];
      mesh_geometry(r.x, Hi, shift, ii, m, &base[0], &arg[0]);
      mesh_geometry(r.y, Hi, shift, ii, m, &base[1], &arg[1]);
      mesh_geometry(r.z, Hi, shift, ii, m, &base[2], &arg[2]);
      int rel0 = base[0] - o0, rel1 = base[1] - o1, rel2 = base[2] - o2;
      rel0 += (rel0 < 0) ? m : 0;
      rel1 += (rel1 < 0) ? m : 0;
      rel2 += (rel2 < 0) ? m : 0;
      real wx[CAO], wy[CAO], wz[CAO];
      bspline_weights<real, CAO, false>(arg[0], wx, nullptr);
      bspline_weights<real, CAO, false>(arg[1], wy, nullptr);
      bspline_weights<real, CAO, false>(arg[2], wz, nullptr);
      real *tile = ii ? tile1 : tile0;
#pragma unroll
      for (int a = 0; a < CAO; a++) {
        const real qa = qp * wx[a];
#pragma unroll
        for (int b = 0; b < CAO; b++) {
          const real qab = qa * wy[b];
          real *row = tile + ((rel0 + a) * T + (rel1 + b)) * T + rel2;
#pragma unroll
          for (int c = 0; c < CAO; c++) atomicAdd(row + c, qab * wz[c]);
        }
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < T3; t += blockDim.x) {
    const int c = t % T, b = (t / T) % T, a = t / (T * T);
    int gi = o0 + a, gj = o1 + b, gk = o2 + c;
    gi -= (gi >= m) ? m : 0;
    gj -= (gj >= m) ? m : 0;
    gk -= (gk >= m) ? m : 0;
    if (gi >= m) gi %= m;
    if (gj >= m) gj %= m;
    if (gk >= m) gk %= m;
    const size_t g = ((size_t)gi * m + gj) * m + gk;
    const real v0 = tile0[t];
    if (v0 != (real)0) atomicAdd(&Q[g].x, v0);
    if (NMESH == 2) {
      const real v1 = tile1[t];
      if (v1 != (real)0) atomicAdd(&Q[g].y, v1);
    }
  }
}

// ------------------------------------------------------------ convolution

__device__ __forceinline__ double dn_op(int i, int m) {
  // Dn[i] = i - round(i/m) m with Dn[m/2] = 0 (p3m-common.c:110-131)
  return (i == m / 2) ? 0.0 : (double)i - round((double)i / (double)m) * (double)m;
}

template <typename real, typename Gt>
__global__ void conv_ik_kernel(const typename cplx<real>::type *__restrict__ Q, const Gt *__restrict__ G, int m,
                               double twopi_over_L, size_t M, typename cplx<real>::type *__restrict__ F) {
  typedef typename cplx<real>::type C;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M) return;
  const int k = (int)(t % m), j = (int)((t / m) % m), i = (int)(t / ((size_t)m * m));
  const C qv = Q[t];
  const real g = (real)G[t];
  const real s = (real)twopi_over_L;
  const real qr = qv.x * g * s, qi = qv.y * g * s;
  const real d0 = (real)dn_op(i, m), d1 = (real)dn_op(j, m), d2 = (real)dn_op(k, m);
  C f;
  f.x = -d0 * qi;
  f.y = d0 * qr;
  F[t] = f;
  f.x = -d1 * qi;
  f.y = d1 * qr;
  F[M + t] = f;
  f.x = -d2 * qi;
  f.y = d2 * qr;
  F[2 * M + t] = f;
}

template <typename real, typename Gt>
__global__ void conv_ad_kernel(typename cplx<real>::type *__restrict__ Q, const Gt *__restrict__ G, size_t M) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M) return;
  const real g = (real)G[t];
  typename cplx<real>::type v = Q[t];
  v.x *= g;
  v.y *= g;
  Q[t] = v;
}

// ---------------------------------------------------------------- gather

// ik: f_d -= scale * q W F_d ; ad: f -= scale * phi * q/L * grad W.
// scale = pref (one mesh) or pref/2 (interlaced, charge-assign.c:646-806).
template <typename real, int CAO, int NMESH, bool AD>
__global__ void __launch_bounds__(ASSIGN_THREADS) gather_kernel(const double4 *__restrict__ sxyzq,
                                                                 const int *__restrict__ sidx, int np, int m,
                                                                 double Hi, double shift, double pref, double Leni,
                                                                 const typename cplx<real>::type *__restrict__ F,
                                                                 size_t M, double *__restrict__ fk, int n) {
  typedef typename cplx<real>::type C;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const double4 r = sxyzq[p];
  const real scale = (real)((NMESH == 2) ? 0.5 * pref : pref);
  real acc0 = 0, acc1 = 0, acc2 = 0;
#pragma unroll
  for (int ii = 0; ii < NMESH; ii++) {
    int base[3], arg[3];
    mesh_geometry(r.x, Hi, shift, ii, m, &base[0], &arg[0]);
    mesh_geometry(r.y, Hi, shift, ii, m, &base[1], &arg[1]);
    mesh_geometry(r.z, Hi, shift, ii, m, &base[2], &arg[2]);
    real wx[CAO], wy[CAO], wz[CAO], dx[CAO], dy[CAO], dz[CAO];
    bspline_weights<real, CAO, AD>(arg[0], wx, dx);
    bspline_weights<real, CAO, AD>(arg[1], wy, dy);
    bspline_weights<real, CAO, AD>(arg[2], wz, dz);
    const real qp = (real)r.w;
    const real qL = (real)(r.w * Leni);
#pragma unroll
    for (int a = 0; a < CAO; a++) {
      int gi = base[0] + a;
      gi -= (gi >= m) ? m : 0;
#pragma unroll
      for (int b = 0; b < CAO; b++) {
        int gj = base[1] + b;
        gj -= (gj >= m) ? m : 0;
        const size_t rowb = ((size_t)gi * m + gj) * m;
        if (!AD) {
          const real qab = qp * wx[a] * wy[b];
#pragma unroll
          for (int c = 0; c < CAO; c++) {
            int gk = base[2] + c;
            gk -= (gk >= m) ? m : 0;
            const size_t g = rowb + gk;
            const real Bw = scale * (qab * wz[c]);
            const C f0 = F[g], f1 = F[M + g], f2 = F[2 * M + g];
            acc0 -= (ii ? f0.y : f0.x) * Bw;
            acc1 -= (ii ? f1.y : f1.x) * Bw;
            acc2 -= (ii ? f2.y : f2.x) * Bw;
          }
        } else {
#pragma unroll
          for (int c = 0; c < CAO; c++) {
            int gk = base[2] + c;
            gk -= (gk >= m) ? m : 0;
            const C v = F[rowb + gk];
            const real Bp = scale * (ii ? v.y : v.x);
            acc0 -= Bp * (dx[a] * wy[b] * wz[c] * qL);
            acc1 -= Bp * (wx[a] * dy[b] * wz[c] * qL);
            acc2 -= Bp * (wx[a] * wy[b] * dz[c] * qL);
          }
        }
      }
    }
  }
  const int o = sidx[p];
  fk[o] += (double)acc0;
  fk[(size_t)n + o] += (double)acc1;
  fk[2 * (size_t)n + o] += (double)acc2;
}

// ---------------------------------------------------------- self forces

// f_tot,d -= b_d(m') q^2 sin(2 pi (m'.x)/h) for the 27 m' (p3m-ad-self-forces.c:114-139)
__global__ void self_force_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                  const double *__restrict__ z, const double *__restrict__ q, int n, double h,
                                  const double *__restrict__ b81, double *__restrict__ f) {
  __shared__ double b[81];
  if (threadIdx.x < 81) b[threadIdx.x] = b81[threadIdx.x];
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double xi = x[i], yi = y[i], zi = z[i], q2 = q[i] * q[i];
  double s0 = 0, s1 = 0, s2 = 0;
  int t = 0;
  for (int a0 = -1; a0 <= 1; a0++)
    for (int a1 = -1; a1 <= 1; a1++)
      for (int a2 = -1; a2 <= 1; a2++) {
        const double arg = __dadd_rn(__dadd_rn(__ddiv_rn(a0 * xi, h), __ddiv_rn(a1 * yi, h)), __ddiv_rn(a2 * zi, h));
        const double st = q2 * sin(__dmul_rn(2.0 * P3MG_PI, arg));
        s0 += b[t] * st;
        s1 += b[t + 1] * st;
        s2 += b[t + 2] * st;
        t += 3;
      }
  f[i] -= s0;
  f[(size_t)n + i] -= s1;
  f[2 * (size_t)n + i] -= s2;
}

// ---------------------------------------------------------------- launch

template <typename real, int CAO, int NMESH>
int launch_scatter(Ctx *c, size_t smem) {
  typedef typename cplx<real>::type C;
  auto kern = scatter_kernel<real, CAO, NMESH>;
  // raise the dynamic shared-memory limit once per instantiation (outside
  // any graph capture: the first step of a shape always runs eagerly)
  static size_t smem_set = 0;
  if (smem > smem_set) {
    P3MG_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    smem_set = 200 * 1024;
  }
  const double Hi = (double)c->mesh / c->L;
  const double shift = (double)((c->cao - 1) / 2);
  const int nbr = c->nbrick1 * c->nbrick1 * c->nbrick1;
  mark(c, EV_K2);
  kern<<<nbr, ASSIGN_THREADS, smem, c->stream>>>(c->sorted_xyzq, c->brick_start, c->mesh, c->brick, c->nbrick1, Hi,
                                                shift, reinterpret_cast<C *>(c->Q));
  c->launches++;
  mark(c, EV_K3);
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

template <typename real, int CAO>
int dispatch_scatter(Ctx *c) {
  const int nmesh = method_interlaced(c->method) ? 2 : 1;
  const int T = brick_tile(c->brick, CAO, nmesh);
  const size_t smem = (size_t)nmesh * T * T * T * sizeof(real);
  if (nmesh == 2) return launch_scatter<real, CAO, 2>(c, smem);
  return launch_scatter<real, CAO, 1>(c, smem);
}

template <typename real, int CAO>
int dispatch_gather(Ctx *c) {
  typedef typename cplx<real>::type C;
  const double Hi = (double)c->mesh / c->L;
  const double shift = (double)((c->cao - 1) / 2);
  const double L3 = c->L * c->L * c->L;
  const double Leni = 1.0 / c->L;
  const int blocks = (c->n + ASSIGN_THREADS - 1) / ASSIGN_THREADS;
  const bool il = method_interlaced(c->method);
  const C *F = reinterpret_cast<const C *>(method_ad(c->method) ? c->Q : c->F);
  mark(c, EV_K4);
  if (method_ad(c->method)) {
    // prefactor Mesh * Leni^3 (p3m-ad.c:202, p3m-ad-i.c:199, p3m-ad-real.c:110)
    const double pref = (double)c->mesh * Leni * Leni * Leni;
    if (il)
      gather_kernel<real, CAO, 2, true><<<blocks, ASSIGN_THREADS, 0, c->stream>>>(
          c->sorted_xyzq, c->sorted_idx, c->n, c->mesh, Hi, shift, pref, Leni, F, c->M, c->fk, c->n);
    else
      gather_kernel<real, CAO, 1, true><<<blocks, ASSIGN_THREADS, 0, c->stream>>>(
          c->sorted_xyzq, c->sorted_idx, c->n, c->mesh, Hi, shift, pref, Leni, F, c->M, c->fk, c->n);
  } else {
    // prefactor 1 / (2 L^3) (p3m-ik.c:242, p3m-ik-i.c:241, p3m-ik-real.c:144)
    const double pref = 1.0 / (2.0 * L3);
    if (il)
      gather_kernel<real, CAO, 2, false><<<blocks, ASSIGN_THREADS, 0, c->stream>>>(
          c->sorted_xyzq, c->sorted_idx, c->n, c->mesh, Hi, shift, pref, Leni, F, c->M, c->fk, c->n);
    else
      gather_kernel<real, CAO, 1, false><<<blocks, ASSIGN_THREADS, 0, c->stream>>>(
          c->sorted_xyzq, c->sorted_idx, c->n, c->mesh, Hi, shift, pref, Leni, F, c->M, c->fk, c->n);
  }
  c->launches++;
  mark(c, EV_K5);
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

template <typename real>
int run_kspace(Ctx *c) {
  typedef typename cplx<real>::type C;
  const size_t M = c->M;
  const int threads = 256;
  const unsigned mblocks = (unsigned)((M + threads - 1) / threads);
  // charge assignment (the brick binning ran in kspace_prepare)
  P3MG_CUDA_TRY(cudaMemsetAsync(c->Q, 0, M * sizeof(C), c->stream));
  switch (c->cao) {
    case 1: P3MG_TRY((dispatch_scatter<real, 1>(c))); break;
    case 2: P3MG_TRY((dispatch_scatter<real, 2>(c))); break;
    case 3: P3MG_TRY((dispatch_scatter<real, 3>(c))); break;
    case 4: P3MG_TRY((dispatch_scatter<real, 4>(c))); break;
    case 5: P3MG_TRY((dispatch_scatter<real, 5>(c))); break;
    case 6: P3MG_TRY((dispatch_scatter<real, 6>(c))); break;
    case 7: P3MG_TRY((dispatch_scatter<real, 7>(c))); break;
  }
  mark(c, EV_S2);
  // forward FFT, convolution, backward FFT(s)
  P3MG_TRY(fft3d(c, c->Q, 1, -1));
  if (method_ad(c->method)) {
    if (c->precision == P3MG_FP64)
      conv_ad_kernel<real, double><<<mblocks, threads, 0, c->stream>>>(reinterpret_cast<C *>(c->Q), c->G, M);
    else
      conv_ad_kernel<real, float><<<mblocks, threads, 0, c->stream>>>(reinterpret_cast<C *>(c->Q), c->G32, M);
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
    P3MG_TRY(fft3d(c, c->Q, 1, +1));
  } else {
    const double s = 2.0 * P3MG_PI / c->L;
    if (c->precision == P3MG_FP64)
      conv_ik_kernel<real, double><<<mblocks, threads, 0, c->stream>>>(reinterpret_cast<const C *>(c->Q), c->G,
                                                                       c->mesh, s, M, reinterpret_cast<C *>(c->F));
    else
      conv_ik_kernel<real, float><<<mblocks, threads, 0, c->stream>>>(reinterpret_cast<const C *>(c->Q), c->G32,
                                                                      c->mesh, s, M, reinterpret_cast<C *>(c->F));
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
    P3MG_TRY(fft3d(c, c->F, 3, +1));
  }
  mark(c, EV_S3);
  // back-interpolation
  switch (c->cao) {
    case 1: P3MG_TRY((dispatch_gather<real, 1>(c))); break;
    case 2: P3MG_TRY((dispatch_gather<real, 2>(c))); break;
    case 3: P3MG_TRY((dispatch_gather<real, 3>(c))); break;
    case 4: P3MG_TRY((dispatch_gather<real, 4>(c))); break;
    case 5: P3MG_TRY((dispatch_gather<real, 5>(c))); break;
    case 6: P3MG_TRY((dispatch_gather<real, 6>(c))); break;
    case 7: P3MG_TRY((dispatch_gather<real, 7>(c))); break;
  }
  if (method_self_force(c->method)) {
    const int blocks = (c->n + threads - 1) / threads;
    self_force_kernel<<<blocks, threads, 0, c->stream>>>(c->x, c->y, c->z, c->q, c->n, c->L / c->mesh, c->self_b,
                                                          c->f);
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
  }
  mark(c, EV_S4);
  return P3MG_OK;
}

}  // namespace
}  // namespace assign_impl
}  // namespace p3mg
