// k-space pipeline of one P3M step on the GPU:
//   bin particles by mesh brick -> tiled charge assignment (scatter) ->
//   forward FFT -> convolution (ik: three differentiated fields, ad: one
//   potential) -> backward FFT(s) -> force back-interpolation (gather)
//   -> ad self-force correction.
//
// Reference counterparts: assign_charge / assign_charge_real /
// assign_charge_and_derivatives(_real) (charge-assign.c:119-305,
// 1067-1348), the convolution loops of P3M_ik / P3M_ik_i / P3M_ik_r /
// P3M_ad / P3M_ad_i / P3M_ad_r (p3m-ik.c:211-232, p3m-ik-i.c:202-228,
// p3m-ik-real.c:113-136, p3m-ad.c:184-193, p3m-ad-i.c:178-187,
// p3m-ad-real.c:92-101), assign_forces* (charge-assign.c:601-922,
// 1352-1539) and Substract_self_forces (p3m-ad-self-forces.c:114-139).
//
// Mesh layout in HBM: one complex mesh Q (m^3 interleaved re/im, index
// ((i m + j) m + k), x slowest) holds the charge density; interlaced
// methods put the unshifted mesh in the real part and the half-cell
// shifted mesh in the imaginary part (p3m-ik-i.c:189-190).  The r2c
// methods (6, 7) use the same complex transform with a zero imaginary
// part: on the k_z <= m/2 half it equals the r2c spectrum and the inverse
// of the Hermitian products equals the c2r result, so their forces are the
// same numbers up to rounding.
//
// Scatter: particles are counting-sorted by the mesh brick (B^3 points)
// that holds the base of their stencil; one CTA per brick accumulates the
// brick's charge into a (B+cao)^3 shared-memory tile with shared-memory
// atomics, then adds the tile to the global mesh (periodic wrap) with one
// global atomic per tile point.
#include <math.h>
#include <stdio.h>

#include "p3mg_internal.cuh"

namespace p3mg {

namespace {


// ---------------------------------------------------------------- binning

__global__ void bin_bricks_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                  const double *__restrict__ z, int n, double Hi, double shift, int m, int B, int nb,
                                  int *__restrict__ key, int *__restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b0, b1, b2, a;
  mesh_geometry(x[i], Hi, shift, 0, m, &b0, &a);
  mesh_geometry(y[i], Hi, shift, 0, m, &b1, &a);
  mesh_geometry(z[i], Hi, shift, 0, m, &b2, &a);
  const int k = ((b0 / B) * nb + (b1 / B)) * nb + (b2 / B);
  key[i] = k;
  atomicAdd(&count[k], 1);
}

__global__ void place_bricks_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                    const double *__restrict__ z, const double *__restrict__ q, int n,
                                    const int *__restrict__ key, const int *__restrict__ start, int *__restrict__ fill,
                                    int *__restrict__ sidx, double4 *__restrict__ sxyzq) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = key[i];
  const int slot = start[k] + atomicAdd(&fill[k], 1);
  sidx[slot] = i;
  sxyzq[slot] = make_double4(x[i], y[i], z[i], q[i]);
}

// single-CTA exclusive scan (sequential chunks, then a block scan of chunk sums)
__global__ void scan_kernel(const int *__restrict__ counts, int *__restrict__ start, int nb) {
  __shared__ int sums[1024];
  const int T = blockDim.x;
  const int chunk = (nb + T - 1) / T;
  const int lo = threadIdx.x * chunk;
  const int hi = min(lo + chunk, nb);
  int s = 0;
  for (int i = lo; i < hi; i++) s += counts[i];
  sums[threadIdx.x] = s;
  __syncthreads();
  for (int off = 1; off < T; off <<= 1) {
    int v = (threadIdx.x >= off) ? sums[threadIdx.x - off] : 0;
    __syncthreads();
    sums[threadIdx.x] += v;
    __syncthreads();
  }
  int run = (threadIdx.x == 0) ? 0 : sums[threadIdx.x - 1];
  for (int i = lo; i < hi; i++) {
    start[i] = run;
    run += counts[i];
  }
  if (threadIdx.x == T - 1) start[nb] = sums[T - 1];
}

__global__ void g_to_f32_kernel(const double *__restrict__ G, float *__restrict__ G32, size_t M) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M) G32[t] = (float)G[t];
}

}  // namespace


int g_to_f32(Ctx *c) {
  const int threads = 256;
  g_to_f32_kernel<<<(unsigned)((c->M + threads - 1) / threads), threads, 0, c->stream>>>(c->G, c->G32, c->M);
  c->launches++;
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

int scan_counts(const int *counts, int *start, int nb, cudaStream_t stream) {
  scan_kernel<<<1, 1024, 0, stream>>>(counts, start, nb);
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

int exclusive_scan(Ctx *c, const int *counts, int *start, int nb) {
  scan_kernel<<<1, 1024, 0, c->stream>>>(counts, start, nb);
  c->launches++;
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

// Sort particles by brick (counting sort) for the tiled scatter / gather.
int kspace_prepare(Ctx *c) {
  const int nb = c->nbrick1;
  const int nbr = nb * nb * nb;
  const int threads = 256;
  const int blocks = (c->n + threads - 1) / threads;
  const double Hi = (double)c->mesh / c->L;
  const double shift = (double)((c->cao - 1) / 2);
  P3MG_CUDA_TRY(cudaMemsetAsync(c->brick_count, 0, sizeof(int) * nbr, c->stream));
  P3MG_CUDA_TRY(cudaMemsetAsync(c->brick_fill, 0, sizeof(int) * nbr, c->stream));
  if (c->n > 0) {
    bin_bricks_kernel<<<blocks, threads, 0, c->stream>>>(c->x, c->y, c->z, c->n, Hi, shift, c->mesh, c->brick, nb,
                                                         c->part_key, c->brick_count);
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
  }
  P3MG_TRY(exclusive_scan(c, c->brick_count, c->brick_start, nbr));
  if (c->n > 0) {
    place_bricks_kernel<<<blocks, threads, 0, c->stream>>>(c->x, c->y, c->z, c->q, c->n, c->part_key, c->brick_start,
                                                           c->brick_fill, c->sorted_idx, c->sorted_xyzq);
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
  }
  return P3MG_OK;
}

int kspace_run_f64(Ctx *c);
int kspace_run_f32(Ctx *c);

int kspace_run(Ctx *c) {
  if (c->precision == P3MG_FP64) return kspace_run_f64(c);
  return kspace_run_f32(c);
}

}  // namespace p3mg
