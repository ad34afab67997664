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
// methods (6, 7) keep the charge in the padded real layout of an in-place
// r2c transform (row pitch m + 2 reals, charge-assign.c:252,257), transform
// it to the half spectrum m x m x (m/2 + 1), convolve there with G indexed
// by the full-mesh r_ind, and transform back with c2r (p3m-ik-real.c:72-76,
// 108-138, p3m-ad-real.c:62-64, 90-104): half the FFT bytes and flops of
// the complex transforms.
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

// Sort key of a particle: its brick (the B^3 mesh points holding the base
// of its stencil), then the stencil base inside the brick in row-major
// order, so that consecutive particles share mesh rows.  The count's
// atomic returns the particle's rank among its key's particles, stored
// beside the key: the placement then needs no second atomic.
__global__ void bin_bricks_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                  const double *__restrict__ z, int n, double Hi, double shift, int m, int B, int nb,
                                  int2 *__restrict__ key, int *__restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b0, b1, b2, a;
  mesh_geometry(x[i], Hi, shift, 0, m, &b0, &a);
  mesh_geometry(y[i], Hi, shift, 0, m, &b1, &a);
  mesh_geometry(z[i], Hi, shift, 0, m, &b2, &a);
  const int brick = ((b0 / B) * nb + (b1 / B)) * nb + (b2 / B);
  const int k = brick * (B * B * B) + ((b0 % B) * B + (b1 % B)) * B + (b2 % B);
  key[i] = make_int2(k, atomicAdd(&count[k], 1));
}

__global__ void place_bricks_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                    const double *__restrict__ z, const double *__restrict__ q, int n,
                                    const int2 *__restrict__ key, const int *__restrict__ start,
                                    int *__restrict__ sidx, double4 *__restrict__ sxyzq) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int2 kr = key[i];
  const int slot = start[kr.x] + kr.y;
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

// Multi-CTA exclusive scan for long count arrays: per-tile sums, a scan of
// the tile sums (scan_kernel), then each tile scanned with its offset.
constexpr int SCAN_TILE = 4096;  // elements per CTA: 1024 threads x 4

__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(1024) scan_tile_sums_kernel(const int *__restrict__ counts, int nb,
                                                               int *__restrict__ tsum) {
  __shared__ int ws[32];
  const int base = blockIdx.x * SCAN_TILE + threadIdx.x * 4;
  int s = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) s += (base + k < nb) ? counts[base + k] : 0;
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = warp_sum(ws[threadIdx.x]);
    if (threadIdx.x == 0) tsum[blockIdx.x] = s;
  }
}

__global__ void __launch_bounds__(1024) scan_tiles_kernel(const int *__restrict__ counts, int nb,
                                                           const int *__restrict__ tstart, int *__restrict__ start) {
  __shared__ int ws[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int base = blockIdx.x * SCAN_TILE + threadIdx.x * 4;
  int v[4];
#pragma unroll
  for (int k = 0; k < 4; k++) v[k] = (base + k < nb) ? counts[base + k] : 0;
  const int t = v[0] + v[1] + v[2] + v[3];
  int incl = t;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += u;
  }
  if (lane == 31) ws[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = ws[lane], wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += u;
    }
    ws[lane] = wi - w;  // exclusive prefix of the warp totals
  }
  __syncthreads();
  int run = tstart[blockIdx.x] + ws[warp] + incl - t;
#pragma unroll
  for (int k = 0; k < 4; k++)
    if (base + k < nb) {
      start[base + k] = run;
      run += v[k];
    }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) start[nb] = tstart[gridDim.x];
}

__global__ void g_to_f32_kernel(const double *__restrict__ G, float *__restrict__ G32, size_t M) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < M) G32[t] = (float)G[t];
}

}  // namespace


int g_to_f32(Ctx *c) { return g_to_f32_n(c, c->G, c->G32, c->M); }

int g_to_f32_n(Ctx *c, const double *G, float *G32, size_t count) {
  const int threads = 256;
  g_to_f32_kernel<<<(unsigned)((count + threads - 1) / threads), threads, 0, c->stream>>>(G, G32, count);
  c->launches++;
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

int scan_counts(const int *counts, int *start, int nb, cudaStream_t stream) {
  scan_kernel<<<1, 1024, 0, stream>>>(counts, start, nb);
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

int scan_tmp_reserve(Ctx *c, int nb) {
  const int need = 2 * (nb / SCAN_TILE + 2);
  if (need <= c->scan_cap) return P3MG_OK;
  if (c->scan_tmp) cudaFree(c->scan_tmp);
  c->scan_tmp = nullptr;
  c->scan_cap = 0;
  P3MG_CUDA_TRY(cudaMalloc(&c->scan_tmp, sizeof(int) * 2 * need));
  c->scan_cap = need;
  return P3MG_OK;
}

// Exclusive scan of nb counts into start[0..nb] (start[nb] = total): one
// CTA for short arrays, the tiled three-launch scan with the context's
// scratch (scan_tmp_reserve, done before any graph capture) otherwise --
// its second slot when the scan is enqueued on stream2, so the two streams
// of a step never share it.
int exclusive_scan(Ctx *c, const int *counts, int *start, int nb) {
  if (nb <= 16 * SCAN_TILE) {
    scan_kernel<<<1, 1024, 0, c->stream>>>(counts, start, nb);
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
    return P3MG_OK;
  }
  const int ntile = (nb + SCAN_TILE - 1) / SCAN_TILE;
  if (2 * (ntile + 1) > c->scan_cap) return P3MG_ERR_STATE;
  int *tmp = c->scan_tmp + ((c->stream2 && c->stream == c->stream2) ? c->scan_cap : 0);
  int *tsum = tmp, *tstart = tmp + ntile + 1;
  scan_tile_sums_kernel<<<ntile, 1024, 0, c->stream>>>(counts, nb, tsum);
  scan_kernel<<<1, 1024, 0, c->stream>>>(tsum, tstart, ntile);
  scan_tiles_kernel<<<ntile, 1024, 0, c->stream>>>(counts, nb, tstart, start);
  c->launches += 3;
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

// Sort particles by brick (counting sort) for the tiled scatter / gather.
int kspace_prepare(Ctx *c) {
  const int nb = c->nbrick1;
  const int nbr = nb * nb * nb * c->brick * c->brick * c->brick;  // sort keys
  const int threads = 256;
  const int blocks = (c->n + threads - 1) / threads;
  const double Hi = (double)c->mesh / c->L;
  const double shift = (double)((c->cao - 1) / 2);
  P3MG_CUDA_TRY(cudaMemsetAsync(c->brick_count, 0, sizeof(int) * nbr, c->stream));
  if (c->n > 0) {
    bin_bricks_kernel<<<blocks, threads, 0, c->stream>>>(c->x, c->y, c->z, c->n, Hi, shift, c->mesh, c->brick, nb,
                                                         c->part_key, c->brick_count);
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
  }
  P3MG_TRY(exclusive_scan(c, c->brick_count, c->brick_start, nbr));
  if (c->n > 0) {
    place_bricks_kernel<<<blocks, threads, 0, c->stream>>>(c->x, c->y, c->z, c->q, c->n, c->part_key, c->brick_start,
                                                           c->sorted_idx, c->sorted_xyzq);
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
  }
  return P3MG_OK;
}

int kspace_run_f64(Ctx *c);
int kspace_run_f32(Ctx *c);
int kspace_batch_f64(Ctx *c, const KspaceBatch &b);
int kspace_batch_f32(Ctx *c, const KspaceBatch &b);

int kspace_run(Ctx *c) {
  if (c->precision == P3MG_FP64) return kspace_run_f64(c);
  return kspace_run_f32(c);
}

int kspace_batch(Ctx *c, const KspaceBatch &b) {
  if (c->precision == P3MG_FP64) return kspace_batch_f64(c, b);
  return kspace_batch_f32(c, b);
}

int adjoint_scatter_f32(Ctx *c);
int adjoint_scatter_f64(Ctx *c);
int adjoint_gather_f32(Ctx *c, const void *Phi, double s, double ge, double *gx, double *gq);
int adjoint_gather_f64(Ctx *c, const void *Phi, double s, double ge, double *gx, double *gq);

int adjoint_scatter(Ctx *c) { return c->precision == P3MG_FP64 ? adjoint_scatter_f64(c) : adjoint_scatter_f32(c); }

int adjoint_gather(Ctx *c, const void *Phi, double s, double ge, double *gx, double *gq) {
  return c->precision == P3MG_FP64 ? adjoint_gather_f64(c, Phi, s, ge, gx, gq)
                                   : adjoint_gather_f32(c, Phi, s, ge, gx, gq);
}

}  // namespace p3mg
