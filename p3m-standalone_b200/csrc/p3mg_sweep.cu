// The reference's alpha sweep (main.c:375-446: for alpha = alphamin;
// alpha <= alphamax; alpha += alphastep, Influence_function then
// Calculate_forces) as one batched GPU pass.
//
// Per chunk of alphas: G_opt and the ad self-force coefficients of every
// alpha in one launch each; the real-space pairs of every alpha in one
// launch (grid.y = alpha over the same cell list); the charge assignment
// and forward FFT once for the whole sweep (they do not depend on alpha);
// then the convolutions, one batched backward FFT over all the chunk's
// meshes, the gather and the self-force correction, each one launch over
// the alphas; finally f = f_self + f_k + f_r and, against reference forces,
// sum |f - f_ref|^2 per alpha.  The kernels are the single-step kernels
// with an alpha index, so each alpha's forces are the ones
// p3mg_influence + p3mg_calculate_forces give.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "p3mg_internal.cuh"

namespace p3mg {

namespace {

// sum_t (f[y 3n + t] - ref[t])^2 into rms2[y]
__global__ void sq_err_kernel(const double *__restrict__ f, const double *__restrict__ ref, size_t n3,
                              double *__restrict__ rms2) {
  __shared__ double red[8];
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (t < n3) {
    const double d = f[(size_t)blockIdx.y * n3 + t] - ref[t];
    v = d * d;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
    if (s != 0.0) atomicAdd(&rms2[blockIdx.y], s);
  }
}

__global__ void combine_batch_kernel(double *__restrict__ f, const double *__restrict__ fk,
                                     const double *__restrict__ fr, size_t count) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < count) f[t] += fk[t] + fr[t];
}

// Sub-buffers of the sweep, carved from one workspace that the context
// keeps between calls (grown when a call needs more).
struct SweepMem {
  double *alphas = nullptr, *G = nullptr, *S26 = nullptr, *b81 = nullptr;
  float *G32 = nullptr;
  void *F = nullptr, *P = nullptr;
  double *f = nullptr, *fk = nullptr, *fr = nullptr, *energy = nullptr, *rms2 = nullptr, *ref = nullptr;
};

// Lay the buffers out from base (nullptr: only count); returns the bytes.
size_t sweep_layout(const Ctx *c, int na, int chunk, bool with_ref, unsigned char *base, SweepMem *w) {
  const size_t n3 = 3 * (size_t)c->n;
  const size_t M = c->M;
  const size_t csz = (c->precision == P3MG_FP64) ? 16 : 8;
  size_t off = 0;
  auto take = [&](size_t bytes) -> void * {
    void *p = base ? (void *)(base + off) : nullptr;
    off += (bytes + 255) & ~(size_t)255;
    return p;
  };
  w->alphas = (double *)take((size_t)na * sizeof(double));
  w->G = (double *)take((size_t)chunk * M * sizeof(double));
  w->S26 = (double *)take(26 * (size_t)chunk * sizeof(double));
  w->b81 = (double *)take(81 * (size_t)chunk * sizeof(double));
  w->G32 = (c->precision != P3MG_FP64) ? (float *)take((size_t)chunk * M * sizeof(float)) : nullptr;
  if (method_ad(c->method)) {
    w->F = take((size_t)chunk * M * csz);
    w->P = nullptr;
  } else {
    w->F = take(3 * (size_t)chunk * M * csz);
    w->P = take((size_t)chunk * (method_interlaced(c->method) ? 2 : 1) * M * 2 * csz);
  }
  w->f = (double *)take((size_t)chunk * n3 * sizeof(double) + 8);
  w->fk = (double *)take((size_t)chunk * n3 * sizeof(double) + 8);
  w->fr = (double *)take((size_t)chunk * n3 * sizeof(double) + 8);
  w->energy = (double *)take((size_t)chunk * sizeof(double));
  w->rms2 = (double *)take((size_t)na * sizeof(double));
  w->ref = with_ref ? (double *)take(n3 * sizeof(double) + 8) : nullptr;
  return off;
}

}  // namespace

// Device bytes one alpha of the sweep needs (meshes, G, forces).
size_t sweep_bytes_per_alpha(const Ctx *c) {
  const size_t csz = (c->precision == P3MG_FP64) ? 16 : 8;
  const size_t M = c->M;
  size_t b = M * sizeof(double) + 81 * sizeof(double) + 26 * sizeof(double);
  if (c->precision != P3MG_FP64) b += M * sizeof(float);
  if (method_ad(c->method))
    b += M * csz;
  else
    b += 3 * M * csz + (method_interlaced(c->method) ? 2 : 1) * M * 2 * csz;
  b += 3 * 3 * (size_t)c->n * sizeof(double) + 2 * sizeof(double);
  return b;
}

int sweep_run(Ctx *c, double rcut, int na, const double *alphas, const double *ref, double *rms_out, double *f_out,
              size_t budget) {
  const size_t n3 = 3 * (size_t)c->n;
  const size_t per = sweep_bytes_per_alpha(c);
  int chunk = (int)(budget / per);
  if (chunk < 1) chunk = 1;
  if (chunk > na) chunk = na;
  const size_t M = c->M;
  SweepMem w;
  int st = P3MG_OK;
  cudaError_t e = cudaSuccess;
  const size_t need = sweep_layout(c, na, chunk, ref != nullptr, nullptr, &w);
  if (need > c->sweep_cap) {
    if (c->sweep_ws) cudaFree(c->sweep_ws);
    c->sweep_ws = nullptr;
    c->sweep_cap = 0;
    e = cudaMalloc(&c->sweep_ws, need);
    if (e != cudaSuccess) {
      record_cuda_error(e);
      return (e == cudaErrorMemoryAllocation) ? P3MG_ERR_ALLOC : P3MG_ERR_CUDA;
    }
    c->sweep_cap = need;
  }
  sweep_layout(c, na, chunk, ref != nullptr, reinterpret_cast<unsigned char *>(c->sweep_ws), &w);
  do {
    e = cudaMemcpyAsync(w.alphas, alphas, (size_t)na * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && ref) e = cudaMemcpyAsync(w.ref, ref, n3 * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.rms2, 0, (size_t)na * sizeof(double), c->stream);
    if (e != cudaSuccess) break;
    if (rcut != 0.0) {
      st = pairs_reserve(c, rcut);
      if (st != P3MG_OK) break;
    }
    if (c->n > 0) {
      st = kspace_prepare(c);
      if (st != P3MG_OK) break;
    }
    for (int a0 = 0; a0 < na && st == P3MG_OK && e == cudaSuccess; a0 += chunk) {
      const int nch = (na - a0 < chunk) ? na - a0 : chunk;
      const double *dal = w.alphas + a0;
      st = influence_batch(c, dal, nch, w.G, w.S26, w.b81);
      if (st != P3MG_OK) break;
      if (c->precision != P3MG_FP64) {
        st = g_to_f32_n(c, w.G, w.G32, (size_t)nch * M);
        if (st != P3MG_OK) break;
      }
      const size_t fb = (size_t)nch * n3 * sizeof(double);
      e = cudaMemsetAsync(w.f, 0, fb, c->stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(w.fk, 0, fb, c->stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(w.fr, 0, fb, c->stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(w.energy, 0, (size_t)nch * sizeof(double), c->stream);
      if (e != cudaSuccess) break;
      if (rcut != 0.0) {
        st = pairs_run(c, rcut, dal, nch, w.fr, w.energy);
        if (st != P3MG_OK) break;
      }
      if (c->n > 0) {
        KspaceBatch kb;
        kb.na = nch;
        kb.G = (c->precision == P3MG_FP64) ? (const void *)w.G : (const void *)w.G32;
        kb.b81 = w.b81;
        kb.F = w.F;
        kb.P = w.P;
        kb.fk = w.fk;
        kb.f = w.f;
        kb.forward = (a0 == 0);
        st = kspace_batch(c, kb);
        if (st != P3MG_OK) break;
        const size_t cnt = (size_t)nch * n3;
        combine_batch_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, c->stream>>>(w.f, w.fk, w.fr, cnt);
        c->launches++;
        if (ref) {
          sq_err_kernel<<<dim3((unsigned)((n3 + 255) / 256), nch), 256, 0, c->stream>>>(w.f, w.ref, n3, w.rms2 + a0);
          c->launches++;
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) break;
      }
      if (f_out) {
        e = cudaMemcpyAsync(f_out + (size_t)a0 * n3, w.f, fb, cudaMemcpyDeviceToHost, c->stream);
        if (e != cudaSuccess) break;
      }
    }
    if (st != P3MG_OK || e != cudaSuccess) break;
    if (rms_out && ref) {
      e = cudaMemcpyAsync(rms_out, w.rms2, (size_t)na * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
      if (e != cudaSuccess) break;
    }
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) break;
    if (rms_out && ref)
      for (int k = 0; k < na; k++) rms_out[k] = sqrt(rms_out[k]) / sqrt((double)(c->n > 0 ? c->n : 1));
  } while (0);
  if (e != cudaSuccess) {
    record_cuda_error(e);
    st = P3MG_ERR_CUDA;
  }
  cudaStreamSynchronize(c->stream);
  return st;
}

}  // namespace p3mg
