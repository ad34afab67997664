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
//
// Many alphas over a narrow range (>= 24 alphas, max/min <= 2.5, no batch
// limit given): the forces are smooth functions of t = 1/alpha^2 -- G_opt
// is a sum of exp(-k^2 t / 4) terms, whose fast high-|k| ones reach the
// forces only through the charge-assignment filter twice, and the pair
// force is made of erfc and Gaussian terms in alpha = t^{-1/2} (G itself
// does not interpolate to the same accuracy: the checks below are on
// forces) -- so they are evaluated exactly as above at R
// Chebyshev nodes in t (10 FP32, 16 FP64) and interpolated to every
// requested alpha.  Two of the requested alphas are evaluated exactly as
// well; the interpolation is used only if it reproduces their forces to
// 1e-6 (FP32) / 1e-12 (FP64) of the RMS force, else every alpha is evaluated.
// Without a force output the interpolation goes straight into the squared
// errors (one kernel reading the node forces once), so an RMS-only sweep
// writes no per-alpha forces.
//
// Reference forces arrive as three host rows; they are uploaded on the
// context's second stream once work is queued on the first, so that a
// pageable copy overlaps the evaluation instead of preceding it.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

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

// out[y n3 + t] = sum_r W[y R + r] fn[r n3 + t] (interpolation from the nodes)
__global__ void interp_kernel(double *__restrict__ out, const double *__restrict__ fn, const double *__restrict__ W,
                              int R, size_t n3) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n3) return;
  const double *w = W + (size_t)blockIdx.y * R;
  double v = 0.0;
  for (int r = 0; r < R; r++) v += w[r] * fn[(size_t)r * n3 + t];
  out[(size_t)blockIdx.y * n3 + t] = v;
}

// acc[2 y] += sum_t (a - b)^2, acc[2 y + 1] += sum_t b^2 over entry y
__global__ void diff_norm_kernel(const double *__restrict__ a, const double *__restrict__ b, size_t n3,
                                 double *__restrict__ acc) {
  __shared__ double red[2][8];
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double d2 = 0.0, b2 = 0.0;
  if (t < n3) {
    const double bv = b[(size_t)blockIdx.y * n3 + t];
    const double d = a[(size_t)blockIdx.y * n3 + t] - bv;
    d2 = d * d;
    b2 = bv * bv;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    d2 += __shfl_xor_sync(0xffffffffu, d2, o);
    b2 += __shfl_xor_sync(0xffffffffu, b2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = d2;
    red[1][threadIdx.x >> 5] = b2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      s0 += red[0][w];
      s1 += red[1][w];
    }
    atomicAdd(&acc[2 * blockIdx.y], s0);
    atomicAdd(&acc[2 * blockIdx.y + 1], s1);
  }
}

// Interpolation straight into squared errors:
// rms2[a] += sum_t (sum_r W[a R + r] fn[r n3 + t] - ref[t])^2 for IE_AB
// alphas per block.  grid.x = alpha blocks (fastest, so the blocks of one t
// tile run together and share its node reads through L2), grid.y = t tiles
// of blockDim.x * IE_ITEMS entries.  RN >= R is the register count for the
// node values.
constexpr int IE_AB = 16;
constexpr int IE_ITEMS = 8;
constexpr int IE_THREADS = 256;

template <int RN>
__global__ void __launch_bounds__(IE_THREADS) interp_err_kernel(const double *__restrict__ fn,
                                                                const double *__restrict__ W, int R, int na,
                                                                const double *__restrict__ ref, size_t n3,
                                                                double *__restrict__ rms2) {
  __shared__ double ws[IE_AB][RN];
  __shared__ double red[IE_THREADS / 32][IE_AB];
  const int a0 = blockIdx.x * IE_AB;
  for (int i = threadIdx.x; i < IE_AB * RN; i += blockDim.x) {
    const int a = i / RN, r = i % RN;
    ws[a][r] = (a0 + a < na && r < R) ? W[(size_t)(a0 + a) * R + r] : 0.0;
  }
  __syncthreads();
  double acc[IE_AB];
#pragma unroll
  for (int a = 0; a < IE_AB; a++) acc[a] = 0.0;
  const size_t base = (size_t)blockIdx.y * blockDim.x * IE_ITEMS + threadIdx.x;
#pragma unroll 1
  for (int it = 0; it < IE_ITEMS; it++) {
    const size_t t = base + (size_t)it * blockDim.x;
    if (t >= n3) break;
    // keeps the weight loads inside the loop (hoisted, they would take
    // IE_AB * RN registers)
    asm volatile("" ::: "memory");
    double f[RN];
#pragma unroll
    for (int r = 0; r < RN; r++) f[r] = (r < R) ? fn[(size_t)r * n3 + t] : 0.0;
    const double rv = ref[t];
#pragma unroll
    for (int a = 0; a < IE_AB; a++) {
      double v = 0.0;
#pragma unroll
      for (int r = 0; r < RN; r++) v = fma(ws[a][r], f[r], v);
      const double d = v - rv;
      acc[a] = fma(d, d, acc[a]);
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < IE_AB; a++) {
    double v = acc[a];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][a] = v;
  }
  __syncthreads();
  if (threadIdx.x < IE_AB && a0 + (int)threadIdx.x < na) {
    double s = 0.0;
    for (int w = 0; w < IE_THREADS / 32; w++) s += red[w][threadIdx.x];
    if (s != 0.0) atomicAdd(&rms2[a0 + threadIdx.x], s);
  }
}

// Host reference rows (x, y, z; n doubles each) to dst (3n doubles) on the
// second stream; the context stream waits for them before its next launch.
cudaError_t upload_ref(Ctx *c, const double *const *ref, double *dst) {
  const size_t n = (size_t)c->n;
  cudaStream_t s = c->stream2 ? c->stream2 : c->stream;
  for (int d = 0; d < 3; d++) {
    const cudaError_t e = cudaMemcpyAsync(dst + d * n, ref[d], n * sizeof(double), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
  }
  if (s == c->stream) return cudaSuccess;
  const cudaError_t e = cudaEventRecord(c->ev_join, s);
  return e != cudaSuccess ? e : cudaStreamWaitEvent(c->stream, c->ev_join, 0);
}

// Lagrange weights of the nodes tn[0..R) at t
void lagrange_weights(const double *tn, int R, double t, double *w) {
  for (int i = 0; i < R; i++) {
    double v = 1.0;
    for (int j = 0; j < R; j++)
      if (j != i) v *= (t - tn[j]) / (tn[i] - tn[j]);
    w[i] = v;
  }
}

constexpr int SWEEP_INTERP_NOT_USED = 1;  // internal: fall back to the exact sweep

// interpolation nodes: 10 (FP32: the checks measure ~2e-7, the FP32
// rounding of the forces, up to max/min = 2; 8 nodes measured up to 1.8e-6
// there), 16 (FP64)
constexpr int sweep_interp_nodes(bool dbl) { return dbl ? 16 : 10; }

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

namespace {

// Every alpha evaluated.  ref: host reference rows x, y, z (or NULL).
// f_dev (device, na 3n doubles, may be NULL) receives the total forces as
// well.  late_ref (host rows, may be NULL) is uploaded to late_dst once the
// evaluation is queued, for the caller's use after it.
// fr_pre (device, na 3n doubles, may be NULL): the real-space forces of
// every alpha, computed elsewhere (the tuning grid shares them between
// contexts that hold the same system); then no pairs run here.  async:
// return once the work is queued, the squared errors left in
// c->sweep_rms2 (device) for the caller to read after synchronising.
int sweep_exact(Ctx *c, double rcut, int na, const double *alphas, const double *const *ref, double *rms_out,
                double *f_out, size_t budget, double *f_dev, const double *const *late_ref = nullptr,
                double *late_dst = nullptr, const double *fr_pre = nullptr, bool async = false) {
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
    if (e == cudaSuccess) e = cudaMemsetAsync(w.rms2, 0, (size_t)na * sizeof(double), c->stream);
    if (e != cudaSuccess) break;
    if (rcut != 0.0 && !fr_pre) {
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
      if (e == cudaSuccess && !fr_pre) e = cudaMemsetAsync(w.fr, 0, fb, c->stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(w.energy, 0, (size_t)nch * sizeof(double), c->stream);
      if (e != cudaSuccess) break;
      if (fr_pre) {
        w.fr = const_cast<double *>(fr_pre) + (size_t)a0 * n3;  // read only
      } else if (rcut != 0.0) {
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
        if (ref && a0 == 0) e = upload_ref(c, ref, w.ref);
        if (e != cudaSuccess) break;
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
      if (f_dev) {
        e = cudaMemcpyAsync(f_dev + (size_t)a0 * n3, w.f, fb, cudaMemcpyDeviceToDevice, c->stream);
        if (e != cudaSuccess) break;
      }
    }
    if (st != P3MG_OK || e != cudaSuccess) break;
    if (late_ref) {
      e = upload_ref(c, late_ref, late_dst);
      if (e != cudaSuccess) break;
    }
    c->sweep_rms2 = w.rms2;
    if (async) return P3MG_OK;
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

// Interpolation in t = 1/alpha^2 from exact evaluations at Chebyshev nodes
// (see the file comment); SWEEP_INTERP_NOT_USED when it does not apply or
// does not reproduce the check alphas.
int sweep_interpolated(Ctx *c, double rcut, int na, const double *alphas, const double *const *ref,
                       double *rms_out, double *f_out, size_t budget) {
  if (na < 24 || c->n == 0) return SWEEP_INTERP_NOT_USED;
  double amin = alphas[0], amax = alphas[0];
  for (int k = 1; k < na; k++) {
    amin = alphas[k] < amin ? alphas[k] : amin;
    amax = alphas[k] > amax ? alphas[k] : amax;
  }
  if (!(amin > 0.0) || amax > 2.5 * amin) return SWEEP_INTERP_NOT_USED;
  const bool dbl = c->precision == P3MG_FP64;
  const int R = sweep_interp_nodes(dbl);
  if (R + 2 > na / 2) return SWEEP_INTERP_NOT_USED;
  const double tol = dbl ? 1e-12 : 1e-6;
  const size_t n3 = 3 * (size_t)c->n;
  // nodes in t, then two requested alphas (a third and two thirds up the sorted list) as checks
  std::vector<double> ex(R + 2), tn(R);
  const double lo = 1.0 / (amax * amax), hi = 1.0 / (amin * amin);
  for (int r = 0; r < R; r++) {
    tn[r] = 0.5 * (lo + hi) + 0.5 * (hi - lo) * cos((2 * r + 1) * P3MG_PI / (2.0 * R));
    ex[r] = 1.0 / sqrt(tn[r]);
  }
  std::vector<double> sorted(alphas, alphas + na);
  std::sort(sorted.begin(), sorted.end());
  ex[R] = sorted[na / 3];
  ex[R + 1] = sorted[(2 * na) / 3];
  // device: node + check forces, interpolated forces (one chunk of alphas
  // with a force output, else the two checks), ref, weights, squared
  // errors and check sums
  const int chunk = f_out ? 16 : 2;
  const size_t nf = (size_t)(R + 2) * n3, nb = (size_t)chunk * n3;
  const size_t total = (nf + nb + (ref ? n3 : 0) + (size_t)na * R + (size_t)na + 8) * sizeof(double);
  if (total > c->interp_cap) {
    if (c->interp_ws) cudaFree(c->interp_ws);
    c->interp_ws = nullptr;
    c->interp_cap = 0;
    P3MG_CUDA_TRY(cudaMalloc(&c->interp_ws, total));
    c->interp_cap = total;
  }
  double *fnode = (double *)c->interp_ws, *fb = fnode + nf, *dref = fb + nb;
  double *dW = dref + (ref ? n3 : 0), *rms2 = dW + (size_t)na * R, *sums = rms2 + na;
  P3MG_TRY(sweep_exact(c, rcut, R + 2, ex.data(), nullptr, nullptr, nullptr, budget, fnode, ref, dref));
  // the checks: interpolate and compare with their exact forces
  std::vector<double> W((size_t)na * R);
  lagrange_weights(tn.data(), R, 1.0 / (ex[R] * ex[R]), W.data());
  lagrange_weights(tn.data(), R, 1.0 / (ex[R + 1] * ex[R + 1]), W.data() + R);
  cudaStream_t st = c->stream;
  P3MG_CUDA_TRY(cudaMemcpyAsync(dW, W.data(), 2 * (size_t)R * sizeof(double), cudaMemcpyHostToDevice, st));
  P3MG_CUDA_TRY(cudaMemsetAsync(sums, 0, 4 * sizeof(double), st));
  const unsigned gx = (unsigned)((n3 + 255) / 256);
  interp_kernel<<<dim3(gx, 2), 256, 0, st>>>(fb, fnode, dW, R, n3);
  diff_norm_kernel<<<dim3(gx, 2), 256, 0, st>>>(fb, fnode + (size_t)R * n3, n3, sums);
  c->launches += 2;
  P3MG_CUDA_TRY(cudaGetLastError());
  double hs[4];
  P3MG_CUDA_TRY(cudaMemcpyAsync(hs, sums, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  P3MG_CUDA_TRY(cudaStreamSynchronize(st));
  c->sweep_check = 0.0;
  for (int j = 0; j < 2; j++) {
    const double rel = hs[2 * j + 1] > 0.0 ? sqrt(hs[2 * j] / hs[2 * j + 1]) : (hs[2 * j] > 0.0 ? INFINITY : 0.0);
    c->sweep_check = rel > c->sweep_check ? rel : c->sweep_check;
  }
  if (!(c->sweep_check <= tol)) return SWEEP_INTERP_NOT_USED;
  // every alpha: with a force output chunk by chunk, else straight into the
  // squared errors
  for (int k = 0; k < na; k++)
    lagrange_weights(tn.data(), R, 1.0 / (alphas[k] * alphas[k]), W.data() + (size_t)k * R);
  P3MG_CUDA_TRY(cudaMemcpyAsync(dW, W.data(), (size_t)na * R * sizeof(double), cudaMemcpyHostToDevice, st));
  if (ref) P3MG_CUDA_TRY(cudaMemsetAsync(rms2, 0, (size_t)na * sizeof(double), st));
  if (f_out) {
    for (int a0 = 0; a0 < na; a0 += chunk) {
      const int nch = (na - a0 < chunk) ? na - a0 : chunk;
      interp_kernel<<<dim3(gx, nch), 256, 0, st>>>(fb, fnode, dW + (size_t)a0 * R, R, n3);
      c->launches++;
      if (ref) {
        sq_err_kernel<<<dim3(gx, nch), 256, 0, st>>>(fb, dref, n3, rms2 + a0);
        c->launches++;
      }
      P3MG_CUDA_TRY(cudaGetLastError());
      P3MG_CUDA_TRY(cudaMemcpyAsync(f_out + (size_t)a0 * n3, fb, (size_t)nch * n3 * sizeof(double),
                                    cudaMemcpyDeviceToHost, st));
    }
  } else if (ref) {
    const dim3 grid((unsigned)((na + IE_AB - 1) / IE_AB),
                    (unsigned)((n3 + (size_t)IE_THREADS * IE_ITEMS - 1) / ((size_t)IE_THREADS * IE_ITEMS)));
    if (R <= 10)
      interp_err_kernel<10><<<grid, IE_THREADS, 0, st>>>(fnode, dW, R, na, dref, n3, rms2);
    else
      interp_err_kernel<16><<<grid, IE_THREADS, 0, st>>>(fnode, dW, R, na, dref, n3, rms2);
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
  }
  if (rms_out && ref)
    P3MG_CUDA_TRY(cudaMemcpyAsync(rms_out, rms2, (size_t)na * sizeof(double), cudaMemcpyDeviceToHost, st));
  P3MG_CUDA_TRY(cudaStreamSynchronize(st));
  if (rms_out && ref)
    for (int k = 0; k < na; k++) rms_out[k] = sqrt(rms_out[k]) / sqrt((double)c->n);
  return P3MG_OK;
}

}  // namespace

int sweep_run(Ctx *c, double rcut, int na, const double *alphas, const double *const *ref, double *rms_out,
              double *f_out, size_t budget, bool exact) {
  c->sweep_nodes = 0;
  c->sweep_check = -1.0;
  if (!exact) {
    const int st = sweep_interpolated(c, rcut, na, alphas, ref, rms_out, f_out, budget);
    if (st != SWEEP_INTERP_NOT_USED) {
      if (st == P3MG_OK) c->sweep_nodes = sweep_interp_nodes(c->precision == P3MG_FP64);
      return st;
    }
  }
  return sweep_exact(c, rcut, na, alphas, ref, rms_out, f_out, budget, nullptr);
}

// The tuning grid: every alpha on every context (same system, different
// mesh / cao / method).  The real-space forces of all alphas are computed
// once on cs[0]'s stream; the other contexts wait for them (an event) and
// run their k-space batches concurrently on their own streams, each with
// its share of the memory budget; one synchronisation at the end.
int sweep_grid_run(Ctx *const *cs, int nctx, double rcut, int na, const double *alphas, const double *const *ref,
                   double *rms_out, size_t budget) {
  Ctx *c0 = cs[0];
  const size_t n3 = 3 * (size_t)c0->n;
  double *shared = nullptr;  // alphas, then na 3n real-space forces and na energies
  cudaEvent_t ready = nullptr;
  int st = P3MG_OK;
  cudaError_t e = cudaSuccess;
  const size_t bytes = ((size_t)na + (size_t)na * n3 + (size_t)na) * sizeof(double);
  e = cudaMalloc(&shared, bytes);
  if (e != cudaSuccess) {
    record_cuda_error(e);
    return e == cudaErrorMemoryAllocation ? P3MG_ERR_ALLOC : P3MG_ERR_CUDA;
  }
  double *d_al = shared, *fr_all = shared + na, *e_all = fr_all + (size_t)na * n3;
  do {
    e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
    if (e != cudaSuccess) break;
    e = cudaMemcpyAsync(d_al, alphas, (size_t)na * sizeof(double), cudaMemcpyHostToDevice, c0->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(fr_all, 0, ((size_t)na * n3 + na) * sizeof(double), c0->stream);
    if (e != cudaSuccess) break;
    if (rcut != 0.0 && c0->n > 0) {
      st = pairs_reserve(c0, rcut);
      if (st == P3MG_OK) st = pairs_run(c0, rcut, d_al, na, fr_all, e_all);
      if (st != P3MG_OK) break;
    }
    e = cudaEventRecord(ready, c0->stream);
    if (e != cudaSuccess) break;
    const size_t share = budget / (size_t)nctx;
    for (int i = 0; i < nctx && st == P3MG_OK; i++) {
      e = cudaStreamWaitEvent(cs[i]->stream, ready, 0);
      if (e != cudaSuccess) break;
      cs[i]->sweep_nodes = 0;
      cs[i]->sweep_check = -1.0;
      st = sweep_exact(cs[i], rcut, na, alphas, ref, nullptr, nullptr, share, nullptr, nullptr, nullptr, fr_all, true);
    }
    if (st != P3MG_OK || e != cudaSuccess) break;
    for (int i = 0; i < nctx; i++) {
      double *row = rms_out + (size_t)i * na;
      e = cudaMemcpyAsync(row, cs[i]->sweep_rms2, (size_t)na * sizeof(double), cudaMemcpyDeviceToHost,
                          cs[i]->stream);
      if (e != cudaSuccess) break;
    }
    if (e != cudaSuccess) break;
    for (int i = 0; i < nctx && e == cudaSuccess; i++) e = cudaStreamSynchronize(cs[i]->stream);
    if (e != cudaSuccess) break;
    for (size_t k = 0; k < (size_t)nctx * na; k++) rms_out[k] = sqrt(rms_out[k]) / sqrt((double)c0->n);
  } while (0);
  if (e != cudaSuccess) {
    record_cuda_error(e);
    st = P3MG_ERR_CUDA;
  }
  for (int i = 0; i < nctx; i++) cudaStreamSynchronize(cs[i]->stream);
  if (ready) cudaEventDestroy(ready);
  cudaFree(shared);
  return st;
}

}  // namespace p3mg
