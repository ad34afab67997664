// Register-tiled FFT passes for FP32 meshes of m = 32, 64 or 128 points per
// side (the transform of p3mg_fft.cu: complex, in place, unnormalised,
// forward sign -1, backward +1, row-major m^3 with the last index fastest).
//
// A pencil of length m = A B is transformed by A threads (the A warps of a
// CTA, one pencil per lane, 32 pencils per CTA) with one Cooley-Tukey split
// (n = t + A j, k = k1 + B k2):
//   thread t: Y_t[k1] = sum_j x[t + A j] W_B^{j k1}   (B-point DFT in registers)
//             Y_t[k1] *= W_m^{t k1}                   (twiddle table)
//   exchange through shared memory (pencil rows of m + 1 entries: lanes
//   touch rows m + 1 apart, so 8-byte accesses are bank-conflict free)
//   thread t: X[k1 + B k2] = sum_t' Y_t'[k1] W_A^{t' k2} for k1 = t + A s
// The small DFTs are radix-2 in registers with the 16th roots of unity as
// constants.  x and y pencils are read and written straight from global
// memory (a warp's lanes are 32 consecutive z, 256 contiguous bytes); z
// pencils are staged through the same shared rows so global accesses stay
// contiguous.  One pass per axis reads and writes the mesh once (the
// Stockham kernel of p3mg_fft.cu makes log_radix(m) shared-memory passes
// with a barrier each).
//
// The ik convolution (conv_ik_kernel: F_d = i D_d(k) G(k) s Q^(k)) is folded
// into the first backward pass: the z pass reads Q^ and G once and writes
// the three field meshes after their z transforms.
#include <math.h>

#include "p3mg_internal.cuh"

namespace p3mg {

namespace {

typedef float2 C32;

template <int M>
struct PencilShape;
template <>
struct PencilShape<32> {
  static constexpr int A = 4, B = 8;
};
template <>
struct PencilShape<64> {
  static constexpr int A = 8, B = 8;
};
template <>
struct PencilShape<128> {
  static constexpr int A = 8, B = 16;
};

constexpr int PENCILS = 32;  // pencils per CTA, one per lane

__device__ __forceinline__ C32 c_mul(C32 a, C32 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ C32 c_add(C32 a, C32 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ C32 c_sub(C32 a, C32 b) { return make_float2(a.x - b.x, a.y - b.y); }

// x exp(SIGN 2 pi i e / 16) for 0 <= e < 16 (e a compile-time constant once
// the callers' loops are unrolled, so the switch folds away)
template <int SIGN>
__device__ __forceinline__ C32 rot16(C32 x, int e) {
  const float c1 = 0.92387953251128675613f;  // cos(pi/8)
  const float s1 = 0.38268343236508977173f;  // sin(pi/8)
  const float h = 0.70710678118654752440f;   // sqrt(1/2)
  float cr, ci;                              // cos, sin of 2 pi e / 16
  switch (e & 15) {
    case 0: return x;
    case 4: return SIGN > 0 ? make_float2(-x.y, x.x) : make_float2(x.y, -x.x);
    case 8: return make_float2(-x.x, -x.y);
    case 12: return SIGN > 0 ? make_float2(x.y, -x.x) : make_float2(-x.y, x.x);
    case 1: cr = c1; ci = s1; break;
    case 2: cr = h; ci = h; break;
    case 3: cr = s1; ci = c1; break;
    case 5: cr = -s1; ci = c1; break;
    case 6: cr = -h; ci = h; break;
    case 7: cr = -c1; ci = s1; break;
    case 9: cr = -c1; ci = -s1; break;
    case 10: cr = -h; ci = -h; break;
    case 11: cr = -s1; ci = -c1; break;
    case 13: cr = s1; ci = -c1; break;
    case 14: cr = h; ci = -h; break;
    default: cr = c1; ci = -s1; break;
  }
  const float wi = SIGN > 0 ? ci : -ci;
  return make_float2(x.x * cr - x.y * wi, x.x * wi + x.y * cr);
}

__host__ __device__ constexpr int bit_reverse(int i, int n) {
  int r = 0;
  for (int b = 1; b < n; b <<= 1) r = (r << 1) | ((i & b) ? 1 : 0);
  return r;
}

// In-place N-point DFT of v (N = 2, 4, 8, 16): radix-2 decimation in time on
// the bit-reversed registers, natural order out.
template <int N, int SIGN>
__device__ __forceinline__ void dft_reg(C32 (&v)[N]) {
  C32 a[N];
#pragma unroll
  for (int i = 0; i < N; i++) a[i] = v[bit_reverse(i, N)];
#pragma unroll
  for (int half = 1; half < N; half <<= 1) {
#pragma unroll
    for (int i = 0; i < N; i += 2 * half) {
#pragma unroll
      for (int k = 0; k < half; k++) {
        // W_{2 half}^k = exp(SIGN 2 pi i k 16 / (2 half) / 16)
        const C32 b = rot16<SIGN>(a[i + k + half], k * (16 / (2 * half)));
        const C32 x = a[i + k];
        a[i + k] = c_add(x, b);
        a[i + k + half] = c_sub(x, b);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < N; i++) v[i] = a[i];
}

// One pencil (the lane's) through the split: v[j] = x[t + A j] on entry,
// w[s][k2] = X[(t + A s) + B k2] on exit.  S must be free on entry (every
// thread past its last read of it); the exchange rows are S + p (m + 1).
template <int M, int SIGN>
__device__ __forceinline__ void pencil_fft(C32 (&v)[PencilShape<M>::B],
                                           C32 (&w)[PencilShape<M>::B / PencilShape<M>::A][PencilShape<M>::A],
                                           C32 *S, const C32 *__restrict__ tw, int t, int p) {
  constexpr int A = PencilShape<M>::A, B = PencilShape<M>::B;
  dft_reg<B, SIGN>(v);
  if (t != 0) {
#pragma unroll
    for (int k1 = 1; k1 < B; k1++) {
      C32 f = __ldg(&tw[t * k1]);  // exp(-2 pi i t k1 / m); t k1 < m
      if (SIGN > 0) f.y = -f.y;
      v[k1] = c_mul(v[k1], f);
    }
  }
  C32 *row = S + p * (M + 1);
#pragma unroll
  for (int k1 = 0; k1 < B; k1++) row[k1 * A + t] = v[k1];
  __syncthreads();
#pragma unroll
  for (int s = 0; s < B / A; s++) {
#pragma unroll
    for (int u = 0; u < A; u++) w[s][u] = row[(t + A * s) * A + u];
    dft_reg<A, SIGN>(w[s]);
  }
}

// The 32 z rows of CTA blockIdx.x (rows r0..r0+31 of the m^2 (x, y) rows)
// from global into S (row stride m + 1) and back.
template <int M>
__device__ __forceinline__ void stage_rows_in(C32 *S, const C32 *__restrict__ src, size_t r0) {
  for (int i = threadIdx.x; i < PENCILS * M; i += blockDim.x) {
    const int r = i / M, e = i % M;
    S[r * (M + 1) + e] = src[(r0 + r) * M + e];
  }
}
template <int M>
__device__ __forceinline__ void stage_rows_out(C32 *__restrict__ dst, const C32 *S, size_t r0) {
  for (int i = threadIdx.x; i < PENCILS * M; i += blockDim.x) {
    const int r = i / M, e = i % M;
    dst[(r0 + r) * M + e] = S[r * (M + 1) + e];
  }
}

// One axis of the 3D transform over grid.y meshes (batch stride bstride).
// AXIS 0: pencils along x (stride m^2), CTA = 32 consecutive (y, z);
// AXIS 1: along y (stride m), CTA = one x and 32 consecutive z;
// AXIS 2: along z (contiguous), CTA = 32 consecutive (x, y) rows.
template <int M, int AXIS, int SIGN>
__global__ void __launch_bounds__(PENCILS *PencilShape<M>::A)
    fft_pencil_kernel(C32 *__restrict__ data, const C32 *__restrict__ tw, size_t bstride) {
  constexpr int A = PencilShape<M>::A, B = PencilShape<M>::B;
  extern __shared__ __align__(16) unsigned char pencil_smem[];
  C32 *S = reinterpret_cast<C32 *>(pencil_smem);
  const int t = threadIdx.x >> 5, p = threadIdx.x & 31;
  C32 *mesh = data + (size_t)blockIdx.y * bstride;
  const size_t M2 = (size_t)M * M;
  C32 v[B];
  size_t base = 0, stride = 0;
  const size_t r0 = (size_t)blockIdx.x * PENCILS;
  if (AXIS == 2) {
    stage_rows_in<M>(S, mesh, r0);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < B; j++) v[j] = S[p * (M + 1) + t + A * j];
    __syncthreads();
  } else {
    if (AXIS == 0) {
      base = r0 + p;
      stride = M2;
    } else {
      const int x = blockIdx.x / (M / PENCILS), z0 = (blockIdx.x % (M / PENCILS)) * PENCILS;
      base = (size_t)x * M2 + z0 + p;
      stride = M;
    }
#pragma unroll
    for (int j = 0; j < B; j++) v[j] = mesh[base + (size_t)(t + A * j) * stride];
  }
  C32 w[B / A][A];
  pencil_fft<M, SIGN>(v, w, S, tw, t, p);
  if (AXIS == 2) {
    __syncthreads();
#pragma unroll
    for (int s = 0; s < B / A; s++)
#pragma unroll
      for (int k2 = 0; k2 < A; k2++) S[p * (M + 1) + (t + A * s) + B * k2] = w[s][k2];
    __syncthreads();
    stage_rows_out<M>(mesh, S, r0);
  } else {
#pragma unroll
    for (int s = 0; s < B / A; s++)
#pragma unroll
      for (int k2 = 0; k2 < A; k2++) mesh[base + (size_t)((t + A * s) + B * k2) * stride] = w[s][k2];
  }
}

// D(i) = i - round(i / m) m with D(m/2) = 0 (dn_op in the convolution)
template <int M>
__device__ __forceinline__ float dn_pencil(int i) {
  return (i == M / 2) ? 0.0f : (float)(i < M / 2 ? i : i - M);
}

// The ik convolution and the backward z pass of the three field meshes in
// one launch: the 32 z rows of Q^ and G of the CTA are staged once as
// b = (Q^.x g s, Q^.y g s) (the products of conv_ik_kernel), and for
// d = 0, 1, 2 the rows F_d = (-D_d b.y, D_d b.x) are transformed and
// written to F + d Mtot.  grid.y = alpha batch: G + y Mtot, F + 3 y Mtot.
template <int M>
__global__ void __launch_bounds__(PENCILS *PencilShape<M>::A)
    ik_conv_zpass_kernel(const C32 *__restrict__ Qh, const float *__restrict__ G, float s, C32 *__restrict__ F,
                         size_t Mtot, const C32 *__restrict__ tw) {
  constexpr int A = PencilShape<M>::A, B = PencilShape<M>::B;
  extern __shared__ __align__(16) unsigned char pencil_smem[];
  C32 *S = reinterpret_cast<C32 *>(pencil_smem);
  const int t = threadIdx.x >> 5, p = threadIdx.x & 31;
  const size_t r0 = (size_t)blockIdx.x * PENCILS;
  G += (size_t)blockIdx.y * Mtot;
  F += (size_t)blockIdx.y * 3 * Mtot;
  for (int i = threadIdx.x; i < PENCILS * M; i += blockDim.x) {
    const int r = i / M, e = i % M;
    const size_t g = (r0 + r) * M + e;
    const C32 qv = Qh[g];
    const float gv = G[g];
    S[r * (M + 1) + e] = make_float2(qv.x * gv * s, qv.y * gv * s);
  }
  __syncthreads();
  C32 b[B];
#pragma unroll
  for (int j = 0; j < B; j++) b[j] = S[p * (M + 1) + t + A * j];
  const int row = (int)(r0 + p);
  const float d0 = dn_pencil<M>(row / M), d1 = dn_pencil<M>(row % M);
  for (int d = 0; d < 3; d++) {
    __syncthreads();  // S free: the staged rows, or the previous mesh's output rows, are read
    C32 v[B];
#pragma unroll
    for (int j = 0; j < B; j++) {
      const float dd = (d == 0) ? d0 : (d == 1) ? d1 : dn_pencil<M>(t + A * j);
      v[j] = make_float2(-dd * b[j].y, dd * b[j].x);
    }
    C32 w[B / A][A];
    pencil_fft<M, +1>(v, w, S, tw, t, p);
    __syncthreads();
#pragma unroll
    for (int s2 = 0; s2 < B / A; s2++)
#pragma unroll
      for (int k2 = 0; k2 < A; k2++) S[p * (M + 1) + (t + A * s2) + B * k2] = w[s2][k2];
    __syncthreads();
    stage_rows_out<M>(F + (size_t)d * Mtot, S, r0);
  }
}

// The last backward pass (x) of the three field meshes with the packing of
// pack_ik_kernel folded in: P[t] = (F_x, F_y, F_z, 0) of the real parts and,
// interlaced (NMESH 2), P[Mtot + t] of the imaginary parts.  Each thread
// keeps the x, y results of its own outputs in shared memory (O, private to
// the thread: no barrier) until the z results are in registers.  grid.y =
// alpha batch: F + 3 y Mtot, P + NMESH y Mtot.
template <int M, int NMESH>
__global__ void __launch_bounds__(PENCILS *PencilShape<M>::A)
    ik_xpass_pack_kernel(const C32 *__restrict__ F, size_t Mtot, float4 *__restrict__ P,
                         const C32 *__restrict__ tw) {
  constexpr int A = PencilShape<M>::A, B = PencilShape<M>::B;
  extern __shared__ __align__(16) unsigned char pencil_smem[];
  C32 *S = reinterpret_cast<C32 *>(pencil_smem);
  C32 *O = S + PENCILS * (M + 1);  // [2][M][PENCILS]
  const int t = threadIdx.x >> 5, p = threadIdx.x & 31;
  F += (size_t)blockIdx.y * 3 * Mtot;
  P += (size_t)blockIdx.y * NMESH * Mtot;
  const size_t M2 = (size_t)M * M;
  const size_t base = (size_t)blockIdx.x * PENCILS + p;
  C32 w[B / A][A];
  for (int d = 0; d < 3; d++) {
    C32 v[B];
#pragma unroll
    for (int j = 0; j < B; j++) v[j] = F[(size_t)d * Mtot + base + (size_t)(t + A * j) * M2];
    if (d > 0) __syncthreads();  // the previous mesh's exchange rows are read
    pencil_fft<M, +1>(v, w, S, tw, t, p);
    if (d < 2) {
#pragma unroll
      for (int s = 0; s < B / A; s++)
#pragma unroll
        for (int k2 = 0; k2 < A; k2++) O[((size_t)d * M + (t + A * s) + B * k2) * PENCILS + p] = w[s][k2];
    }
  }
#pragma unroll
  for (int s = 0; s < B / A; s++)
#pragma unroll
    for (int k2 = 0; k2 < A; k2++) {
      const int e = (t + A * s) + B * k2;
      const C32 fx = O[(size_t)e * PENCILS + p], fy = O[((size_t)M + e) * PENCILS + p], fz = w[s][k2];
      P[base + (size_t)e * M2] = make_float4(fx.x, fy.x, fz.x, 0.0f);
      if (NMESH == 2) P[Mtot + base + (size_t)e * M2] = make_float4(fx.y, fy.y, fz.y, 0.0f);
    }
}

template <int M>
constexpr size_t pack_smem_bytes() {
  return (size_t)PENCILS * (M + 1) * sizeof(C32) + 2 * (size_t)M * PENCILS * sizeof(C32);
}

template <int M>
constexpr size_t pencil_smem_bytes() {
  return (size_t)PENCILS * (M + 1) * sizeof(C32);
}

template <int M, int SIGN>
void launch_pencil_axes(Ctx *c, C32 *d, int nbatch, bool skip_z, bool skip_x = false) {
  const C32 *tw = reinterpret_cast<const C32 *>(c->plan.tw);
  const dim3 grid((unsigned)((size_t)M * M / PENCILS), (unsigned)nbatch);
  const int threads = PENCILS * PencilShape<M>::A;
  const size_t smem = pencil_smem_bytes<M>();
  if (!skip_z) {
    fft_pencil_kernel<M, 2, SIGN><<<grid, threads, smem, c->stream>>>(d, tw, c->M);
    c->launches++;
  }
  fft_pencil_kernel<M, 1, SIGN><<<grid, threads, smem, c->stream>>>(d, tw, c->M);
  c->launches++;
  if (!skip_x) {
    fft_pencil_kernel<M, 0, SIGN><<<grid, threads, smem, c->stream>>>(d, tw, c->M);
    c->launches++;
  }
}

template <int M>
void launch_pencil(Ctx *c, C32 *d, int nbatch, int sign, bool skip_z) {
  if (sign < 0)
    launch_pencil_axes<M, -1>(c, d, nbatch, skip_z);
  else
    launch_pencil_axes<M, +1>(c, d, nbatch, skip_z);
}

template <int M>
void launch_ik_conv_inverse(Ctx *c, const C32 *Qh, const float *G32, float s, C32 *F, int na, float4 *P) {
  const C32 *tw = reinterpret_cast<const C32 *>(c->plan.tw);
  const dim3 grid((unsigned)((size_t)M * M / PENCILS), (unsigned)na);
  const int threads = PENCILS * PencilShape<M>::A;
  ik_conv_zpass_kernel<M><<<grid, threads, pencil_smem_bytes<M>(), c->stream>>>(Qh, G32, s, F, c->M, tw);
  c->launches++;
  launch_pencil_axes<M, +1>(c, F, 3 * na, true, true);
  if (method_interlaced(c->method))
    ik_xpass_pack_kernel<M, 2><<<grid, threads, pack_smem_bytes<M>(), c->stream>>>(F, c->M, P, tw);
  else
    ik_xpass_pack_kernel<M, 1><<<grid, threads, pack_smem_bytes<M>(), c->stream>>>(F, c->M, P, tw);
  c->launches++;
}

template <int M>
int pencil_attrs() {
  P3MG_CUDA_TRY(cudaFuncSetAttribute(ik_xpass_pack_kernel<M, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)pack_smem_bytes<M>()));
  P3MG_CUDA_TRY(cudaFuncSetAttribute(ik_xpass_pack_kernel<M, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)pack_smem_bytes<M>()));
  return P3MG_OK;
}

}  // namespace

bool fft_pencil_ok(const Ctx *c) {
  return c->precision != P3MG_FP64 && (c->mesh == 32 || c->mesh == 64 || c->mesh == 128);
}

int fft_pencil(Ctx *c, void *data, int nbatch, int sign) {
  if (!fft_pencil_ok(c)) return P3MG_ERR_MESH;
  C32 *d = reinterpret_cast<C32 *>(data);
  switch (c->mesh) {
    case 32: launch_pencil<32>(c, d, nbatch, sign, false); break;
    case 64: launch_pencil<64>(c, d, nbatch, sign, false); break;
    default: launch_pencil<128>(c, d, nbatch, sign, false); break;
  }
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

int fft_pencil_init() {
  P3MG_TRY(pencil_attrs<32>());
  P3MG_TRY(pencil_attrs<64>());
  return pencil_attrs<128>();
}

int ik_conv_inverse_pencil(Ctx *c, const void *Qh, const float *G32, double s, void *F, int na, void *Pv) {
  if (!fft_pencil_ok(c)) return P3MG_ERR_MESH;
  const C32 *q = reinterpret_cast<const C32 *>(Qh);
  C32 *f = reinterpret_cast<C32 *>(F);
  float4 *P = reinterpret_cast<float4 *>(Pv);
  switch (c->mesh) {
    case 32: launch_ik_conv_inverse<32>(c, q, G32, (float)s, f, na, P); break;
    case 64: launch_ik_conv_inverse<64>(c, q, G32, (float)s, f, na, P); break;
    default: launch_ik_conv_inverse<128>(c, q, G32, (float)s, f, na, P); break;
  }
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

}  // namespace p3mg
