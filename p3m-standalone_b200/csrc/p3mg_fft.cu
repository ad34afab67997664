// Hand-written 3D FFT for the P3M meshes (radix 2/3/4/5/7, complex, in
// place, unnormalised): forward sign -1, backward +1, row-major m^3 with the
// last index fastest -- the transform the reference plans with FFTW
// (types.h:61-69, p3m-ik.c:84-88, p3m-ad.c:62-64, ...).
//
// One launch per axis.  Each CTA stages a tile of W pencils of length m
// from HBM/L2 into shared memory (coalesced along the contiguous index),
// runs the Stockham autosort passes of the mixed-radix decomposition in
// shared memory (ping-pong buffers, no bit reversal), and writes the tile
// back.  Tile layout is [element][pencil] so that the butterflies of
// neighbouring threads touch neighbouring pencils (bank-conflict free).
// The real-input transforms of methods 6 and 7 (fftw_plan_dft_r2c_3d /
// c2r_3d, p3m-ik-real.c:72-76, p3m-ad-real.c:62-64) run their z axis as an
// m/2-point complex transform of the packed real rows plus a split step
// (fft_real_z_kernel) and their x and y axes on the m/2 + 1 columns of the
// half spectrum.
#include <math.h>
#include <stdio.h>

#include "p3mg_internal.cuh"

namespace p3mg {

namespace {

constexpr int FFT_THREADS = 256;

template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) {
  C r;
  r.x = a.x + b.x;
  r.y = a.y + b.y;
  return r;
}

template <typename C>
__device__ __forceinline__ C csub(C a, C b) {
  C r;
  r.x = a.x - b.x;
  r.y = a.y - b.y;
  return r;
}

// multiply by -i (forward) or +i (backward): sign = -1 / +1
template <typename C>
__device__ __forceinline__ C mul_i(C a, int sign) {
  C r;
  if (sign < 0) {
    r.x = a.y;
    r.y = -a.x;
  } else {
    r.x = -a.y;
    r.y = a.x;
  }
  return r;
}

// twiddle exp(sign * 2 pi i e / m) from the forward table, 0 <= e < m
template <typename C>
__device__ __forceinline__ C twiddle(const C *tw, int e, int sign) {
  C t = tw[e];
  if (sign > 0) t.y = -t.y;
  return t;
}

// One Stockham pass of radix P over W pencils of length m held in
// src[e*LD + c]; writes dst.  Ns = size of the sub-transforms already done;
// j / Ns is taken as __umulhi(j, ns_magic) with ns_magic = ceil(2^32 / Ns)
// (exact for j * Ns < 2^32; here j < 2^13 and Ns <= 512).
template <typename C, int P, int W>
__device__ __forceinline__ void stockham_pass(const C *__restrict__ src, C *__restrict__ dst, const C *tw, int m,
                                              int LD, int Ns, unsigned ns_magic, int sign) {
  const int nb = m / P;  // butterflies per pencil
  const int total = nb * W;
  const int step = m / (Ns * P);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int c = t & (W - 1);
    const int j = t / W;
    const int jq = (Ns == 1) ? j : (int)__umulhi((unsigned)j, ns_magic);
    const int k = j - jq * Ns;
    C v[P];
#pragma unroll
    for (int r = 0; r < P; r++) v[r] = src[(j + r * nb) * LD + c];
    // twiddle by W_{Ns P}^{r k} = exp(sign 2 pi i r k m/(Ns P) / m); r k step < m
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < P; r++) v[r] = cmul(v[r], twiddle(tw, r * k * step, sign));
    }
    C u[P];
    if (P == 2) {
      u[0] = cadd(v[0], v[1]);
      u[1] = csub(v[0], v[1]);
    } else if (P == 4) {
      C a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
      C b0 = cadd(v[1], v[3]), b1 = mul_i(csub(v[1], v[3]), sign);
      u[0] = cadd(a0, b0);
      u[2] = csub(a0, b0);
      u[1] = cadd(a1, b1);
      u[3] = csub(a1, b1);
    } else {
      // generic P-point DFT with W_P^{s r} = tw[s r m / P]
      const int stepP = m / P;
#pragma unroll
      for (int s = 0; s < P; s++) {
        C acc = v[0];
#pragma unroll
        for (int r = 1; r < P; r++) acc = cadd(acc, cmul(v[r], twiddle(tw, ((s * r) % P) * stepP, sign)));
        u[s] = acc;
      }
    }
    const int base = jq * Ns * P + k;
#pragma unroll
    for (int s = 0; s < P; s++) dst[(base + s * Ns) * LD + c] = u[s];
  }
}

struct PassList {
  int npass;
  int radix[24];
  int ns[24];             // sub-transform size before each pass
  unsigned nsmagic[24];   // ceil(2^32 / ns) (unused for ns == 1)
  unsigned mmagic;        // ceil(2^32 / m)
};

// AXIS: 0 = x (stride m^2), 1 = y (stride m), 2 = z (contiguous); W pencils per CTA
// nz: points along z (the row pitch in complex elements): m for the full
// mesh, m/2 + 1 for the half spectrum of a real-input transform (axes 0, 1)
template <typename real, int AXIS, int W>
__global__ void __launch_bounds__(FFT_THREADS) fft_axis_kernel(typename cplx<real>::type *__restrict__ data,
                                                               const typename cplx<real>::type *__restrict__ twg, int m,
                                                               PassList passes, int sign, size_t batch_stride,
                                                               int nz) {
  typedef typename cplx<real>::type C;
  extern __shared__ unsigned char smem_raw[];
  C *tw = reinterpret_cast<C *>(smem_raw);
  const int LD = W + 1;
  C *bufA = tw + m;
  C *bufB = bufA + (size_t)m * LD;

  C *mesh = data + (size_t)blockIdx.y * batch_stride;
  for (int e = threadIdx.x; e < m; e += blockDim.x) tw[e] = twg[e];

  // which pencils does this CTA own?
  const int ngroups_inner = (nz + W - 1) / W;  // column groups along z for axes 0/1
  const int g = blockIdx.x;
  int outer = 0, c0 = 0;
  if (AXIS == 2) {
    c0 = g * W;  // first row index (rows are (i,j) pairs flattened, m*m rows)
  } else {
    outer = g / ngroups_inner;   // i (axis 1) or j (axis 0)
    c0 = (g % ngroups_inner) * W;  // first z index
  }
  const size_t M2 = (size_t)m * m;
  const int nrows = (AXIS == 2) ? (int)M2 : m;

  // load
  for (int t = threadIdx.x; t < W * m; t += blockDim.x) {
    int e, c;
    size_t addr;
    if (AXIS == 2) {
      c = (int)__umulhi((unsigned)t, passes.mmagic);
      e = t - c * m;
      addr = (size_t)(c0 + c) * m + e;
      if (c0 + c >= nrows) continue;
    } else {
      e = t / W;
      c = t & (W - 1);
      if (c0 + c >= nz) continue;
      if (AXIS == 1)
        addr = ((size_t)outer * m + e) * nz + c0 + c;
      else
        addr = ((size_t)e * m + outer) * nz + c0 + c;
    }
    bufA[e * LD + c] = mesh[addr];
  }
  __syncthreads();

  C *src = bufA, *dst = bufB;
  int Ns = 1;
  for (int p = 0; p < passes.npass; p++) {
    const int P = passes.radix[p];
    const unsigned mg = passes.nsmagic[p];
    switch (P) {
      case 2: stockham_pass<C, 2, W>(src, dst, tw, m, LD, Ns, mg, sign); break;
      case 3: stockham_pass<C, 3, W>(src, dst, tw, m, LD, Ns, mg, sign); break;
      case 4: stockham_pass<C, 4, W>(src, dst, tw, m, LD, Ns, mg, sign); break;
      case 5: stockham_pass<C, 5, W>(src, dst, tw, m, LD, Ns, mg, sign); break;
      case 7: stockham_pass<C, 7, W>(src, dst, tw, m, LD, Ns, mg, sign); break;
    }
    Ns *= P;
    __syncthreads();
    C *tmp = src;
    src = dst;
    dst = tmp;
  }

  // store
  for (int t = threadIdx.x; t < W * m; t += blockDim.x) {
    int e, c;
    size_t addr;
    if (AXIS == 2) {
      c = (int)__umulhi((unsigned)t, passes.mmagic);
      e = t - c * m;
      if (c0 + c >= nrows) continue;
      addr = (size_t)(c0 + c) * m + e;
    } else {
      e = t / W;
      c = t & (W - 1);
      if (c0 + c >= nz) continue;
      if (AXIS == 1)
        addr = ((size_t)outer * m + e) * nz + c0 + c;
      else
        addr = ((size_t)e * m + outer) * nz + c0 + c;
    }
    mesh[addr] = src[e * LD + c];
  }
}

static unsigned magic_div(int d) { return d <= 1 ? 0u : (unsigned)((0x100000000ull + (unsigned long long)d - 1) / d); }

template <typename real, int W>
void launch_axes(Ctx *c, typename cplx<real>::type *d, const typename cplx<real>::type *tw, const PassList &pl,
                 int nbatch, int sign, size_t smem) {
  const int m = c->mesh;
  const size_t stride = c->M;
  // axis order: z (contiguous), y, x -- any order gives the same transform
  dim3 g2((unsigned)((size_t)m * m / W + ((size_t)m * m % W ? 1 : 0)), nbatch);
  fft_axis_kernel<real, 2, W><<<g2, FFT_THREADS, smem, c->stream>>>(d, tw, m, pl, sign, stride, m);
  const int gi = (m + W - 1) / W;
  dim3 g01((unsigned)(m * gi), nbatch);
  fft_axis_kernel<real, 1, W><<<g01, FFT_THREADS, smem, c->stream>>>(d, tw, m, pl, sign, stride, m);
  fft_axis_kernel<real, 0, W><<<g01, FFT_THREADS, smem, c->stream>>>(d, tw, m, pl, sign, stride, m);
}

// Axes 0 and 1 of the half spectrum (nz = m/2 + 1 columns), in the order
// the transform direction needs: forward after the z pass, backward before.
template <typename real, int W>
void launch_xy_half(Ctx *c, typename cplx<real>::type *d, const typename cplx<real>::type *tw, const PassList &pl,
                    int nbatch, int sign, size_t smem) {
  const int m = c->mesh, nz = m / 2 + 1;
  const size_t stride = c->M;
  dim3 g01((unsigned)(m * ((nz + W - 1) / W)), nbatch);
  fft_axis_kernel<real, 1, W><<<g01, FFT_THREADS, smem, c->stream>>>(d, tw, m, pl, sign, stride, nz);
  fft_axis_kernel<real, 0, W><<<g01, FFT_THREADS, smem, c->stream>>>(d, tw, m, pl, sign, stride, nz);
}

// Real-input transform along z (the rows of the padded real layout, m
// reals at a pitch of m + 2 = 2 (m/2 + 1) reals, transformed in place).
// Forward (r2c): the m reals of a row are read as m/2 complex values
// z_k = x_2k + i x_2k+1, transformed with an m/2-point complex DFT (the
// Stockham passes of `half`), and split into the m/2 + 1 outputs
//   X_k = E_k + W_m^k O_k,  E_k = (Z_k + conj Z_{m/2-k}) / 2,
//   O_k = (Z_k - conj Z_{m/2-k}) / (2 i),  Z_{m/2} = Z_0.
// Backward (c2r, unnormalised, sign +1): the inverse of those steps,
//   Z'_k = E'_k + i O'_k,  E'_k = X_k + conj X_{m/2-k},
//   O'_k = (X_k - conj X_{m/2-k}) W_m^{-k},
// (imaginary parts of X_0 and X_{m/2}, zero for the spectrum of a real
// mesh up to rounding, are dropped as a c2r transform does), an m/2-point
// backward DFT, and x_2n = Re z_n, x_2n+1 = Im z_n.  W rows per CTA.
template <typename real, int W, bool FORWARD>
__global__ void __launch_bounds__(FFT_THREADS) fft_real_z_kernel(real *__restrict__ data,
                                                                 const typename cplx<real>::type *__restrict__ twg,
                                                                 int m, PassList half, size_t batch_stride) {
  typedef typename cplx<real>::type C;
  extern __shared__ unsigned char smem_raw[];
  const int mh = m / 2, H = mh + 1;
  const int LD = W + 1;
  C *tw = reinterpret_cast<C *>(smem_raw);  // exp(-2 pi i e / m), e < m
  C *twh = tw + m;                          // exp(-2 pi i e / mh), e < mh
  C *bufA = twh + mh;
  C *bufB = bufA + (size_t)H * LD;
  for (int e = threadIdx.x; e < m; e += blockDim.x) {
    const C t = twg[e];
    tw[e] = t;
    if (!(e & 1)) twh[e >> 1] = t;
  }
  C *rows = reinterpret_cast<C *>(data + (size_t)blockIdx.y * batch_stride);  // H complex per row
  const int r0 = blockIdx.x * W;
  const int nrows = m * m;
  const int sign = FORWARD ? -1 : +1;
  __syncthreads();
  if (FORWARD) {
    for (int t = threadIdx.x; t < W * mh; t += blockDim.x) {
      const int c = t / mh, e = t - c * mh;
      if (r0 + c < nrows) bufA[e * LD + c] = rows[(size_t)(r0 + c) * H + e];
    }
  } else {
    for (int t = threadIdx.x; t < W * H; t += blockDim.x) {
      const int c = t / H, e = t - c * H;
      if (r0 + c < nrows) {
        C v = rows[(size_t)(r0 + c) * H + e];
        if (e == 0 || e == mh) v.y = (real)0;
        bufB[e * LD + c] = v;
      }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < W * mh; t += blockDim.x) {
      const int e = t / W, c = t & (W - 1);
      const C a = bufB[e * LD + c], b = bufB[(mh - e) * LD + c];
      C Ep, Op, w = tw[e];
      Ep.x = a.x + b.x;
      Ep.y = a.y - b.y;
      Op.x = a.x - b.x;
      Op.y = a.y + b.y;
      w.y = -w.y;  // W_m^{-e}
      Op = cmul(Op, w);
      C z;
      z.x = Ep.x - Op.y;  // E' + i O'
      z.y = Ep.y + Op.x;
      bufA[e * LD + c] = z;
    }
  }
  __syncthreads();
  C *src = bufA, *dst = bufB;
  int Ns = 1;
  for (int p = 0; p < half.npass; p++) {
    const int P = half.radix[p];
    const unsigned mg = half.nsmagic[p];
    switch (P) {
      case 2: stockham_pass<C, 2, W>(src, dst, twh, mh, LD, Ns, mg, sign); break;
      case 3: stockham_pass<C, 3, W>(src, dst, twh, mh, LD, Ns, mg, sign); break;
      case 4: stockham_pass<C, 4, W>(src, dst, twh, mh, LD, Ns, mg, sign); break;
      case 5: stockham_pass<C, 5, W>(src, dst, twh, mh, LD, Ns, mg, sign); break;
      case 7: stockham_pass<C, 7, W>(src, dst, twh, mh, LD, Ns, mg, sign); break;
    }
    Ns *= P;
    __syncthreads();
    C *tmp = src;
    src = dst;
    dst = tmp;
  }
  if (FORWARD) {
    for (int t = threadIdx.x; t < W * H; t += blockDim.x) {
      const int c = t / H, e = t - c * H;
      if (r0 + c >= nrows) continue;
      const C a = src[(e == mh ? 0 : e) * LD + c], b = src[(e == 0 ? 0 : mh - e) * LD + c];
      // E = (a + conj b) / 2, O = (a - conj b) / (2 i)
      C E, O;
      E.x = (real)0.5 * (a.x + b.x);
      E.y = (real)0.5 * (a.y - b.y);
      O.x = (real)0.5 * (a.y + b.y);
      O.y = (real)-0.5 * (a.x - b.x);
      const C wo = cmul(O, tw[e == mh ? 0 : e]);
      C X;
      if (e == mh) {
        X.x = E.x - O.x;  // W_m^{m/2} = -1
        X.y = E.y - O.y;
      } else {
        X.x = E.x + wo.x;
        X.y = E.y + wo.y;
      }
      rows[(size_t)(r0 + c) * H + e] = X;
    }
  } else {
    for (int t = threadIdx.x; t < W * mh; t += blockDim.x) {
      const int c = t / mh, e = t - c * mh;
      if (r0 + c < nrows) rows[(size_t)(r0 + c) * H + e] = src[e * LD + c];
    }
  }
}

template <typename real>
int launch_fft3d(Ctx *c, void *data, int nbatch, int sign) {
  typedef typename cplx<real>::type C;
  const int m = c->mesh;
  PassList pl;
  pl.npass = c->plan.npass;
  int ns = 1;
  for (int i = 0; i < pl.npass; i++) {
    pl.radix[i] = c->plan.radix[i];
    pl.ns[i] = ns;
    pl.nsmagic[i] = magic_div(ns);
    ns *= pl.radix[i];
  }
  pl.mmagic = magic_div(m);
  // pencils per tile: 128 B of contiguous data per row segment at least
  int W = (sizeof(real) == 8) ? 8 : 16;
  if (c->fft_w == 4 || c->fft_w == 8 || c->fft_w == 16) W = c->fft_w;  // set by the tile autotuner
  if (m * W * 2 * (int)sizeof(C) > 160 * 1024) W = 4;
  const size_t smem = (size_t)m * sizeof(C) + 2 * (size_t)m * (W + 1) * sizeof(C);
  C *d = reinterpret_cast<C *>(data);
  const C *tw = reinterpret_cast<const C *>(c->plan.tw);
  if (W == 16)
    launch_axes<real, 16>(c, d, tw, pl, nbatch, sign, smem);
  else if (W == 8)
    launch_axes<real, 8>(c, d, tw, pl, nbatch, sign, smem);
  else
    launch_axes<real, 4>(c, d, tw, pl, nbatch, sign, smem);
  c->launches += 3;
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

template <typename real, int W>
void launch_real_z(Ctx *c, real *d, const typename cplx<real>::type *tw, const PassList &half, int nbatch,
                   bool forward, size_t smem) {
  const int m = c->mesh;
  const dim3 g((unsigned)(((size_t)m * m + W - 1) / W), nbatch);
  const size_t stride = 2 * c->M;  // reals
  if (forward)
    fft_real_z_kernel<real, W, true><<<g, FFT_THREADS, smem, c->stream>>>(d, tw, m, half, stride);
  else
    fft_real_z_kernel<real, W, false><<<g, FFT_THREADS, smem, c->stream>>>(d, tw, m, half, stride);
}

static PassList pass_list(const int *radix, int npass, int m) {
  PassList pl;
  pl.npass = npass;
  int ns = 1;
  for (int i = 0; i < npass; i++) {
    pl.radix[i] = radix[i];
    pl.ns[i] = ns;
    pl.nsmagic[i] = magic_div(ns);
    ns *= radix[i];
  }
  pl.mmagic = magic_div(m);
  return pl;
}

// 3D real-input transform of nbatch meshes (slot stride M complex): the
// real mesh in the padded layout (row pitch m + 2 reals) <-> the half
// spectrum m x m x (m/2 + 1) (row pitch m/2 + 1 complex), in place.
template <typename real>
int launch_fft3d_real(Ctx *c, void *data, int nbatch, int sign) {
  typedef typename cplx<real>::type C;
  const int m = c->mesh, mh = m / 2;
  if (m % 2 || mh < 1) return P3MG_ERR_MESH;
  int hr[24], hn = 0;
  if (fft_factor(mh, hr, &hn)) return P3MG_ERR_MESH;
  const PassList pl = pass_list(c->plan.radix, c->plan.npass, m);
  const PassList half = pass_list(hr, hn, mh);
  int W = (sizeof(real) == 8) ? 8 : 16;
  if (c->fft_w == 4 || c->fft_w == 8 || c->fft_w == 16) W = c->fft_w;
  if (m * W * 2 * (int)sizeof(C) > 160 * 1024) W = 4;
  const size_t smem_xy = (size_t)m * sizeof(C) + 2 * (size_t)m * (W + 1) * sizeof(C);
  const size_t smem_z = (size_t)(m + mh) * sizeof(C) + 2 * (size_t)(mh + 1) * (W + 1) * sizeof(C);
  C *d = reinterpret_cast<C *>(data);
  real *dr = reinterpret_cast<real *>(data);
  const C *tw = reinterpret_cast<const C *>(c->plan.tw);
  const bool fwd = sign < 0;
  if (fwd) {
    if (W == 16) launch_real_z<real, 16>(c, dr, tw, half, nbatch, true, smem_z);
    else if (W == 8) launch_real_z<real, 8>(c, dr, tw, half, nbatch, true, smem_z);
    else launch_real_z<real, 4>(c, dr, tw, half, nbatch, true, smem_z);
  }
  if (W == 16) launch_xy_half<real, 16>(c, d, tw, pl, nbatch, sign, smem_xy);
  else if (W == 8) launch_xy_half<real, 8>(c, d, tw, pl, nbatch, sign, smem_xy);
  else launch_xy_half<real, 4>(c, d, tw, pl, nbatch, sign, smem_xy);
  if (!fwd) {
    if (W == 16) launch_real_z<real, 16>(c, dr, tw, half, nbatch, false, smem_z);
    else if (W == 8) launch_real_z<real, 8>(c, dr, tw, half, nbatch, false, smem_z);
    else launch_real_z<real, 4>(c, dr, tw, half, nbatch, false, smem_z);
  }
  c->launches += 3;
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

template <typename real, int W>
int set_smem_limits_w() {
  P3MG_CUDA_TRY(cudaFuncSetAttribute(fft_axis_kernel<real, 0, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  P3MG_CUDA_TRY(cudaFuncSetAttribute(fft_axis_kernel<real, 1, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  P3MG_CUDA_TRY(cudaFuncSetAttribute(fft_axis_kernel<real, 2, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  P3MG_CUDA_TRY(cudaFuncSetAttribute(fft_real_z_kernel<real, W, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  P3MG_CUDA_TRY(cudaFuncSetAttribute(fft_real_z_kernel<real, W, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  return P3MG_OK;
}

template <typename real>
int set_smem_limits() {
  P3MG_TRY((set_smem_limits_w<real, 4>()));
  P3MG_TRY((set_smem_limits_w<real, 8>()));
  P3MG_TRY((set_smem_limits_w<real, 16>()));
  return P3MG_OK;
}

}  // namespace

// Factor m into radices 4, 2, 3, 5, 7 (largest supported first); 0 on
// success, -1 when m has another prime factor.
int fft_factor(int m, int *radix, int *npass) {
  int k = 0;
  int r = m;
  while (r % 4 == 0) {
    radix[k++] = 4;
    r /= 4;
  }
  const int pr[4] = {2, 3, 5, 7};
  for (int i = 0; i < 4; i++)
    while (r % pr[i] == 0) {
      radix[k++] = pr[i];
      r /= pr[i];
    }
  *npass = k;
  return r == 1 ? 0 : -1;
}

int fft_plan_init(Ctx *c) {
  const int m = c->mesh;
  if (fft_factor(m, c->plan.radix, &c->plan.npass)) return P3MG_ERR_MESH;
  c->plan.m = m;
  // twiddle table exp(-2 pi i e/m), computed in long double on the host
  const bool dbl = (c->precision == P3MG_FP64);
  const size_t bytes = (size_t)m * (dbl ? sizeof(double2) : sizeof(float2));
  void *host = malloc(bytes);
  for (int e = 0; e < m; e++) {
    long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)e / (long double)m;
    double cr = (double)cosl(a), ci = (double)(-sinl(a));
    if (dbl) {
      ((double2 *)host)[e] = make_double2(cr, ci);
    } else {
      ((float2 *)host)[e] = make_float2((float)cr, (float)ci);
    }
  }
  cudaError_t e = cudaMalloc(&c->plan.tw, bytes);
  if (e != cudaSuccess) {
    free(host);
    record_cuda_error(e);
    return P3MG_ERR_ALLOC;
  }
  e = cudaMemcpy(c->plan.tw, host, bytes, cudaMemcpyHostToDevice);
  free(host);
  P3MG_CUDA_TRY(e);
  if (dbl) {
    P3MG_TRY(set_smem_limits<double>());
  } else {
    P3MG_TRY(set_smem_limits<float>());
    P3MG_TRY(fft_pencil_init());
  }
  return P3MG_OK;
}

void fft_plan_free(Ctx *c) {
  if (c->plan.tw) cudaFree(c->plan.tw);
  c->plan.tw = nullptr;
}

bool fft_real_ok(const Ctx *c) {
  int r[24], k = 0;
  return c->mesh % 2 == 0 && c->mesh >= 4 && fft_factor(c->mesh / 2, r, &k) == 0;
}

int fft3d_real(Ctx *c, void *data, int nbatch, int sign) {
  if (c->precision == P3MG_FP64) return launch_fft3d_real<double>(c, data, nbatch, sign);
  return launch_fft3d_real<float>(c, data, nbatch, sign);
}

int fft3d(Ctx *c, void *data, int nbatch, int sign) {
  if (c->fft_w == 0 && fft_pencil_ok(c)) return fft_pencil(c, data, nbatch, sign);
  if (c->precision == P3MG_FP64) return launch_fft3d<double>(c, data, nbatch, sign);
  return launch_fft3d<float>(c, data, nbatch, sign);
}

}  // namespace p3mg
