// Templated kernels and launchers of the k-space pipeline (included by
// p3mg_assign_f64.cu and p3mg_assign_f32.cu, one precision each).
#pragma once
#include <math.h>

#include <type_traits>

#include "p3mg_internal.cuh"

namespace p3mg {
namespace assign_impl {
namespace {

constexpr int ASSIGN_THREADS = 256;

__host__ __device__ inline int brick_tile(int B, int cao, int nmesh) { return B + cao - 1 + (nmesh == 2 ? 1 : 0); }

// ---------------------------------------------------------------- scatter

// particles staged per round of the scatter (weights and tile offsets)
constexpr int SCATTER_CHUNK = 128;

// staged weight record of one (particle, mesh): W_x (charge and, FP32, the
// tile's fixed-point scale folded in), W_y, W_z, padded to a multiple of 4
// reals so W_x reads as 16-byte vectors
template <int CAO>
__host__ __device__ constexpr int scatter_rec() {
  return (3 * CAO + 3) & ~3;
}

template <typename real, int CAO, int NMESH>
__host__ __device__ constexpr size_t scatter_stage_bytes() {
  return (size_t)NMESH * SCATTER_CHUNK * (scatter_rec<CAO>() * sizeof(real) + sizeof(int)) + 16;
}

// One CTA per mesh brick.  Round by round, SCATTER_CHUNK particles of the
// brick are staged: one thread per particle computes its stencil origin in
// the tile and its B-spline weights (charge folded into the x weights) for
// each mesh.  Then each warp deposits whole particles: each lane owns one
// (b, c) column of the stencil (cao^2 columns over one or two passes of 32
// lanes), forms Wy_b Wz_c once and adds Wx_a Wy_b Wz_c for a = 0..cao-1
// down the column; the host picks the row pitch so that the 32 columns of a
// pass fall in 32 different banks (16 per half-warp for 8-byte elements),
// so one instruction's shared-memory atomics neither collide nor conflict.
// The tile is added to the global mesh at the end (periodic wrap, one
// global atomic per non-zero tile point).
//
// FP32: the tile accumulates in 32-bit fixed point with the brick's own
// scale S = (0.999 * 2^31 - n_brick / 2) / (sum |q| w_max^3) over the
// brick's particles, w_max the largest weight of the order (0.511 for
// cao 7) -- shared-memory integer adds are single native atomics where
// float adds are not.  No tile point can overflow: its sum is at most
// sum |q| w_max^3 plus half a unit of rounding per contribution.  The
// resolution is below the FP32 rounding of the contributions for the few
// hundred particles of a brick at density 1; integer sums also make the
// tile independent of the order of the atomics.  FP64 accumulates doubles.
// EXACT: B-spline weights at the exact in-cell offset instead of the
// reference's 2^-17 table bins (the energy and its adjoint, which must be
// smooth in the positions); the stencil base is the same.
template <typename real, int CAO, int NMESH, bool EXACT = false>
__global__ void __launch_bounds__(ASSIGN_THREADS) scatter_kernel(const double4 *__restrict__ sxyzq,
                                                                  const int *__restrict__ start, int m, int B, int nb,
                                                                  double Hi, double shift, int SR, int SP,
                                                                  const int4 *__restrict__ lanetab,
                                                                  real *__restrict__ Qr, int RP, int ES) {
  constexpr int NPASS = (CAO * CAO + 31) / 32;  // passes of 32 (b, c) columns
  constexpr bool FIXED = std::is_same<real, float>::value;
  typedef typename std::conditional<FIXED, int, real>::type acc_t;
  static_assert(sizeof(acc_t) == sizeof(real), "tile layout");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int T = brick_tile(B, CAO, NMESH);
  const int T3 = T * SP;  // tile elements: T planes of pitch SP, rows of pitch SR
  constexpr int REC = scatter_rec<CAO>();
  acc_t *tile0 = reinterpret_cast<acc_t *>(smem_raw);
  acc_t *tile1 = tile0 + T3;
  // [NMESH*CHUNK][REC] weight records, 16-byte aligned
  real *sw = reinterpret_cast<real *>((reinterpret_cast<uintptr_t>(tile0 + NMESH * T3) + 15) & ~(uintptr_t)15);
  int *soff = reinterpret_cast<int *>(sw + NMESH * SCATTER_CHUNK * REC);  // tile offset of the stencil origin
  const int bid = blockIdx.x;
  const int p0 = start[bid * B * B * B], p1 = start[(bid + 1) * B * B * B];
  if (p0 == p1) return;
  for (int t = threadIdx.x; t < NMESH * T3; t += blockDim.x) tile0[t] = (acc_t)0;
  // FP32: fixed-point scale of this brick from sum |q| (rounded up a little
  // so the bound survives the summation's rounding) and the largest weight
  real scale = (real)1, inv_scale = (real)1;
  if (FIXED) {
    // max over the in-cell offset of the order-CAO weights, rounded up
    constexpr double wmax = CAO <= 2 ? 1.0 : CAO == 3 ? 0.75 : CAO == 4 ? 0.66667 : CAO == 5 ? 0.59896 : CAO == 6 ? 0.55001 : 0.51103;
    __shared__ double qsum_w[ASSIGN_THREADS / 32];
    double qs = 0.0;
    for (int p = p0 + (int)threadIdx.x; p < p1; p += blockDim.x) qs += fabs(sxyzq[p].w);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) qs += __shfl_xor_sync(0xffffffffu, qs, o);
    if ((threadIdx.x & 31) == 0) qsum_w[threadIdx.x >> 5] = qs;
    __syncthreads();
    double R = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) R += qsum_w[w];
    const double bound = R * (1.0 + 1e-6) * wmax * wmax * wmax;
    const double units = 0.999 * 2147483648.0 - 0.5 * (double)(p1 - p0);
    scale = bound > 0.0 ? (real)(units / bound) : (real)0;
    inv_scale = bound > 0.0 ? (real)(bound / units) : (real)0;
  }
  const int bz = bid % nb, by = (bid / nb) % nb, bx = bid / (nb * nb);
  const int o0 = bx * B, o1 = by * B, o2 = bz * B;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  // This lane's stencil columns: tile offset b*SR + c and (b, c), or b < 0
  // (scatter_lane_table).
  int loff[NPASS], lb[NPASS], lc[NPASS];
#pragma unroll
  for (int ps = 0; ps < NPASS; ps++) {
    const int4 e = lanetab[ps * 32 + lane];
    loff[ps] = e.x;
    lb[ps] = e.y;
    lc[ps] = e.z;
  }
  for (int pc = p0; pc < p1; pc += SCATTER_CHUNK) {
    const int cnt = min(SCATTER_CHUNK, p1 - pc);
    __syncthreads();
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
      const double4 r = sxyzq[pc + t];
#pragma unroll
      for (int ii = 0; ii < NMESH; ii++) {
        int base[3], arg[3];
        double uu[3];
        mesh_geometry_u(r.x, Hi, shift, ii, m, &base[0], &arg[0], &uu[0]);
        mesh_geometry_u(r.y, Hi, shift, ii, m, &base[1], &arg[1], &uu[1]);
        mesh_geometry_u(r.z, Hi, shift, ii, m, &base[2], &arg[2], &uu[2]);
        int rel0 = base[0] - o0, rel1 = base[1] - o1, rel2 = base[2] - o2;
        rel0 += (rel0 < 0) ? m : 0;
        rel1 += (rel1 < 0) ? m : 0;
        rel2 += (rel2 < 0) ? m : 0;
        real w[3][CAO];
#pragma unroll
        for (int d = 0; d < 3; d++) {
          if (EXACT)
            bspline_weights_u<real, CAO, false>((real)uu[d], w[d], nullptr);
          else
            bspline_weights<real, CAO, false>(arg[d], w[d], nullptr);
        }
        const int v = t * NMESH + ii;
        real *dst = sw + (size_t)v * REC;
#pragma unroll
        for (int j = 0; j < CAO; j++) {
          // q * W_x (the reference's first product), times the fixed-point scale
          dst[j] = FIXED ? ((real)r.w * w[0][j]) * scale : (real)r.w * w[0][j];
          dst[CAO + j] = w[1][j];
          dst[2 * CAO + j] = w[2][j];
        }
        soff[v] = rel0 * SP + rel1 * SR + rel2;
      }
    }
    __syncthreads();
    for (int v = warp; v < cnt * NMESH; v += nwarp) {
      const real *wv = sw + (size_t)v * REC;
      acc_t *tile = (NMESH == 2 && (v & 1)) ? tile1 : tile0;
      acc_t *org = tile + soff[v];
      // W_x as 16-byte vectors (the record's first CAO reals, padded)
      real wx[(CAO + 3) & ~3];
      if constexpr (FIXED) {
#pragma unroll
        for (int a = 0; a < CAO; a += 4) {
          const float4 t4 = *reinterpret_cast<const float4 *>(wv + a);
          wx[a] = t4.x;
          wx[a + 1] = t4.y;
          wx[a + 2] = t4.z;
          wx[a + 3] = t4.w;
        }
      } else {
#pragma unroll
        for (int a = 0; a < CAO; a += 2) {
          const double2 t2 = *reinterpret_cast<const double2 *>(wv + a);
          wx[a] = t2.x;
          if (a + 1 < ((CAO + 3) & ~3)) wx[a + 1] = t2.y;
        }
      }
#pragma unroll
      for (int ps = 0; ps < NPASS; ps++) {
        if (lb[ps] >= 0) {
          const real wyz = wv[CAO + lb[ps]] * wv[2 * CAO + lc[ps]];
          acc_t *col = org + loff[ps];
#pragma unroll
          for (int a = 0; a < CAO; a++) {
            if constexpr (FIXED)
              atomicAdd(col + a * SP, __float2int_rn(wx[a] * wyz));
            else
              atomicAdd(col + a * SP, wx[a] * wyz);
          }
        }
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < T * T * T; t += blockDim.x) {
    const int c = t % T, b = (t / T) % T, a = t / (T * T);
    const int e = a * SP + b * SR + c;
    int gi = o0 + a, gj = o1 + b, gk = o2 + c;
    gi -= (gi >= m) ? m : 0;
    gj -= (gj >= m) ? m : 0;
    gk -= (gk >= m) ? m : 0;
    if (gi >= m) gi %= m;
    if (gj >= m) gj %= m;
    if (gk >= m) gk %= m;
    // complex mesh (RP = m, ES = 2: real part, imaginary part) or the
    // padded real layout of the r2c methods (RP = m + 2, ES = 1)
    const size_t g = (((size_t)gi * m + gj) * RP + gk) * ES;
    const real v0 = FIXED ? (real)tile0[e] * inv_scale : (real)tile0[e];
    if (NMESH == 2) {
      const real v1 = FIXED ? (real)tile1[e] * inv_scale : (real)tile1[e];
      if (v0 != (real)0) atomicAdd(&Qr[g], v0);
      if (v1 != (real)0) atomicAdd(&Qr[g + 1], v1);
    } else {
      if (v0 != (real)0) atomicAdd(&Qr[g], v0);
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
  // alpha batch (grid.y): G and the three field meshes of entry y
  G += (size_t)blockIdx.y * M;
  F += (size_t)blockIdx.y * 3 * M;
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
// Qout = G Qin (in place when Qout == Qin); alpha batch over grid.y with
// G and Qout of entry y
__global__ void conv_ad_kernel(const typename cplx<real>::type *Qin, const Gt *__restrict__ G, size_t M,
                               typename cplx<real>::type *Qout) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M) return;
  G += (size_t)blockIdx.y * M;
  Qout += (size_t)blockIdx.y * M;
  const real g = (real)G[t];
  typename cplx<real>::type v = Qin[t];
  v.x *= g;
  v.y *= g;
  Qout[t] = v;
}

// The same convolutions on the half spectrum of the real-input methods
// (m x m x (m/2 + 1), row pitch m/2 + 1): the loops of P3M_ik_r / P3M_ad_r
// run k < m/2 + 1 and index G with the full-mesh r_ind = (i m + j) m + k
// (p3m-ik-real.c:113-136, p3m-ad-real.c:92-101).
template <typename real, typename Gt>
__global__ void conv_ik_half_kernel(const typename cplx<real>::type *__restrict__ Q, const Gt *__restrict__ G, int m,
                                    double twopi_over_L, size_t M, typename cplx<real>::type *__restrict__ F) {
  typedef typename cplx<real>::type C;
  const int H = m / 2 + 1;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)m * m * H) return;
  G += (size_t)blockIdx.y * M;
  F += (size_t)blockIdx.y * 3 * M;
  const int k = (int)(t % H);
  const size_t ij = t / H;
  const int j = (int)(ij % m), i = (int)(ij / m);
  const C qv = Q[t];
  const real g = (real)G[ij * m + k];
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
__global__ void conv_ad_half_kernel(const typename cplx<real>::type *Qin, const Gt *__restrict__ G, int m, size_t M,
                                    typename cplx<real>::type *Qout) {
  const int H = m / 2 + 1;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)m * m * H) return;
  G += (size_t)blockIdx.y * M;
  Qout += (size_t)blockIdx.y * M;
  const real g = (real)G[(t / H) * m + t % H];
  typename cplx<real>::type v = Qin[t];
  v.x *= g;
  v.y *= g;
  Qout[t] = v;
}

// ---------------------------------------------------------------- gather

// Pack the three ik field meshes for the back-interpolation: per mesh point
// one vector (F_x, F_y, F_z, 0) of the unshifted mesh (real parts) and, for
// interlaced methods, one of the shifted mesh (imaginary parts), so the
// gather reads one 16-byte (FP32) / 32-byte (FP64) vector per stencil point.
template <typename real, int NMESH>
__global__ void pack_ik_kernel(const typename cplx<real>::type *__restrict__ F, size_t M,
                               typename cplx<real>::vec4 *__restrict__ P) {
  typedef typename cplx<real>::vec4 V;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M) return;
  F += (size_t)blockIdx.y * 3 * M;  // alpha batch (grid.y)
  P += (size_t)blockIdx.y * NMESH * M;
  const typename cplx<real>::type f0 = F[t], f1 = F[M + t], f2 = F[2 * M + t];
  V v;
  v.x = f0.x;
  v.y = f1.x;
  v.z = f2.x;
  v.w = (real)0;
  P[t] = v;
  if (NMESH == 2) {
    v.x = f0.y;
    v.y = f1.y;
    v.z = f2.y;
    P[M + t] = v;
  }
}

// Pack the three real field meshes of method 6 (padded layout, row pitch
// m + 2, one per slot of M complex) into (F_x, F_y, F_z, 0) per mesh point.
template <typename real>
__global__ void pack_ik_real_kernel(const real *__restrict__ F, int m, size_t M,
                                    typename cplx<real>::vec4 *__restrict__ P) {
  typedef typename cplx<real>::vec4 V;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M) return;
  F += (size_t)blockIdx.y * 6 * M;  // alpha batch (grid.y): 3 slots of 2M reals
  P += (size_t)blockIdx.y * M;
  const size_t r = (t / m) * (m + 2) + t % m;
  V v;
  v.x = F[r];
  v.y = F[2 * M + r];
  v.z = F[4 * M + r];
  v.w = (real)0;
  P[t] = v;
}

// ik: f_d -= scale * q W F_d ; ad: f -= scale * phi * q/L * grad W.
// scale = pref (one mesh) or pref/2 (interlaced, charge-assign.c:646-806).
// One thread per brick-sorted particle; ik reads the packed fields (Fv =
// P), ad the potential in the complex mesh (Fv = Q).
template <typename real, int CAO, int NMESH, bool AD>
__global__ void __launch_bounds__(ASSIGN_THREADS) gather_kernel(const double4 *__restrict__ sxyzq,
                                                                 const int *__restrict__ sidx, int np, int m,
                                                                 double Hi, double shift, double pref, double Leni,
                                                                 const void *__restrict__ Fv, size_t M,
                                                                 double *__restrict__ fk, int n, int RP, int ES) {
  typedef typename cplx<real>::type C;
  typedef typename cplx<real>::vec4 V;
  // alpha batch (grid.y): the potential (ad) or packed fields (ik) and the
  // forces of entry y
  // ad: the potential as reals -- complex mesh (RP = m, ES = 2) or the
  // padded real layout of the r2c methods (RP = m + 2, ES = 1)
  const real *__restrict__ Fr = reinterpret_cast<const real *>(Fv) + (size_t)blockIdx.y * 2 * M;
  const V *__restrict__ P = reinterpret_cast<const V *>(Fv) + (size_t)blockIdx.y * NMESH * M;
  fk += (size_t)blockIdx.y * 3 * (size_t)n;
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
          const V *__restrict__ Pm = P + (ii ? M : 0) + rowb;
#pragma unroll
          for (int c = 0; c < CAO; c++) {
            int gk = base[2] + c;
            gk -= (gk >= m) ? m : 0;
            const real Bw = scale * (qab * wz[c]);
            const V f = Pm[gk];
            acc0 -= f.x * Bw;
            acc1 -= f.y * Bw;
            acc2 -= f.z * Bw;
          }
        } else {
          const size_t rowr = ((size_t)gi * m + gj) * RP;
#pragma unroll
          for (int c = 0; c < CAO; c++) {
            int gk = base[2] + c;
            gk -= (gk >= m) ? m : 0;
            const real Bp = scale * Fr[(rowr + gk) * ES + ii];
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

// Piecewise polynomials of the order-CAO cardinal B-spline: c[k * CAO + i]
// is the coefficient of u^i of M_CAO on [k, k + 1) in the local variable u
// = x - k, so the charge-assignment weight of stencil point j at in-cell
// offset u is w_j(u) = M_CAO(u + CAO - 1 - j) = sum_i c[(CAO-1-j) CAO + i] u^i
// (the same weights as bspline_weights_u).  From the recursion on the
// pieces, P_{n,k}(u) = [(k + u) P_{n-1,k}(u) + (n - k - u) P_{n-1,k-1}(u)] / (n - 1),
// P_{1,0} = 1 (de Boor), evaluated on the host in double.
template <typename real>
struct PieceCoef {
  real c[P3MG_MAX_CAO * P3MG_MAX_CAO];
};

template <typename real>
inline PieceCoef<real> bspline_pieces(int cao) {
  double P[P3MG_MAX_CAO][P3MG_MAX_CAO] = {{0.0}};  // [piece][power] of the current order
  P[0][0] = 1.0;
  for (int n = 2; n <= cao; n++) {
    double Q[P3MG_MAX_CAO][P3MG_MAX_CAO] = {{0.0}};
    for (int k = 0; k < n; k++) {
      for (int i = 0; i < n - 1; i++) {
        if (k <= n - 2) {  // (k + u) P_{n-1,k}
          Q[k][i] += k * P[k][i];
          Q[k][i + 1] += P[k][i];
        }
        if (k >= 1) {  // (n - k - u) P_{n-1,k-1}
          Q[k][i] += (n - k) * P[k - 1][i];
          Q[k][i + 1] -= P[k - 1][i];
        }
      }
      for (int i = 0; i < n; i++) Q[k][i] /= (double)(n - 1);
    }
    for (int k = 0; k < P3MG_MAX_CAO; k++)
      for (int i = 0; i < P3MG_MAX_CAO; i++) P[k][i] = Q[k][i];
  }
  PieceCoef<real> out;
  for (int k = 0; k < P3MG_MAX_CAO * P3MG_MAX_CAO; k++) out.c[k] = (real)0;
  for (int k = 0; k < cao; k++)
    for (int i = 0; i < cao; i++) out.c[k * cao + i] = (real)P[k][i];
  return out;
}

// ik back-interpolation with the lanes on the z offsets of the stencil:
// LPP lanes per particle (8 or 16), lane l < NMESH * CAO owns mesh
// ii = l / CAO and z offset c = l % CAO and sums its CAO x CAO (a, b)
// column.  For every (a, b) the CAO lanes of one (particle, mesh) read CAO
// consecutive field vectors, so a load instruction touches a few whole
// cache lines where one thread per particle (gather_kernel) touches one
// scattered line per lane.  Lane c evaluates only the weights of stencil
// index c (one polynomial piece, Horner) on the three axes and takes the
// others from its group's lanes by shuffles; the lane sums are reduced over
// the particle's lanes at the end.  Same geometry, table bins and
// prefactors as gather_kernel.
template <typename real, int CAO, int NMESH>
__global__ void __launch_bounds__(ASSIGN_THREADS) gather_lanes_kernel(const double4 *__restrict__ sxyzq,
                                                                       const int *__restrict__ sidx, int np, int m,
                                                                       double Hi, double shift, double pref,
                                                                       const void *__restrict__ Fv, size_t M,
                                                                       double *__restrict__ fk, int n,
                                                                       const PieceCoef<real> pcoef) {
  typedef typename cplx<real>::vec4 V;
  constexpr int LPP = (NMESH * CAO <= 8) ? 8 : 16;
  static_assert(NMESH * CAO <= 16, "lanes per particle");
  constexpr int PPW = 32 / LPP;
  __shared__ real coef[CAO * CAO];
  if (threadIdx.x < CAO * CAO) coef[threadIdx.x] = pcoef.c[threadIdx.x];
  __syncthreads();
  const V *__restrict__ P = reinterpret_cast<const V *>(Fv) + (size_t)blockIdx.y * NMESH * M;
  fk += (size_t)blockIdx.y * 3 * (size_t)n;
  const int lane = threadIdx.x & 31;
  const int p = (int)(((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * PPW + lane / LPP;
  const int l = lane % LPP;
  const bool act = p < np && l < NMESH * CAO;
  const int lc = act ? l : 0;  // idle lanes mirror lane 0 of their group (their shuffles stay in range)
  const int ii = (NMESH == 2 && lc >= CAO) ? 1 : 0;
  const int c = lc - ii * CAO;
  const int src0 = (lane & ~(LPP - 1)) + ii * CAO;  // lane holding stencil index 0 of this (particle, mesh)
  const double4 r = sxyzq[p < np ? p : (np > 0 ? np - 1 : 0)];
  int base[3], arg[3];
  mesh_geometry(r.x, Hi, shift, ii, m, &base[0], &arg[0]);
  mesh_geometry(r.y, Hi, shift, ii, m, &base[1], &arg[1]);
  mesh_geometry(r.z, Hi, shift, ii, m, &base[2], &arg[2]);
  // this lane's weights: piece CAO-1-c at the three tabulated offsets
  const real *cp = coef + (CAO - 1 - c) * CAO;
  real wc[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const real u = (real)(arg[d] - P3MG_NINTERP / 2) * (real)(1.0 / P3MG_NINTERP) + (real)0.5;
    real h = cp[CAO - 1];
#pragma unroll
    for (int i = CAO - 2; i >= 0; i--) h = h * u + cp[i];
    wc[d] = h;
  }
  real wx[CAO], wy[CAO];
#pragma unroll
  for (int a = 0; a < CAO; a++) {
    wx[a] = __shfl_sync(0xffffffffu, wc[0], src0 + a);
    wy[a] = __shfl_sync(0xffffffffu, wc[1], src0 + a);
  }
  real acc0 = 0, acc1 = 0, acc2 = 0;
  if (act) {
    const real sw = (real)((NMESH == 2) ? 0.5 * pref : pref) * ((real)r.w * wc[2]);
    int gk = base[2] + c;
    gk -= (gk >= m) ? m : 0;
    const V *__restrict__ Pm = P + (ii ? M : 0) + gk;
#pragma unroll
    for (int a = 0; a < CAO; a++) {
      int gi = base[0] + a;
      gi -= (gi >= m) ? m : 0;
      const real swa = sw * wx[a];
      const V *__restrict__ Pa = Pm + (size_t)gi * m * m;
#pragma unroll
      for (int b = 0; b < CAO; b++) {
        int gj = base[1] + b;
        gj -= (gj >= m) ? m : 0;
        const V f = Pa[(size_t)gj * m];
        const real w = swa * wy[b];
        acc0 -= f.x * w;
        acc1 -= f.y * w;
        acc2 -= f.z * w;
      }
    }
  }
#pragma unroll
  for (int o = LPP / 2; o > 0; o >>= 1) {
    acc0 += __shfl_xor_sync(0xffffffffu, acc0, o);
    acc1 += __shfl_xor_sync(0xffffffffu, acc1, o);
    acc2 += __shfl_xor_sync(0xffffffffu, acc2, o);
  }
  if (p < np && l == 0) {
    const int o = sidx[p];
    fk[o] += (double)acc0;
    fk[(size_t)n + o] += (double)acc1;
    fk[2 * (size_t)n + o] += (double)acc2;
  }
}

// The k-space part of the energy's adjoint from the potential meshes Phi
// (complex layout, unshifted mesh in the real part, shifted in the
// imaginary part): per brick-sorted particle, with the weights W and their
// derivatives dW at the exact in-cell offset,
//   gx += ge s q_i (m/L) sum Phi dW/du ...,  gq += ge s sum Phi W,
// s = c / (L^3 nmesh) (c = 1 for the ad, 1/2 for the ik influence
// functions).  Same loop structure as gather_kernel's ad branch.
template <typename real, int CAO, int NMESH>
__global__ void __launch_bounds__(ASSIGN_THREADS) adj_gather_sorted_kernel(const double4 *__restrict__ sxyzq,
                                                                            const int *__restrict__ sidx, int np,
                                                                            int m, double Hi, double shift,
                                                                            const typename cplx<real>::type *__restrict__ Phi,
                                                                            double s, double ge,
                                                                            double *__restrict__ gx,
                                                                            double *__restrict__ gq, int n) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const double4 r = sxyzq[p];
  const real *__restrict__ Pr = reinterpret_cast<const real *>(Phi);
  real sp = 0, s0 = 0, s1 = 0, s2 = 0;
#pragma unroll
  for (int ii = 0; ii < NMESH; ii++) {
    int base[3], arg[3];
    double uu[3];
    mesh_geometry_u(r.x, Hi, shift, ii, m, &base[0], &arg[0], &uu[0]);
    mesh_geometry_u(r.y, Hi, shift, ii, m, &base[1], &arg[1], &uu[1]);
    mesh_geometry_u(r.z, Hi, shift, ii, m, &base[2], &arg[2], &uu[2]);
    real w[3][CAO], dw[3][CAO];
#pragma unroll
    for (int d = 0; d < 3; d++) bspline_weights_u<real, CAO, true>((real)uu[d], w[d], dw[d]);
#pragma unroll
    for (int a = 0; a < CAO; a++) {
      int gi = base[0] + a;
      gi -= (gi >= m) ? m : 0;
#pragma unroll
      for (int b = 0; b < CAO; b++) {
        int gj = base[1] + b;
        gj -= (gj >= m) ? m : 0;
        const size_t row = ((size_t)gi * m + gj) * m;
        real t0 = 0, t1 = 0;  // sum_c phi W_c, sum_c phi dW_c
#pragma unroll
        for (int c = 0; c < CAO; c++) {
          int gk = base[2] + c;
          gk -= (gk >= m) ? m : 0;
          const real ph = Pr[2 * (row + gk) + ii];
          t0 += ph * w[2][c];
          t1 += ph * dw[2][c];
        }
        sp += w[0][a] * w[1][b] * t0;
        s0 += dw[0][a] * w[1][b] * t0;
        s1 += w[0][a] * dw[1][b] * t0;
        s2 += w[0][a] * w[1][b] * t1;
      }
    }
  }
  const int o = sidx[p];
  const double gs = ge * s;
  const double gd = gs * r.w * Hi;  // d/dx = (m/L) d/du
  gx[o] += gd * (double)s0;
  gx[(size_t)n + o] += gd * (double)s1;
  gx[2 * (size_t)n + o] += gd * (double)s2;
  gq[o] += gs * (double)sp;
}

template <typename real, int CAO>
int dispatch_adj_gather(Ctx *c, const void *Phi, double s, double ge, double *gx, double *gq) {
  typedef typename cplx<real>::type C;
  const double Hi = (double)c->mesh / c->L;
  const double shift = (double)((c->cao - 1) / 2);
  const unsigned blocks = (unsigned)((c->n + ASSIGN_THREADS - 1) / ASSIGN_THREADS);
  if (method_interlaced(c->method))
    adj_gather_sorted_kernel<real, CAO, 2><<<blocks, ASSIGN_THREADS, 0, c->stream>>>(
        c->sorted_xyzq, c->sorted_idx, c->n, c->mesh, Hi, shift, reinterpret_cast<const C *>(Phi), s, ge, gx, gq, c->n);
  else
    adj_gather_sorted_kernel<real, CAO, 1><<<blocks, ASSIGN_THREADS, 0, c->stream>>>(
        c->sorted_xyzq, c->sorted_idx, c->n, c->mesh, Hi, shift, reinterpret_cast<const C *>(Phi), s, ge, gx, gq, c->n);
  c->launches++;
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

template <typename real>
int adj_gather_any(Ctx *c, const void *Phi, double s, double ge, double *gx, double *gq) {
  switch (c->cao) {
    case 1: return dispatch_adj_gather<real, 1>(c, Phi, s, ge, gx, gq);
    case 2: return dispatch_adj_gather<real, 2>(c, Phi, s, ge, gx, gq);
    case 3: return dispatch_adj_gather<real, 3>(c, Phi, s, ge, gx, gq);
    case 4: return dispatch_adj_gather<real, 4>(c, Phi, s, ge, gx, gq);
    case 5: return dispatch_adj_gather<real, 5>(c, Phi, s, ge, gx, gq);
    case 6: return dispatch_adj_gather<real, 6>(c, Phi, s, ge, gx, gq);
    case 7: return dispatch_adj_gather<real, 7>(c, Phi, s, ge, gx, gq);
  }
  return P3MG_ERR_CAO;
}

// ---------------------------------------------------------- self forces

// f_tot,d -= b_d(m') q^2 sin(2 pi (m'.x)/h) for the 27 m' (p3m-ad-self-forces.c:114-139)
__global__ void self_force_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                  const double *__restrict__ z, const double *__restrict__ q, int n, double h,
                                  const double *__restrict__ b81, double *__restrict__ f) {
  __shared__ double b[81];
  // alpha batch (grid.y): coefficients and forces of entry y
  b81 += (size_t)blockIdx.y * 81;
  f += (size_t)blockIdx.y * 3 * (size_t)n;
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

// Lane table of the scatter for row pitch SR: entry ps*32 + lane = (b*SR + c,
// b, c, 0) of the (b, c) stencil column that lane owns in pass ps, or
// (0, -1, 0, 0).  Columns are placed greedily in (b, c) order on the first
// free lane of their bank class (b*SR + c modulo 32 for 4-byte elements;
// modulo 16 in each half-warp for 8-byte elements, which are served 16
// lanes at a time).  Returns false when some column finds no lane.
inline bool scatter_lane_table(int cao, int SR, int word_bytes, int4 *tab) {
  const int npass = (cao * cao + 31) / 32;
  const int R = word_bytes == 8 ? 16 : 32;
  for (int e = 0; e < 32 * npass; e++) tab[e] = make_int4(0, -1, 0, 0);
  for (int b = 0; b < cao; b++)
    for (int cc = 0; cc < cao; cc++) {
      const int off = b * SR + cc, cls = off % R;
      bool placed = false;
      for (int ps = 0; ps < npass && !placed; ps++)
        for (int h = 0; h < 32 / R && !placed; h++) {
          int4 &e = tab[ps * 32 + cls + h * R];
          if (e.y < 0) {
            e = make_int4(off, b, cc, 0);
            placed = true;
          }
        }
      if (!placed) return false;
    }
  return true;
}

// Smallest row pitch >= T with a conflict-free lane table (plane pitch
// T * SR); searched once per shape.
inline int scatter_row_pitch(int cao, int T, int word_bytes) {
  static int cache[8][64][2];
  const int wi = word_bytes == 8 ? 1 : 0;
  if (cao < 8 && T < 64 && cache[cao][T][wi]) return cache[cao][T][wi];
  int4 tab[64];
  int sr = T;
  while (sr < T + 64 && !scatter_lane_table(cao, sr, word_bytes, tab)) sr++;
  if (cao < 8 && T < 64) cache[cao][T][wi] = sr;
  return sr;
}

template <typename real, int CAO, int NMESH, bool EXACT = false>
int launch_scatter(Ctx *c, size_t smem, int SR, int SP) {
  auto kern = scatter_kernel<real, CAO, NMESH, EXACT>;
  // raise the dynamic shared-memory limit once per instantiation and device
  // (outside any graph capture: the first step of a shape always runs eagerly)
  static std::atomic<int> smem_set[P3MG_MAX_DEVICES];
  P3MG_CUDA_TRY(raise_smem_limit(kern, (int)(smem > 200 * 1024 ? smem : 200 * 1024), smem_set));
  const double Hi = (double)c->mesh / c->L;
  const double shift = (double)((c->cao - 1) / 2);
  const int nbr = c->nbrick1 * c->nbrick1 * c->nbrick1;
  mark(c, EV_K2);
  if (!c->scatter_tab) {
    // built once per context, on its first (eager, uncaptured) step
    constexpr int NPASS = (CAO * CAO + 31) / 32;
    int4 host[32 * NPASS];
    if (!scatter_lane_table(CAO, SR, (int)sizeof(real), host)) return P3MG_ERR_MESH;
    P3MG_CUDA_TRY(cudaMalloc(&c->scatter_tab, sizeof(int4) * 32 * NPASS));
    P3MG_CUDA_TRY(cudaMemcpy(c->scatter_tab, host, sizeof(int4) * 32 * NPASS, cudaMemcpyHostToDevice));
  }
  const bool rl = !EXACT && kspace_real(c);  // the adjoint keeps the complex mesh
  kern<<<nbr, ASSIGN_THREADS, smem, c->stream>>>(c->sorted_xyzq, c->brick_start, c->mesh, c->brick, c->nbrick1, Hi,
                                                shift, SR, SP, reinterpret_cast<const int4 *>(c->scatter_tab),
                                                reinterpret_cast<real *>(c->Q), rl ? c->mesh + 2 : c->mesh,
                                                rl ? 1 : 2);
  c->launches++;
  mark(c, EV_K3);
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

template <typename real, int CAO, bool EXACT = false>
int dispatch_scatter(Ctx *c) {
  const int nmesh = method_interlaced(c->method) ? 2 : 1;
  const int T = brick_tile(c->brick, CAO, nmesh);
  const int SR = scatter_row_pitch(CAO, T, (int)sizeof(real)), SP = T * SR;
  const size_t tile = (size_t)nmesh * T * SP * sizeof(real);
  if (nmesh == 2) return launch_scatter<real, CAO, 2, EXACT>(c, tile + scatter_stage_bytes<real, CAO, 2>(), SR, SP);
  return launch_scatter<real, CAO, 1, EXACT>(c, tile + scatter_stage_bytes<real, CAO, 1>(), SR, SP);
}

// Gather launch for na batch entries (grid.y): fields / potential Fv of
// entry y at the batch stride of the kernel, forces into fk + 3 n y.
template <typename real, int CAO>
int dispatch_gather(Ctx *c, const void *Fv, double *fk, int na) {
  const double Hi = (double)c->mesh / c->L;
  const double shift = (double)((c->cao - 1) / 2);
  const double L3 = c->L * c->L * c->L;
  const double Leni = 1.0 / c->L;
  const dim3 grid((c->n + ASSIGN_THREADS - 1) / ASSIGN_THREADS, na);
  const bool il = method_interlaced(c->method);
  const int RP = kspace_real(c) ? c->mesh + 2 : c->mesh, ES = kspace_real(c) ? 1 : 2;
  mark(c, EV_K4);
  if (method_ad(c->method)) {
    // prefactor Mesh * Leni^3 (p3m-ad.c:202, p3m-ad-i.c:199, p3m-ad-real.c:110)
    const double pref = (double)c->mesh * Leni * Leni * Leni;
    if (il)
      gather_kernel<real, CAO, 2, true><<<grid, ASSIGN_THREADS, 0, c->stream>>>(
          c->sorted_xyzq, c->sorted_idx, c->n, c->mesh, Hi, shift, pref, Leni, Fv, c->M, fk, c->n, RP, ES);
    else
      gather_kernel<real, CAO, 1, true><<<grid, ASSIGN_THREADS, 0, c->stream>>>(
          c->sorted_xyzq, c->sorted_idx, c->n, c->mesh, Hi, shift, pref, Leni, Fv, c->M, fk, c->n, RP, ES);
  } else if (std::is_same<real, float>::value && c->gather_mode >= 2 && gather_tile_fits(c)) {
    // prefactor 1 / (2 L^3) (p3m-ik.c:242, p3m-ik-i.c:241, p3m-ik-real.c:144);
    // brick tiles in shared memory
    P3MG_TRY(gather_tile_f32(c, Fv, fk, na, 1.0 / (2.0 * L3)));
  } else if (c->gather_mode == 0 && (il ? 2 : 1) * CAO <= 16) {
    // prefactor 1 / (2 L^3) (p3m-ik.c:242, p3m-ik-i.c:241, p3m-ik-real.c:144);
    // lanes on the stencil's z offsets
    const double pref = 1.0 / (2.0 * L3);
    constexpr int LPP2 = (2 * CAO <= 8) ? 8 : 16, LPP1 = (CAO <= 8) ? 8 : 16;
    const size_t lanes = (size_t)c->n * (il ? LPP2 : LPP1);
    const dim3 lgrid((unsigned)((lanes + ASSIGN_THREADS - 1) / ASSIGN_THREADS), na);
    static const PieceCoef<real> pcoef = bspline_pieces<real>(CAO);
    if (il)
      gather_lanes_kernel<real, CAO, (2 * CAO <= 16) ? 2 : 1><<<lgrid, ASSIGN_THREADS, 0, c->stream>>>(
          c->sorted_xyzq, c->sorted_idx, c->n, c->mesh, Hi, shift, pref, Fv, c->M, fk, c->n, pcoef);
    else
      gather_lanes_kernel<real, CAO, 1><<<lgrid, ASSIGN_THREADS, 0, c->stream>>>(
          c->sorted_xyzq, c->sorted_idx, c->n, c->mesh, Hi, shift, pref, Fv, c->M, fk, c->n, pcoef);
  } else {
    // prefactor 1 / (2 L^3) (p3m-ik.c:242, p3m-ik-i.c:241, p3m-ik-real.c:144)
    const double pref = 1.0 / (2.0 * L3);
    if (il)
      gather_kernel<real, CAO, 2, false><<<grid, ASSIGN_THREADS, 0, c->stream>>>(
          c->sorted_xyzq, c->sorted_idx, c->n, c->mesh, Hi, shift, pref, Leni, Fv, c->M, fk, c->n, RP, ES);
    else
      gather_kernel<real, CAO, 1, false><<<grid, ASSIGN_THREADS, 0, c->stream>>>(
          c->sorted_xyzq, c->sorted_idx, c->n, c->mesh, Hi, shift, pref, Leni, Fv, c->M, fk, c->n, RP, ES);
  }
  c->launches++;
  mark(c, EV_K5);
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

template <typename real>
int gather_any(Ctx *c, const void *Fv, double *fk, int na) {
  switch (c->cao) {
    case 1: return dispatch_gather<real, 1>(c, Fv, fk, na);
    case 2: return dispatch_gather<real, 2>(c, Fv, fk, na);
    case 3: return dispatch_gather<real, 3>(c, Fv, fk, na);
    case 4: return dispatch_gather<real, 4>(c, Fv, fk, na);
    case 5: return dispatch_gather<real, 5>(c, Fv, fk, na);
    case 6: return dispatch_gather<real, 6>(c, Fv, fk, na);
    case 7: return dispatch_gather<real, 7>(c, Fv, fk, na);
  }
  return P3MG_ERR_CAO;
}

template <typename real, bool EXACT = false>
int scatter_any(Ctx *c) {
  switch (c->cao) {
    case 1: return dispatch_scatter<real, 1, EXACT>(c);
    case 2: return dispatch_scatter<real, 2, EXACT>(c);
    case 3: return dispatch_scatter<real, 3, EXACT>(c);
    case 4: return dispatch_scatter<real, 4, EXACT>(c);
    case 5: return dispatch_scatter<real, 5, EXACT>(c);
    case 6: return dispatch_scatter<real, 6, EXACT>(c);
    case 7: return dispatch_scatter<real, 7, EXACT>(c);
  }
  return P3MG_ERR_CAO;
}

template <typename real>
int run_kspace(Ctx *c) {
  typedef typename cplx<real>::type C;
  const size_t M = c->M;
  const int threads = 256;
  const unsigned mblocks = (unsigned)((M + threads - 1) / threads);
  // charge assignment (the brick binning ran in kspace_prepare)
  P3MG_CUDA_TRY(cudaMemsetAsync(c->Q, 0, M * sizeof(C), c->stream));
  P3MG_TRY(scatter_any<real>(c));
  mark(c, EV_S2);
  if (kspace_real(c)) {
    // methods 6 / 7: r2c, convolution over the half spectrum, c2r
    typedef typename std::conditional<sizeof(real) == 8, double, float>::type Gt;
    const Gt *G = reinterpret_cast<const Gt *>(c->precision == P3MG_FP64 ? (const void *)c->G : (const void *)c->G32);
    const size_t Mh = (size_t)c->mesh * c->mesh * (c->mesh / 2 + 1);
    const unsigned hblocks = (unsigned)((Mh + threads - 1) / threads);
    P3MG_TRY(fft3d_real(c, c->Q, 1, -1));
    if (method_ad(c->method)) {
      conv_ad_half_kernel<real, Gt><<<hblocks, threads, 0, c->stream>>>(reinterpret_cast<C *>(c->Q), G, c->mesh, M,
                                                                        reinterpret_cast<C *>(c->Q));
      c->launches++;
      P3MG_CUDA_TRY(cudaGetLastError());
      P3MG_TRY(fft3d_real(c, c->Q, 1, +1));
    } else {
      conv_ik_half_kernel<real, Gt><<<hblocks, threads, 0, c->stream>>>(
          reinterpret_cast<const C *>(c->Q), G, c->mesh, 2.0 * P3MG_PI / c->L, M, reinterpret_cast<C *>(c->F));
      c->launches++;
      P3MG_CUDA_TRY(cudaGetLastError());
      P3MG_TRY(fft3d_real(c, c->F, 3, +1));
      typedef typename cplx<real>::vec4 V;
      pack_ik_real_kernel<real><<<mblocks, threads, 0, c->stream>>>(reinterpret_cast<const real *>(c->F), c->mesh, M,
                                                                    reinterpret_cast<V *>(c->P));
      c->launches++;
      P3MG_CUDA_TRY(cudaGetLastError());
    }
    mark(c, EV_S3);
    P3MG_TRY(gather_any<real>(c, method_ad(c->method) ? c->Q : c->P, c->fk, 1));
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
  // forward FFT, convolution, backward FFT(s)
  P3MG_TRY(fft3d(c, c->Q, 1, -1));
  if (method_ad(c->method)) {
    if (c->precision == P3MG_FP64)
      conv_ad_kernel<real, double><<<mblocks, threads, 0, c->stream>>>(reinterpret_cast<C *>(c->Q), c->G, M,
                                                                       reinterpret_cast<C *>(c->Q));
    else
      conv_ad_kernel<real, float><<<mblocks, threads, 0, c->stream>>>(reinterpret_cast<C *>(c->Q), c->G32, M,
                                                                      reinterpret_cast<C *>(c->Q));
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
    P3MG_TRY(fft3d(c, c->Q, 1, +1));
  } else {
    const double s = 2.0 * P3MG_PI / c->L;
    // FP32 pencil FFTs: the convolution folded into the first backward
    // pass, the packing into the last
    const bool fused = c->precision != P3MG_FP64 && c->fft_w == 0 && fft_pencil_ok(c);
    if (fused) {
      P3MG_TRY(ik_conv_inverse_pencil(c, c->Q, c->G32, s, c->F, 1, c->P));
    } else {
      if (c->precision == P3MG_FP64)
        conv_ik_kernel<real, double><<<mblocks, threads, 0, c->stream>>>(reinterpret_cast<const C *>(c->Q), c->G,
                                                                         c->mesh, s, M, reinterpret_cast<C *>(c->F));
      else
        conv_ik_kernel<real, float><<<mblocks, threads, 0, c->stream>>>(reinterpret_cast<const C *>(c->Q), c->G32,
                                                                        c->mesh, s, M, reinterpret_cast<C *>(c->F));
      c->launches++;
      P3MG_CUDA_TRY(cudaGetLastError());
      P3MG_TRY(fft3d(c, c->F, 3, +1));
      typedef typename cplx<real>::vec4 V;
      if (method_interlaced(c->method))
        pack_ik_kernel<real, 2><<<mblocks, threads, 0, c->stream>>>(reinterpret_cast<const C *>(c->F), M,
                                                                    reinterpret_cast<V *>(c->P));
      else
        pack_ik_kernel<real, 1><<<mblocks, threads, 0, c->stream>>>(reinterpret_cast<const C *>(c->F), M,
                                                                    reinterpret_cast<V *>(c->P));
      c->launches++;
      P3MG_CUDA_TRY(cudaGetLastError());
    }
  }
  mark(c, EV_S3);
  // back-interpolation
  P3MG_TRY(gather_any<real>(c, method_ad(c->method) ? c->Q : c->P, c->fk, 1));
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

// The alpha-dependent half of the k-space pass for b.na alphas at once
// (the charge assignment and forward FFT do not depend on alpha and, with
// b.forward, run once into Q): convolution with each alpha's G, the
// backward FFTs of all na meshes in one batched transform, the gather and
// the ad self-force correction, each one launch over grid.y = alpha.
template <typename real>
int run_kspace_batch(Ctx *c, const KspaceBatch &b) {
  typedef typename cplx<real>::type C;
  typedef typename cplx<real>::vec4 V;
  typedef typename std::conditional<sizeof(real) == 8, double, float>::type Gt;
  const size_t M = c->M;
  const int threads = 256;
  const int na = b.na;
  const dim3 mgrid((unsigned)((M + threads - 1) / threads), na);
  const bool rl = kspace_real(c);
  if (b.forward) {
    P3MG_CUDA_TRY(cudaMemsetAsync(c->Q, 0, M * sizeof(C), c->stream));
    P3MG_TRY(scatter_any<real>(c));
    if (rl)
      P3MG_TRY(fft3d_real(c, c->Q, 1, -1));
    else
      P3MG_TRY(fft3d(c, c->Q, 1, -1));
  }
  const Gt *G = reinterpret_cast<const Gt *>(b.G);
  if (rl) {
    // methods 6 / 7: the half spectrum (r2c / c2r)
    const size_t Mh = (size_t)c->mesh * c->mesh * (c->mesh / 2 + 1);
    const dim3 hgrid((unsigned)((Mh + threads - 1) / threads), na);
    if (method_ad(c->method)) {
      conv_ad_half_kernel<real, Gt><<<hgrid, threads, 0, c->stream>>>(reinterpret_cast<const C *>(c->Q), G, c->mesh,
                                                                      M, reinterpret_cast<C *>(b.F));
      c->launches++;
      P3MG_CUDA_TRY(cudaGetLastError());
      P3MG_TRY(fft3d_real(c, b.F, na, +1));
      P3MG_TRY(gather_any<real>(c, b.F, b.fk, na));
    } else {
      conv_ik_half_kernel<real, Gt><<<hgrid, threads, 0, c->stream>>>(
          reinterpret_cast<const C *>(c->Q), G, c->mesh, 2.0 * P3MG_PI / c->L, M, reinterpret_cast<C *>(b.F));
      c->launches++;
      P3MG_CUDA_TRY(cudaGetLastError());
      P3MG_TRY(fft3d_real(c, b.F, 3 * na, +1));
      pack_ik_real_kernel<real><<<mgrid, threads, 0, c->stream>>>(reinterpret_cast<const real *>(b.F), c->mesh, M,
                                                                   reinterpret_cast<V *>(b.P));
      c->launches++;
      P3MG_CUDA_TRY(cudaGetLastError());
      P3MG_TRY(gather_any<real>(c, b.P, b.fk, na));
    }
  } else if (method_ad(c->method)) {
    conv_ad_kernel<real, Gt><<<mgrid, threads, 0, c->stream>>>(reinterpret_cast<const C *>(c->Q), G, M,
                                                               reinterpret_cast<C *>(b.F));
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
    P3MG_TRY(fft3d(c, b.F, na, +1));
    P3MG_TRY(gather_any<real>(c, b.F, b.fk, na));
  } else if (sizeof(real) == 4 && c->fft_w == 0 && fft_pencil_ok(c)) {
    // FP32 pencil FFTs: the convolution folded into the first backward
    // pass, the packing into the last
    P3MG_TRY(ik_conv_inverse_pencil(c, c->Q, reinterpret_cast<const float *>(b.G), 2.0 * P3MG_PI / c->L, b.F, na,
                                    b.P));
    P3MG_TRY(gather_any<real>(c, b.P, b.fk, na));
  } else {
    conv_ik_kernel<real, Gt><<<mgrid, threads, 0, c->stream>>>(reinterpret_cast<const C *>(c->Q), G, c->mesh,
                                                               2.0 * P3MG_PI / c->L, M, reinterpret_cast<C *>(b.F));
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
    P3MG_TRY(fft3d(c, b.F, 3 * na, +1));
    if (method_interlaced(c->method))
      pack_ik_kernel<real, 2><<<mgrid, threads, 0, c->stream>>>(reinterpret_cast<const C *>(b.F), M,
                                                                 reinterpret_cast<V *>(b.P));
    else
      pack_ik_kernel<real, 1><<<mgrid, threads, 0, c->stream>>>(reinterpret_cast<const C *>(b.F), M,
                                                                 reinterpret_cast<V *>(b.P));
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
    P3MG_TRY(gather_any<real>(c, b.P, b.fk, na));
  }
  if (method_self_force(c->method)) {
    const dim3 pgrid((c->n + threads - 1) / threads, na);
    self_force_kernel<<<pgrid, threads, 0, c->stream>>>(c->x, c->y, c->z, c->q, c->n, c->L / c->mesh, b.b81, b.f);
    c->launches++;
    P3MG_CUDA_TRY(cudaGetLastError());
  }
  return P3MG_OK;
}

}  // namespace
}  // namespace assign_impl
}  // namespace p3mg
