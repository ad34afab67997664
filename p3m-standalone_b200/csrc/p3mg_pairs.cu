// Real-space erfc pair forces (the reference's Realteil, realpart.c:124-167):
// for every ordered pair i != j with minimum-image distance r <= rcut
//   f_i += q_i q_j (erfc(alpha r)/r + 2 alpha/sqrt(pi) exp(-alpha^2 r^2)) / r^2 * d
//   E   += 1/2 q_i q_j erfc(alpha r)/r
// The reference loops over all N^2 pairs.  Here particles are counting-sorted
// into a cell list of side > rcut (nc = floor(L / (rcut (1 + 1e-6))) >= 3
// cells per side), each cell split into 2x2x2 half-cells of side h, which
// visits exactly the same pair set.  One CTA per cell stages the half-cells
// around it through shared memory in (J0, J1, J2) order, so each half-cell
// column (J0, J1) is one contiguous range.  Within a CTA each warp takes one
// i at a time: its lanes first clip the 5x5 columns that can hold partners
// of i (xy distance of i from the column <= rcut, z range cut to the
// half-cells the rcut sphere reaches), concatenate the surviving ranges
// (prefix sum + __fns over the lanes), and then test 32 candidates per step
// with every lane busy.  Accepted candidates are compacted (ballot + prefix
// count) into a circular per-warp queue, and 32 interactions are evaluated
// at once whenever the queue holds 32, so the erfc branch runs on full warps.
//
// FP32 applies Newton's third law: a pair is evaluated once, by the CTA of
// the particle that comes first in the staged (J0, J1, J2, slot) order --
// an order every CTA agrees on, because the half-cell offset of j seen from
// i is minus the one of i seen from j -- so a CTA stages only the half-cells
// that can follow one of its own (130 of 216), a warp visits only the
// forward columns, and the partner's force goes into a shared-memory
// accumulator per staged candidate that is added to the global forces with
// FP64 atomics at the end of the chunk (the particle's own force likewise).
// About 90 M evaluations instead of 180 M at the headline workload.  The
// partner accumulators are 32-bit fixed point (shared-memory integer adds
// are single native atomics, float adds are not): partner j's scale is
// S_j = 2^20 / (|q_j| max|q_i| max(alpha^2, 1/rcut^2)) with the maximum over
// the i batch, so its resolution follows its own charge; a contribution
// below 2^24 units is added there, a larger one (the closest pairs) goes
// straight to the global FP64 force; a chunk adds at most 64 contributions
// per partner, so no accumulator passes 2^30.
//
// FP64 keeps every ordered pair, each particle's force summed by one warp in
// a fixed order (bit-reproducible from run to run): a conservative FP32
// filter, then every queued pair is evaluated exactly like the reference (dx -= round(dx/L) L with separately rounded
// products, r <= rcut), so the pair set and the forces are the reference's.
// FP32 (mixed): positions relative to the origin of their cell, neighbour
// offsets added as multiples of the cell side; erfc from a fitted rational
// form; energy summed with compensated (Kahan) FP32 per lane and FP64 across
// lanes.  With fewer than 3 cells per side the all-pairs kernel runs.
#include <math.h>

#include <atomic>

#include "p3mg_internal.cuh"

namespace p3mg {

namespace {

constexpr int BRUTE_THREADS = 256;

// half-cell key of a particle: cell-major, then the 2x2x2 sub-cell; beside
// it the particle's rank in its half-cell (the count's atomic returns it)
__global__ void bin_cells_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                 const double *__restrict__ z, int n, double L, int nc, int2 *__restrict__ key,
                                 int *__restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double s = (double)(2 * nc) / L;
  const int h0 = wrap_full((int)floor(x[i] * s), 2 * nc);
  const int h1 = wrap_full((int)floor(y[i] * s), 2 * nc);
  const int h2 = wrap_full((int)floor(z[i] * s), 2 * nc);
  const int k = (((h0 >> 1) * nc + (h1 >> 1)) * nc + (h2 >> 1)) * 8 + ((h0 & 1) << 2) + ((h1 & 1) << 1) + (h2 & 1);
  key[i] = make_int2(k, atomicAdd(&count[k], 1));
}

template <typename V>
__global__ void place_cells_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                   const double *__restrict__ z, const double *__restrict__ q, int n, double L, int nc,
                                   const int2 *__restrict__ key, const int *__restrict__ start,
                                   int *__restrict__ sidx, V *__restrict__ pos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int2 kr = key[i];
  const int k = kr.x;
  const int slot = start[k] + kr.y;
  sidx[slot] = i;
  if (sizeof(V) == sizeof(double4)) {
    reinterpret_cast<double4 *>(pos)[slot] = make_double4(x[i], y[i], z[i], q[i]);
  } else {
    // position relative to the cell origin, folded into the box
    const double cs = L / nc;
    const int cell = k >> 3;
    const int c2 = cell % nc, c1 = (cell / nc) % nc, c0 = cell / (nc * nc);
    double xr = x[i] - L * floor(x[i] / L) - c0 * cs;
    double yr = y[i] - L * floor(y[i] / L) - c1 * cs;
    double zr = z[i] - L * floor(z[i] / L) - c2 * cs;
    reinterpret_cast<float4 *>(pos)[slot] = make_float4((float)xr, (float)yr, (float)zr, (float)q[i]);
  }
}

__device__ __forceinline__ double min_image(double d, double Li, double L) {
  // d -= round(d / L) * L  (realpart.c:141-146), each operation rounded separately
  return __dadd_rn(d, -__dmul_rn(round(__dmul_rn(d, Li)), L));
}

// erfc(x) for x >= 0 given ex = exp(-x^2):  erfc(x) = t P(t) ex,
// t = 1/(1 + 0.415 x), P a degree-7 polynomial -- the form of Abramowitz &
// Stegun 7.1.26 with coefficients from a least-squares fit of the relative
// error of erfc(x) e^{x^2} / t on [0, 6] (max relative error 8e-8 in exact
// arithmetic, 2e-6 evaluated in FP32 with a fast exp).
__device__ __forceinline__ float erfc_fit(float x, float ex) {
  const float t = __fdividef(1.0f, fmaf(0.415f, x, 1.0f));
  float P = 0.0763478258f;
  P = fmaf(P, t, -0.360062487f);
  P = fmaf(P, t, 0.535669094f);
  P = fmaf(P, t, -0.220555614f);
  P = fmaf(P, t, 0.318725078f);
  P = fmaf(P, t, 0.176562497f);
  P = fmaf(P, t, 0.23950376f);
  P = fmaf(P, t, 0.233809829f);
  return t * P * ex;
}

// CTA shape and shared-memory budget of the cell kernel.
constexpr int PAIR_CTA = 128;
constexpr int PAIR_WARPS = PAIR_CTA / 32;
constexpr int PAIR_JCH = 1536;   // FP64: staged candidates (the whole neighbourhood when it fits)
constexpr int PAIR_JCH32 = 832;  // FP32: staged candidates of the forward half (about 740 at density 1)
constexpr int PAIR_MAXI = 128;   // FP64: i particles per batch
constexpr int PAIR_MAXI32 = 64;  // FP32 (cells hold about 46 at density 1)
constexpr int PAIR_QCAP = 64;    // circular queue per warp (power of two)
constexpr int PAIR_NSEG = 216;   // 6x6x6 half-cells around the cell

// Newton's third law: FP32 with one alpha per CTA (see pairs_cell_kernel)
__host__ __device__ constexpr bool pair_n3(bool dbl, int na) { return !dbl && na == 1; }
__host__ __device__ constexpr int pair_jch(bool dbl, int na, bool adj = false) {
  return pair_n3(dbl, na) && !adj ? PAIR_JCH32 : PAIR_JCH;
}
__host__ __device__ constexpr int pair_maxi(bool dbl) { return dbl ? PAIR_MAXI : PAIR_MAXI32; }

// staged positions, sorted slots, (Newton-3) partner-force accumulators,
// the i batch and its forces per alpha of the group, the warp queues
__host__ __device__ constexpr size_t pair_smem_bytes(bool dbl, int na, bool adj = false) {
  return (size_t)pair_jch(dbl, na, adj) * (sizeof(float4) + sizeof(int) + (pair_n3(dbl, na) && !adj ? 3 * sizeof(float) : 0)) +
         (size_t)pair_maxi(dbl) * sizeof(float4) +
         (size_t)pair_maxi(dbl) * (adj ? 4 : 3) * na * (dbl ? sizeof(double) : sizeof(float)) +
         (size_t)PAIR_WARPS * PAIR_QCAP * sizeof(unsigned short);
}

// alphas per CTA in an alpha batch: the candidate search is shared by the
// group, each pair is evaluated for every alpha of it
constexpr int PAIR_NA32 = 8;
constexpr int PAIR_NA64 = 4;

template <bool DBL>
struct PairAcc {
  typedef float type;
};
template <>
struct PairAcc<true> {
  typedef double type;
};

// Exclusive prefix of the PAIR_NSEG half-cell counts held in seg_pre[1..]
// (seg_pre[sg + 1] = count of segment sg on entry; seg_pre[sg] = the counts
// before sg on exit), by the whole CTA: two entries per thread, a warp scan
// of the pair sums, the warps' totals through wsum.  Ends with a barrier.
__device__ __forceinline__ void scan_segments(int *seg_pre, int *wsum) {
  static_assert(2 * PAIR_CTA >= PAIR_NSEG, "two segments per thread");
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int i1 = 2 * tid + 1, i2 = 2 * tid + 2;
  const int a = i1 <= PAIR_NSEG ? seg_pre[i1] : 0;
  const int b = i2 <= PAIR_NSEG ? seg_pre[i2] : 0;
  int v = a + b;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) wsum[warp] = v;
  __syncthreads();
  int off = 0;
#pragma unroll
  for (int w = 0; w < PAIR_WARPS; w++)
    if (w < warp) off += wsum[w];
  const int incl = v + off;  // counts of segments 0 .. i2 - 1
  if (i1 <= PAIR_NSEG) seg_pre[i1] = incl - b;
  if (i2 <= PAIR_NSEG) seg_pre[i2] = incl;
  if (tid == 0) seg_pre[0] = 0;
  __syncthreads();
}

// FP32 Newton-3 pairs of a DENSE cell: one whose forward half-cells exceed
// the staging arrays (the centre of a clustered system, a cell grid capped
// to fewer, wider cells).  Instead of testing every staged candidate per
// particle, the CTA takes its own half-cells A one at a time and shares one
// candidate list among A's particles: the forward columns that can reach A
// (clipped like a particle's columns, from A's own half-cell on) are listed
// as (column, z) segments, A's particles are staged in blocks of DENSE_ABLK
// and the candidates are streamed through the rest of the staging arrays in
// chunks; a warp tests up to 32 of A's particles against 32 / P candidates
// per instruction (P the power of two >= the block's particle count, lane =
// candidate * P + particle) and queues the hits as (i, j) slot pairs that
// are evaluated 32 at a time.  Both forces of a pair go to 32-bit
// fixed-point accumulators of the two staged slots (slot s counts in units
// fxs / |q_s|, the scale of pairs_cell_kernel with the maximum |q| of the
// staged particles), flushed to the global forces after every chunk; a
// contribution of thr = min(2^24, 2^30 / max(chunk, block)) units or more
// goes straight to the global FP64 force (a slot takes at most that many
// contributions between flushes, so no accumulator passes 2^30).  Pair
// order: a pair belongs to the particle first in (J0, J1, J2, sorted slot)
// order, as in pairs_cell_kernel.  Half-cells u_first .. u_last - 1 and,
// with ab_only >= 0, only their block ab_only (one work unit of
// dense_units_kernel).  Returns this thread's share of the pair energy.
constexpr int DENSE_ABLK = 64;   // particles of a half-cell staged per block (one work unit)
constexpr int DENSE_NSEG = 65;   // (column, z) segments of one half-cell's candidates (13 x 5)

__device__ __noinline__ double dense_cell_pairs(const float4 *__restrict__ pos32, const int *__restrict__ sidx,
                                                const int *seg_src, const int *seg_pre, const double (*cell_off)[3],
                                                const int *own_start, float4 *cf, int *csrc, int *acc,
                                                unsigned *queues, double alpha, double rcut, double cs,
                                                double *__restrict__ fr, int n, int u_first = 0, int u_last = 8,
                                                int ab_only = -1) {
  __shared__ int sa_sg[DENSE_NSEG], sa_cum[DENSE_NSEG + 1], sa_nseg;
  __shared__ unsigned qmax_bits;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int CH = PAIR_JCH32 - DENSE_ABLK;
  const float alphaf = (float)alpha;
  const float rcf = (float)rcut;
  const float fmul = fmaxf(alphaf * alphaf, 1.0f / (rcf * rcf));
  const float rc2f = rcf * rcf;
  const float prune_r2 = (float)(rcut * rcut * (1.0 + 1e-4));
  const float preff = (float)(2.0 * alpha / 1.77245385090551602729816748334);
  const float hf = (float)(0.5 * cs);
  unsigned *q = queues + warp * PAIR_QCAP;
  float e_sum = 0.0f, e_comp = 0.0f;
  unsigned head = 0, tail = 0;
  float fxs = 0.0f, fxs_inv = 0.0f, thr = 0.0f;
  if (tid == 0) qmax_bits = 0u;

  auto deposit = [&](int k, float sc, float ex, float ey, float ez, float fx, float fy, float fz) {
    const float sx = sc * ex, sy = sc * ey, sz = sc * ez;
    if (fmaxf(fabsf(sx), fmaxf(fabsf(sy), fabsf(sz))) < thr) {
      atomicAdd(&acc[3 * k], __float2int_rn(sx));
      atomicAdd(&acc[3 * k + 1], __float2int_rn(sy));
      atomicAdd(&acc[3 * k + 2], __float2int_rn(sz));
    } else {
      const int o = sidx[csrc[k]];
      atomicAdd(&fr[o], (double)fx);
      atomicAdd(&fr[(size_t)n + o], (double)fy);
      atomicAdd(&fr[2 * (size_t)n + o], (double)fz);
    }
  };
  auto process = [&](int take) {
    __syncwarp();
    if (lane < take) {
      const unsigned e = q[(head + lane) & (PAIR_QCAP - 1)];
      const int ki = (int)(e & 0xffffu), kj = (int)(e >> 16);
      const float4 pi = cf[ki], pj = cf[kj];
      const float ex = pi.x - pj.x, ey = pi.y - pj.y, ez = pi.z - pj.z;
      const float rr2 = ex * ex + ey * ey + ez * ez;
      const float rinv = rsqrtf(rr2);
      const float qq = pi.w * pj.w;
      const float ar = alphaf * (rr2 * rinv);
      const float gs = __expf(-ar * ar);
      const float ec = erfc_fit(ar, gs);
      const float kf = (ec * rinv + preff * gs) * (rinv * rinv);  // force / (q_i q_j r)
      const float fak = qq * kf;
      // i: +q_i q_j kf d in units fxs / |q_i| = q_j copysign(fxs, q_i) kf d;
      // j: the opposite force in units fxs / |q_j|; no units without charge
      deposit(ki, (pi.w != 0.0f ? pj.w * copysignf(fxs, pi.w) : 0.0f) * kf, ex, ey, ez, fak * ex, fak * ey,
              fak * ez);
      deposit(kj, -(pj.w != 0.0f ? pi.w * copysignf(fxs, pj.w) : 0.0f) * kf, ex, ey, ez, -fak * ex, -fak * ey,
              -fak * ez);
      const float term = qq * ec * rinv - e_comp;
      const float tsum = e_sum + term;
      e_comp = (tsum - e_sum) - term;
      e_sum = tsum;
    }
    head += take;
    __syncwarp();
  };
  auto warp_incl = [&](int v) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += t;
    }
    return v;
  };

  for (int u = u_first; u < u_last; u++) {
    const int srcA = own_start[u], nA = own_start[u + 1] - srcA;
    if (nA == 0) continue;
    const int U0 = (u >> 2) & 1, U1 = (u >> 1) & 1, U2 = u & 1;
    __syncthreads();
    if (warp == 0) {
      // A's candidate segments in column order (lane r < 25 owns column
      // (J0, J1) = (U0 - 2 + r / 5, U1 - 2 + r % 5); only the forward ones
      // r >= 12; z cut to the half-cells within rcut of A)
      int sgl = 0, nz = 0;
      if (lane >= 12 && lane < 25) {
        const int dj0 = lane / 5 - 2, dj1 = lane % 5 - 2;
        const float dx = (float)max(abs(dj0) - 1, 0) * hf, dy = (float)max(abs(dj1) - 1, 0) * hf;
        const float d2 = dx * dx + dy * dy;
        if (d2 <= prune_r2) {
          const int kz = min(2, 1 + (int)floorf(sqrtf(prune_r2 - d2) / hf));
          const int lo = (lane == 12) ? U2 : U2 - kz, hi = U2 + kz;
          sgl = (U0 + dj0 + 2) * 36 + (U1 + dj1 + 2) * 6 + 2 + lo;
          nz = hi - lo + 1;
        }
      }
      const int len = nz ? seg_pre[sgl + nz] - seg_pre[sgl] : 0;
      const int in_s = warp_incl(nz), in_l = warp_incl(len);
      const int s0 = in_s - nz;
      int cum = in_l - len;
      for (int zz = 0; zz < nz; zz++) {
        const int sg = sgl + zz;
        sa_sg[s0 + zz] = sg;
        sa_cum[s0 + zz] = cum;
        cum += seg_pre[sg + 1] - seg_pre[sg];
      }
      if (lane == 31) {
        sa_nseg = in_s;
        sa_cum[in_s] = in_l;
      }
    }
    __syncthreads();
    const int nseg = sa_nseg, C = sa_cum[nseg];
    for (int ab0 = ab_only >= 0 ? ab_only * DENSE_ABLK : 0; ab0 < (ab_only >= 0 ? min(nA, (ab_only + 1) * DENSE_ABLK) : nA);
         ab0 += DENSE_ABLK) {
      const int nab = min(DENSE_ABLK, nA - ab0);
      for (int cc0 = 0; cc0 < C; cc0 += CH) {
        const int ncand = min(CH, C - cc0);
        __syncthreads();
        // stage the A block (own cell: no offset) and the candidate chunk
        float qm = 0.0f;
        for (int t = tid; t < nab; t += PAIR_CTA) {
          const int src = srcA + ab0 + t;
          const float4 p = pos32[src];
          cf[t] = p;
          csrc[t] = src;
          acc[3 * t] = acc[3 * t + 1] = acc[3 * t + 2] = 0;
          qm = fmaxf(qm, fabsf(p.w));
        }
        for (int t = tid; t < ncand; t += PAIR_CTA) {
          const int c = cc0 + t;
          int sidx_s = 0;
#pragma unroll
          for (int step = 64; step > 0; step >>= 1)
            if (sidx_s + step < nseg && sa_cum[sidx_s + step] <= c) sidx_s += step;
          const int sg = sa_sg[sidx_s];
          const int src = seg_src[sg] + (c - sa_cum[sidx_s]);
          const int J0 = sg / 36, J1 = (sg / 6) % 6, J2 = sg % 6;
          const int cidx = ((J0 / 2) * 3 + J1 / 2) * 3 + J2 / 2;
          const float4 p = pos32[src];
          const int k = DENSE_ABLK + t;
          csrc[k] = src;
          acc[3 * k] = acc[3 * k + 1] = acc[3 * k + 2] = 0;
          cf[k] = make_float4(p.x + (float)cell_off[cidx][0], p.y + (float)cell_off[cidx][1],
                              p.z + (float)cell_off[cidx][2], p.w);
          qm = fmaxf(qm, fabsf(p.w));
        }
        qm = __int_as_float(__reduce_max_sync(0xffffffffu, (unsigned)__float_as_int(qm)));
        if (lane == 0) atomicMax(&qmax_bits, (unsigned)__float_as_int(qm));
        __syncthreads();
        const float fscale = __int_as_float((int)qmax_bits) * fmul;
        fxs = fscale > 0.0f ? 1048576.0f / fscale : 0.0f;
        fxs_inv = fscale * (1.0f / 1048576.0f);
        thr = fminf(16777216.0f, 1073741824.0f / (float)max(ncand, nab));
        for (int a0 = 0; a0 < nab; a0 += 32) {
          const int ng = min(32, nab - a0);
          const int lp = 32 - __clz(ng - 1);  // P = 2^lp >= ng
          const int ia = lane & ((1 << lp) - 1);
          const bool aval = ia < ng;
          const int ki = a0 + (aval ? ia : 0);
          const float4 pa = cf[ki];
          const int srci = csrc[ki];
          const int cpr = 32 >> lp;
          for (int cb = warp * cpr; cb < ncand; cb += PAIR_WARPS * cpr) {
            const int t = cb + (lane >> lp);
            const bool valid = aval && t < ncand;
            const int kk = DENSE_ABLK + (valid ? t : 0);
            const int srcc = csrc[kk];
            const float4 pc = cf[kk];
            const float dx = pa.x - pc.x, dy = pa.y - pc.y, dz = pa.z - pc.z;
            // forward: every candidate outside A; inside A the later slots
            const bool ok = valid & (srcc < srcA || srcc >= srcA + nA || srcc > srci) &
                            (dx * dx + dy * dy + dz * dz <= rc2f);
            const unsigned mask = __ballot_sync(0xffffffffu, ok);
            if (ok)
              q[(tail + __popc(mask & ((1u << lane) - 1u))) & (PAIR_QCAP - 1)] = (unsigned)ki | ((unsigned)kk << 16);
            tail += __popc(mask);
            if (tail - head >= 32) process(32);
          }
        }
        if (tail != head) process((int)(tail - head));
        __syncthreads();
        if (tid == 0) qmax_bits = 0u;  // every thread read it before the barrier above
        for (int k = tid; k < DENSE_ABLK + ncand; k += PAIR_CTA) {
          if (k >= nab && k < DENSE_ABLK) continue;
          const int ix = acc[3 * k], iy = acc[3 * k + 1], iz = acc[3 * k + 2];
          if (ix != 0 || iy != 0 || iz != 0) {
            const float inv = fxs_inv * fabsf(cf[k].w);
            const int o = sidx[csrc[k]];
            atomicAdd(&fr[o], (double)((float)ix * inv));
            atomicAdd(&fr[(size_t)n + o], (double)((float)iy * inv));
            atomicAdd(&fr[2 * (size_t)n + o], (double)((float)iz * inv));
          }
        }
      }
    }
  }
  return (double)e_sum - (double)e_comp;
}

// ADJ (one alpha, no Newton-3): the pair part of the energy's adjoint --
// fr -= ge f_i (dE_r/dx), pot += ge phi_i (dE_r/dq, phi_i = sum_j q_j
// erfc(alpha r)/r), energy[0] += E_r and energy[1] += dE_r/dalpha =
// 1/2 sum q_i q_j (-2/sqrt(pi)) exp(-alpha^2 r^2).
template <bool DBL, int NA, bool ADJ = false>
__global__ void __launch_bounds__(PAIR_CTA) pairs_cell_kernel(const void *__restrict__ posv,
                                                               const int *__restrict__ sidx,
                                                               const int *__restrict__ start, int nc, double L,
                                                               double rcut, double alpha_v,
                                                               const double *__restrict__ alphas, int nalpha,
                                                               double *__restrict__ fr, int n,
                                                               double *__restrict__ energy,
                                                               double *__restrict__ pot = nullptr, double ge = 0.0,
                                                               int2 *__restrict__ units = nullptr,
                                                               int *__restrict__ unit_count = nullptr) {
  typedef typename PairAcc<DBL>::type acc_t;
  static_assert(!ADJ || NA == 1, "the adjoint runs one alpha");
  constexpr int NC = ADJ ? 4 : 3;  // per-i sums: force (and the potential)
  // alpha batch: grid.y = group of NA alphas (alphas on the device), outputs
  // per alpha k at fr + 3 n k and energy + k; without alphas the scalar alpha_v
  const int a0 = blockIdx.y * NA;
  const int nag = alphas ? min(NA, nalpha - a0) : 1;
  double alpha_g[NA];
#pragma unroll
  for (int a = 0; a < NA; a++) alpha_g[a] = alphas ? (a < nag ? alphas[a0 + a] : 0.0) : alpha_v;
  const double alpha = alpha_g[0];
  fr += (size_t)a0 * 3 * (size_t)n;
  energy += a0;
  // FP32 with one alpha per CTA: Newton's third law -- each pair once, by
  // the CTA of the particle that comes first in the staged (J0, J1, J2,
  // slot) order, with the partner's force accumulated in shared memory and
  // added atomically.  FP64 keeps every ordered pair (the reference's loop,
  // reproducible bit for bit from run to run), and so does an alpha group,
  // whose per-alpha partner accumulators would not fit.
  constexpr bool N3 = pair_n3(DBL, NA) && !ADJ;
  constexpr int JCH = pair_jch(DBL, NA, ADJ);
  extern __shared__ __align__(16) unsigned char pair_smem[];
  float4 *cf = reinterpret_cast<float4 *>(pair_smem);
  int *csrc = reinterpret_cast<int *>(cf + JCH);  // sorted slot of each staged candidate
  float *sfj = reinterpret_cast<float *>(csrc + JCH);  // FP32: partner forces of the staged candidates
  float4 *spi = reinterpret_cast<float4 *>(N3 ? reinterpret_cast<unsigned char *>(sfj + 3 * JCH)
                                              : reinterpret_cast<unsigned char *>(csrc + JCH));
  constexpr int MAXI = pair_maxi(DBL);
  acc_t *sfi = reinterpret_cast<acc_t *>(spi + MAXI);  // [MAXI][NA][NC]
  unsigned short *queue = reinterpret_cast<unsigned short *>(sfi + NC * NA * MAXI);
  __shared__ int seg_src[PAIR_NSEG], seg_pre[PAIR_NSEG + 1];
  __shared__ double cell_off[27][3];
  __shared__ double ered[PAIR_WARPS][NA + (ADJ ? 1 : 0)];
  __shared__ float qmax_i_w[PAIR_WARPS];                         // FP32: |q| maxima of the i batch
  int *sfji = reinterpret_cast<int *>(sfj);                        // FP32: fixed-point partner forces
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned short *q = queue + warp * PAIR_QCAP;
  const int cell = blockIdx.x;
  const int c2 = cell % nc, c1 = (cell / nc) % nc, c0 = cell / (nc * nc);
  const double cs = L / nc;
  if (tid < 27) {
    const int d0 = tid / 9 - 1, d1 = (tid / 3) % 3 - 1, d2 = tid % 3 - 1;
    const int u0 = c0 + d0, u1 = c1 + d1, u2 = c2 + d2;
    const int w0 = wrap_full(u0, nc), w1 = wrap_full(u1, nc), w2 = wrap_full(u2, nc);
    if (DBL) {
      cell_off[tid][0] = (double)((u0 - w0) / nc) * L;  // periodic image: 0 or +-L
      cell_off[tid][1] = (double)((u1 - w1) / nc) * L;
      cell_off[tid][2] = (double)((u2 - w2) / nc) * L;
    } else {
      cell_off[tid][0] = d0 * cs;  // neighbour cell origin relative to this one
      cell_off[tid][1] = d1 * cs;
      cell_off[tid][2] = d2 * cs;
    }
  }
  // half-cell segments in grid order: J = 2 d + v in -2..3 per axis, J2 fastest
  for (int sg = tid; sg < PAIR_NSEG; sg += PAIR_CTA) {
    const int J0 = sg / 36 - 2, J1 = (sg / 6) % 6 - 2, J2 = sg % 6 - 2;
    const int d0 = (J0 + 2) / 2 - 1, d1 = (J1 + 2) / 2 - 1, d2 = (J2 + 2) / 2 - 1;
    const int v0 = (J0 + 2) & 1, v1 = (J1 + 2) & 1, v2 = (J2 + 2) & 1;
    const int w0 = wrap_full(c0 + d0, nc), w1 = wrap_full(c1 + d1, nc), w2 = wrap_full(c2 + d2, nc);
    const int key = ((w0 * nc + w1) * nc + w2) * 8 + (v0 << 2) + (v1 << 1) + v2;
    // FP32: only the half-cells that come after one of this cell's own in
    // (J0, J1, J2) order can hold forward partners
    const bool forward = !N3 || J0 >= 1 || (J0 == 0 && (J1 >= 1 || (J1 == 0 && J2 >= 0)));
    seg_src[sg] = start[key];
    seg_pre[sg + 1] = forward ? start[key + 1] - start[key] : 0;
  }
  __syncthreads();
  {
    __shared__ int scan_w[PAIR_WARPS];
    scan_segments(seg_pre, scan_w);
  }
  const int total = seg_pre[PAIR_NSEG];
  const bool fits = total <= JCH;
  const int i0 = start[cell * 8], i1 = start[cell * 8 + 8];
  // this cell's 8 half-cells: sorted-order starts and staged segment starts
  __shared__ int own_start[9], own_seg[8];
  if (tid < 9) own_start[tid] = start[cell * 8 + tid];
  if (tid < 8) own_seg[tid] = seg_pre[(2 + ((tid >> 2) & 1)) * 36 + (2 + ((tid >> 1) & 1)) * 6 + 2 + (tid & 1)];
  __syncthreads();
  const double ox = c0 * cs, oy = c1 * cs, oz = c2 * cs;
  const double Li = 1.0 / L;
  const double wupi = 1.77245385090551602729816748334;
  const float rc2f = DBL ? (float)(rcut * rcut * (1.0 + 1e-4)) : (float)rcut * (float)rcut;
  const float alphaf = (float)alpha;
  float alphaf_g[NA], preff_g[NA];
  double prefd_g[NA];
#pragma unroll
  for (int a = 0; a < NA; a++) {
    alphaf_g[a] = (float)alpha_g[a];
    preff_g[a] = (float)(2.0 * alpha_g[a] / wupi);
    prefd_g[a] = 2.0 * alpha_g[a] / wupi;
  }
  const float hf = (float)(0.5 * cs), hinvf = (float)(2.0 / cs);
  const float prune_r2 = (float)(rcut * rcut * (1.0 + 1e-4));
  const float4 *pos32 = reinterpret_cast<const float4 *>(posv);
  const double4 *pos64 = reinterpret_cast<const double4 *>(posv);
  // pair energy per lane in FP64; FP32 sums each particle's few terms per
  // lane in FP32 first (about 3 per lane at density 1) and adds them here
  double e_d[NA];
#pragma unroll
  for (int a = 0; a < NA; a++) e_d[a] = 0.0;
  // ADJ: dE_r/dalpha, likewise
  double de_d = 0.0;

  double e_dense = 0.0;
  if (N3 && !fits) {
    // FP32 Newton-3 and the forward neighbourhood does not fit: half-cell
    // groups with streamed candidates (dense_cell_pairs), either queued as
    // work units (one per block of DENSE_ABLK particles of an own
    // half-cell) for dense_units_kernel, which spreads a dense cell over
    // many CTAs, or, without a unit list, all here
    if (units) {
      if (tid < 8) {
        const int nA = own_start[tid + 1] - own_start[tid];
        const int nb = (nA + DENSE_ABLK - 1) / DENSE_ABLK;
        if (nb > 0) {
          const int base = atomicAdd(unit_count, nb);
          for (int b = 0; b < nb; b++) units[base + b] = make_int2(cell, (tid << 24) | b);
        }
      }
    } else {
      e_dense = dense_cell_pairs(pos32, sidx, seg_src, seg_pre, cell_off, own_start, cf, csrc, sfji,
                                 reinterpret_cast<unsigned *>(spi), alpha, rcut, cs, fr, n);
    }
  }
  // per i of the batch: its half-cell u (bits 0-2) and its own slot in
  // the flat staged order (bits 3+)
  __shared__ int sui[MAXI];
  for (int ib = i0; ib < ((N3 && !fits) ? i0 : i1); ib += MAXI) {
    const int ni = min(MAXI, i1 - ib);
    __syncthreads();
    float qmi = 0.0f;
    for (int t = tid; t < ni; t += PAIR_CTA) {
      {
        const int isorted = ib + t;
        int u = 0;
#pragma unroll
        for (int v = 1; v < 8; v++)
          if (isorted >= own_start[v]) u = v;
        sui[t] = ((own_seg[u] + (isorted - own_start[u])) << 3) | u;
      }
      if (DBL) {
        const double4 p = pos64[ib + t];
        spi[t] = make_float4((float)(p.x - ox), (float)(p.y - oy), (float)(p.z - oz), (float)p.w);
      } else {
        const float4 p = pos32[ib + t];
        spi[t] = p;
        qmi = fmaxf(qmi, fabsf(p.w));
      }
      for (int a = 0; a < NC * NA; a++) sfi[NC * NA * t + a] = (acc_t)0;
    }
    if (N3) {
      qmi = __int_as_float(__reduce_max_sync(0xffffffffu, (unsigned)__float_as_int(qmi)));
      if (lane == 0) qmax_i_w[warp] = qmi;
    }
    // all candidates in one chunk when they fit (pruned columns), else chunks
    // of the flat candidate order
    for (int k0 = 0; k0 < total; k0 += JCH) {
      const int kn = min(JCH, total - k0);
      __syncthreads();
#pragma unroll 4
      for (int kk = tid; kk < kn; kk += PAIR_CTA) {
        const int k = k0 + kk;
        int sg = 0;
#pragma unroll
        for (int step = 128; step > 0; step >>= 1)
          if (sg + step < PAIR_NSEG && seg_pre[sg + step] <= k) sg += step;
        const int src = seg_src[sg] + (k - seg_pre[sg]);
        const int J0 = sg / 36, J1 = (sg / 6) % 6, J2 = sg % 6;
        const int cidx = ((J0 / 2) * 3 + J1 / 2) * 3 + J2 / 2;
        csrc[kk] = src;
        if (N3) sfji[3 * kk] = sfji[3 * kk + 1] = sfji[3 * kk + 2] = 0;
        if (DBL) {
          const double4 p = pos64[src];
          cf[kk] = make_float4((float)(p.x + cell_off[cidx][0] - ox), (float)(p.y + cell_off[cidx][1] - oy),
                               (float)(p.z + cell_off[cidx][2] - oz), (float)p.w);
        } else {
          const float4 p = pos32[src];
          cf[kk] = make_float4(p.x + (float)cell_off[cidx][0], p.y + (float)cell_off[cidx][1],
                               p.z + (float)cell_off[cidx][2], p.w);
        }
      }
      __syncthreads();
      // FP32: fixed-point scale of the partner accumulators for this chunk,
      // divided by |q_j| per partner, and the squared distance from which on
      // every contribution stays below 2^24 units: |q_i| fxs kf r <= 2^20
      // (1 / r^2 + pref / r) / fmul, below 2^24 for 1 / r < x = (-pref +
      // sqrt(pref^2 + 64 fmul)) / 2 (erfc and the Gaussian at most 1); the
      // closer pairs go to the global FP64 force
      float fxs = 0.0f, fxs_inv = 0.0f, r2min = 0.0f;
      if (N3) {
        const float fm = fmaxf(alphaf * alphaf, 1.0f / ((float)rcut * (float)rcut));
        const float xr = 0.5f * (sqrtf(preff_g[0] * preff_g[0] + 64.0f * fm) - preff_g[0]);
        r2min = 1.02f / (xr * xr);
        float qi = 0.0f;
#pragma unroll
        for (int w = 0; w < PAIR_WARPS; w++) qi = fmaxf(qi, qmax_i_w[w]);
        const float fscale = qi * fmaxf(alphaf * alphaf, 1.0f / ((float)rcut * (float)rcut));
        if (fscale > 0.0f) {
          fxs = 1048576.0f / fscale;
          fxs_inv = fscale * (1.0f / 1048576.0f);
        }
      }
      for (int il = warp; il < ni; il += PAIR_WARPS) {
        const float4 pif = spi[il];
        double4 pid = make_double4(0.0, 0.0, 0.0, 0.0);
        if (DBL) pid = pos64[ib + il];
        // half-cell u of i and its own staged slot (excluded from its pairs)
        const int uk = sui[il];
        const int u = uk & 7;
        const int kself = (uk >> 3) - k0;
        acc_t fx[NA], fy[NA], fz[NA], ph[NA];
        float e_p[NA];  // FP32: this particle's energy terms of this lane
        float de_p = 0.0f;
#pragma unroll
        for (int a = 0; a < NA; a++) {
          fx[a] = fy[a] = fz[a] = ph[a] = (acc_t)0;
          e_p[a] = 0.0f;
        }
        unsigned head = 0, tail = 0;
        // evaluate `take` queued interactions (one per lane) and pop them
        auto process = [&](int take) {
          __syncwarp();
          if (lane < take) {
            const int sl = q[(head + lane) & (PAIR_QCAP - 1)];
            if (DBL) {
              const double4 pj = pos64[csrc[sl]];
              const double ddx = min_image(__dadd_rn(pid.x, -pj.x), Li, L);
              const double ddy = min_image(__dadd_rn(pid.y, -pj.y), Li, L);
              const double ddz = min_image(__dadd_rn(pid.z, -pj.z), Li, L);
              const double rr = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)), __dmul_rn(ddz, ddz)));
              if (rr <= rcut) {
#pragma unroll
                for (int a = 0; a < NA; a++) {
                  if (a < nag) {
                    const double ar = alpha_g[a] * rr;
                    const double ec = erfc(ar);
                    const double gd = exp(-ar * ar);
                    const double fak = pid.w * pj.w * (ec / rr + prefd_g[a] * gd) / (rr * rr);
                    fx[a] += fak * ddx;
                    fy[a] += fak * ddy;
                    fz[a] += fak * ddz;
                    e_d[a] += 0.5 * pid.w * pj.w * ec / rr;
                    if (ADJ) {
                      ph[a] += pj.w * ec / rr;
                      de_d += 0.5 * pid.w * pj.w * (-2.0 / wupi) * gd;
                    }
                  }
                }
              }
            } else {
              const float4 pj = cf[sl];
              const float ex = pif.x - pj.x, ey = pif.y - pj.y, ez = pif.z - pj.z;
              const float rr2 = ex * ex + ey * ey + ez * ez;
              const float rinv = rsqrtf(rr2);
              const float qq = pif.w * pj.w;
#pragma unroll
              for (int a = 0; a < NA; a++) {
                if (a >= nag) break;
              const float ar = alphaf_g[a] * (rr2 * rinv);
              const float gs = __expf(-ar * ar);
              const float ec = erfc_fit(ar, gs);
              const float kf = (ec * rinv + preff_g[a] * gs) * (rinv * rinv);  // force / (q_i q_j r)
              const float fak = qq * kf;
              fx[a] += fak * ex;
              fy[a] += fak * ey;
              fz[a] += fak * ez;
              if (N3) {
                // the partner's force -fak d in its units S_j = fxs / |q_j|:
                // -q_i q_j kf d fxs / |q_j| = -(q_i copysign(fxs, q_j)) kf d,
                // no division; a partner without charge takes no units (its
                // accumulator would otherwise fill with terms the flush
                // multiplies by |q_j| = 0)
                const float sk = -(pif.w * (pj.w != 0.0f ? copysignf(fxs, pj.w) : 0.0f)) * kf;
                const float sx = sk * ex, sy = sk * ey, sz = sk * ez;
                if (rr2 >= r2min) {
                  atomicAdd(&sfji[3 * sl], __float2int_rn(sx));
                  atomicAdd(&sfji[3 * sl + 1], __float2int_rn(sy));
                  atomicAdd(&sfji[3 * sl + 2], __float2int_rn(sz));
                } else {
                  const int o = sidx[csrc[sl]];
                  atomicAdd(&fr[o], (double)(-fak * ex));
                  atomicAdd(&fr[(size_t)n + o], (double)(-fak * ey));
                  atomicAdd(&fr[2 * (size_t)n + o], (double)(-fak * ez));
                }
              }
              e_p[a] = fmaf((N3 ? 1.0f : 0.5f) * qq, ec * rinv, e_p[a]);
              if (ADJ) {
                ph[a] += pj.w * ec * rinv;
                de_p = fmaf(-(float)(1.0 / wupi) * qq, gs, de_p);
              }
              }
            }
          }
          head += take;
          __syncwarp();
        };
        // one candidate test per lane; hits go to the warp's queue
        auto test_push = [&](int kk, bool valid) {
          const float4 pj = cf[valid ? kk : 0];
          const float dx = pif.x - pj.x, dy = pif.y - pj.y, dz = pif.z - pj.z;
          // N3 (only the pruned columns): the own column starts past i's
          // own slot, so every candidate comes after it
          const bool ok = valid & (dx * dx + dy * dy + dz * dz <= rc2f) & (N3 || kk != kself);
          const unsigned mask = __ballot_sync(0xffffffffu, ok);
          if (ok) q[(tail + __popc(mask & ((1u << lane) - 1u))) & (PAIR_QCAP - 1)] = (unsigned short)kk;
          tail += __popc(mask);
          // at most 63 queued: one full round drains it below 32
          if (tail - head >= 32) process(32);
        };
        if (fits) {
          // Candidate columns of this i: lane r < 25 owns the half-cell column
          // (J0, J1) = (U0 - 2 + r / 5, U1 - 2 + r % 5) (cells are wider than
          // rcut, so |J - U| <= 2 covers every partner).  The column is skipped
          // when its xy distance from i exceeds rcut and is otherwise clipped in
          // z to the half-cells the sphere reaches; prune_r2 carries a small
          // margin so no pair the exact test accepts is lost.
          const int U0 = (u >> 2) & 1, U1 = (u >> 1) & 1, U2 = u & 1;
          int ca = 0, clen = 0;
          // FP32 (Newton's third law): only the forward columns; in the own
          // column (lane 12) the half-cells from i's own on
          if (lane < 25 && (!N3 || lane >= 12)) {
            const int J0 = U0 - 2 + lane / 5, J1 = U1 - 2 + lane % 5;
            const float x0 = J0 * hf, y0 = J1 * hf;
            const float ddx = fmaxf(fmaxf(x0 - pif.x, pif.x - (x0 + hf)), 0.0f);
            const float ddy = fmaxf(fmaxf(y0 - pif.y, pif.y - (y0 + hf)), 0.0f);
            const float d2 = ddx * ddx + ddy * ddy;
            if (d2 <= prune_r2) {
              const float zr = sqrtf(prune_r2 - d2);
              const int lo = max((int)floorf((pif.z - zr) * hinvf), (N3 && lane == 12) ? U2 : U2 - 2);
              const int hi = min((int)floorf((pif.z + zr) * hinvf), U2 + 2);
              if (lo <= hi) {
                const int base = (J0 + 2) * 36 + (J1 + 2) * 6 + 2;
                ca = seg_pre[base + lo];
                const int ce = seg_pre[base + hi + 1];
                // Newton-3: i's own column from the slot after its own
                if (N3 && lane == 12) ca = max(ca, kself + 1);
                clen = max(ce - ca, 0);
              }
            }
          }
          // concatenate the non-empty columns: exclusive prefix of the lengths,
          // then lane t holds the start / prefix of the t-th non-empty column
          int incl = clen;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
          }
          const int ntot = __shfl_sync(0xffffffffu, incl, 31);
          const unsigned nem = __ballot_sync(0xffffffffu, clen > 0);
          const int excl = incl - clen;
          const int src = (int)__fns(nem, 0, lane + 1);
          const int colA = __shfl_sync(0xffffffffu, ca, src & 31);
          const int colE = __shfl_sync(0xffffffffu, excl, src & 31);
          const unsigned le = (lane == 31) ? 0xffffffffu : ((2u << lane) - 1u);
          int nbefore = 0;  // non-empty columns that start before this chunk
          for (int c0 = 0; c0 < ntot; c0 += 32) {
            const bool st = (clen > 0) & (excl >= c0) & (excl < c0 + 32);
            const unsigned smask = __reduce_or_sync(0xffffffffu, st ? (1u << ((excl - c0) & 31)) : 0u);
            const int rank = nbefore + __popc(smask & le) - 1;
            nbefore += __popc(smask);
            const int a = __shfl_sync(0xffffffffu, colA, rank & 31);
            const int e = __shfl_sync(0xffffffffu, colE, rank & 31);
            const int k = c0 + lane;
            test_push(a + (k - e), k < ntot);
          }
        } else {
          // the neighbourhood did not fit: this chunk of the flat candidate order
          for (int jb = 0; jb < kn; jb += 32) test_push(jb + lane, jb + lane < kn);
        }
        if (tail != head) process((int)(tail - head));
        if (!DBL) {
#pragma unroll
          for (int a = 0; a < NA; a++) e_d[a] += (double)e_p[a];
          if (ADJ) de_d += (double)de_p;
        }
#pragma unroll
        for (int a = 0; a < NA; a++) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            fx[a] += __shfl_xor_sync(0xffffffffu, fx[a], o);
            fy[a] += __shfl_xor_sync(0xffffffffu, fy[a], o);
            fz[a] += __shfl_xor_sync(0xffffffffu, fz[a], o);
            if (ADJ) ph[a] += __shfl_xor_sync(0xffffffffu, ph[a], o);
          }
          if (lane == 0) {
            acc_t *si = sfi + NC * (NA * il + a);
            si[0] += fx[a];
            si[1] += fy[a];
            si[2] += fz[a];
            if (ADJ) si[3] += ph[a];
          }
        }
      }
      if (N3) {
        // the partners' forces of this chunk, added to the global forces
        __syncthreads();
        for (int kk = tid; kk < kn; kk += PAIR_CTA) {
          const int ix = sfji[3 * kk], iy = sfji[3 * kk + 1], iz = sfji[3 * kk + 2];
          if (ix != 0 || iy != 0 || iz != 0) {
            const float inv = fxs_inv * fabsf(cf[kk].w);
            const float gx = (float)ix * inv, gy = (float)iy * inv, gz = (float)iz * inv;
            const int o = sidx[csrc[kk]];
            atomicAdd(&fr[o], (double)gx);
            atomicAdd(&fr[(size_t)n + o], (double)gy);
            atomicAdd(&fr[2 * (size_t)n + o], (double)gz);
          }
        }
      }
    }
    __syncthreads();
    for (int t = tid; t < ni; t += PAIR_CTA) {
      const int o = sidx[ib + t];
      if (N3) {
        atomicAdd(&fr[o], (double)sfi[3 * t]);
        atomicAdd(&fr[(size_t)n + o], (double)sfi[3 * t + 1]);
        atomicAdd(&fr[2 * (size_t)n + o], (double)sfi[3 * t + 2]);
      } else if (ADJ) {
        const acc_t *si = sfi + NC * t;
        fr[o] -= ge * (double)si[0];
        fr[(size_t)n + o] -= ge * (double)si[1];
        fr[2 * (size_t)n + o] -= ge * (double)si[2];
        pot[o] += ge * (double)si[3];
      } else {
        for (int a = 0; a < nag; a++) {
          double *fa = fr + (size_t)a * 3 * (size_t)n;
          const acc_t *si = sfi + NC * (NA * t + a);
          fa[o] += (double)si[0];
          fa[(size_t)n + o] += (double)si[1];
          fa[2 * (size_t)n + o] += (double)si[2];
        }
      }
    }
  }
#pragma unroll
  for (int a = 0; a < NA; a++) {
    double e_loc = e_d[a] + (a == 0 ? e_dense : 0.0);
    for (int o = 16; o > 0; o >>= 1) e_loc += __shfl_xor_sync(0xffffffffu, e_loc, o);
    if (lane == 0) ered[warp][a] = e_loc;
  }
  if (ADJ) {
    double d_loc = de_d;
    for (int o = 16; o > 0; o >>= 1) d_loc += __shfl_xor_sync(0xffffffffu, d_loc, o);
    if (lane == 0) ered[warp][ADJ ? NA : 0] = d_loc;
  }
  __syncthreads();
  if (tid < nag + (ADJ ? 1 : 0)) {
    double s = 0.0;
    for (int w = 0; w < PAIR_WARPS; w++) s += ered[w][tid];
    if (s != 0.0) atomicAdd(energy + tid, s);
  }
}

// Work units of the dense cells (queued by pairs_cell_kernel<false, 1>):
// a persistent grid takes (cell, own half-cell, block of DENSE_ABLK
// particles) units from the list through an atomic counter, sets up the
// cell's staged segments as pairs_cell_kernel does, and runs that unit of
// dense_cell_pairs.  A cell 13 times denser than the mean (the centre of a
// Gaussian system) thus spreads over tens of CTAs instead of one.
__global__ void __launch_bounds__(PAIR_CTA) dense_units_kernel(const float4 *__restrict__ pos32,
                                                                const int *__restrict__ sidx,
                                                                const int *__restrict__ start, int nc, double L,
                                                                double rcut, const double *__restrict__ alphas,
                                                                double alpha_v, double *__restrict__ fr, int n,
                                                                double *__restrict__ energy,
                                                                const int2 *__restrict__ units,
                                                                const int *__restrict__ unit_count,
                                                                int *__restrict__ unit_next) {
  constexpr int JCH = PAIR_JCH32;
  extern __shared__ __align__(16) unsigned char unit_smem[];
  float4 *cf = reinterpret_cast<float4 *>(unit_smem);
  int *csrc = reinterpret_cast<int *>(cf + JCH);
  int *acc = csrc + JCH;
  unsigned *queues = reinterpret_cast<unsigned *>(acc + 3 * JCH);
  __shared__ int seg_src[PAIR_NSEG], seg_pre[PAIR_NSEG + 1];
  __shared__ double cell_off[27][3];
  __shared__ int own_start[9];
  __shared__ int item_s;
  __shared__ int scan_w[PAIR_WARPS];
  __shared__ double ered[PAIR_WARPS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double alpha = alphas ? alphas[0] : alpha_v;
  const double cs = L / nc;
  const int count = *unit_count;
  if (count == 0) return;  // no dense cell: the usual case at uniform density
  double e_loc = 0.0;
  for (;;) {
    __syncthreads();
    if (tid == 0) item_s = atomicAdd(unit_next, 1);
    __syncthreads();
    const int item = item_s;
    if (item >= count) break;
    const int2 un = units[item];
    const int cell = un.x, u = un.y >> 24, ab = un.y & 0xffffff;
    const int c2 = cell % nc, c1 = (cell / nc) % nc, c0 = cell / (nc * nc);
    if (tid < 27) {
      cell_off[tid][0] = (tid / 9 - 1) * cs;
      cell_off[tid][1] = ((tid / 3) % 3 - 1) * cs;
      cell_off[tid][2] = (tid % 3 - 1) * cs;
    }
    for (int sg = tid; sg < PAIR_NSEG; sg += PAIR_CTA) {
      const int J0 = sg / 36 - 2, J1 = (sg / 6) % 6 - 2, J2 = sg % 6 - 2;
      const int d0 = (J0 + 2) / 2 - 1, d1 = (J1 + 2) / 2 - 1, d2 = (J2 + 2) / 2 - 1;
      const int v0 = (J0 + 2) & 1, v1 = (J1 + 2) & 1, v2 = (J2 + 2) & 1;
      const int w0 = wrap_full(c0 + d0, nc), w1 = wrap_full(c1 + d1, nc), w2 = wrap_full(c2 + d2, nc);
      const int key = ((w0 * nc + w1) * nc + w2) * 8 + (v0 << 2) + (v1 << 1) + v2;
      const bool forward = J0 >= 1 || (J0 == 0 && (J1 >= 1 || (J1 == 0 && J2 >= 0)));
      seg_src[sg] = start[key];
      seg_pre[sg + 1] = forward ? start[key + 1] - start[key] : 0;
    }
    if (tid < 9) own_start[tid] = start[cell * 8 + tid];
    __syncthreads();
    scan_segments(seg_pre, scan_w);
    e_loc += dense_cell_pairs(pos32, sidx, seg_src, seg_pre, cell_off, own_start, cf, csrc, acc, queues, alpha, rcut,
                              cs, fr, n, u, u + 1, ab);
  }
  for (int o = 16; o > 0; o >>= 1) e_loc += __shfl_xor_sync(0xffffffffu, e_loc, o);
  if (lane == 0) ered[warp] = e_loc;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int w = 0; w < PAIR_WARPS; w++) s += ered[w];
    if (s != 0.0) atomicAdd(energy, s);
  }
}

// Launch the cell kernel (FP64 or FP32 positions, already half-cell sorted).
// An alpha batch (alphas with nalpha > 1) runs in groups of PAIR_NA32 /
// PAIR_NA64 alphas per CTA.
template <bool DBL, int NA>
int launch_cells_na(const void *pos, const int *sidx, const int *start, int nc, double L, double rcut, double alpha,
                    const double *alphas, int nalpha, double *fr, int n, double *energy, cudaStream_t s) {
  static std::atomic<int> smem_set[P3MG_MAX_DEVICES];
  const size_t smem = pair_smem_bytes(DBL, NA);
  P3MG_CUDA_TRY(raise_smem_limit(pairs_cell_kernel<DBL, NA>, (int)smem, smem_set));
  const int groups = alphas ? (nalpha + NA - 1) / NA : 1;
  const dim3 grid(nc * nc * nc, groups);
  pairs_cell_kernel<DBL, NA><<<grid, PAIR_CTA, smem, s>>>(pos, sidx, start, nc, L, rcut, alpha, alphas, nalpha, fr,
                                                         n, energy);
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

// The pair part of the energy's adjoint (pairs_cell_kernel with ADJ):
// gx -= ge f, gq += ge phi, sums[0] += E_r, sums[1] += dE_r/dalpha.
template <bool DBL>
int launch_cells_adj(const void *pos, const int *sidx, const int *start, int nc, double L, double rcut, double alpha,
                     double *gx, double *gq, double ge, int n, double *sums, cudaStream_t s) {
  static std::atomic<int> smem_set[P3MG_MAX_DEVICES];
  const size_t smem = pair_smem_bytes(DBL, 1, true);
  P3MG_CUDA_TRY(raise_smem_limit(pairs_cell_kernel<DBL, 1, true>, (int)smem, smem_set));
  pairs_cell_kernel<DBL, 1, true><<<nc * nc * nc, PAIR_CTA, smem, s>>>(pos, sidx, start, nc, L, rcut, alpha, nullptr, 1,
                                                                      gx, n, sums, gq, ge);
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

// FP32, one alpha, with a work-unit list (units: capacity for every
// block of DENSE_ABLK particles of every half-cell; counters: 2 ints the
// caller zeroes before each call): the cell kernel, whose dense cells only
// queue units, then the persistent unit kernel.
int launch_cells_units(const void *pos, const int *sidx, const int *start, int nc, double L, double rcut, double alpha,
                       const double *alphas, double *fr, int n, double *energy, int2 *units, int *counters,
                       cudaStream_t s) {
  static std::atomic<int> smem_set[P3MG_MAX_DEVICES], units_smem_set[P3MG_MAX_DEVICES];
  const size_t smem = pair_smem_bytes(false, 1);
  P3MG_CUDA_TRY(raise_smem_limit(pairs_cell_kernel<false, 1>, (int)smem, smem_set));
  P3MG_CUDA_TRY(raise_smem_limit(dense_units_kernel, (int)smem, units_smem_set));
  pairs_cell_kernel<false, 1><<<nc * nc * nc, PAIR_CTA, smem, s>>>(pos, sidx, start, nc, L, rcut, alpha, alphas, 1, fr,
                                                                  n, energy, nullptr, 0.0, units, counters);
  P3MG_CUDA_TRY(cudaGetLastError());
  // persistent CTAs, as many as the device holds at once (7 per SM on a
  // B200: shared memory), counted once per device: a dense cell's units
  // spread over them; without dense cells each returns after one load
  static std::atomic<int> units_grid[P3MG_MAX_DEVICES];
  int dev = 0;
  P3MG_CUDA_TRY(cudaGetDevice(&dev));
  int grid = (dev >= 0 && dev < P3MG_MAX_DEVICES) ? units_grid[dev].load() : 0;
  if (grid <= 0) {
    int per_sm = 0, sms = 0;
    P3MG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dense_units_kernel, PAIR_CTA, smem));
    P3MG_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    grid = std::max(per_sm, 1) * std::max(sms, 1);
    if (dev >= 0 && dev < P3MG_MAX_DEVICES) units_grid[dev].store(grid);
  }
  dense_units_kernel<<<grid, PAIR_CTA, smem, s>>>(reinterpret_cast<const float4 *>(pos), sidx, start, nc, L, rcut,
                                                  alphas, alpha, fr, n, energy, units, counters, counters + 1);
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

// FP32 alpha sweeps over many alphas: lanes on alphas instead of pairs.
// The alpha-group form of pairs_cell_kernel runs the candidate search once
// per group of PAIR_NA32 alphas and keeps a force sum per alpha of the group
// in every lane (119 registers).  Here one warp per particle i runs the
// search once for up to PAIR_LA alphas; the lane that queued a pair forms
// its geometry once (r, q_i q_j / r^3 d, q_i q_j / (2 r)) and the warp
// broadcasts it, and each lane evaluates erfc and the Gaussian term for its
// own alphas, summing i's force for them in its own registers.  A group of
// more than 32 alphas takes alphas l and l + 32 on lane l; a smaller one is
// rounded up to A = 8, 16 or 32 lanes per pair, so that a step evaluates
// 32 / A pairs (lane = pair * A + alpha) and the sub-groups' sums are
// folded once per particle.  i's forces go straight to the alphas' force
// rows.  Every ordered pair (no Newton's third law), the staging and the
// column search of pairs_cell_kernel's FP32 path.
constexpr int PAIR_LA = 64;     // alphas per CTA (at most two per lane)
constexpr int PAIR_LA_MIN = 9;  // fewer alphas: one group of the alpha-group kernel

__host__ __device__ constexpr size_t pair_la_smem_bytes() {
  return (size_t)PAIR_JCH * sizeof(float4) + (size_t)PAIR_MAXI32 * sizeof(float4) +
         (size_t)PAIR_WARPS * PAIR_QCAP * sizeof(unsigned short);
}

__global__ void __launch_bounds__(PAIR_CTA) pairs_alpha_lanes_kernel(const float4 *__restrict__ pos32,
                                                                      const int *__restrict__ sidx,
                                                                      const int *__restrict__ start, int nc, double L,
                                                                      double rcut, const double *__restrict__ alphas,
                                                                      int nalpha, double *__restrict__ fr, int n,
                                                                      double *__restrict__ energy) {
  // grid.y = group of PAIR_LA alphas; alpha a of the group: forces at
  // fr + 3 n a, energy at energy[a]
  const int a0 = blockIdx.y * PAIR_LA;
  const int nag = min(PAIR_LA, nalpha - a0);
  fr += (size_t)a0 * 3 * (size_t)n;
  energy += a0;
  extern __shared__ __align__(16) unsigned char pair_smem[];
  float4 *cf = reinterpret_cast<float4 *>(pair_smem);  // staged candidates
  float4 *spi = cf + PAIR_JCH;                          // the i batch
  unsigned short *queue = reinterpret_cast<unsigned short *>(spi + PAIR_MAXI32);
  __shared__ int seg_src[PAIR_NSEG], seg_pre[PAIR_NSEG + 1];
  __shared__ float cell_off[27][3];
  __shared__ double ered[PAIR_WARPS][PAIR_LA];
  __shared__ int own_start[9], own_seg[8], sui[PAIR_MAXI32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned short *q = queue + warp * PAIR_QCAP;
  const int cell = blockIdx.x;
  const int c2 = cell % nc, c1 = (cell / nc) % nc, c0 = cell / (nc * nc);
  const double cs = L / nc;
  if (tid < 27) {
    // neighbour cell origin relative to this one
    cell_off[tid][0] = (float)((tid / 9 - 1) * cs);
    cell_off[tid][1] = (float)(((tid / 3) % 3 - 1) * cs);
    cell_off[tid][2] = (float)((tid % 3 - 1) * cs);
  }
  // the 6x6x6 half-cells around the cell in grid order, J2 fastest
  for (int sg = tid; sg < PAIR_NSEG; sg += PAIR_CTA) {
    const int J0 = sg / 36 - 2, J1 = (sg / 6) % 6 - 2, J2 = sg % 6 - 2;
    const int d0 = (J0 + 2) / 2 - 1, d1 = (J1 + 2) / 2 - 1, d2 = (J2 + 2) / 2 - 1;
    const int v0 = (J0 + 2) & 1, v1 = (J1 + 2) & 1, v2 = (J2 + 2) & 1;
    const int w0 = wrap_full(c0 + d0, nc), w1 = wrap_full(c1 + d1, nc), w2 = wrap_full(c2 + d2, nc);
    const int key = ((w0 * nc + w1) * nc + w2) * 8 + (v0 << 2) + (v1 << 1) + v2;
    seg_src[sg] = start[key];
    seg_pre[sg + 1] = start[key + 1] - start[key];
  }
  __syncthreads();
  {
    __shared__ int scan_w[PAIR_WARPS];
    scan_segments(seg_pre, scan_w);
  }
  const int total = seg_pre[PAIR_NSEG];
  const bool fits = total <= PAIR_JCH;
  const int i0 = start[cell * 8], i1 = start[cell * 8 + 8];
  if (tid < 9) own_start[tid] = start[cell * 8 + tid];
  if (tid < 8) own_seg[tid] = seg_pre[(2 + ((tid >> 2) & 1)) * 36 + (2 + ((tid >> 1) & 1)) * 6 + 2 + (tid & 1)];
  // lanes per pair A = 2^lgA and this lane's alphas: a0 + la and, with more
  // than 32 alphas in the group (A = 32), a0 + la + 32; sub = the pair of a
  // step this lane takes (all warp-uniform but sub and la)
  const double wupi = 1.77245385090551602729816748334;
  const bool two = nag > 32;
  const int lgA = nag > 16 ? 5 : nag > 8 ? 4 : 3;
  const int sub = lane >> lgA, la = lane & ((1 << lgA) - 1);
  float al[2], pf[2];
#pragma unroll
  for (int s = 0; s < 2; s++) {
    const double av = la + 32 * s < nag ? alphas[a0 + la + 32 * s] : 0.0;
    al[s] = (float)av;
    pf[s] = (float)(2.0 * av / wupi);
  }
  const float rc2f = (float)rcut * (float)rcut;
  const float hf = (float)(0.5 * cs), hinvf = (float)(2.0 / cs);
  const float prune_r2 = (float)(rcut * rcut * (1.0 + 1e-4));
  double e_d[2] = {0.0, 0.0};
  for (int ib = i0; ib < i1; ib += PAIR_MAXI32) {
    const int ni = min(PAIR_MAXI32, i1 - ib);
    __syncthreads();
    for (int t = tid; t < ni; t += PAIR_CTA) {
      const int isorted = ib + t;
      int u = 0;
#pragma unroll
      for (int v = 1; v < 8; v++)
        if (isorted >= own_start[v]) u = v;
      sui[t] = ((own_seg[u] + (isorted - own_start[u])) << 3) | u;
      spi[t] = pos32[ib + t];
    }
    for (int k0 = 0; k0 < total; k0 += PAIR_JCH) {
      const int kn = min(PAIR_JCH, total - k0);
      __syncthreads();
      for (int kk = tid; kk < kn; kk += PAIR_CTA) {
        const int k = k0 + kk;
        int sg = 0;
#pragma unroll
        for (int step = 128; step > 0; step >>= 1)
          if (sg + step < PAIR_NSEG && seg_pre[sg + step] <= k) sg += step;
        const int src = seg_src[sg] + (k - seg_pre[sg]);
        const int cidx = ((sg / 36 / 2) * 3 + (sg / 6) % 6 / 2) * 3 + (sg % 6) / 2;
        const float4 p = pos32[src];
        cf[kk] = make_float4(p.x + cell_off[cidx][0], p.y + cell_off[cidx][1], p.z + cell_off[cidx][2], p.w);
      }
      __syncthreads();
      for (int il = warp; il < ni; il += PAIR_WARPS) {
        const float4 pif = spi[il];
        const int uk = sui[il];
        const int u = uk & 7;
        const int kself = (uk >> 3) - k0;  // i's own staged slot in this chunk
        float fx[2] = {0.0f, 0.0f}, fy[2] = {0.0f, 0.0f}, fz[2] = {0.0f, 0.0f}, e_p[2] = {0.0f, 0.0f};
        unsigned head = 0, tail = 0;
        // evaluate the first `take` queued pairs for every alpha and pop them
        auto process = [&](int take) {
          __syncwarp();
          float wx = 0.0f, wy = 0.0f, wz = 0.0f, r = 0.0f, qh = 0.0f;
          if (lane < take) {
            const float4 pj = cf[q[(head + lane) & (PAIR_QCAP - 1)]];
            const float ex = pif.x - pj.x, ey = pif.y - pj.y, ez = pif.z - pj.z;
            const float rr2 = ex * ex + ey * ey + ez * ez;
            const float rinv = rsqrtf(rr2);
            const float qq = pif.w * pj.w;
            const float w3 = qq * (rinv * rinv * rinv);
            r = rr2 * rinv;
            wx = w3 * ex;
            wy = w3 * ey;
            wz = w3 * ez;
            qh = 0.5f * qq * rinv;
          }
          for (int p = 0; p < take; p += 32 >> lgA) {
            // pair p + sub of this step (src & 31: the shuffles run on every
            // lane; a lane past the queued pairs discards what it receives)
            const int src = p + sub;
            const float bwx = __shfl_sync(0xffffffffu, wx, src & 31), bwy = __shfl_sync(0xffffffffu, wy, src & 31);
            const float bwz = __shfl_sync(0xffffffffu, wz, src & 31), br = __shfl_sync(0xffffffffu, r, src & 31);
            const float bqh = __shfl_sync(0xffffffffu, qh, src & 31);
            if (src >= take) continue;
#pragma unroll
            for (int s = 0; s < 2; s++) {
              if (s == 1 && !two) break;
              // f = q_i q_j (erfc(a r) + 2 a / sqrt(pi) r exp(-a^2 r^2)) / r^3 d
              const float ar = al[s] * br;
              const float gs = __expf(-ar * ar);
              const float ec = erfc_fit(ar, gs);
              const float sc = fmaf(pf[s] * gs, br, ec);
              fx[s] = fmaf(sc, bwx, fx[s]);
              fy[s] = fmaf(sc, bwy, fy[s]);
              fz[s] = fmaf(sc, bwz, fz[s]);
              e_p[s] = fmaf(bqh, ec, e_p[s]);
            }
          }
          head += take;
          __syncwarp();
        };
        // one candidate test per lane; hits go to the warp's queue
        auto test_push = [&](int kk, bool valid) {
          const float4 pj = cf[valid ? kk : 0];
          const float dx = pif.x - pj.x, dy = pif.y - pj.y, dz = pif.z - pj.z;
          const bool ok = valid & (dx * dx + dy * dy + dz * dz <= rc2f) & (kk != kself);
          const unsigned mask = __ballot_sync(0xffffffffu, ok);
          if (ok) q[(tail + __popc(mask & ((1u << lane) - 1u))) & (PAIR_QCAP - 1)] = (unsigned short)kk;
          tail += __popc(mask);
          // at most 63 queued: one full round drains it below 32
          if (tail - head >= 32) process(32);
        };
        if (fits) {
          // lane r < 25 owns the half-cell column (U0 - 2 + r / 5, U1 - 2 +
          // r % 5), skipped beyond rcut in xy and clipped in z to the
          // half-cells the sphere reaches (as in pairs_cell_kernel)
          const int U0 = (u >> 2) & 1, U1 = (u >> 1) & 1, U2 = u & 1;
          int ca = 0, clen = 0;
          if (lane < 25) {
            const int J0 = U0 - 2 + lane / 5, J1 = U1 - 2 + lane % 5;
            const float x0 = J0 * hf, y0 = J1 * hf;
            const float ddx = fmaxf(fmaxf(x0 - pif.x, pif.x - (x0 + hf)), 0.0f);
            const float ddy = fmaxf(fmaxf(y0 - pif.y, pif.y - (y0 + hf)), 0.0f);
            const float d2 = ddx * ddx + ddy * ddy;
            if (d2 <= prune_r2) {
              const float zr = sqrtf(prune_r2 - d2);
              const int lo = max((int)floorf((pif.z - zr) * hinvf), U2 - 2);
              const int hi = min((int)floorf((pif.z + zr) * hinvf), U2 + 2);
              if (lo <= hi) {
                const int base = (J0 + 2) * 36 + (J1 + 2) * 6 + 2;
                ca = seg_pre[base + lo];
                clen = seg_pre[base + hi + 1] - ca;
              }
            }
          }
          // concatenate the non-empty columns (prefix of the lengths; lane t
          // then holds the start and prefix of the t-th non-empty column)
          int incl = clen;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
          }
          const int ntot = __shfl_sync(0xffffffffu, incl, 31);
          const unsigned nem = __ballot_sync(0xffffffffu, clen > 0);
          const int excl = incl - clen;
          const int src = (int)__fns(nem, 0, lane + 1);
          const int colA = __shfl_sync(0xffffffffu, ca, src & 31);
          const int colE = __shfl_sync(0xffffffffu, excl, src & 31);
          const unsigned le = (lane == 31) ? 0xffffffffu : ((2u << lane) - 1u);
          int nbefore = 0;  // non-empty columns that start before this step
          for (int c0s = 0; c0s < ntot; c0s += 32) {
            const bool st = (clen > 0) & (excl >= c0s) & (excl < c0s + 32);
            const unsigned smask = __reduce_or_sync(0xffffffffu, st ? (1u << ((excl - c0s) & 31)) : 0u);
            const int rank = nbefore + __popc(smask & le) - 1;
            nbefore += __popc(smask);
            const int a = __shfl_sync(0xffffffffu, colA, rank & 31);
            const int e = __shfl_sync(0xffffffffu, colE, rank & 31);
            const int k = c0s + lane;
            test_push(a + (k - e), k < ntot);
          }
        } else {
          // the neighbourhood did not fit: this chunk of the flat candidate order
          for (int jb = 0; jb < kn; jb += 32) test_push(jb + lane, jb + lane < kn);
        }
        if (tail != head) process((int)(tail - head));
        // fewer than 32 lanes per pair: fold the sub-groups' sums of each
        // alpha into the lanes of sub-group 0
        for (int o = 1 << lgA; o < 32; o <<= 1) {
          fx[0] += __shfl_xor_sync(0xffffffffu, fx[0], o);
          fy[0] += __shfl_xor_sync(0xffffffffu, fy[0], o);
          fz[0] += __shfl_xor_sync(0xffffffffu, fz[0], o);
          e_p[0] += __shfl_xor_sync(0xffffffffu, e_p[0], o);
        }
        // i's forces for this lane's alphas (one warp owns i: no race across
        // chunks), its energy terms summed in FP64
        const int o = sidx[ib + il];
        if (sub == 0) {
#pragma unroll
          for (int s = 0; s < 2; s++) {
            if (la + 32 * s < nag) {
              double *fa = fr + (size_t)(la + 32 * s) * 3 * (size_t)n;
              fa[o] += (double)fx[s];
              fa[(size_t)n + o] += (double)fy[s];
              fa[2 * (size_t)n + o] += (double)fz[s];
            }
            e_d[s] += (double)e_p[s];
          }
        }
      }
    }
  }
  ered[warp][lane] = e_d[0];
  ered[warp][lane + 32] = e_d[1];
  __syncthreads();
  if (tid < nag) {
    double s = 0.0;
    for (int w = 0; w < PAIR_WARPS; w++) s += ered[w][tid];
    if (s != 0.0) atomicAdd(energy + tid, s);
  }
}

int launch_cells_alpha_lanes(const void *pos, const int *sidx, const int *start, int nc, double L, double rcut,
                             const double *alphas, int nalpha, double *fr, int n, double *energy, cudaStream_t s) {
  static_assert(pair_la_smem_bytes() <= 48 * 1024, "default dynamic shared-memory limit");
  const dim3 grid(nc * nc * nc, (nalpha + PAIR_LA - 1) / PAIR_LA);
  pairs_alpha_lanes_kernel<<<grid, PAIR_CTA, pair_la_smem_bytes(), s>>>(
      reinterpret_cast<const float4 *>(pos), sidx, start, nc, L, rcut, alphas, nalpha, fr, n, energy);
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

int launch_pairs_cells(bool dbl, const void *pos, const int *sidx, const int *start, int nc, double L, double rcut,
                       double alpha, const double *alphas, int nalpha, double *fr, int n, double *energy,
                       cudaStream_t s) {
  const bool group = alphas != nullptr && nalpha > 1;
  if (!dbl && group && nalpha >= PAIR_LA_MIN)
    return launch_cells_alpha_lanes(pos, sidx, start, nc, L, rcut, alphas, nalpha, fr, n, energy, s);
  if (dbl)
    return group ? launch_cells_na<true, PAIR_NA64>(pos, sidx, start, nc, L, rcut, alpha, alphas, nalpha, fr, n,
                                                     energy, s)
                 : launch_cells_na<true, 1>(pos, sidx, start, nc, L, rcut, alpha, alphas, nalpha, fr, n, energy, s);
  return group ? launch_cells_na<false, PAIR_NA32>(pos, sidx, start, nc, L, rcut, alpha, alphas, nalpha, fr, n,
                                                    energy, s)
               : launch_cells_na<false, 1>(pos, sidx, start, nc, L, rcut, alpha, alphas, nalpha, fr, n, energy, s);
}

// All-pairs fallback (fewer than 3 cells per side): the reference's loop
// order for i, j tiles staged through shared memory.
__global__ void __launch_bounds__(BRUTE_THREADS) pairs_brute_kernel(const double *__restrict__ x,
                                                                     const double *__restrict__ y,
                                                                     const double *__restrict__ z,
                                                                     const double *__restrict__ q, int n, double L,
                                                                     double rcut, double alpha_v,
                                                                     const double *__restrict__ alphas,
                                                                     double *__restrict__ fr,
                                                                     double *__restrict__ energy) {
  // alpha batch as in pairs_cell_kernel
  const double alpha = alphas ? alphas[blockIdx.y] : alpha_v;
  fr += (size_t)blockIdx.y * 3 * (size_t)n;
  energy += blockIdx.y;
  __shared__ double4 sj[BRUTE_THREADS];
  __shared__ double ered[BRUTE_THREADS / 32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = i < n;
  const double Li = 1.0 / L;
  const double pref = 2.0 * alpha / 1.77245385090551602729816748334;
  double4 pi = act ? make_double4(x[i], y[i], z[i], q[i]) : make_double4(0, 0, 0, 0);
  double fx = 0, fy = 0, fz = 0, e_loc = 0;
  for (int jb = 0; jb < n; jb += BRUTE_THREADS) {
    __syncthreads();
    const int jj = jb + threadIdx.x;
    if (jj < n) sj[threadIdx.x] = make_double4(x[jj], y[jj], z[jj], q[jj]);
    __syncthreads();
    const int cnt = min(BRUTE_THREADS, n - jb);
    if (act)
      for (int t = 0; t < cnt; t++) {
        if (jb + t == i) continue;
        const double4 pj = sj[t];
        const double dx = min_image(__dadd_rn(pi.x, -pj.x), Li, L);
        const double dy = min_image(__dadd_rn(pi.y, -pj.y), Li, L);
        const double dz = min_image(__dadd_rn(pi.z, -pj.z), Li, L);
        const double r = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
        if (r <= rcut) {
          const double ar = alpha * r;
          const double ec = erfc(ar);
          const double fak = pi.w * pj.w * (ec / r + pref * exp(-ar * ar)) / (r * r);
          fx += fak * dx;
          fy += fak * dy;
          fz += fak * dz;
          e_loc += 0.5 * pi.w * pj.w * ec / r;
        }
      }
  }
  if (act) {
    fr[i] += fx;
    fr[(size_t)n + i] += fy;
    fr[2 * (size_t)n + i] += fz;
  }
  for (int o = 16; o > 0; o >>= 1) e_loc += __shfl_xor_sync(0xffffffffu, e_loc, o);
  if ((threadIdx.x & 31) == 0) ered[threadIdx.x >> 5] = e_loc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < BRUTE_THREADS / 32; w++) s += ered[w];
    if (s != 0.0) atomicAdd(energy, s);
  }
}

}  // namespace

// Cells strictly wider than rcut (by 1e-6 relative), so every pair within
// rcut lies within two half-cells along each axis.
static int cells_per_side(double L, double rcut) {
  int nc = (int)floor(L / (rcut * (1.0 + 1e-6)));
  return nc > 256 ? 256 : nc;
}

// Allocate the cell-list arrays for this rcut (host-side; called before a
// step is captured into a CUDA graph).  Keys: 8 half-cells per cell.
int pairs_reserve(Ctx *c, double rcut) {
  if (c->n == 0 || rcut <= 0.0) return P3MG_OK;
  const int nc = cells_per_side(c->L, rcut);
  if (nc < 3) return P3MG_OK;
  const int nkey = 8 * nc * nc * nc;
  // FP32 dense-cell work units: at most one per started block of
  // DENSE_ABLK particles of every half-cell, and the two counters
  if (c->precision != P3MG_FP64) {
    const size_t need = (size_t)c->cap / DENSE_ABLK + (size_t)nkey + 8;
    if (need > c->pair_units_cap) {
      if (c->pair_units) cudaFree(c->pair_units);
      c->pair_units = nullptr;
      c->pair_units_cap = 0;
      P3MG_CUDA_TRY(cudaMalloc(&c->pair_units, sizeof(int2) * need + 2 * sizeof(int)));
      c->pair_units_cap = need;
    }
  }
  if (nkey > c->ncell_cap) {
    if (c->cell_count) cudaFree(c->cell_count);
    if (c->cell_start) cudaFree(c->cell_start);
    c->cell_count = c->cell_start = nullptr;
    c->ncell_cap = 0;
    P3MG_CUDA_TRY(cudaMalloc(&c->cell_count, sizeof(int) * nkey));
    P3MG_CUDA_TRY(cudaMalloc(&c->cell_start, sizeof(int) * (nkey + 1)));
    c->ncell_cap = nkey;
    P3MG_TRY(scan_tmp_reserve(c, nkey));
  }
  return P3MG_OK;
}

// Bin the context's particles into the half-cell list of this rcut; sets
// *nc_out to the cells per side (0: fewer than 3, nothing binned).
int pairs_bin(Ctx *c, double rcut, int *nc_out) {
  const int n = c->n;
  *nc_out = 0;
  if (n == 0 || rcut <= 0.0) return P3MG_OK;
  const int nc = cells_per_side(c->L, rcut);
  if (nc < 3) return P3MG_OK;
  const int threads = 256;
  const int blocks = (n + threads - 1) / threads;
  const int nkey = 8 * nc * nc * nc;
  P3MG_TRY(pairs_reserve(c, rcut));
  c->ncell1 = nc;
  P3MG_CUDA_TRY(cudaMemsetAsync(c->cell_count, 0, sizeof(int) * nkey, c->stream));
  bin_cells_kernel<<<blocks, threads, 0, c->stream>>>(c->x, c->y, c->z, n, c->L, nc, c->cell_key, c->cell_count);
  c->launches++;
  P3MG_CUDA_TRY(cudaGetLastError());
  P3MG_TRY(exclusive_scan(c, c->cell_count, c->cell_start, nkey));
  if (c->precision == P3MG_FP64)
    place_cells_kernel<double4><<<blocks, threads, 0, c->stream>>>(c->x, c->y, c->z, c->q, n, c->L, nc, c->cell_key,
                                                                   c->cell_start, c->cell_idx,
                                                                   reinterpret_cast<double4 *>(c->cell_pos));
  else
    place_cells_kernel<float4><<<blocks, threads, 0, c->stream>>>(c->x, c->y, c->z, c->q, n, c->L, nc, c->cell_key,
                                                                  c->cell_start, c->cell_idx,
                                                                  reinterpret_cast<float4 *>(c->cell_pos));
  c->launches++;
  P3MG_CUDA_TRY(cudaGetLastError());
  *nc_out = nc;
  return P3MG_OK;
}

// The pair part of the energy's adjoint on the context's half-cell list
// (binned by pairs_bin with cells_per_side >= 3): gx -= ge dE_r/dx... as
// launch_cells_adj.  Returns P3MG_ERR_STATE when the list is not binned.
int pairs_adjoint(Ctx *c, double rcut, int nc, double ge, double *gx, double *gq, double *sums) {
  if (nc < 3) return P3MG_ERR_STATE;
  if (c->precision == P3MG_FP64)
    P3MG_TRY(launch_cells_adj<true>(c->cell_pos, c->cell_idx, c->cell_start, nc, c->L, rcut, c->alpha, gx, gq, ge, c->n,
                                    sums, c->stream));
  else
    P3MG_TRY(launch_cells_adj<false>(c->cell_pos, c->cell_idx, c->cell_start, nc, c->L, rcut, c->alpha, gx, gq, ge,
                                     c->n, sums, c->stream));
  c->launches++;
  return P3MG_OK;
}

// Real-space forces of the context's particles for nalpha alphas (device
// array) into fr + 3 n k and energy + k, k = 0 .. nalpha-1 (accumulated).
int pairs_run(Ctx *c, double rcut, const double *alphas, int nalpha, double *fr, double *energy) {
  const int n = c->n;
  if (n == 0 || rcut <= 0.0) return P3MG_OK;
  int nc = 0;
  if (cells_per_side(c->L, rcut) < 3) {
    const int threads = 256;
    const int blocks = (n + threads - 1) / threads;
    mark(c, EV_K0);
    pairs_brute_kernel<<<dim3(blocks, nalpha), BRUTE_THREADS, 0, c->stream>>>(c->x, c->y, c->z, c->q, n, c->L, rcut,
                                                                               0.0, alphas, fr, energy);
    c->launches++;
    mark(c, EV_K1);
    P3MG_CUDA_TRY(cudaGetLastError());
    return P3MG_OK;
  }
  P3MG_TRY(pairs_bin(c, rcut, &nc));
  mark(c, EV_K0);
  if (c->precision != P3MG_FP64 && !(alphas != nullptr && nalpha > 1) && c->pair_units) {
    int2 *units = reinterpret_cast<int2 *>(c->pair_units);
    int *counters = reinterpret_cast<int *>(units + c->pair_units_cap);
    P3MG_CUDA_TRY(cudaMemsetAsync(counters, 0, 2 * sizeof(int), c->stream));
    P3MG_TRY(launch_cells_units(c->cell_pos, c->cell_idx, c->cell_start, nc, c->L, rcut, 0.0, alphas, fr, n, energy,
                                units, counters, c->stream));
    c->launches += 2;
  } else {
    P3MG_TRY(launch_pairs_cells(c->precision == P3MG_FP64, c->cell_pos, c->cell_idx, c->cell_start, nc, c->L, rcut,
                                0.0, alphas, nalpha, fr, n, energy, c->stream));
    c->launches++;
  }
  mark(c, EV_K1);
  return P3MG_OK;
}

// ---------------------------------------------------------------------------
// Real-space pair forces without any device allocation.
//
// Some callers cannot let a library allocate device memory: an MD engine or
// framework that owns all device memory through its own pool (a cudaMalloc
// from the library would synchronise the device and fragment that pool),
// or a time-stepping loop that fixes its memory at start-up and must not
// allocate afterwards.  p3mg_real_forces_noalloc serves them: the caller
// passes device-accessible inputs and outputs and a stream, and the cell
// list lives in the file-scope array below, which is part of the loaded
// module (every GPU that loads the library holds it until the process
// exits).  Its capacity bounds the particle count; the cell grid is capped
// so that it fits as well (cells stay at least rcut wide, so the pairs found
// are the same).  The cell list has 8 half-cell keys per cell.  All calls on a device share the one array and it keeps
// the previous call's contents: the per-call counters are cleared on the
// caller's stream before use, and calls that overlap on the GPU (different
// streams, or host threads racing) corrupt each other's cell lists.
// ---------------------------------------------------------------------------

namespace {

constexpr size_t NA_CELL_BYTES = sizeof(int) * (size_t)P3MG_NOALLOC_MAX_CELLS;
constexpr size_t NA_PART_INT_BYTES = sizeof(int) * (size_t)P3MG_NOALLOC_MAX_PARTICLES;
constexpr size_t na_round(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t NA_OFF_COUNT = 0;
constexpr size_t NA_OFF_START = NA_OFF_COUNT + na_round(NA_CELL_BYTES);
constexpr size_t NA_OFF_KEY = NA_OFF_START + na_round(NA_CELL_BYTES + sizeof(int));  // (key, rank) per particle
constexpr size_t NA_OFF_IDX = NA_OFF_KEY + na_round(2 * NA_PART_INT_BYTES);
constexpr size_t NA_OFF_POS = NA_OFF_IDX + na_round(NA_PART_INT_BYTES);
constexpr size_t NA_BYTES = NA_OFF_POS + na_round(sizeof(double4) * (size_t)P3MG_NOALLOC_MAX_PARTICLES);
static_assert(NA_BYTES <= (size_t)P3MG_NOALLOC_SCRATCH_BYTES, "no-alloc scratch layout exceeds its array");

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[P3MG_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int NA_MAX_DEVICES = 64;
std::atomic<unsigned char *> g_na_ptr[NA_MAX_DEVICES];

// Device address of the scratch array for the current device.  In host
// code the symbol name only stands for the array, it is not an address the
// GPU can use, so the address is looked up once per device (with that
// device current) and cached.  Host threads that make their first call on
// a device at the same time each look it up and store the same value; the
// cache slots are atomic so that this is well defined.
int noalloc_scratch(unsigned char **out) {
  int dev = 0;
  P3MG_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NA_MAX_DEVICES) return P3MG_ERR_ARG;
  unsigned char *p = g_na_ptr[dev].load(std::memory_order_acquire);
  if (!p) {
    void *a = nullptr;
    P3MG_CUDA_TRY(cudaGetSymbolAddress(&a, g_noalloc_scratch));
    p = (unsigned char *)a;
    g_na_ptr[dev].store(p, std::memory_order_release);
  }
  *out = p;
  return P3MG_OK;
}

}  // namespace

}  // namespace p3mg

extern "C" int p3mg_real_forces_noalloc(int n, const double *x, const double *y, const double *z, const double *q,
                                        double L, double rcut, double alpha, int precision, double *fr, double *energy,
                                        void *stream) {
  using namespace p3mg;
  if (n < 0 || !(L > 0.0) || !(rcut >= 0.0) || !(alpha >= 0.0)) return P3MG_ERR_ARG;
  if (precision != P3MG_FP64 && precision != P3MG_FP32_MIXED) return P3MG_ERR_PRECISION;
  if (n > P3MG_NOALLOC_MAX_PARTICLES) return P3MG_ERR_NOBUF;
  if (n == 0 || rcut == 0.0) return P3MG_OK;
  if (!x || !y || !z || !q || !fr || !energy) return P3MG_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned char *base = nullptr;
  P3MG_TRY(noalloc_scratch(&base));
  const int threads = 256;
  const int blocks = (n + threads - 1) / threads;
  int nc = cells_per_side(L, rcut);
  if (nc < 3) {
    pairs_brute_kernel<<<blocks, BRUTE_THREADS, 0, s>>>(x, y, z, q, n, L, rcut, alpha, nullptr, fr, energy);
    P3MG_CUDA_TRY(cudaGetLastError());
    return P3MG_OK;
  }
  while (nc > 3 && 8 * nc * nc * nc > P3MG_NOALLOC_MAX_CELLS) nc--;
  const int ncell = 8 * nc * nc * nc;  // half-cell keys
  int *count = (int *)(base + NA_OFF_COUNT);
  int *start = (int *)(base + NA_OFF_START);
  int2 *key = (int2 *)(base + NA_OFF_KEY);
  int *idx = (int *)(base + NA_OFF_IDX);
  void *pos = (void *)(base + NA_OFF_POS);
  // the array keeps the previous call's counters: clear them first
  P3MG_CUDA_TRY(cudaMemsetAsync(count, 0, sizeof(int) * ncell, s));
  bin_cells_kernel<<<blocks, threads, 0, s>>>(x, y, z, n, L, nc, key, count);
  P3MG_CUDA_TRY(cudaGetLastError());
  P3MG_TRY(scan_counts(count, start, ncell, s));
  if (precision == P3MG_FP64) {
    place_cells_kernel<double4><<<blocks, threads, 0, s>>>(x, y, z, q, n, L, nc, key, start, idx,
                                                           reinterpret_cast<double4 *>(pos));
    P3MG_CUDA_TRY(cudaGetLastError());
    P3MG_TRY(launch_pairs_cells(true, pos, idx, start, nc, L, rcut, alpha, nullptr, 1, fr, n, energy, s));
  } else {
    place_cells_kernel<float4><<<blocks, threads, 0, s>>>(x, y, z, q, n, L, nc, key, start, idx,
                                                          reinterpret_cast<float4 *>(pos));
    P3MG_CUDA_TRY(cudaGetLastError());
    P3MG_TRY(launch_pairs_cells(false, pos, idx, start, nc, L, rcut, alpha, nullptr, 1, fr, n, energy, s));
  }
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}
