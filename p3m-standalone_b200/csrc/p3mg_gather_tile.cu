// FP32 ik back-interpolation through shared-memory brick tiles
// (the force assignment of the ik methods, charge-assign.c:646-725 for the
// interlaced pair of meshes, charge-assign.c:560-644 for one mesh).
//
// One CTA per mesh brick (the B^3 stencil bases of the brick-sorted
// particles).  The CTA first stages the packed field vectors (F_x, F_y,
// F_z, 0) of every mesh point its particles' stencils reach -- a tile of
// T = B + cao - 1 (+ 1 for the half-cell-shifted mesh) points per axis per
// mesh -- in shared memory: one TMA tensor copy per mesh when the tile lies
// inside the mesh, plain loads with the periodic wrap otherwise.  Then each
// warp takes one particle at a time with its lanes on the (mesh, b, c)
// columns of the stencil (lane k of round r owns column 32 r + k of the
// NMESH cao^2 columns) and sums the column's cao points a = 0..cao-1.  With
// the tile's row pitch = cao (mod 8) in 16-byte vectors (15 for the
// headline's B = 8, cao 7, interlaced), the 8 lanes of each quarter-warp
// read 8 different 16-byte bank groups, so a load instruction costs the
// minimum four shared-memory wavefronts; the thread-per-particle gather's
// scattered 16-byte global loads touch 8-10 cache lines each.  The weights
// are computed once per particle by a few lanes (geometry with the
// reference's 2^-17 offset bins, FP32 B-spline recursion, the charge and
// prefactor folded into the x weights) and handed over through a per-warp
// shared-memory slot; the column sums are reduced across the warp.
#include <cuda.h>

#include <type_traits>

#include "p3mg_internal.cuh"

namespace p3mg {

namespace {

constexpr int GT_THREADS = 256;  // 8 warps; two CTAs per SM with the B = 8 interlaced tile
constexpr int GT_WARPS = GT_THREADS / 32;
constexpr int GT_GROUP_LANES = 30;  // prologue lanes: (particle, mesh, axis) of a particle group

// particles whose weights a warp prepares at once
__host__ __device__ constexpr int gt_group(int nmesh) { return GT_GROUP_LANES / (3 * nmesh); }

// floats of one particle's weight slot: per mesh 3 axes x CAO weights and
// the tile offset of the stencil origin (as an int)
__host__ __device__ constexpr int gt_slot(int cao, int nmesh) { return nmesh * (3 * cao + 1); }

__host__ __device__ inline int gt_tile_edge(int B, int cao, int nmesh) { return B + cao - 1 + (nmesh == 2 ? 1 : 0); }

// Tile layout of one mesh: [a][b][c] with T planes and rows, a row pitch
// TZ >= T with TZ = cao (mod 8) -- lane k = cao b + c of a round then reads
// vector TZ b + c = k (mod 8) past the stencil origin, a different 16-byte
// bank group for each lane of a quarter-warp -- and the tile stride rounded
// up to a multiple of 8 vectors (128 bytes: the next tile is a TMA
// destination too, and the bank groups of the meshes stay aligned).
__host__ __device__ inline int gt_row_pitch(int T, int cao) { return T + (((cao - T) % 8) + 8) % 8; }
__host__ __device__ inline int gt_tile_stride(int T, int cao) { return (T * T * gt_row_pitch(T, cao) + 7) & ~7; }

__host__ __device__ inline size_t gt_smem_bytes(int B, int cao, int nmesh) {
  const int T = gt_tile_edge(B, cao, nmesh);
  return (size_t)nmesh * gt_tile_stride(T, cao) * 16 + (size_t)GT_WARPS * gt_group(nmesh) * gt_slot(cao, nmesh) * 4 +
         16;
}

// bounded wait on the tile's mbarrier (phase 0), called by whole warps:
// each lane polls until it has seen the TMA copies land itself (its acquire
// of their writes); the warp leaves together, and after about 2^22 polls
// (seconds) it records an error in *status and returns false (the CTA then
// skips its particles)
__device__ __forceinline__ bool gt_wait_tile(uint32_t bar, int *status) {
  bool done = false;
  for (int it = 0; it < (1 << 22); it++) {
    if (!done) {
      uint32_t d;
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}"
          : "=r"(d)
          : "r"(bar), "r"(0)
          : "memory");
      done = d != 0;
    }
    if (__all_sync(0xffffffffu, done)) return true;
  }
  if ((threadIdx.x & 31) == 0 && status) atomicOr(status, 1);
  return false;
}

template <int CAO, int NMESH>
__global__ void __launch_bounds__(GT_THREADS, 2) gather_tile_kernel(
    const __grid_constant__ CUtensorMap tmap, int use_tma, const double4 *__restrict__ sxyzq,
    const int *__restrict__ sidx, const int *__restrict__ start, int m, int B, int nb, double Hi, double shift,
    double pref, const float4 *__restrict__ Pv, size_t M, double *__restrict__ fk, int n, int *status) {
  constexpr int NCOL = NMESH * CAO * CAO;  // (mesh, b, c) columns of a stencil
  constexpr int NR = (NCOL + 31) / 32;     // rounds of 32 columns
  constexpr int GRP = gt_group(NMESH);
  constexpr int SLOT = gt_slot(CAO, NMESH);
  extern __shared__ __align__(128) unsigned char gt_smem[];
  const int T = gt_tile_edge(B, CAO, NMESH);
  const int TZ = gt_row_pitch(T, CAO);  // row pitch (z)
  const int PL = T * TZ;                // plane pitch (y rows of one x)
  const int TS = gt_tile_stride(T, CAO);
  float4 *tile = reinterpret_cast<float4 *>(gt_smem);  // [NMESH][TS]
  float *wslot = reinterpret_cast<float *>(tile + NMESH * TS);  // [warp][GRP][SLOT]
  uint64_t *bar = reinterpret_cast<uint64_t *>(wslot + GT_WARPS * GRP * SLOT);
  const int bid = blockIdx.x;
  const int B3 = B * B * B;
  const int p0 = start[bid * B3], p1 = start[(bid + 1) * B3];
  if (p0 == p1) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int bz = bid % nb, by = (bid / nb) % nb, bx = bid / (nb * nb);
  const int o0 = bx * B, o1 = by * B, o2 = bz * B;
  const float4 *__restrict__ P = Pv + (size_t)blockIdx.y * NMESH * M;  // alpha batch (grid.y)
  fk += (size_t)blockIdx.y * 3 * (size_t)n;

  // ---- stage the tile(s).  TMA: one box of (4 floats, TZ, T, T) per mesh
  // (the TZ - T extra z points are never read; past the mesh end the copy
  // fills zeros), when the T^3 points needed lie inside the mesh
  const bool inside = use_tma && o0 + T <= m && o1 + T <= m && o2 + T <= m;
  const uint32_t bar_s = (uint32_t)__cvta_generic_to_shared(bar);
  if (inside) {
    if (tid == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_s), "r"(1) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      const uint32_t bytes = (uint32_t)(NMESH * T * PL * 16);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_s), "r"(bytes) : "memory");
#pragma unroll
      for (int ii = 0; ii < NMESH; ii++) {
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(tile + ii * TS);
        // coordinates innermost first: vector component 0 (a 16-byte aligned
        // start), z, y, x, mesh plane of this batch entry
        const int plane = (int)blockIdx.y * NMESH + ii;
        asm volatile(
            "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
            "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(0), "r"(o2), "r"(o1), "r"(o0), "r"(plane), "r"(bar_s)
            : "memory");
      }
    }
  } else {
    // plain loads with the periodic wrap: one tile row (T <= 16 consecutive
    // z) per half-warp, rows spread over the warps
    for (int row = warp * 2 + (lane >> 4); row < NMESH * T * T; row += 2 * GT_WARPS) {
      const int c = lane & 15;
      if (c < T) {
        const int ii = row / (T * T), rr = row - ii * T * T, a = rr / T, b = rr - a * T;
        int gi = o0 + a, gj = o1 + b, gk = o2 + c;
        gi -= (gi >= m) ? m : 0;
        gj -= (gj >= m) ? m : 0;
        gk -= (gk >= m) ? m : 0;
        if (gi >= m) gi %= m;
        if (gj >= m) gj %= m;
        if (gk >= m) gk %= m;
        tile[ii * TS + a * PL + b * TZ + c] = P[(size_t)ii * M + ((size_t)gi * m + gj) * m + gk];
      }
    }
  }
  __syncthreads();  // the barrier is initialised (TMA) or the tile is loaded (plain loads)
  // TMA: each warp computes its first group's weights before it waits for
  // the tile
  bool tile_ready = !inside;

  // ---- this lane's columns.  Full rounds: column 32 r + lane of the
  // NCOL (mesh, b, c) columns, its tile offset past the mesh's stencil
  // origin and its y / z weight indices in a particle slot.  The LEFT
  // columns past the full rounds are summed point by point: lane t of a
  // point pass takes point (column, a) = (32 NFULL + t / CAO, t % CAO).
  constexpr int NFULL = NCOL / 32;
  constexpr int LEFT = NCOL - 32 * NFULL;
  constexpr int NPP = (LEFT * CAO + 31) / 32;
  constexpr int WY = NMESH * CAO, WZ = 2 * NMESH * CAO, OFF = 3 * NMESH * CAO;  // slot layout (floats)
  int coff[NFULL > 0 ? NFULL : 1], cwy[NFULL > 0 ? NFULL : 1], cwz[NFULL > 0 ? NFULL : 1];
  bool cii[NFULL > 0 ? NFULL : 1];
#pragma unroll
  for (int r = 0; r < NFULL; r++) {
    const int k = 32 * r + lane;
    const int ii = k / (CAO * CAO), bc = k - ii * CAO * CAO, b = bc / CAO, c = bc - b * CAO;
    coff[r] = ii * TS + b * TZ + c;
    cii[r] = ii != 0;
    cwy[r] = WY + ii * CAO + b;
    cwz[r] = WZ + ii * CAO + c;
  }
  int poff[NPP > 0 ? NPP : 1], pwy[NPP > 0 ? NPP : 1], pwz[NPP > 0 ? NPP : 1], pwx[NPP > 0 ? NPP : 1];
  bool pii[NPP > 0 ? NPP : 1];
#pragma unroll
  for (int r = 0; r < NPP; r++) {
    const int t = 32 * r + lane;
    if (t < LEFT * CAO) {
      const int k = 32 * NFULL + t / CAO, a = t % CAO;
      const int ii = k / (CAO * CAO), bc = k - ii * CAO * CAO, b = bc / CAO, c = bc - b * CAO;
      poff[r] = ii * TS + a * PL + b * TZ + c;
      pii[r] = ii != 0;
      pwy[r] = WY + ii * CAO + b;
      pwz[r] = WZ + ii * CAO + c;
      pwx[r] = a * NMESH + ii;
    } else {
      poff[r] = -1;
      pii[r] = false;
      pwy[r] = pwz[r] = pwx[r] = 0;
    }
  }
  const double scale = (NMESH == 2) ? 0.5 * pref : pref;
  float *myslot = wslot + warp * GRP * SLOT;
  const int np = p1 - p0;
  // prologue lane (j, ii, d): axis d of mesh ii of particle j of a group
  const int pj = lane / (NMESH * 3), pmi = (lane / 3) % NMESH, pd = lane % 3;
  const bool plane_ok = lane < GRP * NMESH * 3;
  // the first group's particle, loaded ahead (each later one is loaded
  // while the previous group is summed)
  int g0 = warp * GRP;
  double4 rnext = make_double4(0.0, 0.0, 0.0, 0.0);
  if (plane_ok && g0 + pj < np) rnext = sxyzq[p0 + g0 + pj];
  for (; g0 < np; g0 += GT_WARPS * GRP) {
    __syncwarp();
    const bool act = plane_ok && g0 + pj < np;
    {
      const double4 r = rnext;
      const double xc = pd == 0 ? r.x : (pd == 1 ? r.y : r.z);
      int base, arg;
      mesh_geometry(xc, Hi, shift, pmi, m, &base, &arg);
      int rel = base - (pd == 0 ? o0 : (pd == 1 ? o1 : o2));
      rel += (rel < 0) ? m : 0;
      // tile offset of the stencil origin: the three axes' parts summed
      // on the lane of axis 0
      const int part = rel * (pd == 0 ? PL : (pd == 1 ? TZ : 1));
      const int part1 = __shfl_down_sync(0xffffffffu, part, 1);
      const int part2 = __shfl_down_sync(0xffffffffu, part, 2);
      if (act) {
        float w[CAO];
        bspline_weights<float, CAO, false>(arg, w, nullptr);
        float *sp = myslot + pj * SLOT;
        if (pd == 0) {
          // -(scale q) folded into the x weights (f -= scale q W F), stored
          // as (mesh 0, mesh 1) pairs per a
          const float fold = (float)(-scale * r.w);
#pragma unroll
          for (int t = 0; t < CAO; t++) sp[t * NMESH + pmi] = w[t] * fold;
          reinterpret_cast<int *>(sp)[OFF + pmi] = part + part1 + part2;
        } else {
#pragma unroll
          for (int t = 0; t < CAO; t++) sp[(pd == 1 ? WY : WZ) + pmi * CAO + t] = w[t];
        }
      }
    }
    const int gn = min(GRP, np - g0);
    // lane j < gn keeps particle j's force; its output slot and current
    // force and the next group's particles are loaded while the group is
    // summed
    const int oidx = lane < gn ? sidx[p0 + g0 + lane] : 0;
    double fk0 = 0.0, fk1 = 0.0, fk2 = 0.0;
    if (lane < gn) {
      fk0 = fk[oidx];
      fk1 = fk[(size_t)n + oidx];
      fk2 = fk[2 * (size_t)n + oidx];
    }
    {
      const int gnext = g0 + GT_WARPS * GRP;
      if (plane_ok && gnext + pj < np) rnext = sxyzq[p0 + gnext + pj];
    }
    __syncwarp();
    if (!tile_ready) {
      if (!gt_wait_tile(bar_s, status)) return;
      tile_ready = true;
    }
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    for (int j = 0; j < gn; j++) {
      const float *s = myslot + j * SLOT;
      float wx0[CAO], wx1[CAO];
#pragma unroll
      for (int a = 0; a < CAO; a++) {
        if (NMESH == 2) {
          const float2 v = reinterpret_cast<const float2 *>(s)[a];
          wx0[a] = v.x;
          wx1[a] = v.y;
        } else {
          wx0[a] = wx1[a] = s[a];
        }
      }
      int org0, org1;
      if (NMESH == 2) {
        const int2 o2v = *reinterpret_cast<const int2 *>(s + OFF);
        org0 = o2v.x;
        org1 = o2v.y;
      } else {
        org0 = org1 = reinterpret_cast<const int *>(s)[OFF];
      }
      float ax = 0.0f, ay = 0.0f, az = 0.0f;
#pragma unroll
      for (int r = 0; r < NFULL; r++) {
        // rounds wholly on one mesh (known once the loop is unrolled) take
        // that mesh's x weights without a per-lane select
        const bool all0 = 32 * r + 31 < CAO * CAO, all1 = 32 * r >= CAO * CAO;
        const bool m1 = all1 || (!all0 && cii[r]);
        const float wbc = s[cwy[r]] * s[cwz[r]];
        const float4 *col = tile + (m1 ? org1 : org0) + coff[r];
#pragma unroll
        for (int a = 0; a < CAO; a++) {
          const float4 f = col[a * PL];
          const float w = wbc * (m1 ? wx1[a] : wx0[a]);
          ax = fmaf(f.x, w, ax);
          ay = fmaf(f.y, w, ay);
          az = fmaf(f.z, w, az);
        }
      }
#pragma unroll
      for (int r = 0; r < NPP; r++) {
        if (poff[r] >= 0) {
          const float w = s[pwy[r]] * s[pwz[r]] * s[pwx[r]];
          const float4 f = tile[(pii[r] ? org1 : org0) + poff[r]];
          ax = fmaf(f.x, w, ax);
          ay = fmaf(f.y, w, ay);
          az = fmaf(f.z, w, az);
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
      }
      if (lane == j) {
        fx = ax;
        fy = ay;
        fz = az;
      }
    }
    if (lane < gn) {
      fk[oidx] = fk0 + (double)fx;
      fk[(size_t)n + oidx] = fk1 + (double)fy;
      fk[2 * (size_t)n + oidx] = fk2 + (double)fz;
    }
  }
}

typedef CUresult (*encode_tiled_t)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda); nullptr when the driver does not provide it
encode_tiled_t encode_fn() {
  static encode_tiled_t fn = nullptr;
  static bool looked = false;
  if (!looked) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<encode_tiled_t>(p);
    else
      cudaGetLastError();
    looked = true;
  }
  return fn;
}

template <int CAO, int NMESH>
int launch_tile(Ctx *c, const void *Fv, double *fk, int na, double pref, bool tma) {
  const int B = c->brick, nb = c->nbrick1, m = c->mesh;
  const int T = gt_tile_edge(B, CAO, NMESH);
  const int TZ = gt_row_pitch(T, CAO);
  const size_t smem = gt_smem_bytes(B, CAO, NMESH);
  if (smem > 227 * 1024 || T > 16) return P3MG_ERR_ARG;
  static std::atomic<int> smem_set[P3MG_MAX_DEVICES];
  P3MG_CUDA_TRY(raise_smem_limit(gather_tile_kernel<CAO, NMESH>, (int)smem, smem_set));
  CUtensorMap tmap;
  memset(&tmap, 0, sizeof(tmap));
  int use_tma = 0;
  // TMA: a 16-byte aligned base (the strides are multiples of 16 bytes)
  if (tma && T <= m && (reinterpret_cast<uintptr_t>(Fv) & 15) == 0) {
    encode_tiled_t enc = encode_fn();
    if (enc) {
      const cuuint64_t dims[5] = {4, (cuuint64_t)m, (cuuint64_t)m, (cuuint64_t)m, (cuuint64_t)(NMESH * na)};
      const cuuint64_t strides[4] = {16, 16 * (cuuint64_t)m, 16 * (cuuint64_t)m * m, 16 * (cuuint64_t)c->M};
      const cuuint32_t box[5] = {4, (cuuint32_t)TZ, (cuuint32_t)T, (cuuint32_t)T, 1};
      const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
      if (enc(&tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, const_cast<void *>(Fv), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS)
        use_tma = 1;
    }
  }
  const double Hi = (double)m / c->L;
  const double shift = (double)((CAO - 1) / 2);
  const dim3 grid(nb * nb * nb, na);
  gather_tile_kernel<CAO, NMESH><<<grid, GT_THREADS, smem, c->stream>>>(
      tmap, use_tma, c->sorted_xyzq, c->sorted_idx, c->brick_start, m, B, nb, Hi, shift, pref,
      reinterpret_cast<const float4 *>(Fv), c->M, fk, c->n, c->dev_status);
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

}  // namespace

// FP32 ik gather through brick tiles (gather_mode 2: TMA-staged tiles where
// they lie inside the mesh, 3: plain loads for every tile).  Returns
// P3MG_ERR_ARG when the tile does not fit in shared memory.
int gather_tile_f32(Ctx *c, const void *Fv, double *fk, int na, double pref) {
  const bool il = method_interlaced(c->method);
  const bool tma = c->gather_mode == 2;
#define GT_CASE(K)                                                                          \
  case K:                                                                                   \
    return il ? launch_tile<K, 2>(c, Fv, fk, na, pref, tma) : launch_tile<K, 1>(c, Fv, fk, na, pref, tma);
  switch (c->cao) {
    GT_CASE(1)
    GT_CASE(2)
    GT_CASE(3)
    GT_CASE(4)
    GT_CASE(5)
    GT_CASE(6)
    GT_CASE(7)
  }
#undef GT_CASE
  return P3MG_ERR_CAO;
}

bool gather_tile_fits(const Ctx *c) {
  const int nmesh = method_interlaced(c->method) ? 2 : 1;
  return gt_smem_bytes(c->brick, c->cao, nmesh) <= 227 * 1024 && gt_tile_edge(c->brick, c->cao, nmesh) <= 16;
}

}  // namespace p3mg
