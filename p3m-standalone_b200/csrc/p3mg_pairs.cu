// Real-space erfc pair forces (the reference's Realteil, realpart.c:124-167):
// for every ordered pair i != j with minimum-image distance r <= rcut
//   f_i += q_i q_j (erfc(alpha r)/r + 2 alpha/sqrt(pi) exp(-alpha^2 r^2)) / r^2 * d
//   E   += 1/2 q_i q_j erfc(alpha r)/r
// The reference loops over all N^2 pairs; here particles are counting-sorted
// into a cell list of side >= rcut (nc = floor(L/rcut) >= 3 cells per side),
// which visits exactly the same pair set.  One CTA per cell: its particles
// are the i's (one per thread), the 27 neighbour cells are staged through
// shared memory and every thread reads them as broadcasts.
//
// FP64: absolute positions and the reference's minimum-image rounding
// (dx -= round(dx/L) L) with separately rounded products, so the r <= rcut
// decisions are the reference's.  FP32 (mixed): positions relative to the
// origin of their cell (exact in FP32 to ~1e-7 of a cell), neighbour image
// offsets added as integer multiples of the cell side; energy summed with
// compensated (Kahan) FP32 per thread and FP64 across threads.
// With fewer than 3 cells per side the all-pairs kernel runs instead.
#include <math.h>

#include "p3mg_internal.cuh"

namespace p3mg {

namespace {

constexpr int PAIR_THREADS = 64;
constexpr int BRUTE_THREADS = 256;

__global__ void bin_cells_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                 const double *__restrict__ z, int n, double L, int nc, int *__restrict__ key,
                                 int *__restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double s = (double)nc / L;
  int c0 = wrap_full((int)floor(x[i] * s), nc);
  int c1 = wrap_full((int)floor(y[i] * s), nc);
  int c2 = wrap_full((int)floor(z[i] * s), nc);
  const int k = (c0 * nc + c1) * nc + c2;
  key[i] = k;
  atomicAdd(&count[k], 1);
}

template <typename V>
__global__ void place_cells_kernel(const double *__restrict__ x, const double *__restrict__ y,
                                   const double *__restrict__ z, const double *__restrict__ q, int n, double L, int nc,
                                   const int *__restrict__ key, const int *__restrict__ start, int *__restrict__ fill,
                                   int *__restrict__ sidx, V *__restrict__ pos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = key[i];
  const int slot = start[k] + atomicAdd(&fill[k], 1);
  sidx[slot] = i;
  if (sizeof(V) == sizeof(double4)) {
    reinterpret_cast<double4 *>(pos)[slot] = make_double4(x[i], y[i], z[i], q[i]);
  } else {
    // position relative to the cell origin, folded into the box
    const double cs = L / nc;
    const int c2 = k % nc, c1 = (k / nc) % nc, c0 = k / (nc * nc);
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

__global__ void __launch_bounds__(PAIR_THREADS) pairs_fp64_kernel(const double4 *__restrict__ pos,
                                                                   const int *__restrict__ sidx,
                                                                   const int *__restrict__ start, int nc, double L,
                                                                   double rcut, double alpha, double *__restrict__ fr,
                                                                   int n, double *__restrict__ energy) {
  __shared__ double4 sj[PAIR_THREADS];
  __shared__ double ered[PAIR_THREADS / 32];
  const int cell = blockIdx.x;
  const int c2 = cell % nc, c1 = (cell / nc) % nc, c0 = cell / (nc * nc);
  const int i0 = start[cell], i1 = start[cell + 1];
  const double Li = 1.0 / L;
  const double wupi = 1.77245385090551602729816748334;
  const double pref = 2.0 * alpha / wupi;
  double e_loc = 0.0;
  for (int ib = i0; ib < i1; ib += PAIR_THREADS) {
    const int i = ib + threadIdx.x;
    const bool act = i < i1;
    double4 pi = act ? pos[i] : make_double4(0, 0, 0, 0);
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int nb = 0; nb < 27; nb++) {
      const int d0 = nb / 9 - 1, d1 = (nb / 3) % 3 - 1, d2 = nb % 3 - 1;
      const int nc0 = wrap_full(c0 + d0, nc), nc1 = wrap_full(c1 + d1, nc), nc2 = wrap_full(c2 + d2, nc);
      const int ncell = (nc0 * nc + nc1) * nc + nc2;
      const int j0 = start[ncell], j1 = start[ncell + 1];
      for (int jb = j0; jb < j1; jb += PAIR_THREADS) {
        __syncthreads();
        if (jb + threadIdx.x < j1) sj[threadIdx.x] = pos[jb + threadIdx.x];
        __syncthreads();
        const int cnt = min(PAIR_THREADS, j1 - jb);
        if (act) {
          for (int t = 0; t < cnt; t++) {
            if (jb + t == i) continue;
            const double4 pj = sj[t];
            const double dx = min_image(__dadd_rn(pi.x, -pj.x), Li, L);
            const double dy = min_image(__dadd_rn(pi.y, -pj.y), Li, L);
            const double dz = min_image(__dadd_rn(pi.z, -pj.z), Li, L);
            const double r2s = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            const double r = sqrt(r2s);
            if (r <= rcut) {
              const double ar = alpha * r;
              const double ec = erfc(ar);
              const double r2 = r * r;
              const double fak = pi.w * pj.w * (ec / r + pref * exp(-ar * ar)) / r2;
              fx += fak * dx;
              fy += fak * dy;
              fz += fak * dz;
              e_loc += 0.5 * pi.w * pj.w * ec / r;
            }
          }
        }
      }
    }
    if (act) {
      const int o = sidx[i];
      fr[o] += fx;
      fr[(size_t)n + o] += fy;
      fr[2 * (size_t)n + o] += fz;
    }
  }
  // energy: warp then block reduction, one atomic per CTA
  for (int o = 16; o > 0; o >>= 1) e_loc += __shfl_xor_sync(0xffffffffu, e_loc, o);
  if ((threadIdx.x & 31) == 0) ered[threadIdx.x >> 5] = e_loc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < PAIR_THREADS / 32; w++) s += ered[w];
    if (s != 0.0) atomicAdd(energy, s);
  }
}

__global__ void __launch_bounds__(PAIR_THREADS) pairs_fp32_kernel(const float4 *__restrict__ pos,
                                                                   const int *__restrict__ sidx,
                                                                   const int *__restrict__ start, int nc, float cs,
                                                                   float rcut, float alpha, double *__restrict__ fr,
                                                                   int n, double *__restrict__ energy) {
  __shared__ float4 sj[PAIR_THREADS];
  __shared__ double ered[PAIR_THREADS / 32];
  const int cell = blockIdx.x;
  const int c2 = cell % nc, c1 = (cell / nc) % nc, c0 = cell / (nc * nc);
  const int i0 = start[cell], i1 = start[cell + 1];
  const float pref = 2.0f * alpha / 1.7724538509055160273f;
  const float rc2 = rcut * rcut;
  float e_sum = 0.0f, e_comp = 0.0f;  // Kahan
  for (int ib = i0; ib < i1; ib += PAIR_THREADS) {
    const int i = ib + threadIdx.x;
    const bool act = i < i1;
    float4 pi = act ? pos[i] : make_float4(0, 0, 0, 0);
    float fx = 0.f, fy = 0.f, fz = 0.f;
    for (int nb = 0; nb < 27; nb++) {
      const int d0 = nb / 9 - 1, d1 = (nb / 3) % 3 - 1, d2 = nb % 3 - 1;
      const int nc0 = wrap_full(c0 + d0, nc), nc1 = wrap_full(c1 + d1, nc), nc2 = wrap_full(c2 + d2, nc);
      const int ncell = (nc0 * nc + nc1) * nc + nc2;
      const int j0 = start[ncell], j1 = start[ncell + 1];
      // i relative to the neighbour cell's origin: pi - d*cs
      const float ox = pi.x - d0 * cs, oy = pi.y - d1 * cs, oz = pi.z - d2 * cs;
      for (int jb = j0; jb < j1; jb += PAIR_THREADS) {
        __syncthreads();
        if (jb + threadIdx.x < j1) sj[threadIdx.x] = pos[jb + threadIdx.x];
        __syncthreads();
        const int cnt = min(PAIR_THREADS, j1 - jb);
        if (act) {
          for (int t = 0; t < cnt; t++) {
            const float4 pj = sj[t];
            const float dx = ox - pj.x, dy = oy - pj.y, dz = oz - pj.z;
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 <= rc2 && (jb + t) != i) {
              const float rinv = rsqrtf(r2);
              const float r = r2 * rinv;
              const float ar = alpha * r;
              const float ec = erfcf(ar);
              const float qq = pi.w * pj.w;
              const float fak = qq * (ec * rinv + pref * __expf(-ar * ar)) * (rinv * rinv);
              fx += fak * dx;
              fy += fak * dy;
              fz += fak * dz;
              const float term = 0.5f * qq * ec * rinv - e_comp;
              const float tsum = e_sum + term;
              e_comp = (tsum - e_sum) - term;
              e_sum = tsum;
            }
          }
        }
      }
    }
    if (act) {
      const int o = sidx[i];
      fr[o] += (double)fx;
      fr[(size_t)n + o] += (double)fy;
      fr[2 * (size_t)n + o] += (double)fz;
    }
  }
  double e_loc = (double)e_sum - (double)e_comp;
  for (int o = 16; o > 0; o >>= 1) e_loc += __shfl_xor_sync(0xffffffffu, e_loc, o);
  if ((threadIdx.x & 31) == 0) ered[threadIdx.x >> 5] = e_loc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < PAIR_THREADS / 32; w++) s += ered[w];
    if (s != 0.0) atomicAdd(energy, s);
  }
}

// All-pairs fallback (fewer than 3 cells per side): the reference's loop
// order for i, j tiles staged through shared memory.
__global__ void __launch_bounds__(BRUTE_THREADS) pairs_brute_kernel(const double *__restrict__ x,
                                                                     const double *__restrict__ y,
                                                                     const double *__restrict__ z,
                                                                     const double *__restrict__ q, int n, double L,
                                                                     double rcut, double alpha, double *__restrict__ fr,
                                                                     double *__restrict__ energy) {
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

static int cells_per_side(double L, double rcut) {
  int nc = (int)floor(L / rcut);
  return nc > 256 ? 256 : nc;
}

// Allocate the cell-list arrays for this rcut (host-side; called before a
// step is captured into a CUDA graph).
int pairs_reserve(Ctx *c, double rcut) {
  if (c->n == 0 || rcut <= 0.0) return P3MG_OK;
  const int nc = cells_per_side(c->L, rcut);
  if (nc < 3) return P3MG_OK;
  const int ncell = nc * nc * nc;
  if (ncell > c->ncell_cap) {
    if (c->cell_count) cudaFree(c->cell_count);
    if (c->cell_start) cudaFree(c->cell_start);
    if (c->cell_fill) cudaFree(c->cell_fill);
    c->cell_count = c->cell_start = c->cell_fill = nullptr;
    c->ncell_cap = 0;
    P3MG_CUDA_TRY(cudaMalloc(&c->cell_count, sizeof(int) * ncell));
    P3MG_CUDA_TRY(cudaMalloc(&c->cell_start, sizeof(int) * (ncell + 1)));
    P3MG_CUDA_TRY(cudaMalloc(&c->cell_fill, sizeof(int) * ncell));
    c->ncell_cap = ncell;
  }
  return P3MG_OK;
}

int pairs_run(Ctx *c, double rcut, double alpha) {
  const int n = c->n;
  if (n == 0 || rcut <= 0.0) return P3MG_OK;
  const int nc = cells_per_side(c->L, rcut);
  const int threads = 256;
  const int blocks = (n + threads - 1) / threads;
  if (nc < 3) {
    mark(c, EV_K0);
    pairs_brute_kernel<<<blocks, BRUTE_THREADS, 0, c->stream>>>(c->x, c->y, c->z, c->q, n, c->L, rcut, alpha, c->fr,
                                                                 c->energy);
    c->launches++;
    mark(c, EV_K1);
    P3MG_CUDA_TRY(cudaGetLastError());
    return P3MG_OK;
  }
  const int ncell = nc * nc * nc;
  P3MG_TRY(pairs_reserve(c, rcut));
  c->ncell1 = nc;
  P3MG_CUDA_TRY(cudaMemsetAsync(c->cell_count, 0, sizeof(int) * ncell, c->stream));
  P3MG_CUDA_TRY(cudaMemsetAsync(c->cell_fill, 0, sizeof(int) * ncell, c->stream));
  bin_cells_kernel<<<blocks, threads, 0, c->stream>>>(c->x, c->y, c->z, n, c->L, nc, c->cell_key, c->cell_count);
  c->launches++;
  P3MG_CUDA_TRY(cudaGetLastError());
  P3MG_TRY(exclusive_scan(c, c->cell_count, c->cell_start, ncell));
  if (c->precision == P3MG_FP64) {
    place_cells_kernel<double4><<<blocks, threads, 0, c->stream>>>(c->x, c->y, c->z, c->q, n, c->L, nc, c->cell_key,
                                                                   c->cell_start, c->cell_fill, c->cell_idx,
                                                                   reinterpret_cast<double4 *>(c->cell_pos));
    P3MG_CUDA_TRY(cudaGetLastError());
    mark(c, EV_K0);
    pairs_fp64_kernel<<<ncell, PAIR_THREADS, 0, c->stream>>>(reinterpret_cast<const double4 *>(c->cell_pos),
                                                             c->cell_idx, c->cell_start, nc, c->L, rcut, alpha, c->fr,
                                                             n, c->energy);
  } else {
    place_cells_kernel<float4><<<blocks, threads, 0, c->stream>>>(c->x, c->y, c->z, c->q, n, c->L, nc, c->cell_key,
                                                                  c->cell_start, c->cell_fill, c->cell_idx,
                                                                  reinterpret_cast<float4 *>(c->cell_pos));
    P3MG_CUDA_TRY(cudaGetLastError());
    mark(c, EV_K0);
    pairs_fp32_kernel<<<ncell, PAIR_THREADS, 0, c->stream>>>(reinterpret_cast<const float4 *>(c->cell_pos),
                                                             c->cell_idx, c->cell_start, nc, (float)(c->L / nc),
                                                             (float)rcut, (float)alpha, c->fr, n, c->energy);
  }
  c->launches += 2;
  mark(c, EV_K1);
  P3MG_CUDA_TRY(cudaGetLastError());
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
// are the same).  All calls on a device share the one array and it keeps
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
constexpr size_t NA_OFF_FILL = NA_OFF_START + na_round(NA_CELL_BYTES + sizeof(int));
constexpr size_t NA_OFF_KEY = NA_OFF_FILL + na_round(NA_CELL_BYTES);
constexpr size_t NA_OFF_IDX = NA_OFF_KEY + na_round(NA_PART_INT_BYTES);
constexpr size_t NA_OFF_POS = NA_OFF_IDX + na_round(NA_PART_INT_BYTES);
constexpr size_t NA_BYTES = NA_OFF_POS + na_round(sizeof(double4) * (size_t)P3MG_NOALLOC_MAX_PARTICLES);
static_assert(NA_BYTES <= (size_t)P3MG_NOALLOC_SCRATCH_BYTES, "no-alloc scratch layout exceeds its array");

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[P3MG_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int NA_MAX_DEVICES = 64;
unsigned char *g_na_ptr[NA_MAX_DEVICES] = {nullptr};

// Device address of the scratch array for the current device.  In host
// code the symbol name only stands for the array, it is not an address the
// GPU can use, so the address is looked up once per device (with that
// device current) and cached.
int noalloc_scratch(unsigned char **out) {
  int dev = 0;
  P3MG_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NA_MAX_DEVICES) return P3MG_ERR_ARG;
  if (!g_na_ptr[dev]) {
    void *p = nullptr;
    P3MG_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_na_ptr[dev] = (unsigned char *)p;
  }
  *out = g_na_ptr[dev];
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
    pairs_brute_kernel<<<blocks, BRUTE_THREADS, 0, s>>>(x, y, z, q, n, L, rcut, alpha, fr, energy);
    P3MG_CUDA_TRY(cudaGetLastError());
    return P3MG_OK;
  }
  while (nc > 3 && nc * nc * nc > P3MG_NOALLOC_MAX_CELLS) nc--;
  const int ncell = nc * nc * nc;
  int *count = (int *)(base + NA_OFF_COUNT);
  int *start = (int *)(base + NA_OFF_START);
  int *fill = (int *)(base + NA_OFF_FILL);
  int *key = (int *)(base + NA_OFF_KEY);
  int *idx = (int *)(base + NA_OFF_IDX);
  void *pos = (void *)(base + NA_OFF_POS);
  // the array keeps the previous call's counters: clear them first
  P3MG_CUDA_TRY(cudaMemsetAsync(count, 0, sizeof(int) * ncell, s));
  P3MG_CUDA_TRY(cudaMemsetAsync(fill, 0, sizeof(int) * ncell, s));
  bin_cells_kernel<<<blocks, threads, 0, s>>>(x, y, z, n, L, nc, key, count);
  P3MG_CUDA_TRY(cudaGetLastError());
  P3MG_TRY(scan_counts(count, start, ncell, s));
  if (precision == P3MG_FP64) {
    place_cells_kernel<double4><<<blocks, threads, 0, s>>>(x, y, z, q, n, L, nc, key, start, fill, idx,
                                                           reinterpret_cast<double4 *>(pos));
    P3MG_CUDA_TRY(cudaGetLastError());
    pairs_fp64_kernel<<<ncell, PAIR_THREADS, 0, s>>>(reinterpret_cast<const double4 *>(pos), idx, start, nc, L, rcut,
                                                     alpha, fr, n, energy);
  } else {
    place_cells_kernel<float4><<<blocks, threads, 0, s>>>(x, y, z, q, n, L, nc, key, start, fill, idx,
                                                          reinterpret_cast<float4 *>(pos));
    P3MG_CUDA_TRY(cudaGetLastError());
    pairs_fp32_kernel<<<ncell, PAIR_THREADS, 0, s>>>(reinterpret_cast<const float4 *>(pos), idx, start, nc,
                                                     (float)(L / nc), (float)rcut, (float)alpha, fr, n, energy);
  }
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}
