// Internal declarations of the p3mg library: context, device helpers and
// the kernel launchers shared by the translation units.  sm_100a only.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <atomic>

#include "../../include/p3mg.h"

#define P3MG_PI 3.14159265358979323846264338327950288
#define P3MG_MAX_MESH 512
#define P3MG_MAX_CAO 7
// largest alias range of the inhomogeneous error estimate ((2 mc + 1)^3 - 1 alias vectors)
#define P3MG_MAX_INHOMO_MC 10
// tabulated in-cell offset resolution of the reference: 2*MaxInterpol
// = 131072 bins per mesh spacing (interpol.h:149, charge-assign.c:156)
#define P3MG_NINTERP 131072

namespace p3mg {

// ------------------------------------------------------------ error handling
void record_cuda_error(cudaError_t e);

#define P3MG_CUDA_TRY(expr)                       \
  do {                                            \
    cudaError_t e_ = (expr);                      \
    if (e_ != cudaSuccess) {                      \
      ::p3mg::record_cuda_error(e_);              \
      return (e_ == cudaErrorMemoryAllocation) ? P3MG_ERR_ALLOC : P3MG_ERR_CUDA; \
    }                                             \
  } while (0)

#define P3MG_TRY(expr)      \
  do {                      \
    int s_ = (expr);        \
    if (s_ != P3MG_OK) return s_; \
  } while (0)

// Dynamic shared-memory limit of a kernel, raised to at least `bytes` once
// per device: the attribute belongs to each device's copy of the kernel, so a
// process that drives several GPUs sets it on each.  `cache` (one slot per
// device, zero-initialised static storage) holds the value set; host threads
// racing here set the same value, and the atomic slots keep that defined.
constexpr int P3MG_MAX_DEVICES = 64;
template <typename T>
inline cudaError_t raise_smem_limit(T *kernel, int bytes, std::atomic<int> *cache) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < P3MG_MAX_DEVICES && cache[dev].load(std::memory_order_relaxed) >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && dev >= 0 && dev < P3MG_MAX_DEVICES) cache[dev].store(bytes, std::memory_order_relaxed);
  return e;
}

// ------------------------------------------------------------ method traits
__host__ __device__ inline bool method_interlaced(int m) { return m == 1 || m == 3; }
__host__ __device__ inline bool method_ad(int m) { return m == 2 || m == 3 || m == 7; }
__host__ __device__ inline bool method_self_force(int m) { return m == 2 || m == 7; }

template <typename real>
struct cplx;
template <>
struct cplx<double> {
  typedef double2 type;
  typedef double4 vec4;
};
template <>
struct cplx<float> {
  typedef float2 type;
  typedef float4 vec4;
};

// ------------------------------------------------------------ FFT plan
struct FftPlan {
  int m = 0;
  int npass = 0;
  int radix[24];
  void *tw = nullptr;  // m complex entries exp(-2 pi i e / m), real type of the context
};

// ------------------------------------------------------------ context
struct Ctx {
  int method = 0, mesh = 0, cao = 0, mc = 1, precision = P3MG_FP64;
  int device = 0;
  cudaStream_t stream = nullptr;
  // second stream of a step: the real-space pairs run on it beside the
  // k-space chain (fork / join events on the context stream)
  cudaStream_t stream2 = nullptr;
  bool overlap = true;  // the pairs on stream2 beside the k-space chain (p3mg_set_overlap)
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;

  // particles
  int n = 0, cap = 0;
  double L = 0.0;
  double *x = nullptr, *y = nullptr, *z = nullptr, *q = nullptr;  // inputs (device)
  double *f = nullptr, *fk = nullptr, *fr = nullptr;              // outputs, 3n each (device)
  double *energy = nullptr;                                        // device: [0] pair energy, [1] compensation
  // device status word: kernels with bounded waits set bit 0 when a wait
  // gave up (read and cleared by the host-synchronising entry points)
  int *dev_status = nullptr;

  // scatter lane table (int2 per lane and iteration, built on the first step)
  void *scatter_tab = nullptr;

  // k-space binning by mesh brick (particles sorted by the brick of their stencil base)
  int brick = 8;
  int fft_w = 0;    // FFT: 0 automatic (pencil kernels where they apply), 4/8/16 Stockham tile width
  // ik gather: 0 lanes on the stencil's z offsets, 1 one thread per
  // particle, 2 FP32 brick tiles in shared memory staged by TMA (plain loads
  // where a tile wraps around the mesh), 3 the same tiles with plain loads
  // only (set by p3mg_create)
  int gather_mode = 0;
  int nbrick1 = 0;  // bricks per dimension
  // particle counts / starts per sort key: brick, then mesh point in the
  // brick (B^3 keys per brick); the range of brick b is
  // brick_start[b B^3] .. brick_start[(b + 1) B^3]
  int *brick_count = nullptr, *brick_start = nullptr;
  int2 *part_key = nullptr;    // sort key per particle (input order) and its rank among that key's particles
  int *sorted_idx = nullptr;   // input index of each sorted particle
  double4 *sorted_xyzq = nullptr;

  // pair cell list
  int ncell1 = 0, ncell_cap = 0;
  double cell_rcut = -1.0;
  int *cell_count = nullptr, *cell_start = nullptr;
  int2 *cell_key = nullptr;  // half-cell key per particle and its rank in that half-cell
  int *cell_idx = nullptr;
  void *cell_pos = nullptr;  // double4 (FP64) or float4 (FP32: position relative to the cell origin, q)
  void *pair_units = nullptr;  // FP32 dense-cell work units (int2) + 2 counters
  size_t pair_units_cap = 0;

  // mesh data (real type = double for FP64, float for FP32_MIXED)
  size_t M = 0;               // mesh^3
  void *Q = nullptr;          // complex mesh
  void *F = nullptr;          // 3 complex meshes (ik methods)
  void *P = nullptr;          // ik: packed fields per mesh point (Fx, Fy, Fz, 0), unshifted then shifted mesh
  double *G = nullptr;        // FP64 influence function (full mesh)
  float *G32 = nullptr;       // FP32 copy for the mixed path
  double *self_b = nullptr;   // 81 self-force coefficients (device)
  double self_b_host[81];
  FftPlan plan;

  double alpha = 0.0;
  double *d_alpha = nullptr;  // device: [0] alpha of G (read by the step's kernels), [1] scratch
  double h_alpha_arg = 0.0;   // host source of the [1] upload
  bool have_G = false;

  // timing: CUDA events on the context stream (see EV_* below)
  bool timing = false;
  cudaEvent_t ev[12];
  bool ev_ok = false;
  double stage_ms[4] = {0, 0, 0, 0};   // t_c, t_g, t_f, t_r
  double kernel_ms[3] = {0, 0, 0};     // pair kernel, scatter kernel, gather kernel
  bool stage_pending = false;

  // kernels launched by this context (host-side count)
  long long launches = 0;

  // CUDA graph of one p3mg_compute step (replayed when the same rcut/n repeat)
  bool use_graph = false;
  cudaGraphExec_t gexec = nullptr;
  double graph_rcut = -1.0;
  int graph_n = -1;
  long long graph_launches = 0;  // kernels per replay

  // scratch of the tiled scan: two slots of scan_cap ints, the second for
  // scans enqueued on stream2
  int *scan_tmp = nullptr;
  int scan_cap = 0;           // ints per slot
  void *sweep_ws = nullptr;  // workspace of p3mg_sweep, kept between calls
  int sweep_nodes = 0;       // last p3mg_sweep: interpolation nodes used (0: every alpha evaluated)
  void *interp_ws = nullptr;  // buffers of the interpolated sweep, kept between calls
  size_t interp_cap = 0;
  double sweep_check = -1.0; // its check: RMS(interpolated - evaluated) / RMS(evaluated), -1: none
  // energy / adjoint buffers (allocated on first use): G and dG/dalpha at
  // alpha, the potential mesh, 8 reduction slots, the gradients (3 n + n)
  double *adj_G = nullptr, *adj_dG = nullptr, *adj_sums = nullptr, *adj_grad = nullptr;
  // alpha and box length adj_G / adj_dG were computed for (-1: none yet)
  double adj_key_alpha = -1.0, adj_key_L = -1.0;
  double *sweep_rms2 = nullptr;  // the last sweep's squared errors per alpha (device, in its workspace)
  // per-axis alias tables of G_opt (influence_tables), kept between calls
  double *infl_tab = nullptr;
  size_t infl_cap = 0;
  double *self_R = nullptr;  // per-axis factors of the ad self-force sums
  void *adj_phi = nullptr;
  int adj_cap = 0;
  size_t sweep_cap = 0;
};

// event slots: stage markers and kernel brackets
enum {
  EV_S0 = 0,   // step start
  EV_S1 = 1,   // after real space (on the stream the pairs ran on)
  EV_S2 = 2,   // after binning + charge assignment
  EV_S3 = 3,   // after FFTs + convolution
  EV_S4 = 4,   // after back-interpolation + self-force
  EV_K0 = 5,   // pair kernel start / end
  EV_K1 = 6,
  EV_K2 = 7,   // scatter kernel start / end
  EV_K3 = 8,
  EV_K4 = 9,   // gather kernel start / end
  EV_K5 = 10,
  EV_S1K = 11,  // start of the k-space chain (after the pairs, or beside them on stream2)
};

inline void mark(Ctx *c, int slot) {
  if (c->timing && c->ev_ok) cudaEventRecord(c->ev[slot], c->stream);
}

int alloc_system(Ctx *c, int n);
int free_all(Ctx *c);

// ------------------------------------------------------------ launchers
// FFT (p3mg_fft.cu)
int fft_plan_init(Ctx *c);
void fft_plan_free(Ctx *c);
int fft3d(Ctx *c, void *data, int nbatch, int sign);
// real-input transforms (methods 6, 7; even meshes whose half is 2/3/5/7-smooth):
// padded real layout (row pitch m + 2 reals) <-> half spectrum
// m x m x (m/2 + 1), in place, nbatch meshes at a slot stride of M complex
bool fft_real_ok(const Ctx *c);
int fft3d_real(Ctx *c, void *data, int nbatch, int sign);
// methods 6 and 7 run the real-input transforms (r2c / c2r) where the mesh allows
inline bool kspace_real(const Ctx *c) { return (c->method == 6 || c->method == 7) && fft_real_ok(c); }
// register-tiled pencil passes (p3mg_fft_pencil.cu): FP32, m = 32, 64, 128
bool fft_pencil_ok(const Ctx *c);
int fft_pencil(Ctx *c, void *data, int nbatch, int sign);
// ik convolution of Q^ with the G of na alphas (FP32, na M), the backward
// FFTs of their field meshes (F: 3 na M complex work space) and the packing
// for the gather (P: NMESH na M float4), the convolution fused into the
// first pass and the packing into the last
int fft_pencil_init();
int ik_conv_inverse_pencil(Ctx *c, const void *Qh, const float *G32, double s, void *F, int na, void *P);
int fft_factor(int m, int *radix, int *npass);  // 0 when m factors into 2, 3, 4, 5, 7

// inhomogeneous error estimate and error map (p3mg_inhomo.cu)
int inhomo_error(Ctx *c, double alpha, int uniform, int mesh, int cao, int mc, int collect_mesh, int collect_cao,
                 double *estimate, double *mesh_out);
int error_map(Ctx *c, int mesh, int cao, const double *fk[3], const double *ref[3], double *map, double totals[2]);

// influence (p3mg_influence.cu)
int influence_compute(Ctx *c, double alpha);

// FP32 ik back-interpolation through shared-memory brick tiles
// (p3mg_gather_tile.cu; gather_mode 2 and 3)
bool gather_tile_fits(const Ctx *c);
int gather_tile_f32(Ctx *c, const void *Fv, double *fk, int na, double pref);

// charge assignment / back-interpolation (p3mg_assign.cu)
int kspace_prepare(Ctx *c);
int kspace_run(Ctx *c);  // scatter, FFTs, convolution, gather, self-force into c->fk / c->f

// analytic error estimates (p3mg_influence.cu): est = total, k space, real space
int error_estimates(int method, int m, int cao, int n, double L, double q2, double alpha, double rcut, int mc_est,
                    cudaStream_t stream, long long *launches, double est[3]);

// FP64 Ewald reference (p3mg_ewald.cu)
int ewald_parameters(int n, double q2, double L, int mesh_param, double *alpha, int *kmax);
int ewald_forces(Ctx *c, int nt, const int *d_tgt, double alpha, int kmax, bool shell, double rcut_real,
                 double *d_out, double *d_fk);
double ewald_error(int n, double q2, double L, double rcut, int kmax, double alpha);

// real space (p3mg_pairs.cu)
int pairs_reserve(Ctx *c, double rcut);
int pairs_run(Ctx *c, double rcut, const double *alphas, int nalpha, double *fr, double *energy);
int pairs_bin(Ctx *c, double rcut, int *nc_out);
int pairs_adjoint(Ctx *c, double rcut, int nc, double ge, double *gx, double *gq, double *sums);
int influence_with_derivative(Ctx *c, double *G_out, double *dG_out);
int adjoint(Ctx *c, double rcut, double ge, double *gx, double *gq, double energy[5], double *dalpha, double *dL);

// Buffers of a batched k-space pass over na alphas (all on the device):
// G (na meshes, FP64 or FP32 by precision), b81 (81 self-force
// coefficients per alpha), mesh scratch for the na field meshes (ik: 3 na
// complex meshes in F, na x (1 or 2) packed meshes in P; ad: na complex
// meshes in F), and the outputs fk (gather) and f (self forces), 3 n per
// alpha, both accumulated.
struct KspaceBatch {
  int na = 0;
  const void *G = nullptr;
  const double *b81 = nullptr;
  void *F = nullptr;
  void *P = nullptr;
  double *fk = nullptr;
  double *f = nullptr;
  bool forward = true;  // run the scatter and forward FFT into Q first
};
int kspace_batch(Ctx *c, const KspaceBatch &b);
// the energy's adjoint on the brick-sorted particles (kspace_prepare first):
// exact-weight charge assignment into the complex mesh Q, and the gradient
// gather from the potential meshes Phi (see adj_gather_sorted_kernel)
int adjoint_scatter(Ctx *c);
int adjoint_gather(Ctx *c, const void *Phi, double s, double ge, double *gx, double *gq);
int influence_batch(Ctx *c, const double *d_alphas, int na, double *G_all, double *S26, double *b81_all);
int g_to_f32_n(Ctx *c, const double *G, float *G32, size_t count);
size_t sweep_bytes_per_alpha(const Ctx *c);
// ref: host reference rows x, y, z (n doubles each), or NULL
int sweep_run(Ctx *c, double rcut, int na, const double *alphas, const double *const *ref, double *rms_out,
              double *f_out, size_t budget, bool exact);
int sweep_grid_run(Ctx *const *cs, int nctx, double rcut, int na, const double *alphas, const double *const *ref,
                   double *rms_out, size_t budget);

// misc kernels (p3mg_api.cu)
int zero_forces(Ctx *c);
int combine_forces(Ctx *c);

// FP32 copy of the FP64 influence function (mixed precision)
int g_to_f32(Ctx *c);

// single-CTA exclusive scan of counts[0..nb) into start[0..nb] (start[nb] = total)
int exclusive_scan(Ctx *c, const int *counts, int *start, int nb);
int scan_tmp_reserve(Ctx *c, int nb);
int scan_counts(const int *counts, int *start, int nb, cudaStream_t stream);

// ------------------------------------------------------------ device helpers

__host__ __device__ inline int wrap_full(int i, int m) {
  int r = i % m;
  return r < 0 ? r + m : r;
}

// Mesh geometry of one coordinate, with the reference's rounding
// (charge-assign.c:148-157): pos = x*Hi - shift (+ 0.5 for the shifted mesh),
// nmp = floor(pos + 0.5), arg = floor((pos - nmp + 0.5) * 131072).
// __dmul_rn/__dadd_rn keep each operation separately rounded (no FMA),
// so the tabulated bin `arg` is the one the reference selects.
__device__ inline void mesh_geometry(double xc, double Hi, double shift, int ii, int m, int *base, int *arg) {
  double pos = __dadd_rn(__dmul_rn(xc, Hi), -shift);
  if (ii) pos = __dadd_rn(pos, 0.5);
  double nf = floor(__dadd_rn(pos, 0.5));
  int nmp = (int)nf;
  double frac = __dadd_rn(__dadd_rn(pos, -nf), 0.5);
  int a = (int)floor(__dmul_rn(frac, (double)P3MG_NINTERP));
  a = a < 0 ? 0 : (a > P3MG_NINTERP - 1 ? P3MG_NINTERP - 1 : a);
  *base = wrap_full(nmp, m);
  *arg = a;
}

// mesh_geometry plus the exact in-cell offset u = frac in [0, 1) of the
// same rounded position (so the stencil base always agrees with the
// binning's).
__device__ inline void mesh_geometry_u(double xc, double Hi, double shift, int ii, int m, int *base, int *arg,
                                       double *u) {
  double pos = __dadd_rn(__dmul_rn(xc, Hi), -shift);
  if (ii) pos = __dadd_rn(pos, 0.5);
  double nf = floor(__dadd_rn(pos, 0.5));
  int nmp = (int)nf;
  double frac = __dadd_rn(__dadd_rn(pos, -nf), 0.5);
  int a = (int)floor(__dmul_rn(frac, (double)P3MG_NINTERP));
  a = a < 0 ? 0 : (a > P3MG_NINTERP - 1 ? P3MG_NINTERP - 1 : a);
  *base = wrap_full(nmp, m);
  *arg = a;
  *u = frac;
}

// Cardinal B-spline weights of order CAO at the tabulated offset of bin
// `arg` (x = (arg - 65536)/131072 in [-0.5, 0.5)):  w[j] = M_CAO(u + CAO-1-j),
// u = x + 1/2, with the recursion M_n(u) = [u M_{n-1}(u) + (n-u) M_{n-1}(u-1)]/(n-1)
// (de Boor; Essmann et al. 1995) and dw[j] = M_{CAO-1}(u+k) - M_{CAO-1}(u+k-1),
// k = CAO-1-j.  These are the charge-assignment polynomials of
// window-functions.c:46-183.
// The same weights at an arbitrary offset u = x + 1/2 in [0, 1) (used
// where the weights must be smooth functions of the position).
template <typename real, int CAO, bool DERIV>
__device__ __forceinline__ void bspline_weights_u(real u, real *w, real *dw) {
  real a[CAO];
  real prev[CAO];
  a[0] = (real)1;
#pragma unroll
  for (int k = 1; k < CAO; k++) a[k] = (real)0;
#pragma unroll
  for (int n = 2; n <= CAO; n++) {
#pragma unroll
    for (int k = 0; k < CAO; k++) prev[k] = a[k];
    const real inv = (real)1 / (real)(n - 1);
#pragma unroll
    for (int k = 0; k < CAO; k++) {
      if (k < n) {
        real lo = (k < n - 1) ? prev[k] : (real)0;
        real hi = (k > 0) ? prev[k - 1] : (real)0;
        a[k] = ((u + (real)k) * lo + ((real)n - u - (real)k) * hi) * inv;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < CAO; j++) {
    const int k = CAO - 1 - j;
    w[j] = a[k];
    if (DERIV) {
      if (CAO == 1)
        dw[j] = (real)0;
      else
        dw[j] = prev[k] - (k > 0 ? prev[k - 1] : (real)0);
    }
  }
}

template <typename real, int CAO, bool DERIV>
__device__ __forceinline__ void bspline_weights(int arg, real *w, real *dw) {
  const real u = (real)(arg - P3MG_NINTERP / 2) * (real)(1.0 / P3MG_NINTERP) + (real)0.5;
  bspline_weights_u<real, CAO, DERIV>(u, w, dw);
}

// Stencil base and exact in-cell offset u in [0, 1) of a coordinate (the
// geometry of mesh_geometry without the 2^-17 quantisation of the offset).
__device__ inline void mesh_geometry_exact(double xc, double Hi, double shift, int ii, int m, int *base, double *u) {
  double pos = xc * Hi - shift;
  if (ii) pos += 0.5;
  const double nf = floor(pos + 0.5);
  *u = pos - nf + 0.5;
  *base = wrap_full((int)nf, m);
}

}  // namespace p3mg
