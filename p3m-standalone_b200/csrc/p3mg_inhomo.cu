// Inhomogeneous k-space error estimate and error map on the GPU (FP64).
//
// inhomo_error restates Generic_error_estimate_inhomo (p3m-common.c:437-719):
//   rho2(r)  = sum_i q_i^2 W(r - x_i) on the estimator's mesh
//              (assign_charge_q2, charge-assign.c:1544-1590), or the uniform
//              sum q^2 / mesh^3;
//   K_d(k)   = -2 pi i k_d / L (U2 G_opt - Ghat), the homogeneous kernel
//              (p3m-common.c:489-534) with G_opt = B/A of p3m-common.c:359-392
//              taken with no alias images, so U2 G_opt - Ghat vanishes up to
//              rounding;
//   K_d^a(k) for each alias vector a in [-mc, mc]^3 without 0
//              (p3m-common.c:558-625): -i (k_d/L) 2 pi U(k) U(-k - a m) G_opt(k)
//              times S_d(a) = sum_{k' != 0} (k'_d/L) 2 pi U(k') U(k' + a m) G_opt(k').
//              The reference adds the product term by term over k' for every
//              k (mesh^6 work per alias vector); the sum over k' factors out
//              and is formed once here by a reduction;
//   K2(r)    = sum_d Re(IDFT K_d)^2 + sum_a sum_d Re(IDFT K_d^a)^2;
//   E        = IDFT[DFT(rho2) * DFT(K2)], the product component by component
//              (re*re, im*im, p3m-common.c:664-672);
//   estimate = sqrt(sum_i q_i^2 sum_stencil W E / n)
//              (collect_rms_nocf, charge-assign.c:1650-1705).
// The reference's collection step takes its mesh spacing, stencil shift and
// stencil length from the force method's parameters while the window table
// has the estimator's order; collect_mesh / collect_cao carry those values
// here.  Table entries past the estimator's order (which the reference reads
// past its table rows, interpol.c:38-44) are 0, and indices wrap modulo the
// mesh (the reference wraps once, charge-assign.c:37-40, which is the same
// whenever collect_mesh < 2 mesh and collect_cao <= mesh).
//
// error_map restates Error_map (p3m-common.c:402-435): |fk_ref - fk|^2 of
// every particle assigned to a mesh with the window of the given order
// (assign_charge_nocf, charge-assign.c:1592-1648).
//
// All DFTs are the unnormalised FFTW conventions the reference plans:
// backward +i, forward -i.  Sums over particles and mesh points are
// deterministic (fixed-order block reductions).
#include <stdlib.h>

#include "p3mg_internal.cuh"

namespace p3mg {
namespace {

constexpr int kThreads = 256;
constexpr int kSumBlocks = 296;  // 2 per SM

__device__ inline double sinc_pi(double d) {
  const double a = P3MG_PI * d;
  return d == 0.0 ? 1.0 : sin(a) / a;
}

// (sinc(a/m) sinc(b/m) sinc(c/m))^e  (U, U2: p3m-common.c:351-357)
__device__ inline double window_hat(int a, int b, int c, int m, int e) {
  return pow(sinc_pi((double)a / m) * sinc_pi((double)b / m) * sinc_pi((double)c / m), (double)e);
}

__device__ inline int half_signed(int i, int m) { return (i >= m / 2) ? i - m : i; }

__device__ inline void mesh_point(size_t t, int m, int tn[3]) {
  const int k = (int)(t % m);
  const size_t r = t / m;
  const int j = (int)(r % m);
  const int i = (int)(r / m);
  tn[0] = half_signed(i, m);
  tn[1] = half_signed(j, m);
  tn[2] = half_signed(k, m);
}

// B-spline weights of order cao at tabulated bin arg, zero past the order.
__device__ inline void weights_any(int cao, int arg, double *w) {
#pragma unroll
  for (int j = 0; j < P3MG_MAX_CAO; j++) w[j] = 0.0;
  switch (cao) {
    case 1: bspline_weights<double, 1, false>(arg, w, nullptr); break;
    case 2: bspline_weights<double, 2, false>(arg, w, nullptr); break;
    case 3: bspline_weights<double, 3, false>(arg, w, nullptr); break;
    case 4: bspline_weights<double, 4, false>(arg, w, nullptr); break;
    case 5: bspline_weights<double, 5, false>(arg, w, nullptr); break;
    case 6: bspline_weights<double, 6, false>(arg, w, nullptr); break;
    default: bspline_weights<double, 7, false>(arg, w, nullptr); break;
  }
}

struct Stencil {
  int base[3];
  double w[3][P3MG_MAX_CAO];
};

// Geometry (mesh spacing L/mesh_h, shift) with indices wrapped onto a mesh
// of m points, weights of order tab_cao.
__device__ inline void make_stencil(double x, double y, double z, double Hi, double shift, int m, int tab_cao,
                                    Stencil &s) {
  const double c[3] = {x, y, z};
#pragma unroll
  for (int d = 0; d < 3; d++) {
    int arg;
    mesh_geometry(c[d], Hi, shift, 0, m, &s.base[d], &arg);
    weights_any(tab_cao, arg, s.w[d]);
  }
}

// value * W assigned to a real-part mesh of m^3 complex points (stride 2
// doubles) or a plain real mesh (stride 1).
__device__ inline void assign(const Stencil &s, int count, int m, double value, double *mesh, int stride) {
  for (int a = 0; a < count; a++) {
    const int I = (s.base[0] + a) % m;
    const double t0 = value * s.w[0][a];
    for (int b = 0; b < count; b++) {
      const int J = (s.base[1] + b) % m;
      const double t1 = t0 * s.w[1][b];
      const size_t row = ((size_t)I * m + J) * m;
      for (int c = 0; c < count; c++) {
        const int K = (s.base[2] + c) % m;
        atomicAdd(mesh + stride * (row + K), t1 * s.w[2][c]);
      }
    }
  }
}

__global__ void rho2_kernel(const double *x, const double *y, const double *z, const double *q, int n, double Hi,
                            double shift, int m, int cao, double2 *R) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Stencil s;
  make_stencil(x[i], y[i], z[i], Hi, shift, m, cao, s);
  assign(s, cao, m, q[i] * q[i], reinterpret_cast<double *>(R), 2);
}

__global__ void uniform_kernel(const double *q2sum, size_t M, double2 *R) {
  const double v = q2sum[0] / (double)M;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < M; t += (size_t)gridDim.x * blockDim.x)
    R[t] = make_double2(v, 0.0);
}

// Block partial sums of v[i] (SQUARE: v[i]^2) over a grid-stride range,
// tree-reduced in a fixed order.
template <bool SQUARE>
__global__ void partial_sum_kernel(const double *v, size_t n, double *partial) {
  __shared__ double sh[kThreads];
  double acc = 0.0;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
    acc += SQUARE ? v[t] * v[t] : v[t];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// out[j] = sum_b partial[j * nb + b] in order, one thread per output.
__global__ void final_sum_kernel(const double *partial, int nb, int nout, double *out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nout) return;
  double s = 0.0;
  for (int b = 0; b < nb; b++) s += partial[(size_t)j * nb + b];
  out[j] = s;
}

// Homogeneous kernel K_d(k) (imaginary parts; the k = 0 bin is 0), and per
// bin G_opt (no alias images) and U for the alias terms.
__global__ void homo_kernel(int m, int cao, double L, double alpha, double2 *K, double *gopt, double *uw) {
  const size_t M = (size_t)m * m * m;
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= M) return;
  int tn[3];
  mesh_point(t, m, tn);
  uw[t] = window_hat(tn[0], tn[1], tn[2], m, cao);
  double kv[3] = {0.0, 0.0, 0.0};
  double g = 0.0;
  if (tn[0] != 0 || tn[1] != 0 || tn[2] != 0) {
    const double w = 2.0 * P3MG_PI / L;
    const double k2 = (w * w) * ((double)tn[0] * tn[0] + (double)tn[1] * tn[1] + (double)tn[2] * tn[2]);
    const double ghat = (4 * P3MG_PI / k2) * exp(-k2 / (4 * alpha * alpha));
    const double u2 = window_hat(tn[0], tn[1], tn[2], m, 2 * cao);
    g = (u2 * ghat * k2) / (u2 * (k2 * u2));
    const double v = u2 * g - ghat;
#pragma unroll
    for (int d = 0; d < 3; d++) kv[d] = -2 * P3MG_PI * tn[d] / L * v;
  }
  gopt[t] = g;
#pragma unroll
  for (int d = 0; d < 3; d++) K[d * M + t] = make_double2(0.0, kv[d]);
}

// Alias vector number ia (reference loop order mx, my, mz; 0 skipped).
__device__ inline void alias_vector(int ia, int mc, int a[3]) {
  const int w = 2 * mc + 1;
  const int center = (w * w * w - 1) / 2;
  const int u = ia < center ? ia : ia + 1;
  a[0] = u / (w * w) - mc;
  a[1] = (u / w) % w - mc;
  a[2] = u % w - mc;
}

// Block partials of S_d(a) = sum_{k != 0} (k_d/L) 2 pi U(k) U(k + a m) G_opt(k)
// for the alias vector blockIdx.y.
__global__ void alias_sum_kernel(int m, int cao, int mc, double L, const double *gopt, const double *uw,
                                 double *partial) {
  __shared__ double sh[3][kThreads];
  const size_t M = (size_t)m * m * m;
  int a[3];
  alias_vector(blockIdx.y, mc, a);
  double acc[3] = {0.0, 0.0, 0.0};
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < M; t += (size_t)gridDim.x * blockDim.x) {
    int tn[3];
    mesh_point(t, m, tn);
    if (tn[0] == 0 && tn[1] == 0 && tn[2] == 0) continue;
    const double k1 = 2 * P3MG_PI * uw[t] * window_hat(tn[0] + a[0] * m, tn[1] + a[1] * m, tn[2] + a[2] * m, m, cao) *
                      gopt[t];
#pragma unroll
    for (int d = 0; d < 3; d++) acc[d] += (tn[d] / L) * k1;
  }
#pragma unroll
  for (int d = 0; d < 3; d++) sh[d][threadIdx.x] = acc[d];
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
#pragma unroll
      for (int d = 0; d < 3; d++) sh[d][threadIdx.x] += sh[d][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int d = 0; d < 3; d++) partial[((size_t)blockIdx.y * 3 + d) * gridDim.x + blockIdx.x] = sh[d][0];
}

// K_d^a(k) for the alias vectors ia0 + blockIdx.y (3 meshes each).
__global__ void alias_kernel(int m, int cao, int mc, double L, int ia0, const double *gopt, const double *uw,
                             const double *S, double2 *K) {
  const size_t M = (size_t)m * m * m;
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= M) return;
  const int ia = ia0 + blockIdx.y;
  int a[3], tn[3];
  alias_vector(ia, mc, a);
  mesh_point(t, m, tn);
  double kv[3] = {0.0, 0.0, 0.0};
  if (tn[0] != 0 || tn[1] != 0 || tn[2] != 0) {
    const double k2 = 2 * P3MG_PI * uw[t] *
                      window_hat(-tn[0] - a[0] * m, -tn[1] - a[1] * m, -tn[2] - a[2] * m, m, cao) * gopt[t];
#pragma unroll
    for (int d = 0; d < 3; d++) kv[d] = -(tn[d] / L) * k2 * S[ia * 3 + d];
  }
  double2 *Kb = K + (size_t)blockIdx.y * 3 * M;
#pragma unroll
  for (int d = 0; d < 3; d++) Kb[d * M + t] = make_double2(0.0, kv[d]);
}

// K2(r) (+)= sum over nb kernel triples of sum_d Re(K_d)^2, in order.
__global__ void ksq_kernel(const double2 *K, int nb, size_t M, int accumulate, double2 *K2) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= M) return;
  double acc = accumulate ? K2[t].x : 0.0;
  for (int b = 0; b < nb; b++) {
    const double2 *Kb = K + (size_t)b * 3 * M;
    double kr = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) kr += Kb[d * M + t].x * Kb[d * M + t].x;
    acc = (!accumulate && b == 0) ? kr : acc + kr;
  }
  K2[t] = make_double2(acc, 0.0);
}

__global__ void product_kernel(const double2 *K2, double2 *E, size_t M) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= M) return;
  const double2 k = K2[t];
  double2 e = E[t];
  e.x *= k.x;
  e.y *= k.y;
  E[t] = e;
}

__global__ void collect_kernel(const double *x, const double *y, const double *z, const double *q, int n, double Hi,
                               double shift, int m, int tab_cao, int count, const double2 *E, double *rms) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Stencil s;
  make_stencil(x[i], y[i], z[i], Hi, shift, m, tab_cao, s);
  const double q2 = q[i] * q[i];
  double r = 0.0;
  for (int a = 0; a < count; a++) {
    const int I = (s.base[0] + a) % m;
    const double t0 = q2 * s.w[0][a];
    for (int b = 0; b < count; b++) {
      const int J = (s.base[1] + b) % m;
      const double t1 = t0 * s.w[1][b];
      const size_t row = ((size_t)I * m + J) * m;
      for (int c = 0; c < count; c++) r += E[row + (s.base[2] + c) % m].x * (t1 * s.w[2][c]);
    }
  }
  rms[i] = r;
}

__global__ void error_map_kernel(const double *x, const double *y, const double *z, const double *F, int n,
                                 double Hi, double shift, int m, int cao, double *map, double *dF) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // F: fk x, y, z blocks, then the reference forces' x, y, z blocks
  double v = 0.0;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double e = F[(size_t)(3 + d) * n + i] - F[(size_t)d * n + i];
    v += e * e;
  }
  dF[i] = v;
  Stencil s;
  make_stencil(x[i], y[i], z[i], Hi, shift, m, cao, s);
  assign(s, cao, m, v, map, 1);
}

unsigned blocks_for(size_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// Deterministic sum of v[0..n) (SQUARE: of squares) into d_out[0].
template <bool SQUARE>
void device_sum(const double *v, size_t n, double *partial, double *d_out, cudaStream_t st, long long *launches) {
  partial_sum_kernel<SQUARE><<<kSumBlocks, kThreads, 0, st>>>(v, n, partial);
  final_sum_kernel<<<1, 32, 0, st>>>(partial, kSumBlocks, 1, d_out);
  *launches += 2;
}

// Device / host allocations released on scope exit.
struct DevBuf {
  void *p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};
struct HostBuf {
  double *p = nullptr;
  ~HostBuf() { free(p); }
};

// Frees the estimator's FFT plan and adds the kernels launched to the
// context's count on every exit.
struct PlanGuard {
  Ctx *sc;
  Ctx *c;
  long long launches = 0;
  ~PlanGuard() {
    c->launches += launches + sc->launches;
    fft_plan_free(sc);
  }
};

}  // namespace

int inhomo_error(Ctx *c, double alpha, int uniform, int mesh, int cao, int mc, int collect_mesh, int collect_cao,
                 double *estimate, double *mesh_out) {
  if (!estimate || collect_mesh < 1 || mc < 0 || mc > P3MG_MAX_INHOMO_MC || !(alpha > 0.0)) return P3MG_ERR_ARG;
  if (cao < 1 || cao > P3MG_MAX_CAO || collect_cao < 1 || collect_cao > P3MG_MAX_CAO) return P3MG_ERR_CAO;
  {
    int radix[24], np;
    if (mesh < 4 || mesh > P3MG_MAX_MESH || fft_factor(mesh, radix, &np)) return P3MG_ERR_MESH;
  }
  if (!(c->L > 0.0)) return P3MG_ERR_NOSYS;
  cudaSetDevice(c->device);
  // FFT plan of the estimator's mesh, on the context's stream
  Ctx sc;
  sc.mesh = mesh;
  sc.M = (size_t)mesh * mesh * mesh;
  sc.precision = P3MG_FP64;
  sc.device = c->device;
  sc.stream = c->stream;
  PlanGuard guard{&sc, c};
  P3MG_TRY(fft_plan_init(&sc));

  const size_t M = sc.M;
  const int w = 2 * mc + 1;
  const int na = w * w * w - 1;  // alias vectors
  // alias vectors per batched pass: at most 1 GiB of kernel meshes
  const size_t per_alias = 3 * M * sizeof(double2);
  int nb = (int)(((size_t)1 << 30) / per_alias);
  if (nb < 1) nb = 1;
  if (nb > na) nb = na;
  const int nk = na > 0 ? nb : 1;  // kernel triples held (the homogeneous part needs 1)
  const int n = c->n;
  const unsigned sum_rows = 3u * (unsigned)(na > 0 ? na : 1);
  // one allocation (doubles): R, E, K2 (complex, adjacent), gopt, uw,
  // K (3 nk complex), S (3 na), partial sums, rms (n), scalars
  const size_t off_R = 0, off_E = off_R + 2 * M, off_K2 = off_E + 2 * M, off_g = off_K2 + 2 * M, off_u = off_g + M;
  const size_t off_K = off_u + M, off_S = off_K + 6 * M * (size_t)nk;
  const size_t off_P = off_S + sum_rows;
  const size_t off_rms = off_P + (size_t)kSumBlocks * sum_rows, off_sc = off_rms + (size_t)(n > 0 ? n : 1);
  DevBuf buf;
  P3MG_CUDA_TRY(cudaMalloc(&buf.p, (off_sc + 2) * sizeof(double)));
  double *base = (double *)buf.p;
  double2 *R = (double2 *)(base + off_R), *E = (double2 *)(base + off_E), *K2 = (double2 *)(base + off_K2);
  double2 *K = (double2 *)(base + off_K);
  double *gopt = base + off_g, *uw = base + off_u, *S = base + off_S, *partial = base + off_P;
  double *rms = base + off_rms, *scal = base + off_sc;
  cudaStream_t st = c->stream;
  long long &launches = guard.launches;
  const unsigned gM = blocks_for(M);
  const unsigned gN = blocks_for((size_t)(n > 0 ? n : 1));

  // rho^2 on the estimator's mesh
  P3MG_CUDA_TRY(cudaMemsetAsync(R, 0, M * sizeof(double2), st));
  if (!uniform) {
    if (n > 0) {
      rho2_kernel<<<gN, kThreads, 0, st>>>(c->x, c->y, c->z, c->q, n, (double)mesh / c->L, (double)((cao - 1) / 2),
                                          mesh, cao, R);
      launches++;
    }
  } else {
    device_sum<true>(c->q, (size_t)n, partial, scal, st, &launches);
    uniform_kernel<<<kSumBlocks, kThreads, 0, st>>>(scal, M, R);
    launches++;
  }

  // homogeneous kernel -> K2(r)
  homo_kernel<<<gM, kThreads, 0, st>>>(mesh, cao, c->L, alpha, K, gopt, uw);
  launches++;
  P3MG_TRY(fft3d(&sc, K, 3, +1));
  ksq_kernel<<<gM, kThreads, 0, st>>>(K, 1, M, 0, K2);
  launches++;

  // alias terms, nb alias vectors per pass
  if (na > 0) {
    alias_sum_kernel<<<dim3(kSumBlocks, na), kThreads, 0, st>>>(mesh, cao, mc, c->L, gopt, uw, partial);
    final_sum_kernel<<<(sum_rows + 127) / 128, 128, 0, st>>>(partial, kSumBlocks, (int)sum_rows, S);
    launches += 2;
    for (int ia0 = 0; ia0 < na; ia0 += nb) {
      const int cnt = (na - ia0) < nb ? (na - ia0) : nb;
      alias_kernel<<<dim3(gM, cnt), kThreads, 0, st>>>(mesh, cao, mc, c->L, ia0, gopt, uw, S, K);
      launches++;
      P3MG_TRY(fft3d(&sc, K, 3 * cnt, +1));
      ksq_kernel<<<gM, kThreads, 0, st>>>(K, cnt, M, 1, K2);
      launches++;
    }
  }

  // E = IDFT[DFT(rho2) * DFT(K2)]; E and K2 are adjacent, one batched forward FFT
  P3MG_CUDA_TRY(cudaMemcpyAsync(E, R, M * sizeof(double2), cudaMemcpyDeviceToDevice, st));
  P3MG_TRY(fft3d(&sc, E, 2, -1));
  product_kernel<<<gM, kThreads, 0, st>>>(K2, E, M);
  launches++;
  P3MG_TRY(fft3d(&sc, E, 1, +1));

  // collect at the particles
  if (n > 0) {
    collect_kernel<<<gN, kThreads, 0, st>>>(c->x, c->y, c->z, c->q, n, (double)collect_mesh / c->L,
                                            (double)((collect_cao - 1) / 2), mesh, cao, collect_cao, E, rms);
    launches++;
    device_sum<false>(rms, (size_t)n, partial, scal + 1, st, &launches);
  } else {
    P3MG_CUDA_TRY(cudaMemsetAsync(scal + 1, 0, sizeof(double), st));
  }
  P3MG_CUDA_TRY(cudaGetLastError());
  double sum = 0.0;
  P3MG_CUDA_TRY(cudaMemcpyAsync(&sum, scal + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
  HostBuf host;
  if (mesh_out) {
    host.p = (double *)malloc(6 * M * sizeof(double));  // R, E, K2
    if (!host.p) return P3MG_ERR_ALLOC;
    P3MG_CUDA_TRY(cudaMemcpyAsync(host.p, base + off_R, 6 * M * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  P3MG_CUDA_TRY(cudaStreamSynchronize(st));
  *estimate = sqrt(sum / n);
  if (mesh_out) {
    const double *hR = host.p, *hE = host.p + 2 * M, *hK = host.p + 4 * M;
    for (size_t t = 0; t < M; t++) {
      mesh_out[5 * t + 0] = hR[2 * t];
      mesh_out[5 * t + 1] = hE[2 * t];
      mesh_out[5 * t + 2] = hE[2 * t + 1];
      mesh_out[5 * t + 3] = hK[2 * t];
      mesh_out[5 * t + 4] = hK[2 * t + 1];
    }
  }
  return P3MG_OK;
}

int error_map(Ctx *c, int mesh, int cao, const double *fk[3], const double *ref[3], double *map, double totals[2]) {
  if (!map) return P3MG_ERR_ARG;
  for (int d = 0; d < 3; d++)
    if (c->n > 0 && (!fk[d] || !ref[d])) return P3MG_ERR_ARG;
  if (cao < 1 || cao > P3MG_MAX_CAO) return P3MG_ERR_CAO;
  if (mesh < 1 || mesh > P3MG_MAX_MESH) return P3MG_ERR_MESH;
  if (!(c->L > 0.0)) return P3MG_ERR_NOSYS;
  cudaSetDevice(c->device);
  const int n = c->n;
  const size_t M = (size_t)mesh * mesh * mesh;
  const size_t nn = (size_t)(n > 0 ? n : 1);
  // layout (doubles): map (M), forces (6 n), dF (n), partial sums, 2 totals
  const size_t off_F = M, off_dF = off_F + 6 * nn, off_P = off_dF + nn, off_T = off_P + kSumBlocks;
  DevBuf buf;
  P3MG_CUDA_TRY(cudaMalloc(&buf.p, (off_T + 2) * sizeof(double)));
  double *base = (double *)buf.p;
  cudaStream_t st = c->stream;
  long long launches = 0;
  P3MG_CUDA_TRY(cudaMemsetAsync(base, 0, M * sizeof(double), st));
  P3MG_CUDA_TRY(cudaMemsetAsync(base + off_T, 0, 2 * sizeof(double), st));
  if (n > 0) {
    for (int d = 0; d < 3; d++) {
      P3MG_CUDA_TRY(cudaMemcpyAsync(base + off_F + (size_t)d * n, fk[d], n * sizeof(double), cudaMemcpyHostToDevice, st));
      P3MG_CUDA_TRY(
          cudaMemcpyAsync(base + off_F + (size_t)(3 + d) * n, ref[d], n * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    error_map_kernel<<<blocks_for((size_t)n), kThreads, 0, st>>>(c->x, c->y, c->z, base + off_F, n,
                                                                 (double)mesh / c->L, (double)((cao - 1) / 2), mesh,
                                                                 cao, base, base + off_dF);
    launches++;
    device_sum<false>(base + off_dF, (size_t)n, base + off_P, base + off_T, st, &launches);
  }
  device_sum<false>(base, M, base + off_P, base + off_T + 1, st, &launches);
  P3MG_CUDA_TRY(cudaMemcpyAsync(map, base, M * sizeof(double), cudaMemcpyDeviceToHost, st));
  double tot[2];
  P3MG_CUDA_TRY(cudaMemcpyAsync(tot, base + off_T, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  P3MG_CUDA_TRY(cudaStreamSynchronize(st));
  P3MG_CUDA_TRY(cudaGetLastError());
  if (totals) {
    totals[0] = tot[0];
    totals[1] = tot[1];
  }
  c->launches += launches;
  return P3MG_OK;
}

}  // namespace p3mg
