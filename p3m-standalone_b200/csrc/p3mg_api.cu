// C ABI of the p3mg library (declared in include/p3mg.h): context
// lifecycle, host/device particle I/O and the step orchestration that
// mirrors Calculate_forces (common.c:268-327).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <new>

#include <vector>

#include "p3mg_internal.cuh"

namespace p3mg {

static char g_last_cuda_error[256] = "";

void record_cuda_error(cudaError_t e) {
  snprintf(g_last_cuda_error, sizeof(g_last_cuda_error), "%s: %s", cudaGetErrorName(e), cudaGetErrorString(e));
}

int fft_factor(int m, int *radix, int *npass);

namespace {

__global__ void combine_kernel(double *__restrict__ f, const double *__restrict__ fk, const double *__restrict__ fr,
                               size_t n3) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n3) f[t] += fk[t] + fr[t];
}

template <typename T>
void dfree(T *&p) {
  if (p) cudaFree((void *)p);
  p = nullptr;
}

}  // namespace

int zero_forces(Ctx *c) {
  const size_t b = 3 * (size_t)c->n * sizeof(double);
  P3MG_CUDA_TRY(cudaMemsetAsync(c->f, 0, b, c->stream));
  P3MG_CUDA_TRY(cudaMemsetAsync(c->fk, 0, b, c->stream));
  P3MG_CUDA_TRY(cudaMemsetAsync(c->fr, 0, b, c->stream));
  P3MG_CUDA_TRY(cudaMemsetAsync(c->energy, 0, 2 * sizeof(double), c->stream));
  return P3MG_OK;
}

int combine_forces(Ctx *c) {
  const size_t n3 = 3 * (size_t)c->n;
  if (n3 == 0) return P3MG_OK;
  combine_kernel<<<(unsigned)((n3 + 255) / 256), 256, 0, c->stream>>>(c->f, c->fk, c->fr, n3);
  c->launches++;
  P3MG_CUDA_TRY(cudaGetLastError());
  return P3MG_OK;
}

int alloc_system(Ctx *c, int n) {
  if (n <= c->cap && c->x) {
    c->n = n;
    return P3MG_OK;
  }
  dfree(c->x);
  dfree(c->y);
  dfree(c->z);
  dfree(c->q);
  dfree(c->f);
  dfree(c->fk);
  dfree(c->fr);
  dfree(c->part_key);
  dfree(c->sorted_idx);
  dfree(c->sorted_xyzq);
  dfree(c->cell_key);
  dfree(c->cell_idx);
  dfree(c->cell_pos);
  const size_t cap = (size_t)(n > 0 ? n : 1);
  P3MG_CUDA_TRY(cudaMalloc(&c->x, cap * sizeof(double)));
  P3MG_CUDA_TRY(cudaMalloc(&c->y, cap * sizeof(double)));
  P3MG_CUDA_TRY(cudaMalloc(&c->z, cap * sizeof(double)));
  P3MG_CUDA_TRY(cudaMalloc(&c->q, cap * sizeof(double)));
  P3MG_CUDA_TRY(cudaMalloc(&c->f, 3 * cap * sizeof(double)));
  P3MG_CUDA_TRY(cudaMalloc(&c->fk, 3 * cap * sizeof(double)));
  P3MG_CUDA_TRY(cudaMalloc(&c->fr, 3 * cap * sizeof(double)));
  P3MG_CUDA_TRY(cudaMalloc(&c->part_key, cap * sizeof(int2)));
  P3MG_CUDA_TRY(cudaMalloc(&c->sorted_idx, cap * sizeof(int)));
  P3MG_CUDA_TRY(cudaMalloc(&c->sorted_xyzq, cap * sizeof(double4)));
  P3MG_CUDA_TRY(cudaMalloc(&c->cell_key, cap * sizeof(int2)));
  P3MG_CUDA_TRY(cudaMalloc(&c->cell_idx, cap * sizeof(int)));
  P3MG_CUDA_TRY(cudaMalloc(&c->cell_pos, cap * sizeof(double4)));
  c->cap = (int)cap;
  c->n = n;
  return P3MG_OK;
}

int free_all(Ctx *c) {
  dfree(c->x);
  dfree(c->y);
  dfree(c->z);
  dfree(c->q);
  dfree(c->f);
  dfree(c->fk);
  dfree(c->fr);
  dfree(c->energy);
  dfree(c->dev_status);
  dfree(c->d_alpha);
  dfree(c->brick_count);
  dfree(c->brick_start);
  dfree(c->part_key);
  dfree(c->sorted_idx);
  dfree(c->sorted_xyzq);
  dfree(c->cell_count);
  dfree(c->cell_start);
  dfree(c->cell_key);
  dfree(c->cell_idx);
  dfree(c->cell_pos);
  dfree(c->pair_units);
  c->pair_units_cap = 0;
  dfree(c->Q);
  dfree(c->F);
  dfree(c->P);
  dfree(c->G);
  dfree(c->G32);
  dfree(c->self_b);
  dfree(c->scan_tmp);
  dfree(c->scatter_tab);
  if (c->sweep_ws) cudaFree(c->sweep_ws);
  c->sweep_ws = nullptr;
  c->sweep_cap = 0;
  if (c->interp_ws) cudaFree(c->interp_ws);
  c->interp_ws = nullptr;
  c->interp_cap = 0;
  dfree(c->adj_G);
  dfree(c->adj_dG);
  dfree(c->adj_sums);
  dfree(c->adj_grad);
  dfree(c->adj_phi);
  c->adj_cap = 0;
  dfree(c->infl_tab);
  c->infl_cap = 0;
  dfree(c->self_R);
  fft_plan_free(c);
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  c->gexec = nullptr;
  if (c->ev_ok)
    for (int i = 0; i < 12; i++) cudaEventDestroy(c->ev[i]);
  c->ev_ok = false;
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  c->ev_fork = c->ev_join = nullptr;
  if (c->stream2) cudaStreamDestroy(c->stream2);
  c->stream2 = nullptr;
  if (c->stream) cudaStreamDestroy(c->stream);
  c->stream = nullptr;
  return P3MG_OK;
}

// Enqueue one force evaluation on the context stream (Calculate_forces,
// common.c:268-327): zero, real space (rcut != 0, common.c:290-294),
// k-space with self-force, f += f_k + f_r.
// The real-space pairs (instruction-issue bound) and the k-space chain
// (shared-memory atomics, L1 and HBM bound) touch disjoint buffers, so the
// pairs run on stream2 beside the k-space chain: forked after the forces
// are zeroed, joined before they are combined.  Stage and kernel events
// follow the stream their work runs on (t_r from the step start to the
// pairs' end on stream2, t_c from the k-space start on the context stream).
static int enqueue_pairs_on_stream2(Ctx *c, double rcut) {
  P3MG_CUDA_TRY(cudaEventRecord(c->ev_fork, c->stream));
  P3MG_CUDA_TRY(cudaStreamWaitEvent(c->stream2, c->ev_fork, 0));
  cudaStream_t main_stream = c->stream;
  c->stream = c->stream2;
  const int st = pairs_run(c, rcut, c->d_alpha, 1, c->fr, c->energy);
  mark(c, EV_S1);
  c->stream = main_stream;
  // join even after an error, so no work is left outside the context stream
  P3MG_CUDA_TRY(cudaEventRecord(c->ev_join, c->stream2));
  return st;
}

static int enqueue_step(Ctx *c, double rcut) {
  P3MG_TRY(zero_forces(c));
  const bool timed = c->timing && c->ev_ok && c->n > 0;
  if (timed) {
    // brackets of stages that may not run this step must still be recorded
    for (int s = EV_K0; s <= EV_K5; s++) cudaEventRecord(c->ev[s], c->stream);
  }
  const bool overlap = rcut != 0.0 && c->n > 0 && c->stream2 && c->overlap;
  mark(c, EV_S0);
  int st = P3MG_OK;
  if (overlap) {
    st = enqueue_pairs_on_stream2(c, rcut);
  } else {
    if (rcut != 0.0) st = pairs_run(c, rcut, c->d_alpha, 1, c->fr, c->energy);
    mark(c, EV_S1);
  }
  mark(c, EV_S1K);
  if (st == P3MG_OK && c->n > 0) {
    st = kspace_prepare(c);
    if (st == P3MG_OK) st = kspace_run(c);
  }
  if (overlap) P3MG_CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
  P3MG_TRY(st);
  P3MG_TRY(combine_forces(c));
  c->stage_pending = timed;
  return P3MG_OK;
}

static void collect_stage_times(Ctx *c) {
  if (!c->stage_pending) return;
  cudaEventSynchronize(c->ev[EV_S4]);
  cudaEventSynchronize(c->ev[EV_S1]);
  float t;
  const int st[4][2] = {{EV_S1K, EV_S2}, {EV_S2, EV_S3}, {EV_S3, EV_S4}, {EV_S0, EV_S1}};
  for (int i = 0; i < 4; i++)
    if (cudaEventElapsedTime(&t, c->ev[st[i][0]], c->ev[st[i][1]]) == cudaSuccess) c->stage_ms[i] = t;
  const int kt[3][2] = {{EV_K0, EV_K1}, {EV_K2, EV_K3}, {EV_K4, EV_K5}};
  for (int i = 0; i < 3; i++)
    if (cudaEventElapsedTime(&t, c->ev[kt[i][0]], c->ev[kt[i][1]]) == cudaSuccess) c->kernel_ms[i] = t;
  c->stage_pending = false;
}

static void drop_graph(Ctx *c) {
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  c->gexec = nullptr;
  c->graph_rcut = -1.0;
  c->graph_n = -1;
}

// One step: eager, or replay of a captured CUDA graph when graphs are on.
// The first step for a given (n, rcut) runs eagerly (allocations, function
// attributes), the second captures and replays, later ones replay.
static int step_device(Ctx *c, double rcut) {
  if (!c->use_graph || c->timing) return enqueue_step(c, rcut);
  if (c->gexec && c->graph_rcut == rcut && c->graph_n == c->n) {
    P3MG_CUDA_TRY(cudaGraphLaunch(c->gexec, c->stream));
    c->launches += c->graph_launches;
    return P3MG_OK;
  }
  if (c->graph_rcut != rcut || c->graph_n != c->n) {
    // eager warm-up for this shape; capture on the next call
    drop_graph(c);
    P3MG_TRY(pairs_reserve(c, rcut));
    c->graph_rcut = rcut;
    c->graph_n = c->n;
    return enqueue_step(c, rcut);
  }
  cudaGraph_t g = nullptr;
  P3MG_CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  const long long before = c->launches;
  int st = enqueue_step(c, rcut);
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (st != P3MG_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess) {
    record_cuda_error(e);
    return P3MG_ERR_CUDA;
  }
  c->graph_launches = c->launches - before;
  c->launches = before;
  e = cudaGraphInstantiate(&c->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    c->gexec = nullptr;
    record_cuda_error(e);
    return P3MG_ERR_CUDA;
  }
  P3MG_CUDA_TRY(cudaGraphLaunch(c->gexec, c->stream));
  c->launches += c->graph_launches;
  return P3MG_OK;
}

}  // namespace p3mg

using namespace p3mg;

struct p3mg_ctx {
  Ctx c;
};

extern "C" {

const char *p3mg_strerror(int s) {
  switch (s) {
    case P3MG_OK: return "ok";
    case P3MG_ERR_ARG: return "invalid argument";
    case P3MG_ERR_METHOD: return "unknown method id (supported: 0, 1, 2, 3, 6, 7)";
    case P3MG_ERR_CAO: return "charge assignment order must be 1..7";
    case P3MG_ERR_MESH: return "unsupported mesh size (need max(cao,4) <= mesh <= 512, prime factors 2,3,5,7, even for methods 6/7)";
    case P3MG_ERR_NOSYS: return "no particles set";
    case P3MG_ERR_CUDA: return "CUDA runtime error";
    case P3MG_ERR_ALLOC: return "device memory allocation failed";
    case P3MG_ERR_STATE: return "influence function not computed (call p3mg_influence first)";
    case P3MG_ERR_PRECISION: return "unknown precision mode";
    case P3MG_ERR_NOBUF: return "buffer capacity exceeded";
  }
  return "unknown status";
}

const char *p3mg_last_cuda_error(void) { return g_last_cuda_error; }

int p3mg_create(p3mg_ctx **out, int method_id, int mesh, int cao, int mc, int precision) {
  if (!out) return P3MG_ERR_ARG;
  *out = nullptr;
  if (!(method_id == 0 || method_id == 1 || method_id == 2 || method_id == 3 || method_id == 6 || method_id == 7))
    return P3MG_ERR_METHOD;
  if (cao < 1 || cao > P3MG_MAX_CAO) return P3MG_ERR_CAO;
  if (precision != P3MG_FP64 && precision != P3MG_FP32_MIXED) return P3MG_ERR_PRECISION;
  if (mc < 0) return P3MG_ERR_ARG;
  int rad[24], np;
  if (mesh < 4 || mesh < cao || mesh > P3MG_MAX_MESH || fft_factor(mesh, rad, &np) != 0) return P3MG_ERR_MESH;
  if ((method_id == 6 || method_id == 7) && (mesh % 2)) return P3MG_ERR_MESH;
  p3mg_ctx *h = new (std::nothrow) p3mg_ctx();
  if (!h) return P3MG_ERR_ALLOC;
  Ctx *c = &h->c;
  c->method = method_id;
  c->mesh = mesh;
  c->cao = cao;
  c->mc = mc;
  c->precision = precision;
  // ik gather: lanes on the stencil's z offsets for the 32-byte FP64 field
  // vectors, TMA-staged brick tiles in shared memory for the 16-byte FP32
  // ones (each the fastest at the 1M-particle headline on a B200; a tile
  // that does not fit falls back to one thread per particle)
  c->gather_mode = (precision == P3MG_FP64) ? 0 : 2;
  c->M = (size_t)mesh * mesh * mesh;
  int st = P3MG_OK;
  do {
    cudaError_t e = cudaGetDevice(&c->device);
    if (e != cudaSuccess) {
      record_cuda_error(e);
      st = P3MG_ERR_CUDA;
      break;
    }
    // equal priorities: with the k-space stream ahead, its gather and the
    // pair kernel share SMs and both slow down (they lean on the same L1 /
    // shared-memory pipe), which measured slower than letting them follow
    // the launch order
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      record_cuda_error(e);
      st = P3MG_ERR_CUDA;
      break;
    }
    const size_t csz = (precision == P3MG_FP64) ? sizeof(double2) : sizeof(float2);
    // brick edge for the tiled charge assignment
    c->brick = (mesh >= 64) ? 8 : 4;
    c->nbrick1 = (mesh + c->brick - 1) / c->brick;
    // sort keys: bricks x mesh points per brick
    const int nbr = c->nbrick1 * c->nbrick1 * c->nbrick1 * c->brick * c->brick * c->brick;
#define ALLOC(ptr, bytes)                              \
  e = cudaMalloc((void **)&(ptr), (bytes));            \
  if (e != cudaSuccess) {                              \
    record_cuda_error(e);                              \
    st = P3MG_ERR_ALLOC;                               \
    break;                                             \
  }
    ALLOC(c->Q, c->M * csz);
    if (!method_ad(method_id)) {
      ALLOC(c->F, 3 * c->M * csz);
      ALLOC(c->P, (method_interlaced(method_id) ? 2 : 1) * c->M * 2 * csz);
    }
    ALLOC(c->G, c->M * sizeof(double));
    if (precision != P3MG_FP64) {
      ALLOC(c->G32, c->M * sizeof(float));
    }
    ALLOC(c->self_b, 81 * sizeof(double));
    ALLOC(c->energy, 2 * sizeof(double));
    ALLOC(c->dev_status, sizeof(int));
    ALLOC(c->d_alpha, 2 * sizeof(double));
    ALLOC(c->brick_count, nbr * sizeof(int));
    ALLOC(c->brick_start, (nbr + 1) * sizeof(int));
#undef ALLOC
    st = scan_tmp_reserve(c, nbr);
    if (st != P3MG_OK) break;
    cudaMemset(c->self_b, 0, 81 * sizeof(double));
    cudaMemset(c->dev_status, 0, sizeof(int));
    memset(c->self_b_host, 0, sizeof(c->self_b_host));
    st = fft_plan_init(c);
    if (st != P3MG_OK) break;
    c->ev_ok = true;
    for (int i = 0; i < 12; i++)
      if (cudaEventCreate(&c->ev[i]) != cudaSuccess) c->ev_ok = false;
  } while (0);
  if (st != P3MG_OK) {
    free_all(c);
    delete h;
    return st;
  }
  *out = h;
  return P3MG_OK;
}

void p3mg_destroy(p3mg_ctx *h) {
  if (!h) return;
  cudaSetDevice(h->c.device);
  if (h->c.stream) cudaStreamSynchronize(h->c.stream);
  free_all(&h->c);
  delete h;
}

static int set_system_common(Ctx *c, int n, const double *x, const double *y, const double *z, const double *q,
                             double L, cudaMemcpyKind kind) {
  if (n < 0 || !(L > 0.0) || !isfinite(L)) return P3MG_ERR_ARG;
  if (n > 0 && (!x || !y || !z || !q)) return P3MG_ERR_ARG;
  cudaSetDevice(c->device);
  // a captured step holds the old buffers, sizes and box (cell counts,
  // mesh spacing are kernel arguments)
  const bool same_shape = (n == c->n) && c->x != nullptr && L == c->L;
  if (!same_shape) drop_graph(c);
  P3MG_TRY(alloc_system(c, n));
  if (L != c->L) c->have_G = false;  // G_opt and the self-force depend on L
  c->L = L;
  const size_t b = (size_t)n * sizeof(double);
  if (n > 0) {
    P3MG_CUDA_TRY(cudaMemcpyAsync(c->x, x, b, kind, c->stream));
    P3MG_CUDA_TRY(cudaMemcpyAsync(c->y, y, b, kind, c->stream));
    P3MG_CUDA_TRY(cudaMemcpyAsync(c->z, z, b, kind, c->stream));
    P3MG_CUDA_TRY(cudaMemcpyAsync(c->q, q, b, kind, c->stream));
  }
  return P3MG_OK;
}

int p3mg_set_system(p3mg_ctx *h, int n, const double *x, const double *y, const double *z, const double *q, double L) {
  if (!h) return P3MG_ERR_ARG;
  return set_system_common(&h->c, n, x, y, z, q, L, cudaMemcpyHostToDevice);
}

int p3mg_set_system_device(p3mg_ctx *h, int n, const double *x, const double *y, const double *z, const double *q,
                           double L) {
  if (!h) return P3MG_ERR_ARG;
  return set_system_common(&h->c, n, x, y, z, q, L, cudaMemcpyDeviceToDevice);
}

int p3mg_influence(p3mg_ctx *h, double alpha) {
  if (!h) return P3MG_ERR_ARG;
  Ctx *c = &h->c;
  if (!(c->L > 0.0)) return P3MG_ERR_NOSYS;
  if (!isfinite(alpha) || alpha < 0.0) return P3MG_ERR_ARG;
  cudaSetDevice(c->device);
  return influence_compute(c, alpha);
}

// Device status word of the context's kernels (set when a bounded wait
// gave up); read after the stream has been synchronised, then cleared.
static int check_device_status(Ctx *c) {
  int st = 0;
  P3MG_CUDA_TRY(cudaMemcpyAsync(&st, c->dev_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  P3MG_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (st == 0) return P3MG_OK;
  P3MG_CUDA_TRY(cudaMemsetAsync(c->dev_status, 0, sizeof(int), c->stream));
  snprintf(g_last_cuda_error, sizeof(g_last_cuda_error), "a kernel's bounded wait gave up (device status %d)", st);
  return P3MG_ERR_CUDA;
}

static int copy_out3(Ctx *c, const double *src, double *hx, double *hy, double *hz, bool accumulate) {
  const size_t n = (size_t)c->n;
  if (n == 0) return P3MG_OK;
  double *dst[3] = {hx, hy, hz};
  if (!accumulate) {
    for (int d = 0; d < 3; d++)
      if (dst[d]) P3MG_CUDA_TRY(cudaMemcpyAsync(dst[d], src + d * n, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    P3MG_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return P3MG_OK;
  }
  double *tmp = (double *)malloc(3 * n * sizeof(double));
  if (!tmp) return P3MG_ERR_ALLOC;
  cudaError_t e = cudaMemcpyAsync(tmp, src, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    free(tmp);
    record_cuda_error(e);
    return P3MG_ERR_CUDA;
  }
  for (int d = 0; d < 3; d++)
    if (dst[d])
      for (size_t i = 0; i < n; i++) dst[d][i] += tmp[d * n + i];
  free(tmp);
  return P3MG_OK;
}

int p3mg_kspace_forces(p3mg_ctx *h, double *fk_x, double *fk_y, double *fk_z, double *ft_x, double *ft_y,
                       double *ft_z) {
  if (!h) return P3MG_ERR_ARG;
  Ctx *c = &h->c;
  if (c->n > 0 && (!fk_x || !fk_y || !fk_z)) return P3MG_ERR_ARG;
  if (!c->have_G) return P3MG_ERR_STATE;
  cudaSetDevice(c->device);
  P3MG_TRY(zero_forces(c));
  if (c->n > 0) {
    P3MG_TRY(kspace_prepare(c));
    P3MG_TRY(kspace_run(c));
  }
  collect_stage_times(c);
  P3MG_TRY(copy_out3(c, c->fk, fk_x, fk_y, fk_z, true));
  if (method_self_force(c->method) && (ft_x || ft_y || ft_z)) P3MG_TRY(copy_out3(c, c->f, ft_x, ft_y, ft_z, true));
  return check_device_status(c);
}

int p3mg_real_forces(p3mg_ctx *h, double rcut, double alpha, double *fr_x, double *fr_y, double *fr_z,
                     double *energy) {
  if (!h) return P3MG_ERR_ARG;
  Ctx *c = &h->c;
  if (c->n > 0 && (!fr_x || !fr_y || !fr_z)) return P3MG_ERR_ARG;
  if (!(c->L > 0.0)) return P3MG_ERR_NOSYS;
  if (!(rcut >= 0.0) || !(alpha >= 0.0)) return P3MG_ERR_ARG;
  cudaSetDevice(c->device);
  P3MG_TRY(zero_forces(c));
  c->h_alpha_arg = alpha;
  P3MG_CUDA_TRY(cudaMemcpyAsync(c->d_alpha + 1, &c->h_alpha_arg, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  P3MG_TRY(pairs_run(c, rcut, c->d_alpha + 1, 1, c->fr, c->energy));
  P3MG_TRY(copy_out3(c, c->fr, fr_x, fr_y, fr_z, true));
  if (energy) {
    double e;
    P3MG_CUDA_TRY(cudaMemcpy(&e, c->energy, sizeof(double), cudaMemcpyDeviceToHost));
    *energy += e;
  }
  return P3MG_OK;
}

int p3mg_compute(p3mg_ctx *h, double rcut) {
  if (!h) return P3MG_ERR_ARG;
  Ctx *c = &h->c;
  if (!(c->L > 0.0)) return P3MG_ERR_NOSYS;
  if (!c->have_G) return P3MG_ERR_STATE;
  if (!(rcut >= 0.0)) return P3MG_ERR_ARG;
  cudaSetDevice(c->device);
  return step_device(c, rcut);
}

int p3mg_get_forces(p3mg_ctx *h, double *f_x, double *f_y, double *f_z, double *fk_x, double *fk_y, double *fk_z,
                    double *fr_x, double *fr_y, double *fr_z, double *energy) {
  if (!h) return P3MG_ERR_ARG;
  Ctx *c = &h->c;
  cudaSetDevice(c->device);
  collect_stage_times(c);
  P3MG_TRY(copy_out3(c, c->f, f_x, f_y, f_z, false));
  P3MG_TRY(copy_out3(c, c->fk, fk_x, fk_y, fk_z, false));
  P3MG_TRY(copy_out3(c, c->fr, fr_x, fr_y, fr_z, false));
  if (energy) P3MG_CUDA_TRY(cudaMemcpy(energy, c->energy, sizeof(double), cudaMemcpyDeviceToHost));
  return check_device_status(c);
}

int p3mg_calculate_forces(p3mg_ctx *h, double rcut, double *f_x, double *f_y, double *f_z, double *fk_x, double *fk_y,
                          double *fk_z, double *fr_x, double *fr_y, double *fr_z, double *energy) {
  if (!h) return P3MG_ERR_ARG;
  Ctx *c = &h->c;
  if (c->n > 0 && (!f_x || !f_y || !f_z)) return P3MG_ERR_ARG;
  P3MG_TRY(p3mg_compute(h, rcut));
  return p3mg_get_forces(h, f_x, f_y, f_z, fk_x, fk_y, fk_z, fr_x, fr_y, fr_z, energy);
}

int p3mg_get_forces_device(p3mg_ctx *h, const double **f, const double **fk, const double **fr) {
  if (!h) return P3MG_ERR_ARG;
  if (f) *f = h->c.f;
  if (fk) *fk = h->c.fk;
  if (fr) *fr = h->c.fr;
  return P3MG_OK;
}

int p3mg_enable_timing(p3mg_ctx *h, int on) {
  if (!h) return P3MG_ERR_ARG;
  h->c.timing = on != 0;
  return P3MG_OK;
}

int p3mg_stage_times(p3mg_ctx *h, double t[4]) {
  if (!h || !t) return P3MG_ERR_ARG;
  collect_stage_times(&h->c);
  for (int i = 0; i < 4; i++) t[i] = h->c.stage_ms[i];
  return P3MG_OK;
}

int p3mg_get_influence(p3mg_ctx *h, double *G, double *self81) {
  if (!h) return P3MG_ERR_ARG;
  Ctx *c = &h->c;
  if (!c->have_G) return P3MG_ERR_STATE;
  cudaSetDevice(c->device);
  if (G) P3MG_CUDA_TRY(cudaMemcpy(G, c->G, c->M * sizeof(double), cudaMemcpyDeviceToHost));
  if (self81) memcpy(self81, c->self_b_host, sizeof(c->self_b_host));
  return P3MG_OK;
}

void *p3mg_stream(p3mg_ctx *h) { return h ? (void *)h->c.stream : nullptr; }

int p3mg_set_graph(p3mg_ctx *h, int on) {
  if (!h) return P3MG_ERR_ARG;
  h->c.use_graph = on != 0;
  if (!h->c.use_graph) drop_graph(&h->c);
  return P3MG_OK;
}

int p3mg_set_overlap(p3mg_ctx *h, int on) {
  if (!h) return P3MG_ERR_ARG;
  drop_graph(&h->c);
  h->c.overlap = on != 0;
  return P3MG_OK;
}

int p3mg_launch_count(p3mg_ctx *h, long long *count) {
  if (!h || !count) return P3MG_ERR_ARG;
  *count = h->c.launches;
  return P3MG_OK;
}

int p3mg_kernel_times(p3mg_ctx *h, double t[3]) {
  if (!h || !t) return P3MG_ERR_ARG;
  collect_stage_times(&h->c);
  for (int i = 0; i < 3; i++) t[i] = h->c.kernel_ms[i];
  return P3MG_OK;
}

}  // extern "C"

// sum of q^2 (system_t.q2, io.c:150) from the context's device copy
static int host_q2(Ctx *c, double *q2) {
  *q2 = 0.0;
  const size_t n = (size_t)c->n;
  if (n == 0) return P3MG_OK;
  double *hq = (double *)malloc(n * sizeof(double));
  if (!hq) return P3MG_ERR_ALLOC;
  cudaError_t e = cudaMemcpy(hq, c->q, n * sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    free(hq);
    record_cuda_error(e);
    return P3MG_ERR_CUDA;
  }
  double s = 0.0;
  for (size_t i = 0; i < n; i++) s += hq[i] * hq[i];
  free(hq);
  *q2 = s;
  return P3MG_OK;
}

extern "C" int p3mg_error_estimate(p3mg_ctx *h, double alpha, double rcut, int mc_est, double est[3]) {
  if (!h || !est) return P3MG_ERR_ARG;
  Ctx *c = &h->c;
  if (!(c->L > 0.0)) return P3MG_ERR_NOSYS;
  if (!(alpha > 0.0) || !(rcut >= 0.0) || mc_est < 0) return P3MG_ERR_ARG;
  cudaSetDevice(c->device);
  double q2 = 0.0;
  P3MG_TRY(host_q2(c, &q2));
  return error_estimates(c->method, c->mesh, c->cao, c->n, c->L, q2, alpha, rcut, mc_est, c->stream, &c->launches,
                         est);
}

extern "C" int p3mg_estimate_errors(int method_id, int mesh, int cao, int mc_est, int n, double q2, double L,
                                    double alpha, double rcut, double est[3]) {
  if (!est) return P3MG_ERR_ARG;
  if (!(method_id == 0 || method_id == 1 || method_id == 2 || method_id == 3 || method_id == 6 || method_id == 7))
    return P3MG_ERR_METHOD;
  if (cao < 1 || cao > P3MG_MAX_CAO) return P3MG_ERR_CAO;
  if (mesh < 2 || mesh > P3MG_MAX_MESH || (mesh % 2)) return P3MG_ERR_MESH;
  if (n < 1 || !(q2 >= 0.0) || !(L > 0.0) || !(alpha > 0.0) || !(rcut >= 0.0) || mc_est < 0) return P3MG_ERR_ARG;
  return error_estimates(method_id, mesh, cao, n, L, q2, alpha, rcut, mc_est, cudaStreamPerThread, nullptr, est);
}

extern "C" int p3mg_inhomo_error(p3mg_ctx *h, double alpha, int uniform, int mesh, int cao, int mc,
                                 int collect_mesh, int collect_cao, double *estimate, double *mesh_out) {
  if (!h) return P3MG_ERR_ARG;
  return inhomo_error(&h->c, alpha, uniform, mesh, cao, mc, collect_mesh, collect_cao, estimate, mesh_out);
}

extern "C" int p3mg_error_map(p3mg_ctx *h, int mesh, int cao, const double *fk_x, const double *fk_y,
                              const double *fk_z, const double *ref_x, const double *ref_y, const double *ref_z,
                              double *map, double totals[2]) {
  if (!h) return P3MG_ERR_ARG;
  const double *fk[3] = {fk_x, fk_y, fk_z};
  const double *ref[3] = {ref_x, ref_y, ref_z};
  return error_map(&h->c, mesh, cao, fk, ref, map, totals);
}

extern "C" int p3mg_alpha_range(double alphamin, double alphamax, double alphastep, int cap, double *alphas) {
  if (!(alphastep > 0.0) || !isfinite(alphamin) || !isfinite(alphamax) || cap < 0) return P3MG_ERR_ARG;
  // the reference's loop: alpha accumulated in double (main.c:375)
  int k = 0;
  for (double a = alphamin; a <= alphamax; a += alphastep) {
    if (alphas && k < cap) alphas[k] = a;
    k++;
    if (k > (1 << 24)) return P3MG_ERR_ARG;
  }
  return k;
}

extern "C" int p3mg_sweep(p3mg_ctx *h, double rcut, int nalpha, const double *alphas, const double *ref_x,
                          const double *ref_y, const double *ref_z, double *rms_out, double *f_out, int max_batch) {
  if (!h || nalpha < 0 || (nalpha > 0 && !alphas) || max_batch < 0) return P3MG_ERR_ARG;
  Ctx *c = &h->c;
  if (!(c->L > 0.0)) return P3MG_ERR_NOSYS;
  if (!(rcut >= 0.0)) return P3MG_ERR_ARG;
  const bool want_ref = ref_x || ref_y || ref_z;
  if (want_ref && !(ref_x && ref_y && ref_z)) return P3MG_ERR_ARG;
  if (rms_out && !want_ref) return P3MG_ERR_ARG;
  for (int k = 0; k < nalpha; k++)
    if (!isfinite(alphas[k]) || alphas[k] < 0.0) return P3MG_ERR_ARG;
  if (nalpha == 0) return P3MG_OK;
  cudaSetDevice(c->device);
  const double *const ref[3] = {ref_x, ref_y, ref_z};
  size_t free_b = 0, total_b = 0;
  P3MG_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
  size_t budget = free_b / 2;
  const size_t cap = (size_t)16 << 30;
  if (budget > cap) budget = cap;
  if (max_batch > 0) {
    const size_t b = (size_t)max_batch * sweep_bytes_per_alpha(c);
    if (b < budget) budget = b;
  }
  P3MG_TRY(sweep_run(c, rcut, nalpha, alphas, want_ref ? ref : nullptr, rms_out, f_out, budget, max_batch > 0));
  return check_device_status(c);
}

extern "C" int p3mg_sweep_grid(p3mg_ctx *const *hs, int nctx, double rcut, int nalpha, const double *alphas,
                               const double *ref_x, const double *ref_y, const double *ref_z, double *rms_out) {
  if (!hs || nctx < 1 || nalpha < 0 || (nalpha > 0 && !alphas) || !ref_x || !ref_y || !ref_z || !rms_out)
    return P3MG_ERR_ARG;
  if (!(rcut >= 0.0)) return P3MG_ERR_ARG;
  for (int k = 0; k < nalpha; k++)
    if (!isfinite(alphas[k]) || alphas[k] < 0.0) return P3MG_ERR_ARG;
  std::vector<Ctx *> cs((size_t)nctx);
  for (int i = 0; i < nctx; i++) {
    if (!hs[i]) return P3MG_ERR_ARG;
    cs[i] = &hs[i]->c;
    if (!(cs[i]->L > 0.0)) return P3MG_ERR_NOSYS;
    // one system: the shared real-space forces must fit every context
    if (cs[i]->n != cs[0]->n || cs[i]->L != cs[0]->L || cs[i]->precision != cs[0]->precision ||
        cs[i]->device != cs[0]->device)
      return P3MG_ERR_ARG;
    for (int j = 0; j < i; j++)
      if (cs[j] == cs[i]) return P3MG_ERR_ARG;
  }
  if (nalpha == 0) return P3MG_OK;
  cudaSetDevice(cs[0]->device);
  const double *const ref[3] = {ref_x, ref_y, ref_z};
  size_t free_b = 0, total_b = 0;
  P3MG_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
  size_t budget = free_b / 2;
  const size_t cap = (size_t)32 << 30;
  if (budget > cap) budget = cap;
  P3MG_TRY(sweep_grid_run(cs.data(), nctx, rcut, nalpha, alphas, ref, rms_out, budget));
  for (int i = 0; i < nctx; i++) P3MG_TRY(check_device_status(cs[i]));
  return P3MG_OK;
}

extern "C" int p3mg_sweep_nodes(p3mg_ctx *h, int *nodes, double *check) {
  if (!h || !nodes) return P3MG_ERR_ARG;
  *nodes = h->c.sweep_nodes;
  if (check) *check = h->c.sweep_check;
  return P3MG_OK;
}

extern "C" int p3mg_backward(p3mg_ctx *h, double rcut, double grad_E, double *grad_x, double *grad_y,
                             double *grad_z, double *grad_q, double *grad_alpha, double *grad_L, double parts[5]) {
  if (!h) return P3MG_ERR_ARG;
  Ctx *c = &h->c;
  if (!(c->L > 0.0)) return P3MG_ERR_NOSYS;
  if (!c->have_G) return P3MG_ERR_STATE;
  if (!(c->alpha > 0.0) || !(rcut >= 0.0) || !isfinite(grad_E)) return P3MG_ERR_ARG;
  const bool want_x = grad_x || grad_y || grad_z;
  if (want_x && !(grad_x && grad_y && grad_z)) return P3MG_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t n = (size_t)c->n;
  if (!c->adj_grad || c->adj_cap < c->n) {
    if (c->adj_grad) cudaFree(c->adj_grad);
    c->adj_grad = nullptr;
    c->adj_cap = 0;
    P3MG_CUDA_TRY(cudaMalloc(&c->adj_grad, 4 * (n > 0 ? n : 1) * sizeof(double)));
    c->adj_cap = c->n;
  }
  double *gx = c->adj_grad, *gq = c->adj_grad + 3 * n;
  P3MG_CUDA_TRY(cudaMemsetAsync(c->adj_grad, 0, 4 * n * sizeof(double), c->stream));
  double e5[5], da = 0.0, dl = 0.0;
  P3MG_TRY(adjoint(c, rcut, grad_E, gx, gq, e5, &da, &dl));
  if (parts)
    for (int k = 0; k < 5; k++) parts[k] = e5[k];
  if (grad_alpha) *grad_alpha = da;
  if (grad_L) *grad_L = dl;
  double *dst[4] = {grad_x, grad_y, grad_z, grad_q};
  for (int k = 0; k < 4; k++)
    if (dst[k] && n) P3MG_CUDA_TRY(cudaMemcpyAsync(dst[k], c->adj_grad + k * n, n * sizeof(double),
                                                   cudaMemcpyDeviceToHost, c->stream));
  P3MG_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return P3MG_OK;
}

extern "C" int p3mg_backward_device(p3mg_ctx *h, double rcut, double grad_E, const double **grad_xyz,
                                    const double **grad_q, double *grad_alpha, double *grad_L, double parts[5]) {
  if (!h) return P3MG_ERR_ARG;
  Ctx *c = &h->c;
  if (!(c->L > 0.0)) return P3MG_ERR_NOSYS;
  if (!c->have_G) return P3MG_ERR_STATE;
  if (!(c->alpha > 0.0) || !(rcut >= 0.0) || !isfinite(grad_E)) return P3MG_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t n = (size_t)c->n;
  if (!c->adj_grad || c->adj_cap < c->n) {
    if (c->adj_grad) cudaFree(c->adj_grad);
    c->adj_grad = nullptr;
    c->adj_cap = 0;
    P3MG_CUDA_TRY(cudaMalloc(&c->adj_grad, 4 * (n > 0 ? n : 1) * sizeof(double)));
    c->adj_cap = c->n;
  }
  double *gx = c->adj_grad, *gq = c->adj_grad + 3 * n;
  P3MG_CUDA_TRY(cudaMemsetAsync(c->adj_grad, 0, 4 * n * sizeof(double), c->stream));
  double e5[5], da = 0.0, dl = 0.0;
  P3MG_TRY(adjoint(c, rcut, grad_E, gx, gq, e5, &da, &dl));
  if (parts)
    for (int k = 0; k < 5; k++) parts[k] = e5[k];
  if (grad_alpha) *grad_alpha = da;
  if (grad_L) *grad_L = dl;
  if (grad_xyz) *grad_xyz = gx;
  if (grad_q) *grad_q = gq;
  return P3MG_OK;
}

extern "C" int p3mg_energy(p3mg_ctx *h, double rcut, double parts[5]) {
  if (!parts) return P3MG_ERR_ARG;
  return p3mg_backward(h, rcut, 0.0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, parts);
}

// Brick edge of the charge-assignment tiles and the FFT kernel (0: pencil
// kernels where they apply, else Stockham with the default width; 4, 8, 16:
// Stockham with that many pencils per tile).
static int set_tiles(Ctx *c, int brick, int fft_w) {
  if (brick != 4 && brick != 8) return P3MG_ERR_ARG;
  if (fft_w != 0 && fft_w != 4 && fft_w != 8 && fft_w != 16) return P3MG_ERR_ARG;
  drop_graph(c);
  c->fft_w = fft_w;
  if (brick == c->brick) return P3MG_OK;
  c->brick = brick;
  c->nbrick1 = (c->mesh + brick - 1) / brick;
  const size_t nkey = (size_t)c->nbrick1 * c->nbrick1 * c->nbrick1 * brick * brick * brick;
  dfree(c->brick_count);
  dfree(c->brick_start);
  dfree(c->scatter_tab);  // its pitches depend on the tile edge; rebuilt on the next step
  P3MG_CUDA_TRY(cudaMalloc(&c->brick_count, nkey * sizeof(int)));
  P3MG_CUDA_TRY(cudaMalloc(&c->brick_start, (nkey + 1) * sizeof(int)));
  return scan_tmp_reserve(c, (int)nkey);
}

extern "C" int p3mg_set_tiles(p3mg_ctx *h, int brick, int fft_w) {
  if (!h) return P3MG_ERR_ARG;
  cudaSetDevice(h->c.device);
  return set_tiles(&h->c, brick, fft_w);
}

extern "C" int p3mg_set_gather(p3mg_ctx *h, int mode) {
  if (!h) return P3MG_ERR_ARG;
  if (mode < 0 || mode > 3) return P3MG_ERR_ARG;
  if (mode >= 2 && (h->c.precision == P3MG_FP64 || !gather_tile_fits(&h->c))) return P3MG_ERR_ARG;
  drop_graph(&h->c);
  h->c.gather_mode = mode;
  return P3MG_OK;
}

// Mean device time of `reps` steps after `warm` untimed ones (events on the
// context stream; no graph).
static int time_steps(Ctx *c, double rcut, int warm, int reps, double *ms) {
  for (int i = 0; i < warm; i++) P3MG_TRY(enqueue_step(c, rcut));
  cudaEvent_t a, b;
  P3MG_CUDA_TRY(cudaEventCreate(&a));
  P3MG_CUDA_TRY(cudaEventCreate(&b));
  cudaEventRecord(a, c->stream);
  int st = P3MG_OK;
  for (int i = 0; i < reps && st == P3MG_OK; i++) st = enqueue_step(c, rcut);
  cudaEventRecord(b, c->stream);
  cudaError_t e = cudaEventSynchronize(b);
  float t = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (st != P3MG_OK) return st;
  if (e != cudaSuccess) {
    record_cuda_error(e);
    return P3MG_ERR_CUDA;
  }
  *ms = (double)t / reps;
  return P3MG_OK;
}

extern "C" int p3mg_autotune(p3mg_ctx *h, double rcut, int *brick_out, int *fft_w_out, double *ms_out) {
  if (!h) return P3MG_ERR_ARG;
  Ctx *c = &h->c;
  if (!(c->L > 0.0)) return P3MG_ERR_NOSYS;
  if (!c->have_G) return P3MG_ERR_STATE;
  if (!(rcut >= 0.0)) return P3MG_ERR_ARG;
  cudaSetDevice(c->device);
  const bool timing = c->timing;
  c->timing = false;
  P3MG_TRY(pairs_reserve(c, rcut));
  // FFT: 0 = automatic (the pencil kernels where they apply), then the
  // Stockham tile widths
  const int bricks[2] = {4, 8}, ws[4] = {0, 4, 8, 16};
  int bb = c->brick, bw = c->fft_w, bg = c->gather_mode;
  double best = 1e300;
  int st = P3MG_OK;
  // the gather variants apply to ik methods: lanes on z offsets, thread
  // per particle and (FP32) the TMA-staged brick tiles
  const int ngm = method_ad(c->method) ? 1 : (c->precision == P3MG_FP64 ? 2 : 3);
  for (int ig = 0; ig < ngm && st == P3MG_OK; ig++)
    for (int ib = 0; ib < 2 && st == P3MG_OK; ib++)
      for (int iw = 0; iw < 4 && st == P3MG_OK; iw++) {
        if (bricks[ib] > c->mesh) continue;
        c->gather_mode = ig;
        st = set_tiles(c, bricks[ib], ws[iw]);
        double ms = 0.0;
        if (st == P3MG_OK) st = time_steps(c, rcut, 2, 5, &ms);
        if (st == P3MG_OK && ms < best) {
          best = ms;
          bb = bricks[ib];
          bw = ws[iw];
          bg = ig;
        }
      }
  c->gather_mode = bg;
  if (st == P3MG_OK) st = set_tiles(c, bb, bw);
  c->timing = timing;
  if (st != P3MG_OK) return st;
  if (brick_out) *brick_out = bb;
  if (fft_w_out) *fft_w_out = bw;
  if (ms_out) *ms_out = best;
  return P3MG_OK;
}

// Even mesh sizes the FFT supports (2^a 3^b 5^c 7^d), ascending, in [lo, hi].
static int smooth_meshes(int lo, int hi, int *out, int cap) {
  int k = 0;
  int rad[24], np;
  for (int m = lo; m <= hi && k < cap; m++)
    if (m % 2 == 0 && fft_factor(m, rad, &np) == 0) out[k++] = m;
  return k;
}

extern "C" int p3mg_tune(int method_id, int precision, int n, const double *x, const double *y, const double *z,
                         const double *q, double L, double rcut, double target, int cao_fixed, int mesh_max,
                         int *mesh_out, int *cao_out, double *alpha_out, double *est_out, double *ms_out) {
  if (n < 1 || !x || !y || !z || !q || !(L > 0.0) || !(rcut > 0.0) || !(target > 0.0)) return P3MG_ERR_ARG;
  if (cao_fixed < 0 || cao_fixed > P3MG_MAX_CAO) return P3MG_ERR_CAO;
  if (mesh_max <= 0) mesh_max = 256;
  if (mesh_max > P3MG_MAX_MESH) mesh_max = P3MG_MAX_MESH;
  double q2 = 0.0;
  for (int i = 0; i < n; i++) q2 += q[i] * q[i];
  // alpha from the real-space estimate at rcut (tuning.c:292)
  const double V = L * L * L;
  const double arg = (target * sqrt((double)n * rcut * V)) / (2.0 * sqrt(2.0) * q2);
  if (!(arg > 0.0 && arg < 1.0)) return P3MG_ERR_ARG;
  const double alpha = sqrt(-log(arg)) / rcut;
  int meshes[512];
  const int nm = smooth_meshes(8, mesh_max, meshes, 512);
  const int cmin = cao_fixed ? cao_fixed : 1, cmax = cao_fixed ? cao_fixed : P3MG_MAX_CAO;
  double best = 1e300, best_est = 0.0;
  int bm = 0, bc = 0, cao_last = cmax;
  bool success = false;
  // the reference's search (tuning.c:250-370): meshes ascending; per mesh
  // cao descending while the estimate meets the target, each candidate
  // timed; stop when the cheapest cao of a mesh is already slower than
  // the best, or no cao below the last working one is left
  for (int im = 0; im < nm; im++) {
    const int m = meshes[im];
    int cstart = cmax;
    if (success) {
      if (cao_last <= cmin) break;
      cstart = cao_last - 1;
    }
    double tmin = 1e300;
    for (int cao = cstart; cao >= cmin; cao--) {
      if (cao > m) continue;
      double est[3];
      int st = p3mg_estimate_errors(method_id, m, cao, 1, n, q2, L, alpha, rcut, est);
      if (st != P3MG_OK) return st;
      if (est[0] > target) break;
      cao_last = cao;
      success = true;
      p3mg_ctx *ctx = nullptr;
      st = p3mg_create(&ctx, method_id, m, cao, 1, precision);
      if (st == P3MG_OK) st = p3mg_set_system(ctx, n, x, y, z, q, L);
      if (st == P3MG_OK) st = p3mg_influence(ctx, alpha);
      double ms = 0.0;
      if (st == P3MG_OK) st = pairs_reserve(&ctx->c, rcut);
      if (st == P3MG_OK) st = time_steps(&ctx->c, rcut, 2, 5, &ms);
      p3mg_destroy(ctx);
      if (st != P3MG_OK) return st;
      if (ms < tmin) tmin = ms;
      if (ms < best) {
        best = ms;
        bm = m;
        bc = cao;
        best_est = est[0];
      }
    }
    if (success && tmin > best) break;
  }
  if (!success) return P3MG_ERR_ARG;
  if (mesh_out) *mesh_out = bm;
  if (cao_out) *cao_out = bc;
  if (alpha_out) *alpha_out = alpha;
  if (est_out) *est_out = best_est;
  if (ms_out) *ms_out = best;
  return P3MG_OK;
}

// ---------------------------------------------------------------------------
// Batches of independent systems (no counterpart in the reference): one CUDA
// graph whose parallel branches are the force evaluations of several
// contexts (each on its own stream, joined to the batch stream for the
// capture), launched as one unit so that small systems fill the GPU
// together.  The first run of a batch is eager (allocations, lane tables),
// the second captures, later runs replay; a change of any context's
// particle count or of the cutoffs re-captures.
struct p3mg_batch {
  std::vector<p3mg_ctx *> ctx;
  std::vector<double> rcut;
  std::vector<int> n;
  std::vector<double> L;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, done = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t gexec = nullptr;
  int runs = 0;
  long long launches = 0;
  int device = 0;
};

extern "C" int p3mg_batch_create(p3mg_batch **out, p3mg_ctx *const *ctxs, int count) {
  if (!out || !ctxs || count < 1) return P3MG_ERR_ARG;
  *out = nullptr;
  for (int i = 0; i < count; i++)
    if (!ctxs[i] || ctxs[i]->c.device != ctxs[0]->c.device) return P3MG_ERR_ARG;
  for (int i = 0; i < count; i++)
    for (int j = i + 1; j < count; j++)
      if (ctxs[i] == ctxs[j]) return P3MG_ERR_ARG;
  p3mg_batch *b = new (std::nothrow) p3mg_batch();
  if (!b) return P3MG_ERR_ALLOC;
  b->ctx.assign(ctxs, ctxs + count);
  b->device = ctxs[0]->c.device;
  cudaSetDevice(b->device);
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
  b->join.assign(count, nullptr);
  for (int i = 0; i < count && e == cudaSuccess; i++) e = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    record_cuda_error(e);
    p3mg_batch_destroy(b);
    return P3MG_ERR_CUDA;
  }
  *out = b;
  return P3MG_OK;
}

extern "C" void p3mg_batch_destroy(p3mg_batch *b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  for (cudaEvent_t ev : b->join)
    if (ev) cudaEventDestroy(ev);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->done) cudaEventDestroy(b->done);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

// All branches: fork from the batch stream, one step per context, join.
static int batch_enqueue(p3mg_batch *b, const double *rcuts) {
  P3MG_CUDA_TRY(cudaEventRecord(b->fork, b->stream));
  for (size_t i = 0; i < b->ctx.size(); i++) {
    Ctx *c = &b->ctx[i]->c;
    P3MG_CUDA_TRY(cudaStreamWaitEvent(c->stream, b->fork, 0));
    P3MG_TRY(enqueue_step(c, rcuts[i]));
    P3MG_CUDA_TRY(cudaEventRecord(b->join[i], c->stream));
    P3MG_CUDA_TRY(cudaStreamWaitEvent(b->stream, b->join[i], 0));
  }
  return P3MG_OK;
}

extern "C" int p3mg_batch_compute(p3mg_batch *b, const double *rcuts) {
  if (!b || !rcuts) return P3MG_ERR_ARG;
  const size_t k = b->ctx.size();
  for (size_t i = 0; i < k; i++) {
    Ctx *c = &b->ctx[i]->c;
    if (!(c->L > 0.0)) return P3MG_ERR_NOSYS;
    if (!c->have_G) return P3MG_ERR_STATE;
    if (!(rcuts[i] >= 0.0)) return P3MG_ERR_ARG;
  }
  cudaSetDevice(b->device);
  bool same = (b->rcut.size() == k);
  for (size_t i = 0; same && i < k; i++)
    same = (b->rcut[i] == rcuts[i]) && (b->n[i] == b->ctx[i]->c.n) && (b->L[i] == b->ctx[i]->c.L);
  if (!same) {
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
    b->runs = 0;
    b->rcut.assign(rcuts, rcuts + k);
    b->n.resize(k);
    b->L.resize(k);
    for (size_t i = 0; i < k; i++) {
      b->n[i] = b->ctx[i]->c.n;
      b->L[i] = b->ctx[i]->c.L;
    }
  }
  // stage timing events are not captured; switch them off for the batch
  std::vector<bool> timing(k);
  for (size_t i = 0; i < k; i++) {
    timing[i] = b->ctx[i]->c.timing;
    b->ctx[i]->c.timing = false;
  }
  int st = P3MG_OK;
  if (b->runs == 0) {
    for (size_t i = 0; i < k && st == P3MG_OK; i++) st = pairs_reserve(&b->ctx[i]->c, rcuts[i]);
    if (st == P3MG_OK) st = batch_enqueue(b, rcuts);
    if (st == P3MG_OK) b->runs = 1;
  } else {
    if (!b->gexec) {
      cudaGraph_t g = nullptr;
      long long before = 0;
      for (size_t i = 0; i < k; i++) before += b->ctx[i]->c.launches;
      cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        st = batch_enqueue(b, rcuts);
        e = cudaStreamEndCapture(b->stream, &g);
      }
      long long after = 0;
      for (size_t i = 0; i < k; i++) after += b->ctx[i]->c.launches;
      b->launches = after - before;
      if (st == P3MG_OK && e == cudaSuccess) e = cudaGraphInstantiate(&b->gexec, g, 0);
      if (g) cudaGraphDestroy(g);
      if (st == P3MG_OK && e != cudaSuccess) {
        record_cuda_error(e);
        b->gexec = nullptr;
        st = P3MG_ERR_CUDA;
      }
    }
    if (st == P3MG_OK) {
      cudaError_t e = cudaGraphLaunch(b->gexec, b->stream);
      if (e != cudaSuccess) {
        record_cuda_error(e);
        st = P3MG_ERR_CUDA;
      }
      // the captured launches count towards the first context
      b->ctx[0]->c.launches += b->launches;
      b->runs++;
    }
  }
  // later work on each context stream follows the batch
  if (st == P3MG_OK) {
    cudaError_t e = cudaEventRecord(b->done, b->stream);
    for (size_t i = 0; i < k && e == cudaSuccess; i++) e = cudaStreamWaitEvent(b->ctx[i]->c.stream, b->done, 0);
    if (e != cudaSuccess) {
      record_cuda_error(e);
      st = P3MG_ERR_CUDA;
    }
  }
  for (size_t i = 0; i < k; i++) b->ctx[i]->c.timing = timing[i];
  return st;
}

extern "C" int p3mg_batch_synchronize(p3mg_batch *b) {
  if (!b) return P3MG_ERR_ARG;
  cudaSetDevice(b->device);
  P3MG_CUDA_TRY(cudaStreamSynchronize(b->stream));
  for (p3mg_ctx *h : b->ctx) P3MG_TRY(check_device_status(&h->c));
  return P3MG_OK;
}

// Shared body of the Ewald entries: checks the targets, uploads them, runs
// the Ewald kernels and copies the requested outputs (f and/or fk, each
// three host arrays of nt doubles or NULL) back to the host.
static int ewald_common(Ctx *c, int nt, const int *targets, double alpha, int kmax, bool shell, double rcut_real,
                        double *const f[3], double *const fk[3]) {
  if (nt == 0) return P3MG_OK;
  int *d_tgt = nullptr;
  double *d_out = nullptr, *d_fk = nullptr;
  const size_t bytes = 3 * (size_t)nt * sizeof(double);
  int st = P3MG_OK;
  cudaError_t e = cudaSuccess;
  if (f) e = cudaMalloc(&d_out, bytes);
  if (e == cudaSuccess && fk) e = cudaMalloc(&d_fk, bytes);
  if (e == cudaSuccess && targets) {
    e = cudaMalloc(&d_tgt, (size_t)nt * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(d_tgt, targets, (size_t)nt * sizeof(int), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    record_cuda_error(e);
    st = (e == cudaErrorMemoryAllocation) ? P3MG_ERR_ALLOC : P3MG_ERR_CUDA;
  } else {
    st = ewald_forces(c, nt, d_tgt, alpha, kmax, shell, rcut_real, d_out, d_fk);
    for (int w = 0; w < 2 && st == P3MG_OK; w++) {
      double *const *dst = w ? fk : f;
      const double *src = w ? d_fk : d_out;
      for (int d = 0; dst && d < 3 && e == cudaSuccess; d++)
        e = cudaMemcpy(dst[d], src + (size_t)d * nt, (size_t)nt * sizeof(double), cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) {
        record_cuda_error(e);
        st = P3MG_ERR_CUDA;
      }
    }
  }
  if (d_tgt) cudaFree(d_tgt);
  if (d_out) cudaFree(d_out);
  if (d_fk) cudaFree(d_fk);
  return st;
}

static int check_targets(const Ctx *c, int nt, const int *targets) {
  if (nt < 0 || (!targets && nt != c->n)) return P3MG_ERR_ARG;
  if (targets)
    for (int t = 0; t < nt; t++)
      if (targets[t] < 0 || targets[t] >= c->n) return P3MG_ERR_ARG;
  return P3MG_OK;
}

extern "C" int p3mg_ewald_reference(p3mg_ctx *h, int nt, const int *targets, double *f_x, double *f_y, double *f_z,
                                    double *fk_x, double *fk_y, double *fk_z, double *alpha_out, int *kmax_out,
                                    double *precision_out) {
  if (!h) return P3MG_ERR_ARG;
  Ctx *c = &h->c;
  if (!(c->L > 0.0)) return P3MG_ERR_NOSYS;
  const bool want_f = f_x || f_y || f_z, want_fk = fk_x || fk_y || fk_z;
  if (want_f && !(f_x && f_y && f_z)) return P3MG_ERR_ARG;
  if (want_fk && !(fk_x && fk_y && fk_z)) return P3MG_ERR_ARG;
  P3MG_TRY(check_targets(c, nt, targets));
  cudaSetDevice(c->device);
  double q2 = 0.0;
  P3MG_TRY(host_q2(c, &q2));
  double alpha = 0.0;
  int kmax = 0;
  P3MG_TRY(ewald_parameters(c->n, q2, c->L, c->mesh, &alpha, &kmax));
  if (alpha_out) *alpha_out = alpha;
  if (kmax_out) *kmax_out = kmax;
  if (precision_out) *precision_out = ewald_error(c->n, q2, c->L, 0.49 * c->L, kmax, alpha);
  double *const f[3] = {f_x, f_y, f_z};
  double *const fk[3] = {fk_x, fk_y, fk_z};
  return ewald_common(c, nt, targets, alpha, kmax, true, 0.49 * c->L, want_f ? f : nullptr, want_fk ? fk : nullptr);
}

extern "C" int p3mg_ewald_forces(p3mg_ctx *h, int nt, const int *targets, double *f_x, double *f_y, double *f_z,
                                 double *alpha_out, int *kmax_out) {
  if (h && nt > 0 && (!f_x || !f_y || !f_z)) return P3MG_ERR_ARG;
  return p3mg_ewald_reference(h, nt, targets, f_x, f_y, f_z, nullptr, nullptr, nullptr, alpha_out, kmax_out,
                              nullptr);
}

extern "C" int p3mg_ewald_kspace_forces(p3mg_ctx *h, double alpha, int kmax, int nt, const int *targets,
                                        double *fk_x, double *fk_y, double *fk_z) {
  if (!h) return P3MG_ERR_ARG;
  Ctx *c = &h->c;
  if (!(c->L > 0.0)) return P3MG_ERR_NOSYS;
  if (!(alpha > 0.0) || kmax < 1 || kmax > 4096) return P3MG_ERR_ARG;
  if (nt > 0 && (!fk_x || !fk_y || !fk_z)) return P3MG_ERR_ARG;
  P3MG_TRY(check_targets(c, nt, targets));
  cudaSetDevice(c->device);
  double *const fk[3] = {fk_x, fk_y, fk_z};
  return ewald_common(c, nt, targets, alpha, kmax, false, 0.0, nullptr, fk);
}
