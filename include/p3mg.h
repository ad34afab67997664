/* p3mg — P3M electrostatics on one NVIDIA B200 (sm_100a), C ABI.
 *
 * Drop-in GPU replacement for the k-space force path and the real-space
 * pair loop of the p3m-standalone program.  The reference's plugin table is
 *   method_t { id, name, short_name, flags, Init, Influence_function,
 *              Kspace_force, Error, Error_k }          (types.h:306-316)
 * with the methods registered under ids 0/1/2/3/6/7 (p3m-ik.c:46-49,
 * p3m-ik-i.c:40-43, p3m-ad.c:39-41, p3m-ad-i.c:39-41, p3m-ik-real.c:43-46,
 * p3m-ad-real.c:39-41).  Each entry below names the reference interface it
 * replaces.  Conventions:
 *   - every function returns a status: P3MG_OK (0) or a negative P3MG_ERR_*;
 *     the library never calls exit() (the reference does: parameters.c:137,
 *     io.c:81-84, main.c:341-344);
 *   - particle data are caller-owned SoA host arrays of doubles, one array
 *     per coordinate (the reference's vector_array_t fields, types.h:126-132);
 *   - force outputs ACCUMULATE (+=) exactly like Kspace_force and Realteil;
 *   - a context owns all device memory and one CUDA stream; contexts are
 *     independent, a single context is not re-entrant.
 */
#ifndef P3MG_H
#define P3MG_H

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* status codes */
#define P3MG_OK 0
#define P3MG_ERR_ARG (-1)       /* NULL pointer, n < 0, L <= 0, ... */
#define P3MG_ERR_METHOD (-2)    /* method id not in {0,1,2,3,6,7} (main.c:341-344 exits 126) */
#define P3MG_ERR_CAO (-3)       /* cao not in 1..7 (charge-assign.c:209-211 prints and skips) */
#define P3MG_ERR_MESH (-4)      /* mesh < max(cao,4), > 512, prime factor > 7, or odd for methods 6/7 */
#define P3MG_ERR_NOSYS (-5)     /* no particles set yet */
#define P3MG_ERR_CUDA (-6)      /* CUDA runtime error (see p3mg_last_cuda_error) */
#define P3MG_ERR_ALLOC (-7)     /* device allocation failed */
#define P3MG_ERR_STATE (-8)     /* influence function not computed for this context */
#define P3MG_ERR_PRECISION (-9) /* unknown precision mode */
#define P3MG_ERR_NOBUF (-10)    /* capacity of a caller-provided buffer exceeded */

/* precision modes */
#define P3MG_FP64 0       /* everything in FP64: parity path (<= 1e-10 relative RMS vs the reference) */
#define P3MG_FP32_MIXED 1 /* FP32 mesh, FFTs, weights and pair forces; FP64 G_opt, self-force and geometry */

/* method ids: the reference's enum (types.h:109-118) */
#define P3MG_METHOD_IK 0
#define P3MG_METHOD_IK_I 1
#define P3MG_METHOD_AD 2
#define P3MG_METHOD_AD_I 3
#define P3MG_METHOD_IK_R 6
#define P3MG_METHOD_AD_R 7

typedef struct p3mg_ctx p3mg_ctx;

/* Create a context on the current CUDA device for one method and mesh.
 * mc is the aliasing-sum range P3M_BRILLOUIN (p3m-common.c:33, CLI "mc").
 * Replaces method.Init (e.g. Init_ik p3m-ik.c:75-90, Init_ad_r
 * p3m-ad-real.c:54-67) and Init_data (p3m-common.c:145-232). */
int p3mg_create(p3mg_ctx **ctx, int method_id, int mesh, int cao, int mc, int precision);

/* Release all device memory of the context (Free_data, p3m-common.c:234). */
void p3mg_destroy(p3mg_ctx *ctx);

/* Load n particles (host arrays) and the box length.  Positions are
 * expected in [0, L) like the reference's (charge-assign.c:37-40); other
 * values are folded into the box.  Replaces filling system_t (types.h:163-183). */
int p3mg_set_system(p3mg_ctx *ctx, int n, const double *x, const double *y, const double *z, const double *q,
                    double L);

/* Same with DEVICE pointers (on the context's device); the data are copied
 * into the context on its stream. */
int p3mg_set_system_device(p3mg_ctx *ctx, int n, const double *x, const double *y, const double *z,
                           const double *q, double L);

/* Optimal influence function G_opt for this alpha on the GPU in FP64, and
 * for methods 2 and 7 the ad self-force coefficients.  Replaces
 * method.Influence_function (p3m-ik.c:135-173, p3m-ik-i.c:126-166,
 * p3m-ad.c:111-158 + p3m-ad-self-forces.c:93-112, p3m-ad-i.c:121-150). */
int p3mg_influence(p3mg_ctx *ctx, double alpha);

/* k-space forces accumulated into fk (+=); for methods 2 and 7 the
 * self-force correction is subtracted from ft (may be NULL to skip).
 * Replaces method.Kspace_force (P3M_ik p3m-ik.c:179-245, P3M_ik_i
 * p3m-ik-i.c:169-246, P3M_ad p3m-ad.c:161-210, P3M_ad_i p3m-ad-i.c:153-203,
 * P3M_ik_r p3m-ik-real.c:83-147, P3M_ad_r p3m-ad-real.c:69-118). */
int p3mg_kspace_forces(p3mg_ctx *ctx, double *fk_x, double *fk_y, double *fk_z, double *ft_x, double *ft_y,
                       double *ft_z);

/* Real-space erfc pair forces for all ordered pairs i != j with
 * minimum-image distance <= rcut, accumulated into fr (+=); *energy
 * (may be NULL) receives the pair energy sum 1/2 q_i q_j erfc(alpha r)/r.
 * Replaces Realteil (realpart.c:124-167). */
int p3mg_real_forces(p3mg_ctx *ctx, double rcut, double alpha, double *fr_x, double *fr_y, double *fr_z,
                     double *energy);

/* One force evaluation exactly like Calculate_forces (common.c:268-327):
 * f, f_k and f_r are ZEROED, then real space (skipped when rcut == 0),
 * k-space and self-force, then f += f_k + f_r.  Any of fk_*, fr_* may be
 * NULL; f_* may not.  Uses the alpha of the last p3mg_influence. */
int p3mg_calculate_forces(p3mg_ctx *ctx, double rcut, double *f_x, double *f_y, double *f_z, double *fk_x,
                          double *fk_y, double *fk_z, double *fr_x, double *fr_y, double *fr_z, double *energy);

/* The same step with inputs and outputs resident in device memory: runs
 * on the context's stream and returns without synchronising.  Results are
 * read with p3mg_get_forces / p3mg_get_forces_device. */
int p3mg_compute(p3mg_ctx *ctx, double rcut);

/* Copy the forces of the last p3mg_compute to host arrays (any may be NULL). */
int p3mg_get_forces(p3mg_ctx *ctx, double *f_x, double *f_y, double *f_z, double *fk_x, double *fk_y,
                    double *fk_z, double *fr_x, double *fr_y, double *fr_z, double *energy);

/* Device pointers to the context's force arrays (3n doubles each: x block,
 * y block, z block), valid until the next p3mg_set_system or p3mg_destroy. */
int p3mg_get_forces_device(p3mg_ctx *ctx, const double **f, const double **fk, const double **fr);

/* Stage times of the last step in milliseconds, measured with CUDA events
 * on the context's stream: t[0] charge assignment, t[1] FFTs and
 * convolution, t[2] force assignment and self-force, t[3] real space.
 * Mirrors the reference's tuning timers t_c/t_g/t_f (p3m-common.h:48-57).
 * Stage timing is on only after p3mg_enable_timing(ctx, 1). */
int p3mg_enable_timing(p3mg_ctx *ctx, int on);
int p3mg_stage_times(p3mg_ctx *ctx, double t[4]);

/* The method's analytic RMS force error estimates for the context's system
 * at (alpha, rcut), computed on the GPU: est[0] total = sqrt(est[1]^2 +
 * est[2]^2), est[1] k-space, est[2] real space.  mc_est is the aliasing
 * range P3M_BRILLOUIN_TUNING (CLI "mc_est", default 1).  Replaces
 * method.Error / method.Error_k (p3m-ik.c:249-336, p3m-ik-i.c:249-320,
 * p3m-ad.c:436-505, p3m-ad-i.c:205-294) and Realspace_error
 * (realpart.c:343-346).  For ik (0, 6) and ik-i (1) at the meshes the
 * reference tabulates (q.c:1), cao 1..7 and alpha*L <= 100 the reference
 * interpolates precomputed sums at alpha*L = 0, 1, ..., 100
 * (find_error.c:84-107); this evaluates the sums at the two bracketing
 * points and interpolates the same way. */
int p3mg_error_estimate(p3mg_ctx *ctx, double alpha, double rcut, int mc_est, double est[3]);

/* The same estimates without a context, from the system's particle count n,
 * q2 = sum q_i^2 and box length L (all the reference's estimate functions
 * read from system_t), on the calling thread's current device.  The form a
 * method table's Error(system_t*, parameters_t*) / Error_k entry can call
 * (types.h:306-316).  mesh must be even (the estimate loops run over
 * -mesh/2 .. mesh/2-1). */
int p3mg_estimate_errors(int method_id, int mesh, int cao, int mc_est, int n, double q2, double L, double alpha,
                         double rcut, double est[3]);

/* The alphas of the reference's sweep loop `for (alpha = alphamin; alpha
 * <= alphamax; alpha += alphastep)` (main.c:375), accumulated in double as
 * there (0.1 .. 2.5 step 0.05 gives 49 values, the last
 * 2.4999999999999991).  Writes min(count, cap) values to alphas (may be
 * NULL) and returns the count (>= 0), or P3MG_ERR_ARG. */
int p3mg_alpha_range(double alphamin, double alphamax, double alphastep, int cap, double *alphas);

/* The alpha sweep of the reference's main loop (main.c:375-446) as one
 * batched GPU pass: for each of the nalpha alphas, G_opt (as p3mg_influence)
 * and one force evaluation (as p3mg_calculate_forces with rcut).  The
 * charge assignment and forward FFT run once; G, pairs, convolution,
 * backward FFTs, gather and self forces run batched over the alphas.  Each
 * alpha's forces are the ones the single calls give.
 * With max_batch 0, at least 24 alphas and max alpha <= 2.5 min alpha, the
 * forces are instead evaluated at 10 (FP32) / 16 (FP64) Chebyshev nodes in
 * 1/alpha^2 and interpolated to every alpha, provided two of the requested
 * alphas, also evaluated, agree with the interpolation to 1e-6 (FP32) /
 * 1e-12 (FP64) of their RMS force; otherwise every alpha is evaluated.
 * p3mg_sweep_nodes reports which happened.
 *   ref_x/y/z (host, n each, may all be NULL): reference forces; then
 *   rms_out (host, nalpha, may be NULL) receives sqrt(sum |f - ref|^2) /
 *   sqrt(n) per alpha (Calculate_errors, error.c:21-34, main.c:446).  The
 *   rows are read while the sweep runs, not copied first.
 *   f_out (host, 3 n nalpha doubles, may be NULL): total forces, alpha k
 *   component d particle i at f_out[(k * 3 + d) * n + i].
 *   max_batch: most alphas per batched pass (0: as many as half the free
 *   device memory holds, at most 16 GiB of buffers); a positive value also
 *   has every alpha evaluated.
 * The context's own influence function and forces are left as they were
 * (its charge mesh is overwritten). */
int p3mg_sweep(p3mg_ctx *ctx, double rcut, int nalpha, const double *alphas, const double *ref_x,
               const double *ref_y, const double *ref_z, double *rms_out, double *f_out, int max_batch);

/* The tuning grid over (mesh, cao) of the reference's Tune (tuning.c:250-370)
 * at every alpha: nctx contexts holding the SAME system (particle count,
 * positions, charges, box, precision; each its own method, mesh and cao,
 * distinct contexts) each evaluated at the nalpha alphas like p3mg_sweep
 * with max_batch > 0 (every alpha exact).  The real-space forces depend
 * on neither mesh nor cao: they are computed once per alpha (on ctxs[0]'s
 * stream) and shared; the contexts' k-space passes then run concurrently
 * on their own streams.  rms_out (host, nctx x nalpha, row = context)
 * receives sqrt(sum |f - ref|^2) / sqrt(n) against the reference forces
 * ref_x/y/z (host, n each).  No counterpart in the reference, which runs
 * Calculate_forces point by point. */
int p3mg_sweep_grid(p3mg_ctx *const *ctxs, int nctx, double rcut, int nalpha, const double *alphas,
                    const double *ref_x, const double *ref_y, const double *ref_z, double *rms_out);

/* Interpolation nodes the context's last p3mg_sweep used (0: every alpha
 * was evaluated) and, in check (may be NULL), the larger relative RMS
 * difference between interpolated and evaluated forces at its two check
 * alphas (-1 when no interpolation was tried).  No counterpart in the
 * reference. */
int p3mg_sweep_nodes(p3mg_ctx *ctx, int *nodes, double *check);

/* Electrostatic energy of the P3M approximation (no counterpart in the
 * reference, which computes no P3M energy): parts = {total, k space, real
 * space, self, neutralising}, with
 *   E_k    = c/(2 L^3 nmesh) sum_k G(k) |Q^(k)|^2 over the method's mesh(es)
 *            (charge assignment with the exact B-spline offsets, G = the
 *            context's G_opt at its alpha; nmesh = 2 for interlaced methods;
 *            c = 1 for ad and 1/2 for ik influence functions, matching the
 *            normalisation of their forces),
 *   E_r    = 1/2 sum_{i != j, r <= rcut} q_i q_j erfc(alpha r)/r,
 *   E_self = -alpha/sqrt(pi) sum q^2 (as ewald.c:60-62),
 *   E_neut = -pi Q^2/(2 alpha^2 L^3) for net charge Q.
 * Needs p3mg_influence first (alpha > 0). */
int p3mg_energy(p3mg_ctx *ctx, double rcut, double parts[5]);

/* Adjoint of p3mg_energy (no counterpart in the reference): grad_E times
 * dE/dx, dE/dy, dE/dz and dE/dq (host arrays of n, each may be NULL; x, y, z
 * all or none), dE/dalpha and dE/dL (box length at fixed fractional
 * coordinates; -L dE/dL is the isotropic virial) in grad_alpha / grad_L
 * (may be NULL), and the energy parts (may be NULL).  dE/dx is minus the
 * exact force of this energy: for ad methods the ad force without the
 * self-force correction, for ik methods the gradient of E, which differs
 * from the ik force by its discretisation error. */
int p3mg_backward(p3mg_ctx *ctx, double rcut, double grad_E, double *grad_x, double *grad_y, double *grad_z,
                  double *grad_q, double *grad_alpha, double *grad_L, double parts[5]);

/* The same adjoint with the gradients left in device memory (no
 * counterpart in the reference): *grad_xyz receives a device pointer to
 * grad_E dE/dx (3n doubles: x block, y block, z block) and *grad_q one to
 * grad_E dE/dq (n doubles), both valid until the next backward call, the
 * next p3mg_set_system or p3mg_destroy (either may be NULL).  The scalars
 * are returned as by p3mg_backward; the call returns once they are known. */
int p3mg_backward_device(p3mg_ctx *ctx, double rcut, double grad_E, const double **grad_xyz, const double **grad_q,
                         double *grad_alpha, double *grad_L, double parts[5]);

/* Tile shapes (no counterpart in the reference): brick edge of the
 * charge-assignment tiles (4 or 8 mesh points; the default is 8 for meshes
 * of 64 and more, else 4) and the FFT kernel: 0 (the default) for the
 * register-tiled pencil kernels on FP32 meshes of 32, 64 and 128 points
 * (with the ik convolution folded into the first backward pass) and the
 * shared-memory Stockham kernel with 16 (FP32) / 8 (FP64) pencils per tile
 * otherwise; 4, 8 or 16 for the Stockham kernel with that many pencils.
 * Results differ only by the rounding of the floating-point operations. */
int p3mg_set_tiles(p3mg_ctx *ctx, int brick, int fft_w);

/* Back-interpolation kernel of the ik methods (0, 1, 6; no counterpart in
 * the reference): 0 puts one lane on each z offset of a particle's stencil
 * (8 or 16 lanes per particle, each lane reading a column of consecutive
 * mesh points), 1 runs one thread per particle; P3MG_FP32_MIXED only: 2
 * stages each mesh brick's field tile in shared memory with TMA tensor
 * copies (plain loads where the tile wraps around the periodic mesh) and
 * puts a warp's lanes on the (mesh, b, c) columns of one particle at a
 * time, 3 the same with plain loads only.  The default is 0 for P3MG_FP64
 * and 2 for P3MG_FP32_MIXED (the fastest for each on a B200; a tile that
 * does not fit in shared memory runs mode 1).  Modes 2 and 3 return
 * P3MG_ERR_ARG for P3MG_FP64 contexts.  Results differ only by the
 * rounding of the floating-point sums. */
int p3mg_set_gather(p3mg_ctx *ctx, int mode);

/* Tile autotuner (no counterpart in the reference): times the context's
 * force evaluation with rcut for every brick edge, FFT kernel and gather
 * kernel, keeps the fastest and returns its brick edge, FFT kernel and
 * mean time in ms (outputs may be NULL).  Needs p3mg_influence first. */
int p3mg_autotune(p3mg_ctx *ctx, double rcut, int *brick, int *fft_w, double *ms);

/* The reference's parameter tuner (Tune, tuning.c:250-370) on the GPU: for
 * the given system, method, precision mode and real-space cutoff, alpha
 * from the real-space estimate at rcut (tuning.c:292); then over the even
 * mesh sizes this library transforms (2^a 3^b 5^c 7^d, 8 .. mesh_max, 0 =
 * 256) in ascending order and cao from the top down (cao_fixed != 0: that
 * cao only) while the analytic estimate (mc_est 1) meets target, each
 * candidate's full force evaluation is timed on the GPU; the fastest wins.
 * The reference's search stops the same way (a mesh whose cheapest cao is
 * slower than the best ends it).  Returns mesh, cao, alpha, the estimate and
 * the time in ms (outputs may be NULL); P3MG_ERR_ARG when no candidate
 * meets the target. */
int p3mg_tune(int method_id, int precision, int n, const double *x, const double *y, const double *z,
              const double *q, double L, double rcut, double target, int cao_fixed, int mesh_max, int *mesh,
              int *cao, double *alpha, double *estimate, double *ms);

/* Batches of independent systems (no counterpart in the reference): the
 * force evaluations of several contexts (their own systems, meshes, methods
 * and precisions, on one device) run as the parallel branches of one CUDA
 * graph, so that many small systems occupy the GPU together.  Each
 * context's results are read as after p3mg_compute (p3mg_get_forces or
 * p3mg_get_forces_device).  The first p3mg_batch_compute of a batch runs
 * eagerly, the second captures the graph, later ones replay it; new
 * particle counts, box lengths or cutoffs re-capture.  A context belongs to at most one
 * batch at a time and must not be used on its own while a batch call is in
 * flight; p3mg_batch_destroy leaves the contexts alive. */
typedef struct p3mg_batch p3mg_batch;
int p3mg_batch_create(p3mg_batch **batch, p3mg_ctx *const *ctxs, int count);
int p3mg_batch_compute(p3mg_batch *batch, const double *rcuts);
int p3mg_batch_synchronize(p3mg_batch *batch);
void p3mg_batch_destroy(p3mg_batch *batch);

/* FP64 Ewald reference forces for the context's particles, evaluated on nt
 * target particles (targets: host array of particle indices, or NULL with
 * nt == n for all), written (not accumulated) to the host arrays f_x/f_y/f_z
 * (nt each): real space with rcut = 0.49 L plus the Ewald k-space sum, alpha
 * and kmax chosen like the reference (alpha by bisection with the context's
 * mesh as kmax, then kmax = 2, 4, ... until the estimate <= 1e-8).
 * alpha_out / kmax_out may be NULL.  Replaces Calculate_reference_forces
 * (common.c:329-363) with Ewald_k_space (ewald.c:122-173); the reference's
 * Ewald energy is not reproduced (ewald.c:169 accumulates only the last k). */
int p3mg_ewald_forces(p3mg_ctx *ctx, int nt, const int *targets, double *f_x, double *f_y, double *f_z,
                      double *alpha_out, int *kmax_out);

/* The same reference computation with every output of
 * Calculate_reference_forces: total forces f_* and k-space forces fk_*
 * (either triple may be NULL), alpha, kmax and the Ewald error estimate the
 * reference prints as "Reference precision" (method_ewald.Error,
 * ewald.c:199-201, common.c:361).  What Write_exact_forces (io.c:159-177)
 * writes for reference_out. */
int p3mg_ewald_reference(p3mg_ctx *ctx, int nt, const int *targets, double *f_x, double *f_y, double *f_z,
                         double *fk_x, double *fk_y, double *fk_z, double *alpha_out, int *kmax_out,
                         double *precision_out);

/* FP64 Ewald k-space forces at a given alpha with the spherical cutoff
 * 0 < |n|^2 <= kmax^2, written to fk_* (nt each) for the target particles
 * (as p3mg_ewald_forces).  The reference's method 4 Kspace_force as
 * main.c:392-396 uses it for the "error_k" column: Ewald_init with the P3M
 * mesh and Ewald_compute_influence_function (ewald.c:84-119), i.e. kmax =
 * mesh - 1, at each alpha of the sweep. */
int p3mg_ewald_kspace_forces(p3mg_ctx *ctx, double alpha, int kmax, int nt, const int *targets, double *fk_x,
                             double *fk_y, double *fk_z);

/* Inhomogeneous k-space error estimate of the context's particles
 * (Generic_error_estimate_inhomo, p3m-common.c:437-719, the "inhomo_error"
 * column of main.c:436-447), in FP64 on the GPU:
 *   mesh, cao: the estimator's mesh and window order (main.c "inhomo_mesh",
 *     "inhomo_cao"; mesh 4 .. 512 with prime factors 2, 3, 5, 7 only);
 *   mc: alias range (main.c "inhomo_mc", 0 .. 10); with mc = 0 the kernel
 *     is U2 G_opt - Ghat with an alias-free G_opt, which vanishes up to
 *     rounding, as in the reference;
 *   uniform: rho^2 = sum q^2 / mesh^3 instead of the assigned q_i^2
 *     ("inhomo_uniform");
 *   collect_mesh, collect_cao: mesh spacing L/collect_mesh, stencil shift
 *     and stencil length of the final interpolation at the particles.  The
 *     reference uses the force method's mesh and cao there
 *     (charge-assign.c:1650-1705 called with the method's parameters);
 *     pass the estimator's own values for a self-consistent estimate.
 *     Window weights past the estimator's order count as 0 (the reference
 *     reads past its table rows there).  Indices wrap modulo mesh (the
 *     reference wraps once, which is the same whenever collect_mesh <
 *     2 mesh and collect_cao <= mesh).
 *   estimate: sqrt(sum_i rms_i / n);
 *   mesh_out (host, 5 mesh^3 doubles, may be NULL): per mesh point
 *     (index (i*mesh + j)*mesh + k) rho^2, Re and Im of the error density,
 *     Re and Im of DFT(K^2): the columns of the reference's "inhomo_output"
 *     file (p3m-common.c:683-696). */
int p3mg_inhomo_error(p3mg_ctx *ctx, double alpha, int uniform, int mesh, int cao, int mc, int collect_mesh,
                      int collect_cao, double *estimate, double *mesh_out);

/* Error map (Error_map, p3m-common.c:402-435, main.c "error_map"): the
 * squared k-space force error |ref - fk|^2 of each particle of the context
 * assigned to a mesh of `mesh` points per side with the window of order
 * cao (1 .. 7).  fk_* and ref_* are host arrays of n doubles; map (host,
 * mesh^3 doubles, index (i*mesh + j)*mesh + k) receives the mesh;
 * totals (may be NULL) = {sum of the particles' squared errors, sum over
 * the mesh} (the reference prints both). */
int p3mg_error_map(p3mg_ctx *ctx, int mesh, int cao, const double *fk_x, const double *fk_y, const double *fk_z,
                   const double *ref_x, const double *ref_y, const double *ref_z, double *map, double totals[2]);

/* Copy the FP64 influence function (mesh^3 doubles, full mesh, index
 * (i*mesh + j)*mesh + k as r_ind, p3m-common.h:25) and the 81 ad self-force
 * coefficients (zeros for other methods) to host memory; either may be NULL. */
int p3mg_get_influence(p3mg_ctx *ctx, double *G, double *self_coeffs81);

/* Times in milliseconds of single kernels in the last timed step:
 * t[0] real-space pair kernel, t[1] charge-assignment (scatter) kernel,
 * t[2] back-interpolation (gather) kernel.  Needs p3mg_enable_timing. */
int p3mg_kernel_times(p3mg_ctx *ctx, double t[3]);

/* Replay p3mg_compute as a CUDA graph: the first step for a given particle
 * count and rcut runs eagerly, the next is captured, later ones replay the
 * graph (one launch instead of ~20).  Off by default; stage timing
 * disables it.  No reference counterpart (the reference is single-threaded C). */
int p3mg_set_graph(p3mg_ctx *ctx, int on);

/* Concurrency of a step's two halves (no reference counterpart): on (the
 * default), p3mg_compute runs the real-space pairs on a second stream beside
 * the k-space chain; off, the pairs run first on the context stream and the
 * k-space chain after them, so each kernel has the GPU to itself (what
 * p3mg_kernel_times then reports is each kernel's own duration).  The
 * forces are the same either way. */
int p3mg_set_overlap(p3mg_ctx *ctx, int on);

/* Real-space erfc pair forces that allocate no device memory.
 * No counterpart in the reference.
 * For callers that cannot let a library allocate GPU memory: an engine
 * whose allocator owns all device memory (a library cudaMalloc would
 * synchronise the device and fragment its pool), or a stepping loop that
 * must not allocate after start-up.  The caller passes device-accessible
 * inputs x, y, z, q (n doubles each), the output fr (3n doubles: x block,
 * y block, z block; forces are ADDED, like Realteil) and energy (one double,
 * the pair energy is ADDED), and a cudaStream_t (NULL = default stream).
 * The cell list lives in one static device array of
 * P3MG_NOALLOC_SCRATCH_BYTES in the library, held by every GPU that loads
 * it until the process exits; n above P3MG_NOALLOC_MAX_PARTICLES returns
 * P3MG_ERR_NOBUF.  The first call on a device looks up that array's device
 * address (make it before any stream capture).  Calls share the array:
 * calls that overlap on the GPU race and corrupt each other's results.
 * The call is asynchronous on the given stream. */
#define P3MG_NOALLOC_MAX_PARTICLES 131072
#define P3MG_NOALLOC_MAX_CELLS 32768
#define P3MG_NOALLOC_SCRATCH_BYTES (6u << 20)
int p3mg_real_forces_noalloc(int n, const double *x, const double *y, const double *z, const double *q, double L,
                             double rcut, double alpha, int precision, double *fr, double *energy, void *stream);

/* Number of CUDA kernels this context has launched so far. */
int p3mg_launch_count(p3mg_ctx *ctx, long long *count);

/* The context's CUDA stream (cudaStream_t) as an opaque pointer. */
void *p3mg_stream(p3mg_ctx *ctx);

/* Human-readable text for a status code. */
const char *p3mg_strerror(int status);

/* Text of the last CUDA runtime error seen by any context ("" if none). */
const char *p3mg_last_cuda_error(void);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* P3MG_H */
