/* p3m_gpu: drop-in for the reference's p3m program (main.c:93-470) with the
 * force evaluations on the GPU.  Same "<key> [<value>]" parameters, the
 * same system files, method ids, console table and out.dat columns:
 *
 *   p3m_gpu particles 1000 box 10 mesh 16 cao 7 rcut 3.0 method 7 \
 *           alphamin 0.1 alphamax 2.5 alphastep 0.05
 *
 * For each alpha = alphamin, alphamin + alphastep, ... <= alphamax
 * (accumulated in double, main.c:375) it computes G_opt, one force
 * evaluation (timed), the RMS error against the reference forces (Ewald
 * on the GPU, or a forces file), and the analytic estimates.
 *
 * Additions: "fp32" runs the FP32-mixed pipeline instead of FP64; "alpha"
 * alone runs that single alpha; "batched" computes the whole alpha range
 * in one batched GPU pass (p3mg_sweep) and reports its time divided evenly
 * over the alphas (not with error_k, which needs each alpha's k-space
 * forces); "tune" with "prec" picks mesh, cao (cao 0: any; otherwise that
 * cao) and alpha with the reference's tuning search (tuning.c:250-370,
 * which the reference's main parses but never runs) timed on the GPU, then
 * runs that single alpha.  "inhomo_error" (with inhomo_mesh, inhomo_cao,
 * inhomo_mc, inhomo_uniform, inhomo_output) fills the err_inhomo column
 * from the inhomogeneous estimate on the GPU (main.c:436-440), and
 * "error_map" (with error_k, error_map_mesh, error_map_cao) writes
 * error_map.dat and error_map_2d.dat (main.c:403-424).  Parameters the
 * reference parses for its other analysis side paths (rdf, rdf_species,
 * cdf) are accepted and reported as not provided here. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "p3m_host.h"

static double wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* Petersen's k-space estimate for plain Ewald with kmax = mesh - 1
 * (main.c:79-90): the out.dat column "ewald_error_k_est". */
static double ewald_error_k_estimate(const system_t *s, const parameters_t *p, double alpha) {
  const double pi = 3.14159265358979323846264338328;
  const int kmax = p->mesh - 1;
  return 2.0 * s->q2 * alpha / s->length * sqrt(1.0 / (pi * kmax * s->nparticles)) *
         exp(-(pi * kmax / (alpha * s->length)) * (pi * kmax / (alpha * s->length)));
}

static void write_vtf(const char *filename, const system_t *s) {
  FILE *f = fopen(filename, "w");
  if (!f) {
    fprintf(stderr, "Could not open '%s' for writing.", filename);
    return;
  }
  for (int i = 0; i < s->nparticles; i++) fprintf(f, "a %d t %c r 0.5\n", i, (s->q[i] < 0.0) ? 'O' : 'H');
  fprintf(f, "timestep indexed\n");
  for (int i = 0; i < s->nparticles; i++) fprintf(f, "%d %lf %lf %lf\n", i, s->p->x[i], s->p->y[i], s->p->z[i]);
  fclose(f);
}

/* Smallest minimum-image pair distance (printed before reference_out). */
static double min_distance(const system_t *s) {
  double best = INFINITY;
  const double L = s->length;
  for (int i = 0; i < s->nparticles; i++)
    for (int j = i + 1; j < s->nparticles; j++) {
      double r2 = 0.0;
      for (int d = 0; d < 3; d++) {
        double dx = s->p->fields[d][i] - s->p->fields[d][j];
        dx -= L * round(dx / L);
        r2 += dx * dx;
      }
      if (r2 < best) best = r2;
    }
  return sqrt(best);
}

/* Error map of the k-space forces against the Ewald k-space forces
 * (main.c:403-424, Error_map p3m-common.c:402-435): error_map.dat holds every
 * mesh point, error_map_2d.dat the plane nx = 0.5 mesh.  Both are rewritten
 * and closed at every alpha, so they hold the last alpha's map (the
 * reference leaves its streams open, main.c:407-423, and with several alphas
 * the earlier streams' buffers land in its files at exit). */
static void write_error_map(data_t *data, const forces_t *f, const forces_t *f_ref, int mesh, int cao) {
  puts("Writing error map.");
  const size_t M = (size_t)mesh * mesh * mesh;
  double *map = (double *)malloc((M > 0 ? M : 1) * sizeof(double));
  if (!map) {
    fputs("out of memory\n", stderr);
    exit(1);
  }
  double totals[2] = {0.0, 0.0};
  const int st = p3mg_error_map(data->ctx, mesh, cao, f->f_k->x, f->f_k->y, f->f_k->z, f_ref->f_k->x, f_ref->f_k->y,
                                f_ref->f_k->z, map, totals);
  if (st != P3MG_OK) p3m_host_die(st, "p3mg_error_map");
  printf("dF_total %e dF_total_mesh %e\n", totals[0], totals[1]);
  FILE *out = fopen("error_map.dat", "w");
  FILE *out2d = fopen("error_map_2d.dat", "w");
  if (!out || !out2d) {
    fputs("Could not open error_map.dat / error_map_2d.dat for writing.\n", stderr);
    exit(127);
  }
  const int plane = (int)(0.5 * mesh);
  printf("2d cut plane is nx = %d\n", plane);
  for (int i = 0; i < mesh; i++)
    for (int j = 0; j < mesh; j++)
      for (int k = 0; k < mesh; k++) {
        const double v = map[((size_t)i * mesh + j) * mesh + k];
        fprintf(out, "%d %d %d %e\n", i, j, k, v);
        if (i == plane) fprintf(out2d, "%d %d %e\n", j, k, v);
      }
  fclose(out);
  fclose(out2d);
  free(map);
}

/* Inhomogeneous error estimate as main.c:436-440 calls it: the estimator's
 * mesh, cao and alias range, with the force method's mesh and cao for the
 * final interpolation (collect_rms_nocf gets the method's parameters there).
 * With out_file, one line per mesh point as p3m-common.c:683-692 writes. */
static double inhomo_estimate(data_t *data, const parameters_t *p, int uniform, int mesh, int cao, int mc,
                              const char *out_file) {
  double est = 0.0;
  double *cols = NULL;
  const size_t M = (size_t)mesh * mesh * mesh;
  if (out_file) {
    cols = (double *)malloc(5 * (M > 0 ? M : 1) * sizeof(double));
    if (!cols) {
      fputs("out of memory\n", stderr);
      exit(1);
    }
  }
  const int st = p3mg_inhomo_error(data->ctx, p->alpha, uniform, mesh, cao, mc, p->mesh, p->cao, &est, cols);
  if (st != P3MG_OK) p3m_host_die(st, "p3mg_inhomo_error");
  if (out_file) {
    FILE *f = fopen(out_file, "w");
    if (f) {
      for (int i = 0; i < mesh; i++)
        for (int j = 0; j < mesh; j++)
          for (int k = 0; k < mesh; k++) {
            const double *c = cols + 5 * (((size_t)i * mesh + j) * mesh + k);
            fprintf(f, "%d %d %d %e %e %e %e %e %e\n", i, j, k, c[0], c[1], c[2], c[3], c[4], c[1] * c[0]);
          }
      fclose(f);
    }
    free(cols);
  }
  return est;
}

int main(int argc, char **argv) {
  int methodnr = -1, npart = 0, form_factor = 0, rdf_bins = 100;
  int inhomo_mesh = 64, inhomo_cao = 5, inhomo_mc = 0, error_map_mesh = 64, error_map_cao = 1, nthreads = 0;
  double alphamin = 0, alphamax = 0, alphastep = 0, alpha = 0, length = 0, prec = 0, charge = 1.0;
  double rdf_min = 0, rdf_max = 0;
  char *pos_file = NULL, *force_file = NULL, *out_file = NULL, *ref_out = NULL, *sys_out = NULL, *rdf_file = NULL;
  char *vtf_file = NULL, *cdf_file = NULL, *inhomo_output = NULL;
  parameters_t parameters;
  memset(&parameters, 0, sizeof parameters);
  parameters.mc = 1;
  parameters.mc_est = 1;

  cmd_parameters_t params = {NULL, 0, 0};
  add_param("rcut", ARG_TYPE_FLOAT, ARG_REQUIRED, &parameters.rcut, &params);
  add_param("alphamin", ARG_TYPE_FLOAT, ARG_OPTIONAL, &alphamin, &params);
  add_param("alphamax", ARG_TYPE_FLOAT, ARG_OPTIONAL, &alphamax, &params);
  add_param("alphastep", ARG_TYPE_FLOAT, ARG_OPTIONAL, &alphastep, &params);
  add_param("alpha", ARG_TYPE_FLOAT, ARG_OPTIONAL, &alpha, &params);
  add_param("positions", ARG_TYPE_STRING, ARG_OPTIONAL, &pos_file, &params);
  add_param("error_k", ARG_TYPE_NONE, ARG_OPTIONAL, NULL, &params);
  add_param("forces", ARG_TYPE_STRING, ARG_OPTIONAL, &force_file, &params);
  add_param("mesh", ARG_TYPE_INT, ARG_REQUIRED, &parameters.mesh, &params);
  add_param("cao", ARG_TYPE_INT, ARG_REQUIRED, &parameters.cao, &params);
  add_param("method", ARG_TYPE_INT, ARG_REQUIRED, &methodnr, &params);
  add_param("mc", ARG_TYPE_INT, ARG_OPTIONAL, &parameters.mc, &params);
  add_param("mc_est", ARG_TYPE_INT, ARG_OPTIONAL, &parameters.mc_est, &params);
  add_param("no_estimate", ARG_TYPE_NONE, ARG_OPTIONAL, NULL, &params);
  add_param("outfile", ARG_TYPE_STRING, ARG_OPTIONAL, &out_file, &params);
  add_param("particles", ARG_TYPE_INT, ARG_OPTIONAL, &npart, &params);
  add_param("box", ARG_TYPE_FLOAT, ARG_OPTIONAL, &length, &params);
  add_param("tune", ARG_TYPE_NONE, ARG_OPTIONAL, NULL, &params);
  add_param("prec", ARG_TYPE_FLOAT, ARG_OPTIONAL, &prec, &params);
  add_param("reference_out", ARG_TYPE_STRING, ARG_OPTIONAL, &ref_out, &params);
  add_param("system_out", ARG_TYPE_STRING, ARG_OPTIONAL, &sys_out, &params);
  add_param("verlet_lists", ARG_TYPE_NONE, ARG_OPTIONAL, NULL, &params);
  add_param("charge", ARG_TYPE_FLOAT, ARG_OPTIONAL, &charge, &params);
  add_param("system_type", ARG_TYPE_INT, ARG_OPTIONAL, &form_factor, &params);
  add_param("rdf", ARG_TYPE_STRING, ARG_OPTIONAL, &rdf_file, &params);
  add_param("rdf_bins", ARG_TYPE_INT, ARG_OPTIONAL, &rdf_bins, &params);
  add_param("rdf_rmin", ARG_TYPE_FLOAT, ARG_OPTIONAL, &rdf_min, &params);
  add_param("rdf_rmax", ARG_TYPE_FLOAT, ARG_OPTIONAL, &rdf_max, &params);
  add_param("cdf", ARG_TYPE_STRING, ARG_OPTIONAL, &cdf_file, &params);
  add_param("no_calculation", ARG_TYPE_NONE, ARG_OPTIONAL, NULL, &params);
  add_param("vtf_file", ARG_TYPE_STRING, ARG_OPTIONAL, &vtf_file, &params);
  add_param("rdf_species", ARG_TYPE_NONE, ARG_OPTIONAL, NULL, &params);
  add_param("no_reference_force", ARG_TYPE_NONE, ARG_OPTIONAL, NULL, &params);
  add_param("threads", ARG_TYPE_INT, ARG_OPTIONAL, &nthreads, &params);
  add_param("inhomo_error", ARG_TYPE_NONE, ARG_OPTIONAL, NULL, &params);
  add_param("inhomo_mesh", ARG_TYPE_INT, ARG_OPTIONAL, &inhomo_mesh, &params);
  add_param("inhomo_cao", ARG_TYPE_INT, ARG_OPTIONAL, &inhomo_cao, &params);
  add_param("inhomo_mc", ARG_TYPE_INT, ARG_OPTIONAL, &inhomo_mc, &params);
  add_param("inhomo_output", ARG_TYPE_STRING, ARG_OPTIONAL, &inhomo_output, &params);
  add_param("inhomo_uniform", ARG_TYPE_NONE, ARG_OPTIONAL, NULL, &params);
  add_param("error_map", ARG_TYPE_NONE, ARG_OPTIONAL, NULL, &params);
  add_param("error_map_mesh", ARG_TYPE_INT, ARG_OPTIONAL, &error_map_mesh, &params);
  add_param("error_map_cao", ARG_TYPE_INT, ARG_OPTIONAL, &error_map_cao, &params);
  add_param("fp32", ARG_TYPE_NONE, ARG_OPTIONAL, NULL, &params);
  add_param("batched", ARG_TYPE_NONE, ARG_OPTIONAL, NULL, &params);

  parse_parameters(argc - 1, argv + 1, &params);

  const int calc_k_error = param_isset("error_k", &params);
  const int calc_est = !param_isset("no_estimate", &params);
  parameters.cao3 = parameters.cao * parameters.cao * parameters.cao;
  parameters.ip = parameters.cao - 1;
  parameters.alpha = 0.0;
  parameters.precision = param_isset("fp32", &params) ? P3MG_FP32_MIXED : P3MG_FP64;

  const int tune = param_isset("tune", &params);
  const int have_range =
      param_isset("alphamin", &params) && param_isset("alphamax", &params) && param_isset("alphastep", &params);
  if (tune && !param_isset("prec", &params)) {
    puts("Need 'prec' (target RMS force error) with 'tune'.");
    exit(1);
  }
  if (!have_range && !param_isset("alpha", &params) && !tune) {
    puts("Need to provide either alpha-range (alphamin, alphamax, alphastep) or alpha.");
    exit(1);
  }
  if (!have_range) {
    alphamin = alphamax = alpha;
    alphastep = 1.0;
  }
  if (!(alphastep > 0.0)) {
    puts("alphastep must be positive.");
    exit(1);
  }
  if (!param_isset("positions", &params) && !(param_isset("box", &params) && param_isset("particles", &params))) {
    puts("Need to provide either 'positions' or 'box' and 'particles'.");
    exit(1);
  }

  static const char *const side_paths[] = {"rdf", "rdf_species", "cdf"};
  for (size_t i = 0; i < sizeof side_paths / sizeof side_paths[0]; i++)
    if (param_isset(side_paths[i], &params))
      fprintf(stderr, "Note: '%s' is not provided by this program; ignored.\n", side_paths[i]);

  system_t *system;
  if (param_isset("positions", &params)) {
    puts("Reading file");
    system = Read_system(&parameters, pos_file);
    puts("Done.");
  } else {
    puts("Generating system.");
    if (param_isset("system_type", &params)) {
      printf("Using system type %d\n", form_factor);
      system = generate_system(form_factor, npart, length, charge);
    } else {
      system = generate_system(SYSTEM_RANDOM, npart, length, charge);
    }
    if (!system) exit(1);
    puts("Done.");
  }

  if (tune) {
    if (!method_by_id(methodnr)) {
      fprintf(stderr, "Method %d not know.", methodnr);
      exit(126);
    }
    int tm = 0, tc = 0;
    double ta = 0.0, te = 0.0, tms = 0.0;
    const int st = p3mg_tune(methodnr, parameters.precision, system->nparticles, system->p->x, system->p->y,
                             system->p->z, system->q, system->length, parameters.rcut, prec, parameters.cao, 0, &tm,
                             &tc, &ta, &te, &tms);
    if (st != P3MG_OK) p3m_host_die(st, "p3mg_tune");
    printf("Tuned for precision %e: mesh %d cao %d alpha %lf (estimate %e, %e ms per force evaluation)\n", prec, tm,
           tc, ta, te, tms);
    parameters.mesh = tm;
    parameters.cao = tc;
    parameters.cao3 = tc * tc * tc;
    parameters.ip = tc - 1;
    alphamin = alphamax = ta;
    alphastep = 1.0;
  }

  if (param_isset("vtf_file", &params)) write_vtf(vtf_file, system);

  forces_t *forces = Init_forces(system->nparticles);
  forces_t *forces_ewald = Init_forces(system->nparticles);

  if (param_isset("reference_out", &params)) {
    if (system->nparticles <= 100000) printf("Minimal distance: %.*f\n", 17, min_distance(system));
    puts("Calculating reference forces.");
    printf("Reference precision %e\n.", Calculate_reference_forces(system, &parameters));
    puts("Done.");
    printf("Writing reference forces to '%s'\n", ref_out);
    Write_exact_forces(system, ref_out);
    puts("Done.");
  }

  if (param_isset("system_out", &params)) {
    printf("Writing system to '%s'\n", sys_out);
    Write_system(system, sys_out);
    puts("Done.");
  }

  if (param_isset("forces", &params)) {
    printf("Reading reference forces from '%s'.\n", force_file);
    Read_exact_forces(system, force_file);
    puts("Done.");
  } else if (!param_isset("no_reference_force", &params)) {
    if (!param_isset("reference_out", &params)) {
      puts("Calculating reference forces.");
      printf("Reference precision %e\n.", Calculate_reference_forces(system, &parameters));
      puts("Done.");
    }
  } else {
    puts("Skipping reference force calculation.");
  }

  const method_t *method = method_by_id(methodnr);
  if (!method) {
    fprintf(stderr, "Method %d not know.", methodnr);
    exit(126);
  }

  fprintf(stderr, "Using %s.\n", method->method_name);

  FILE *fout = fopen(param_isset("outfile", &params) ? out_file : "out.dat", "w");
  if (!fout) {
    fprintf(stderr, "Could not open '%s' for writing.\n", param_isset("outfile", &params) ? out_file : "out.dat");
    exit(127);
  }

  printf("Init");
  fflush(stdout);
  data_t *data = method->Init(system, &parameters);
  printf(".\n");

  const size_t n = (size_t)system->nparticles;
  double walltime = 0.0, estimate = 0.0, error_k_est = 0.0;

  /* batched sweep: every alpha's RMS error from one p3mg_sweep call */
  double *batch_rms = NULL, batch_time = 0.0;
  const int batched = param_isset("batched", &params) && !calc_k_error && !param_isset("no_calculation", &params);
  if (param_isset("batched", &params) && !batched)
    fprintf(stderr, "Note: 'batched' is not combined with error_k or no_calculation; running alpha by alpha.\n");
  if (batched) {
    const int na = p3mg_alpha_range(alphamin, alphamax, alphastep, 0, NULL);
    if (na < 0) p3m_host_die(na, "p3mg_alpha_range");
    double *al = (double *)malloc((size_t)(na > 0 ? na : 1) * sizeof(double));
    batch_rms = (double *)calloc((size_t)(na > 0 ? na : 1), sizeof(double));
    if (!al || !batch_rms) {
      fputs("out of memory\n", stderr);
      exit(1);
    }
    p3mg_alpha_range(alphamin, alphamax, alphastep, na, al);
    const forces_t *r = system->reference;
    batch_time = wtime();
    const int st = p3mg_sweep(data->ctx, parameters.rcut, na, al, r->f->x, r->f->y, r->f->z, batch_rms, NULL, 0);
    batch_time = wtime() - batch_time;
    if (st != P3MG_OK) p3m_host_die(st, "p3mg_sweep");
    if (na > 0) batch_time /= na;
    free(al);
  }
  int ia = 0;
  printf("# %8s\t%8s\t%8s\t%8s\t%8s\n", "alpha", "DeltaF", "Estimate", "R-Error-Est",
         "K-Error-Est Generic-K-Space-err");
  for (parameters.alpha = alphamin; parameters.alpha <= alphamax; parameters.alpha += alphastep, ia++) {
    if (!batched) method->Influence_function(system, &parameters, data);

    if (batched) {
      walltime = batch_time;
    } else if (!param_isset("no_calculation", &params)) {
      walltime = wtime();
      Calculate_forces(method, system, &parameters, data, forces);
      walltime = wtime() - walltime;
    }

    double error_k = 0.0;
    if (calc_k_error) {
      const int st = p3mg_ewald_kspace_forces(data->ctx, parameters.alpha, parameters.mesh - 1, system->nparticles,
                                              NULL, forces_ewald->f_k->x, forces_ewald->f_k->y, forces_ewald->f_k->z);
      if (st != P3MG_OK) p3m_host_die(st, "p3mg_ewald_kspace_forces");
      for (size_t i = 0; i < n; i++)
        for (int j = 0; j < 3; j++) {
          const double dv = forces->f_k->fields[j][i] - forces_ewald->f_k->fields[j][i];
          error_k += dv * dv;
        }
      error_k = sqrt(error_k) / sqrt((double)n);
      if (param_isset("error_map", &params)) write_error_map(data, forces, forces_ewald, error_map_mesh, error_map_cao);
    }

    const double ewald_error_k_est = ewald_error_k_estimate(system, &parameters, parameters.alpha);
    double ef = 0.0;
    if (batched) {
      ef = batch_rms[ia] * sqrt((double)n);
    } else {
      for (size_t i = 0; i < n; i++)
        for (int j = 0; j < 3; j++) {
          const double dv = forces->f->fields[j][i] - system->reference->f->fields[j][i];
          ef += dv * dv;
        }
      ef = sqrt(ef);
    }

    if (calc_est) {
      estimate = method->Error(system, &parameters);
      error_k_est = method->Error_k(system, &parameters);
    }
    double err_inhomo = 0.0;
    if (param_isset("inhomo_error", &params))
      err_inhomo = inhomo_estimate(data, &parameters, param_isset("inhomo_uniform", &params), inhomo_mesh, inhomo_cao,
                                   inhomo_mc, param_isset("inhomo_output", &params) ? inhomo_output : NULL);
    const double rs_error = Realspace_error(system, &parameters);

    printf("%8lf\t%8e\t%8e\t %8e %8e\t %8e sec\t %8e %8e\n", parameters.alpha, ef / sqrt((double)n), estimate,
           rs_error, error_k_est, walltime, err_inhomo, error_k);
    fprintf(fout, "% lf\t% e\t% e\t% e\t% e\t% e\t% e\t% e\n", parameters.alpha, ef / sqrt((double)n), estimate,
            rs_error, error_k_est, error_k, ewald_error_k_est, err_inhomo);
    fflush(stdout);
    fflush(fout);
  }
  fclose(fout);
  free(batch_rms);

  Free_data(data);
  Free_forces(forces);
  Free_forces(forces_ewald);
  Free_system(system);
  free(params.list);
  return 0;
}
