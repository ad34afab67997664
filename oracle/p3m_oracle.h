/* ORACLE — test infrastructure only (see p3m_oracle.c). */
#ifndef P3M_ORACLE_H
#define P3M_ORACLE_H

void oracle_bspline(int cao, double x, double *w, double *dw);
int oracle_influence(int method, int mesh, int cao, int mc, double alpha, double L, double *G);
int oracle_self_force_coeffs(int mesh, int cao, double L, const double *G, double *b81);
int oracle_kspace(int method, int mesh, int cao, int mc, double alpha, int n, const double *x, const double *y,
                  const double *z, const double *q, double L, const double *G, double *fk, double *ftot);
int oracle_realspace(int n, const double *x, const double *y, const double *z, const double *q, double L, double rcut,
                     double alpha, double *fr, double *energy, int cells);
int oracle_forces(int method, int mesh, int cao, int mc, double alpha, double rcut, int n, const double *x,
                  const double *y, const double *z, const double *q, double L, const double *G, double *f, double *fk,
                  double *fr, double *energy, int cells);
int oracle_ewald_parameters(int n, double q2, double L, int mesh_param, double *alpha, int *kmax);
int oracle_ewald_kspace(int n, const double *x, const double *y, const double *z, const double *q, double L, double alpha,
                        int kmax, int nt, const int *tgt, double *fk);
int oracle_ewald_kspace_plain(int n, const double *x, const double *y, const double *z, const double *q, double L,
                              double alpha, int kmax, int nt, const int *tgt, double *fk);
int oracle_ewald(int n, const double *x, const double *y, const double *z, const double *q, double L, int mesh_param,
                 int nt, const int *tgt, double *f, double *fk, double *fr, double *alpha_out, int *kmax_out);
double oracle_rms_error(int n, const double *f, const double *ref);
double oracle_realspace_error(int n, double q2, double L, double rcut, double alpha);
int oracle_estimate_table_mesh(int mesh);
double oracle_kspace_error(int method, int mesh, int cao, int mc_est, double alpha, int n, double q2, double L);
int oracle_inhomo_error(int n, const double *x, const double *y, const double *z, const double *q, double L,
                        double alpha, int uniform, int mesh, int cao, int mc, int collect_mesh, int collect_cao,
                        double *estimate, double *mesh_out);
int oracle_error_map(int n, const double *x, const double *y, const double *z, double L, const double *fk,
                     const double *fk_ref, int mesh, int cao, double *map);

#endif
