/* Host side of the drop-in p3m program: the reference's command line, file
 * formats and method table, with every force evaluation on the GPU through
 * the p3mg C ABI (include/p3mg.h).
 *
 * The types mirror the reference's (types.h): SoA particle data
 * (fields[3][N] + q[N], types.h:100-140), forces_t with f, f_k, f_r
 * (types.h:150-160), parameters_t (types.h:170-190) and the method table
 * method_t {id, name, short_name, flags, Init, Influence_function,
 * Kspace_force, Error, Error_k} (types.h:306-316) under the same ids. */
#ifndef P3M_HOST_H
#define P3M_HOST_H

#include <stdio.h>

#include "p3mg.h"

/* SoA vector field: fields[0..2] alias x, y, z (types.h:100-112). */
typedef struct {
  double *fields[3];
  double *x, *y, *z;
  int size;
} vector_array_t;

typedef struct {
  vector_array_t *f, *f_k, *f_r;
} forces_t;

typedef struct {
  int nparticles;
  double length;
  double q2;          /* sum q_i^2, used by the estimates (io.c:152) */
  vector_array_t *p;  /* positions */
  double *q;
  forces_t *reference;  /* reference (Ewald or file) forces */
  double energy;
} system_t;

typedef struct {
  double alpha;
  double rcut;
  int mesh;
  int cao;
  int cao3;
  int ip;
  int tuning;
  int mc;         /* P3M_BRILLOUIN: aliasing range of G_opt */
  int mc_est;     /* P3M_BRILLOUIN_TUNING: aliasing range of the estimates */
  int precision;  /* P3MG_FP64 or P3MG_FP32_MIXED */
} parameters_t;

/* Method-owned state: the GPU context (meshes, G, plans, device copies). */
typedef struct {
  p3mg_ctx *ctx;
  int method_id;
  const system_t *system;
  double runtime[4]; /* stage times of the last step, seconds: t_c, t_g, t_f, t_r */
} data_t;

enum {
  METHOD_FLAG_none = 0,
  METHOD_FLAG_ik = 1,
  METHOD_FLAG_ad = 2,
  METHOD_FLAG_interlaced = 4,
  METHOD_FLAG_nshift = 8,
  METHOD_FLAG_G_hat = 16,
  METHOD_FLAG_Qmesh = 32,
  METHOD_FLAG_ca = 64,
  METHOD_FLAG_self_force_correction = 128
};
#define METHOD_FLAG_P3M (METHOD_FLAG_nshift | METHOD_FLAG_G_hat | METHOD_FLAG_Qmesh | METHOD_FLAG_ca)

typedef struct {
  int method_id;
  const char *method_name;
  const char *method_name_short;
  int flags;
  data_t *(*Init)(system_t *, parameters_t *);
  void (*Influence_function)(system_t *, parameters_t *, data_t *);
  void (*Kspace_force)(system_t *, parameters_t *, data_t *, forces_t *);
  double (*Error)(system_t *, parameters_t *);
  double (*Error_k)(system_t *, parameters_t *);
} method_t;

/* methods.c */
extern const method_t method_p3m_ik, method_p3m_ik_i, method_p3m_ad, method_p3m_ad_i, method_p3m_ik_r,
    method_p3m_ad_r;
const method_t *method_by_id(int id);
void Free_data(data_t *d);
void Calculate_forces(const method_t *m, system_t *s, parameters_t *p, data_t *d, forces_t *f);
double Calculate_reference_forces(system_t *s, parameters_t *p);
double Realspace_error(const system_t *s, const parameters_t *p);
void p3m_host_die(int status, const char *what);

/* io.c */
vector_array_t *Init_vector_array(int n);
void Free_vector_array(vector_array_t *v);
forces_t *Init_forces(int n);
void Free_forces(forces_t *f);
system_t *Init_system(int n);
void Free_system(system_t *s);
system_t *Read_system(parameters_t *p, const char *filename);
void Write_system(const system_t *s, const char *filename);
void Read_exact_forces(system_t *s, const char *filename);
void Write_exact_forces(const system_t *s, const char *filename);

/* generate.c */
enum {
  SYSTEM_RANDOM = 0,
  SYSTEM_INNER_BOX = 1,
  SYSTEM_MADELUNG = 2,
  SYSTEM_SEPARATED_DIPOLE = 3,
  SYSTEM_GAUSSIAN = 4,
  SYSTEM_SLAB = 5
};
system_t *generate_system(int type, int size, double box, double charge);

/* params.c */
enum { ARG_TYPE_INT, ARG_TYPE_FLOAT, ARG_TYPE_STRING, ARG_TYPE_NONE };
enum { ARG_OPTIONAL, ARG_REQUIRED };
typedef struct {
  const char *name;
  int type;
  int required;
  void *value;
  int is_set;
} cmd_parameter_t;
typedef struct {
  cmd_parameter_t *list;
  int n, cap;
} cmd_parameters_t;
void add_param(const char *name, int type, int reqopt, void *value, cmd_parameters_t *params);
int param_isset(const char *name, const cmd_parameters_t *params);
void parse_parameters(int argc, char **argv, cmd_parameters_t *params);

#endif
