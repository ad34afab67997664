/* Particle and force files in the reference's formats (io.c:70-225):
 *
 *   positions:   "# Teilchenzahl: <n>", "# Len: <L>", then n lines "x y z q"
 *   forces in:   n lines "<i> fx fy fz" (io.c:70-98); lines may also carry
 *                the three k-space columns that Write_exact_forces adds
 *   forces out:  n lines "<i> fx fy fz fkx fky fkz" (io.c:159-177)
 *
 * Unreadable files exit 127 and malformed ones -1 (255), as in the
 * reference.  Widenings, for the reference's own data sets
 * (Data/ReferenceDataVincent):
 *   - further "#" lines after the header (the "# Mesh:", "# kmax:",
 *     "# alpha:" ... lines of the Konfig_NN.dat files) are skipped;
 *   - a positions file without the "#" header is read as the simulation
 *     snapshots konfig_N: a line with the count, a line with the box
 *     length, then "x y z q" with unwrapped coordinates, which are folded
 *     into [0, L) here (the reference's mesh code wraps only once,
 *     charge-assign.c:37-40);
 *   - a forces file may have 4 or 7 columns per line (the reference reader
 *     only parses 4, so it cannot read back its own 7-column output), and a
 *     4-column line whose first field is not an integer is a Konfig_NN.exact
 *     line "E fx fy fz" (total Coulomb energy, then the force). */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "p3m_host.h"

vector_array_t *Init_vector_array(int n) {
  vector_array_t *v = (vector_array_t *)calloc(1, sizeof(vector_array_t));
  double *buf = (double *)calloc(3 * (size_t)(n > 0 ? n : 1), sizeof(double));
  if (!v || !buf) {
    fputs("out of memory\n", stderr);
    exit(1);
  }
  for (int d = 0; d < 3; d++) v->fields[d] = buf + (size_t)d * n;
  v->x = v->fields[0];
  v->y = v->fields[1];
  v->z = v->fields[2];
  v->size = n;
  return v;
}

void Free_vector_array(vector_array_t *v) {
  if (!v) return;
  free(v->fields[0]);
  free(v);
}

forces_t *Init_forces(int n) {
  forces_t *f = (forces_t *)calloc(1, sizeof(forces_t));
  if (!f) {
    fputs("out of memory\n", stderr);
    exit(1);
  }
  f->f = Init_vector_array(n);
  f->f_k = Init_vector_array(n);
  f->f_r = Init_vector_array(n);
  return f;
}

void Free_forces(forces_t *f) {
  if (!f) return;
  Free_vector_array(f->f);
  Free_vector_array(f->f_k);
  Free_vector_array(f->f_r);
  free(f);
}

system_t *Init_system(int n) {
  system_t *s = (system_t *)calloc(1, sizeof(system_t));
  if (!s) {
    fputs("out of memory\n", stderr);
    exit(1);
  }
  s->nparticles = n;
  s->p = Init_vector_array(n);
  s->q = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  s->reference = Init_forces(n);
  if (!s->q) {
    fputs("out of memory\n", stderr);
    exit(1);
  }
  return s;
}

void Free_system(system_t *s) {
  if (!s) return;
  Free_vector_array(s->p);
  free(s->q);
  Free_forces(s->reference);
  free(s);
}

static FILE *open_or_die(const char *filename, const char *mode) {
  FILE *fp = fopen(filename, mode);
  if (!fp) {
    fprintf(stderr, "Could not open '%s' for %s.\n", filename, mode[0] == 'r' ? "reading" : "writing");
    exit(127);
  }
  return fp;
}

static void bad_file(const char *filename, FILE *fp) {
  fprintf(stderr, "Error while reading file '%s'\n", filename);
  fclose(fp);
  exit(-1);
}

/* x folded into [0, L) */
static double fold(double x, double L) {
  double r = x - L * floor(x / L);
  return (r >= L || r < 0.0) ? 0.0 : r;
}

/* konfig_N snapshot: count line, length line, n lines "x y z q" */
static system_t *read_konfig(const char *filename, FILE *fp) {
  int n = -1;
  double len = 0.0;
  if (fscanf(fp, "%d", &n) != 1 || fscanf(fp, "%lf", &len) != 1 || n < 0 || !(len > 0.0)) bad_file(filename, fp);
  system_t *s = Init_system(n);
  s->length = len;
  s->q2 = 0.0;
  for (int i = 0; i < n; i++) {
    double x, y, z;
    if (fscanf(fp, "%lf %lf %lf %lf", &x, &y, &z, &s->q[i]) != 4) bad_file(filename, fp);
    s->p->x[i] = fold(x, len);
    s->p->y[i] = fold(y, len);
    s->p->z[i] = fold(z, len);
    s->q2 += s->q[i] * s->q[i];
  }
  fclose(fp);
  return s;
}

system_t *Read_system(parameters_t *p, const char *filename) {
  (void)p;
  FILE *fp = open_or_die(filename, "r");
  int n = -1;
  double len = 0.0;
  int first;
  while ((first = fgetc(fp)) == ' ' || first == '\t' || first == '\n' || first == '\r') {
  }
  if (first == EOF) bad_file(filename, fp);
  ungetc(first, fp);
  if (first != '#') return read_konfig(filename, fp);
  if (fscanf(fp, " # Teilchenzahl: %d", &n) != 1 || fscanf(fp, " # Len: %lf", &len) != 1 || n < 0)
    bad_file(filename, fp);
  /* skip any further comment lines */
  int ch;
  for (;;) {
    while ((ch = fgetc(fp)) == ' ' || ch == '\t' || ch == '\n' || ch == '\r') {
    }
    if (ch != '#') {
      if (ch != EOF) ungetc(ch, fp);
      break;
    }
    while ((ch = fgetc(fp)) != '\n' && ch != EOF) {
    }
  }
  system_t *s = Init_system(n);
  s->length = len;
  s->q2 = 0.0;
  for (int i = 0; i < n; i++) {
    if (fscanf(fp, "%lf %lf %lf %lf", &s->p->x[i], &s->p->y[i], &s->p->z[i], &s->q[i]) != 4) bad_file(filename, fp);
    s->q2 += s->q[i] * s->q[i];
  }
  fclose(fp);
  return s;
}

void Write_system(const system_t *s, const char *filename) {
  FILE *fp = open_or_die(filename, "w");
  fprintf(fp, "# Teilchenzahl: %d\n", s->nparticles);
  fprintf(fp, "# Len: %lf\n", s->length);
  for (int i = 0; i < s->nparticles; i++)
    fprintf(fp, "%lf\t%lf\t%lf\t%lf\n", s->p->x[i], s->p->y[i], s->p->z[i], s->q[i]);
  fclose(fp);
}

void Read_exact_forces(system_t *s, const char *filename) {
  printf("npart %d\n", s->nparticles);
  FILE *fp = open_or_die(filename, "r");
  char line[1024];
  int i = 0;
  while (i < s->nparticles && fgets(line, sizeof line, fp)) {
    double v[7];
    const int got = sscanf(line, "%lf %lf %lf %lf %lf %lf %lf", v + 6, v, v + 1, v + 2, v + 3, v + 4, v + 5);
    if (got == EOF || got == 0) continue; /* blank line */
    /* the first field: an index (reference layout) or, with 4 fields and a
     * fraction or exponent in it, the energy of a .exact line */
    const char *t = line + strspn(line, " \t");
    const size_t tl = strcspn(t, " \t\r\n");
    const int integer = memchr(t, '.', tl) == NULL && memchr(t, 'e', tl) == NULL && memchr(t, 'E', tl) == NULL;
    if ((got != 4 && got != 7) || (got == 7 && !integer)) {
      fprintf(stderr, "Error while reading file '%s' (%d) (%d)\n", filename, got, i);
      fclose(fp);
      exit(-1);
    }
    s->reference->f->x[i] = v[0];
    s->reference->f->y[i] = v[1];
    s->reference->f->z[i] = v[2];
    if (got == 7) {
      s->reference->f_k->x[i] = v[3];
      s->reference->f_k->y[i] = v[4];
      s->reference->f_k->z[i] = v[5];
    }
    i++;
  }
  fclose(fp);
  if (i != s->nparticles) {
    fprintf(stderr, "Error while reading file '%s' (%d) (%d)\n", filename, 0, i);
    exit(-1);
  }
}

void Write_exact_forces(const system_t *s, const char *filename) {
  FILE *fp = open_or_die(filename, "w");
  const forces_t *r = s->reference;
  for (int i = 0; i < s->nparticles; i++)
    fprintf(fp, "%d\t%lf\t%lf\t%lf\t%lf\t%lf\t%lf\n", i, r->f->x[i], r->f->y[i], r->f->z[i], r->f_k->x[i],
            r->f_k->y[i], r->f_k->z[i]);
  fclose(fp);
}
