/* Command-line parameters of the form "<key> [<value>]" in any order, with
 * the reference's behaviour (parameters.c:41-160): a key takes the next
 * word as its value unless it is a flag; an unknown key prints
 * "Unknown parameter '<key>'" and exits 23; a missing required key prints
 * "Required parameter '<key>' missing." and exits -1 (255). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "p3m_host.h"

void add_param(const char *name, int type, int reqopt, void *value, cmd_parameters_t *params) {
  if (params->n == params->cap) {
    params->cap = params->cap ? 2 * params->cap : 32;
    params->list = (cmd_parameter_t *)realloc(params->list, (size_t)params->cap * sizeof(cmd_parameter_t));
    if (!params->list) {
      fputs("out of memory\n", stderr);
      exit(1);
    }
  }
  cmd_parameter_t *p = &params->list[params->n++];
  p->name = name;
  p->type = type;
  p->required = (reqopt == ARG_REQUIRED);
  p->value = value;
  p->is_set = 0;
}

static cmd_parameter_t *find(const cmd_parameters_t *params, const char *name) {
  for (int i = 0; i < params->n; i++)
    if (strcmp(params->list[i].name, name) == 0) return &params->list[i];
  return NULL;
}

int param_isset(const char *name, const cmd_parameters_t *params) {
  const cmd_parameter_t *p = find(params, name);
  return p ? p->is_set : 0;
}

static void print_parameter(const cmd_parameter_t *p) {
  if (!p->is_set) {
    printf("'%s' = not set, ", p->name);
    return;
  }
  switch (p->type) {
    case ARG_TYPE_INT: printf("'%s' = %d, ", p->name, *(int *)p->value); break;
    case ARG_TYPE_FLOAT: printf("'%s' = %lf, ", p->name, *(double *)p->value); break;
    case ARG_TYPE_STRING: printf("'%s' = '%s', ", p->name, *(char **)p->value); break;
    default: printf("'%s' is set, ", p->name);
  }
}

void parse_parameters(int argc, char **argv, cmd_parameters_t *params) {
  int nreq = 0;
  for (int i = 0; i < params->n; i++) nreq += params->list[i].required;
  printf("Parsing for %d required and %d optional parameters.\n", nreq, params->n - nreq);
  for (int a = 0; a < argc; a++) {
    cmd_parameter_t *p = find(params, argv[a]);
    if (!p) {
      printf("Unknown parameter '%s'\n", argv[a]);
      exit(23);
    }
    if (p->type != ARG_TYPE_NONE) {
      if (a + 1 >= argc) {
        printf("Parameter '%s' needs a value.\n", argv[a]);
        exit(23);
      }
      const char *v = argv[++a];
      if (p->type == ARG_TYPE_INT)
        *(int *)p->value = atoi(v);
      else if (p->type == ARG_TYPE_FLOAT)
        *(double *)p->value = atof(v);
      else
        *(char **)p->value = (char *)v;
    }
    p->is_set = 1;
  }
  for (int i = 0; i < params->n; i++)
    if (params->list[i].required) {
      if (!params->list[i].is_set) {
        printf("Required parameter '%s' missing.\n", params->list[i].name);
        exit(-1);
      }
      print_parameter(&params->list[i]);
    }
  for (int i = 0; i < params->n; i++)
    if (!params->list[i].required && params->list[i].is_set) print_parameter(&params->list[i]);
  putchar('\n');
}
