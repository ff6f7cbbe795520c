// C interface of the CPU restatement (test infrastructure; see oracle.cpp).
#pragma once
#include "oneflow_b200.h"
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
void *oro_create(const ofg_params *p);
void oro_destroy(void *h);
int oro_set_mesh(void *h, int nn, const double *x, const double *y, const double *z, int nf, const int *fnc,
                 const int *fn, const int *l, const int *r, int nc, int nb, const int *bct, const double *wd);
int oro_init_flowfield(void *h);
int oro_step(void *h, int n);
int oro_task(void *h, const char *name);
int64_t oro_field(void *h, const char *name, double *out);
int oro_set_q(void *h, const double *qin);
long oro_outer_steps(void *h);
int oro_forces(void *h, double aref, double *out);   /* out[13], see Oracle::forces */
void *oro_ins_create(void *h);
void oro_ins_destroy(void *s);
int oro_ins_set_wall(void *s, const double *uvw);
int oro_ins_init(void *s);
int oro_ins_run(void *s, int maxIter);
int oro_ins_stats(void *s, double *out);             /* out[13] */
int64_t oro_ins_field(void *s, const char *name, double *out);
#ifdef __cplusplus
}
#endif
