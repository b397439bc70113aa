/*
 * Test infrastructure only: a minimal stand-in for <nlopt.h> so that the
 * reference's LaueMatchingCPU.c compiles here without the NLopt library
 * (NLopt is not installed and cannot be downloaded on this machine).
 *
 * The reference calls NLopt only from its orientation refinement
 * (LaueMatchingHeaders.h FitOrientation, lines 769-778).  This stand-in
 * "optimises" by evaluating the objective once at the start point and
 * returning that point unchanged, so the refinement step is an identity.
 * The compare and forward-simulation arithmetic never touch NLopt.
 *
 * The product's own post-stage offers the same evaluate-once mode, which is
 * what makes solutions.txt comparable byte for byte between the two.
 */
#ifndef LMB_ORACLE_NLOPT_STUB_H
#define LMB_ORACLE_NLOPT_STUB_H

#include <stdlib.h>

typedef enum { NLOPT_LN_BOBYQA = 34, NLOPT_LN_NELDERMEAD = 28 } nlopt_algorithm;
typedef enum { NLOPT_FAILURE = -1, NLOPT_SUCCESS = 1 } nlopt_result;
typedef double (*nlopt_func)(unsigned n, const double *x, double *grad,
                             void *data);

struct lmb_stub_nlopt_s {
  unsigned n;
  nlopt_func f;
  void *data;
};
typedef struct lmb_stub_nlopt_s *nlopt_opt;

static inline nlopt_opt nlopt_create(nlopt_algorithm a, unsigned n) {
  (void)a;
  nlopt_opt o = (nlopt_opt)calloc(1, sizeof(*o));
  if (o) o->n = n;
  return o;
}
static inline void nlopt_destroy(nlopt_opt o) { free(o); }
static inline nlopt_result nlopt_set_lower_bounds(nlopt_opt o, const double *lb) {
  (void)o; (void)lb; return NLOPT_SUCCESS;
}
static inline nlopt_result nlopt_set_upper_bounds(nlopt_opt o, const double *ub) {
  (void)o; (void)ub; return NLOPT_SUCCESS;
}
static inline nlopt_result nlopt_set_min_objective(nlopt_opt o, nlopt_func f,
                                                   void *data) {
  o->f = f; o->data = data; return NLOPT_SUCCESS;
}
static inline nlopt_result nlopt_set_ftol_rel(nlopt_opt o, double t) {
  (void)o; (void)t; return NLOPT_SUCCESS;
}
static inline nlopt_result nlopt_set_xtol_rel(nlopt_opt o, double t) {
  (void)o; (void)t; return NLOPT_SUCCESS;
}
static inline nlopt_result nlopt_set_maxeval(nlopt_opt o, int m) {
  (void)o; (void)m; return NLOPT_SUCCESS;
}
/* One evaluation at x; x is left unchanged. */
static inline nlopt_result nlopt_optimize(nlopt_opt o, double *x, double *minf) {
  if (!o || !o->f) return NLOPT_FAILURE;
  *minf = o->f(o->n, x, NULL, o->data);
  return NLOPT_SUCCESS;
}

#endif
