/*
 * Test infrastructure only (parity tests and bench.py's baseline legs): the
 * reference's own refinement objective, exported for comparison.
 *
 * This file holds no reference code.  It includes the reference tree's
 * LaueMatchingHeaders.h where it lies (oracle/Makefile, target ref-objective,
 * compiles it with the reference's C flags into _ref/libref_objective.so),
 * defines the globals that header declares (as LaueMatchingCPU.c:14-22 does)
 * and wraps, with plain pointer arguments:
 *   OrientMat2Euler       LaueMatchingHeaders.h:313-332
 *   prefilterHKLs         :513-561
 *   problem_function      :640-694 (calcOverlapFiltered :564-636, calcV :371-377)
 */
#include <stdlib.h>

#include "LaueMatchingHeaders.h"

double tol_LatC[6];
double tol_c_over_a;
double c_over_a_orig;
int sg_num;
double cellVol;
double phiVol;
int nSym;
double Symm[24][4];
int useBobyqa = 1;

/* The crystal globals as LaueMatchingCPU.c's parameter reader and main set
 * them (tol_latc already zeroed by the caller when tol_c_over_a != 0). */
void refobj_set_crystal(const double latc[6], const double tol_latc[6], double tca, int sg) {
  double lat[6];
  for (int i = 0; i < 6; i++) {
    lat[i] = latc[i];
    tol_LatC[i] = tol_latc[i];
  }
  tol_c_over_a = tca;
  sg_num = sg;
  c_over_a_orig = lat[2] / lat[0];
  calcV(lat);
}

void refobj_euler(const double om[9], double euler[3]) {
  double m[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) m[i][j] = om[i * 3 + j];
  OrientMat2Euler(m, euler);
}

void refobj_euler_to_om(const double euler[3], double om[9]) {
  double e[3] = {euler[0], euler[1], euler[2]}, m[3][3];
  Euler2OrientMat(e, m);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) om[i * 3 + j] = m[i][j];
}

static void to33(const double *a, double m[3][3]) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) m[i][j] = a[i * 3 + j];
}

int refobj_prefilter(int *hkls, int nhkls, const double euler[3], const double recip[9], int W,
                     int H, const double rt[9], const double p[3], double pxX, double pxY,
                     double Elo, double Ehi, int *valid) {
  double e[3] = {euler[0], euler[1], euler[2]}, rc[3][3], rtm[3][3];
  double pa[3] = {p[0], p[1], p[2]};
  to33(recip, rc);
  to33(rt, rtm);
  return prefilterHKLs(hkls, nhkls, e, rc, W, H, rtm, pa, pxX, pxY, Elo, Ehi, valid, nhkls);
}

double refobj_problem(unsigned n, const double *x, float *image, int *hkls, int nhkls, int W,
                      int H, const double latc[6], const double recip[9], int max_spots,
                      const double rt[9], const double p[3], double pxX, double pxY, double Elo,
                      double Ehi, int *valid, int nvalid) {
  struct dataFit f;
  memset(&f, 0, sizeof(f));
  f.image = image;
  f.hkls = hkls;
  f.nhkls = nhkls;
  f.nrPxX = W;
  f.nrPxY = H;
  for (int i = 0; i < 6; i++) f.LatCOrig[i] = latc[i];
  to33(recip, f.recip);
  to33(rt, f.rotTranspose);
  for (int i = 0; i < 3; i++) f.pArr[i] = p[i];
  f.pxX = pxX;
  f.pxY = pxY;
  f.Elo = Elo;
  f.Ehi = Ehi;
  f.maxNrSpots = max_spots;
  f.validHKLIdx = valid;
  f.nValidHKL = nvalid;
  f.outArrThis = (double *)calloc(3 * (size_t)max_spots, sizeof(double));
  const double r = problem_function(n, x, NULL, &f);
  free(f.outArrThis);
  return r;
}
