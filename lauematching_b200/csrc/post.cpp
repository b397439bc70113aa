// Host post-stage after the compare pass: duplicate merge, orientation
// refinement objective, solutions/spots text.
//
// Restates, in the reference's operation order (FP64, glibc libm, printf):
//   mergeDuplicateOrientations  LaueMatchingHeaders.h:969-1065
//   fitAndWriteOrientations     LaueMatchingHeaders.h:1072-1153
//   (prefilterHKLs :513-561, calcOverlapFiltered :564-636, problem_function
//    :640-694, FitOrientation :696-801, writeCalcOverlap :805-947, and the
//    quaternion / Euler / symmetry utilities :147-347).
// The symmetry quaternion tables must hold the reference's values (5-decimal
// roundings) in the reference's order, because the fundamental-region
// reduction keeps the first maximum; they are data, listed below.
//
// Refinement.  The reference refines each grain with NLopt (BOBYQA or
// Nelder-Mead, 200 evaluations).  NLopt is not available here, so the
// optimiser of this stage evaluates the objective once at the start point and
// returns it unchanged; the reference built against the same evaluate-once
// NLopt stand-in writes byte-identical files.
//
// Output order.  The reference writes grains from an OpenMP loop inside a
// critical section, so its line order depends on thread timing; here grains
// are evaluated in parallel and written in grain order (the reference's order
// with one thread).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lmb200.h"
#include "merge.h"
#include "refine.h"

namespace lmb {
void set_error(const char *fmt, ...);
}

namespace {

constexpr double kDeg2Rad = 0.0174532925199433;  // LaueMatchingHeaders.h:32
constexpr double kRad2Deg = 57.2957795130823;    // :33
constexpr double kEps = 1E-12;                    // :42
constexpr double kHc = 1.2398419739;              // :41
constexpr int kMergeMax = 50000;                  // :953
constexpr int kFitMaxEval = 200;                  // nlopt_set_maxeval, :775
// From this many grains on, a post-stage with a device refines on it (fewer:
// host threads are as fast, the per-round launch latency dominates).
constexpr int kDeviceRefineMin = 2048;

// Symmetry quaternions (w, x, y, z) per crystal system, LaueMatchingHeaders.h:83-145.
const double kTric[1][4] = {{1, 0, 0, 0}};
const double kMono[2][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}};
const double kOrth[4][4] = {{1, 0, 0, 0}, {1, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};
const double kTetr[8][4] = {{1, 0, 0, 0},          {0.70711, 0, 0, 0.70711}, {0, 0, 0, 1},
                            {0.70711, -0.0, -0.0, -0.70711}, {0, 1, 0, 0},   {0, 0, 1, 0},
                            {0, 0.70711, 0.70711, 0},        {0, -0.70711, 0.70711, 0}};
const double kTrig[6][4] = {{1, 0, 0, 0},          {0, 0.86603, -0.5, 0}, {0.5, 0, 0, 0.86603},
                            {0, 0, 1, 0},          {0.5, -0.0, -0.0, -0.86603},
                            {0, 0.86603, 0.5, 0}};
const double kHexa[12][4] = {{1, 0, 0, 0},           {0.86603, 0, 0, 0.5},
                             {0.5, 0, 0, 0.86603},   {0, 0, 0, 1},
                             {0.5, -0.0, -0.0, -0.86603}, {0.86603, -0.0, -0.0, -0.5},
                             {0, 1, 0, 0},           {0, 0.86603, 0.5, 0},
                             {0, 0.5, 0.86603, 0},   {0, 0, 1, 0},
                             {0, -0.5, 0.86603, 0},  {0, -0.86603, 0.5, 0}};
const double kCubi[24][4] = {
    {1, 0, 0, 0},          {0.70711, 0.70711, 0, 0},  {0, 1, 0, 0},
    {0.70711, -0.70711, 0, 0}, {0.70711, 0, 0.70711, 0}, {0, 0, 1, 0},
    {0.70711, 0, -0.70711, 0}, {0.70711, 0, 0, 0.70711}, {0, 0, 0, 1},
    {0.70711, 0, 0, -0.70711}, {0.5, 0.5, 0.5, 0.5},      {0.5, -0.5, -0.5, -0.5},
    {0.5, -0.5, 0.5, 0.5},     {0.5, 0.5, -0.5, -0.5},    {0.5, 0.5, -0.5, 0.5},
    {0.5, -0.5, 0.5, -0.5},    {0.5, -0.5, -0.5, 0.5},    {0.5, 0.5, 0.5, -0.5},
    {0, 0.70711, 0.70711, 0},  {0, -0.70711, 0.70711, 0}, {0, 0.70711, 0, 0.70711},
    {0, 0.70711, 0, -0.70711}, {0, 0, 0.70711, 0.70711}, {0, 0, 0.70711, -0.70711}};

struct Sym {
  int n = 1;
  double q[24][4];
};

Sym make_sym(int sg) {  // MakeSymmetries, :180-219
  Sym s;
  const double(*t)[4];
  if (sg <= 2) {
    s.n = 1, t = kTric;
  } else if (sg <= 15) {
    s.n = 2, t = kMono;
  } else if (sg <= 74) {
    s.n = 4, t = kOrth;
  } else if (sg <= 142) {
    s.n = 8, t = kTetr;
  } else if (sg <= 167) {
    s.n = 6, t = kTrig;
  } else if (sg <= 194) {
    s.n = 12, t = kHexa;
  } else {
    s.n = 24, t = kCubi;
  }
  for (int i = 0; i < s.n; i++)
    for (int j = 0; j < 4; j++) s.q[i][j] = t[i][j];
  return s;
}

inline double length3(double x, double y, double z) { return std::sqrt(x * x + y * y + z * z); }
inline double zero_out(double v) { return (std::fabs(v) < kEps) ? 0 : v; }

void normalize4(double q[4]) {
  const double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  q[0] /= n;
  q[1] /= n;
  q[2] /= n;
  q[3] /= n;
}

// Quaternion product as LaueMatchingHeaders.h:166-178 (w>=0 hemisphere, normalised).
void qmul(const double q[4], const double r[4], double Q[4]) {
  Q[0] = r[0] * q[0] - r[1] * q[1] - r[2] * q[2] - r[3] * q[3];
  Q[1] = r[1] * q[0] + r[0] * q[1] + r[3] * q[2] - r[2] * q[3];
  Q[2] = r[2] * q[0] + r[0] * q[2] + r[1] * q[3] - r[3] * q[1];
  Q[3] = r[3] * q[0] + r[0] * q[3] + r[2] * q[1] - r[1] * q[2];
  if (Q[0] < 0) {
    Q[0] = -Q[0];
    Q[1] = -Q[1];
    Q[2] = -Q[2];
    Q[3] = -Q[3];
  }
  normalize4(Q);
}

void to_fundamental(const Sym &S, const double in[4], double out[4]) {  // :221-245
  int best = 0;
  double best_w = -10000, cand[24][4];
  for (int i = 0; i < S.n; i++) {
    qmul(in, S.q[i], cand[i]);
    if (best_w < cand[i][0]) {
      best_w = cand[i][0];
      best = i;
    }
  }
  for (int j = 0; j < 4; j++) out[j] = cand[best][j];
  normalize4(out);
}

double misorientation_deg(const Sym &S, const double a[4], const double b[4]) {  // :247-260
  double af[4], bf[4], ai[4], p[4], m[4];
  to_fundamental(S, a, af);
  to_fundamental(S, b, bf);
  ai[0] = -af[0];
  ai[1] = af[1];
  ai[2] = af[2];
  ai[3] = af[3];
  qmul(ai, bf, p);
  to_fundamental(S, p, m);
  if (m[0] > 1) m[0] = 1;
  return 2 * (std::acos(m[0])) * kRad2Deg;
}

// ---- the duplicate merge on the device (merge.cu) ------------------------------
constexpr int64_t kDeviceMergeMin = 1024;  // fewer candidates: the host loop is quick

struct DecideCtx {
  const Sym *S;
  const double *quat;
  double max_angle;
};

// The host's own comparison for a pair the device left undecided (l > g, the
// reference's argument order).
bool decide_pair(void *ctx, int64_t l, int64_t g) {
  const DecideCtx *c = static_cast<const DecideCtx *>(ctx);
  return (float)misorientation_deg(*c->S, &c->quat[l * 4], &c->quat[g * 4]) <= c->max_angle;
}

int merge_on_gpu(int device, double band, const Sym &S, double max_angle,
                 const std::vector<double> &quat,
                 const std::vector<uint64_t> &rows, const std::vector<double> &sc,
                 std::vector<int> *dcount, std::vector<int> *best_row,
                 std::vector<double> *best_score) {
  const int64_t n = (int64_t)rows.size();
  lmb::MergeHost h{};
  h.device = device;
  h.n = n;
  h.quat = quat.data();
  h.score = sc.data();
  h.nsym = S.n;
  for (int i = 0; i < 24; i++)
    for (int j = 0; j < 4; j++) h.sym[i][j] = S.q[i][j];
  h.max_angle = max_angle;
  h.rad2deg = kRad2Deg;
  // (float)x <= max_angle changes value where x crosses the midpoint of the
  // two floats around max_angle; pairs whose device angle is within a band far
  // wider than the device/host acos difference of it are decided on the host
  float f1 = (float)max_angle;
  if ((double)f1 > max_angle) f1 = std::nextafterf(f1, -INFINITY);
  const float f2 = std::nextafterf(f1, INFINITY);
  h.mid = ((double)f1 + (double)f2) / 2;
  h.window = std::isfinite(h.mid) ? std::fmax(1e-12 * std::fmax(1.0, std::fabs(h.mid)), band)
                                   : -1.0;
  DecideCtx ctx{&S, quat.data(), max_angle};
  h.decide = decide_pair;
  h.ctx = &ctx;
  std::vector<int64_t> bi((size_t)n);
  std::vector<int32_t> cnt((size_t)n);
  int32_t nc = 0;
  std::vector<std::pair<uint32_t, uint32_t>> unsure;
  bool overflow = false;
  const int rc = lmb::merge_device_run(h, &nc, bi.data(), cnt.data(), &unsure, &overflow);
  if (rc) return rc;
  if (overflow) {
    lmb::set_error("device merge: too many candidate pairs at the MaxAngle boundary");
    return LMB_ERR_OVERFLOW;
  }
  for (int32_t c = 0; c < nc; c++) {
    dcount->push_back(cnt[c]);
    best_row->push_back((int)rows[bi[c]]);
    best_score->push_back(sc[bi[c]]);
  }
  return LMB_OK;
}

void om_to_quat(const double m[9], double q[4]) {  // OrientMat2Quat, :262-302
  const double tr = m[0] + m[4] + m[8];
  if (tr > 0) {
    const double s = 0.5 / std::sqrt(tr + 1.0);
    q[0] = 0.25 / s;
    q[1] = (m[7] - m[5]) * s;
    q[2] = (m[2] - m[6]) * s;
    q[3] = (m[3] - m[1]) * s;
  } else if (m[0] > m[4] && m[0] > m[8]) {
    const double s = 2.0 * std::sqrt(1.0 + m[0] - m[4] - m[8]);
    q[0] = (m[7] - m[5]) / s;
    q[1] = 0.25 * s;
    q[2] = (m[1] + m[3]) / s;
    q[3] = (m[2] + m[6]) / s;
  } else if (m[4] > m[8]) {
    const double s = 2.0 * std::sqrt(1.0 + m[4] - m[0] - m[8]);
    q[0] = (m[2] - m[6]) / s;
    q[1] = (m[1] + m[3]) / s;
    q[2] = 0.25 * s;
    q[3] = (m[5] + m[7]) / s;
  } else {
    const double s = 2.0 * std::sqrt(1.0 + m[8] - m[0] - m[4]);
    q[0] = (m[3] - m[1]) / s;
    q[1] = (m[2] + m[6]) / s;
    q[2] = (m[5] + m[7]) / s;
    q[3] = 0.25 * s;
  }
  if (q[0] < 0) {
    q[0] = -q[0];
    q[1] = -q[1];
    q[2] = -q[2];
    q[3] = -q[3];
  }
  normalize4(q);
}

inline double angle_from_sc(double s, double c) {  // sin_cos_to_angle, :149-151
  return (s >= 0.0) ? std::acos(c) : 2.0 * M_PI - std::acos(c);
}

void om_to_euler(const double m[3][3], double e[3]) {  // OrientMat2Euler, :313-332
  double psi, phi, theta;
  if (std::fabs(m[2][2] - 1.0) < kEps)
    phi = 0;
  else
    phi = std::acos(m[2][2]);
  const double sph = std::sin(phi);
  if (std::fabs(sph) < kEps) {
    psi = 0.0;
    theta = (std::fabs(m[2][2] - 1.0) < kEps) ? angle_from_sc(m[1][0], m[0][0])
                                               : angle_from_sc(-m[1][0], m[0][0]);
  } else {
    psi = (std::fabs(-m[1][2] / sph) <= 1.0) ? angle_from_sc(m[0][2] / sph, -m[1][2] / sph)
                                             : angle_from_sc(m[0][2] / sph, 1);
    theta = (std::fabs(m[2][1] / sph) <= 1.0) ? angle_from_sc(m[2][0] / sph, m[2][1] / sph)
                                              : angle_from_sc(m[2][0] / sph, 1);
  }
  e[0] = psi;
  e[1] = phi;
  e[2] = theta;
}

void euler_to_om(const double e[3], double m[3][3]) {  // Euler2OrientMat, :334-347
  const double psi = e[0], phi = e[1], theta = e[2];
  const double cps = std::cos(psi), cph = std::cos(phi), cth = std::cos(theta);
  const double sps = std::sin(psi), sph = std::sin(phi), sth = std::sin(theta);
  m[0][0] = cth * cps - sth * cph * sps;
  m[0][1] = -cth * cph * sps - sth * cps;
  m[0][2] = sph * sps;
  m[1][0] = cth * sps + sth * cph * cps;
  m[1][1] = cth * cph * cps - sth * sps;
  m[1][2] = -sph * cps;
  m[2][0] = sth * sph;
  m[2][1] = cth * sph;
  m[2][2] = cph;
}

void mat33(const double m[3][3], const double n[3][3], double r[3][3]) {  // :349-357
  for (int i = 0; i < 3; i++) {
    r[i][0] = m[i][0] * n[0][0] + m[i][1] * n[1][0] + m[i][2] * n[2][0];
    r[i][1] = m[i][0] * n[0][1] + m[i][1] * n[1][1] + m[i][2] * n[2][1];
    r[i][2] = m[i][0] * n[0][2] + m[i][1] * n[1][2] + m[i][2] * n[2][2];
  }
}

void matvec(const double m[3][3], const double v[3], double r[3]) {  // :361-369
  r[0] = 0;
  r[1] = 0;
  r[2] = 0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) r[i] += m[i][j] * v[j];
}

void recip_of(const double lat[6], int sg, double recip[3][3]) {  // calcRecipArray, :379-436
  const double a = lat[0], b = lat[1], c = lat[2];
  const bool rh = sg == 146 || sg == 148 || sg == 155 || sg == 160 || sg == 161 || sg == 166 ||
                  sg == 167;
  const double ca = std::cos(lat[3] * kDeg2Rad), cb = std::cos(lat[4] * kDeg2Rad);
  const double cg = std::cos(lat[5] * kDeg2Rad), sgm = std::sin(lat[5] * kDeg2Rad);
  const double phi = std::sqrt(1.0 - ca * ca - cb * cb - cg * cg + 2 * ca * cb * cg);
  const double pv = (2 * M_PI) / (a * b * c * phi);
  double a0, a1, a2, b0, b1, b2, c0, c1, c2;
  if (!rh) {
    a0 = zero_out(a), a1 = zero_out(0.0), a2 = zero_out(0.0);
    b0 = b * cg, b1 = zero_out(b * sgm), b2 = zero_out(0.0);
    c0 = c * cb, c1 = c * (ca - cb * cg) / sgm, c2 = zero_out(c * phi / sgm);
  } else {
    const double p = std::sqrt(1.0 + 2 * ca), q = std::sqrt(1.0 - ca);
    const double pmq = (a / 3.0) * (p - q), p2q = (a / 3.0) * (p + 2 * q);
    a0 = p2q, a1 = pmq, a2 = pmq, b0 = pmq, b1 = p2q, b2 = pmq, c0 = pmq, c1 = pmq, c2 = p2q;
  }
  recip[0][0] = zero_out((b1 * c2 - b2 * c1) * pv);
  recip[1][0] = zero_out((b2 * c0 - b0 * c2) * pv);
  recip[2][0] = zero_out((b0 * c1 - b1 * c0) * pv);
  recip[0][1] = zero_out((c1 * a2 - c2 * a1) * pv);
  recip[1][1] = zero_out((c2 * a0 - c0 * a2) * pv);
  recip[2][1] = zero_out((c0 * a1 - c1 * a0) * pv);
  recip[0][2] = zero_out((a1 * b2 - a2 * b1) * pv);
  recip[1][2] = zero_out((a2 * b0 - a0 * b2) * pv);
  recip[2][2] = zero_out((a0 * b1 - a1 * b0) * pv);
}

struct Detector {
  double rt[3][3];
  double p[3];
  double px_x, px_y, elo, ehi;
  int W, H;
};

// One reflection through the detector model (steps shared by prefilterHKLs,
// calcOverlapFiltered and writeCalcOverlap).  Returns false when rejected;
// px/py are the unrounded pixel coordinates.
inline bool project(const double OM[3][3], const int *hkl, const Detector &d, double qhat[3],
                    double &px, double &py, double &qlen) {
  const double h[3] = {(double)hkl[0], (double)hkl[1], (double)hkl[2]};
  double q[3];
  matvec(OM, h, q);
  qlen = length3(q[0], q[1], q[2]);
  if (qlen == 0) return false;
  qhat[0] = q[0] / qlen;
  qhat[1] = q[1] / qlen;
  qhat[2] = q[2] / qlen;
  const double dot = qhat[2];
  const double kf[3] = {0 - 2 * dot * qhat[0], 0 - 2 * dot * qhat[1], 1.0 - 2 * dot * qhat[2]};
  double xyz[3];
  matvec(d.rt, kf, xyz);
  if (xyz[2] <= 0) return false;
  const double x = xyz[0] * d.p[2] / xyz[2];
  const double y = xyz[1] * d.p[2] / xyz[2];
  const double xp = x - d.p[0], yp = y - d.p[1];
  px = (xp / d.px_x) + (0.5 * (d.W - 1));
  if (px < 0 || px > (d.W - 1)) return false;
  py = (yp / d.px_y) + (0.5 * (d.H - 1));
  if (py < 0 || py > (d.H - 1)) return false;
  const double sin_th = -qhat[2];
  const double e = kHc * qlen / (4 * M_PI * sin_th);
  if (e < d.elo || e > d.ehi) return false;
  return true;
}

// de-duplication of refinement spots by scattering direction (:487-495)
inline bool seen_qhat(const std::vector<double> &acc, int n, const double qh[3]) {
  for (int i = 0; i < n; i++)
    if ((std::fabs(qh[0] - acc[3 * i + 0]) * 100000 < 0.1) &&
        (std::fabs(qh[1] - acc[3 * i + 1]) * 100000 < 0.1) &&
        (std::fabs(qh[2] - acc[3 * i + 2]) * 100000 < 0.1))
      return true;
  return false;
}

struct Crystal {
  double lat[6];
  int sg;
  double tol_latc[6];
  double tol_c_over_a;
  double c_over_a_orig;
  double cell_vol, phi_vol;  // calcV of the params lattice, :371-377
};

// The matrix OM . recip of the refinement at x (problem_function :651-673 and
// calcOverlapFiltered :567-570): the lattice of x when n > 3, else recip0.
void point_matrix(unsigned n, const double *x, const Crystal &cr, const double recip0[3][3],
                  double OM[3][3]) {
  double recip[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) recip[i][j] = recip0[i][j];
  if (n > 3) {
    double lat[6];
    int c = 0;
    for (int i = 0; i < 6; i++) {
      if (cr.tol_latc[i] != 0)
        lat[i] = x[3 + c++];
      else
        lat[i] = cr.lat[i];
    }
    if (cr.tol_c_over_a != 0) {
      const double a_new = std::cbrt(cr.cell_vol / (x[3] * cr.phi_vol));
      lat[0] = a_new;
      lat[1] = a_new;
      lat[2] = x[3] * a_new;
    }
    recip_of(lat, cr.sg, recip);
  }
  const double eul[3] = {x[0], x[1], x[2]};
  double OMt[3][3];
  euler_to_om(eul, OMt);
  mat33(OMt, recip, OM);
}

// calcOverlapFiltered (:564-636) at the matrix OM, with problem_function's
// sign: -(nrPos * sqrt(sum of the kept spots' positive pixels)).
double overlap_at(const double OM[3][3], const Detector &d, const float *img,
                  const int32_t *hkls, const int *valid, int nvalid, int max_spots,
                  std::vector<double> &acc) {
  double result = 0;
  int nspot = 0, npos = 0;
  for (int vi = 0; vi < nvalid; vi++) {
    double qh[3], px, py, ql;
    if (!project(OM, hkls + 3 * valid[vi], d, qh, px, py, ql)) continue;
    if (seen_qhat(acc, nspot, qh)) continue;
    acc[3 * nspot + 0] = qh[0];
    acc[3 * nspot + 1] = qh[1];
    acc[3 * nspot + 2] = qh[2];
    const float v = img[(size_t)((size_t)py * d.W + (size_t)px)];
    if (v > 0) {
      result += v;
      npos++;
    }
    if (++nspot == max_spots) break;
  }
  return -(npos * std::sqrt(result));
}

// Objective of the refinement at x (problem_function, :640-694 with
// calcOverlapFiltered :564-636).
double objective(unsigned n, const double *x, const Crystal &cr, const double recip0[3][3],
                 const Detector &d, const float *img, const int32_t *hkls, const int *valid,
                 int nvalid, int max_spots, std::vector<double> &acc) {
  double OM[3][3];
  point_matrix(n, x, cr, recip0, OM);
  return overlap_at(OM, d, img, hkls, valid, nvalid, max_spots, acc);
}

// The crystal of the refinement (tol_c_over_a != 0 zeroes tol_LatC, as the
// reference's parameter reader does) with calcV's volumes (:371-377).
Crystal make_crystal(const lmb_post_params *pp) {
  Crystal cr;
  for (int i = 0; i < 6; i++) {
    cr.lat[i] = pp->lattice[i];
    cr.tol_latc[i] = pp->tol_c_over_a != 0 ? 0.0 : pp->tol_latc[i];
  }
  cr.sg = pp->space_group;
  cr.tol_c_over_a = pp->tol_c_over_a;
  cr.c_over_a_orig = cr.lat[2] / cr.lat[0];
  const double ca = std::cos(cr.lat[3] * kDeg2Rad), cb = std::cos(cr.lat[4] * kDeg2Rad);
  const double cg = std::cos(cr.lat[5] * kDeg2Rad);
  cr.phi_vol = std::sqrt(1.0 - ca * ca - cb * cb - cg * cg + 2 * ca * cb * cg);
  cr.cell_vol = cr.lat[0] * cr.lat[1] * cr.lat[2] * cr.phi_vol;
  return cr;
}

void make_detector(const lmb_geometry *geo, Detector *d, double recip[3][3]) {
  for (int i = 0; i < 3; i++) {
    d->p[i] = geo->p[i];
    for (int j = 0; j < 3; j++) {
      recip[i][j] = geo->recip[i * 3 + j];
      d->rt[i][j] = geo->rot_t[i * 3 + j];
    }
  }
  d->px_x = geo->px_x;
  d->px_y = geo->px_y;
  d->elo = geo->elo;
  d->ehi = geo->ehi;
  d->W = geo->nr_px_x;
  d->H = geo->nr_px_y;
}

// FitOrientation's dimension count (:705-716): 3 Euler angles plus the
// lattice entries with a tolerance, or 4 with a c/a tolerance.
unsigned fit_dims(const Crystal &cr) {
  int nz = 0;
  for (int i = 0; i < 6; i++)
    if (cr.tol_latc[i] != 0) nz++;
  unsigned n = 3 + nz;
  if (cr.tol_c_over_a != 0) n = 4;
  return n;
}

struct GrainOut {
  bool keep = false;
  std::string sol, spots;
};

// Append printf-formatted text.
void appendf(std::string &s, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
void appendf(std::string &s, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  const int n = vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (n < (int)sizeof(buf)) {
    s.append(buf, n > 0 ? n : 0);
  } else {
    std::vector<char> big(n + 1);
    va_start(ap, fmt);
    vsnprintf(big.data(), big.size(), fmt, ap);
    va_end(ap);
    s.append(big.data(), n);
  }
}

// mergeDuplicateOrientations (:969-1065) after the cap, on candidates rows/sc
// in input order: clusters (count, kept row, kept score).  device >= 0 and at
// least kDeviceMergeMin candidates: the pair matrix and greedy pass on that
// CUDA device (band > 0 widens the band of pairs decided on the host);
// otherwise the host loop.
int merge_clusters(int device, double band, const Sym &S, double max_angle,
                   const double *orients, const std::vector<uint64_t> &rows,
                   const std::vector<double> &sc, int nthreads, std::vector<int> *dcount,
                   std::vector<int> *best_row, std::vector<double> *best_score) {
  const int64_t nr = (int64_t)rows.size();
  std::vector<double> quat((size_t)nr * 4);
#pragma omp parallel for num_threads(nthreads)
  for (int64_t i = 0; i < nr; i++) om_to_quat(orients + rows[i] * 9, &quat[i * 4]);
  if (device >= 0 && nr >= kDeviceMergeMin)
    return merge_on_gpu(device, band, S, max_angle, quat, rows, sc, dcount, best_row, best_score);
  std::vector<float> miso((size_t)nr * (nr > 0 ? nr - 1 : 0) / 2);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic)
  for (int64_t i = 1; i < nr; i++)
    for (int64_t j = 0; j < i; j++)
      miso[(size_t)i * (i - 1) / 2 + j] = (float)misorientation_deg(S, &quat[i * 4], &quat[j * 4]);
  std::vector<int> done(nr, 0);
  for (int64_t g = 0; g < nr; g++) {
    if (done[g]) continue;
    done[g] = 1;
    int bs = (int)rows[g];
    double bsc = sc[g];
    for (int64_t l = g + 1; l < nr; l++) {
      if (done[l] > 0) continue;
      if (miso[(size_t)l * (l - 1) / 2 + g] <= max_angle) {
        done[l] = 1;
        done[g]++;
        if (sc[l] > bsc) {
          bsc = sc[l];
          bs = (int)rows[l];
        }
      }
    }
    dcount->push_back(done[g]);
    best_row->push_back(bs);
    best_score->push_back(bsc);
  }
  return LMB_OK;
}

}  // namespace

namespace {

// Refinement handles of the post-stage, kept between calls: a handle on a
// device holds device buffers, and creating and freeing those per image would
// put cudaMalloc/cudaFree (and cudaFree's device-wide synchronisation) into
// every frame of the streaming daemon's writer threads.  A call checks out an
// idle handle made for the same device, geometry, parameters and HKL list (or
// creates one) and returns it afterwards; concurrent calls each hold their
// own.  At most kRefinePoolIdle idle handles are kept; the pool lives until
// the process exits.
constexpr size_t kRefinePoolIdle = 8;

struct RefineKey {
  int device = -1;
  lmb_geometry geo{};
  lmb_post_params pp{};
  std::vector<int32_t> hkls;
  bool operator==(const RefineKey &o) const {
    return device == o.device && memcmp(&geo, &o.geo, sizeof(geo)) == 0 &&
           memcmp(&pp, &o.pp, sizeof(pp)) == 0 && hkls == o.hkls;
  }
};

struct RefinePool {
  std::mutex mu;
  std::vector<std::pair<RefineKey, lmb_refine *>> idle;
};

RefinePool &refine_pool() {
  static RefinePool *pool = new RefinePool();  // never destroyed: no CUDA calls at exit
  return *pool;
}

int refine_checkout(int device, const lmb_geometry *geo, const lmb_post_params *pp,
                    const int32_t *hkls, int32_t nh, RefineKey *key, lmb_refine **out) {
  key->device = device;
  memcpy(&key->geo, geo, sizeof(lmb_geometry));
  memcpy(&key->pp, pp, sizeof(lmb_post_params));
  key->hkls.assign(hkls, hkls + 3 * (size_t)nh);
  {
    RefinePool &pool = refine_pool();
    std::lock_guard<std::mutex> lk(pool.mu);
    for (size_t i = 0; i < pool.idle.size(); i++)
      if (pool.idle[i].first == *key) {
        *out = pool.idle[i].second;
        pool.idle.erase(pool.idle.begin() + (ptrdiff_t)i);
        return LMB_OK;
      }
  }
  return lmb_refine_create(device, geo, pp, hkls, nh, out);
}

void refine_return(RefineKey &&key, lmb_refine *rf, bool reusable) {
  if (!rf) return;
  if (reusable) {
    RefinePool &pool = refine_pool();
    std::lock_guard<std::mutex> lk(pool.mu);
    if (pool.idle.size() < kRefinePoolIdle) {
      pool.idle.emplace_back(std::move(key), rf);
      return;
    }
  }
  lmb_refine_destroy(rf);
}

// What the calling thread's last lmb_post_process refined, and where.
struct PostRefineStats {
  int32_t device = -2;  // -2: no refinement; -1: host threads; else the device
  int64_t points = 0;
  int32_t rounds = 0;
  float kernel_ms = 0.0f;
};
thread_local PostRefineStats t_post_refine;

}  // namespace

extern "C" int lmb_post_last_refine_stats(int32_t *device, int64_t *points, int32_t *rounds,
                                          float *kernel_ms) {
  if (device) *device = t_post_refine.device;
  if (points) *points = t_post_refine.points;
  if (rounds) *rounds = t_post_refine.rounds;
  if (kernel_ms) *kernel_ms = t_post_refine.kernel_ms;
  return LMB_OK;
}

extern "C" int lmb_post_process(const lmb_geometry *geo, const lmb_post_params *pp,
                                const double *orients, uint64_t n_orients, const uint64_t *ids,
                                const double *scores, int64_t n_results, const float *image,
                                const int32_t *hkls, int32_t nh, lmb_post_output *out) {
  if (!geo || !pp || !out || (!orients && n_orients) || (n_results > 0 && (!ids || !scores)) ||
      !image || (!hkls && nh) || (pp->optimizer != 0 && pp->optimizer != 1)) {
    lmb::set_error("null argument");
    return LMB_ERR_INVALID;
  }
  for (int64_t i = 0; i < n_results; i++)
    if (ids[i] >= n_orients) {
      lmb::set_error("survivor id %llu outside the %llu orientations",
                     (unsigned long long)ids[i], (unsigned long long)n_orients);
      return LMB_ERR_INVALID;
    }
  const int nthreads = pp->num_threads > 0 ? pp->num_threads : 1;
  const Sym S = make_sym(pp->space_group);
  const Crystal cr = make_crystal(pp);
  double recip[3][3];
  Detector d;
  make_detector(geo, &d, recip);
  const int max_spots = 3 * geo->max_nr_spots;  // LaueMatchingCPU.c:740
  const double tol = 3 * kDeg2Rad;                // :739

  // ---- duplicate merge (:969-1065) ---------------------------------------------
  int64_t nr = n_results;
  std::vector<uint64_t> rows(ids, ids + nr);
  std::vector<double> sc(scores, scores + nr);
  const int64_t cap = pp->max_results > 0 ? pp->max_results : kMergeMax;
  if (nr > cap) {
    fprintf(stderr,
            "WARNING: %lld coarse matches exceed merge cap %lld; keeping the top-scored before "
            "clustering.\n",
            (long long)nr, (long long)cap);
    struct SR {
      double score;
      size_t row;
    };
    std::vector<SR> sr(nr);
    for (int64_t i = 0; i < nr; i++) sr[i] = {sc[i], (size_t)rows[i]};
    qsort(sr.data(), (size_t)nr, sizeof(SR), [](const void *a, const void *b) {
      const double x = ((const SR *)a)->score, y = ((const SR *)b)->score;
      return (x < y) - (x > y);
    });
    for (int64_t i = 0; i < cap; i++) {
      sc[i] = sr[i].score;
      rows[i] = sr[i].row;
    }
    nr = cap;
  }
  std::vector<int> dcount, best_row;
  std::vector<double> best_score;
  {
    const int rc = merge_clusters(pp->merge_on_device - 1, 0.0, S, pp->max_angle, orients, rows,
                                  sc, nthreads, &dcount, &best_row, &best_score);
    if (rc) return rc;
  }
  const int nsol = (int)dcount.size();

  // ---- refine + write (:1072-1153) ---------------------------------------------
  // optimizer 1: this library's bounded Nelder-Mead over all grains at once
  // (lmb_refine_fit; its evaluations on the merge's device when there is one
  // and the grains are many, on host threads otherwise; the same fits either
  // way); optimizer 0 (below): evaluate once, as the reference built without
  // NLopt does
  std::vector<double> nm_x, nm_ov;
  t_post_refine = PostRefineStats{};
  if (pp->optimizer == 1 && nsol > 0) {
    lmb_refine *rf = nullptr;
    const int rdev = (pp->merge_on_device > 0 && nsol >= kDeviceRefineMin)
                         ? pp->merge_on_device - 1
                         : -1;
    RefineKey key;
    int rc = refine_checkout(rdev, geo, pp, hkls, nh, &key, &rf);
    std::vector<double> om((size_t)nsol * 9);
    std::vector<int32_t> im((size_t)nsol, 0);
    for (int it = 0; it < nsol; it++)
      memcpy(&om[(size_t)it * 9], orients + (size_t)best_row[it] * 9, 9 * sizeof(double));
    int32_t nd = 0;
    if (!rc) rc = lmb_refine_set_images(rf, &image, 1);
    if (!rc) rc = lmb_refine_set_grains(rf, om.data(), im.data(), nsol, nullptr);
    if (!rc) rc = lmb_refine_dims(rf, &nd);
    if (!rc) {
      nm_x.resize((size_t)nsol * nd);
      nm_ov.resize((size_t)nsol);
      rc = lmb_refine_fit(rf, 1, kFitMaxEval, 0.0, nm_x.data(), nm_ov.data(), nullptr);
    }
    if (!rc) {
      t_post_refine.device = rdev;
      rc = lmb_refine_last_stats(rf, &t_post_refine.points, &t_post_refine.rounds,
                                 &t_post_refine.kernel_ms);
    }
    refine_return(std::move(key), rf, rc == LMB_OK);
    if (rc) return rc;
  }
  std::vector<GrainOut> go(nsol);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic)
  for (int it = 0; it < nsol; it++) {
    double ob[3][3], eb[3], ef[3], of[3][3], q1[4], q2[4];
    const double *m = orients + (size_t)best_row[it] * 9;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) ob[i][j] = m[i * 3 + j];
    om_to_euler(ob, eb);
    // HKLs that project onto the detector at the coarse orientation (:513-561)
    std::vector<int> valid;
    {
      double OMt[3][3], OM[3][3];
      euler_to_om(eb, OMt);
      mat33(OMt, recip, OM);
      for (int h = 0; h < nh; h++) {
        double qh[3], px, py, ql;
        if (project(OM, hkls + 3 * h, d, qh, px, py, ql)) valid.push_back(h);
      }
    }
    // FitOrientation (:696-801) with the evaluate-once optimiser
    const unsigned n = fit_dims(cr);
    std::vector<double> x(n);
    x[0] = eb[0];
    x[1] = eb[1];
    x[2] = eb[2];
    {
      int c = 3;
      for (int i = 0; i < 6; i++)
        if (cr.tol_latc[i] != 0) x[c++] = cr.lat[i];
      if (cr.tol_c_over_a != 0) x[3] = cr.c_over_a_orig;
    }
    (void)tol;  // bounds of the search box (used by lmb_refine_set_grains)
    std::vector<double> acc((size_t)3 * max_spots, 0.0);
    double mv;
    if (pp->optimizer == 1) {
      for (unsigned i = 0; i < n; i++) x[i] = nm_x[(size_t)it * n + i];
      mv = nm_ov[it];
    } else {
      mv = -objective(n, x.data(), cr, recip, d, image, hkls, valid.data(), (int)valid.size(),
                      max_spots, acc);
    }
    for (int i = 0; i < 3; i++) ef[i] = x[i];
    double latf[6];
    {
      int c = 0;
      for (int i = 0; i < 6; i++) latf[i] = (cr.tol_latc[i] != 0) ? x[3 + c++] : cr.lat[i];
      if (cr.tol_c_over_a != 0) {
        const double a_new = std::cbrt(cr.cell_vol / (x[3] * cr.phi_vol));
        latf[0] = a_new;
        latf[1] = a_new;
        latf[2] = x[3] * a_new;
      }
    }
    euler_to_om(ef, of);
    double qb[9], qf[9];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        qb[i * 3 + j] = ob[i][j];
        qf[i * 3 + j] = of[i][j];
      }
    om_to_quat(qb, q1);
    om_to_quat(qf, q2);
    double recf[3][3];
    recip_of(latf, cr.sg, recf);
    // writeCalcOverlap (:805-947): spots of the refined grain on positive pixels
    std::fill(acc.begin(), acc.end(), 0.0);
    double OMt[3][3], OM[3][3];
    euler_to_om(ef, OMt);
    mat33(OMt, recf, OM);
    const int grain_nr = it + 1;
    int nspot = 0, npos = 0;
    std::string spots;
    for (int h = 0; h < nh; h++) {
      double qh[3], px, py, ql;
      if (!project(OM, hkls + 3 * h, d, qh, px, py, ql)) continue;
      if (seen_qhat(acc, nspot, qh)) continue;
      acc[3 * nspot + 0] = qh[0];
      acc[3 * nspot + 1] = qh[1];
      acc[3 * nspot + 2] = qh[2];
      const float v = image[(size_t)((size_t)py * d.W + (size_t)px)];
      if (v > 0) {
        const int *hk = hkls + 3 * h;
        if (pp->image_num > 0)
          appendf(spots, "%d\t%d\t%d\t%d\t%d\t%d\t%5d\t%5d\t%lf\t%lf\t%lf\t%lf\n", pp->image_num,
                  grain_nr, nspot, hk[0], hk[1], hk[2], (int)px, (int)py, qh[0], qh[1], qh[2],
                  (double)v);
        else
          appendf(spots, "%d\t%d\t%d\t%d\t%d\t%5d\t%5d\t%lf\t%lf\t%lf\t%lf\n", grain_nr, nspot,
                  hk[0], hk[1], hk[2], (int)px, (int)py, qh[0], qh[1], qh[2], (double)v);
        npos++;
      }
      if (++nspot == max_spots) break;
    }
    // the reference's spot buffer holds max_spots*256 bytes (snprintf-truncated)
    const size_t cap = (size_t)max_spots * 256;
    if (spots.size() > cap - 1) spots.resize(cap - 1);
    go[it].spots = spots;
    if (npos >= pp->min_nr_spots) {
      const double mis = misorientation_deg(S, q1, q2);
      double OF[3][3];
      mat33(of, recf, OF);
      std::string &s = go[it].sol;
      if (pp->image_num > 0) appendf(s, "%d\t", pp->image_num);
      appendf(s, "%d\t%d\t", it + 1, dcount[it]);
      appendf(s, "%-13.4lf\t", (mv / npos) * (mv / npos));
      appendf(s, "%-13.4lf\t", npos * (mv / npos) * (mv / npos));
      appendf(s, "%-13.4lf\t", mv);
      appendf(s, "%d\t", npos);
      appendf(s, "%d\t", nspot);
      for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++) appendf(s, "%-13.7lf\t\t", OF[k][l]);
      for (int k = 0; k < 6; k++) appendf(s, "%-13.7lf\t\t", latf[k]);
      for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++) appendf(s, "%-13.7lf\t\t", of[k][l]);
      appendf(s, "%-13.4lf\t%-13.7lf\t%d\n", best_score[it], mis, best_row[it]);
      go[it].keep = true;
    }
  }
  std::string sol, spt;
  for (int it = 0; it < nsol; it++) {
    spt += go[it].spots;
    if (go[it].keep) sol += go[it].sol;
  }
  out->n_unique = nsol;
  out->solutions = (char *)malloc(sol.size() + 1);
  out->spots = (char *)malloc(spt.size() + 1);
  if (!out->solutions || !out->spots) {
    free(out->solutions);
    free(out->spots);
    out->solutions = out->spots = nullptr;
    lmb::set_error("out of host memory for the solution text");
    return LMB_ERR_OOM;
  }
  memcpy(out->solutions, sol.c_str(), sol.size() + 1);
  memcpy(out->spots, spt.c_str(), spt.size() + 1);
  out->solutions_len = sol.size();
  out->spots_len = spt.size();
  return LMB_OK;
}

extern "C" int lmb_merge_clusters(int32_t device, int32_t space_group, double max_angle,
                                  double host_band, const double *orients, uint64_t n_orients,
                                  const uint64_t *rows, const double *scores, int64_t n,
                                  int32_t num_threads, int32_t *n_clusters, uint64_t *best_rows,
                                  double *best_scores, int32_t *counts) {
  if ((n > 0 && (!rows || !scores || !orients || !best_rows || !best_scores || !counts)) ||
      !n_clusters || n < 0 || !(host_band >= 0.0)) {
    lmb::set_error("bad argument");
    return LMB_ERR_INVALID;
  }
  for (int64_t i = 0; i < n; i++)
    if (rows[i] >= n_orients) {
      lmb::set_error("row %llu outside the %llu orientations", (unsigned long long)rows[i],
                     (unsigned long long)n_orients);
      return LMB_ERR_INVALID;
    }
  const Sym S = make_sym(space_group);
  std::vector<uint64_t> rv(rows, rows + n);
  std::vector<double> sv(scores, scores + n);
  std::vector<int> dcount, best_row;
  std::vector<double> best_score;
  const int rc = merge_clusters(device, host_band, S, max_angle, orients, rv, sv,
                                num_threads > 0 ? num_threads : 1, &dcount, &best_row,
                                &best_score);
  if (rc) return rc;
  *n_clusters = (int32_t)dcount.size();
  for (size_t c = 0; c < dcount.size(); c++) {
    best_rows[c] = (uint64_t)best_row[c];
    best_scores[c] = best_score[c];
    counts[c] = dcount[c];
  }
  return LMB_OK;
}

extern "C" void lmb_post_free(lmb_post_output *out) {
  if (!out) return;
  free(out->solutions);
  free(out->spots);
  out->solutions = out->spots = nullptr;
  out->solutions_len = out->spots_len = 0;
}

// ---- batched refinement (FitOrientation :696-801 over many grains) -------------
//
// One context holds the detector, the crystal and the HKL list of a
// parameter set, the float images of a batch and the grains to refine (their
// coarse orientations and prefiltered HKL lists).  Evaluations run on a CUDA
// device (device >= 0, refine.cu) or on host threads (device < 0) with the
// same arithmetic, so both give identical objective values.
struct lmb_refine {
  int device = -1;
  Detector d{};
  Crystal cr{};
  double recip[3][3];
  int max_spots = 0, nthreads = 1;
  unsigned n = 3;
  std::vector<int32_t> hkls;
  int nh = 0;
  std::vector<float> frames;  // host evaluation: the images, W x H each
  int n_img = 0;
  lmb::RefineDev *dev = nullptr;
  std::vector<double> hout[lmb::kRefineBufs];  // host evaluation: values per buffer
  int ng = 0;
  std::vector<int32_t> gimg, nvalid;
  std::vector<std::vector<int>> valid;  // host evaluation: per grain
  std::vector<double> x0, xl, xu;
  // statistics of the last evaluate / fit call
  int64_t last_points = 0;
  int32_t last_rounds = 0;
  float last_kernel_ms = 0.f;
};

namespace {

// problem_function at m points (grain[k], x[k][n]), in evaluation buffer b:
// eval_submit forms the points' matrices (into page-locked memory for the
// device) and queues the evaluation (on the host: computes it), eval_collect
// waits for it and hands out the m values (valid until b is submitted again).
int eval_submit(lmb_refine *r, int b, const int32_t *grain, const double *x, int64_t m) {
  const int nt = m >= 64 ? r->nthreads : 1;
  if (r->device >= 0) {
    double *T = nullptr;
    int32_t *gd = nullptr;
    int rc = lmb::refine_dev_stage(r->dev, b, m, &T, &gd);
    if (rc) return rc;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t k = 0; k < m; k++) {
      double OM[3][3];
      point_matrix(r->n, x + (size_t)k * r->n, r->cr, r->recip, OM);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) T[(size_t)k * 9 + i * 3 + j] = OM[i][j];
      gd[k] = grain[k];
    }
    return lmb::refine_dev_submit(r->dev, b, r->max_spots);
  }
  std::vector<double> &out = r->hout[b];
  out.resize((size_t)m);
  const size_t npx = (size_t)r->d.W * r->d.H;
#pragma omp parallel num_threads(nt)
  {
    std::vector<double> acc((size_t)3 * r->max_spots, 0.0);
#pragma omp for schedule(dynamic, 16)
    for (int64_t k = 0; k < m; k++) {
      const int g = grain[k];
      double OM[3][3];
      point_matrix(r->n, x + (size_t)k * r->n, r->cr, r->recip, OM);
      out[k] = overlap_at(OM, r->d, r->frames.data() + npx * r->gimg[g], r->hkls.data(),
                          r->valid[g].data(), r->nvalid[g], r->max_spots, acc);
    }
  }
  return LMB_OK;
}

int eval_collect(lmb_refine *r, int b, const double **obj, float *kernel_ms) {
  if (r->device >= 0) return lmb::refine_dev_collect(r->dev, b, obj, kernel_ms);
  *obj = r->hout[b].data();
  if (kernel_ms) *kernel_ms = 0.f;
  return LMB_OK;
}

// The two steps at once, values into obj[m].
int refine_eval(lmb_refine *r, const int32_t *grain, const double *x, int64_t m, double *obj,
                float *kernel_ms) {
  int rc = eval_submit(r, 0, grain, x, m);
  if (rc) return rc;
  const double *v = nullptr;
  rc = eval_collect(r, 0, &v, kernel_ms);
  if (rc) return rc;
  if (m) memcpy(obj, v, sizeof(double) * m);
  return LMB_OK;
}

// Bounded Nelder-Mead (Nelder & Mead 1965, with the coefficients of Lagarias,
// Reeds, Wright & Wright 1998: reflection 1, expansion 2, contraction 1/2,
// shrink 1/2), trial points clamped into the box.  This library's own
// optimiser, not NLopt's: its steps and stopping differ from NLopt's
// NELDERMEAD and BOBYQA.  One state per grain; every round each running
// grain proposes its next points and all of them are evaluated together.
constexpr int kMaxDims = 9;  // 3 Euler angles + 6 lattice parameters

struct NMGrain {
  double v[(kMaxDims + 1) * kMaxDims];  // n+1 vertices of n coordinates
  double f[kMaxDims + 1];               // their values
  double xr[kMaxDims], xb[kMaxDims];    // reflection, centroid of the n best
  double fr = 0;
  int phase = 0;  // 0 start simplex, 1 reflect, 2 expand, 3 outside / 4 inside contraction,
                  // 5 shrink, 6 done
  int evals = 0;
  int npend = 0;                                // points to evaluate this round
  double pend[(kMaxDims + 1) * kMaxDims];
};

constexpr double kTolRel = 1e-6;  // ftol_rel and xtol_rel of FitOrientation (:773-774)
// Start simplex: x0 and x0 + h_i e_i, h_i this fraction of coordinate i's box
// (Euler: 6 degrees wide).  Spots are a few pixels wide, so large first steps
// land every vertex off all spots.
constexpr double kInitStep = 0.02;
// From this many grains on, the fit runs them as two alternating groups.
constexpr int kSplitGrains = 64;

void nm_clamp(const lmb_refine *r, int g, double *x) {
  for (unsigned i = 0; i < r->n; i++)
    x[i] = std::min(std::max(x[i], r->xl[(size_t)g * r->n + i]), r->xu[(size_t)g * r->n + i]);
}

void nm_propose(NMGrain &s, unsigned n, const double *x) {
  for (unsigned i = 0; i < n; i++) s.pend[i] = x[i];
  s.npend = 1;
}

// Vertices in ascending value, ties in their current order (a stable sort).
void nm_sort(NMGrain &s, unsigned n) {
  for (unsigned i = 1; i <= n; i++) {
    const double fi = s.f[i];
    double vi[kMaxDims];
    for (unsigned c = 0; c < n; c++) vi[c] = s.v[i * n + c];
    unsigned j = i;
    for (; j > 0 && s.f[j - 1] > fi; j--) {
      s.f[j] = s.f[j - 1];
      for (unsigned c = 0; c < n; c++) s.v[j * n + c] = s.v[(j - 1) * n + c];
    }
    s.f[j] = fi;
    for (unsigned c = 0; c < n; c++) s.v[j * n + c] = vi[c];
  }
}

// Order the simplex, test the stopping rules, propose the reflection.
void nm_step(const lmb_refine *r, int g, NMGrain &s, int max_eval) {
  const unsigned n = r->n;
  nm_sort(s, n);
  s.npend = 0;
  bool stop = s.evals + 1 > max_eval;
  if (!stop && s.f[n] - s.f[0] <= kTolRel * std::fabs(s.f[0])) stop = true;
  if (!stop) {
    bool small = true;
    for (unsigned j = 1; j <= n && small; j++)
      for (unsigned i = 0; i < n; i++)
        if (std::fabs(s.v[j * n + i] - s.v[i]) > kTolRel * std::fabs(s.v[i])) {
          small = false;
          break;
        }
    stop = small;
  }
  if (stop) {
    s.phase = 6;
    return;
  }
  for (unsigned i = 0; i < n; i++) s.xb[i] = 0.0;
  for (unsigned j = 0; j < n; j++)
    for (unsigned i = 0; i < n; i++) s.xb[i] += s.v[j * n + i];
  for (unsigned i = 0; i < n; i++) s.xb[i] /= n;
  for (unsigned i = 0; i < n; i++) s.xr[i] = s.xb[i] + (s.xb[i] - s.v[n * n + i]);
  nm_clamp(r, g, s.xr);
  nm_propose(s, n, s.xr);
  s.phase = 1;
}

void nm_replace_worst(NMGrain &s, unsigned n, const double *x, double fx) {
  for (unsigned i = 0; i < n; i++) s.v[n * n + i] = x[i];
  s.f[n] = fx;
}

void nm_shrink(const lmb_refine *r, int g, NMGrain &s, int max_eval) {
  (void)g;
  const unsigned n = r->n;
  if (s.evals + (int)n > max_eval) {
    nm_sort(s, n);
    s.npend = 0;
    s.phase = 6;
    return;
  }
  for (unsigned j = 1; j <= n; j++)
    for (unsigned i = 0; i < n; i++) s.v[j * n + i] = s.v[i] + 0.5 * (s.v[j * n + i] - s.v[i]);
  for (unsigned k = 0; k < n * n; k++) s.pend[k] = s.v[n + k];
  s.npend = (int)n;
  s.phase = 5;
}

// Take this round's values (res[0..) in the order of s.pend) and move on.
void nm_consume(const lmb_refine *r, int g, NMGrain &s, const double *res, int max_eval) {
  const unsigned n = r->n;
  const double *xb = s.xb;
  switch (s.phase) {
    case 0:
      for (unsigned j = 0; j <= n; j++) s.f[j] = res[j];
      s.evals += n + 1;
      nm_step(r, g, s, max_eval);
      return;
    case 1: {
      s.fr = res[0];
      s.evals++;
      if (s.fr >= s.f[0] && s.fr < s.f[n - 1]) {
        nm_replace_worst(s, n, s.xr, s.fr);
        nm_step(r, g, s, max_eval);
      } else if (s.fr < s.f[0]) {
        if (s.evals + 1 > max_eval) {
          nm_replace_worst(s, n, s.xr, s.fr);
          nm_step(r, g, s, max_eval);
          return;
        }
        double x[kMaxDims];
        for (unsigned i = 0; i < n; i++) x[i] = xb[i] + 2.0 * (xb[i] - s.v[n * n + i]);
        nm_clamp(r, g, x);
        nm_propose(s, n, x);
        s.phase = 2;
      } else {
        if (s.evals + 1 > max_eval) {
          nm_step(r, g, s, max_eval);
          return;
        }
        double x[kMaxDims];
        if (s.fr < s.f[n]) {
          for (unsigned i = 0; i < n; i++) x[i] = xb[i] + 0.5 * (s.xr[i] - xb[i]);
          s.phase = 3;
        } else {
          for (unsigned i = 0; i < n; i++) x[i] = xb[i] + 0.5 * (s.v[n * n + i] - xb[i]);
          s.phase = 4;
        }
        nm_propose(s, n, x);
      }
      return;
    }
    case 2:
      s.evals++;
      if (res[0] < s.fr)
        nm_replace_worst(s, n, s.pend, res[0]);
      else
        nm_replace_worst(s, n, s.xr, s.fr);
      nm_step(r, g, s, max_eval);
      return;
    case 3:
      s.evals++;
      if (res[0] <= s.fr) {
        nm_replace_worst(s, n, s.pend, res[0]);
        nm_step(r, g, s, max_eval);
      } else {
        nm_shrink(r, g, s, max_eval);
      }
      return;
    case 4:
      s.evals++;
      if (res[0] < s.f[n]) {
        nm_replace_worst(s, n, s.pend, res[0]);
        nm_step(r, g, s, max_eval);
      } else {
        nm_shrink(r, g, s, max_eval);
      }
      return;
    case 5:
      for (unsigned j = 1; j <= n; j++) s.f[j] = res[j - 1];
      s.evals += n;
      nm_step(r, g, s, max_eval);
      return;
    default:
      return;
  }
}

}  // namespace

extern "C" int lmb_refine_create(int32_t device, const lmb_geometry *geo,
                                 const lmb_post_params *pp, const int32_t *hkls, int32_t nh,
                                 lmb_refine **out) {
  if (!geo || !pp || !out || nh < 0 || (!hkls && nh) || geo->nr_px_x <= 0 ||
      geo->nr_px_y <= 0 || geo->max_nr_spots <= 0) {
    lmb::set_error("bad argument");
    return LMB_ERR_INVALID;
  }
  lmb_refine *r = new lmb_refine();
  r->device = device;
  r->cr = make_crystal(pp);
  make_detector(geo, &r->d, r->recip);
  r->max_spots = 3 * geo->max_nr_spots;  // LaueMatchingCPU.c:740
  r->nthreads = pp->num_threads > 0 ? pp->num_threads : 1;
  r->n = fit_dims(r->cr);
  r->hkls.assign(hkls, hkls + 3 * (size_t)nh);
  r->nh = nh;
  if (device >= 0) {
    lmb::RefineGeoHost g{};
    for (int i = 0; i < 3; i++) {
      g.p[i] = r->d.p[i];
      for (int j = 0; j < 3; j++) g.rt[i * 3 + j] = r->d.rt[i][j];
    }
    g.px_x = r->d.px_x;
    g.px_y = r->d.px_y;
    g.elo = r->d.elo;
    g.ehi = r->d.ehi;
    g.W = r->d.W;
    g.H = r->d.H;
    const int rc = lmb::refine_dev_create(device, g, hkls, nh, &r->dev);
    if (rc) {
      delete r;
      return rc;
    }
  }
  *out = r;
  return LMB_OK;
}

extern "C" int lmb_refine_destroy(lmb_refine *r) {
  if (!r) return LMB_OK;
  lmb::refine_dev_destroy(r->dev);
  delete r;
  return LMB_OK;
}

extern "C" int lmb_refine_dims(lmb_refine *r, int32_t *n) {
  if (!r || !n) {
    lmb::set_error("bad argument");
    return LMB_ERR_INVALID;
  }
  *n = (int32_t)r->n;
  return LMB_OK;
}

extern "C" int lmb_refine_set_images(lmb_refine *r, const float *const *frames,
                                     int32_t n_images) {
  if (!r || n_images < 0 || (!frames && n_images)) {
    lmb::set_error("bad argument");
    return LMB_ERR_INVALID;
  }
  for (int i = 0; i < n_images; i++)
    if (!frames[i]) {
      lmb::set_error("null frame %d", i);
      return LMB_ERR_INVALID;
    }
  r->ng = 0;
  if (r->device >= 0) {
    const int rc = lmb::refine_dev_images(r->dev, frames, n_images);
    if (rc) return rc;
  } else {
    const size_t npx = (size_t)r->d.W * r->d.H;
    r->frames.resize(npx * n_images);
    for (int i = 0; i < n_images; i++)
      memcpy(r->frames.data() + npx * i, frames[i], npx * sizeof(float));
  }
  r->n_img = n_images;
  return LMB_OK;
}

extern "C" int lmb_refine_set_grains(lmb_refine *r, const double *orients, const int32_t *image,
                                     int32_t n_grains, int32_t *n_valid) {
  if (!r || n_grains < 0 || (n_grains && (!orients || !image))) {
    lmb::set_error("bad argument");
    return LMB_ERR_INVALID;
  }
  for (int g = 0; g < n_grains; g++)
    if (image[g] < 0 || image[g] >= r->n_img) {
      lmb::set_error("grain %d: image %d outside the %d images", g, image[g], r->n_img);
      return LMB_ERR_INVALID;
    }
  const unsigned n = r->n;
  const double tol = 3 * kDeg2Rad;  // LaueMatchingCPU.c:739
  r->ng = 0;
  r->gimg.assign(image, image + n_grains);
  r->x0.assign((size_t)n_grains * n, 0.0);
  r->xl = r->x0;
  r->xu = r->x0;
  std::vector<double> T((size_t)n_grains * 9);
#pragma omp parallel for num_threads(r->nthreads) schedule(static)
  for (int g = 0; g < n_grains; g++) {
    // fitAndWriteOrientations (:1090-1112): Euler angles of the coarse matrix,
    // FitOrientation's start point and box (:718-743)
    double ob[3][3], eb[3], OMt[3][3], OM[3][3];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) ob[i][j] = orients[(size_t)g * 9 + i * 3 + j];
    om_to_euler(ob, eb);
    double *x = &r->x0[(size_t)g * n], *xl = &r->xl[(size_t)g * n], *xu = &r->xu[(size_t)g * n];
    for (int i = 0; i < 3; i++) {
      x[i] = eb[i];
      xl[i] = eb[i] - tol;
      xu[i] = eb[i] + tol;
    }
    int c = 3;
    for (int i = 0; i < 6; i++)
      if (r->cr.tol_latc[i] != 0) {
        x[c] = r->cr.lat[i];
        xl[c] = r->cr.lat[i] * (1 - r->cr.tol_latc[i]);
        xu[c] = r->cr.lat[i] * (1 + r->cr.tol_latc[i]);
        c++;
      }
    if (r->cr.tol_c_over_a != 0) {
      x[3] = r->cr.c_over_a_orig;
      xl[3] = r->cr.c_over_a_orig * (1 - r->cr.tol_c_over_a);
      xu[3] = r->cr.c_over_a_orig * (1 + r->cr.tol_c_over_a);
    }
    // prefilterHKLs (:513-561) at the coarse angles with the parameters' lattice
    euler_to_om(eb, OMt);
    mat33(OMt, r->recip, OM);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) T[(size_t)g * 9 + i * 3 + j] = OM[i][j];
  }
  r->nvalid.assign(n_grains, 0);
  if (r->device >= 0) {
    const int rc = lmb::refine_dev_prefilter(r->dev, T.data(), image, n_grains, r->nvalid.data(),
                                             nullptr);
    if (rc) return rc;
  } else {
    r->valid.assign(n_grains, {});
#pragma omp parallel for num_threads(r->nthreads) schedule(dynamic)
    for (int g = 0; g < n_grains; g++) {
      double OM[3][3];
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) OM[i][j] = T[(size_t)g * 9 + i * 3 + j];
      for (int h = 0; h < r->nh; h++) {
        double qh[3], px, py, ql;
        if (project(OM, r->hkls.data() + 3 * h, r->d, qh, px, py, ql)) r->valid[g].push_back(h);
      }
      r->nvalid[g] = (int32_t)r->valid[g].size();
    }
  }
  if (n_valid) memcpy(n_valid, r->nvalid.data(), sizeof(int32_t) * n_grains);
  r->ng = n_grains;
  return LMB_OK;
}

extern "C" int lmb_refine_start(lmb_refine *r, double *x0, double *lower, double *upper) {
  if (!r) {
    lmb::set_error("bad argument");
    return LMB_ERR_INVALID;
  }
  const size_t k = (size_t)r->ng * r->n;
  if (x0) memcpy(x0, r->x0.data(), k * sizeof(double));
  if (lower) memcpy(lower, r->xl.data(), k * sizeof(double));
  if (upper) memcpy(upper, r->xu.data(), k * sizeof(double));
  return LMB_OK;
}

extern "C" int lmb_refine_evaluate(lmb_refine *r, const int32_t *grain, const double *x,
                                   int64_t m, double *objective) {
  if (!r || m < 0 || (m && (!grain || !x || !objective))) {
    lmb::set_error("bad argument");
    return LMB_ERR_INVALID;
  }
  for (int64_t k = 0; k < m; k++)
    if (grain[k] < 0 || grain[k] >= r->ng) {
      lmb::set_error("point %lld: grain %d outside the %d grains", (long long)k, grain[k], r->ng);
      return LMB_ERR_INVALID;
    }
  float ms = 0.f;
  const int rc = refine_eval(r, grain, x, m, objective, &ms);
  r->last_points = m;
  r->last_rounds = 1;
  r->last_kernel_ms = ms;
  return rc;
}

extern "C" int lmb_refine_fit(lmb_refine *r, int32_t optimizer, int32_t max_eval,
                              double init_step, double *x_fit, double *overlap, int32_t *evals) {
  if (!r || (optimizer != 0 && optimizer != 1) || max_eval < 1 || !(init_step < 1.0) ||
      (r->ng && (!x_fit || !overlap))) {
    lmb::set_error("bad argument");
    return LMB_ERR_INVALID;
  }
  const unsigned n = r->n;
  const int ng = r->ng;
  r->last_points = 0;
  r->last_rounds = 0;
  r->last_kernel_ms = 0.f;
  if (ng == 0) return LMB_OK;
  if (optimizer == 0 || max_eval < (int)n + 1) {
    // the evaluate-once stand-in: x stays at the start point
    std::vector<int32_t> gi(ng);
    std::vector<double> f(ng);
    for (int g = 0; g < ng; g++) gi[g] = g;
    float ms = 0.f;
    const int rc = refine_eval(r, gi.data(), r->x0.data(), ng, f.data(), &ms);
    if (rc) return rc;
    memcpy(x_fit, r->x0.data(), sizeof(double) * ng * n);
    for (int g = 0; g < ng; g++) {
      overlap[g] = -f[g];
      if (evals) evals[g] = 1;
    }
    r->last_points = ng;
    r->last_rounds = 1;
    r->last_kernel_ms = ms;
    return LMB_OK;
  }
  std::vector<NMGrain> st(ng);
  for (int g = 0; g < ng; g++) {
    NMGrain &s = st[g];
    const double *x0 = &r->x0[(size_t)g * n];
    for (unsigned j = 0; j <= n; j++) {
      s.f[j] = 0.0;
      for (unsigned i = 0; i < n; i++) s.v[j * n + i] = x0[i];
    }
    for (unsigned i = 0; i < n; i++) {
      const double lo = r->xl[(size_t)g * n + i], hi = r->xu[(size_t)g * n + i];
      const double h = (init_step > 0 ? init_step : kInitStep) * (hi - lo);
      double y = x0[i] + h;
      if (y > hi) y = x0[i] - h;
      s.v[(i + 1) * n + i] = y;
    }
    for (unsigned k = 0; k < (n + 1) * n; k++) s.pend[k] = s.v[k];
    s.npend = (int)n + 1;
    s.phase = 0;
  }
  // Two groups of grains alternate: while the device evaluates one group's
  // round, the host takes the other group's values and forms its next points.
  // Each grain's steps depend on its own values only, so the grouping changes
  // no result.
  struct Group {
    int g0 = 0, g1 = 0;
    std::vector<int32_t> pg;  // host evaluation: grain of each point
    std::vector<double> px;   // host evaluation: the points
    std::vector<int64_t> off;
    int64_t m = 0;
    bool pending = false;
  };
  const int ngroups = ng >= kSplitGrains ? 2 : 1;
  Group grp[2];
  for (int b = 0; b < ngroups; b++) {
    grp[b].g0 = (int)((int64_t)ng * b / ngroups);
    grp[b].g1 = (int)((int64_t)ng * (b + 1) / ngroups);
    grp[b].off.assign(grp[b].g1 - grp[b].g0 + 1, 0);
  }
  const int nt = r->nthreads;
  // One round of group b in one parallel region: the optimiser steps on the
  // values pf (none on the first round), the round's points in grain order,
  // and (device) their matrices straight into the page-locked staging
  // buffer; then the evaluation is queued (device) or done (host).
  auto round = [&](int b, const double *pf) -> int {
    Group &G = grp[b];
    const int cnt = G.g1 - G.g0;
    const bool dev = r->device >= 0;
    int64_t tot = 0;
    int lrc = LMB_OK;
    double *T = nullptr;
    int32_t *gd = nullptr;
#pragma omp parallel num_threads(nt) if (cnt >= 256)
    {
      if (pf) {
#pragma omp for schedule(dynamic, 32)
        for (int g = G.g0; g < G.g1; g++)
          if (st[g].phase != 6) nm_consume(r, g, st[g], pf + G.off[g - G.g0], max_eval);
      }
#pragma omp master
      {
        for (int g = G.g0; g < G.g1; g++) {
          G.off[g - G.g0] = tot;
          if (st[g].phase != 6) tot += st[g].npend;
        }
        G.off[cnt] = tot;
        if (tot > 0 && dev) {
          lrc = lmb::refine_dev_stage(r->dev, b, tot, &T, &gd);
        } else if (tot > 0) {
          G.pg.resize((size_t)tot);
          G.px.resize((size_t)tot * n);
        }
      }
#pragma omp barrier
      if (tot > 0 && lrc == LMB_OK) {
#pragma omp for schedule(static)
        for (int g = G.g0; g < G.g1; g++) {
          if (st[g].phase == 6) continue;
          const int64_t o = G.off[g - G.g0], k = G.off[g - G.g0 + 1] - o;
          for (int64_t j = 0; j < k; j++) {
            const double *x = st[g].pend + (size_t)j * n;
            if (dev) {
              double OM[3][3];
              point_matrix(n, x, r->cr, r->recip, OM);
              double *t = T + (size_t)(o + j) * 9;
              for (int i = 0; i < 3; i++)
                for (int c = 0; c < 3; c++) t[i * 3 + c] = OM[i][c];
              gd[o + j] = g;
            } else {
              G.pg[(size_t)(o + j)] = g;
              std::copy(x, x + n, G.px.begin() + (size_t)(o + j) * n);
            }
          }
        }
      }
    }
    if (lrc) return lrc;
    G.m = tot;
    if (tot == 0) return LMB_OK;
    lrc = dev ? lmb::refine_dev_submit(r->dev, b, r->max_spots)
              : eval_submit(r, b, G.pg.data(), G.px.data(), tot);
    G.pending = lrc == LMB_OK;
    return lrc;
  };
  auto drain = [&]() {  // after an error: wait for what is still queued
    for (int b = 0; b < ngroups; b++)
      if (grp[b].pending) {
        const double *v;
        eval_collect(r, b, &v, nullptr);
        grp[b].pending = false;
      }
  };
  int rc = LMB_OK;
  for (int b = 0; b < ngroups && !rc; b++) rc = round(b, nullptr);
  for (bool any = true; any && !rc;) {
    any = false;
    for (int b = 0; b < ngroups && !rc; b++) {
      Group &G = grp[b];
      if (!G.pending) continue;
      any = true;
      const double *pf = nullptr;
      float ms = 0.f;
      G.pending = false;
      rc = eval_collect(r, b, &pf, &ms);
      if (rc) break;
      r->last_points += G.m;
      r->last_rounds++;
      r->last_kernel_ms += ms;
      rc = round(b, pf);
    }
  }
  if (rc) {
    drain();
    return rc;
  }
  for (int g = 0; g < ng; g++) {
    memcpy(x_fit + (size_t)g * n, st[g].v, sizeof(double) * n);
    overlap[g] = -st[g].f[0];
    if (evals) evals[g] = st[g].evals;
  }
  return LMB_OK;
}

extern "C" int lmb_refine_last_stats(lmb_refine *r, int64_t *points, int32_t *rounds,
                                     float *kernel_ms) {
  if (!r) {
    lmb::set_error("bad argument");
    return LMB_ERR_INVALID;
  }
  if (points) *points = r->last_points;
  if (rounds) *rounds = r->last_rounds;
  if (kernel_ms) *kernel_ms = r->last_kernel_ms;
  return LMB_OK;
}
