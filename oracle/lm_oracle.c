/*
 * lm_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A plain-C, FP64 restatement of the reference LaueMatching CPU algorithm for
 * the orientation-matching hot path.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load this library; the product never
 * does.  Every function cites the reference lines it restates
 * (paths relative to the LaueMatching source tree).
 *
 * Bit-exactness rules followed here (they are what make the oracle a pin):
 *   - every FP64 expression is evaluated in the reference's order, with the
 *     reference's parenthesisation (C evaluates a*b+c as (a*b)+c; the build
 *     uses -ffp-contract=off so no fused multiply-add is formed);
 *   - (int) casts use C truncation, as the reference does.
 *
 * Deviations from the reference, each where the reference has undefined
 * behaviour on malformed input:
 *   - a record whose count exceeds MaxNrLaueSpots is clamped to it (the
 *     reference CPU would read into the next record; the reference GPU kernel
 *     clamps, LaueMatchingGPU.cu:54-55);
 *   - a pixel outside the detector is skipped (the reference CPU would read
 *     outside the image; the reference GPU kernel skips, LaueMatchingGPU.cu:65).
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_HC_KEVNM 1.2398419739 /* LaueMatchingHeaders.h:41 */
#define ORC_DEG2RAD 0.0174532925199433 /* LaueMatchingHeaders.h:32 */
#define ORC_EPS 1E-12 /* LaueMatchingHeaders.h:42 */

static double orc_zero_out(double v) { return (fabs(v) < ORC_EPS) ? 0 : v; }

/* Detector rotation from R_Array (Rodrigues) and its transpose.
 * Restates LaueMatchingCPU.c:225-239.  R = (0,0,0) yields NaN, as in the
 * reference (division by |R|). */
void orc_detector_rot_t(const double r[3], double rot_t[9]) {
  double ang = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  double v[3] = {r[0] / ang, r[1] / ang, r[2] / ang};
  double c = cos(ang), s = sin(ang);
  double rot[3][3] = {
      {c + (1 - c) * (v[0] * v[0]), (1 - c) * v[0] * v[1] - s * v[2],
       (1 - c) * v[0] * v[2] + s * v[1]},
      {(1 - c) * v[1] * v[0] + s * v[2], c + (1 - c) * (v[1] * v[1]),
       (1 - c) * v[1] * v[2] - s * v[0]},
      {(1 - c) * v[2] * v[0] - s * v[1], (1 - c) * v[2] * v[1] + s * v[0],
       c + (1 - c) * (v[2] * v[2])}};
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) rot_t[i * 3 + j] = rot[j][i];
}

/* Reciprocal basis, 2*pi/V convention.  Restates calcRecipArray,
 * LaueMatchingHeaders.h:379-436 (rhombohedral space groups included). */
void orc_recip(const double lat[6], int sg, double recip[9]) {
  double a = lat[0], b = lat[1], c = lat[2];
  int rh = (sg == 146 || sg == 148 || sg == 155 || sg == 160 || sg == 161 ||
            sg == 166 || sg == 167);
  double ca = cos(lat[3] * ORC_DEG2RAD), cb = cos(lat[4] * ORC_DEG2RAD);
  double cg = cos(lat[5] * ORC_DEG2RAD), sg_ = sin(lat[5] * ORC_DEG2RAD);
  double phi = sqrt(1.0 - ca * ca - cb * cb - cg * cg + 2 * ca * cb * cg);
  double vc = a * b * c * phi;
  double pv = (2 * M_PI) / vc;
  double a0, a1, a2, b0, b1, b2, c0, c1, c2;
  if (!rh) {
    a0 = a; a1 = 0.0; a2 = 0.0;
    b0 = b * cg; b1 = b * sg_; b2 = 0;
    c0 = c * cb; c1 = c * (ca - cb * cg) / sg_; c2 = c * phi / sg_;
    a0 = orc_zero_out(a0); a1 = orc_zero_out(a1); a2 = orc_zero_out(a2);
    b1 = orc_zero_out(b1); b2 = orc_zero_out(b2); c2 = orc_zero_out(c2);
  } else {
    double p = sqrt(1.0 + 2 * ca), q = sqrt(1.0 - ca);
    double pmq = (a / 3.0) * (p - q), p2q = (a / 3.0) * (p + 2 * q);
    a0 = p2q; a1 = pmq; a2 = pmq;
    b0 = pmq; b1 = p2q; b2 = pmq;
    c0 = pmq; c1 = pmq; c2 = p2q;
  }
  recip[0 * 3 + 0] = orc_zero_out((b1 * c2 - b2 * c1) * pv);
  recip[1 * 3 + 0] = orc_zero_out((b2 * c0 - b0 * c2) * pv);
  recip[2 * 3 + 0] = orc_zero_out((b0 * c1 - b1 * c0) * pv);
  recip[0 * 3 + 1] = orc_zero_out((c1 * a2 - c2 * a1) * pv);
  recip[1 * 3 + 1] = orc_zero_out((c2 * a0 - c0 * a2) * pv);
  recip[2 * 3 + 1] = orc_zero_out((c0 * a1 - c1 * a0) * pv);
  recip[0 * 3 + 2] = orc_zero_out((a1 * b2 - a2 * b1) * pv);
  recip[1 * 3 + 2] = orc_zero_out((a2 * b0 - a0 * b2) * pv);
  recip[2 * 3 + 2] = orc_zero_out((a0 * b1 - a1 * b0) * pv);
}

/* Forward simulation of one orientation into one record uint16[1+2S].
 * Restates LaueMatchingCPU.c:595-667 (MatrixMultF33 / MatrixMultF from
 * LaueMatchingHeaders.h:349-369).  `seen` is a caller-owned scratch list of
 * accepted pixels (equality on (ipx, ipy) is exactly the reference's
 * occupancy-mask test at :638-641). */
static void orc_forward_one(const double *om, const int *hkls, int nh,
                            const double *recip, const double *rot_t,
                            const double *p, double px_x, double px_y, int W,
                            int H, double elo, double ehi, int S,
                            uint16_t *rec) {
  double t[3][3];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++)
      t[r][c] = om[r * 3 + 0] * recip[0 * 3 + c] +
                om[r * 3 + 1] * recip[1 * 3 + c] +
                om[r * 3 + 2] * recip[2 * 3 + c];
  int n = 0;
  memset(rec, 0, sizeof(uint16_t) * (size_t)(1 + 2 * S));
  for (int h = 0; h < nh && n < S; h++) {
    double hkl[3] = {hkls[3 * h + 0], hkls[3 * h + 1], hkls[3 * h + 2]};
    double q[3];
    for (int i = 0; i < 3; i++) {
      q[i] = 0;
      for (int j = 0; j < 3; j++) q[i] += t[i][j] * hkl[j];
    }
    double ql = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
    if (ql == 0) continue;
    double qh[3] = {q[0] / ql, q[1] / ql, q[2] / ql};
    double dot = qh[2];
    double kf[3] = {0 - 2 * dot * qh[0], 0 - 2 * dot * qh[1],
                    1.0 - 2 * dot * qh[2]};
    double xyz[3];
    for (int i = 0; i < 3; i++) {
      xyz[i] = 0;
      for (int j = 0; j < 3; j++) xyz[i] += rot_t[i * 3 + j] * kf[j];
    }
    if (xyz[2] <= 0) continue;
    double x = xyz[0] * p[2] / xyz[2];
    double y = xyz[1] * p[2] / xyz[2];
    double xp = x - p[0], yp = y - p[1];
    int ipx = (int)((xp / px_x) + (0.5 * (W - 1)));
    if (ipx < 0 || ipx > (W - 1)) continue;
    int ipy = (int)((yp / px_y) + (0.5 * (H - 1)));
    if (ipy < 0 || ipy > (H - 1)) continue;
    double sin_th = -qh[2];
    double e = ORC_HC_KEVNM * ql / (4 * M_PI * sin_th);
    if (e < elo || e > ehi) continue;
    int dup = 0;
    for (int s = 0; s < n; s++)
      if (rec[1 + 2 * s] == (uint16_t)ipx && rec[2 + 2 * s] == (uint16_t)ipy) {
        dup = 1;
        break;
      }
    if (dup) continue;
    rec[1 + 2 * n] = (uint16_t)ipx;
    rec[2 + 2 * n] = (uint16_t)ipy;
    n++;
  }
  rec[0] = (uint16_t)n;
}

void orc_forward(const double *orients, int64_t n, const int *hkls, int nh,
                 const double *recip, const double *rot_t, const double *p,
                 double px_x, double px_y, int W, int H, double elo,
                 double ehi, int S, uint16_t *out, int nthreads) {
  size_t R = (size_t)(1 + 2 * S);
#pragma omp parallel for schedule(static) num_threads(nthreads)
  for (int64_t i = 0; i < n; i++)
    orc_forward_one(orients + 9 * i, hkls, nh, recip, rot_t, p, px_x, px_y, W,
                    H, elo, ehi, S, out + R * (size_t)i);
}

/* uint8 quantisation.  Restates LaueMatchingCPU.c:356-375.  Returns imScale. */
double orc_quantize(const double *img, int64_t npx, uint8_t *out) {
  double mx = 0;
  for (int64_t i = 0; i < npx; i++)
    if (img[i] > mx) mx = img[i];
  double scale = (mx > 0) ? mx / 255.0 : 1.0;
  double inv = (mx > 0) ? 255.0 / mx : 0.0;
  for (int64_t i = 0; i < npx; i++) {
    if (img[i] > 0) {
      double v = img[i] * inv;
      out[i] = (v >= 255.0) ? 255 : (v < 1.0) ? 1 : (uint8_t)v;
    } else {
      out[i] = 0;
    }
  }
  return scale;
}

/* Compare one record against the image.  mode 0: the uint8 image scaled by
 * im_scale (LaueMatchingCPU.c:668-682, DoFwd 0); mode 1: the float64 image
 * read directly (LaueMatchingCPU.c:649-653, the DoFwd 1 path). */
static inline void orc_compare_one(const uint16_t *rec, int S, int mode,
                                   const uint8_t *u8, const double *f64,
                                   double im_scale, int W, int H, int *n_sp,
                                   int *sum_u8, double *tot) {
  int c = rec[0];
  if (c > S) c = S;
  int ns = 0, su = 0;
  double t = 0;
  for (int s = 0; s < c; s++) {
    int x = rec[1 + 2 * s], y = rec[2 + 2 * s];
    if (x >= W || y >= H) continue;
    size_t px = (size_t)y * (size_t)W + (size_t)x;
    if (mode == 0) {
      uint8_t raw = u8[px];
      if (raw > 0) {
        t += (double)raw * im_scale;
        ns++;
        su += raw;
      }
    } else {
      double v = f64[px];
      if (v > 0) {
        t += v;
        ns++;
        su += u8 ? u8[px] : 0;
      }
    }
  }
  *n_sp = ns;
  *sum_u8 = su;
  *tot = t;
}

/* Full compare pass: survivors in ascending orientation ID, exactly the
 * collection order of LaueMatchingCPU.c:781-788.  A survivor is an
 * orientation with nSpots >= min_nr_spots and totInt >= min_intensity
 * (:683) whose score totInt*sqrt(nSpots) (:688) is non-zero (:783).
 * *n_pass receives the reference's nrResults (:686), which also counts
 * passing orientations whose score is zero.  Returns the survivor count, or
 * -(count) when it exceeds cap (outputs then hold the first cap). */
int64_t orc_compare(const uint16_t *recs, int64_t n, int S, int mode,
                    const uint8_t *u8, const double *f64, double im_scale,
                    int W, int H, int min_nr_spots, double min_intensity,
                    int64_t *ids, int32_t *n_spots, int32_t *sum_u8,
                    double *tot_int, double *score, int64_t cap,
                    int64_t *n_pass, int nthreads) {
  size_t R = (size_t)(1 + 2 * S);
  if (nthreads < 1) nthreads = 1;
  int64_t *cnt = (int64_t *)calloc((size_t)nthreads + 1, sizeof(int64_t));
  int64_t *pas = (int64_t *)calloc((size_t)nthreads + 1, sizeof(int64_t));
  int64_t chunk = (n + nthreads - 1) / nthreads;
  /* pass 1: per-thread survivor counts over contiguous slabs */
#pragma omp parallel num_threads(nthreads)
  {
    int tid = omp_get_thread_num();
    int64_t lo = (int64_t)tid * chunk, hi = lo + chunk;
    if (hi > n) hi = n;
    int64_t k = 0, np = 0;
    for (int64_t i = lo; i < hi; i++) {
      int ns, su;
      double t;
      orc_compare_one(recs + R * (size_t)i, S, mode, u8, f64, im_scale, W, H,
                      &ns, &su, &t);
      if (ns >= min_nr_spots && t >= min_intensity) {
        np++;
        if (t * sqrt((double)ns) != 0) k++;
      }
    }
    cnt[tid + 1] = k;
    pas[tid + 1] = np;
  }
  for (int i = 0; i < nthreads; i++) {
    cnt[i + 1] += cnt[i];
    pas[i + 1] += pas[i];
  }
  int64_t total = cnt[nthreads];
  /* pass 2: write survivors at each slab's prefix offset (ID order) */
#pragma omp parallel num_threads(nthreads)
  {
    int tid = omp_get_thread_num();
    int64_t lo = (int64_t)tid * chunk, hi = lo + chunk;
    if (hi > n) hi = n;
    int64_t k = cnt[tid];
    for (int64_t i = lo; i < hi; i++) {
      int ns, su;
      double t;
      orc_compare_one(recs + R * (size_t)i, S, mode, u8, f64, im_scale, W, H,
                      &ns, &su, &t);
      if (ns >= min_nr_spots && t >= min_intensity) {
        double sc = t * sqrt((double)ns);
        if (sc == 0) continue;
        if (k < cap) {
          ids[k] = i;
          n_spots[k] = ns;
          sum_u8[k] = su;
          tot_int[k] = t;
          score[k] = sc;
        }
        k++;
      }
    }
  }
  if (n_pass) *n_pass = pas[nthreads];
  free(cnt);
  free(pas);
  return total <= cap ? total : -total;
}
