// Host-side FP64 geometry: detector rotation and reciprocal basis.
//
// Both are evaluated once per run on the host, in the reference's operation
// order, with the same libm (cos, sin, sqrt), so the matrices are bitwise the
// ones the reference computes.  Built with -ffp-contract=off.
#include <cmath>

#include "../../include/lmb200.h"

namespace lmb {
void set_error(const char *fmt, ...);
}

namespace {
constexpr double kDeg2Rad = 0.0174532925199433;  // LaueMatchingHeaders.h:32
constexpr double kEps = 1E-12;                    // LaueMatchingHeaders.h:42

double zero_out(double v) { return (std::fabs(v) < kEps) ? 0 : v; }

// Rodrigues rotation of R_Array and its transpose (LaueMatchingCPU.c:225-239).
void detector_rot_t(const double r[3], double rot_t[9]) {
  const double ang = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  const double v[3] = {r[0] / ang, r[1] / ang, r[2] / ang};
  const double c = std::cos(ang), s = std::sin(ang);
  const double m[3][3] = {
      {c + (1 - c) * (v[0] * v[0]), (1 - c) * v[0] * v[1] - s * v[2],
       (1 - c) * v[0] * v[2] + s * v[1]},
      {(1 - c) * v[1] * v[0] + s * v[2], c + (1 - c) * (v[1] * v[1]),
       (1 - c) * v[1] * v[2] - s * v[0]},
      {(1 - c) * v[2] * v[0] - s * v[1], (1 - c) * v[2] * v[1] + s * v[0],
       c + (1 - c) * (v[2] * v[2])}};
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) rot_t[i * 3 + j] = m[j][i];
}

// Reciprocal basis, 2*pi/V convention, rhombohedral settings for the
// trigonal space groups (calcRecipArray, LaueMatchingHeaders.h:379-436).
void recip_basis(const double lat[6], int sg, double out[9]) {
  const double a = lat[0], b = lat[1], c = lat[2];
  const bool rh = sg == 146 || sg == 148 || sg == 155 || sg == 160 || sg == 161 || sg == 166 ||
                  sg == 167;
  const double ca = std::cos(lat[3] * kDeg2Rad), cb = std::cos(lat[4] * kDeg2Rad);
  const double cg = std::cos(lat[5] * kDeg2Rad), sgm = std::sin(lat[5] * kDeg2Rad);
  const double phi = std::sqrt(1.0 - ca * ca - cb * cb - cg * cg + 2 * ca * cb * cg);
  const double vc = a * b * c * phi;
  const double pv = (2 * M_PI) / vc;
  double a0, a1, a2, b0, b1, b2, c0, c1, c2;
  if (!rh) {
    a0 = zero_out(a);
    a1 = zero_out(0.0);
    a2 = zero_out(0.0);
    b0 = b * cg;
    b1 = zero_out(b * sgm);
    b2 = zero_out(0.0);
    c0 = c * cb;
    c1 = c * (ca - cb * cg) / sgm;
    c2 = zero_out(c * phi / sgm);
  } else {
    const double p = std::sqrt(1.0 + 2 * ca), q = std::sqrt(1.0 - ca);
    const double pmq = (a / 3.0) * (p - q), p2q = (a / 3.0) * (p + 2 * q);
    a0 = p2q;
    a1 = pmq;
    a2 = pmq;
    b0 = pmq;
    b1 = p2q;
    b2 = pmq;
    c0 = pmq;
    c1 = pmq;
    c2 = p2q;
  }
  out[0] = zero_out((b1 * c2 - b2 * c1) * pv);
  out[3] = zero_out((b2 * c0 - b0 * c2) * pv);
  out[6] = zero_out((b0 * c1 - b1 * c0) * pv);
  out[1] = zero_out((c1 * a2 - c2 * a1) * pv);
  out[4] = zero_out((c2 * a0 - c0 * a2) * pv);
  out[7] = zero_out((c0 * a1 - c1 * a0) * pv);
  out[2] = zero_out((a1 * b2 - a2 * b1) * pv);
  out[5] = zero_out((a2 * b0 - a0 * b2) * pv);
  out[8] = zero_out((a0 * b1 - a1 * b0) * pv);
}
}  // namespace

extern "C" int lmb_geometry_init(const double lattice[6], int32_t space_group,
                                 const double p_array[3], const double r_array[3], double px_x,
                                 double px_y, int32_t nr_px_x, int32_t nr_px_y, double elo,
                                 double ehi, int32_t max_nr_spots, lmb_geometry *out) {
  if (!lattice || !p_array || !r_array || !out) {
    lmb::set_error("null argument");
    return LMB_ERR_INVALID;
  }
  lmb_geometry g{};
  recip_basis(lattice, space_group, g.recip);
  detector_rot_t(r_array, g.rot_t);
  for (int i = 0; i < 3; i++) g.p[i] = p_array[i];
  g.px_x = px_x;
  g.px_y = px_y;
  g.elo = elo;
  g.ehi = ehi;
  g.nr_px_x = nr_px_x;
  g.nr_px_y = nr_px_y;
  g.max_nr_spots = max_nr_spots;
  *out = g;
  return LMB_OK;
}
