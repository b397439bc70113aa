// Host-side interface of the device refinement objective (refine.cu), usable
// from host-only translation units (post.cpp).
#pragma once

#include <cstdint>

namespace lmb {

// Detector model of the refinement (calcOverlapFiltered's arguments).
struct RefineGeoHost {
  double rt[9];  // rotTranspose, row-major
  double p[3];   // pArr
  double px_x, px_y, elo, ehi;
  int W, H;      // nrPxX, nrPxY
};

struct RefineDev;

int refine_dev_create(int device, const RefineGeoHost &g, const int32_t *hkls, int nh,
                      RefineDev **out);
void refine_dev_destroy(RefineDev *r);
// n float frames of W x H (image[py * W + px]) copied to the device.
int refine_dev_images(RefineDev *r, const float *const *frames, int n);
// prefilterHKLs for ng grains at the matrices T[ng][9] (OM . recip at the
// coarse Euler angles); each grain's image index in image[ng].  The valid
// lists stay on the device; their lengths go to nvalid[ng] (host) and, when
// valid is not null, the lists themselves to valid[ng][nh] (host).
int refine_dev_prefilter(RefineDev *r, const double *T, const int32_t *image, int ng,
                         int32_t *nvalid, int32_t *valid);
// problem_function for many points, in two steps so that the host can work
// while the device evaluates: refine_dev_stage hands out page-locked room for
// m points of evaluation buffer b (T[m][9]: matrix of point k; grain[m]: its
// grain), refine_dev_submit queues the copy, the kernel and the copy back,
// refine_dev_collect waits for them and points *objective at the m values
// (-(nrPos * sqrt(sum)) over the grain's valid list), valid until the buffer
// is staged again.  kernel_ms (optional): the kernel's device time.
constexpr int kRefineBufs = 2;
int refine_dev_stage(RefineDev *r, int b, int64_t m, double **T, int32_t **grain);
int refine_dev_submit(RefineDev *r, int b, int max_spots);
int refine_dev_collect(RefineDev *r, int b, const double **objective, float *kernel_ms);

}  // namespace lmb
