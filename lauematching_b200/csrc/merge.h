// Host-side interface of the device duplicate merge (merge.cu), usable from
// host-only translation units (post.cpp).
#pragma once

#include <cstdint>
#include <utility>
#include <vector>

namespace lmb {

struct MergeHost {
  int device;
  int64_t n;
  const double *quat;   // [n][4] candidates' quaternions, input order
  const double *score;  // [n]
  int nsym;
  double sym[24][4];
  double max_angle, rad2deg;
  double mid, window;  // float rounding boundary at max_angle, band decided on the host
  bool (*decide)(void *ctx, int64_t l, int64_t g);  // host comparison of a close call
  void *ctx;
};

// Clusters in input order: best_idx[c] (index into the candidates), counts[c];
// n_clusters of them.  unsure_out receives the (l, g) pairs decided on the host.
int merge_device_run(const MergeHost &h, int32_t *n_clusters, int64_t *best_idx, int32_t *counts,
                     std::vector<std::pair<uint32_t, uint32_t>> *unsure_out, bool *overflow);

}  // namespace lmb
