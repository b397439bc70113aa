// Refinement objective on the device: prefilterHKLs and calcOverlapFiltered
// (LaueMatchingHeaders.h:513-561, :564-636) as problem_function (:640-694)
// calls them, for many (grain, point) pairs in one launch.
//
// The reference evaluates the objective up to 200 times per grain inside
// NLopt, one grain per host thread.  Here the optimiser stays on the host and
// proposes one point (or a few) per grain per round; all grains' points of a
// round go to the device together.  The host forms each point's matrix
// T = Euler2OrientMat(x) . recip(x) with the C library's trigonometry (the
// same calls as the host objective), so the device part is pure IEEE FP64
// arithmetic (products, sums, quotients, square roots, each rounded alone as
// on the x86-64 host without FMA) and the objective is bit-identical.
//
// One warp per point.  Lanes project 32 of the grain's valid HKLs at once and
// gather their pixels; the spots are then taken in list order (the
// de-duplication by scattering direction depends on it): for each projected
// HKL the warp compares its direction with the spots kept so far (lanes over
// the kept list, one ballot), and the kept ones add their pixel value to the
// FP64 sum in order.  Prefiltering is one warp per grain over all HKLs with
// ballot compaction, which keeps the HKL order.
#include <algorithm>
#include <cstring>
#include <vector>

#include "kernels.cuh"
#include "refine.h"

namespace lmb {

namespace {

constexpr double kHc = 1.2398419739;                       // LaueMatchingHeaders.h:41
constexpr double kFourPiR = 4.0 * 3.14159265358979323846;  // 4 * M_PI as C folds it

struct RGeo {
  double rt[9];
  double p0, p1, p2;
  double px_x, px_y;
  double cx, cy;  // 0.5 * (nrPxX - 1), 0.5 * (nrPxY - 1)
  double wm1, hm1;  // nrPxX - 1, nrPxY - 1 as doubles
  double elo, ehi;
  int W, H;
};

// One reflection through the detector model in calcOverlapFiltered's order
// (:577-605).  prefilterHKLs (:531-555) writes kf as (-2 * dot) * qhat where
// this writes 0 - (2 * dot) * qhat: the two differ at most in the sign of a
// zero, which changes no comparison and no pixel.
__device__ __forceinline__ bool reflect(const double T[9], const int4 hk, const RGeo &g,
                                        double &h0, double &h1, double &h2, double &px,
                                        double &py) {
  const double h = (double)hk.x, k = (double)hk.y, l = (double)hk.z;
  const double q0 = dadd(dadd(dadd(0.0, dmul(T[0], h)), dmul(T[1], k)), dmul(T[2], l));
  const double q1 = dadd(dadd(dadd(0.0, dmul(T[3], h)), dmul(T[4], k)), dmul(T[5], l));
  const double q2 = dadd(dadd(dadd(0.0, dmul(T[6], h)), dmul(T[7], k)), dmul(T[8], l));
  const double ql = dsqrt(dadd(dadd(dmul(q0, q0), dmul(q1, q1)), dmul(q2, q2)));
  if (ql == 0.0) return false;
  h0 = ddiv(q0, ql);
  h1 = ddiv(q1, ql);
  h2 = ddiv(q2, ql);
  const double td = dmul(2.0, h2);
  const double k0 = dsub(0.0, dmul(td, h0));
  const double k1 = dsub(0.0, dmul(td, h1));
  const double k2 = dsub(1.0, dmul(td, h2));
  const double x = dadd(dadd(dadd(0.0, dmul(g.rt[0], k0)), dmul(g.rt[1], k1)), dmul(g.rt[2], k2));
  const double y = dadd(dadd(dadd(0.0, dmul(g.rt[3], k0)), dmul(g.rt[4], k1)), dmul(g.rt[5], k2));
  const double z = dadd(dadd(dadd(0.0, dmul(g.rt[6], k0)), dmul(g.rt[7], k1)), dmul(g.rt[8], k2));
  if (z <= 0.0) return false;
  const double xp = dsub(ddiv(dmul(x, g.p2), z), g.p0);
  const double yp = dsub(ddiv(dmul(y, g.p2), z), g.p1);
  px = dadd(ddiv(xp, g.px_x), g.cx);
  if (px < 0.0 || px > g.wm1) return false;
  py = dadd(ddiv(yp, g.px_y), g.cy);
  if (py < 0.0 || py > g.hm1) return false;
  const double e = ddiv(dmul(kHc, ql), dmul(kFourPiR, -h2));
  if (e < g.elo || e > g.ehi) return false;
  return true;
}

__device__ __forceinline__ void load_T(const double *__restrict__ T, int64_t k, double t[9]) {
#pragma unroll
  for (int i = 0; i < 9; i++) t[i] = __ldg(T + k * 9 + i);
}

// prefilterHKLs: valid[g][0..nvalid[g]) = HKL numbers that project onto the
// detector inside the energy band at grain g's coarse matrix, in HKL order.
__global__ void __launch_bounds__(128) prefilter_kernel(const double *__restrict__ T, int ng,
                                                        const int4 *__restrict__ hkl, int nh,
                                                        RGeo g, int32_t *__restrict__ valid,
                                                        int32_t *__restrict__ nvalid) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (gw >= ng) return;  // warp-uniform
  double t[9];
  load_T(T, gw, t);
  int cnt = 0;
  int32_t *out = valid + (size_t)gw * nh;
  for (int base = 0; base < nh; base += 32) {
    const int h = base + lane;
    bool ok = false;
    if (h < nh) {
      double a, b, c, px, py;
      ok = reflect(t, __ldg(hkl + h), g, a, b, c, px, py);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, ok);
    if (ok) out[cnt + __popc(bal & ((1u << lane) - 1u))] = h;
    cnt += __popc(bal);
  }
  if (lane == 0) nvalid[gw] = cnt;
}

// calcOverlapFiltered + problem_function's sign: obj[k] = -(nrPos * sqrt(sum))
// for point k (matrix T[k], grain grain[k]).  acc: per warp, the directions
// of the spots kept so far (max_spots x 3 doubles, outArrThis).
__global__ void __launch_bounds__(128, 7) objective_kernel(
    const double *__restrict__ T, const int32_t *__restrict__ grain, int64_t m,
    const int4 *__restrict__ hkl, int nh, const int32_t *__restrict__ valid,
    const int32_t *__restrict__ nvalid, const int32_t *__restrict__ gimg,
    const float *__restrict__ img, RGeo g, int max_spots, double *__restrict__ obj) {
  extern __shared__ double acc_all[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t k = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
  if (k >= m) return;  // warp-uniform
  double *acc = acc_all + (size_t)wib * max_spots * 3;
  double t[9];
  load_T(T, k, t);
  const int gi = __ldg(grain + k);
  const int nv = __ldg(nvalid + gi);
  const int32_t *vl = valid + (size_t)gi * nh;
  const float *im = img + (size_t)__ldg(gimg + gi) * (size_t)g.W * (size_t)g.H;
  double result = 0.0;
  int npos = 0, nspot = 0;
  bool done = false;
  for (int base = 0; base < nv && !done; base += 32) {
    const int vi = base + lane;
    bool ok = false;
    double h0 = 0, h1 = 0, h2 = 0;
    float v = 0.f;
    if (vi < nv) {
      double px, py;
      ok = reflect(t, __ldg(hkl + __ldg(vl + vi)), g, h0, h1, h2, px, py);
      if (ok) v = __ldg(im + ((size_t)py * (size_t)g.W + (size_t)px));
    }
    unsigned bal = __ballot_sync(0xffffffffu, ok);
    while (bal) {
      const int j = __ffs(bal) - 1;
      bal &= bal - 1u;
      const double c0 = __shfl_sync(0xffffffffu, h0, j);
      const double c1 = __shfl_sync(0xffffffffu, h1, j);
      const double c2 = __shfl_sync(0xffffffffu, h2, j);
      const float cv = __shfl_sync(0xffffffffu, v, j);
      bool seen = false;
      for (int a = lane; a < nspot; a += 32)
        seen |= (dmul(fabs(dsub(c0, acc[3 * a + 0])), 100000.0) < 0.1) &&
                (dmul(fabs(dsub(c1, acc[3 * a + 1])), 100000.0) < 0.1) &&
                (dmul(fabs(dsub(c2, acc[3 * a + 2])), 100000.0) < 0.1);
      if (__any_sync(0xffffffffu, seen)) continue;
      if (lane == 0) {
        acc[3 * nspot + 0] = c0;
        acc[3 * nspot + 1] = c1;
        acc[3 * nspot + 2] = c2;
      }
      __syncwarp();
      if (cv > 0.f) {
        result = dadd(result, (double)cv);
        npos++;
      }
      if (++nspot == max_spots) {
        done = true;
        break;
      }
    }
  }
  if (lane == 0) obj[k] = -dmul((double)npos, dsqrt(result));
}

template <class Tp>
int grow(Tp **p, size_t *cap, size_t need, bool pinned) {
  if (need <= *cap) return LMB_OK;
  size_t n = std::max(need, *cap * 2);
  if (*p) {
    if (pinned)
      cudaFreeHost(*p);
    else
      cudaFree(*p);
    *p = nullptr;
    *cap = 0;
  }
  const cudaError_t e = pinned ? cudaMallocHost((void **)p, n * sizeof(Tp))
                               : cudaMalloc((void **)p, n * sizeof(Tp));
  if (e != cudaSuccess) {
    *p = nullptr;
    set_error("refinement buffers: %s", cudaGetErrorString(e));
    return LMB_ERR_OOM;
  }
  *cap = n;
  return LMB_OK;
}

}  // namespace

// One set of evaluation buffers: the host stages m point matrices and their
// grain numbers in page-locked memory (T[m][9], then grain[m]), one copy moves
// them, the kernel writes m values, one copy brings them back.  Two sets let
// the host prepare one group of grains while the device evaluates the other.
struct EvalBuf {
  unsigned char *h_in = nullptr, *d_in = nullptr;
  double *h_out = nullptr, *d_out = nullptr;
  size_t h_in_cap = 0, d_in_cap = 0, h_out_cap = 0, d_out_cap = 0;
  int64_t m = 0;
  bool pending = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, done = nullptr;  // kernel start, end; copy back
};

struct RefineDev {
  int device = 0;
  RGeo g{};
  int nh = 0;
  int4 *hkl = nullptr;
  float *img = nullptr;
  size_t img_cap = 0;
  int n_img = 0;
  int32_t *gimg = nullptr, *valid = nullptr, *nvalid = nullptr;
  size_t gimg_cap = 0, valid_cap = 0, nvalid_cap = 0;
  int ng = 0;
  double *T = nullptr, *hT = nullptr;  // prefilter matrices
  size_t T_cap = 0, hT_cap = 0;
  EvalBuf buf[kRefineBufs];
  cudaStream_t st = nullptr;
};

int refine_dev_create(int device, const RefineGeoHost &gh, const int32_t *hkls, int nh,
                      RefineDev **out) {
  LMB_REQUIRE(out && nh >= 0 && (hkls || nh == 0) && gh.W > 0 && gh.H > 0, "bad argument");
  LMB_CUDA(cudaSetDevice(device));
  RefineDev *r = new RefineDev();
  r->device = device;
  RGeo &g = r->g;
  for (int i = 0; i < 9; i++) g.rt[i] = gh.rt[i];
  g.p0 = gh.p[0];
  g.p1 = gh.p[1];
  g.p2 = gh.p[2];
  g.px_x = gh.px_x;
  g.px_y = gh.px_y;
  g.cx = 0.5 * (gh.W - 1);
  g.cy = 0.5 * (gh.H - 1);
  g.wm1 = (double)(gh.W - 1);
  g.hm1 = (double)(gh.H - 1);
  g.elo = gh.elo;
  g.ehi = gh.ehi;
  g.W = gh.W;
  g.H = gh.H;
  r->nh = nh;
  int rc = LMB_OK;
  cudaError_t e = cudaStreamCreateWithFlags(&r->st, cudaStreamNonBlocking);
  for (int b = 0; b < kRefineBufs && e == cudaSuccess; b++) {
    e = cudaEventCreate(&r->buf[b].ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&r->buf[b].ev1);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->buf[b].done, cudaEventDisableTiming);
  }
  if (e == cudaSuccess && nh > 0) {
    std::vector<int4> h4(nh);
    for (int i = 0; i < nh; i++) h4[i] = make_int4(hkls[3 * i], hkls[3 * i + 1], hkls[3 * i + 2], 0);
    e = cudaMalloc((void **)&r->hkl, sizeof(int4) * nh);
    if (e == cudaSuccess)
      e = cudaMemcpy(r->hkl, h4.data(), sizeof(int4) * nh, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) rc = cuda_fail(e, "refinement set-up", __FILE__, __LINE__);
  if (rc) {
    refine_dev_destroy(r);
    return rc;
  }
  *out = r;
  return LMB_OK;
}

void refine_dev_destroy(RefineDev *r) {
  if (!r) return;
  cudaSetDevice(r->device);
  if (r->st) cudaStreamSynchronize(r->st);
  cudaFree(r->hkl);
  cudaFree(r->img);
  cudaFree(r->gimg);
  cudaFree(r->valid);
  cudaFree(r->nvalid);
  cudaFree(r->T);
  cudaFreeHost(r->hT);
  for (EvalBuf &b : r->buf) {
    cudaFreeHost(b.h_in);
    cudaFreeHost(b.h_out);
    cudaFree(b.d_in);
    cudaFree(b.d_out);
    if (b.ev0) cudaEventDestroy(b.ev0);
    if (b.ev1) cudaEventDestroy(b.ev1);
    if (b.done) cudaEventDestroy(b.done);
  }
  if (r->st) cudaStreamDestroy(r->st);
  delete r;
}

int refine_dev_images(RefineDev *r, const float *const *frames, int n) {
  LMB_REQUIRE(r && n >= 0 && (frames || n == 0), "bad argument");
  LMB_CUDA(cudaSetDevice(r->device));
  const size_t npx = (size_t)r->g.W * r->g.H;
  int rc = grow(&r->img, &r->img_cap, std::max<size_t>(1, npx * n), false);
  if (rc) return rc;
  for (int i = 0; i < n; i++) {
    LMB_REQUIRE(frames[i], "null frame %d", i);
    LMB_CUDA(cudaMemcpyAsync(r->img + npx * i, frames[i], npx * sizeof(float),
                             cudaMemcpyHostToDevice, r->st));
  }
  LMB_CUDA(cudaStreamSynchronize(r->st));
  r->n_img = n;
  r->ng = 0;  // grains refer to image numbers of the previous set
  return LMB_OK;
}

int refine_dev_prefilter(RefineDev *r, const double *T, const int32_t *image, int ng,
                         int32_t *nvalid, int32_t *valid) {
  LMB_REQUIRE(r && ng >= 0 && (ng == 0 || (T && image && nvalid)), "bad argument");
  for (int i = 0; i < ng; i++)
    LMB_REQUIRE(image[i] >= 0 && image[i] < r->n_img, "grain %d: image %d outside the %d images",
                i, image[i], r->n_img);
  LMB_CUDA(cudaSetDevice(r->device));
  r->ng = 0;
  if (ng == 0) return LMB_OK;
  int rc = grow(&r->gimg, &r->gimg_cap, ng, false);
  if (!rc) rc = grow(&r->nvalid, &r->nvalid_cap, ng, false);
  if (!rc) rc = grow(&r->valid, &r->valid_cap, std::max<size_t>(1, (size_t)ng * r->nh), false);
  if (!rc) rc = grow(&r->T, &r->T_cap, (size_t)ng * 9, false);
  if (!rc) rc = grow(&r->hT, &r->hT_cap, (size_t)ng * 9, true);
  if (rc) return rc;
  memcpy(r->hT, T, sizeof(double) * 9 * ng);
  LMB_CUDA(cudaMemcpyAsync(r->T, r->hT, sizeof(double) * 9 * ng, cudaMemcpyHostToDevice, r->st));
  LMB_CUDA(cudaMemcpyAsync(r->gimg, image, sizeof(int32_t) * ng, cudaMemcpyHostToDevice, r->st));
  const int threads = 128, wpb = threads / 32;
  prefilter_kernel<<<(ng + wpb - 1) / wpb, threads, 0, r->st>>>(r->T, ng, r->hkl, r->nh, r->g,
                                                                  r->valid, r->nvalid);
  LMB_CUDA(cudaGetLastError());
  LMB_CUDA(cudaMemcpyAsync(nvalid, r->nvalid, sizeof(int32_t) * ng, cudaMemcpyDeviceToHost,
                           r->st));
  if (valid && r->nh > 0)
    LMB_CUDA(cudaMemcpyAsync(valid, r->valid, sizeof(int32_t) * ng * r->nh,
                             cudaMemcpyDeviceToHost, r->st));
  LMB_CUDA(cudaStreamSynchronize(r->st));
  r->ng = ng;
  return LMB_OK;
}

int refine_dev_stage(RefineDev *r, int b, int64_t m, double **T, int32_t **grain) {
  LMB_REQUIRE(r && b >= 0 && b < kRefineBufs && m >= 0 && m <= (int64_t)1 << 30 && T && grain,
              "bad argument");
  EvalBuf &B = r->buf[b];
  LMB_REQUIRE(!B.pending, "evaluation buffer %d still in flight", b);
  LMB_CUDA(cudaSetDevice(r->device));
  const size_t in_bytes = (size_t)m * (9 * sizeof(double) + sizeof(int32_t));
  int rc = grow(&B.h_in, &B.h_in_cap, std::max<size_t>(1, in_bytes), true);
  if (!rc) rc = grow(&B.h_out, &B.h_out_cap, std::max<size_t>(1, (size_t)m), true);
  if (rc) return rc;
  *T = reinterpret_cast<double *>(B.h_in);
  *grain = reinterpret_cast<int32_t *>(B.h_in + (size_t)m * 9 * sizeof(double));
  B.m = m;
  return LMB_OK;
}

int refine_dev_submit(RefineDev *r, int b, int max_spots) {
  LMB_REQUIRE(r && b >= 0 && b < kRefineBufs && max_spots >= 1, "bad argument");
  EvalBuf &B = r->buf[b];
  LMB_REQUIRE(!B.pending, "evaluation buffer %d still in flight", b);
  const int64_t m = B.m;
  if (m == 0) {
    B.pending = true;
    return LMB_OK;
  }
  const int32_t *grain = reinterpret_cast<const int32_t *>(B.h_in + (size_t)m * 9 * sizeof(double));
  for (int64_t i = 0; i < m; i++)
    LMB_REQUIRE(grain[i] >= 0 && grain[i] < r->ng, "point %lld: grain %d outside the %d grains",
                (long long)i, grain[i], r->ng);
  LMB_CUDA(cudaSetDevice(r->device));
  const size_t in_bytes = (size_t)m * (9 * sizeof(double) + sizeof(int32_t));
  int rc = grow(&B.d_in, &B.d_in_cap, in_bytes, false);
  if (!rc) rc = grow(&B.d_out, &B.d_out_cap, (size_t)m, false);
  if (rc) return rc;
  // warps per block: as many as fit 48 KiB of kept-spot directions, at most 4
  const size_t per_warp = sizeof(double) * 3 * (size_t)max_spots;
  const int wpb = (int)std::max<size_t>(1, std::min<size_t>(4, (48 * 1024) / per_warp));
  const size_t smem = per_warp * wpb;
  if (smem > 48 * 1024) {
    LMB_REQUIRE(smem <= 200 * 1024, "max_spots %d needs too much shared memory", max_spots);
    LMB_CUDA(cudaFuncSetAttribute(objective_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
  }
  LMB_CUDA(cudaMemcpyAsync(B.d_in, B.h_in, in_bytes, cudaMemcpyHostToDevice, r->st));
  LMB_CUDA(cudaEventRecord(B.ev0, r->st));
  const double *dT = reinterpret_cast<const double *>(B.d_in);
  const int32_t *dg = reinterpret_cast<const int32_t *>(B.d_in + (size_t)m * 9 * sizeof(double));
  const int64_t blocks = (m + wpb - 1) / wpb;
  objective_kernel<<<(unsigned)blocks, 32 * wpb, smem, r->st>>>(
      dT, dg, m, r->hkl, r->nh, r->valid, r->nvalid, r->gimg, r->img, r->g, max_spots, B.d_out);
  LMB_CUDA(cudaGetLastError());
  LMB_CUDA(cudaEventRecord(B.ev1, r->st));
  LMB_CUDA(cudaMemcpyAsync(B.h_out, B.d_out, sizeof(double) * m, cudaMemcpyDeviceToHost, r->st));
  LMB_CUDA(cudaEventRecord(B.done, r->st));
  B.pending = true;
  return LMB_OK;
}

int refine_dev_collect(RefineDev *r, int b, const double **objective, float *kernel_ms) {
  LMB_REQUIRE(r && b >= 0 && b < kRefineBufs && objective, "bad argument");
  EvalBuf &B = r->buf[b];
  LMB_REQUIRE(B.pending, "evaluation buffer %d was not submitted", b);
  B.pending = false;
  if (kernel_ms) *kernel_ms = 0.f;
  *objective = B.h_out;
  if (B.m == 0) return LMB_OK;
  LMB_CUDA(cudaSetDevice(r->device));
  LMB_CUDA(cudaEventSynchronize(B.done));
  if (kernel_ms) LMB_CUDA(cudaEventElapsedTime(kernel_ms, B.ev0, B.ev1));
  return LMB_OK;
}

}  // namespace lmb
