// Duplicate merge on the device: the pairwise misorientation matrix and the
// greedy clustering of mergeDuplicateOrientations (LaueMatchingHeaders.h:969-1065).
//
// The reference (and the host post-stage, post.cpp) computes, for every pair
// (l > g) of candidates in input order, the misorientation angle in FP64
// (GetMisOrientation, :247-260: both quaternions brought to the fundamental
// region, the relative rotation, brought down again), stores it as float and
// then merges greedily: candidate g, if not yet taken, takes every later
// untaken l with (float)angle <= MaxAngle and keeps the highest score (the
// first one on ties).  That is O(n^2) FP64 work with ~75 normalised
// quaternion products per pair, seconds on the host for 1e4 candidates.
//
// Here one thread evaluates 32 pairs (g, 32w..32w+31) and writes one bit word
// of "l merges into g" (column g, bits over l).  Every operation is the
// host's, in the host's order, rounded the same way (no contraction) except
// acos, for which CUDA's result may differ from the host library's in the last
// bits; a pair whose angle lands so close to the float rounding boundary at
// MaxAngle that such a difference could flip the comparison is listed and
// decided again on the host with the host's function.  The greedy pass runs
// in one block: a shared-memory bit set of taken candidates, each untaken g
// in order claims the set bits of its column, and a block reduction picks the
// best score.
#include <cmath>

#include "kernels.cuh"
#include "merge.h"

namespace lmb {

namespace {

__device__ __forceinline__ void d_normalize4(double q[4]) {
  const double n = dsqrt(dadd(dadd(dadd(dmul(q[0], q[0]), dmul(q[1], q[1])), dmul(q[2], q[2])),
                              dmul(q[3], q[3])));
  q[0] = ddiv(q[0], n);
  q[1] = ddiv(q[1], n);
  q[2] = ddiv(q[2], n);
  q[3] = ddiv(q[3], n);
}

// QuaternionProduct (LaueMatchingHeaders.h:166-178): w >= 0, normalised.
__device__ __forceinline__ void d_qmul(const double q[4], const double r[4], double Q[4]) {
  Q[0] = dsub(dsub(dsub(dmul(r[0], q[0]), dmul(r[1], q[1])), dmul(r[2], q[2])), dmul(r[3], q[3]));
  Q[1] = dsub(dadd(dadd(dmul(r[1], q[0]), dmul(r[0], q[1])), dmul(r[3], q[2])), dmul(r[2], q[3]));
  Q[2] = dsub(dadd(dadd(dmul(r[2], q[0]), dmul(r[0], q[2])), dmul(r[1], q[3])), dmul(r[3], q[1]));
  Q[3] = dsub(dadd(dadd(dmul(r[3], q[0]), dmul(r[0], q[3])), dmul(r[2], q[1])), dmul(r[1], q[2]));
  if (Q[0] < 0) {
    Q[0] = -Q[0];
    Q[1] = -Q[1];
    Q[2] = -Q[2];
    Q[3] = -Q[3];
  }
  d_normalize4(Q);
}

// BringDownToFundamentalRegion (:221-245): the first symmetry-equivalent with
// the largest w, normalised once more.
__device__ __forceinline__ void d_fundamental(const MergeArgs &a, const double in[4], double out[4]) {
  double best_w = -10000;
  for (int i = 0; i < a.nsym; i++) {
    double c[4];
    d_qmul(in, a.sym[i], c);
    if (best_w < c[0]) {
      best_w = c[0];
      out[0] = c[0];
      out[1] = c[1];
      out[2] = c[2];
      out[3] = c[3];
    }
  }
  d_normalize4(out);
}

__global__ void merge_fr_kernel(MergeArgs a) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  double q[4] = {a.quat[4 * i], a.quat[4 * i + 1], a.quat[4 * i + 2], a.quat[4 * i + 3]};
  double f[4];
  d_fundamental(a, q, f);
  for (int k = 0; k < 4; k++) a.fr[4 * i + k] = f[k];
}

// Column g, word w: bit b set when l = 32w + b > g and l merges into g.
__global__ void merge_pairs_kernel(MergeArgs a) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= a.n * a.W) return;
  const int64_t g = t / a.W, w = t % a.W;
  const int64_t l0 = 32 * w;
  uint32_t bits = 0;
  if (l0 + 31 > g) {
    // the reference evaluates GetMisOrientation(quat[l], quat[g]) for l > g:
    // the inverse of l's fundamental-region quaternion times g's
    const double gf[4] = {a.fr[4 * g], a.fr[4 * g + 1], a.fr[4 * g + 2], a.fr[4 * g + 3]};
    for (int b = 0; b < 32; b++) {
      const int64_t l = l0 + b;
      if (l <= g || l >= a.n) continue;
      const double li[4] = {-a.fr[4 * l], a.fr[4 * l + 1], a.fr[4 * l + 2], a.fr[4 * l + 3]};
      double p[4], m[4];
      d_qmul(li, gf, p);
      d_fundamental(a, p, m);
      if (m[0] > 1) m[0] = 1;
      const double ang = dmul(dmul(2.0, acos(m[0])), a.rad2deg);
      if (fabs(ang - a.mid) <= a.window) {  // too close to call: the host decides
        const unsigned k = atomicAdd(a.n_unsure, 1u);
        if (k < a.cap_unsure) {
          a.unsure[2 * k] = (uint32_t)l;
          a.unsure[2 * k + 1] = (uint32_t)g;
        }
        continue;
      }
      if ((double)__double2float_rn(ang) <= a.max_angle) bits |= 1u << b;
    }
  }
  a.bits[t] = bits;
}

// Greedy clustering in input order, one block.  done: shared bit set.
__global__ void __launch_bounds__(1024) merge_greedy_kernel(MergeArgs a) {
  extern __shared__ uint32_t done[];
  __shared__ double s_best[32];
  __shared__ int64_t s_bl[32];
  __shared__ int s_cnt[32];
  for (int64_t w = threadIdx.x; w < a.W; w += blockDim.x) done[w] = 0;
  __syncthreads();
  int nc = 0;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int64_t g = 0; g < a.n; g++) {
    if ((done[g >> 5] >> (g & 31)) & 1u) continue;  // block-uniform
    __syncthreads();
    if (threadIdx.x == 0) done[g >> 5] |= 1u << (g & 31);
    __syncthreads();
    double best = -INFINITY;
    int64_t bl = INT64_MAX;
    int cnt = 0;
    const uint32_t *col = a.bits + g * a.W;
    for (int64_t w = (g >> 5) + threadIdx.x; w < a.W; w += blockDim.x) {
      const uint32_t nb = col[w] & ~done[w];
      if (!nb) continue;
      done[w] |= nb;  // each word has one owner thread in this sweep
      cnt += __popc(nb);
      uint32_t m = nb;
      while (m) {
        const int b = __ffs(m) - 1;
        m &= m - 1;
        const int64_t l = 32 * w + b;
        const double s = a.score[l];
        if (s > best) {  // ascending l within the thread: first maximum
          best = s;
          bl = l;
        }
      }
    }
    // block reduction: largest score, smallest index on ties
    for (int o = 16; o; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int64_t ol = __shfl_xor_sync(0xffffffffu, bl, o);
      cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
      if (ob > best || (ob == best && ol < bl)) {
        best = ob;
        bl = ol;
      }
    }
    if (lane == 0) {
      s_best[wid] = best;
      s_bl[wid] = bl;
      s_cnt[wid] = cnt;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      // the merged candidates' best (first of the largest scores) replaces g
      // only when strictly larger, as the host's ascending scan does
      double mb = -INFINITY;
      int64_t ml = INT64_MAX;
      int c0 = 1;
      for (int k = 0; k < nw; k++) {
        c0 += s_cnt[k];
        if (s_best[k] > mb || (s_best[k] == mb && s_bl[k] < ml)) {
          mb = s_best[k];
          ml = s_bl[k];
        }
      }
      a.out_best[nc] = (mb > a.score[g]) ? ml : g;
      a.out_count[nc] = c0;
    }
    nc++;
    __syncthreads();
  }
  if (threadIdx.x == 0) *a.n_clusters = nc;
}

}  // namespace

int merge_device_run(const MergeHost &h, int32_t *n_clusters, int64_t *best_idx, int32_t *counts,
                     std::vector<std::pair<uint32_t, uint32_t>> *unsure_out, bool *overflow) {
  const int64_t n = h.n;
  *n_clusters = 0;
  *overflow = false;
  if (n <= 0) return LMB_OK;
  LMB_CUDA(cudaSetDevice(h.device));
  const int64_t W = (n + 31) / 32;
  LMB_REQUIRE(n <= 200000, "%lld candidates exceed the device merge (at most 200000; its "
              "pair matrix takes n*n/8 bytes)", (long long)n);
  cudaStream_t st = nullptr;
  LMB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  // one stream-ordered allocation for everything (no device-wide synchronisation)
  const size_t b_quat = (size_t)n * 32, b_score = (size_t)n * 8, b_bits = (size_t)n * W * 4;
  const size_t cap_unsure = 1u << 16;
  const size_t b_unsure = cap_unsure * 8, b_out = (size_t)n * 12 + 16;
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t total = 2 * al(b_quat) + al(b_score) + al(b_bits) + al(b_unsure) + al(b_out) + 256;
  char *mem = nullptr;
  cudaError_t ce = cudaMallocAsync((void **)&mem, total, st);
  int rc = LMB_OK;
  MergeArgs a{};
  if (ce == cudaSuccess) {
    size_t o = 0;
    auto take = [&](size_t b) {
      char *p = mem + o;
      o += al(b);
      return p;
    };
    a.quat = reinterpret_cast<double *>(take(b_quat));
    a.fr = reinterpret_cast<double *>(take(b_quat));
    a.score = reinterpret_cast<double *>(take(b_score));
    a.bits = reinterpret_cast<uint32_t *>(take(b_bits));
    a.unsure = reinterpret_cast<uint32_t *>(take(b_unsure));
    char *outp = take(b_out);
    a.out_best = reinterpret_cast<int64_t *>(outp);
    a.out_count = reinterpret_cast<int32_t *>(outp + (size_t)n * 8);
    a.n_unsure = reinterpret_cast<unsigned *>(take(256));
    a.n_clusters = reinterpret_cast<int *>(reinterpret_cast<char *>(a.n_unsure) + 8);
    a.n = n;
    a.W = W;
    a.cap_unsure = (unsigned)cap_unsure;
    a.nsym = h.nsym;
    for (int i = 0; i < 24; i++)
      for (int j = 0; j < 4; j++) a.sym[i][j] = h.sym[i][j];
    a.max_angle = h.max_angle;
    a.rad2deg = h.rad2deg;
    a.mid = h.mid;
    a.window = h.window;
    ce = cudaMemcpyAsync(a.quat, h.quat, b_quat, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(a.score, h.score, b_score, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(a.n_unsure, 0, 256, st);
    if (ce == cudaSuccess) {
      merge_fr_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a);
      const int64_t th = n * W;
      merge_pairs_kernel<<<(unsigned)((th + 255) / 256), 256, 0, st>>>(a);
      ce = cudaGetLastError();
    }
    unsigned nu = 0;
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&nu, a.n_unsure, 4, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce == cudaSuccess && nu > cap_unsure) *overflow = true;
    if (ce == cudaSuccess && !*overflow && nu) {
      // decide the close calls with the host's own function, patch their bits
      std::vector<uint32_t> u((size_t)nu * 2);
      ce = cudaMemcpyAsync(u.data(), a.unsure, u.size() * 4, cudaMemcpyDeviceToHost, st);
      if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
      std::vector<uint32_t> words;
      std::vector<int64_t> where;
      if (ce == cudaSuccess) {
        for (unsigned k = 0; k < nu; k++) unsure_out->push_back({u[2 * k], u[2 * k + 1]});
        // read-modify-write of the affected words on the host side
        for (unsigned k = 0; k < nu; k++) {
          const int64_t l = u[2 * k], g = u[2 * k + 1];
          if (h.decide(h.ctx, l, g)) where.push_back(g * W + l / 32), words.push_back(1u << (l % 32));
        }
      }
      for (size_t k = 0; k < where.size() && ce == cudaSuccess; k++) {
        uint32_t cur = 0;
        ce = cudaMemcpyAsync(&cur, a.bits + where[k], 4, cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
        cur |= words[k];
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(a.bits + where[k], &cur, 4, cudaMemcpyHostToDevice, st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
      }
    }
    if (ce == cudaSuccess && !*overflow) {
      const int smem = (int)(W * 4);
      if (smem > 48 * 1024)
        ce = cudaFuncSetAttribute(merge_greedy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  smem);
      if (ce == cudaSuccess) {
        merge_greedy_kernel<<<1, 1024, smem, st>>>(a);
        ce = cudaGetLastError();
      }
      int nc = 0;
      if (ce == cudaSuccess) ce = cudaMemcpyAsync(&nc, a.n_clusters, 4, cudaMemcpyDeviceToHost, st);
      if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
      if (ce == cudaSuccess && nc > 0) {
        ce = cudaMemcpyAsync(best_idx, a.out_best, (size_t)nc * 8, cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess)
          ce = cudaMemcpyAsync(counts, a.out_count, (size_t)nc * 4, cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
      }
      *n_clusters = nc;
    }
    cudaFreeAsync(mem, st);
  }
  const cudaError_t se = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (ce != cudaSuccess) rc = cuda_fail(ce, "device duplicate merge", __FILE__, __LINE__);
  else if (se != cudaSuccess) rc = cuda_fail(se, "device duplicate merge", __FILE__, __LINE__);
  return rc;
}

}  // namespace lmb
