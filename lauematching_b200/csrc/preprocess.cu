// Frame preprocessing on the device: the steps of preprocess_image
// (laue_index/preprocess.py:221-338) as the reference runs them with numpy,
// scipy and OpenCV, with identical results:
//
//   background   exact square median (scipy.ndimage.median_filter, mirrored
//                borders): pixels become ranks among the frame's distinct
//                values; one warp per (column, row segment) slides its window
//                down, keeping 8-bit-digit rank histograms level by level and
//                refilling a deeper level only when the digit above it moves.
//   threshold    order statistics (np.median, np.percentile) by radix
//                selection over order-preserving 64-bit keys, on the device.
//   components   union-find over 8-neighbours (atomicMin on the parent
//                array); OpenCV numbers components by the raster order of
//                the first 2x2 pixel block each touches, so labels come from
//                a prefix sum over per-block flags.
//   centres      integer moments per component (exact), one division each.
//   blur width   closest pair of centres: cell grid, brute force when the
//                pair is farther apart than a cell.
//   blur         separable float64 passes in scipy's summation order.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <cmath>
#include <cstring>
#include <limits>
#include <type_traits>

#include "common.cuh"
#include "kernels.cuh"

using namespace lmb;

namespace {

constexpr int kT = 256;            // threads of the elementwise kernels
constexpr int kMedWarps = 8;       // warps per median block
constexpr int kMedLevels = 4;      // 8-bit digits of a rank (ranks < 2^32)
constexpr int kCell = 32;          // cell side of the closest-pair grid (pixels)
constexpr int kKeepShift = 40;     // the 8-bit pass that reads the frame and keeps its keys
constexpr int kHist16Threads = 1024;
constexpr size_t kHist16Smem = 32768 * sizeof(unsigned);  // 65536 packed 16-bit counters
constexpr int kPreEvents = 12;
enum PreEv : int {
  EV_SEG0 = 0, EV_SEG_UP, EV_SEG_THR, EV_SEG_CC, EV_BLUR0, EV_BLUR_K, EV_BLUR_DL, EV_MED0, EV_MED_UP,
  EV_MED_RANK, EV_MED_K, EV_MED_PASS
};

enum SelMode : int { SEL_NZ = 0, SEL_ABSDEV = 1, SEL_ALL = 2 };

// ---- small helpers -----------------------------------------------------------
// scipy's 'reflect' border (d c b a | a b c d | d c b a), periodic.
__host__ __device__ __forceinline__ int mirror(int i, int n) {
  if (i >= 0 && i < n) return i;
  if (n == 1) return 0;
  const int p = 2 * n;
  i %= p;
  if (i < 0) i += p;
  return i < n ? i : p - 1 - i;
}

// Order-preserving key of a double (total order; -0 sorts just below +0).
__device__ __forceinline__ unsigned long long okey(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double okey_value(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

// numpy's float64 -> uint16 (x86-64): truncate to int32, keep 16 bits.
__device__ __forceinline__ uint16_t u16_cast(double v) {
  return (uint16_t)((unsigned)x86_trunc_i32(v) & 0xFFFFu);
}

template <typename T>
__device__ __forceinline__ double to_f64(T v) {
  return (double)v;
}

size_t grid_for(size_t n, int num_sms) {
  return std::max<size_t>(1, std::min<size_t>((n + kT - 1) / kT, (size_t)num_sms * 16));
}

// ---- device state of one frame -----------------------------------------------
struct Select {
  unsigned long long n;          // candidates
  unsigned long long k[2];       // residual ranks sought (k[1] = k[0] + 1 when two)
  unsigned long long prefix[2];  // key bits fixed so far
  unsigned long long n_compact;  // candidates kept for the later passes
  unsigned long long kmin[2], kmax[2];  // extremes of the keys under each prefix (this pass)
  int two;
  int valid;
  int done[2];                   // the rank's key is known (all keys under its prefix equal)
  int pad;
};

struct PreState {
  Select sel;
  __align__(16) unsigned int hist[2][256];
  double med;
  double thresh;
  unsigned int blocks_done;  // blocks of the running selection pass that finished
  unsigned int nonint;       // a candidate value was not an integer in [0, 65535]
  unsigned int value_path;   // the threshold came from the value histogram
  unsigned int n_comp;      // components
  unsigned int n_labels;    // components + 1
  unsigned int n_keep;      // components with area >= min_area
  unsigned long long best;  // bits of the smallest squared centre distance
};

static_assert(offsetof(PreState, hist) % 16 == 0, "histogram rows are read as 16-byte vectors");

// ---- conversions -------------------------------------------------------------
template <typename T>
__global__ void to_f64_kernel(const T *__restrict__ in, double *__restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = to_f64(in[i]);
}

// np.maximum(raw - background, 0.0): NaN stays NaN, -0 stays -0.
template <typename T>
__global__ void subtract_kernel(const T *__restrict__ raw, const double *__restrict__ bg,
                                double *__restrict__ sub, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double d = lmb::dsub(to_f64(raw[i]), bg[i]);
    sub[i] = (d >= 0.0 || isnan(d)) ? d : 0.0;
  }
}

// ---- order statistics ----------------------------------------------------------
__global__ void sel_init_kernel(PreState *st, int mode, unsigned long long n,
                                unsigned long long k0, int two, int new_frame) {
  const int t = threadIdx.x;
  for (int i = t; i < 512; i += blockDim.x) (&st->hist[0][0])[i] = 0;
  if (t == 0) {
    if (new_frame) {
      st->nonint = 0;
      st->value_path = 0;
    }
    Select &s = st->sel;
    s.n = mode == SEL_ALL ? n : 0;
    s.k[0] = k0;
    s.k[1] = k0 + 1;
    s.prefix[0] = s.prefix[1] = 0;
    s.n_compact = 0;
    s.kmin[0] = s.kmin[1] = ~0ull;
    s.kmax[0] = s.kmax[1] = 0;
    s.done[0] = s.done[1] = 0;
    s.two = mode == SEL_ALL ? two : 0;
    s.valid = 1;
  }
}

// Digit holding residual rank k among 256 bins, lane l holding bins
// 8l..8l+7 in c[]; one warp.
__device__ __forceinline__ unsigned warp_find_in(const unsigned (&c)[8], unsigned long long &k) {
  const int lane = threadIdx.x & 31;
  unsigned long long sum = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) sum += c[j];
  unsigned long long incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const unsigned long long excl = incl - sum;
  const unsigned msk = __ballot_sync(0xffffffffu, k < incl);
  const int f = msk ? __ffs(msk) - 1 : 31;
  unsigned digit = 0;
  unsigned long long r = 0;
  if (lane == f) {
    r = k - excl;
    int j = 0;
    while (j < 7 && r >= c[j]) r -= c[j++];
    digit = (unsigned)(lane * 8 + j);
  }
  digit = __shfl_sync(0xffffffffu, digit, f);
  k = __shfl_sync(0xffffffffu, r, f);
  return digit;
}

// The same over a 16-byte aligned shared-memory histogram.
__device__ __forceinline__ unsigned warp_find_digit(const unsigned *h, unsigned long long &k) {
  const int lane = threadIdx.x & 31;
  const uint4 a = reinterpret_cast<const uint4 *>(h)[lane * 2];
  const uint4 b = reinterpret_cast<const uint4 *>(h)[lane * 2 + 1];
  const unsigned c[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
  return warp_find_in(c, k);
}

// Per-thread run of equal digits, flushed into the block's histogram when the
// digit changes: a frame's values crowd a few bins, so most values only bump
// a register.
struct DigitRun {
  unsigned d = 0x100u, n = 0;
  __device__ __forceinline__ void add(unsigned *hh, unsigned dig) {
    if (dig == d) {
      ++n;
      return;
    }
    if (n) atomicAdd(hh + d, n);
    d = dig;
    n = 1;
  }
  __device__ __forceinline__ void flush(unsigned *hh) {
    if (n) atomicAdd(hh + d, n);
    n = 0;
  }
};

// After a pass (warp 0 of the grid's last block): fix the digit of each
// sought rank and clear the histograms.  Pass 0 also learns the candidate
// count (SEL_NZ / SEL_ABSDEV: the median's ranks, two for an even count).
__device__ void sel_pick(PreState *st, int mode, int shift) {
  Select &s = st->sel;
  const int lane = threadIdx.x & 31;
  unsigned c0[8], c1[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    c0[j] = __ldcg(&st->hist[0][lane * 8 + j]);
    c1[j] = __ldcg(&st->hist[1][lane * 8 + j]);
  }
  if (s.valid) {
    for (int L = 0; L < (s.two ? 2 : 1); ++L) {
      if (s.done[L]) continue;
      const int src = L;
      if (s.kmin[src] == s.kmax[src]) {  // every key under the prefix is this one
        if (lane == 0) {
          s.prefix[L] = s.kmin[src];
          s.done[L] = 1;
        }
        __syncwarp();
        continue;
      }
      unsigned long long k = s.k[L];
      const unsigned d = warp_find_in(src == 0 ? c0 : c1, k);
      if (lane == 0) {
        s.k[L] = k;
        s.prefix[L] |= (unsigned long long)d << shift;
      }
      __syncwarp();
    }
  }
  __syncwarp();
  if (lane == 0) {
    s.kmin[0] = s.kmin[1] = ~0ull;
    s.kmax[0] = s.kmax[1] = 0;
  }
  for (int j = lane; j < 512; j += 32) (&st->hist[0][0])[j] = 0;
}

// Key of a selection candidate: non-negative values (every candidate of
// SEL_NZ and SEL_ABSDEV) only need the sign bit set.
__device__ __forceinline__ unsigned long long sel_key(int mode, double v) {
  return mode == SEL_ALL ? okey(v)
                         : ((unsigned long long)__double_as_longlong(v) | 0x8000000000000000ull);
}

// One radix pass: histogram of the digit at `shift` of the candidates whose
// higher digits equal each sought rank's prefix.  Passes 0..2 read the frame
// (pass 2 also keeps the surviving keys), later passes read those keys.  The
// last block to finish picks the digits for the next pass.
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
  for (int o = 16; o; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
  for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__global__ void __launch_bounds__(kT, 4)
    sel_hist_kernel(const double *frame, size_t n, PreState *st, int mode, int shift,
                    unsigned long long *compact) {
  constexpr int U = 8;  // values per thread per round
  __shared__ unsigned int h[2][256];
  __shared__ Select ss;
  __shared__ bool last;
  __shared__ unsigned long long stage[kT * U];  // kept keys of one round
  __shared__ unsigned n_stage;
  __shared__ unsigned long long base_s;
  __shared__ unsigned long long ext[4][kT / 32];
  for (int i = threadIdx.x; i < 512; i += blockDim.x) (&h[0][0])[i] = 0;
  if (threadIdx.x == 0) {
    ss = st->sel;
    n_stage = 0;
  }
  __syncthreads();
  const Select s = ss;
  const bool two = s.two != 0;
  // ranks whose key is known already need no more passes
  if (!s.valid || (s.done[0] && (!two || s.done[1]))) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool act0 = !s.done[0], act1 = two && !s.done[1];
  const unsigned long long hi = ~0ull << (shift + 8);
  const unsigned long long p0 = s.prefix[0] & hi, p1 = s.prefix[1] & hi;
  const double med = st->med;
  const bool from_frame = shift >= kKeepShift;
  const bool keep = shift == kKeepShift;
  const unsigned m = from_frame ? (unsigned)n : (unsigned)s.n_compact;
  const unsigned stride = gridDim.x * blockDim.x;
  const unsigned rounds = (m + stride * U - 1) / (stride * U);
  DigitRun run0, run1;
  unsigned long long mn0 = ~0ull, mx0 = 0, mn1 = ~0ull, mx1 = 0;
  for (unsigned it = 0; it < rounds; ++it) {
    unsigned long long key[U];
    bool hit0[U], hit1[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const unsigned i = (it * U + u) * stride + blockIdx.x * blockDim.x + threadIdx.x;
      hit0[u] = hit1[u] = false;
      key[u] = 0;
      if (i < m) {
        bool cand = true;
        if (from_frame) {
          const double v = frame[i];
          cand = mode == SEL_ALL || v > 0.0;
          key[u] = sel_key(mode, mode == SEL_ABSDEV ? fabs(lmb::dsub(v, med)) : v);
        } else {
          key[u] = compact[i];
        }
        hit0[u] = cand && act0 && (key[u] & hi) == p0;
        hit1[u] = cand && act1 && (key[u] & hi) == p1;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const unsigned d = (unsigned)(key[u] >> shift) & 255u;
      if (hit0[u]) {
        run0.add(h[0], d);
        mn0 = min(mn0, key[u]);
        mx0 = max(mx0, key[u]);
      }
      if (hit1[u]) {
        run1.add(h[1], d);
        mn1 = min(mn1, key[u]);
        mx1 = max(mx1, key[u]);
      }
      if (keep) {  // warp-aggregated slot in the block's staging area
        const bool k = hit0[u] || hit1[u];
        const unsigned msk = __ballot_sync(0xffffffffu, k);
        if (msk) {
          unsigned base = 0;
          if (lane == __ffs(msk) - 1) base = atomicAdd(&n_stage, (unsigned)__popc(msk));
          base = __shfl_sync(0xffffffffu, base, __ffs(msk) - 1);
          if (k) stage[base + __popc(msk & ((1u << lane) - 1u))] = key[u];
        }
      }
    }
    if (keep) {  // one reservation per block and round for the kept keys
      __syncthreads();
      const unsigned ns = n_stage;
      if (threadIdx.x == 0 && ns) base_s = atomicAdd(&st->sel.n_compact, (unsigned long long)ns);
      __syncthreads();
      for (unsigned q = threadIdx.x; q < ns; q += blockDim.x) compact[base_s + q] = stage[q];
      __syncthreads();
      if (threadIdx.x == 0) n_stage = 0;
      __syncthreads();
    }
  }
  run0.flush(h[0]);
  run1.flush(h[1]);
  mn0 = warp_min_u64(mn0);
  mx0 = warp_max_u64(mx0);
  mn1 = warp_min_u64(mn1);
  mx1 = warp_max_u64(mx1);
  if (lane == 0) {
    ext[0][warp] = mn0;
    ext[1][warp] = mx0;
    ext[2][warp] = mn1;
    ext[3][warp] = mx1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kT / 32; ++w) {
      mn0 = min(mn0, ext[0][w]);
      mx0 = max(mx0, ext[1][w]);
      mn1 = min(mn1, ext[2][w]);
      mx1 = max(mx1, ext[3][w]);
    }
    if (mn0 != ~0ull) {
      atomicMin(&st->sel.kmin[0], mn0);
      atomicMax(&st->sel.kmax[0], mx0);
    }
    if (mn1 != ~0ull) {
      atomicMin(&st->sel.kmin[1], mn1);
      atomicMax(&st->sel.kmax[1], mx1);
    }
  }
  for (int i = threadIdx.x; i < 512; i += blockDim.x) {
    const unsigned v = (&h[0][0])[i];
    if (v) atomicAdd(&(&st->hist[0][0])[i], v);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&st->blocks_done, 1u) == gridDim.x - 1;
  __syncthreads();
  if (last && threadIdx.x < 32) {
    __threadfence();
    sel_pick(st, mode, shift);
    if (threadIdx.x == 0) st->blocks_done = 0;
  }
}

// ---- first selection pass: 16-bit digits --------------------------------------
// The top 16 key bits (sign, exponent, 4 mantissa bits) of every candidate are
// counted in 65536 packed 16-bit counters in shared memory (a block handles at
// most 65535 values), flushed to a 65536-bin histogram in global memory; the
// grid's last block finds the bins of the sought ranks with all its threads.
struct Digit16Run {
  unsigned d = 0xffffffffu, n = 0;
  __device__ __forceinline__ void add(unsigned *words, unsigned dig) {
    if (dig == d) {
      ++n;
      return;
    }
    flush(words);
    d = dig;
    n = 1;
  }
  __device__ __forceinline__ void flush(unsigned *words) {
    if (n) atomicAdd(words + (d >> 1), n << (16 * (d & 1)));
    n = 0;
  }
};

__device__ __forceinline__ unsigned key16(int mode, double v) {
  return (unsigned)(sel_key(mode, v) >> 48);
}

// Block of 1024 threads: each owns 64 consecutive bins.
__device__ void sel_pick16(PreState *st, unsigned *g16, int mode) {
  __shared__ unsigned long long warp_tot[32];
  __shared__ unsigned long long total_s;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const uint4 *src = reinterpret_cast<const uint4 *>(g16 + t * 64);
  unsigned long long mine = 0;
  {
    uint4 q[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) q[j] = __ldcg(src + j);
#pragma unroll
    for (int j = 0; j < 16; ++j) mine += (unsigned long long)q[j].x + q[j].y + q[j].z + q[j].w;
  }
  unsigned long long incl = mine;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warp_tot[w] = incl;
  __syncthreads();
  if (w == 0) {
    unsigned long long v = warp_tot[lane], x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long u = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += u;
    }
    warp_tot[lane] = x - v;  // exclusive prefix of the warps
    if (lane == 31) total_s = x;
  }
  __syncthreads();
  const unsigned long long excl = warp_tot[w] + incl - mine;
  Select &s = st->sel;
  if (t == 0) {
    const unsigned long long tot = total_s;
    if (mode != SEL_ALL) {
      s.n = tot;
      s.k[0] = tot ? (tot - 1) / 2 : 0;
      s.k[1] = s.k[0] + 1;
      s.two = tot > 0 && (tot % 2) == 0;
    }
    if (s.n == 0) s.valid = 0;
  }
  __syncthreads();
  if (s.valid) {
    for (int L = 0; L < (s.two ? 2 : 1); ++L) {
      const unsigned long long k = s.k[L];
      if (k >= excl && k < excl + mine) {
        unsigned long long r = k - excl;
        int jj = 63;
        for (int j = 0; j < 16 && jj == 63; ++j) {
          const uint4 q = __ldcg(src + j);
          const unsigned cc[4] = {q.x, q.y, q.z, q.w};
          for (int e = 0; e < 4; ++e) {
            if (4 * j + e == 63) break;
            if (r < cc[e]) {
              jj = 4 * j + e;
              break;
            }
            r -= cc[e];
          }
        }
        s.k[L] = r;
        s.prefix[L] = (unsigned long long)(t * 64 + jj) << 48;
      }
    }
  }
  __syncthreads();
  uint4 *dst = reinterpret_cast<uint4 *>(g16 + t * 64);
#pragma unroll
  for (int j = 0; j < 16; ++j) dst[j] = make_uint4(0, 0, 0, 0);
}

// Pass A over the subtracted frame.
__global__ void __launch_bounds__(kHist16Threads, 1)
    sel_hist16_kernel(const double *__restrict__ sub, unsigned n, PreState *st, unsigned *g16,
                      int mode) {
  extern __shared__ unsigned words[];
  __shared__ bool last;
  for (int i = threadIdx.x; i < 32768; i += blockDim.x) words[i] = 0;
  __syncthreads();
  const double med = st->med;
  Digit16Run run;
  constexpr int U = 4;
  const unsigned stride = gridDim.x * blockDim.x;
  const unsigned rounds = (n + stride * U - 1) / (stride * U);
  for (unsigned it = 0; it < rounds; ++it) {
    double v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const unsigned i = (it * U + u) * stride + blockIdx.x * blockDim.x + threadIdx.x;
      v[u] = i < n ? sub[i] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const unsigned i = (it * U + u) * stride + blockIdx.x * blockDim.x + threadIdx.x;
      if (i < n && (mode == SEL_ALL || v[u] > 0.0))
        run.add(words, key16(mode, mode == SEL_ABSDEV ? fabs(lmb::dsub(v[u], med)) : v[u]));
    }
  }
  run.flush(words);
  __syncthreads();
  for (int wd = threadIdx.x; wd < 32768; wd += blockDim.x) {
    const unsigned x = words[wd];
    if (x & 0xffffu) atomicAdd(g16 + 2 * wd, x & 0xffffu);
    if (x >> 16) atomicAdd(g16 + 2 * wd + 1, x >> 16);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&st->blocks_done, 1u) == gridDim.x - 1;
  __syncthreads();
  if (last) {
    __threadfence();
    sel_pick16(st, g16, mode);
    if (threadIdx.x == 0) st->blocks_done = 0;
  }
}

// ---- threshold statistics of integer-valued frames ---------------------------------
// A detector frame minus a median background holds integers.  When every
// candidate value is an integer in [0, 65535], one pass counts the values
// themselves (65536 packed 16-bit counters per block, flushed into the global
// histogram); the grid's last block turns the histogram into prefix sums and
// finds the order statistics by binary search: np.median / np.percentile
// directly, and the median of |v - median| as the smallest distance d with
// more than k values within d of the median.  Any other value (fraction,
// negative zero, NaN, above 65535) leaves the work to the radix selection.
__device__ __forceinline__ unsigned long long vh_count_le(const unsigned *P, int v) {
  return v < 0 ? 0ull : (unsigned long long)__ldcg(P + v);
}

// Smallest x in [lo, hi] with pred(x), pred monotone and true at hi; the
// whole warp probes 32 points per round.
template <typename Pred>
__device__ long long warp_search(long long lo, long long hi, Pred pred) {
  const int lane = threadIdx.x & 31;
  while (hi - lo + 1 > 32) {
    const long long step = (hi - lo + 1 + 31) / 32;
    long long x = lo + (long long)(lane + 1) * step - 1;
    if (x > hi) x = hi;
    const unsigned m = __ballot_sync(0xffffffffu, pred(x));
    const int f = __ffs(m) - 1;
    long long nhi = lo + (long long)(f + 1) * step - 1;
    if (nhi > hi) nhi = hi;
    lo = lo + (long long)f * step;
    hi = nhi;
  }
  const long long x = lo + lane;
  const unsigned m = __ballot_sync(0xffffffffu, x <= hi && pred(x));
  return lo + __ffs(m) - 1;
}

// Smallest value v >= lo with more than r values in [lo, v].
__device__ int vh_rank(const unsigned *P, int lo, unsigned long long r) {
  const unsigned long long base = vh_count_le(P, lo - 1);
  return (int)warp_search(lo, 65535, [&](long long v) {
    return vh_count_le(P, (int)v) - base > r;
  });
}

// Values in [lo, 65535] within t/2 of med.
__device__ unsigned long long vh_within(const unsigned *P, int lo, double med, long long t) {
  const double h = 0.5 * (double)t;
  long long a = (long long)ceil(med - h), b = (long long)floor(med + h);
  if (a < lo) a = lo;
  if (b > 65535) b = 65535;
  if (b < a) return 0ull;
  return vh_count_le(P, (int)b) - vh_count_le(P, (int)a - 1);
}

// Smallest distance (a multiple of 1/2) with more than r values within it.
__device__ double vh_dist(const unsigned *P, int lo, double med, unsigned long long r) {
  const long long t = warp_search(0, 2 * 65536, [&](long long x) {
    return vh_within(P, lo, med, x) > r;
  });
  return 0.5 * (double)t;
}

// Last block (1024 threads): prefix sums in place, then the threshold (warp 0).
__device__ void vh_finish(PreState *st, unsigned *g16, int mode, unsigned long long k0, int two,
                          double gamma) {
  __shared__ unsigned long long warp_tot[32];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int nq = 65536 / 4 / blockDim.x;  // uint4 words of bins per thread
  uint4 *src = reinterpret_cast<uint4 *>(g16) + (size_t)t * nq;
  unsigned mine = 0;
  for (int j0 = 0; j0 < nq; j0 += 16) {
    uint4 q[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) q[j] = __ldcg(src + j0 + j);
#pragma unroll
    for (int j = 0; j < 16; ++j) mine += q[j].x + q[j].y + q[j].z + q[j].w;
  }
  unsigned long long incl = mine;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warp_tot[w] = incl;
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    unsigned long long v = lane < nw ? warp_tot[lane] : 0ull, x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long u = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += u;
    }
    if (lane < nw) warp_tot[lane] = x - v;
  }
  __syncthreads();
  unsigned run = (unsigned)(warp_tot[w] + incl - mine);  // counts fit 32 bits (frames < 2^31 px)
  for (int j = 0; j < nq; ++j) {
    uint4 q = __ldcg(src + j);
    q.x = (run += q.x);
    q.y = (run += q.y);
    q.z = (run += q.z);
    q.w = (run += q.w);
    src[j] = q;
  }
  __threadfence();
  __syncthreads();
  if (w == 0) {
    const unsigned *P = g16;
    double thresh;
    if (mode == SEL_ALL) {  // np.percentile over every pixel
      const double a = (double)vh_rank(P, 0, k0);
      const double b = two ? (double)vh_rank(P, 0, k0 + 1) : a;
      const double diff = lmb::dsub(b, a);
      thresh = lmb::dadd(a, lmb::dmul(diff, gamma));
      if (gamma >= 0.5) thresh = lmb::dsub(b, lmb::dmul(diff, lmb::dsub(1.0, gamma)));
    } else {  // the adaptive noise floor over the nonzero pixels
      const unsigned long long n = vh_count_le(P, 65535) - vh_count_le(P, 0);
      if (n == 0) {
        thresh = 1.0;
      } else {
        const unsigned long long k = (n - 1) / 2;
        const bool even = (n % 2) == 0;
        const double a = (double)vh_rank(P, 1, k);
        const double med =
            even ? lmb::ddiv(lmb::dadd(a, (double)vh_rank(P, 1, k + 1)), 2.0) : a;
        const double m1 = vh_dist(P, 1, med, k);
        const double md = even ? lmb::ddiv(lmb::dadd(m1, vh_dist(P, 1, med, k + 1)), 2.0) : m1;
        const double mad = lmb::dmul(1.4826, md);
        const double thr = lmb::dadd(med, lmb::dmul(4.0, mad));
        thresh = (1.0 > thr) ? 1.0 : thr;
      }
    }
    if (lane == 0) {
      st->thresh = thresh;
      st->value_path = 1;
    }
  }
  __syncthreads();
  for (int j = 0; j < nq; ++j) src[j] = make_uint4(0, 0, 0, 0);
}

// Subtraction fused with the value histogram (see above).  Each block counts
// values below kVhLocal in shared memory (runs of equal values in registers)
// and adds larger ones straight into the global 65536-bin histogram.
constexpr int kVhLocal = 4096;
constexpr int kVhThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kVhThreads, 4)
    value_hist_kernel(const T *__restrict__ raw, const double *__restrict__ bg,
                      double *__restrict__ sub, unsigned n, PreState *st, unsigned *g16, int mode,
                      unsigned long long k0, int two, double gamma) {
  __shared__ unsigned h[kVhLocal];
  __shared__ bool last;
  __shared__ int nonint_s;
  for (int i = threadIdx.x; i < kVhLocal; i += blockDim.x) h[i] = 0;
  if (threadIdx.x == 0) nonint_s = 0;
  __syncthreads();
  DigitRun run;  // bins below kVhLocal
  bool nonint = false;
  constexpr int U = 8;
  const unsigned stride = gridDim.x * blockDim.x;
  const unsigned rounds = (n + stride * U - 1) / (stride * U);
  for (unsigned it = 0; it < rounds; ++it) {
    double v[U];
    bool in[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const unsigned i = (it * U + u) * stride + blockIdx.x * blockDim.x + threadIdx.x;
      in[u] = i < n;
      v[u] = 0.0;
      if (in[u]) {
        const double d = lmb::dsub(to_f64(raw[i]), bg[i]);
        v[u] = (d >= 0.0 || isnan(d)) ? d : 0.0;
        sub[i] = v[u];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!in[u] || !(mode == SEL_ALL || v[u] > 0.0)) continue;
      const double x = v[u];
      if (x == trunc(x) && x <= 65535.0 && !signbit(x)) {
        const unsigned b = (unsigned)x;
        if (b < (unsigned)kVhLocal) run.add(h, b);
        else atomicAdd(g16 + b, 1u);
      } else {
        nonint = true;  // also NaN: every comparison with it is false
      }
    }
  }
  run.flush(h);
  if (nonint) nonint_s = 1;
  __syncthreads();
  if (threadIdx.x == 0 && nonint_s) atomicOr(&st->nonint, 1u);
  for (int b = threadIdx.x; b < kVhLocal; b += blockDim.x)
    if (h[b]) atomicAdd(g16 + b, h[b]);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&st->blocks_done, 1u) == gridDim.x - 1;
  __syncthreads();
  if (last) {
    __threadfence();
    if (__ldcg(&st->nonint) == 0) {
      vh_finish(st, g16, mode, k0, two, gamma);
    } else {  // leave an empty histogram for the radix selection
      for (int q = threadIdx.x; q < 65536 / 4; q += blockDim.x)
        reinterpret_cast<uint4 *>(g16)[q] = make_uint4(0, 0, 0, 0);
    }
    if (threadIdx.x == 0) st->blocks_done = 0;
  }
}

__device__ __forceinline__ double sel_value(const Select &s, int L) {
  return okey_value(s.prefix[L]);
}

// np.median of the candidates: the middle one, or the mean of the two.
__device__ __forceinline__ double sel_median(const Select &s) {
  const double a = sel_value(s, 0);
  return s.two ? lmb::ddiv(lmb::dadd(a, sel_value(s, 1)), 2.0) : a;
}

__global__ void finish_median_kernel(PreState *st) {
  st->med = st->sel.valid ? sel_median(st->sel) : 0.0;
}

// thresholds.py:35-45: max(med + 4 * (1.4826 * mad), 1.0); 1.0 without candidates.
__global__ void finish_adaptive_kernel(PreState *st) {
  if (!st->sel.valid) {
    st->thresh = 1.0;
    return;
  }
  const double mad = lmb::dmul(1.4826, sel_median(st->sel));
  const double t = lmb::dadd(st->med, lmb::dmul(4.0, mad));
  st->thresh = (1.0 > t) ? 1.0 : t;
}

// numpy's _lerp(a, b, gamma) of the two order statistics.
__global__ void finish_percentile_kernel(PreState *st, double gamma) {
  const Select &s = st->sel;
  const double a = sel_value(s, 0);
  const double b = s.two ? sel_value(s, 1) : a;
  const double diff = lmb::dsub(b, a);
  double r = lmb::dadd(a, lmb::dmul(diff, gamma));
  if (gamma >= 0.5) r = lmb::dsub(b, lmb::dmul(diff, lmb::dsub(1.0, gamma)));
  st->thresh = r;
}

__global__ void set_thresh_kernel(PreState *st, double t) { st->thresh = t; }

__global__ void reset_counts_kernel(PreState *st) {
  st->n_comp = 0;
  st->best = 0x7ff0000000000000ull;  // +inf
}

// ---- threshold, uint16, components ---------------------------------------------
// Threshold and uint16 cast (thresholds.py:29-32, preprocess.py:291), and
// the union-find parents along row runs (see init_parents_kernel).
__global__ void apply_kernel(const double *__restrict__ sub, const PreState *st,
                             uint16_t *__restrict__ t16, int *__restrict__ par, int nx, size_t n) {
  const double thr = st->thresh;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double v = sub[i];
    const uint16_t u = (v <= thr) ? (uint16_t)0 : u16_cast(v);
    t16[i] = u;
    bool left = false;
    if (u && (i % nx) != 0) {
      const double vl = sub[i - 1];
      left = !(vl <= thr) && u16_cast(vl) != 0;
    }
    par[i] = u ? (left ? (int)i - 1 : (int)i) : -1;
  }
}

// Parents start along row runs: a foreground pixel points at its left
// neighbour when that one is foreground too.
__global__ void init_parents_kernel(const uint16_t *t16, int *par, int nx, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    par[i] = t16[i] ? ((i % nx) != 0 && t16[i - 1] ? (int)i - 1 : (int)i) : -1;
}

__device__ __forceinline__ int uf_find(int *L, int x) {
  int p = __ldcg(L + x);
  while (p != x) {
    x = p;
    p = __ldcg(L + x);
  }
  return x;
}

// Hang the larger root under the smaller; retry when another thread moved it.
__device__ void uf_union(int *L, int a, int b) {
  for (;;) {
    a = uf_find(L, a);
    b = uf_find(L, b);
    if (a == b) return;
    if (a > b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicMin(L + b, a);
    if (old == b) return;
    b = old;
  }
}

// Joins each row run S = [s, e] to every run R of the row above that touches
// it (8-connectivity).  Row runs are already chained, so one join per pair
// suffices: at q, the leftmost pixel of R within [s-1, e+1], from the pixel
// max(s, q-1) of S.  Seen from a pixel x of S: the upper-left neighbour when
// x = s; the upper one when x = s and the upper-left is background; the
// upper-right one when the upper one is background.
__global__ void merge_kernel(const uint16_t *t16, int *L, int nx, const unsigned *fg,
                             const unsigned *n_fg) {
  const unsigned nf = *n_fg;
  for (unsigned f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
    const unsigned i = fg[f];
    const int y = (int)(i / nx), x = (int)(i % nx);
    if (y == 0) continue;
    const int p = (int)i;
    const bool left = x > 0 && t16[i - 1];
    const uint16_t *up = t16 + (i - nx);
    const bool ul = x > 0 && up[-1], uc = up[0], ur = x + 1 < nx && up[1];
    if (ul && !left) uf_union(L, p, p - nx - 1);
    if (uc && !left && !ul) uf_union(L, p, p - nx);
    if (ur && !uc) uf_union(L, p, p - nx + 1);
  }
}


struct Comps {
  int *area, *x0, *y0, *x1, *y1;
  unsigned *fb;  // first 2x2 block (raster index)
  unsigned long long *sw, *swx, *swy;
  int *label, *keep;
};

// Every foreground pixel points straight at its root; each root takes the
// next component id.
__global__ void compress_kernel(int *L, int *cid, PreState *st, Comps c, const unsigned *fg,
                                const unsigned *n_fg) {
  const unsigned nf = *n_fg;
  for (unsigned f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
    const unsigned i = fg[f];
    const int r = uf_find(L, (int)i);
    if (r != (int)i) {
      L[i] = r;
      continue;
    }
    const unsigned id = atomicAdd(&st->n_comp, 1u);
    cid[i] = (int)id;
    c.area[id] = 0;
    c.x0[id] = INT_MAX;
    c.y0[id] = INT_MAX;
    c.x1[id] = -1;
    c.y1[id] = -1;
    c.fb[id] = 0xffffffffu;
    c.sw[id] = c.swx[id] = c.swy[id] = 0;
  }
}

__global__ void moments_kernel(const int *L, const int *cid, const uint16_t *t16, Comps c, int nx,
                               const unsigned *fg, const unsigned *n_fg) {
  const unsigned nf = *n_fg;
  const unsigned bw = (unsigned)(nx + 1) / 2;
  for (unsigned f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
    const unsigned i = fg[f];
    const int r = L[i];
    const int id = cid[r];
    const int y = (int)(i / nx), x = (int)(i % nx);
    const unsigned long long w = t16[i];
    atomicAdd(c.area + id, 1);
    atomicMin(c.x0 + id, x);
    atomicMin(c.y0 + id, y);
    atomicMax(c.x1 + id, x);
    atomicMax(c.y1 + id, y);
    atomicMin(c.fb + id, (unsigned)(y >> 1) * bw + (unsigned)(x >> 1));
    atomicAdd(c.sw + id, w);
    atomicAdd(c.swx + id, w * (unsigned long long)x);
    atomicAdd(c.swy + id, w * (unsigned long long)y);
  }
}

// Flag each component's first block: low word counts components, high word
// kept ones; a prefix sum over blocks then numbers them in OpenCV's order.
__global__ void flags_kernel(const PreState *st, Comps c, int min_area,
                             unsigned long long *flags, size_t cap) {
  const size_t nc = st->n_comp;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < nc && id < cap;
       id += (size_t)gridDim.x * blockDim.x) {
    const bool keep = c.area[id] >= min_area;
    flags[c.fb[id]] = 1ull | (keep ? (1ull << 32) : 0ull);
  }
}

__global__ void label_kernel(PreState *st, Comps c, int min_area, const unsigned long long *pos,
                             size_t nblocks, double *centres, int *stats) {
  const size_t nc = st->n_comp;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < nc;
       id += (size_t)gridDim.x * blockDim.x) {
    const unsigned long long p = pos[c.fb[id]];
    const int label = (int)(p & 0xffffffffull);
    const bool keep = c.area[id] >= min_area;
    c.label[id] = label;
    const int x0 = c.x0[id], y0 = c.y0[id];
    int *sr = stats + (size_t)(label - 1) * 5;
    sr[0] = x0;
    sr[1] = y0;
    sr[2] = c.x1[id] - x0 + 1;
    sr[3] = c.y1[id] - y0 + 1;
    sr[4] = c.area[id];
    if (keep) {
      const int k = (int)(p >> 32) - 1;
      c.keep[id] = k;
      const unsigned long long sw = c.sw[id];
      const double rx = (double)(c.swx[id] - (unsigned long long)x0 * sw);
      const double ry = (double)(c.swy[id] - (unsigned long long)y0 * sw);
      double *cr = centres + (size_t)k * 4;
      cr[0] = (double)label;
      cr[1] = lmb::dadd(lmb::ddiv(rx, (double)sw), (double)x0);
      cr[2] = lmb::dadd(lmb::ddiv(ry, (double)sw), (double)y0);
      cr[3] = (double)c.area[id];
    } else {
      c.keep[id] = -1;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const unsigned long long t = nblocks ? pos[nblocks - 1] : 0;
    st->n_labels = (unsigned)(t & 0xffffffffull) + 1u;
    st->n_keep = (unsigned)(t >> 32);
  }
}

// The filtered frame (kept components' pixels) over a zeroed frame.
__global__ void filt_kernel(const int *__restrict__ L, const int *__restrict__ cid,
                            const uint16_t *__restrict__ t16, Comps c, uint16_t *__restrict__ filt,
                            const unsigned *fg, const unsigned *n_fg) {
  const unsigned nf = *n_fg;
  for (unsigned f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
    const unsigned i = fg[f];
    if (c.keep[cid[L[i]]] >= 0) filt[i] = t16[i];
  }
}

// Labels of all and of the kept components over zeroed frames (built only
// when a caller asks for them).
__global__ void labels_kernel(const int *__restrict__ L, const int *__restrict__ cid, Comps c,
                              int *__restrict__ labels, int *__restrict__ flabels,
                              const unsigned *fg, const unsigned *n_fg) {
  const unsigned nf = *n_fg;
  for (unsigned f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
    const unsigned i = fg[f];
    const int id = cid[L[i]];
    const int lab = c.label[id];
    labels[i] = lab;
    if (c.keep[id] >= 0) flabels[i] = lab;
  }
}

// Foreground test of the list selection.
struct IsForeground {
  const uint16_t *t16;
  __device__ __forceinline__ bool operator()(const unsigned &i) const { return t16[i] != 0; }
};

// ---- closest pair of centres (blur width) ---------------------------------------
__device__ __forceinline__ double pair_d2(const double *a, const double *b) {
  const double dx = lmb::dsub(a[1], b[1]), dy = lmb::dsub(a[2], b[2]);
  return lmb::dadd(lmb::dmul(dx, dx), lmb::dmul(dy, dy));
}

// Smallest double over the warp, one atomic per warp that found a pair.
__device__ __forceinline__ void warp_min_to(unsigned long long *dst, double v) {
  for (int o = 16; o; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0 && v < __longlong_as_double(0x7ff0000000000000ll))
    atomicMin(dst, (unsigned long long)__double_as_longlong(v));
}

__global__ void cell_insert_kernel(const PreState *st, const double *centres, int *head, int *next,
                                   int gcx, int gcy) {
  const unsigned n = st->n_keep;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int cx = min(max((int)(centres[(size_t)i * 4 + 1] / kCell), 0), gcx - 1);
    const int cy = min(max((int)(centres[(size_t)i * 4 + 2] / kCell), 0), gcy - 1);
    next[i] = atomicExch(head + cy * gcx + cx, (int)i);
  }
}

__global__ void cell_pairs_kernel(PreState *st, const double *centres, const int *head,
                                  const int *next, int gcx, int gcy) {
  const unsigned n = st->n_keep;
  double best = __longlong_as_double(0x7ff0000000000000ll);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double *a = centres + (size_t)i * 4;
    const int cx = min(max((int)(a[1] / kCell), 0), gcx - 1);
    const int cy = min(max((int)(a[2] / kCell), 0), gcy - 1);
    for (int yy = max(cy - 1, 0); yy <= min(cy + 1, gcy - 1); ++yy)
      for (int xx = max(cx - 1, 0); xx <= min(cx + 1, gcx - 1); ++xx)
        for (int j = head[yy * gcx + xx]; j >= 0; j = next[j])
          if ((unsigned)j > i) best = fmin(best, pair_d2(a, centres + (size_t)j * 4));
  }
  warp_min_to(&st->best, best);
}

// Pairs in cells that are not neighbours lie more than a cell apart, so the
// grid's answer is exact when it is within a cell; otherwise every pair.
__global__ void brute_pairs_kernel(PreState *st, const double *centres) {
  const double cell2 = (double)kCell * (double)kCell;
  if (__longlong_as_double((long long)st->best) <= cell2) return;
  const unsigned n = st->n_keep;
  double best = __longlong_as_double(0x7ff0000000000000ll);
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (unsigned j = i + 1; j < n; ++j)
      best = fmin(best, pair_d2(centres + (size_t)i * 4, centres + (size_t)j * 4));
  warp_min_to(&st->best, best);
}

// ---- Gaussian blur ---------------------------------------------------------------
// scipy's symmetric correlation: w_c*x_0, then + (x_-j + x_+j) * w_j from the
// outermost pair inwards, every operation rounded on its own.
template <typename TIn>
__global__ void blur_rows_kernel(const TIn *in, const double *wts, int r, int ny, int nx,
                                 double *out) {
  extern __shared__ double w[];
  for (int j = threadIdx.x; j <= 2 * r; j += blockDim.x) w[j] = wts[j];
  __syncthreads();
  const size_t n = (size_t)ny * nx;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / nx), x = (int)(i % nx);
    double acc = lmb::dmul(to_f64(in[i]), w[r]);
    for (int j = r; j >= 1; --j) {
      const double a = to_f64(in[(size_t)mirror(y - j, ny) * nx + x]);
      const double b = to_f64(in[(size_t)mirror(y + j, ny) * nx + x]);
      acc = lmb::dadd(acc, lmb::dmul(lmb::dadd(a, b), w[r - j]));
    }
    out[i] = acc;
  }
}

template <typename TOut>
__global__ void blur_cols_kernel(const double *in, const double *wts, int r, int ny, int nx,
                                 TOut *out) {
  extern __shared__ double w[];
  for (int j = threadIdx.x; j <= 2 * r; j += blockDim.x) w[j] = wts[j];
  __syncthreads();
  const size_t n = (size_t)ny * nx;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const double *row = in + (i - x);
    double acc = lmb::dmul(row[x], w[r]);
    for (int j = r; j >= 1; --j)
      acc = lmb::dadd(acc, lmb::dmul(lmb::dadd(row[mirror(x - j, nx)], row[mirror(x + j, nx)]), w[r - j]));
    out[i] = (TOut)acc;
  }
}

// Both passes for a 32x32 output tile: the mirrored input tile with its halo
// in shared memory, the axis-0 pass over the tile's rows and halo columns,
// then the axis-1 pass; the same operations in the same order as the two
// separate passes, without the float64 intermediate in global memory.
constexpr int kBlurTile = 32;
constexpr int kBlurTileMaxR = 32;

size_t blur_tile_smem(int r) {
  const int W = kBlurTile + 2 * r;
  return (size_t)(2 * r + 1 + kBlurTile * W) * sizeof(double) + (size_t)W * W * sizeof(uint16_t);
}

template <typename TOut>
__global__ void __launch_bounds__(256)
    blur_tile_kernel(const uint16_t *__restrict__ in, const double *__restrict__ wts, int r, int ny,
                     int nx, TOut *__restrict__ out) {
  extern __shared__ double sm[];
  const int W = kBlurTile + 2 * r;
  double *w = sm;
  double *vert = sm + (2 * r + 1);
  uint16_t *tile = reinterpret_cast<uint16_t *>(vert + kBlurTile * W);
  const int x0 = blockIdx.x * kBlurTile, y0 = blockIdx.y * kBlurTile;
  const int tid = threadIdx.x;
  for (int j = tid; j <= 2 * r; j += blockDim.x) w[j] = wts[j];
  for (int idx = tid; idx < W * W; idx += blockDim.x) {
    const int ty = idx / W, tx = idx - ty * W;
    tile[idx] = in[(size_t)mirror(y0 - r + ty, ny) * nx + mirror(x0 - r + tx, nx)];
  }
  __syncthreads();
  for (int idx = tid; idx < kBlurTile * W; idx += blockDim.x) {
    const int ty = idx / W, tx = idx - ty * W;
    const uint16_t *col = tile + (ty + r) * W + tx;
    double acc = lmb::dmul((double)col[0], w[r]);
    for (int j = r; j >= 1; --j)
      acc = lmb::dadd(acc, lmb::dmul(lmb::dadd((double)col[-j * W], (double)col[j * W]), w[r - j]));
    vert[idx] = acc;
  }
  __syncthreads();
  for (int idx = tid; idx < kBlurTile * kBlurTile; idx += blockDim.x) {
    const int ty = idx / kBlurTile, tx = idx - ty * kBlurTile;
    const int gy = y0 + ty, gx = x0 + tx;
    if (gy >= ny || gx >= nx) continue;
    const double *row = vert + ty * W + tx + r;
    double acc = lmb::dmul(row[0], w[r]);
    for (int j = r; j >= 1; --j) acc = lmb::dadd(acc, lmb::dmul(lmb::dadd(row[-j], row[j]), w[r - j]));
    out[(size_t)gy * nx + gx] = (TOut)acc;
  }
}

// The same for radius R known at compile time (1..8; sigma 1 gives R = 4):
// each thread keeps a 4-output segment of a column (axis-0 pass) and then of
// a row (axis-1 pass) in registers, 4 + 2R inputs, each converted once.
constexpr int kBlurFixedMaxR = 8;

template <int R, typename TOut>
__global__ void __launch_bounds__(256)
    blur_tile_r_kernel(const uint16_t *__restrict__ in, const double *__restrict__ wts, int ny,
                       int nx, TOut *__restrict__ out) {
  constexpr int W = kBlurTile + 2 * R;
  __shared__ double w[2 * R + 1];
  __shared__ double vert[kBlurTile * W];
  __shared__ uint16_t tile[W * W];
  const int x0 = blockIdx.x * kBlurTile, y0 = blockIdx.y * kBlurTile;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (t <= 2 * R) w[t] = wts[t];
  // mirrored source columns of this lane (W <= 48 < 64)
  const int c0 = mirror(x0 - R + lane, nx);
  const int c1 = lane + 32 < W ? mirror(x0 - R + lane + 32, nx) : 0;
  for (int row = warp; row < W; row += 8) {
    const uint16_t *src = in + (size_t)mirror(y0 - R + row, ny) * nx;
    tile[row * W + lane] = src[c0];
    if (lane + 32 < W) tile[row * W + lane + 32] = src[c1];
  }
  __syncthreads();
  // axis 0: task = (group of 4 output rows, tile column)
  for (int task = t; task < 8 * W; task += 256) {
    const int rg = task / W, col = task - rg * W;
    double v[4 + 2 * R];
#pragma unroll
    for (int q = 0; q < 4 + 2 * R; ++q) v[q] = (double)tile[(rg * 4 + q) * W + col];
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      double acc = lmb::dmul(v[o + R], w[R]);
#pragma unroll
      for (int j = R; j >= 1; --j)
        acc = lmb::dadd(acc, lmb::dmul(lmb::dadd(v[o + R - j], v[o + R + j]), w[R - j]));
      vert[(rg * 4 + o) * W + col] = acc;
    }
  }
  __syncthreads();
  // axis 1: task = (output row, group of 4 output columns)
  {
    const int row = t >> 3, cg = (t & 7) * 4;
    const double *src = vert + row * W + cg;
    double v[4 + 2 * R];
#pragma unroll
    for (int q = 0; q < 4 + 2 * R; ++q) v[q] = src[q];
    const int gy = y0 + row;
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      double acc = lmb::dmul(v[o + R], w[R]);
#pragma unroll
      for (int j = R; j >= 1; --j)
        acc = lmb::dadd(acc, lmb::dmul(lmb::dadd(v[o + R - j], v[o + R + j]), w[R - j]));
      const int gx = x0 + cg + o;
      if (gy < ny && gx < nx) out[(size_t)gy * nx + gx] = (TOut)acc;
    }
  }
}

template <typename TOut>
void blur_tile_r_launch(int r, dim3 grid, const uint16_t *in, const double *w, int ny, int nx,
                        TOut *out, cudaStream_t st) {
  switch (r) {
    case 1: blur_tile_r_kernel<1, TOut><<<grid, 256, 0, st>>>(in, w, ny, nx, out); break;
    case 2: blur_tile_r_kernel<2, TOut><<<grid, 256, 0, st>>>(in, w, ny, nx, out); break;
    case 3: blur_tile_r_kernel<3, TOut><<<grid, 256, 0, st>>>(in, w, ny, nx, out); break;
    case 4: blur_tile_r_kernel<4, TOut><<<grid, 256, 0, st>>>(in, w, ny, nx, out); break;
    case 5: blur_tile_r_kernel<5, TOut><<<grid, 256, 0, st>>>(in, w, ny, nx, out); break;
    case 6: blur_tile_r_kernel<6, TOut><<<grid, 256, 0, st>>>(in, w, ny, nx, out); break;
    case 7: blur_tile_r_kernel<7, TOut><<<grid, 256, 0, st>>>(in, w, ny, nx, out); break;
    default: blur_tile_r_kernel<8, TOut><<<grid, 256, 0, st>>>(in, w, ny, nx, out); break;
  }
}

// ---- median ------------------------------------------------------------------------
__global__ void rank_keys_kernel(const double *img, unsigned long long *keys, unsigned *idx,
                                 size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    keys[i] = okey(img[i]);
    idx[i] = (unsigned)i;
  }
}

__global__ void rank_flags_kernel(const unsigned long long *keys, unsigned *flag, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

__global__ void rank_scatter_kernel(const unsigned long long *keys, const unsigned *idx,
                                    const unsigned *flag, const unsigned *incl, unsigned *rank,
                                    double *vals, unsigned *n_distinct, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const unsigned r = incl[i] - 1u;
    rank[idx[i]] = r;
    if (flag[i]) vals[r] = okey_value(keys[i]);
    if (i == n - 1) *n_distinct = incl[i];
  }
}

__device__ __forceinline__ unsigned med_digit(unsigned r, int l, int L) {
  return (r >> (8 * (L - 1 - l))) & 255u;
}
__device__ __forceinline__ unsigned med_prefix(unsigned r, int l, int L) {
  const int sh = 8 * (L - l);
  return sh >= 32 ? 0u : (r >> sh);
}

// Add `delta` for rank r to every level whose path prefix it follows, and
// count it into `below` of the levels where its digit lies under the path's.
__device__ __forceinline__ void med_update(unsigned *h, const unsigned (&pp)[kMedLevels],
                                           const int (&path)[kMedLevels], int (&below)[kMedLevels],
                                           int L, unsigned r, int delta) {
#pragma unroll
  for (int l = 0; l < kMedLevels; ++l) {
    if (l >= L || med_prefix(r, l, L) != pp[l]) break;
    const unsigned d = med_digit(r, l, L);
    atomicAdd(h + l * 256 + d, (unsigned)delta);
    below[l] += (int)d < path[l] ? delta : 0;
  }
}

// Fill level l from the whole window (ranks whose digits above l equal pp).
__device__ void med_fill(unsigned *h, int l, int L, unsigned pp, const unsigned *rk, int ny,
                         int nx, int x, int y, int lo, int hi) {
  const int lane = threadIdx.x & 31;
  for (int j = lane; j < 256; j += 32) h[l * 256 + j] = 0;
  __syncwarp();
  for (int dy = -lo; dy <= hi; ++dy) {
    const unsigned *row = rk + (size_t)mirror(y + dy, ny) * nx;
    for (int dx = -lo + lane; dx <= hi; dx += 32) {
      const unsigned r = row[mirror(x + dx, nx)];
      if (l == 0 || med_prefix(r, l, L) == pp) atomicAdd(h + l * 256 + med_digit(r, l, L), 1u);
    }
  }
  __syncwarp();
}

// One warp per (column x, segment of rows): the window's ranks are kept as
// per-level histograms of 8-bit digits.  Level 0 counts every rank; level l
// counts the ranks whose higher digits equal the median's path so far, and
// below[l] how many of those have a smaller digit at l than the path.  When
// the window slides down one row, the leaving and entering rows update both.
// The median's digit at a level is kept while below <= k < below + count
// (the common case: a background changes slowly); otherwise a short walk
// over neighbouring bins or a scan of the level finds it, and the levels
// under a moved digit are refilled from the whole window.
__global__ void __launch_bounds__(kMedWarps * 32, 4)
    median_kernel(const unsigned *rk, const double *vals, const unsigned *n_distinct, int ny, int nx,
                  int s, int seg, double *out) {
  __shared__ __align__(16) unsigned hist[kMedWarps][kMedLevels * 256];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nseg = (ny + seg - 1) / seg;
  const long long task = (long long)blockIdx.x * kMedWarps + warp;
  if (task >= (long long)nx * nseg) return;
  const int x = (int)(task % nx), sg = (int)(task / nx);
  const int y0 = sg * seg, y1 = min(ny, y0 + seg);
  const unsigned D = *n_distinct;
  const int bits = D <= 1 ? 1 : 32 - __clz(D - 1);
  const int L = (bits + 7) / 8;
  unsigned *h = hist[warp];
  int path[kMedLevels], below[kMedLevels];
  unsigned pp[kMedLevels];
#pragma unroll
  for (int l = 0; l < kMedLevels; ++l) {
    path[l] = -1;
    below[l] = 0;
    pp[l] = 0xffffffffu;
  }
  pp[0] = 0;
  const int lo = s / 2, hi = s - 1 - lo;
  const unsigned long long k = ((unsigned long long)s * s) / 2;
  med_fill(h, 0, L, 0, rk, ny, nx, x, y0, lo, hi);
  int rb = 0;  // shallowest level whose digit must be found by a full scan
  for (int y = y0; y < y1; ++y) {
    if (y > y0) {
      int mine[kMedLevels];
#pragma unroll
      for (int l = 0; l < kMedLevels; ++l) mine[l] = 0;
      const unsigned *ro = rk + (size_t)mirror(y - 1 - lo, ny) * nx;
      const unsigned *ri = rk + (size_t)mirror(y + hi, ny) * nx;
      for (int dx = -lo + lane; dx <= hi; dx += 32) {
        const int c = mirror(x + dx, nx);
        med_update(h, pp, path, mine, L, ro[c], -1);
        med_update(h, pp, path, mine, L, ri[c], 1);
      }
#pragma unroll
      for (int l = 0; l < kMedLevels; ++l)
        if (l < L) below[l] += __reduce_add_sync(0xffffffffu, mine[l]);
      __syncwarp();
    }
    unsigned long long kres = k;
    unsigned rank = 0;
#pragma unroll
    for (int l = 0; l < kMedLevels; ++l) {
      if (l >= L) break;
      const unsigned *hl = h + l * 256;
      bool found = false;
      if (l < rb) {
        // keep the digit, or walk a few bins from it
        long long b = below[l];
        int d = path[l];
        for (int step = 0; step < 8; ++step) {
          const long long c = hl[d];
          if ((long long)kres < b) {
            if (d == 0) break;
            --d;
            b -= hl[d];
          } else if ((long long)kres >= b + c) {
            if (d == 255) break;
            b += c;
            ++d;
          } else {
            found = true;
            break;
          }
        }
        if (found) {
          kres -= (unsigned long long)b;
          below[l] = (int)b;
          if (d != path[l]) {
            path[l] = d;
            if (rb > l + 1) rb = l + 1;
          }
        }
      } else if (l > 0) {
        med_fill(h, l, L, pp[l], rk, ny, nx, x, y, lo, hi);
      }
      if (!found) {
        const unsigned long long k0 = kres;
        const int d = (int)warp_find_digit(hl, kres);
        below[l] = (int)(k0 - kres);
        if (d != path[l]) {
          path[l] = d;
          if (rb > l + 1) rb = l + 1;
        }
        if (rb <= l) rb = l + 1;
      }
      rank = (rank << 8) | (unsigned)path[l];
      if (l + 1 < kMedLevels) pp[l + 1] = rank;
    }
    // a rank outside the distinct values would mean inconsistent histograms
    if (lane == 0)
      out[(size_t)y * nx + x] = rank < D ? vals[rank] : __longlong_as_double(0x7ff8000000000000ll);
  }
}

}  // namespace

// ---- handle ------------------------------------------------------------------------
struct lmb_pre {
  int device = 0, ny = 0, nx = 0, num_sms = 148;
  size_t npx = 0, nblocks = 0;
  cudaStream_t st = nullptr;
  void *d_raw = nullptr;
  double *d_bg = nullptr, *d_sub = nullptr, *d_tmp = nullptr;
  void *d_out = nullptr;
  uint16_t *d_t16 = nullptr, *d_filt = nullptr;
  int *d_par = nullptr, *d_cid = nullptr, *d_lab = nullptr, *d_flab = nullptr;
  Comps c{};
  unsigned long long *d_flags = nullptr, *d_pos = nullptr, *d_compact = nullptr;
  unsigned *d_hist16 = nullptr;  // 65536-bin histogram of the first selection pass
  unsigned *d_fg = nullptr, *d_nfg = nullptr;  // foreground pixel list and its length
  void *d_fg_tmp = nullptr;
  size_t fg_bytes = 0;
  bool labels_ready = false;  // label images of the last segment built
  double *d_centres = nullptr, *d_w = nullptr;
  int *d_stats = nullptr, *d_head = nullptr, *d_next = nullptr;
  int gcx = 1, gcy = 1;
  PreState *d_state = nullptr, *h_state = nullptr;
  void *d_cub = nullptr;
  size_t cub_bytes = 0;
  // median scratch, allocated on first use
  unsigned long long *m_keys = nullptr, *m_keys2 = nullptr;
  unsigned *m_idx = nullptr, *m_idx2 = nullptr, *m_flag = nullptr, *m_incl = nullptr,
           *m_rank = nullptr, *m_nd = nullptr;
  double *m_vals = nullptr, *m_img = nullptr;
  void *m_cub = nullptr;
  size_t m_cub_bytes = 0;
  bool segmented = false;
  lmb_pre_counts last{};
  // stage events: frame upload, threshold, components, blur, download, median ranks, median
  cudaEvent_t ev[kPreEvents] = {};
  float ms[LMB_PRE_STAGES] = {};
  // blurred frame handed to an engine: ready on this stream, free once the
  // engine's quantisation has read it
  cudaEvent_t ev_out_ready = nullptr, ev_out_free = nullptr;
  bool out_in_use = false;
};

namespace {

int check_pre(lmb_pre *p) {
  if (!p) {
    set_error("null preprocessing handle");
    return LMB_ERR_INVALID;
  }
  LMB_CUDA(cudaSetDevice(p->device));
  return LMB_OK;
}

void free_pre(lmb_pre *p) {
  if (!p) return;
  cudaSetDevice(p->device);
  if (p->st) cudaStreamSynchronize(p->st);
  void *bufs[] = {p->d_raw, p->d_bg, p->d_sub, p->d_tmp, p->d_out, p->d_t16, p->d_filt, p->d_par,
                  p->d_cid, p->d_lab, p->d_flab, p->c.area, p->c.x0, p->c.y0, p->c.x1, p->c.y1,
                  p->c.fb, p->c.sw, p->c.swx, p->c.swy, p->c.label, p->c.keep, p->d_flags,
                  p->d_pos, p->d_compact, p->d_centres, p->d_w, p->d_stats, p->d_head, p->d_next,
                  p->d_state, p->d_cub, p->d_hist16, p->d_fg, p->d_nfg, p->d_fg_tmp, p->m_keys, p->m_keys2, p->m_idx, p->m_idx2, p->m_flag,
                  p->m_incl, p->m_rank, p->m_nd, p->m_vals, p->m_img, p->m_cub};
  for (void *b : bufs)
    if (b) cudaFree(b);
  if (p->h_state) cudaFreeHost(p->h_state);
  for (auto &e : p->ev)
    if (e) cudaEventDestroy(e);
  if (p->ev_out_ready) cudaEventDestroy(p->ev_out_ready);
  if (p->ev_out_free) cudaEventDestroy(p->ev_out_free);
  if (p->st) cudaStreamDestroy(p->st);
  delete p;
}

template <typename T>
int alloc(T **ptr, size_t count) {
  LMB_CUDA(cudaMalloc(reinterpret_cast<void **>(ptr), std::max<size_t>(count, 1) * sizeof(T)));
  return LMB_OK;
}

size_t pre_dtype_bytes(int dtype) {
  return dtype == LMB_F64 ? 8 : dtype == LMB_F32 ? 4 : dtype == LMB_U16 ? 2 : 1;
}

template <typename F>
int by_dtype(int dtype, F &&f) {
  switch (dtype) {
    case LMB_F64: return f((const double *)nullptr);
    case LMB_F32: return f((const float *)nullptr);
    case LMB_U16: return f((const uint16_t *)nullptr);
    case LMB_U8: return f((const uint8_t *)nullptr);
  }
  set_error("unknown dtype %d", dtype);
  return LMB_ERR_INVALID;
}

int upload_frame(lmb_pre *p, const void *frame, int dtype) {
  LMB_REQUIRE(frame, "null frame");
  LMB_CUDA(cudaMemcpyAsync(p->d_raw, frame, p->npx * pre_dtype_bytes(dtype),
                           cudaMemcpyHostToDevice, p->st));
  return LMB_OK;
}

// Blocks of the 16-bit pass: each handles at most 65535 values.
unsigned hist16_grid(const lmb_pre *p) {
  return (unsigned)std::max<size_t>((size_t)p->num_sms, p->npx / 60000 + 1);
}

// One order-statistic search.  The 16-bit first pass has run (fused with
// the subtraction, or launched here when `first_pass`); the 8-bit passes
// follow, the first over the frame, the rest over the keys it kept.
int run_select(lmb_pre *p, int mode, bool first_pass) {
  if (first_pass)
    sel_hist16_kernel<<<hist16_grid(p), kHist16Threads, kHist16Smem, p->st>>>(
        p->d_sub, (unsigned)p->npx, p->d_state, p->d_hist16, mode);
  for (int shift = kKeepShift; shift >= 0; shift -= 8) {
    // one wave of blocks over the frame; the kept keys' count is on the device
    const unsigned gp = (unsigned)(p->num_sms * (shift == kKeepShift ? 4 : 2));
    sel_hist_kernel<<<gp, kT, 0, p->st>>>(p->d_sub, p->npx, p->d_state, mode, shift, p->d_compact);
  }
  LMB_CUDA(cudaGetLastError());
  return LMB_OK;
}

// Subtraction fused with the value histogram; *done when every candidate was
// an integer in [0, 65535] and the threshold is set (else the frame's
// subtraction is in place for the radix selection).
int value_select(lmb_pre *p, int dtype, int mode, unsigned long long k0, int two, double gamma,
                 bool *done) {
  int rc = by_dtype(dtype, [&](auto tag) {
    using T = std::remove_const_t<std::remove_pointer_t<decltype(tag)>>;
    value_hist_kernel<T><<<(unsigned)(p->num_sms * 4), kVhThreads, 0, p->st>>>(
        static_cast<const T *>(p->d_raw), p->d_bg, p->d_sub, (unsigned)p->npx, p->d_state,
        p->d_hist16, mode, k0, two, gamma);
    return LMB_OK;
  });
  if (rc) return rc;
  LMB_CUDA(cudaGetLastError());
  LMB_CUDA(cudaMemcpyAsync(&p->h_state->value_path, &p->d_state->value_path, sizeof(unsigned),
                           cudaMemcpyDeviceToHost, p->st));
  LMB_CUDA(cudaStreamSynchronize(p->st));
  *done = p->h_state->value_path != 0;
  return LMB_OK;
}


// np.percentile's order statistics and weight for n values (linear method).
void percentile_plan(size_t n, double pct, unsigned long long *k0, int *two, double *gamma) {
  const double q = pct / 100.0;
  const double vi = (double)(n - 1) * q;
  double prev = std::floor(vi);
  if (vi >= (double)(n - 1)) {
    *k0 = n - 1;
    *two = 0;
    prev = -1.0;
  } else if (vi < 0) {
    *k0 = 0;
    *two = 0;
    prev = 0.0;
  } else {
    *k0 = (unsigned long long)prev;
    *two = 1;
  }
  *gamma = vi - prev;
}

// Components, centres and closest pair from d_t16 / d_par.
int segment_tail(lmb_pre *p, int min_area, lmb_pre_counts *counts, bool parents_ready) {
  const unsigned g = (unsigned)grid_for(p->npx, p->num_sms);
  cudaStream_t st = p->st;
  if (!parents_ready) init_parents_kernel<<<g, kT, 0, st>>>(p->d_t16, p->d_par, p->nx, p->npx);
  // the foreground pixels, in raster order; the component kernels run over them
  size_t sb = p->fg_bytes;
  LMB_CUDA(cub::DeviceSelect::If(p->d_fg_tmp, sb, thrust::counting_iterator<unsigned>(0u),
                                 p->d_fg, p->d_nfg, (int)p->npx, IsForeground{p->d_t16}, st));
  merge_kernel<<<g, kT, 0, st>>>(p->d_t16, p->d_par, p->nx, p->d_fg, p->d_nfg);
  reset_counts_kernel<<<1, 1, 0, st>>>(p->d_state);
  compress_kernel<<<g, kT, 0, st>>>(p->d_par, p->d_cid, p->d_state, p->c, p->d_fg, p->d_nfg);
  moments_kernel<<<g, kT, 0, st>>>(p->d_par, p->d_cid, p->d_t16, p->c, p->nx, p->d_fg, p->d_nfg);
  LMB_CUDA(cudaMemsetAsync(p->d_flags, 0, p->nblocks * sizeof(unsigned long long), st));
  const unsigned gc = (unsigned)grid_for(p->nblocks, p->num_sms);
  flags_kernel<<<gc, kT, 0, st>>>(p->d_state, p->c, min_area, p->d_flags, p->nblocks);
  size_t tb = p->cub_bytes;
  LMB_CUDA(cub::DeviceScan::InclusiveSum(p->d_cub, tb, p->d_flags, p->d_pos, (int)p->nblocks, st));
  label_kernel<<<gc, kT, 0, st>>>(p->d_state, p->c, min_area, p->d_pos, p->nblocks,
                                  p->d_centres, p->d_stats);
  LMB_CUDA(cudaMemsetAsync(p->d_filt, 0, p->npx * sizeof(uint16_t), st));
  filt_kernel<<<g, kT, 0, st>>>(p->d_par, p->d_cid, p->d_t16, p->c, p->d_filt, p->d_fg, p->d_nfg);
  p->labels_ready = false;
  // closest pair of kept centres
  LMB_CUDA(cudaMemsetAsync(p->d_head, 0xff, (size_t)p->gcx * p->gcy * sizeof(int), st));
  cell_insert_kernel<<<gc, kT, 0, st>>>(p->d_state, p->d_centres, p->d_head, p->d_next, p->gcx,
                                        p->gcy);
  cell_pairs_kernel<<<gc, kT, 0, st>>>(p->d_state, p->d_centres, p->d_head, p->d_next, p->gcx,
                                       p->gcy);
  brute_pairs_kernel<<<p->num_sms * 2, kT, 0, st>>>(p->d_state, p->d_centres);
  LMB_CUDA(cudaGetLastError());
  LMB_CUDA(cudaEventRecord(p->ev[EV_SEG_CC], st));
  PreState *hs = p->h_state;
  LMB_CUDA(cudaMemcpyAsync(hs, p->d_state, sizeof(PreState), cudaMemcpyDeviceToHost, st));
  LMB_CUDA(cudaStreamSynchronize(st));
  lmb_pre_counts out{};
  out.threshold = hs->thresh;
  out.n_labels = (int32_t)hs->n_labels;
  out.n_centres = (int32_t)hs->n_keep;
  double best;
  memcpy(&best, &hs->best, sizeof(best));
  out.min_dist2 = hs->n_keep >= 2 ? best : std::numeric_limits<double>::infinity();
  p->last = out;
  p->segmented = true;
  if (counts) *counts = out;
  return LMB_OK;
}

// Elapsed device time between two recorded events (the stream is synchronised).
int stage_times(lmb_pre *p, int a, int b, int slot) {
  float ms = 0.f;
  LMB_CUDA(cudaEventElapsedTime(&ms, p->ev[a], p->ev[b]));
  p->ms[slot] = ms;
  return LMB_OK;
}

int ensure_median_scratch(lmb_pre *p) {
  if (p->m_keys) return LMB_OK;
  int rc;
  if ((rc = alloc(&p->m_keys, p->npx)) || (rc = alloc(&p->m_keys2, p->npx)) ||
      (rc = alloc(&p->m_idx, p->npx)) || (rc = alloc(&p->m_idx2, p->npx)) ||
      (rc = alloc(&p->m_flag, p->npx)) || (rc = alloc(&p->m_incl, p->npx)) ||
      (rc = alloc(&p->m_rank, p->npx)) || (rc = alloc(&p->m_nd, 1)) ||
      (rc = alloc(&p->m_vals, p->npx)) || (rc = alloc(&p->m_img, p->npx)))
    return rc;
  size_t a = 0, b = 0;
  LMB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, a, p->m_keys, p->m_keys2, p->m_idx, p->m_idx2,
                                           (int)p->npx));
  LMB_CUDA(cub::DeviceScan::InclusiveSum(nullptr, b, p->m_flag, p->m_incl, (int)p->npx));
  p->m_cub_bytes = std::max(a, b);
  LMB_CUDA(cudaMalloc(&p->m_cub, p->m_cub_bytes));
  return LMB_OK;
}

// One median pass of d_in into d_out (both float64 on the device).
int median_pass(lmb_pre *p, const double *d_in, double *d_out, int size) {
  cudaStream_t st = p->st;
  const unsigned g = (unsigned)grid_for(p->npx, p->num_sms);
  LMB_CUDA(cudaEventRecord(p->ev[EV_MED_PASS], st));
  rank_keys_kernel<<<g, kT, 0, st>>>(d_in, p->m_keys, p->m_idx, p->npx);
  size_t tb = p->m_cub_bytes;
  LMB_CUDA(cub::DeviceRadixSort::SortPairs(p->m_cub, tb, p->m_keys, p->m_keys2, p->m_idx,
                                           p->m_idx2, (int)p->npx, 0, 64, st));
  rank_flags_kernel<<<g, kT, 0, st>>>(p->m_keys2, p->m_flag, p->npx);
  tb = p->m_cub_bytes;
  LMB_CUDA(cub::DeviceScan::InclusiveSum(p->m_cub, tb, p->m_flag, p->m_incl, (int)p->npx, st));
  rank_scatter_kernel<<<g, kT, 0, st>>>(p->m_keys2, p->m_idx2, p->m_flag, p->m_incl, p->m_rank,
                                        p->m_vals, p->m_nd, p->npx);
  // row segments: enough warps to fill every SM several times over
  const long long want = (long long)p->num_sms * 64 * 2;
  int seg = (int)std::max<long long>(16, ((long long)p->ny * p->nx + want - 1) / want);
  seg = std::min(seg, p->ny);
  const long long tasks = (long long)p->nx * ((p->ny + seg - 1) / seg);
  const unsigned blocks = (unsigned)((tasks + kMedWarps - 1) / kMedWarps);
  LMB_CUDA(cudaEventRecord(p->ev[EV_MED_RANK], st));
  median_kernel<<<blocks, kMedWarps * 32, 0, st>>>(p->m_rank, p->m_vals, p->m_nd, p->ny, p->nx,
                                                   size, seg, d_out);
  LMB_CUDA(cudaGetLastError());
  LMB_CUDA(cudaEventRecord(p->ev[EV_MED_K], st));
  return LMB_OK;
}

}  // namespace

extern "C" {

int lmb_pre_create(int32_t device, int32_t nr_px_y, int32_t nr_px_x, lmb_pre **out) {
  LMB_REQUIRE(out, "null output");
  *out = nullptr;
  LMB_REQUIRE(nr_px_y > 0 && nr_px_x > 0, "frame size %d x %d", nr_px_y, nr_px_x);
  LMB_REQUIRE((long long)nr_px_y * nr_px_x < (1ll << 31), "frame of %lld pixels is too large",
              (long long)nr_px_y * nr_px_x);
  LMB_CUDA(cudaSetDevice(device));
  lmb_pre *p = new lmb_pre();
  p->device = device;
  p->ny = nr_px_y;
  p->nx = nr_px_x;
  p->npx = (size_t)nr_px_y * nr_px_x;
  p->nblocks = (size_t)((nr_px_y + 1) / 2) * ((nr_px_x + 1) / 2);
  p->gcx = (nr_px_x + kCell - 1) / kCell;
  p->gcy = (nr_px_y + kCell - 1) / kCell;
  cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, device);
  int rc = LMB_OK;
  auto fail = [&](int r) {
    free_pre(p);
    return r;
  };
  if (cudaStreamCreateWithFlags(&p->st, cudaStreamNonBlocking) != cudaSuccess)
    return fail(cuda_fail(cudaGetLastError(), "cudaStreamCreate", __FILE__, __LINE__));
  const size_t n = p->npx, nb = p->nblocks;
  if ((rc = alloc(reinterpret_cast<double **>(&p->d_raw), n)) || (rc = alloc(&p->d_bg, n)) ||
      (rc = alloc(&p->d_sub, n)) || (rc = alloc(&p->d_tmp, n)) ||
      (rc = alloc(reinterpret_cast<double **>(&p->d_out), n)) || (rc = alloc(&p->d_t16, n)) ||
      (rc = alloc(&p->d_filt, n)) || (rc = alloc(&p->d_par, n)) || (rc = alloc(&p->d_cid, n)) ||
      (rc = alloc(&p->d_lab, n)) || (rc = alloc(&p->d_flab, n)) || (rc = alloc(&p->c.area, nb)) ||
      (rc = alloc(&p->c.x0, nb)) || (rc = alloc(&p->c.y0, nb)) || (rc = alloc(&p->c.x1, nb)) ||
      (rc = alloc(&p->c.y1, nb)) || (rc = alloc(&p->c.fb, nb)) || (rc = alloc(&p->c.sw, nb)) ||
      (rc = alloc(&p->c.swx, nb)) || (rc = alloc(&p->c.swy, nb)) ||
      (rc = alloc(&p->c.label, nb)) || (rc = alloc(&p->c.keep, nb)) ||
      (rc = alloc(&p->d_flags, nb)) || (rc = alloc(&p->d_pos, nb)) ||
      (rc = alloc(&p->d_compact, n)) || (rc = alloc(&p->d_centres, nb * 4)) ||
      (rc = alloc(&p->d_w, 1024)) || (rc = alloc(&p->d_stats, nb * 5)) ||
      (rc = alloc(&p->d_head, (size_t)p->gcx * p->gcy)) || (rc = alloc(&p->d_next, nb)) ||
      (rc = alloc(&p->d_state, 1)) || (rc = alloc(&p->d_hist16, 65536)) ||
      (rc = alloc(&p->d_fg, n)) || (rc = alloc(&p->d_nfg, 1)))
    return fail(rc);
  {
    size_t fb = 0;
    if (cub::DeviceSelect::If(nullptr, fb, thrust::counting_iterator<unsigned>(0u), p->d_fg,
                              p->d_nfg, (int)n, IsForeground{p->d_t16}) != cudaSuccess ||
        cudaMalloc(&p->d_fg_tmp, std::max<size_t>(fb, 1)) != cudaSuccess)
      return fail(cuda_fail(cudaGetLastError(), "foreground list set-up", __FILE__, __LINE__));
    p->fg_bytes = fb;
  }
  if (cudaMemset(p->d_hist16, 0, 65536 * sizeof(unsigned)) != cudaSuccess)
    return fail(cuda_fail(cudaGetLastError(), "cudaMemset", __FILE__, __LINE__));
  {
    // the 16-bit selection pass uses 128 KiB of shared memory per block
    const int b = (int)kHist16Smem;
    cudaError_t e = cudaFuncSetAttribute(sel_hist16_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaFuncSetAttribute", __FILE__, __LINE__));
  }
  for (auto &e : p->ev)
    if (cudaEventCreate(&e) != cudaSuccess)
      return fail(cuda_fail(cudaGetLastError(), "cudaEventCreate", __FILE__, __LINE__));
  if (cudaEventCreateWithFlags(&p->ev_out_ready, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->ev_out_free, cudaEventDisableTiming) != cudaSuccess)
    return fail(cuda_fail(cudaGetLastError(), "cudaEventCreate", __FILE__, __LINE__));
  if (cudaMallocHost(&p->h_state, sizeof(PreState)) != cudaSuccess)
    return fail(cuda_fail(cudaErrorMemoryAllocation, "cudaMallocHost", __FILE__, __LINE__));
  memset(p->h_state, 0, sizeof(PreState));
  p->h_state->best = 0x7ff0000000000000ull;
  if (cudaMemset(p->d_bg, 0, n * sizeof(double)) != cudaSuccess ||
      cudaMemset(p->d_state, 0, sizeof(PreState)) != cudaSuccess)
    return fail(cuda_fail(cudaGetLastError(), "cudaMemset", __FILE__, __LINE__));
  size_t tb = 0;
  if (cub::DeviceScan::InclusiveSum(nullptr, tb, p->d_flags, p->d_pos, (int)nb) != cudaSuccess)
    return fail(cuda_fail(cudaGetLastError(), "scan sizing", __FILE__, __LINE__));
  p->cub_bytes = tb;
  if (cudaMalloc(&p->d_cub, std::max<size_t>(tb, 1)) != cudaSuccess)
    return fail(cuda_fail(cudaErrorMemoryAllocation, "cudaMalloc", __FILE__, __LINE__));
  *out = p;
  return LMB_OK;
}

int lmb_pre_destroy(lmb_pre *p) {
  if (!p) return LMB_OK;
  free_pre(p);
  return LMB_OK;
}

int lmb_pre_set_background(lmb_pre *p, const double *background) {
  int rc = check_pre(p);
  if (rc) return rc;
  if (background)
    LMB_CUDA(cudaMemcpyAsync(p->d_bg, background, p->npx * sizeof(double), cudaMemcpyHostToDevice,
                             p->st));
  else
    LMB_CUDA(cudaMemsetAsync(p->d_bg, 0, p->npx * sizeof(double), p->st));
  LMB_CUDA(cudaStreamSynchronize(p->st));
  return LMB_OK;
}

int lmb_pre_get_background(lmb_pre *p, double *out) {
  int rc = check_pre(p);
  if (rc) return rc;
  LMB_REQUIRE(out, "null output");
  LMB_CUDA(cudaMemcpyAsync(out, p->d_bg, p->npx * sizeof(double), cudaMemcpyDeviceToHost, p->st));
  LMB_CUDA(cudaStreamSynchronize(p->st));
  return LMB_OK;
}

int lmb_pre_median(lmb_pre *p, const void *frame, int32_t dtype, int32_t size, int32_t passes,
                   double *out) {
  int rc = check_pre(p);
  if (rc) return rc;
  LMB_REQUIRE(size >= 1, "median size %d", size);
  LMB_REQUIRE(!(p->ny > 1 && size >= 8 * p->ny) && !(p->nx > 1 && size >= 8 * p->nx),
              "median size %d reaches 8x the %d x %d frame", size, p->ny, p->nx);
  LMB_CUDA(cudaEventRecord(p->ev[EV_MED0], p->st));
  if ((rc = upload_frame(p, frame, dtype))) return rc;
  LMB_CUDA(cudaEventRecord(p->ev[EV_MED_UP], p->st));
  if ((rc = ensure_median_scratch(p))) return rc;
  const unsigned g = (unsigned)grid_for(p->npx, p->num_sms);
  rc = by_dtype(dtype, [&](auto tag) {
    using T = std::remove_const_t<std::remove_pointer_t<decltype(tag)>>;
    to_f64_kernel<T><<<g, kT, 0, p->st>>>(static_cast<const T *>(p->d_raw), p->d_bg, p->npx);
    return LMB_OK;
  });
  if (rc) return rc;
  if (size > 1) {
    for (int i = 0; i < passes; ++i) {
      LMB_CUDA(cudaMemcpyAsync(p->m_img, p->d_bg, p->npx * sizeof(double),
                               cudaMemcpyDeviceToDevice, p->st));
      if ((rc = median_pass(p, p->m_img, p->d_bg, size))) return rc;
    }
  }
  if (out)
    LMB_CUDA(cudaMemcpyAsync(out, p->d_bg, p->npx * sizeof(double), cudaMemcpyDeviceToHost, p->st));
  LMB_CUDA(cudaStreamSynchronize(p->st));
  if (size > 1 && passes > 0)
    return stage_times(p, EV_MED0, EV_MED_UP, 5) || stage_times(p, EV_MED_PASS, EV_MED_RANK, 6) ||
           stage_times(p, EV_MED_RANK, EV_MED_K, 7);
  return stage_times(p, EV_MED0, EV_MED_UP, 5);
}

int lmb_pre_segment(lmb_pre *p, const void *frame, int32_t dtype, const lmb_pre_params *prm,
                    lmb_pre_counts *counts) {
  int rc = check_pre(p);
  if (rc) return rc;
  LMB_REQUIRE(prm, "null parameters");
  LMB_CUDA(cudaEventRecord(p->ev[EV_SEG0], p->st));
  if ((rc = upload_frame(p, frame, dtype))) return rc;
  LMB_CUDA(cudaEventRecord(p->ev[EV_SEG_UP], p->st));
  const unsigned g = (unsigned)grid_for(p->npx, p->num_sms);
  if (prm->override_thresh > 0 || prm->threshold_method == LMB_THR_FIXED) {
    rc = by_dtype(dtype, [&](auto tag) {
      using T = std::remove_const_t<std::remove_pointer_t<decltype(tag)>>;
      subtract_kernel<T><<<g, kT, 0, p->st>>>(static_cast<const T *>(p->d_raw), p->d_bg,
                                              p->d_sub, p->npx);
      return LMB_OK;
    });
    if (rc) return rc;
    set_thresh_kernel<<<1, 1, 0, p->st>>>(
        p->d_state, prm->override_thresh > 0 ? prm->override_thresh : prm->threshold_value);
  } else if (prm->threshold_method == LMB_THR_PERCENTILE) {
    unsigned long long k0;
    int two;
    double gamma;
    LMB_REQUIRE(prm->threshold_percentile >= 0.0 && prm->threshold_percentile <= 100.0,
                "Percentiles must be in the range [0, 100]");
    percentile_plan(p->npx, prm->threshold_percentile, &k0, &two, &gamma);
    sel_init_kernel<<<1, kT, 0, p->st>>>(p->d_state, SEL_ALL, p->npx, k0, two, 1);
    bool done = false;
    if ((rc = value_select(p, dtype, SEL_ALL, k0, two, gamma, &done))) return rc;
    if (!done) {
      if ((rc = run_select(p, SEL_ALL, true))) return rc;
      finish_percentile_kernel<<<1, 1, 0, p->st>>>(p->d_state, gamma);
    }
  } else {
    LMB_REQUIRE(prm->threshold_method == LMB_THR_ADAPTIVE, "threshold method %d",
                prm->threshold_method);
    sel_init_kernel<<<1, kT, 0, p->st>>>(p->d_state, SEL_NZ, p->npx, 0, 0, 1);
    bool done = false;
    if ((rc = value_select(p, dtype, SEL_NZ, 0, 0, 0.0, &done))) return rc;
    if (!done) {
      if ((rc = run_select(p, SEL_NZ, true))) return rc;
      finish_median_kernel<<<1, 1, 0, p->st>>>(p->d_state);
      sel_init_kernel<<<1, kT, 0, p->st>>>(p->d_state, SEL_ABSDEV, p->npx, 0, 0, 0);
      if ((rc = run_select(p, SEL_ABSDEV, true))) return rc;
      finish_adaptive_kernel<<<1, 1, 0, p->st>>>(p->d_state);
    }
  }
  apply_kernel<<<g, kT, 0, p->st>>>(p->d_sub, p->d_state, p->d_t16, p->d_par, p->nx, p->npx);
  LMB_CUDA(cudaGetLastError());
  LMB_CUDA(cudaEventRecord(p->ev[EV_SEG_THR], p->st));
  rc = segment_tail(p, prm->min_area, counts, true);
  if (rc) return rc;
  return stage_times(p, EV_SEG0, EV_SEG_UP, 0) || stage_times(p, EV_SEG_UP, EV_SEG_THR, 1) ||
         stage_times(p, EV_SEG_THR, EV_SEG_CC, 2);
}

int lmb_pre_segment_thresholded(lmb_pre *p, const uint16_t *thresholded, int32_t min_area,
                                lmb_pre_counts *counts) {
  int rc = check_pre(p);
  if (rc) return rc;
  LMB_REQUIRE(thresholded, "null frame");
  LMB_CUDA(cudaMemcpyAsync(p->d_t16, thresholded, p->npx * sizeof(uint16_t),
                           cudaMemcpyHostToDevice, p->st));
  set_thresh_kernel<<<1, 1, 0, p->st>>>(p->d_state, 0.0);
  LMB_CUDA(cudaGetLastError());
  return segment_tail(p, min_area, counts, false);
}

int lmb_pre_centres(lmb_pre *p, double *centres, int32_t cap) {
  int rc = check_pre(p);
  if (rc) return rc;
  LMB_REQUIRE(p->segmented, "no frame segmented yet");
  const int n = std::min(cap, p->last.n_centres);
  LMB_REQUIRE(centres || n == 0, "null output");
  if (n > 0)
    LMB_CUDA(cudaMemcpy(centres, p->d_centres, (size_t)n * 4 * sizeof(double),
                        cudaMemcpyDeviceToHost));
  return LMB_OK;
}

int lmb_pre_stats(lmb_pre *p, int32_t *stats, int32_t cap) {
  int rc = check_pre(p);
  if (rc) return rc;
  LMB_REQUIRE(p->segmented, "no frame segmented yet");
  const int n = std::min(cap, p->last.n_labels - 1);
  LMB_REQUIRE(stats || n == 0, "null output");
  if (n > 0)
    LMB_CUDA(cudaMemcpy(stats, p->d_stats, (size_t)n * 5 * sizeof(int32_t),
                        cudaMemcpyDeviceToHost));
  return LMB_OK;
}

int lmb_pre_images(lmb_pre *p, uint16_t *thresholded, int32_t *labels, uint16_t *filt_img,
                   int32_t *filt_labels) {
  int rc = check_pre(p);
  if (rc) return rc;
  LMB_REQUIRE(p->segmented, "no frame segmented yet");
  const size_t n = p->npx;
  if ((labels || filt_labels) && !p->labels_ready) {
    LMB_CUDA(cudaMemsetAsync(p->d_lab, 0, n * sizeof(int), p->st));
    LMB_CUDA(cudaMemsetAsync(p->d_flab, 0, n * sizeof(int), p->st));
    labels_kernel<<<(unsigned)grid_for(n, p->num_sms), kT, 0, p->st>>>(
        p->d_par, p->d_cid, p->c, p->d_lab, p->d_flab, p->d_fg, p->d_nfg);
    LMB_CUDA(cudaGetLastError());
    p->labels_ready = true;
  }
  if (thresholded)
    LMB_CUDA(cudaMemcpyAsync(thresholded, p->d_t16, n * 2, cudaMemcpyDeviceToHost, p->st));
  if (labels) LMB_CUDA(cudaMemcpyAsync(labels, p->d_lab, n * 4, cudaMemcpyDeviceToHost, p->st));
  if (filt_img)
    LMB_CUDA(cudaMemcpyAsync(filt_img, p->d_filt, n * 2, cudaMemcpyDeviceToHost, p->st));
  if (filt_labels)
    LMB_CUDA(cudaMemcpyAsync(filt_labels, p->d_flab, n * 4, cudaMemcpyDeviceToHost, p->st));
  LMB_CUDA(cudaStreamSynchronize(p->st));
  return LMB_OK;
}

}  // extern "C"

namespace {

// Both blur passes of the last segment's filtered frame into p->d_out.
int blur_launch(lmb_pre *p, const double *weights, int32_t radius, int32_t out_dtype) {
  LMB_REQUIRE(p->segmented, "no frame segmented yet");
  LMB_REQUIRE(weights, "null weights");
  LMB_REQUIRE(radius >= 0 && 2 * radius + 1 <= 1024, "blur radius %d outside 0..511", radius);
  LMB_REQUIRE(out_dtype == LMB_F64 || out_dtype == LMB_F32, "blur output dtype %d", out_dtype);
  if (p->out_in_use) {  // an engine may still be reading the previous blurred frame
    LMB_CUDA(cudaStreamWaitEvent(p->st, p->ev_out_free, 0));
    p->out_in_use = false;
  }
  LMB_CUDA(cudaEventRecord(p->ev[EV_BLUR0], p->st));
  LMB_CUDA(cudaMemcpyAsync(p->d_w, weights, (size_t)(2 * radius + 1) * sizeof(double),
                           cudaMemcpyHostToDevice, p->st));
  const unsigned g = (unsigned)grid_for(p->npx, p->num_sms);
  if (radius >= 1 && radius <= kBlurFixedMaxR) {
    const dim3 tg((p->nx + kBlurTile - 1) / kBlurTile, (p->ny + kBlurTile - 1) / kBlurTile);
    if (out_dtype == LMB_F64)
      blur_tile_r_launch<double>(radius, tg, p->d_filt, p->d_w, p->ny, p->nx,
                                 static_cast<double *>(p->d_out), p->st);
    else
      blur_tile_r_launch<float>(radius, tg, p->d_filt, p->d_w, p->ny, p->nx,
                                static_cast<float *>(p->d_out), p->st);
  } else if (radius <= kBlurTileMaxR) {
    const dim3 tg((p->nx + kBlurTile - 1) / kBlurTile, (p->ny + kBlurTile - 1) / kBlurTile);
    const size_t tsm = blur_tile_smem(radius);
    if (out_dtype == LMB_F64)
      blur_tile_kernel<double><<<tg, 256, tsm, p->st>>>(p->d_filt, p->d_w, radius, p->ny, p->nx,
                                                        static_cast<double *>(p->d_out));
    else
      blur_tile_kernel<float><<<tg, 256, tsm, p->st>>>(p->d_filt, p->d_w, radius, p->ny, p->nx,
                                                       static_cast<float *>(p->d_out));
  } else {
    const size_t sm = (size_t)(2 * radius + 1) * sizeof(double);
    blur_rows_kernel<uint16_t><<<g, kT, sm, p->st>>>(p->d_filt, p->d_w, radius, p->ny, p->nx,
                                                     p->d_tmp);
    if (out_dtype == LMB_F64)
      blur_cols_kernel<double><<<g, kT, sm, p->st>>>(p->d_tmp, p->d_w, radius, p->ny, p->nx,
                                                     static_cast<double *>(p->d_out));
    else
      blur_cols_kernel<float><<<g, kT, sm, p->st>>>(p->d_tmp, p->d_w, radius, p->ny, p->nx,
                                                    static_cast<float *>(p->d_out));
  }
  LMB_CUDA(cudaGetLastError());
  LMB_CUDA(cudaEventRecord(p->ev[EV_BLUR_K], p->st));
  return LMB_OK;
}

}  // namespace

extern "C" {

int lmb_pre_blur(lmb_pre *p, const double *weights, int32_t radius, void *out, int32_t out_dtype) {
  int rc = check_pre(p);
  if (rc) return rc;
  LMB_REQUIRE(out, "null output");
  if ((rc = blur_launch(p, weights, radius, out_dtype))) return rc;
  LMB_CUDA(cudaMemcpyAsync(out, p->d_out, p->npx * (out_dtype == LMB_F64 ? 8 : 4),
                           cudaMemcpyDeviceToHost, p->st));
  LMB_CUDA(cudaEventRecord(p->ev[EV_BLUR_DL], p->st));
  LMB_CUDA(cudaStreamSynchronize(p->st));
  return stage_times(p, EV_BLUR0, EV_BLUR_K, 3) || stage_times(p, EV_BLUR_K, EV_BLUR_DL, 4);
}

int lmb_pre_blur_to_slot(lmb_pre *p, const double *weights, int32_t radius, lmb_engine *e,
                         int32_t slot, int32_t frame_dtype, double *im_scale) {
  int rc = check_pre(p);
  if (rc) return rc;
  LMB_REQUIRE(e, "null engine");
  LMB_REQUIRE(engine_device(e) == p->device, "engine on device %d, preprocessing on device %d",
              engine_device(e), p->device);
  if ((rc = blur_launch(p, weights, radius, frame_dtype))) return rc;
  LMB_CUDA(cudaEventRecord(p->ev_out_ready, p->st));
  rc = engine_load_device_frame(e, slot, p->d_out, frame_dtype, p->ny, p->nx, p->ev_out_ready,
                                p->ev_out_free, im_scale);
  if (rc) return rc;
  p->out_in_use = true;
  LMB_CUDA(cudaStreamSynchronize(p->st));
  return stage_times(p, EV_BLUR0, EV_BLUR_K, 3);
}

int lmb_pre_timings(lmb_pre *p, float *ms, int32_t n) {
  LMB_REQUIRE(p && ms, "null argument");
  for (int i = 0; i < n && i < LMB_PRE_STAGES; ++i) ms[i] = p->ms[i];
  return LMB_OK;
}

}  // extern "C"
