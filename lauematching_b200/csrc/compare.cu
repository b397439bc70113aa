// Compare pass: image quantisation, the batched DB pass, survivor ordering.
//
// Quantisation restates LaueMatchingCPU.c:345-375.  The compare restates
// LaueMatchingCPU.c:668-690 and replaces the reference's compare kernels
// (LaueMatchingGPU.cu:45-81, LaueMatchingGPUStream.cu:69-100); survivors are
// delivered in ascending orientation ID like LaueMatchingCPU.c:781-788.
//
// Batched pass.  Up to 64 images ("slots") are matched in one pass over the
// DB.  For every pixel the occupancy word holds bit k set when slot k's
// uint8 pixel is positive, so one 8-byte gather per spot gives the hit/miss
// of that spot in every image at once; per-slot spot counts are kept as
// bit-sliced counters (bit b of all 64 counters in one word).  Only an
// orientation whose count reaches MinNrSpots in some slot ("candidate") goes
// back over its spots to sum the intensity of that slot in FP64, in record
// order, exactly as the reference does; candidates are rare, so the DB
// stream and the 8-byte gathers are the cost.
//
// DB stream.  A persistent grid walks tiles of TILE consecutive records;
// tile bytes are moved into shared memory by 1-D TMA bulk copies
// (cp.async.bulk) through a STAGES-deep mbarrier ring, so the stream is
// coalesced regardless of the 122-byte record stride.  Waits are bounded
// (2 s of global time) and report through an error word.
#include <climits>
#include <mutex>
#include <vector>

#include "kernels.cuh"

namespace lmb {

// cudaFuncSetAttribute once per (device, kernel, size): later launches, and
// launches captured into a CUDA graph, need no attribute call.
static int ensure_smem(const void *fn, int bytes) {
  static std::mutex mu;
  struct Done {
    int dev;
    const void *fn;
    int bytes;
  };
  static std::vector<Done> done;
  int dev = 0;
  LMB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  for (const auto &d : done)
    if (d.dev == dev && d.fn == fn && d.bytes >= bytes) return LMB_OK;
  LMB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  done.push_back({dev, fn, bytes});
  return LMB_OK;
}

// ----------------------------------------------------------------------------
// Quantisation: max of the positive pixels, then uint8 + occupancy bit.
// ----------------------------------------------------------------------------
template <typename T>
__global__ void quant_max_kernel(const T *__restrict__ img, size_t npx,
                                 unsigned long long *__restrict__ max_bits) {
  double m = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < npx;
       i += (size_t)gridDim.x * blockDim.x) {
    const double v = (double)img[i];
    if (v > m) m = v;  // NaN never compares greater (LaueMatchingCPU.c:357-359)
  }
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double sm[32];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = (threadIdx.x < (blockDim.x >> 5)) ? sm[threadIdx.x] : 0.0;
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    // non-negative doubles order like their bit patterns
    if (threadIdx.x == 0 && m > 0.0) atomicMax(max_bits, (unsigned long long)__double_as_longlong(m));
  }
}

// u8 = v>=255 ? 255 : v<1 ? 1 : (uint8)v  with v = pixel * (255/max), for
// positive pixels; 0 otherwise (LaueMatchingCPU.c:367-375).
template <typename T>
__global__ void quant_u8_kernel(const T *__restrict__ img, size_t npx,
                                const unsigned long long *__restrict__ max_bits,
                                uint8_t *__restrict__ u8, double *__restrict__ f64_keep,
                                unsigned long long *__restrict__ occ, unsigned long long bit,
                                double *__restrict__ scale_out) {
  const double mx = __longlong_as_double((long long)*max_bits);
  const double inv = (mx > 0) ? ddiv(255.0, mx) : 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) *scale_out = (mx > 0) ? ddiv(mx, 255.0) : 1.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < npx;
       i += (size_t)gridDim.x * blockDim.x) {
    const double x = (double)img[i];
    uint8_t q = 0;
    if (x > 0) {
      const double v = dmul(x, inv);
      // (uint8_t)v of a double: x86 converts via a 32-bit cvttsd2si (NaN -> 0)
      q = (v >= 255.0) ? 255 : (v < 1.0) ? 1 : (uint8_t)(x86_trunc_i32(v) & 0xFF);
    }
    u8[i] = q;
    if (f64_keep) f64_keep[i] = x;
    const unsigned long long w = occ[i];
    occ[i] = q ? (w | bit) : (w & ~bit);
  }
}

// Sparse frame upload.  slot_clear: zero the slot's previous positive pixels
// (found through its uint8 image) and their occupancy bits.  sparse_scatter:
// quantise the positive pixels of the new frame (index, value) with the scale
// of its maximum `mx` (computed by the host over the same values) exactly as
// quant_u8_kernel does, and set their occupancy bits.
__global__ void slot_clear_kernel(uint8_t *__restrict__ u8, unsigned long long *__restrict__ occ,
                                  unsigned long long bit, size_t npx) {
  // 16-pixel vector path only when the slot starts on a 16-byte boundary
  const size_t n16 = (reinterpret_cast<uintptr_t>(u8) & 15) ? 0 : npx / 16;
  uint4 *u = reinterpret_cast<uint4 *>(u8);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n16;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint4 v = u[i];
    if ((v.x | v.y | v.z | v.w) == 0u) continue;
    const uint8_t *b = reinterpret_cast<const uint8_t *>(&v);
#pragma unroll
    for (int j = 0; j < 16; j++)
      if (b[j]) occ[i * 16 + j] &= ~bit;
    u[i] = make_uint4(0u, 0u, 0u, 0u);
  }
  for (size_t i = n16 * 16 + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < npx;
       i += (size_t)gridDim.x * blockDim.x) {
    if (u8[i]) {
      occ[i] &= ~bit;
      u8[i] = 0;
    }
  }
}

template <typename T>
__global__ void sparse_scatter_kernel(const uint32_t *__restrict__ idx, const T *__restrict__ val,
                                      size_t nnz, double mx, uint8_t *__restrict__ u8,
                                      unsigned long long *__restrict__ occ, unsigned long long bit,
                                      double *__restrict__ scale_out) {
  const double inv = (mx > 0) ? ddiv(255.0, mx) : 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) *scale_out = (mx > 0) ? ddiv(mx, 255.0) : 1.0;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < nnz;
       j += (size_t)gridDim.x * blockDim.x) {
    const double x = (double)val[j];  // > 0 by construction
    const double v = dmul(x, inv);
    const uint8_t q = (v >= 255.0) ? 255 : (v < 1.0) ? 1 : (uint8_t)(x86_trunc_i32(v) & 0xFF);
    const uint32_t p = idx[j];
    u8[p] = q;
    occ[p] |= bit;
  }
}

int sparse_load_launch(const uint32_t *d_idx, const void *d_val, int dtype, size_t nnz, double mx,
                       uint8_t *d_u8, unsigned long long *d_occ, int slot, double *d_scale_slot,
                       size_t npx, int num_sms, cudaStream_t st) {
  const unsigned long long bit = 1ull << slot;
  const unsigned cb = (unsigned)std::min<size_t>((npx / 16 + 255) / 256 + 1, (size_t)num_sms * 8);
  slot_clear_kernel<<<cb, 256, 0, st>>>(d_u8, d_occ, bit, npx);
  const unsigned sb = (unsigned)std::max<size_t>(1, std::min<size_t>((nnz + 255) / 256, (size_t)num_sms * 8));
  if (dtype == LMB_F64)
    sparse_scatter_kernel<double><<<sb, 256, 0, st>>>(d_idx, static_cast<const double *>(d_val),
                                                      nnz, mx, d_u8, d_occ, bit, d_scale_slot);
  else if (dtype == LMB_F32)
    sparse_scatter_kernel<float><<<sb, 256, 0, st>>>(d_idx, static_cast<const float *>(d_val), nnz,
                                                     mx, d_u8, d_occ, bit, d_scale_slot);
  else
    sparse_scatter_kernel<uint8_t><<<sb, 256, 0, st>>>(
        d_idx, static_cast<const uint8_t *>(d_val), nnz, mx, d_u8, d_occ, bit, d_scale_slot);
  LMB_CUDA(cudaGetLastError());
  return LMB_OK;
}

// Batched sparse upload: blockIdx.y selects the frame.  The arithmetic per
// pixel is that of sparse_scatter_kernel / quant_u8_kernel; the occupancy
// updates are atomic because several slots' bits live in one word.
__global__ void batch_clear_kernel(const SparseFrameDesc *__restrict__ desc,
                                   uint8_t *__restrict__ u8_base,
                                   unsigned long long *__restrict__ occ, size_t npx) {
  const int slot = desc[blockIdx.y].slot;
  uint8_t *u8 = u8_base + (size_t)slot * npx;
  const unsigned long long keep = ~(1ull << slot);
  const size_t n16 = (reinterpret_cast<uintptr_t>(u8) & 15) ? 0 : npx / 16;
  uint4 *u = reinterpret_cast<uint4 *>(u8);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n16;
       i += (size_t)gridDim.x * blockDim.x) {
    const uint4 v = u[i];
    if ((v.x | v.y | v.z | v.w) == 0u) continue;
    const uint8_t *b = reinterpret_cast<const uint8_t *>(&v);
#pragma unroll
    for (int j = 0; j < 16; j++)
      if (b[j]) atomicAnd(&occ[i * 16 + j], keep);
    u[i] = make_uint4(0u, 0u, 0u, 0u);
  }
  for (size_t i = n16 * 16 + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < npx;
       i += (size_t)gridDim.x * blockDim.x) {
    if (u8[i]) {
      atomicAnd(&occ[i], keep);
      u8[i] = 0;
    }
  }
}

template <typename T>
__global__ void batch_scatter_kernel(const SparseFrameDesc *__restrict__ desc,
                                     const uint32_t *__restrict__ idx, const T *__restrict__ val,
                                     uint8_t *__restrict__ u8_base,
                                     unsigned long long *__restrict__ occ,
                                     double *__restrict__ scale, size_t npx) {
  const SparseFrameDesc d = desc[blockIdx.y];
  const double inv = (d.mx > 0) ? ddiv(255.0, d.mx) : 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) scale[d.slot] = (d.mx > 0) ? ddiv(d.mx, 255.0) : 1.0;
  uint8_t *u8 = u8_base + (size_t)d.slot * npx;
  const unsigned long long bit = 1ull << d.slot;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < d.nnz;
       j += (size_t)gridDim.x * blockDim.x) {
    const double x = (double)val[d.off + j];  // > 0 by construction
    const double v = dmul(x, inv);
    const uint8_t q = (v >= 255.0) ? 255 : (v < 1.0) ? 1 : (uint8_t)(x86_trunc_i32(v) & 0xFF);
    const uint32_t p = idx[d.off + j];
    u8[p] = q;
    atomicOr(&occ[p], bit);
  }
}

int batch_sparse_load_launch(const SparseFrameDesc *d_desc, int nframes, uint32_t max_nnz,
                             const uint32_t *d_idx, const void *d_val, int dtype, uint8_t *d_u8,
                             unsigned long long *d_occ, double *d_scale, size_t npx, int num_sms,
                             cudaStream_t st) {
  if (nframes <= 0) return LMB_OK;
  LMB_REQUIRE(nframes <= LMB_MAX_SLOTS, "batch of %d frames", nframes);
  const size_t budget = std::max<size_t>(1, (size_t)num_sms * 8 / nframes);
  const unsigned cb = (unsigned)std::min<size_t>((npx / 16 + 255) / 256 + 1, budget);
  batch_clear_kernel<<<dim3(cb, nframes), 256, 0, st>>>(d_desc, d_u8, d_occ, npx);
  const unsigned sb =
      (unsigned)std::max<size_t>(1, std::min<size_t>(((size_t)max_nnz + 255) / 256, budget));
  const dim3 g(sb, nframes);
  if (dtype == LMB_F64)
    batch_scatter_kernel<double><<<g, 256, 0, st>>>(
        d_desc, d_idx, static_cast<const double *>(d_val), d_u8, d_occ, d_scale, npx);
  else if (dtype == LMB_F32)
    batch_scatter_kernel<float><<<g, 256, 0, st>>>(
        d_desc, d_idx, static_cast<const float *>(d_val), d_u8, d_occ, d_scale, npx);
  else
    batch_scatter_kernel<uint8_t><<<g, 256, 0, st>>>(
        d_desc, d_idx, static_cast<const uint8_t *>(d_val), d_u8, d_occ, d_scale, npx);
  LMB_CUDA(cudaGetLastError());
  return LMB_OK;
}

// ----------------------------------------------------------------------------
// The DB pass.
// ----------------------------------------------------------------------------


static constexpr uint64_t kWaitNs = 2000000000ull;  // bounded TMA waits: 2 s

// Stage and round of consecutive tiles of a ring of ST stages (tile i sits in
// stage i % ST of round i / ST), advanced by step <= ST tiles without a 64-bit
// division per tile.
__device__ __forceinline__ void ring_next(int &st, uint32_t &rd, int ST, int step = 1) {
  st += step;
  if (st >= ST) {
    st -= ST;
    rd++;
  }
}
static constexpr int kGather = 8;                    // spots gathered per group
static constexpr int kSumGroup = 4;                  // pixel values loaded per group
static constexpr int kDirect = 16;  // compact pass: a chunk with this many passable records is
                                    // counted in place, one with fewer goes through the queue

// The spots of one orientation, in record order, as detector pixel indices.
// RecSpots reads the reference record ({count, x0, y0, ...}) and skips
// off-detector pixels like LaueMatchingGPU.cu:65; ListSpots reads the compact
// layout, which holds the on-detector pixels only (same order).
struct RecSpots {
  const uint16_t *rec;
  __device__ __forceinline__ bool pixel(const CmpArgs &a, int s, size_t &p) const {
    const int x = rec[1 + 2 * s], y = rec[2 + 2 * s];
    if (x >= a.W || y >= a.H) return false;
    p = (size_t)y * a.W + x;
    return true;
  }
};
struct ListSpots {
  const uint32_t *sp;
  __device__ __forceinline__ bool pixel(const CmpArgs &, int s, size_t &p) const {
    p = sp[s];
    return true;
  }
};

// Intensity of slot k over one record, in record order (LaueMatchingCPU.c:671-681
// for the uint8 image; :649-653 for the float64 image).  Returns the spot
// count; tot/su receive the FP64 sum and the uint8 sum.
template <class Spots>
__device__ __forceinline__ int slot_sum_body(const CmpArgs &a, const Spots sp, int c, int k,
                                             double &tot_out, int &su_out) {
  const uint8_t *img = a.u8 + (size_t)k * a.npx;
  const double *fim = a.f64 ? a.f64 + (size_t)k * a.npx : nullptr;
  const double sc = a.scale[k];
  int ns = 0, su = 0;
  double tot = 0.0;
  // pixel values loaded kSumGroup at a time (independent loads in flight
  // together), then summed strictly in record order
  for (int s0 = 0; s0 < c; s0 += kSumGroup) {
    uint8_t raw[kSumGroup];
    double fv[kSumGroup];
#pragma unroll
    for (int j = 0; j < kSumGroup; j++) {
      raw[j] = 0;
      fv[j] = 0.0;
      size_t p;
      if (s0 + j < c && sp.pixel(a, s0 + j, p)) {
        raw[j] = img[p];
        if (a.mode != LMB_VALUE_U8) fv[j] = fim[p];
      }
    }
#pragma unroll
    for (int j = 0; j < kSumGroup; j++) {
      if (a.mode == LMB_VALUE_U8) {
        if (raw[j] > 0) {
          tot = dadd(tot, dmul((double)raw[j], sc));
          ns++;
          su += raw[j];
        }
      } else if (fv[j] > 0) {
        tot = dadd(tot, fv[j]);
        ns++;
        su += raw[j];
      }
    }
  }
  tot_out = tot;
  su_out = su;
  return ns;
}

// Called out of line by kernels without a tight register bound; kernels
// bounded for high occupancy (TAG > 1) take it inline, within their bound.
template <class Spots>
__device__ __noinline__ int slot_sum(const CmpArgs &a, const Spots sp, int c, int k,
                                     double &tot_out, int &su_out) {
  return slot_sum_body(a, sp, c, k, tot_out, su_out);
}

// Called by all 32 lanes of a warp (lanes without a record pass valid=false,
// c=0).  c = the record's spot count, clamped to S.
template <int B, class Spots, int TAG = 1>
__device__ __forceinline__ void process(const CmpArgs &a, const Spots sp, int c, uint64_t oid,
                                        uint64_t pol, bool valid) {
  // nSpots <= c, so a record with c < MinNrSpots fails the spot threshold of
  // LaueMatchingCPU.c:683 in every image: nothing to gather or count
  if (!a.full_gather && c < a.min_spots) {
    valid = false;
    c = 0;
  }
  unsigned long long cnt[B];
#pragma unroll
  for (int b = 0; b < B; b++) cnt[b] = 0ull;
  // gathers issued kGather at a time so their L2 latencies overlap
  for (int s0 = 0; s0 < c; s0 += kGather) {
    unsigned long long m[kGather];
#pragma unroll
    for (int j = 0; j < kGather; j++) {
      m[j] = 0ull;
      const int s = s0 + j;
      size_t p;
      if (s < c && sp.pixel(a, s, p)) m[j] = ld_nc_hint(a.occ + p, pol);
    }
#pragma unroll
    for (int j = 0; j < kGather; j++) {
      unsigned long long v = m[j] & a.active;
      if (v) {
#pragma unroll
        for (int b = 0; b < B; b++) {
          const unsigned long long t = cnt[b] & v;
          cnt[b] ^= v;
          v = t;
        }
      }
    }
  }
  // count >= min_spots, bit-sliced, from the most significant bit down
  unsigned long long gt = 0ull, eq = ~0ull;
#pragma unroll
  for (int b = B - 1; b >= 0; b--) {
    if ((a.min_spots >> b) & 1) {
      eq &= cnt[b];
    } else {
      gt |= eq & cnt[b];
      eq &= ~cnt[b];
    }
  }
  const unsigned long long cand = valid ? ((gt | eq) & a.active) : 0ull;
  // Candidates, slot by slot, warp-uniformly: the lanes whose orientation is
  // a candidate for slot k sum it; one leader reserves the warp's survivor
  // positions with a single atomic (warp-aggregated compaction).
  unsigned long long wc = ((unsigned long long)__reduce_or_sync(0xffffffffu, (unsigned)(cand >> 32))
                           << 32) |
                          __reduce_or_sync(0xffffffffu, (unsigned)cand);
  const int lane = threadIdx.x & 31;
  while (wc) {
    const int k = __ffsll((long long)wc) - 1;
    wc &= wc - 1;
    bool pass = false, surv = false;
    double tot = 0.0, score = 0.0;
    int ns = 0, su = 0;
    if ((cand >> k) & 1) {
      if constexpr (TAG > 1)
        ns = slot_sum_body(a, sp, c, k, tot, su);
      else
        ns = slot_sum(a, sp, c, k, tot, su);
      pass = ns >= a.min_spots && tot >= a.min_int;
      if (pass) {
        score = dmul(tot, dsqrt((double)ns));
        surv = score != 0.0;  // collection skips zero scores (LaueMatchingCPU.c:783)
      }
    }
    const unsigned pm = __ballot_sync(0xffffffffu, pass);
    const unsigned sm = __ballot_sync(0xffffffffu, surv);
    unsigned base = 0;
    if (lane == 0) {
      if (pm) atomicAdd(&a.pass_cnt[k], (unsigned)__popc(pm));
      if (sm) base = atomicAdd(&a.surv_cnt[k], (unsigned)__popc(sm));
    }
    base = __shfl_sync(0xffffffffu, base, 0);
    if (surv) {
      const unsigned pos = base + __popc(sm & ((1u << lane) - 1u));
      if (pos < a.cap) {
        lmb_survivor sv;
        sv.id = oid;
        sv.n_spots = ns;
        sv.sum_u8 = su;
        sv.tot_int = tot;
        sv.score = score;
        a.surv[(size_t)k * a.cap + pos] = sv;
      }
    }
  }
}

// One record of the reference layout.
template <int B>
__device__ __forceinline__ void process_rec(const CmpArgs &a, const uint16_t *rec, uint64_t oid,
                                            uint64_t pol, bool valid) {
  int c = valid ? rec[0] : 0;
  if (c > a.S) c = a.S;  // clamp like LaueMatchingGPU.cu:54-55
  process<B>(a, RecSpots{rec}, c, oid, pol, valid);
}

// Variant 0: every thread consumes; thread 0 refills the ring after a block
// barrier.  One orientation per thread per tile.
template <int B>
__global__ void __launch_bounds__(256) compare_ring_kernel(const __grid_constant__ CmpArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
  unsigned char *ring = smem + 256;
  const uint32_t TILE = a.tile;
  const uint64_t G = gridDim.x;
  const int stages = a.stages;
  const uint64_t pol_db = l2_evict_first(), pol_occ = l2_evict_last();

  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; s++) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; s++) {
      const uint64_t tile = blockIdx.x + (uint64_t)s * G;
      if (tile < a.full_tiles) {
        mbar_expect_tx(&bars[s], a.tile_bytes);
        bulk_g2s_hint(ring + (size_t)s * a.tile_bytes,
                      reinterpret_cast<const unsigned char *>(a.db) + tile * a.tile_bytes,
                      a.tile_bytes, &bars[s], pol_db);
      }
    }
  }
  uint64_t it = 0;
  for (uint64_t tile = blockIdx.x; tile < a.ntiles; tile += G, ++it) {
    const int s = (int)(it % stages);
    const uint32_t parity = (uint32_t)((it / stages) & 1);
    const uint64_t oid = tile * TILE + threadIdx.x;
    if (tile < a.full_tiles) {
      const bool ok = mbar_wait_bounded(&bars[s], parity, kWaitNs);
      if (__syncthreads_or(!ok)) {  // block-uniform give-up
        if (threadIdx.x == 0) {
          atomicExch(a.err, DEV_TIMEOUT_TMA);
          // let every copy this block still has in flight land before leaving
          for (int d = 0; d < stages; d++) {
            const uint64_t it2 = it + (uint64_t)d;
            if (blockIdx.x + it2 * G < a.full_tiles)
              mbar_wait_bounded(&bars[it2 % stages], (uint32_t)((it2 / stages) & 1), kWaitNs);
          }
        }
        return;
      }
      const uint16_t *rec = reinterpret_cast<const uint16_t *>(ring + (size_t)s * a.tile_bytes) +
                            (size_t)threadIdx.x * a.R;
      process_rec<B>(a, rec, oid, pol_occ, true);
    } else {
      const bool v = oid < a.n;  // partial last tile: direct loads, whole warps
      process_rec<B>(a, v ? a.db + oid * a.R : a.db, oid, pol_occ, v);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const uint64_t nt = tile + (uint64_t)stages * G;
      if (nt < a.full_tiles) {
        mbar_expect_tx(&bars[s], a.tile_bytes);
        bulk_g2s_hint(ring + (size_t)s * a.tile_bytes,
                      reinterpret_cast<const unsigned char *>(a.db) + nt * a.tile_bytes,
                      a.tile_bytes, &bars[s], pol_db);
      }
    }
  }
}

// Variant 1: warp-specialised.  Warp 0 (one lane) is the producer: it
// refills a stage as soon as the consumers release it (empty barrier), so
// there is no block barrier on the stream.  Consumer warps are grouped: a
// group of tile_sub warps takes one tile (each warp 32 orientations), the
// groups take successive tiles of this block in turn.  Tiles that share a
// stage belong to the same group (stages % groups == 0), so no waiter is ever
// more than one barrier phase ahead.
template <int B>
__global__ void __launch_bounds__(576, 1) compare_ws_kernel(const __grid_constant__ CmpArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int ST = a.stages;
  uint64_t *full = reinterpret_cast<uint64_t *>(smem);
  uint64_t *empty = full + 16;
  unsigned char *ring = smem + 256;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int TS = a.tile_sub;
  const int NG = a.consumers / TS;
  const uint64_t G = gridDim.x;
  const uint64_t my_tiles = (a.ntiles > blockIdx.x) ? (a.ntiles - 1 - blockIdx.x) / G + 1 : 0;
  const uint64_t my_full =
      (a.full_tiles > blockIdx.x) ? (a.full_tiles - 1 - blockIdx.x) / G + 1 : 0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], TS);
    }
    fence_mbar_init();
  }
  __syncthreads();
  if (warp == 0) {
    if (lane != 0) return;
    const uint64_t pol_db = l2_evict_first();
    uint64_t issued = 0;
    int ps = 0;
    uint32_t pr = 0;
    for (uint64_t i = 0; i < my_full; i++, ring_next(ps, pr, ST)) {
      const int s = ps;
      if (pr > 0 && !mbar_wait_bounded(&empty[s], (pr - 1) & 1u, kWaitNs)) {
        atomicExch(a.err, DEV_TIMEOUT_TMA);
        break;
      }
      mbar_expect_tx(&full[s], a.tile_bytes);
      bulk_g2s_hint(ring + (size_t)s * a.tile_bytes,
                    reinterpret_cast<const unsigned char *>(a.db) +
                        (blockIdx.x + i * G) * (uint64_t)a.tile_bytes,
                    a.tile_bytes, &full[s], pol_db);
      issued = i + 1;
    }
    // stay until the last copies have landed (bounded)
    {
      const uint64_t j0 = issued > (uint64_t)ST ? issued - ST : 0;
      int ds = (int)(j0 % ST);
      uint32_t dr = (uint32_t)(j0 / ST);
      for (uint64_t j = j0; j < issued; j++, ring_next(ds, dr, ST))
        mbar_wait_bounded(&full[ds], dr & 1u, kWaitNs);
    }
    return;
  }
  const int cw = warp - 1;
  const int g = cw / TS, sub = cw % TS;
  if (g >= NG) return;
  const uint64_t pol_occ = l2_evict_last();
  int cs = g;  // stage and round of tile i (g < NG <= ST; stages are a multiple of NG)
  uint32_t cr = 0;
  for (uint64_t i = g; i < my_tiles; i += NG, ring_next(cs, cr, ST, NG)) {
    const uint64_t tile = blockIdx.x + i * G;
    const uint64_t oid = tile * a.tile + (uint64_t)sub * 32 + lane;
    if (i < my_full) {
      const int s = cs;
      const bool ok = mbar_wait_bounded(&full[s], cr & 1u, kWaitNs);
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) atomicExch(a.err, DEV_TIMEOUT_TMA);
        return;
      }
      const uint16_t *rec = reinterpret_cast<const uint16_t *>(ring + (size_t)s * a.tile_bytes) +
                            (size_t)(sub * 32 + lane) * a.R;
      process_rec<B>(a, rec, oid, pol_occ, true);
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    } else {
      const bool v = oid < a.n;  // partial last tile: direct loads, whole warps
      process_rec<B>(a, v ? a.db + oid * a.R : a.db, oid, pol_occ, v);
    }
  }
}

// Variant 2: warp-specialised over the compact layout (clist.cu): fixed-size
// tiles of tile_bytes, tile t at cl + t*tile_bytes, each holding nch whole
// 32-record chunks (header: first record, nch; then the uint8 per-chunk
// maximum counts, the uint8 counts, the uint32 chunk bases, the uint32
// on-detector pixel indices in record order).  The producer lane moves whole
// tiles into the ring (one bulk copy each, no table lookup).  The consumer
// warps vote over the per-chunk maxima, 32 chunks at a time, for the chunks
// holding a record with at least MinNrSpots spots (no other record can pass),
// share those out round-robin (the turn carries over from tile to tile, so
// tiles with few such chunks still use every warp), find each lane's first
// spot with a warp prefix sum of the counts, and run the per-record logic of
// the other variants.
template <int B, int MINB>
__global__ void __launch_bounds__(MINB > 1 ? 128 : 576, MINB)
    compare_clist_kernel(const __grid_constant__ CmpArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int ST = a.stages;
  uint64_t *full = reinterpret_cast<uint64_t *>(smem);
  uint64_t *empty = full + 16;
  unsigned char *ring = smem + 256;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int NC = a.consumers;
  const uint64_t G = gridDim.x;
  const uint64_t my_tiles = (a.ntiles > blockIdx.x) ? (a.ntiles - 1 - blockIdx.x) / G + 1 : 0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NC);
    }
    if (a.test_consumer_wait_ns) mbar_init(&full[15], 1);  // nothing ever arrives (ST <= 15)
    fence_mbar_init();
  }
  __syncthreads();
  if (warp == 0) {
    if (lane != 0) return;
    const uint64_t pol_db = l2_evict_first();
    uint64_t issued = 0;
    int ps = 0;
    uint32_t pr = 0;
    for (uint64_t i = 0; i < my_tiles; i++, ring_next(ps, pr, ST)) {
      const int s = ps;
      if (pr > 0 && !mbar_wait_bounded(&empty[s], (pr - 1) & 1u, kWaitNs)) {
        atomicExch(a.err, DEV_TIMEOUT_TMA);
        break;
      }
      const uint64_t t = blockIdx.x + i * G;
      mbar_expect_tx(&full[s], a.tile_bytes);
      bulk_g2s_hint(ring + (size_t)s * a.tile_bytes, a.cl + t * a.tile_bytes, a.tile_bytes,
                    &full[s], pol_db);
      issued = i + 1;
    }
    {
      const uint64_t j0 = issued > (uint64_t)ST ? issued - ST : 0;
      int ds = (int)(j0 % ST);
      uint32_t dr = (uint32_t)(j0 / ST);
      for (uint64_t j = j0; j < issued; j++, ring_next(ds, dr, ST))
        mbar_wait_bounded(&full[ds], dr & 1u, kWaitNs);
    }
    return;
  }
  const int cw = warp - 1;
  if (cw >= NC) return;
  const uint64_t pol_occ = l2_evict_last();
  // This warp's queue of records that can pass, copied out of the ring (id,
  // count, pixel indices at an odd stride): a chunk with few of them feeds the
  // queue, and the queue is counted 32 records at a time on a full warp.
  const uint32_t SP = clist_queue_stride(a.qS);
  unsigned char *qb = ring + (size_t)ST * a.tile_bytes + (size_t)cw * clist_queue_bytes(a.qS);
  uint64_t *q_oid = reinterpret_cast<uint64_t *>(qb);
  uint32_t *q_c = reinterpret_cast<uint32_t *>(qb + 256);
  uint32_t *q_sp = reinterpret_cast<uint32_t *>(qb + 384);
  int qn = 0;
  auto flush = [&]() {
    __syncwarp();
    const bool v = lane < qn;
    process<B, ListSpots, MINB>(a, ListSpots{q_sp + lane * SP}, v ? (int)q_c[lane] : 0,
                                v ? q_oid[lane] : 0,
               pol_occ, v);
    __syncwarp();
    qn = 0;
  };
  uint32_t turn = 0;  // the consumer warp that takes the next chunk
  int cs = 0;
  uint32_t cr = 0;
  for (uint64_t i = 0; i < my_tiles; i++, ring_next(cs, cr, ST)) {
    const int s = cs;
    const bool ok = a.test_consumer_wait_ns
                        ? mbar_wait_bounded(&full[15], 0, a.test_consumer_wait_ns)
                        : mbar_wait_bounded(&full[s], cr & 1u, kWaitNs);
    if (!__all_sync(0xffffffffu, ok)) {
      if (lane == 0) atomicExch(a.err, DEV_TIMEOUT_TMA);
      return;
    }
    const unsigned char *tb = ring + (size_t)s * a.tile_bytes;
    const uint64_t first = *reinterpret_cast<const uint64_t *>(tb);
    const uint32_t nch = *reinterpret_cast<const uint32_t *>(tb + 8);
    const unsigned char *cmax = tb + 16;
    const unsigned char *cnt = tb + clist_cnt_offset(nch);
    const uint32_t *base = reinterpret_cast<const uint32_t *>(tb + clist_base_offset(nch));
    const uint32_t *spots = reinterpret_cast<const uint32_t *>(tb + clist_spot_offset(nch));
    // chunks with a record of at least MinNrSpots spots (every chunk when
    // gathering everything), 32 per vote; the k-th of them in the block's
    // running order goes to consumer warp k mod NC
    const int need = a.full_gather ? 0 : a.min_spots;
    for (uint32_t j0 = 0; j0 < nch; j0 += 32) {
      unsigned m = __ballot_sync(0xffffffffu, j0 + lane < nch && cmax[j0 + lane] >= need);
      while (m) {
        const uint32_t ch = j0 + (uint32_t)(__ffs(m) - 1);
        m &= m - 1;
        const bool mine = turn == (uint32_t)cw;
        turn = (turn + 1 == (uint32_t)NC) ? 0 : turn + 1;
        if (!mine) continue;
        const uint64_t oid = first + ch * 32 + lane;
        const bool valid = oid < a.n;
        const int c = valid ? cnt[ch * 32 + lane] : 0;
        int x = c;  // inclusive prefix sum of the counts over the warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, x, o);
          if (lane >= o) x += y;
        }
        const uint32_t *my = spots + base[ch] + (x - c);
        // a record longer than a queue entry cannot come from a layout whose
        // largest count sized the queue; should one appear, fail the pass
        if (valid && c >= need && c > a.qS) atomicExch(a.err, DEV_BAD_QUEUE);
        unsigned qm = __ballot_sync(0xffffffffu, valid && c >= need && c <= a.qS);
        if (__popc(qm) >= kDirect) {  // many can pass: count the chunk in place
          process<B, ListSpots, MINB>(a, ListSpots{my}, c, oid, pol_occ, valid);
          continue;
        }
        while (qm) {  // into the queue, emptying it whenever it fills
          unsigned rest = qm;
          for (int r = 32 - qn; r > 0 && rest; r--) rest &= rest - 1;
          const unsigned take = qm & ~rest;
          if ((take >> lane) & 1u) {
            const int pos = qn + __popc(take & ((1u << lane) - 1u));
            q_oid[pos] = oid;
            q_c[pos] = (uint32_t)c;
            for (int k = 0; k < c; k++) q_sp[pos * SP + k] = my[k];
          }
          qn += __popc(take);
          qm = rest;
          if (qn == 32) flush();
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
  if (qn) flush();
}

// ----------------------------------------------------------------------------
// Variant 4: the compact layout filtered by the batch's cell mask.
//
// With detector geometries that put ~15-20 spots of every orientation on the
// detector, nearly every record can reach MinNrSpots and the pass is the
// 8-byte occupancy gathers of all their spots (~1.5e9 per pass at 1e8
// records), not the DB stream.  But the batch's frames are sparse: at K = 64
// the union of their positive pixels covers ~12 % of the detector.  The cell
// mask holds one bit per cell of 2^cm_shift consecutive pixels, set when a
// pixel of the cell is positive in some slot of the pass; it is built per
// pass (cellmask_kernel) and copied into each block's shared memory.  A spot
// on an unmarked cell is zero in every slot, so
//   * it adds nothing to any count or sum and is dropped from the record's
//     spot list (the remaining spots keep record order, so the FP64 sums are
//     those of the reference: zero pixels are skipped there too);
//   * a record with fewer than MinNrSpots spots on marked cells cannot pass
//     in any slot (LaueMatchingCPU.c:683) and is not gathered at all.
// Consumer warps go through a chunk's spot array 32 spots at a time (one
// conflict-free shared-memory read per lane), test each spot's cell, and
// compact the hits into the warp's hit list in order; per window the hit
// bits and the hits before it give every record its hit range with two
// lookups.  The records that can still pass are counted from their hit
// ranges with the per-record logic of the other variants.
// ----------------------------------------------------------------------------
__global__ void cellmask_kernel(const unsigned long long *__restrict__ occ, uint64_t npx,
                                unsigned long long active, int shift, uint64_t nslots,
                                uint32_t *__restrict__ mask) {
  // thread per cell; nslots (32 x the mask words) and the grid stride are
  // multiples of 32, so whole warps run every iteration together
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < nslots;
       c += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p0 = c << shift;
    const uint64_t p1 = p0 + (1ull << shift) < npx ? p0 + (1ull << shift) : npx;
    unsigned long long any = 0ull;
    for (uint64_t p = p0; p < p1; p++) any |= occ[p];
    const unsigned b = __ballot_sync(0xffffffffu, (any & active) != 0ull);
    if ((threadIdx.x & 31) == 0) mask[c >> 5] = b;
  }
}

int cellmask_launch(const unsigned long long *d_occ, uint64_t npx, unsigned long long active,
                    int shift, uint32_t cm_bytes, uint32_t *d_mask, int num_sms, cudaStream_t st) {
  const uint64_t nslots = (uint64_t)(cm_bytes / 4) * 32;
  const unsigned blocks =
      (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((nslots + 255) / 256, (uint64_t)num_sms * 8));
  cellmask_kernel<<<blocks, 256, 0, st>>>(d_occ, npx, active, shift, nslots, d_mask);
  LMB_CUDA(cudaGetLastError());
  return LMB_OK;
}

template <int B>
__global__ void __launch_bounds__(32 * 13, 1) compare_cell_kernel(const __grid_constant__ CmpArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  const int ST = a.stages;
  uint64_t *full = reinterpret_cast<uint64_t *>(smem);
  uint64_t *empty = full + 16;
  uint32_t *cm = reinterpret_cast<uint32_t *>(smem + 256);
  unsigned char *ring = smem + 256 + a.cm_bytes;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int NC = a.consumers;
  const uint64_t G = gridDim.x;
  const uint64_t my_tiles = (a.ntiles > blockIdx.x) ? (a.ntiles - 1 - blockIdx.x) / G + 1 : 0;
  {  // the pass's cell mask into shared memory
    const uint4 *src = reinterpret_cast<const uint4 *>(a.cellmask);
    uint4 *dst = reinterpret_cast<uint4 *>(cm);
    for (uint32_t i = threadIdx.x; i < a.cm_bytes / 16; i += blockDim.x) dst[i] = src[i];
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NC);
    }
    if (a.test_consumer_wait_ns) mbar_init(&full[15], 1);  // nothing ever arrives (ST <= 15)
    fence_mbar_init();
  }
  __syncthreads();
  if (warp == 0) {
    if (lane != 0) return;
    const uint64_t pol_db = l2_evict_first();
    uint64_t issued = 0;
    int ps = 0;
    uint32_t pr = 0;
    for (uint64_t i = 0; i < my_tiles; i++, ring_next(ps, pr, ST)) {
      const int s = ps;
      if (pr > 0 && !mbar_wait_bounded(&empty[s], (pr - 1) & 1u, kWaitNs)) {
        atomicExch(a.err, DEV_TIMEOUT_TMA);
        break;
      }
      const uint64_t t = blockIdx.x + i * G;
      mbar_expect_tx(&full[s], a.tile_bytes);
      bulk_g2s_hint(ring + (size_t)s * a.tile_bytes, a.cl + t * a.tile_bytes, a.tile_bytes,
                    &full[s], pol_db);
      issued = i + 1;
    }
    {
      const uint64_t j0 = issued > (uint64_t)ST ? issued - ST : 0;
      int ds = (int)(j0 % ST);
      uint32_t dr = (uint32_t)(j0 / ST);
      for (uint64_t j = j0; j < issued; j++, ring_next(ds, dr, ST))
        mbar_wait_bounded(&full[ds], dr & 1u, kWaitNs);
    }
    return;
  }
  const int cw = warp - 1;
  if (cw >= NC) return;
  const uint64_t pol_occ = l2_evict_last();
  const uint32_t QS = (uint32_t)(a.qS < 1 ? 1 : a.qS);
  unsigned char *wb = ring + (size_t)ST * a.tile_bytes +
                      (size_t)cw * cell_warp_bytes(a.qS, a.cell_queue);
  uint32_t *hl = reinterpret_cast<uint32_t *>(wb);
  uint32_t *wm = hl + 32u * QS;  // per window: hit bits
  uint32_t *cum = wm + QS;       // per window: hits before it
  // the candidate queue (cell_queue): id, count, marked spots at an odd stride
  const uint32_t SP = clist_queue_stride(a.qS);
  unsigned char *qb = wb + cell_warp_bytes(a.qS);
  uint64_t *q_oid = reinterpret_cast<uint64_t *>(qb);
  uint32_t *q_c = reinterpret_cast<uint32_t *>(qb + 256);
  uint32_t *q_sp = reinterpret_cast<uint32_t *>(qb + 384);
  int qn = 0;
  auto flush = [&]() {
    __syncwarp();
    const bool v = lane < qn;
    process<B, ListSpots, 1>(a, ListSpots{q_sp + lane * SP}, v ? (int)q_c[lane] : 0,
                             v ? q_oid[lane] : 0, pol_occ, v);
    __syncwarp();
    qn = 0;
  };
  const unsigned lt = (1u << lane) - 1u;
  const int need = a.full_gather ? 0 : a.min_spots;
  const int sh = a.cm_shift;
  uint32_t turn = 0;
  int cs = 0;
  uint32_t cr = 0;
  for (uint64_t i = 0; i < my_tiles; i++, ring_next(cs, cr, ST)) {
    const int s = cs;
    const bool ok = a.test_consumer_wait_ns
                        ? mbar_wait_bounded(&full[15], 0, a.test_consumer_wait_ns)
                        : mbar_wait_bounded(&full[s], cr & 1u, kWaitNs);
    if (!__all_sync(0xffffffffu, ok)) {
      if (lane == 0) atomicExch(a.err, DEV_TIMEOUT_TMA);
      return;
    }
    const unsigned char *tb = ring + (size_t)s * a.tile_bytes;
    const uint64_t first = *reinterpret_cast<const uint64_t *>(tb);
    const uint32_t nch = *reinterpret_cast<const uint32_t *>(tb + 8);
    const unsigned char *cmax = tb + 16;
    const unsigned char *cnt = tb + clist_cnt_offset(nch);
    const uint32_t *base = reinterpret_cast<const uint32_t *>(tb + clist_base_offset(nch));
    const uint32_t *spots = reinterpret_cast<const uint32_t *>(tb + clist_spot_offset(nch));
    for (uint32_t j0 = 0; j0 < nch; j0 += 32) {
      unsigned m = __ballot_sync(0xffffffffu, j0 + lane < nch && cmax[j0 + lane] >= need);
      while (m) {
        const uint32_t ch = j0 + (uint32_t)(__ffs(m) - 1);
        m &= m - 1;
        const bool mine = turn == (uint32_t)cw;
        turn = (turn + 1 == (uint32_t)NC) ? 0 : turn + 1;
        if (!mine) continue;
        const uint64_t oid = first + ch * 32 + lane;
        const bool valid = oid < a.n;
        const int c = valid ? cnt[ch * 32 + lane] : 0;
        if (valid && c > a.qS) atomicExch(a.err, DEV_BAD_QUEUE);  // cannot come from this layout
        int x = c;  // inclusive prefix sum of the counts over the warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, x, o);
          if (lane >= o) x += y;
        }
        // the chunk's spots in windows of 32 (total <= 32 * qS: at most qS windows)
        const uint32_t total = min((uint32_t)__shfl_sync(0xffffffffu, x, 31), 32u * QS);
        const uint32_t *sp = spots + base[ch];
        uint32_t hb = 0;
        for (uint32_t w0 = 0; w0 < total; w0 += 32) {
          const uint32_t k = w0 + lane;
          uint32_t p = 0;
          bool h = false;
          if (k < total) {
            p = sp[k];
            const uint32_t q = p >> sh;
            h = (cm[q >> 5] >> (q & 31u)) & 1u;
          }
          const unsigned hm = __ballot_sync(0xffffffffu, h);
          if (h) hl[hb + __popc(hm & lt)] = p;
          if (lane == 0) {
            wm[w0 >> 5] = hm;
            cum[w0 >> 5] = hb;
          }
          hb += (uint32_t)__popc(hm);
        }
        __syncwarp();
        // this record's spots are [x - c, x) of the chunk; its hits, in order,
        // are [h0, h1) of the hit list
        auto hits_before = [&](uint32_t k) -> uint32_t {
          if (k >= total) return hb;
          const uint32_t w = k >> 5;
          return cum[w] + (uint32_t)__popc(wm[w] & ((1u << (k & 31u)) - 1u));
        };
        const uint32_t xe = min((uint32_t)x, total), xs = min((uint32_t)(x - c), total);
        const uint32_t h0 = hits_before(xs);
        const int ub = (int)(hits_before(xe) - h0);
        const bool cand = valid && c <= a.qS && ub >= need;
        if (a.cell_queue) {
          // into the queue (marked spots only, in order), emptied when full
          unsigned qm = __ballot_sync(0xffffffffu, cand);
          while (qm) {
            unsigned rest = qm;
            for (int r = 32 - qn; r > 0 && rest; r--) rest &= rest - 1;
            const unsigned take = qm & ~rest;
            if ((take >> lane) & 1u) {
              const int pos = qn + __popc(take & ((1u << lane) - 1u));
              q_oid[pos] = oid;
              q_c[pos] = (uint32_t)ub;
              for (int k = 0; k < ub; k++) q_sp[pos * SP + k] = hl[h0 + k];
            }
            qn += __popc(take);
            qm = rest;
            if (qn == 32) flush();
          }
        } else if (__any_sync(0xffffffffu, cand)) {
          process<B, ListSpots, 1>(a, ListSpots{hl + h0}, cand ? ub : 0, oid, pol_occ, cand);
        }
        __syncwarp();
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
  if (qn) flush();
}

// ----------------------------------------------------------------------------
// Variant 5: the cell-mask filter and the counting of its candidates as two
// kernels.
//
// In one kernel (variant 4) the per-record counting logic rides along with
// the spot filter: its registers and branches weigh on every chunk, and the
// chunks of a tile are dealt out across all consumer warps, so each warp
// walks every chunk of every tile.  Here the filter kernel only streams and
// filters: one ring stage per consumer warp, the warp takes whole tiles (the
// producer prefetches the warp's next tile into L2 while the warp works),
// tests each spot's cell 64 spots at a time, and appends the records that can
// still pass (at least MinNrSpots spots on marked cells) with their marked
// pixels, in record order, to its block's region of a candidate buffer.  The
// counting kernel then runs the per-record logic of the other variants on
// full warps of candidates.  Survivors and pass counts are those of the other
// variants (the candidate set and each candidate's nonzero spots are the
// same; order is restored by the ordering kernel).
// ----------------------------------------------------------------------------
__global__ void __launch_bounds__(32 * 25, 1) cell_filter_kernel(const __grid_constant__ CmpArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  // consumers / stages warps share a ring stage (its tiles), splitting each
  // tile's chunks between them
  const int ST = a.stages;
  const int CPT = a.consumers / a.stages;
  uint64_t *full = reinterpret_cast<uint64_t *>(smem);
  uint64_t *empty = full + 16;
  uint32_t *ctr = reinterpret_cast<uint32_t *>(smem + 256);  // entries, pixels, warps done
  uint32_t *cm = reinterpret_cast<uint32_t *>(smem + 384);
  unsigned char *ring = smem + 384 + a.cm_bytes;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int NC = a.consumers;
  const uint64_t G = gridDim.x;
  const uint64_t my_tiles = (a.ntiles > blockIdx.x) ? (a.ntiles - 1 - blockIdx.x) / G + 1 : 0;
  {  // the pass's cell mask into shared memory
    const uint4 *src = reinterpret_cast<const uint4 *>(a.cellmask);
    uint4 *dst = reinterpret_cast<uint4 *>(cm);
    for (uint32_t i = threadIdx.x; i < a.cm_bytes / 16; i += blockDim.x) dst[i] = src[i];
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], CPT);
    }
    ctr[0] = ctr[1] = ctr[2] = 0u;
    fence_mbar_init();
  }
  __syncthreads();
  if (warp == 0) {
    if (lane != 0) return;
    const uint64_t pol_db = l2_evict_first();
    uint64_t issued = 0;
    int ps = 0;
    uint32_t pr = 0;
    for (uint64_t i = 0; i < my_tiles; i++, ring_next(ps, pr, ST)) {
      const int s = ps;
      if (pr > 0 && !mbar_wait_bounded(&empty[s], (pr - 1) & 1u, kWaitNs)) {
        atomicExch(a.err, DEV_TIMEOUT_TMA);
        break;
      }
      const uint64_t t = blockIdx.x + i * G;
      mbar_expect_tx(&full[s], a.tile_bytes);
      bulk_g2s_hint(ring + (size_t)s * a.tile_bytes, a.cl + t * a.tile_bytes, a.tile_bytes,
                    &full[s], pol_db);
      // the stage's next tile, into L2 while this one is worked on
      if (i + ST < my_tiles) bulk_prefetch_l2(a.cl + (t + ST * G) * a.tile_bytes, a.tile_bytes);
      issued = i + 1;
    }
    {
      const uint64_t j0 = issued > (uint64_t)ST ? issued - ST : 0;
      int ds = (int)(j0 % ST);
      uint32_t dr = (uint32_t)(j0 / ST);
      for (uint64_t j = j0; j < issued; j++, ring_next(ds, dr, ST))
        mbar_wait_bounded(&full[ds], dr & 1u, kWaitNs);
    }
    return;
  }
  const int cw = warp - 1;
  if (cw >= NC) return;
  const uint32_t QS = (uint32_t)(a.qS < 1 ? 1 : a.qS);
  uint32_t *wm = reinterpret_cast<uint32_t *>(ring + (size_t)ST * a.tile_bytes +
                                              (size_t)cw * filter_warp_bytes(a.qS));
  const unsigned lt = (1u << lane) - 1u;
  const int need = a.full_gather ? 0 : a.min_spots;
  const int sh = a.cm_shift;
  const uint64_t e_base = a.cq_ebase[blockIdx.x], e_cap = a.cq_ebase[blockIdx.x + 1] - e_base;
  const uint64_t p_base = a.cq_pbase[blockIdx.x], p_cap = a.cq_pbase[blockIdx.x + 1] - p_base;
  CandEntry *E = a.cq_e + e_base;
  uint32_t *P = a.cq_pix + p_base;
  const int s = cw / CPT, sub = cw % CPT;  // this warp's ring stage, its share of the chunks
  uint32_t rd = 0;  // round of tile i (i / ST)
  for (uint64_t i = (uint64_t)s; i < my_tiles; i += (uint64_t)ST, rd++) {
    const bool ok = mbar_wait_bounded(&full[s], rd & 1u, kWaitNs);
    if (!__all_sync(0xffffffffu, ok)) {
      if (lane == 0) atomicExch(a.err, DEV_TIMEOUT_TMA);
      break;
    }
    const unsigned char *tb = ring + (size_t)s * a.tile_bytes;
    const uint64_t first = *reinterpret_cast<const uint64_t *>(tb);
    const uint32_t nch = *reinterpret_cast<const uint32_t *>(tb + 8);
    const unsigned char *cmax = tb + 16;
    const unsigned char *cnt = tb + clist_cnt_offset(nch);
    const uint32_t *base = reinterpret_cast<const uint32_t *>(tb + clist_base_offset(nch));
    const uint32_t *spots = reinterpret_cast<const uint32_t *>(tb + clist_spot_offset(nch));
    uint32_t turn = 0;  // the k-th chunk that can pass goes to sub-warp k mod CPT
    for (uint32_t j0 = 0; j0 < nch; j0 += 32) {
      unsigned m = __ballot_sync(0xffffffffu, j0 + lane < nch && cmax[j0 + lane] >= need);
      while (m) {
        const uint32_t ch = j0 + (uint32_t)(__ffs(m) - 1);
        m &= m - 1;
        const bool take = turn == (uint32_t)sub;
        turn = (turn + 1 == (uint32_t)CPT) ? 0 : turn + 1;
        if (!take) continue;
        const uint64_t oid = first + ch * 32 + lane;
        const bool valid = oid < a.n;
        const int c = valid ? cnt[ch * 32 + lane] : 0;
        if (valid && c > a.qS) atomicExch(a.err, DEV_BAD_QUEUE);  // cannot come from this layout
        int x = c;  // inclusive prefix sum of the counts over the warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, x, o);
          if (lane >= o) x += y;
        }
        const uint32_t total = min((uint32_t)__shfl_sync(0xffffffffu, x, 31), 32u * QS);
        const uint32_t *sp = spots + base[ch];
        // hit bits of the chunk's spots, four 32-spot windows per step
        for (uint32_t w0 = 0; w0 < total; w0 += 128) {
          bool h[4];
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const uint32_t k = w0 + 32u * (uint32_t)u + (uint32_t)lane;
            h[u] = false;
            if (k < total) {
              const uint32_t q = sp[k] >> sh;
              h[u] = (cm[q >> 5] >> (q & 31u)) & 1u;
            }
          }
          unsigned bw[4];
#pragma unroll
          for (int u = 0; u < 4; u++) bw[u] = __ballot_sync(0xffffffffu, h[u]);
          if (lane == 0) {
#pragma unroll
            for (int u = 0; u < 4; u++)
              if (w0 + 32u * (uint32_t)u < total) wm[(w0 >> 5) + (uint32_t)u] = bw[u];
          }
        }
        __syncwarp();
        // this record's spots are [xs, xe) of the chunk: its marked ones
        const uint32_t xe = min((uint32_t)x, total), xs = min((uint32_t)(x - c), total);
        int ub = 0;
        for (uint32_t w = xs >> 5; xe > xs && w <= (xe - 1) >> 5; w++) {
          unsigned mw = wm[w];
          const int lo = (int)xs - (int)(w << 5), hi = (int)xe - (int)(w << 5);
          if (lo > 0) mw &= ~0u << lo;
          if (hi < 32) mw &= (1u << hi) - 1u;
          ub += __popc(mw);
        }
        const bool cand = valid && c <= a.qS && ub >= need;
        const unsigned cmk = __ballot_sync(0xffffffffu, cand);
        if (cmk) {
          // the warp's places in the block's region, one reservation per
          // chunk: an entry per candidate, and pixel room for all the chunk's
          // spots, so a candidate's pixels go where its spots sit in the chunk
          // (its count prefix; the room a region holds covers every spot)
          uint32_t e0 = 0, p0 = 0;
          if (lane == 0) {
            e0 = atomicAdd(&ctr[0], (uint32_t)__popc(cmk));
            p0 = atomicAdd(&ctr[1], total);
          }
          e0 = __shfl_sync(0xffffffffu, e0, 0);
          p0 = __shfl_sync(0xffffffffu, p0, 0);
          if (cand) {
            const uint64_t e = (uint64_t)e0 + (uint64_t)__popc(cmk & lt);
            const uint64_t off = (uint64_t)p0 + (uint64_t)xs;
            if (e < e_cap && off + (uint64_t)ub <= p_cap) {
              CandEntry ce;
              ce.oid = oid;
              ce.off = (uint32_t)off;
              ce.n = (uint32_t)ub;
              E[e] = ce;
              uint32_t k = 0;  // its marked pixels in record order (none when xe == xs)
              for (uint32_t w = xs >> 5; xe > xs && w <= (xe - 1) >> 5; w++) {
                unsigned mw = wm[w];
                const int lo = (int)xs - (int)(w << 5), hi = (int)xe - (int)(w << 5);
                if (lo > 0) mw &= ~0u << lo;
                if (hi < 32) mw &= (1u << hi) - 1u;
                while (mw) {
                  const int b = __ffs(mw) - 1;
                  mw &= mw - 1;
                  P[off + k++] = sp[(w << 5) + (uint32_t)b];
                }
              }
            } else {
              atomicExch(a.err, DEV_BAD_QUEUE);  // regions hold every record: cannot happen
            }
          }
        }
        __syncwarp();
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
  // the last consumer warp to finish publishes the block's counts
  __syncwarp();
  if (lane == 0) {
    __threadfence_block();
    if (atomicAdd(&ctr[2], 1u) == (uint32_t)NC - 1) {
      a.cq_count[2 * blockIdx.x] = atomicAdd(&ctr[0], 0u);
      a.cq_count[2 * blockIdx.x + 1] = atomicAdd(&ctr[1], 0u);
    }
  }
}

// The filter's candidates, 32 per warp: the per-record logic of the other
// variants over each candidate's marked pixels.  blockIdx.y = the filter
// block whose region is read.
template <int B>
__global__ void __launch_bounds__(256) cell_count_kernel(const __grid_constant__ CmpArgs a) {
  const uint32_t b = blockIdx.y;
  const uint64_t cap = a.cq_ebase[b + 1] - a.cq_ebase[b];
  const uint64_t n = min((uint64_t)a.cq_count[2 * b], cap);
  const CandEntry *E = a.cq_e + a.cq_ebase[b];
  const uint32_t *P = a.cq_pix + a.cq_pbase[b];
  const int lane = threadIdx.x & 31;
  const uint64_t wpb = blockDim.x >> 5;
  const uint64_t nw = gridDim.x * wpb;
  const uint64_t pol_occ = l2_evict_last();
  for (uint64_t g = (blockIdx.x * wpb + (threadIdx.x >> 5)) * 32; g < n; g += nw * 32) {
    const uint64_t e = g + lane;
    const bool v = e < n;
    CandEntry ce{0ull, 0u, 0u};
    if (v) ce = E[e];
    process<B, ListSpots, 1>(a, ListSpots{P + ce.off}, v ? (int)ce.n : 0, ce.oid, pol_occ, v);
  }
}

// ----------------------------------------------------------------------------
// Ordering: per slot, sort survivors by ID (keys id<<24 | index), bitonic.
// ----------------------------------------------------------------------------


static constexpr uint32_t kSmemSortMax = 8192;

__device__ __forceinline__ void bitonic(unsigned long long *keys, uint32_t P) {
  for (uint32_t size = 2; size <= P; size <<= 1) {
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t i = threadIdx.x; i < (P >> 1); i += blockDim.x) {
        const uint32_t lo = 2 * i - (i & (stride - 1));
        const uint32_t hi = lo + stride;
        const bool asc = (lo & size) == 0;
        const unsigned long long x = keys[lo], y = keys[hi];
        if ((x > y) == asc) {
          keys[lo] = y;
          keys[hi] = x;
        }
      }
      __syncthreads();
    }
  }
}

// One compare-exchange step of the bitonic network over the pairs (lo, lo +
// stride) of keys[0, m), m a power of two; `base` is keys[0]'s index in the
// whole sequence, which decides each pair's direction for this `size`.
__device__ __forceinline__ void bitonic_step(unsigned long long *keys, uint32_t m, uint32_t base,
                                             uint32_t size, uint32_t stride) {
  for (uint32_t i = threadIdx.x; i < (m >> 1); i += blockDim.x) {
    const uint32_t lo = 2 * i - (i & (stride - 1));
    const uint32_t hi = lo + stride;
    const bool asc = ((base + lo) & size) == 0;
    const unsigned long long x = keys[lo], y = keys[hi];
    if ((x > y) == asc) {
      keys[lo] = y;
      keys[hi] = x;
    }
  }
  __syncthreads();
}

// The bitonic network of bitonic() over P > kSmemSortMax keys in global
// memory (P a power of two), with every stage whose pairs lie within one
// tile of kSmemSortMax keys run on that tile in shared memory: the tiles are
// sorted there first (sizes up to the tile), and each larger size runs its
// strides of a tile or more over global memory and then the smaller strides
// tile by tile.  Same comparisons as bitonic(), so the same order; global
// passes per size log2(size / tile) instead of log2(size).
__device__ void bitonic_tiled(unsigned long long *g, uint32_t P, unsigned long long *sk) {
  constexpr uint32_t T = kSmemSortMax;
  for (uint32_t t0 = 0; t0 < P; t0 += T) {
    for (uint32_t i = threadIdx.x; i < T; i += blockDim.x) sk[i] = g[t0 + i];
    __syncthreads();
    for (uint32_t size = 2; size <= T; size <<= 1)
      for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) bitonic_step(sk, T, t0, size, stride);
    for (uint32_t i = threadIdx.x; i < T; i += blockDim.x) g[t0 + i] = sk[i];
    __syncthreads();
  }
  for (uint32_t size = 2 * T; size <= P; size <<= 1) {
    for (uint32_t stride = size >> 1; stride >= T; stride >>= 1) bitonic_step(g, P, 0, size, stride);
    for (uint32_t t0 = 0; t0 < P; t0 += T) {
      for (uint32_t i = threadIdx.x; i < T; i += blockDim.x) sk[i] = g[t0 + i];
      __syncthreads();
      for (uint32_t stride = T >> 1; stride > 0; stride >>= 1) bitonic_step(sk, T, t0, size, stride);
      for (uint32_t i = threadIdx.x; i < T; i += blockDim.x) g[t0 + i] = sk[i];
      __syncthreads();
    }
  }
}

__global__ void __launch_bounds__(1024) order_kernel(OrderArgs a) {
  extern __shared__ __align__(16) unsigned long long sk[];  // kSmemSortMax keys
  const int k = a.slots[blockIdx.x];
  const uint32_t n = min(a.surv_cnt[k], a.cap);
  if (n == 0) return;
  uint32_t P = 1;
  while (P < n) P <<= 1;
  unsigned long long *keys = (P <= kSmemSortMax) ? sk : a.scratch + (size_t)k * a.cap2;
  const lmb_survivor *src = a.surv + (size_t)k * a.cap;
  for (uint32_t i = threadIdx.x; i < P; i += blockDim.x)
    keys[i] = (i < n) ? ((src[i].id << 24) | i) : ~0ull;
  __syncthreads();
  if (P <= kSmemSortMax)
    bitonic(keys, P);
  else
    bitonic_tiled(keys, P, sk);
  lmb_survivor *dst = a.out + (size_t)k * a.cap;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[keys[i] & 0xFFFFFFull];
}

// ----------------------------------------------------------------------------
// Launchers
// ----------------------------------------------------------------------------
int quantize_launch(const void *d_img, int dtype, size_t npx, unsigned long long *d_max_bits,
                    uint8_t *d_u8, double *d_f64_keep, unsigned long long *d_occ, int slot,
                    double *d_scale_slot, int num_sms, cudaStream_t st) {
  LMB_CUDA(cudaMemsetAsync(d_max_bits, 0, sizeof(unsigned long long), st));
  const unsigned blocks = (unsigned)std::min<size_t>((npx + 255) / 256, (size_t)num_sms * 8);
  const unsigned long long bit = 1ull << slot;
  if (dtype == LMB_F64) {
    const double *p = static_cast<const double *>(d_img);
    quant_max_kernel<double><<<blocks, 256, 0, st>>>(p, npx, d_max_bits);
    quant_u8_kernel<double><<<blocks, 256, 0, st>>>(p, npx, d_max_bits, d_u8, d_f64_keep, d_occ,
                                                     bit, d_scale_slot);
  } else if (dtype == LMB_F32) {
    const float *p = static_cast<const float *>(d_img);
    quant_max_kernel<float><<<blocks, 256, 0, st>>>(p, npx, d_max_bits);
    quant_u8_kernel<float><<<blocks, 256, 0, st>>>(p, npx, d_max_bits, d_u8, d_f64_keep, d_occ,
                                                    bit, d_scale_slot);
  } else {
    const uint8_t *p = static_cast<const uint8_t *>(d_img);
    quant_max_kernel<uint8_t><<<blocks, 256, 0, st>>>(p, npx, d_max_bits);
    quant_u8_kernel<uint8_t><<<blocks, 256, 0, st>>>(p, npx, d_max_bits, d_u8, d_f64_keep, d_occ,
                                                      bit, d_scale_slot);
  }
  LMB_CUDA(cudaGetLastError());
  return LMB_OK;
}

static int counter_bits(int S) {
  int b = 1;
  while ((1 << b) <= S) b++;
  return b;
}

// Launch shape for records of R uint16: the fields set in `req` (from the
// tuning table), defaults for the rest, clamped to what fits.
CompareTuning compare_config(int R, const CompareTuning &req) {
  CompareTuning c = req;
  const size_t rb = (size_t)R * 2;
  if (c.variant == 5) {  // cell-mask filter + counting kernel: one filter block per SM
    c.tile_sub = 0;
    // stages (tiles in flight) and consumer warps, a multiple of them: the
    // warps of a stage split its tiles' chunks; 25 warps at most
    // (__launch_bounds__ of the kernel)
    if (c.stages <= 0) c.stages = 12;
    c.stages = std::max(1, std::min(c.stages, 16));
    if (c.consumers <= 0) c.consumers = 2 * c.stages;
    int cpt = std::max(1, c.consumers / c.stages);
    while (cpt > 1 && c.stages * cpt > 24) cpt--;
    c.consumers = c.stages * cpt;
    c.blocks_per_sm = 1;
    c.grid_mult = 1;
    return c;
  }
  if (c.variant == 4) {  // compact layout + cell mask: one block per SM
    c.tile_sub = 0;
    if (c.consumers <= 0) c.consumers = 12;
    c.consumers = std::min(c.consumers, 12);  // 13 warps: __launch_bounds__ of the kernel
    c.stages = c.stages > 0 ? std::max(2, std::min(c.stages, 16)) : 0;  // 0: as many as fit
    c.blocks_per_sm = 1;
    c.grid_mult = 1;
    return c;
  }
  if (c.variant == 2 || c.variant == 3) {  // compact layout: the tile shape comes with it
    c.tile_sub = 0;
    if (c.consumers <= 0) c.consumers = 16;
    c.consumers = std::min(c.consumers, 17);
    c.stages = c.stages > 0 ? std::max(2, std::min(c.stages, 16)) : 0;  // 0: as many as fit
    c.blocks_per_sm = 1;
    return c;
  }
  if (c.variant == 1) {
    if (c.tile_sub <= 0) c.tile_sub = 8;
    while (c.tile_sub > 1 && (size_t)c.tile_sub * 32 * rb * 3 > 200 * 1024) c.tile_sub /= 2;
    if (c.stages <= 0) c.stages = (int)std::min<size_t>(12, (200 * 1024) / ((size_t)c.tile_sub * 32 * rb));
    if (c.consumers <= 0) c.consumers = 16;
    c.consumers = std::min(c.consumers, 17);  // 18 warps per block at most
    int groups = std::max(1, c.consumers / c.tile_sub);
    while (groups > 1 && c.stages % groups) groups--;
    c.consumers = groups * c.tile_sub;
    c.blocks_per_sm = 1;
  } else {
    c.variant = 0;
    if (c.tile_sub <= 0 || c.tile_sub > 8) c.tile_sub = 8;  // one thread per orientation, <= 256
    while (c.tile_sub > 1 && (size_t)c.tile_sub * 32 * rb > 48 * 1024) c.tile_sub /= 2;
    const size_t tb = (size_t)c.tile_sub * 32 * rb;
    if (c.stages <= 0) c.stages = (int)std::min<size_t>(4, std::max<size_t>(2, (96 * 1024) / tb));
    if (c.blocks_per_sm <= 0) c.blocks_per_sm = 2;
    c.consumers = c.tile_sub;
  }
  if (c.stages > 16) c.stages = 16;
  if (c.stages < 2) c.stages = 2;
  return c;
}

template <int B, int MINB>
static int launch_clist_bounded(const CmpArgs &a, unsigned grid, size_t smem, cudaStream_t st) {
  const int rc = ensure_smem((const void *)compare_clist_kernel<B, MINB>, (int)smem);
  if (rc) return rc;
  compare_clist_kernel<B, MINB><<<grid, 128, smem, st>>>(a);
  return LMB_OK;
}

template <int B>
static int launch_b(const CmpArgs &a, const CompareTuning &c, unsigned grid, size_t smem,
                    int nblk, cudaStream_t st) {
  if (c.variant == 5) {
    int rc = ensure_smem((const void *)cell_filter_kernel, (int)smem);
    if (rc) return rc;
    cell_filter_kernel<<<grid, 32 * (1 + c.consumers), smem, st>>>(a);
    LMB_CUDA(cudaGetLastError());
    // the counting kernel: four 256-thread blocks per filter block's region
    cell_count_kernel<B><<<dim3(4, grid), 256, 0, st>>>(a);
  } else if (c.variant == 4) {
    const int rc = ensure_smem((const void *)compare_cell_kernel<B>, (int)smem);
    if (rc) return rc;
    compare_cell_kernel<B><<<grid, 32 * (1 + c.consumers), smem, st>>>(a);
  } else if (c.variant == 2 && nblk >= 6) {
    // six to eight 128-thread blocks per SM: registers bounded for that occupancy
    const int rc = nblk >= 8   ? launch_clist_bounded<B, 8>(a, grid, smem, st)
                   : nblk == 7 ? launch_clist_bounded<B, 7>(a, grid, smem, st)
                               : launch_clist_bounded<B, 6>(a, grid, smem, st);
    if (rc) return rc;
  } else if (c.variant == 2) {
    const int rc = ensure_smem((const void *)compare_clist_kernel<B, 1>, (int)smem);
    if (rc) return rc;
    compare_clist_kernel<B, 1><<<grid, 32 * (1 + c.consumers), smem, st>>>(a);
  } else if (c.variant == 1) {
    const int rc = ensure_smem((const void *)compare_ws_kernel<B>, (int)smem);
    if (rc) return rc;
    compare_ws_kernel<B><<<grid, 32 * (1 + c.consumers), smem, st>>>(a);
  } else {
    const int rc = ensure_smem((const void *)compare_ring_kernel<B>, (int)smem);
    if (rc) return rc;
    compare_ring_kernel<B><<<grid, a.tile, smem, st>>>(a);
  }
  LMB_CUDA(cudaGetLastError());
  return LMB_OK;
}

int compare_launch(CmpArgs a, const CompareTuning &req, int num_sms, cudaStream_t st) {
  LMB_REQUIRE((reinterpret_cast<uintptr_t>(a.db) & 15) == 0,
              "DB device pointer must be 16-byte aligned");
  CompareTuning c = compare_config(a.R, req);
  a.test_consumer_wait_ns = (uint64_t)std::max(0, c.test_consumer_wait_us) * 1000ull;
  LMB_REQUIRE(!a.test_consumer_wait_ns || c.variant == 2 || c.variant == 4,
              "the test wait applies to variants 2 and 4");
  size_t fixed = 256;  // barriers
  if (c.variant == 5) {
    // barriers and block counters, the cell mask, and per consumer warp one
    // ring stage (set below) and its window words
    LMB_REQUIRE(a.cellmask && a.cm_bytes > 0 && a.cm_bytes % 128 == 0 &&
                    a.cm_bytes <= kCellMaskBytes && (reinterpret_cast<uintptr_t>(a.cellmask) & 15) == 0,
                "cell mask missing or malformed");
    LMB_REQUIRE(a.cq_e && a.cq_pix && a.cq_ebase && a.cq_pbase && a.cq_count,
                "candidate buffer missing");
    LMB_REQUIRE(a.qS >= 1 && a.qS <= a.S, "filter windows for %d spots per record", a.qS);
    LMB_REQUIRE(!c.test_consumer_wait_us, "the test wait applies to variants 2 and 4");
    // fewer stages (keeping the warps per stage) until the ring fits
    const int cpt = c.consumers / c.stages;
    while (c.stages > 1 && 384 + (size_t)a.cm_bytes + (size_t)c.stages * a.tile_bytes +
                                   (size_t)c.stages * cpt * filter_warp_bytes(a.qS) >
                               227 * 1024)
      c.stages--;
    c.consumers = c.stages * cpt;
    fixed = 384 + a.cm_bytes + (size_t)c.consumers * filter_warp_bytes(a.qS);
  }
  if (c.variant == 4) {
    // the cell mask, and per consumer warp its hit list and window words; as
    // many consumer warps as leave room for a two-stage ring
    LMB_REQUIRE(a.cellmask && a.cm_bytes > 0 && a.cm_bytes % 128 == 0 &&
                    a.cm_bytes <= kCellMaskBytes && (reinterpret_cast<uintptr_t>(a.cellmask) & 15) == 0,
                "cell mask missing or malformed");
    LMB_REQUIRE(a.qS >= 1 && a.qS <= a.S, "cell pass hit lists of %d spots per record", a.qS);
    a.cell_queue = c.cell_queue ? 1 : 0;
    const size_t per_warp = cell_warp_bytes(a.qS, a.cell_queue);
    while (c.consumers > 1 &&
           256 + (size_t)a.cm_bytes + (size_t)c.consumers * per_warp + 2 * (size_t)a.tile_bytes >
               227 * 1024)
      c.consumers--;
    fixed += a.cm_bytes + (size_t)c.consumers * per_warp;
  }
  a.consumers = c.consumers;
  if (c.variant == 2 || c.variant == 4 || c.variant == 5) {
    // a.cl_tiles tiles of a.tile_bytes come from the compact layout; every
    // tile, the last included, is one bulk copy
    LMB_REQUIRE(a.cl && a.cl_tiles > 0 && a.tile_bytes > 0 && a.tile_bytes % 128 == 0,
                "compact layout missing or malformed");
    LMB_REQUIRE((reinterpret_cast<uintptr_t>(a.cl) & 127) == 0, "compact layout misaligned");
    a.tile_sub = 0;
    a.tile = 0;
    a.ntiles = a.cl_tiles;
    a.full_tiles = a.ntiles;
    LMB_REQUIRE(a.qS >= 1 && a.qS <= a.S, "compact pass queue entry of %d spots", a.qS);
    const size_t qbytes =
        c.variant >= 4 ? fixed - 256 : (size_t)c.consumers * clist_queue_bytes(a.qS);
    const size_t room = 227 * 1024 > 256 + qbytes ? 227 * 1024 - 256 - qbytes : 0;
    // barrier 15 is the test wait's when one is set
    const int fit = (int)std::min<size_t>(a.test_consumer_wait_ns ? 15 : 16, room / a.tile_bytes);
    if (c.variant == 5) {  // one stage per consumer warp, sized above
      LMB_REQUIRE(c.stages >= 1 && c.stages <= fit && c.stages <= 16,
                  "compact tiles of %u bytes leave no room for the filter's stages", a.tile_bytes);
    } else {
      LMB_REQUIRE(fit >= 2, "compact tiles of %u bytes leave no room for a ring", a.tile_bytes);
      c.stages = c.stages > 0 ? std::min(c.stages, fit) : fit;
    }
  } else {
    a.tile_sub = c.tile_sub;
    a.tile = (uint32_t)c.tile_sub * 32;
    a.tile_bytes = (uint32_t)((size_t)a.tile * a.R * 2);  // tile multiple of 8 -> multiple of 16
    a.full_tiles = a.n / a.tile;
    a.ntiles = (a.n + a.tile - 1) / a.tile;
  }
  a.stages = c.stages;
  if (a.ntiles == 0 || a.active == 0) return LMB_OK;
  size_t smem = 256 + (size_t)c.stages * a.tile_bytes;
  if (c.variant == 2) smem += (size_t)c.consumers * clist_queue_bytes(a.qS);
  if (c.variant >= 4) smem = fixed + (size_t)c.stages * a.tile_bytes;
  LMB_REQUIRE(smem <= 227 * 1024, "compare ring of %zu bytes exceeds shared memory", smem);
  const int mult = c.grid_mult > 0 ? c.grid_mult : 1;
  const unsigned grid = (unsigned)std::min<uint64_t>(
      a.ntiles, (uint64_t)num_sms * c.blocks_per_sm * (uint64_t)mult);
  LMB_REQUIRE(c.variant != 5 || grid == a.cq_blocks,
              "candidate regions laid out for %u filter blocks, grid of %u", a.cq_blocks, grid);
  const int B = counter_bits(a.S);
  // six to eight 128-thread compact-pass blocks per SM (the tuned shapes) get
  // a kernel whose registers are bounded for that occupancy
  const int nblk = (c.variant == 2 && c.consumers == 3) ? std::min(mult, 8) : 0;
  if (B <= 3) return launch_b<3>(a, c, grid, smem, nblk, st);
  if (B <= 5) return launch_b<5>(a, c, grid, smem, nblk, st);
  if (B <= 6) return launch_b<6>(a, c, grid, smem, nblk, st);
  if (B <= 7) return launch_b<7>(a, c, grid, smem, nblk, st);
  if (B <= 9) return launch_b<9>(a, c, grid, smem, nblk, st);
  if (B <= 11) return launch_b<11>(a, c, grid, smem, nblk, st);
  return launch_b<16>(a, c, grid, smem, nblk, st);
}

// Zero the survivor and pass counters of the pass's slots only: the counters
// of other slots keep the results of their own last pass, so a pass can be
// queued before the previous one has been collected.
__global__ void status_reset_kernel(unsigned int *__restrict__ status, unsigned long long mask) {
  const int k = threadIdx.x;
  if (k < LMB_MAX_SLOTS && ((mask >> k) & 1ull)) {
    status[k] = 0u;
    status[LMB_MAX_SLOTS + k] = 0u;
  }
}

int status_reset_launch(unsigned int *d_status, uint64_t mask, cudaStream_t st) {
  status_reset_kernel<<<1, LMB_MAX_SLOTS, 0, st>>>(d_status, (unsigned long long)mask);
  LMB_CUDA(cudaGetLastError());
  return LMB_OK;
}

// blockIdx.y = position in the slot list; 16-byte words of the 32-byte survivors.
__global__ void gather_kernel(const __grid_constant__ GatherArgs g) {
  const int i = blockIdx.y;
  const uint32_t cnt = g.off[i + 1] - g.off[i];
  const uint4 *src = reinterpret_cast<const uint4 *>(g.src + (size_t)g.slot[i] * g.cap);
  uint4 *dst = reinterpret_cast<uint4 *>(g.dst + g.off[i]);
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < 2 * cnt; w += gridDim.x * blockDim.x)
    dst[w] = src[w];
}

int gather_launch(const GatherArgs &g, cudaStream_t st) {
  if (g.n <= 0) return LMB_OK;
  LMB_REQUIRE(g.n <= LMB_MAX_SLOTS, "gather of %d lists", g.n);
  uint32_t mx = 0;
  for (int i = 0; i < g.n; i++) mx = std::max(mx, g.off[i + 1] - g.off[i]);
  const unsigned bx = std::max(1u, std::min(64u, (2 * mx + 255) / 256));
  gather_kernel<<<dim3(bx, g.n), 256, 0, st>>>(g);
  LMB_CUDA(cudaGetLastError());
  return LMB_OK;
}

int order_launch(const OrderArgs &a, int nslots, cudaStream_t st) {
  if (nslots == 0) return LMB_OK;
  const int smem = (int)(kSmemSortMax * sizeof(unsigned long long));
  const int rc = ensure_smem((const void *)order_kernel, smem);
  if (rc) return rc;
  order_kernel<<<nslots, 1024, smem, st>>>(a);
  LMB_CUDA(cudaGetLastError());
  return LMB_OK;
}

}  // namespace lmb
