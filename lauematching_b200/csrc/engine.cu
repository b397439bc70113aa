// C ABI of liblmb200: engine lifetime, device residency of the DB and the
// image slots, pass orchestration on one CUDA stream.  See include/lmb200.h.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include <omp.h>

#include "kernels.cuh"

namespace lmb {

static thread_local char g_err[2048] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
  set_error("%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  return e == cudaErrorMemoryAllocation ? LMB_ERR_OOM : LMB_ERR_CUDA;
}

}  // namespace lmb

using namespace lmb;

// Status words copied back after every pass: [0,64) survivor counts,
// [64,128) pass counts, [128] device error word (sticky).  A pass resets only
// its own slots' counters and copies all words into the next entry of a
// small pinned ring, so several passes can be in flight and each slot's
// results are read from the entry of the last pass that included it.
static constexpr int kStatusWords = 2 * LMB_MAX_SLOTS + 1;
static constexpr int kStatusRing = 4;

static constexpr int kSparseRing = 4;  // pinned staging buffers for sparse frames

// Configuration of one pass; a captured graph is reusable for an equal key.
struct PassKey {
  uint64_t mask = 0;
  int min_spots = 0;
  double min_int = 0;
  int mode = 0;
  CompareTuning tuning{};
  bool operator==(const PassKey &o) const {
    return mask == o.mask && min_spots == o.min_spots &&
           memcmp(&min_int, &o.min_int, sizeof(double)) == 0 && mode == o.mode &&
           memcmp(&tuning, &o.tuning, sizeof(CompareTuning)) == 0;
  }
};

struct PassGraph {
  PassKey key;
  cudaGraphExec_t exec;
};

struct lmb_engine {
  int device = 0;
  int num_sms = 148;
  lmb_geometry geo{};
  size_t npx = 0;
  int S = 0, R = 0;
  cudaStream_t st = nullptr;
  // resident DB
  uint16_t *d_db = nullptr;
  uint64_t n = 0;
  // compact layout derived from it for compare variant 2 (built on first use)
  unsigned char *d_cl = nullptr;
  uint64_t cl_tiles = 0;
  uint32_t cl_stage = 0;  // bytes per tile
  uint64_t cl_bytes = 0;
  int cl_state = 0;  // 0 not built, 1 built, -1 this DB cannot use it
  unsigned long long cl_hist[256] = {};  // records per on-detector spot count
  int cl_qs = 0;  // largest on-detector spot count of a record (sizes the pass's queues)
  // per tile of the compact layout: its chunks and its spots (sizes the
  // variant-5 candidate regions: at most every record and spot of a tile)
  std::vector<uint32_t> cl_tile_nch;
  std::vector<uint64_t> cl_tile_spots;
  // variant 5: candidate buffer, per filter block a region of entries and one
  // of pixels (bases [G+1] each, in one allocation), counts written per block
  CandEntry *d_cq_e = nullptr;
  uint32_t *d_cq_pix = nullptr;
  uint64_t *d_cq_base = nullptr;
  uint32_t *d_cq_count = nullptr;
  uint32_t cq_blocks = 0;
  // image slots
  uint8_t *d_u8 = nullptr;
  double *d_f64 = nullptr;  // allocated on first keep_f64 load
  unsigned long long *d_occ = nullptr;
  uint32_t *d_cellmask = nullptr;  // compare variant 4: the pass's cell mask
  uint32_t cm_bytes = 0;
  int cm_shift = 0;
  double *d_scale = nullptr;
  unsigned long long *d_max_bits = nullptr;
  void *d_stage = nullptr;  // one image in its wire dtype
  uint64_t loaded_mask = 0, f64_mask = 0;
  // survivors
  uint32_t cap = 0, cap2 = 0;
  lmb_survivor *d_surv = nullptr, *d_sorted = nullptr;
  unsigned long long *d_scratch = nullptr;
  unsigned int *d_status = nullptr;
  unsigned int *h_status = nullptr;  // pinned, kStatusRing x kStatusWords
  cudaEvent_t ev_done[kStatusRing] = {};  // a pass and its status copy finished
  uint64_t pass_seq = 0;                  // passes enqueued so far
  int slot_ring[LMB_MAX_SLOTS] = {};      // status entry of each slot's last pass
  uint64_t done_mask = 0;                 // slots that have been in a pass
  cudaStream_t dl = nullptr;              // survivor downloads
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  // image uploads run on their own stream so they overlap a running pass:
  // a pass waits for its slots' uploads, an upload waits until the last pass
  // that read its slot has finished.
  cudaStream_t ld = nullptr;
  cudaEvent_t ev_loaded[LMB_MAX_SLOTS] = {};
  cudaEvent_t ev_released[LMB_MAX_SLOTS] = {};
  // automatic variant with the compact pass's tuned shape (2 stages, 3 consumer
  // warps, 8 blocks per SM)
  CompareTuning tuning{3, 0, 2, 3, 1, 8, 0, 0, 0, 0, 0};
  int last_variant = -1;  // variant the latest pass ran
  std::vector<PassGraph> graphs;  // captured passes, most recent last
  bool use_graphs = true;
  bool sparse_uploads = true;               // frames cross the link as pairs when sparse
  double dense_share = 0.33;                // of page-locked frames in a batch, sent dense
  void *sp_host[kSparseRing] = {};          // pinned (index, value) staging ring (lazy)
  cudaEvent_t sp_ev[kSparseRing] = {};
  int sp_next = 0;
  uint64_t sparse_loads = 0;
  void *h_stage[2] = {nullptr, nullptr};   // pinned upload staging (lazy)
  cudaEvent_t ev_stage[2] = {nullptr, nullptr};
  uint64_t bytes_h2d = 0, bytes_d2h = 0;   // host<->device bytes moved so far
  // batched sparse uploads: per-task scan output (pageable), a two-deep ring
  // of pinned packed staging buffers, the device copy of the packed batch
  std::vector<uint32_t> bt_idx;
  std::vector<unsigned char> bt_val;
  void *bt_host[2] = {nullptr, nullptr};
  size_t bt_host_cap[2] = {0, 0};
  cudaEvent_t bt_ev[2] = {nullptr, nullptr};
  int bt_next = 0;
  void *d_batch = nullptr;
  size_t d_batch_cap = 0;
  // survivors of a batch of slots packed for one device-to-host copy
  lmb_survivor *d_gather = nullptr;
  uint64_t d_gather_cap = 0;
};

namespace {

void free_candidates(lmb_engine *e) {
  cudaFree(e->d_cq_e);
  cudaFree(e->d_cq_pix);
  cudaFree(e->d_cq_base);
  cudaFree(e->d_cq_count);
  e->d_cq_e = nullptr;
  e->d_cq_pix = nullptr;
  e->d_cq_base = nullptr;
  e->d_cq_count = nullptr;
  e->cq_blocks = 0;
}

// The variant-5 candidate buffer for a filter grid of G blocks (block b takes
// tiles b, b + G, ...): per block room for every record and every spot of its
// tiles, so the filter cannot run out of room whatever the frames.  Made
// before the first such pass (never inside a captured pass).
int ensure_candidates(lmb_engine *e, uint32_t G) {
  if (e->d_cq_e && e->cq_blocks == G) return LMB_OK;
  free_candidates(e);
  std::vector<uint64_t> base(2 * ((size_t)G + 1), 0);
  uint64_t *eb = base.data(), *pb = base.data() + G + 1;
  for (uint64_t t = 0; t < e->cl_tiles; t++) {
    const uint64_t b = t % G;
    eb[b + 1] += 32ull * e->cl_tile_nch[t];
    pb[b + 1] += e->cl_tile_spots[t];
  }
  for (uint32_t b = 0; b < G; b++) {
    eb[b + 1] += eb[b];
    pb[b + 1] += pb[b];
  }
  LMB_REQUIRE(pb[G] < (1ull << 40), "candidate pixel buffer too large");
  for (uint32_t b = 0; b < G; b++)
    LMB_REQUIRE(pb[b + 1] - pb[b] < (1ull << 32), "candidate region of block %u too large", b);
  cudaError_t ce = cudaMalloc(&e->d_cq_e, std::max<uint64_t>(eb[G], 1) * sizeof(CandEntry));
  if (ce == cudaSuccess)
    ce = cudaMalloc(&e->d_cq_pix, std::max<uint64_t>(pb[G], 1) * sizeof(uint32_t));
  if (ce == cudaSuccess) ce = cudaMalloc(&e->d_cq_base, base.size() * sizeof(uint64_t));
  if (ce == cudaSuccess) ce = cudaMalloc(&e->d_cq_count, 2ull * G * sizeof(uint32_t));
  if (ce == cudaSuccess)
    ce = cudaMemcpy(e->d_cq_base, base.data(), base.size() * sizeof(uint64_t),
                    cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMemset(e->d_cq_count, 0, 2ull * G * sizeof(uint32_t));
  if (ce != cudaSuccess) {
    free_candidates(e);
    return cuda_fail(ce, "variant-5 candidate buffer", __FILE__, __LINE__);
  }
  e->cq_blocks = G;
  return LMB_OK;
}

int check_engine(lmb_engine *e) {
  if (!e) {
    set_error("null engine");
    return LMB_ERR_INVALID;
  }
  LMB_CUDA(cudaSetDevice(e->device));
  return LMB_OK;
}

void free_engine(lmb_engine *e) {
  if (!e) return;
  cudaSetDevice(e->device);
  if (e->st) cudaStreamSynchronize(e->st);
  if (e->ld) cudaStreamSynchronize(e->ld);
  cudaFree(e->d_db);
  cudaFree(e->d_cl);
  cudaFree(e->d_cq_e);
  cudaFree(e->d_cq_pix);
  cudaFree(e->d_cq_base);
  cudaFree(e->d_cq_count);
  cudaFree(e->d_u8);
  cudaFree(e->d_f64);
  cudaFree(e->d_occ);
  cudaFree(e->d_cellmask);
  cudaFree(e->d_scale);
  cudaFree(e->d_max_bits);
  cudaFree(e->d_stage);
  cudaFree(e->d_surv);
  cudaFree(e->d_sorted);
  cudaFree(e->d_scratch);
  cudaFree(e->d_status);
  cudaFreeHost(e->h_status);
  for (auto &v : e->ev_done)
    if (v) cudaEventDestroy(v);
  if (e->dl) {
    cudaStreamSynchronize(e->dl);
    cudaStreamDestroy(e->dl);
  }
  for (auto &g : e->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  for (int i = 0; i < kSparseRing; i++) {
    if (e->sp_host[i]) cudaFreeHost(e->sp_host[i]);
    if (e->sp_ev[i]) cudaEventDestroy(e->sp_ev[i]);
  }
  for (int i = 0; i < 2; i++) {
    if (e->h_stage[i]) cudaFreeHost(e->h_stage[i]);
    if (e->ev_stage[i]) cudaEventDestroy(e->ev_stage[i]);
    if (e->bt_host[i]) cudaFreeHost(e->bt_host[i]);
    if (e->bt_ev[i]) cudaEventDestroy(e->bt_ev[i]);
  }
  cudaFree(e->d_batch);
  cudaFree(e->d_gather);
  for (auto &v : e->ev)
    if (v) cudaEventDestroy(v);
  for (int k = 0; k < LMB_MAX_SLOTS; k++) {
    if (e->ev_loaded[k]) cudaEventDestroy(e->ev_loaded[k]);
    if (e->ev_released[k]) cudaEventDestroy(e->ev_released[k]);
  }
  if (e->st) cudaStreamDestroy(e->st);
  if (e->ld) cudaStreamDestroy(e->ld);
  delete e;
}

size_t dtype_bytes(int dtype) {
  return dtype == LMB_F64 ? 8 : dtype == LMB_F32 ? 4 : 1;
}

// Host->device copy of a large pageable buffer (a memory-mapped cache or
// orientation file) through the engine's two pinned 64 MiB staging chunks:
// the host copy into chunk b (split over OpenMP threads) overlaps the DMA of
// chunk b^1.
int upload_chunked(lmb_engine *e, void *dst, const void *src, size_t bytes, cudaStream_t st) {
  const size_t kChunk = 64ull << 20;
  e->bytes_h2d += bytes;
  if (bytes <= (4ull << 20)) {
    LMB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    LMB_CUDA(cudaStreamSynchronize(st));
    return LMB_OK;
  }
  for (int i = 0; i < 2; i++) {
    if (!e->h_stage[i]) LMB_CUDA(cudaHostAlloc(&e->h_stage[i], kChunk, cudaHostAllocDefault));
    if (!e->ev_stage[i]) LMB_CUDA(cudaEventCreateWithFlags(&e->ev_stage[i], cudaEventDisableTiming));
  }
  size_t off = 0;
  int b = 0;
  while (off < bytes) {
    const size_t len = std::min(kChunk, bytes - off);
    LMB_CUDA(cudaEventSynchronize(e->ev_stage[b]));  // chunk b free again
    char *dstp = static_cast<char *>(e->h_stage[b]);
    const char *srcp = static_cast<const char *>(src) + off;
    const size_t piece = 4ull << 20;
    const long np = (long)((len + piece - 1) / piece);
#pragma omp parallel for schedule(static) num_threads(8)
    for (long i = 0; i < np; i++) {
      const size_t o = (size_t)i * piece;
      memcpy(dstp + o, srcp + o, std::min(piece, len - o));
    }
    LMB_CUDA(cudaMemcpyAsync(static_cast<char *>(dst) + off, dstp, len, cudaMemcpyHostToDevice, st));
    LMB_CUDA(cudaEventRecord(e->ev_stage[b], st));
    off += len;
    b ^= 1;
  }
  LMB_CUDA(cudaStreamSynchronize(st));
  return LMB_OK;
}

int alloc_db(lmb_engine *e, uint64_t n) {
  LMB_REQUIRE(n < (1ull << 40), "at most 2^40 orientations are supported (got %llu)",
              (unsigned long long)n);
  for (auto &g : e->graphs)  // captured passes name the old DB
    if (g.exec) cudaGraphExecDestroy(g.exec);
  e->graphs.clear();
  cudaFree(e->d_db);
  e->d_db = nullptr;
  e->n = 0;
  cudaFree(e->d_cl);
  e->d_cl = nullptr;
  e->cl_tiles = 0;
  e->cl_state = 0;
  e->cl_bytes = 0;
  e->cl_qs = 0;
  free_candidates(e);
  const size_t bytes = (size_t)n * e->R * 2;
  const size_t alloc = ((bytes + 255) / 256) * 256 + 256;
  LMB_CUDA(cudaMalloc(&e->d_db, alloc));
  LMB_CUDA(cudaMemsetAsync(e->d_db, 0, alloc, e->st));
  e->n = n;
  return LMB_OK;
}

int upload_hkls(const int32_t *hkls, int nh, int4 **d_out) {
  std::vector<int4> h((size_t)std::max(nh, 1));
  for (int i = 0; i < nh; i++) h[i] = make_int4(hkls[3 * i], hkls[3 * i + 1], hkls[3 * i + 2], 0);
  LMB_CUDA(cudaMalloc(d_out, h.size() * sizeof(int4)));
  LMB_CUDA(cudaMemcpy(*d_out, h.data(), (size_t)nh * sizeof(int4), cudaMemcpyHostToDevice));
  return LMB_OK;
}


// Host scan of a frame: if its positive pixels, as (uint32 index, value)
// pairs, take less than half the dense bytes, upload the pairs (through a
// ring of pinned staging buffers) and scatter them on the load stream;
// otherwise leave *sparse false for the dense path.  The maximum is taken over
// the same positive values the device would see (NaN and non-positive
// pixels quantise to 0 and are not listed).
// Positive (and not NaN) pixel test on the bits: uint8 != 0; IEEE floats
// with the sign bit clear, not zero, and at most +infinity.
inline bool positive(uint8_t v) { return v != 0; }
inline bool positive(float v) {
  uint32_t b;
  memcpy(&b, &v, 4);
  return b - 1u < 0x7F800000u;
}
inline bool positive(double v) {
  uint64_t b;
  memcpy(&b, &v, 8);
  return b - 1ull < 0x7FF0000000000000ull;
}

// Visit the positive pixels of px[lo, hi) in order, skipping all-zero 64-byte
// blocks (a thresholded frame is mostly zero bytes).
template <typename T, typename F>
inline void for_positive(const T *px, size_t lo, size_t hi, F &&f) {
  constexpr size_t kPer = 64 / sizeof(T);
  size_t i = lo;
  while (i < hi && (i % kPer)) {
    if (positive(px[i])) f(i, px[i]);
    i++;
  }
  for (; i + kPer <= hi; i += kPer) {
    uint64_t w[8];
    memcpy(w, px + i, 64);
    if ((w[0] | w[1] | w[2] | w[3] | w[4] | w[5] | w[6] | w[7]) == 0) continue;
    for (size_t j = 0; j < kPer; j++)
      if (positive(px[i + j])) f(i + j, px[i + j]);
  }
  for (; i < hi; i++)
    if (positive(px[i])) f(i, px[i]);
}

template <typename T>
int try_sparse(lmb_engine *e, const T *px, int slot, int dtype, bool *sparse) {
  *sparse = false;
  const size_t npx = e->npx;
  const size_t vb = sizeof(T);
  const size_t limit = npx * vb / (2 * (4 + vb));
  const int nt = (int)std::max<size_t>(
      1, std::min<size_t>(std::min(16, omp_get_num_procs()), npx / (1 << 16) + 1));
  std::vector<size_t> cnt((size_t)nt + 1, 0);
  std::vector<double> mxs((size_t)nt, 0.0);
#pragma omp parallel num_threads(nt)
  {
    const int t = omp_get_thread_num();
    const size_t lo = npx * t / nt, hi = npx * (t + 1) / nt;
    size_t c = 0;
    double m = 0.0;
    for_positive(px, lo, hi, [&](size_t, T v) {
      c++;
      if ((double)v > m) m = (double)v;
    });
    cnt[t + 1] = c;
    mxs[t] = m;
  }
  for (int t = 0; t < nt; t++) cnt[t + 1] += cnt[t];
  const size_t nnz = cnt[nt];
  if (nnz > limit) return LMB_OK;
  double mx = 0.0;
  for (int t = 0; t < nt; t++)
    if (mxs[t] > mx) mx = mxs[t];
  const int r = e->sp_next;
  e->sp_next = (r + 1) % kSparseRing;
  const size_t cap = npx * 4 + 64;
  if (!e->sp_host[r]) LMB_CUDA(cudaHostAlloc(&e->sp_host[r], cap, cudaHostAllocDefault));
  if (!e->sp_ev[r]) LMB_CUDA(cudaEventCreateWithFlags(&e->sp_ev[r], cudaEventDisableTiming));
  LMB_CUDA(cudaEventSynchronize(e->sp_ev[r]));  // ring entry free again
  uint32_t *hidx = static_cast<uint32_t *>(e->sp_host[r]);
  const size_t voff = ((nnz * 4 + 15) / 16) * 16;
  T *hval = reinterpret_cast<T *>(static_cast<char *>(e->sp_host[r]) + voff);
#pragma omp parallel num_threads(nt)
  {
    const int t = omp_get_thread_num();
    const size_t lo = npx * t / nt, hi = npx * (t + 1) / nt;
    size_t o = cnt[t];
    for_positive(px, lo, hi, [&](size_t i, T v) {
      hidx[o] = (uint32_t)i;
      hval[o] = v;
      o++;
    });
  }
  const size_t bytes = voff + nnz * vb;
  LMB_CUDA(cudaMemcpyAsync(e->d_stage, e->sp_host[r], bytes, cudaMemcpyHostToDevice, e->ld));
  LMB_CUDA(cudaEventRecord(e->sp_ev[r], e->ld));
  e->bytes_h2d += bytes;
  const int rc = sparse_load_launch(
      static_cast<const uint32_t *>(e->d_stage), static_cast<const char *>(e->d_stage) + voff,
      dtype, nnz, mx, e->d_u8 + (size_t)slot * npx, e->d_occ, slot, e->d_scale + slot, npx,
      e->num_sms, e->ld);
  if (rc) return rc;
  e->sparse_loads++;
  *sparse = true;
  return LMB_OK;
}

// Automatic variant.  Each spot the pass gathers costs the same in both
// layouts; what the compact layout saves is the stream of the records'
// padding.  Measured on B200 at 1e8 records (two detector geometries, K=64),
// the compact pass is as fast or faster while the records that can pass
// (at least min_spots on-detector spots) hold up to ~3 spots per DB record
// on average, and up to 1.4x slower beyond (dense records, where the
// reference records' stream is no longer the cost).
constexpr double kAutoGather = 3.0;
// the cell-mask pass the automatic variant runs beyond that
constexpr int kAutoCellVariant = 5;

double gathered_per_record(const lmb_engine *e, int min_spots) {
  const int m = std::max(0, min_spots);
  double g = 0;
  for (int c = m; c < 256; c++) g += (double)c * (double)e->cl_hist[c];
  return e->n ? g / (double)e->n : 0.0;
}

// Tile size of the compact layout of a dense DB (one whose passes run the
// cell-mask filter): a dozen ring stages of it fit beside the 128 KiB cell
// mask, and a tile holds an even number of chunks at ~15 spots per record,
// so the two warps of a stage split it evenly (measured on B200 at 1e8
// records, K = 64: 3.72 ms per pass against 4.1-5.4 ms with 4-10 KiB tiles
// at the same warp count, 3.70 ms with 12 KiB tiles and three warps per stage).
constexpr uint64_t kCellTileBytes = 8192;

// One pass: status reset, compare, ordering, status copy-back, on e->st.
// Derive the compact layout of the resident DB (see clist.cu): spots per
// 32-record chunk on the device; on the host, the tile size (about 64 chunks
// of the DB's average size, 4-24 KiB, at least the largest chunk) and a
// greedy packing of consecutive chunks into tiles; then the tiles on the
// device.  min_spots: MinNrSpots of the pass that asks for the layout; a DB
// dense at that threshold gets the cell-mask filter's tile size.
int build_compact(lmb_engine *e, int min_spots) {
  e->cl_state = -1;
  if (e->S > 255 || e->n == 0) return LMB_OK;  // counts are uint8
  const uint64_t n = e->n, nch = (n + 31) / 32;
  uint32_t *d_aux = nullptr;  // chunk spots, then 4 arrays of the packing; count histogram
  LMB_CUDA(cudaMalloc(&d_aux, nch * 4 * 4 + 256 * sizeof(unsigned long long)));
  unsigned long long *d_hist = reinterpret_cast<unsigned long long *>(d_aux + 4 * nch);
  std::vector<uint32_t> cs(nch);
  int rc = clist_chunk_launch(e->d_db, n, e->R, e->S, e->geo.nr_px_x, e->geo.nr_px_y, d_aux,
                              d_hist, e->st);
  cudaError_t ce = cudaSuccess;
  if (rc == LMB_OK) ce = cudaMemcpyAsync(cs.data(), d_aux, nch * 4, cudaMemcpyDeviceToHost, e->st);
  if (ce == cudaSuccess)
    ce = cudaMemcpyAsync(e->cl_hist, d_hist, sizeof(e->cl_hist), cudaMemcpyDeviceToHost, e->st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->st);
  if (rc || ce != cudaSuccess) {
    cudaFree(d_aux);
    return rc ? rc : cuda_fail(ce, "compact layout: chunk counts", __FILE__, __LINE__);
  }
  e->cl_qs = 1;
  for (int c = 255; c >= 1; c--)
    if (e->cl_hist[c]) {
      e->cl_qs = c;
      break;
    }
  uint64_t total_spots = 0, max_spots = 0;
  for (uint64_t c = 0; c < nch; c++) {
    total_spots += cs[c];
    max_spots = std::max<uint64_t>(max_spots, cs[c]);
  }
  auto round128 = [](uint64_t b) { return ((b + 127) / 128) * 128; };
  const uint64_t avg_chunk = 36 + (4 * total_spots + nch - 1) / nch;
  uint64_t TB = std::min<uint64_t>(24 * 1024, std::max<uint64_t>(4096, round128(64 * avg_chunk)));
  if (gathered_per_record(e, min_spots) > kAutoGather) {
    // the automatic variant will run the cell-mask filter over it: its tile
    // size, whatever the tuning of this pass
    TB = kCellTileBytes;
  } else {
    // room for the pass shape's blocks (three consumer warps, a two-stage
    // ring; six per SM, or up to eight when the tuning asks for more) on an
    // SM, when the largest chunk allows it
    int per_sm = 0, reserved = 0;
    cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, e->device);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, e->device);
    const int nb = std::max(6, std::min(8, e->tuning.grid_mult));
    const int64_t room =
        (int64_t)per_sm / nb - reserved - 256 - 3 * (int64_t)clist_queue_bytes(e->cl_qs);
    if (room > 2 * 4096) TB = std::min<uint64_t>(TB, (uint64_t)(room / 2) / 128 * 128);
  }
  TB = std::max<uint64_t>(TB, round128(clist_spot_offset(1) + 4 * max_spots));
  if (2 * TB + 256 > 227 * 1024) {  // a huge S with dense records: keep the reference layout
    cudaFree(d_aux);
    return LMB_OK;
  }
  // greedy packing: chunk c into the current tile while it still fits
  std::vector<uint32_t> ctile(nch), cpos(nch), cbase(nch), tnch;
  uint32_t nt_chunks = 0;
  uint64_t t_spots = 0;
  for (uint64_t c = 0; c < nch; c++) {
    if (nt_chunks && clist_spot_offset(nt_chunks + 1) + 4 * (t_spots + cs[c]) > TB) {
      tnch.push_back(nt_chunks);
      nt_chunks = 0;
      t_spots = 0;
    }
    ctile[c] = (uint32_t)tnch.size();
    cpos[c] = nt_chunks;
    cbase[c] = (uint32_t)t_spots;
    nt_chunks++;
    t_spots += cs[c];
  }
  tnch.push_back(nt_chunks);
  const uint64_t nt = tnch.size();
  const uint64_t total = nt * TB;
  uint32_t *d_tnch = nullptr;
  ce = cudaMemcpy(d_aux + nch, ctile.data(), nch * 4, cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMemcpy(d_aux + 2 * nch, cpos.data(), nch * 4, cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMemcpy(d_aux + 3 * nch, cbase.data(), nch * 4, cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMalloc(&d_tnch, nt * 4);
  if (ce == cudaSuccess) ce = cudaMemcpy(d_tnch, tnch.data(), nt * 4, cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMalloc(&e->d_cl, total);
  if (ce == cudaSuccess) ce = cudaMemsetAsync(e->d_cl, 0, total, e->st);
  if (ce == cudaSuccess)
    rc = clist_fill_launch(e->d_db, n, e->R, e->S, e->geo.nr_px_x, e->geo.nr_px_y, (uint32_t)TB,
                           d_aux + nch, d_aux + 2 * nch, d_aux + 3 * nch, d_tnch, e->d_cl, e->st);
  if (ce == cudaSuccess && rc == LMB_OK) ce = cudaStreamSynchronize(e->st);
  cudaFree(d_aux);
  cudaFree(d_tnch);
  if (ce != cudaSuccess || rc) {
    cudaFree(e->d_cl);
    e->d_cl = nullptr;
    return rc ? rc : cuda_fail(ce, "compact layout", __FILE__, __LINE__);
  }
  e->cl_tiles = nt;
  e->cl_stage = (uint32_t)TB;
  e->cl_bytes = total;
  e->cl_state = 1;
  e->cl_tile_nch = tnch;
  e->cl_tile_spots.assign(nt, 0);
  for (uint64_t c = 0; c < nch; c++) e->cl_tile_spots[ctile[c]] += cs[c];
  return LMB_OK;
}


// The cell-mask pass needs its mask, a hit list per consumer warp and a
// two-stage ring of the layout's tiles in one block's shared memory.
bool cell_pass_fits(const lmb_engine *e) {
  const size_t need = 256 + (size_t)e->cm_bytes +
                      cell_warp_bytes(e->cl_qs > 0 ? e->cl_qs : e->S, e->tuning.cell_queue) +
                      2 * (size_t)e->cl_stage;
  return e->d_cellmask && need <= 227 * 1024;
}

int enqueue_pass(lmb_engine *e, const PassKey &k, bool capturing) {
  // timing events recorded inside a captured graph must be external to be
  // observable (and timed) after each replay
  const unsigned evf = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
  {
    const int rc = status_reset_launch(e->d_status, k.mask, e->st);
    if (rc) return rc;
  }
  LMB_CUDA(cudaEventRecordWithFlags(e->ev[0], e->st, evf));
  CmpArgs a{};
  a.db = e->d_db;
  a.n = e->n;
  a.R = e->R;
  a.S = e->S;
  a.qS = e->cl_qs > 0 ? e->cl_qs : e->S;
  a.W = e->geo.nr_px_x;
  a.H = e->geo.nr_px_y;
  a.occ = e->d_occ;
  a.active = k.mask;
  a.u8 = e->d_u8;
  a.f64 = k.mode == LMB_VALUE_F64 ? e->d_f64 : nullptr;
  a.npx = e->npx;
  a.scale = e->d_scale;
  a.mode = k.mode;
  // count >= MinNrSpots can only hold for MinNrSpots <= S; <= 0 always holds
  a.min_spots = k.min_spots < 0 ? 0 : k.min_spots;
  a.min_int = k.min_int;
  a.surv = e->d_surv;
  a.cap = e->cap;
  a.surv_cnt = e->d_status;
  a.pass_cnt = e->d_status + LMB_MAX_SLOTS;
  a.err = reinterpret_cast<int *>(e->d_status + 2 * LMB_MAX_SLOTS);
  a.full_gather = k.tuning.full_gather;
  if (k.tuning.variant == 2 || k.tuning.variant >= 4) {
    a.cl = e->d_cl;
    a.cl_tiles = e->cl_tiles;
    a.tile_bytes = e->cl_stage;
  }
  if (k.tuning.variant >= 4) {
    a.cellmask = e->d_cellmask;
    a.cm_bytes = e->cm_bytes;
    a.cm_shift = e->cm_shift;
  }
  if (k.tuning.variant == 5) {
    a.cq_e = e->d_cq_e;
    a.cq_pix = e->d_cq_pix;
    a.cq_ebase = e->d_cq_base;
    a.cq_pbase = e->d_cq_base + e->cq_blocks + 1;
    a.cq_count = e->d_cq_count;
    a.cq_blocks = e->cq_blocks;
  }
  if (k.min_spots <= e->S && !std::isnan(k.min_int)) {
    if (k.tuning.variant >= 4) {  // the cell mask of this pass's slots, then the pass
      const int rc = cellmask_launch(e->d_occ, e->npx, k.mask, e->cm_shift, e->cm_bytes,
                                     e->d_cellmask, e->num_sms, e->st);
      if (rc) return rc;
    }
    const int rc = compare_launch(a, k.tuning, e->num_sms, e->st);
    if (rc) return rc;
  }
  LMB_CUDA(cudaEventRecordWithFlags(e->ev[1], e->st, evf));
  OrderArgs o{};
  o.surv = e->d_surv;
  o.out = e->d_sorted;
  o.surv_cnt = e->d_status;
  o.cap = e->cap;
  o.scratch = e->d_scratch;
  o.cap2 = e->cap2;
  int ns = 0;
  for (int i = 0; i < LMB_MAX_SLOTS; i++)
    if (k.mask >> i & 1) o.slots[ns++] = i;
  const int rc = order_launch(o, ns, e->st);
  if (rc) return rc;
  LMB_CUDA(cudaEventRecordWithFlags(e->ev[2], e->st, evf));
  return LMB_OK;
}

}  // namespace

extern "C" {

const char *lmb_version(void) { return "lmb200 0.1.0 sm_100a"; }

int lmb_device_info(int32_t device, uint64_t *free_bytes, uint64_t *total_bytes,
                    int32_t *l2_bytes, int32_t *sm_count) {
  LMB_CUDA(cudaSetDevice(device));
  size_t fr = 0, tot = 0;
  LMB_CUDA(cudaMemGetInfo(&fr, &tot));
  int l2 = 0, sms = 0;
  LMB_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device));
  LMB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  if (free_bytes) *free_bytes = fr;
  if (total_bytes) *total_bytes = tot;
  if (l2_bytes) *l2_bytes = l2;
  if (sm_count) *sm_count = sms;
  return LMB_OK;
}
const char *lmb_last_error(void) { return g_err; }

int lmb_geometry_init(const double lattice[6], int32_t space_group, const double p_array[3],
                      const double r_array[3], double px_x, double px_y, int32_t nr_px_x,
                      int32_t nr_px_y, double elo, double ehi, int32_t max_nr_spots,
                      lmb_geometry *out);  // geometry.cpp

int lmb_engine_create(int32_t device, const lmb_geometry *geo, uint64_t survivor_capacity,
                      lmb_engine **out) {
  LMB_REQUIRE(geo && out, "null argument");
  LMB_REQUIRE(geo->nr_px_x > 0 && geo->nr_px_y > 0 && geo->nr_px_x <= 65535 &&
                  geo->nr_px_y <= 65535,
              "detector size %d x %d outside 1..65535", geo->nr_px_x, geo->nr_px_y);
  LMB_REQUIRE(geo->max_nr_spots >= 1 && geo->max_nr_spots <= 32767,
              "MaxNrLaueSpots=%d outside 1..32767", geo->max_nr_spots);
  if (survivor_capacity == 0) survivor_capacity = 262144;
  LMB_REQUIRE(survivor_capacity <= (1u << 24), "survivor capacity above 2^24");
  *out = nullptr;
  lmb_engine *e = new lmb_engine();
  e->device = device;
  e->geo = *geo;
  e->npx = (size_t)geo->nr_px_x * geo->nr_px_y;
  e->S = geo->max_nr_spots;
  e->R = 1 + 2 * e->S;
  e->cap = (uint32_t)survivor_capacity;
  e->cap2 = 1;
  while (e->cap2 < e->cap) e->cap2 <<= 1;
  auto fail = [&](int rc) {
    free_engine(e);
    return rc;
  };
  cudaError_t ce = cudaSetDevice(device);
  if (ce != cudaSuccess) return fail(cuda_fail(ce, "cudaSetDevice", __FILE__, __LINE__));
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  e->num_sms = sms > 0 ? sms : 148;
#define TRY(call)                                                              \
  do {                                                                         \
    cudaError_t _e = (call);                                                   \
    if (_e != cudaSuccess) return fail(cuda_fail(_e, #call, __FILE__, __LINE__)); \
  } while (0)
  TRY(cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking));
  TRY(cudaStreamCreateWithFlags(&e->ld, cudaStreamNonBlocking));
  TRY(cudaStreamCreateWithFlags(&e->dl, cudaStreamNonBlocking));
  for (auto &v : e->ev_done) TRY(cudaEventCreateWithFlags(&v, cudaEventDisableTiming));
  for (auto &v : e->ev) TRY(cudaEventCreate(&v));
  for (int k = 0; k < LMB_MAX_SLOTS; k++) {
    TRY(cudaEventCreateWithFlags(&e->ev_loaded[k], cudaEventDisableTiming));
    TRY(cudaEventCreateWithFlags(&e->ev_released[k], cudaEventDisableTiming));
  }
  TRY(cudaMalloc(&e->d_u8, e->npx * LMB_MAX_SLOTS));
  TRY(cudaMemset(e->d_u8, 0, e->npx * LMB_MAX_SLOTS));
  TRY(cudaMalloc(&e->d_occ, e->npx * sizeof(unsigned long long)));
  TRY(cudaMemset(e->d_occ, 0, e->npx * sizeof(unsigned long long)));
  e->cm_shift = cellmask_shift(e->npx);
  e->cm_bytes = cellmask_bytes(e->npx);
  TRY(cudaMalloc(&e->d_cellmask, e->cm_bytes));
  TRY(cudaMemset(e->d_cellmask, 0, e->cm_bytes));
  TRY(cudaMalloc(&e->d_scale, LMB_MAX_SLOTS * sizeof(double)));
  TRY(cudaMemset(e->d_scale, 0, LMB_MAX_SLOTS * sizeof(double)));
  TRY(cudaMalloc(&e->d_max_bits, sizeof(unsigned long long)));
  TRY(cudaMalloc(&e->d_stage, e->npx * sizeof(double)));
  TRY(cudaMalloc(&e->d_surv, (size_t)LMB_MAX_SLOTS * e->cap * sizeof(lmb_survivor)));
  TRY(cudaMalloc(&e->d_sorted, (size_t)LMB_MAX_SLOTS * e->cap * sizeof(lmb_survivor)));
  TRY(cudaMalloc(&e->d_scratch, (size_t)LMB_MAX_SLOTS * e->cap2 * sizeof(unsigned long long)));
  TRY(cudaMalloc(&e->d_status, kStatusWords * sizeof(unsigned int)));
  TRY(cudaMemset(e->d_status, 0, kStatusWords * sizeof(unsigned int)));
  TRY(cudaHostAlloc(&e->h_status, kStatusRing * kStatusWords * sizeof(unsigned int),
                    cudaHostAllocDefault));
  memset(e->h_status, 0, kStatusRing * kStatusWords * sizeof(unsigned int));
#undef TRY
  *out = e;
  return LMB_OK;
}

int lmb_engine_destroy(lmb_engine *e) {
  if (!e) return LMB_OK;
  free_engine(e);
  return LMB_OK;
}

void *lmb_engine_stream(lmb_engine *e) { return e ? (void *)e->st : nullptr; }

int lmb_db_upload(lmb_engine *e, const uint16_t *records, uint64_t n) {
  int rc = check_engine(e);
  if (rc) return rc;
  LMB_REQUIRE(records || n == 0, "null records");
  LMB_CUDA(cudaStreamSynchronize(e->st));
  rc = alloc_db(e, n);
  if (rc) return rc;
  LMB_CUDA(cudaStreamSynchronize(e->st));
  return upload_chunked(e, e->d_db, records, (size_t)n * e->R * 2, e->st);
}

static int db_build_common(lmb_engine *e, const double *orients, uint64_t seed, bool synthetic,
                           uint64_t n, const int32_t *hkls, int32_t nh, double *orients_out,
                           uint32_t flags) {
  int rc = check_engine(e);
  if (rc) return rc;
  LMB_REQUIRE(nh >= 0 && (hkls || nh == 0), "bad HKL list");
  LMB_REQUIRE(synthetic || orients || n == 0, "null orientations");
  LMB_CUDA(cudaStreamSynchronize(e->st));
  rc = alloc_db(e, n);
  if (rc) return rc;
  int4 *d_hkl = nullptr;
  rc = upload_hkls(hkls, nh, &d_hkl);
  if (rc) return rc;
  const uint64_t kChunk = 4ull << 20;  // orientations per chunk (288 MB of matrices)
  double *d_om = nullptr;
  cudaError_t ce = cudaMalloc(&d_om, std::min(kChunk, std::max<uint64_t>(n, 1)) * 72);
  if (ce != cudaSuccess) {
    cudaFree(d_hkl);
    return cuda_fail(ce, "cudaMalloc(orientation chunk)", __FILE__, __LINE__);
  }
  for (uint64_t off = 0; off < n && rc == LMB_OK; off += kChunk) {
    const uint64_t len = std::min(kChunk, n - off);
    if (synthetic) {
      rc = synth_orient_launch(seed, off, len, d_om, e->st, flags);
    } else {
      rc = upload_chunked(e, d_om, orients + off * 9, len * 72, e->st);
    }
    if (rc == LMB_OK)
      rc = dbbuild_launch(d_om, len, d_hkl, nh, e->geo, e->d_db + off * e->R, e->st,
                          (flags & LMB_BUILD_EXACT_FP64) != 0);
    if (rc == LMB_OK && synthetic && orients_out) {
      ce = cudaMemcpyAsync(orients_out + off * 9, d_om, len * 72, cudaMemcpyDeviceToHost, e->st);
      e->bytes_d2h += len * 72;
      if (ce != cudaSuccess) rc = cuda_fail(ce, "orientation download", __FILE__, __LINE__);
    }
    ce = cudaStreamSynchronize(e->st);
    if (ce != cudaSuccess && rc == LMB_OK) rc = cuda_fail(ce, "DB build", __FILE__, __LINE__);
  }
  cudaFree(d_om);
  cudaFree(d_hkl);
  return rc;
}

int lmb_db_build(lmb_engine *e, const double *orients, uint64_t n, const int32_t *hkls,
                 int32_t nh) {
  return db_build_common(e, orients, 0, false, n, hkls, nh, nullptr, 0);
}

int lmb_db_build_ex(lmb_engine *e, const double *orients, uint64_t n, const int32_t *hkls,
                    int32_t nh, uint32_t flags) {
  return db_build_common(e, orients, 0, false, n, hkls, nh, nullptr, flags);
}

int lmb_db_build_synthetic(lmb_engine *e, uint64_t seed, uint64_t n, const int32_t *hkls,
                           int32_t nh, double *orients_out) {
  return db_build_common(e, nullptr, seed, true, n, hkls, nh, orients_out, 0);
}

int lmb_db_build_synthetic_ex(lmb_engine *e, uint64_t seed, uint64_t n, const int32_t *hkls,
                              int32_t nh, double *orients_out, uint32_t flags) {
  LMB_REQUIRE((flags & ~(uint32_t)(LMB_BUILD_EXACT_FP64 | LMB_BUILD_SYNTH_HEX_FZ)) == 0,
              "unknown build flags 0x%x", flags);
  return db_build_common(e, nullptr, seed, true, n, hkls, nh, orients_out, flags);
}

int lmb_synth_orientations(lmb_engine *e, uint64_t seed, uint64_t first, uint64_t n,
                           double *out) {
  return lmb_synth_orientations_ex(e, seed, first, n, out, 0);
}

int lmb_synth_orientations_ex(lmb_engine *e, uint64_t seed, uint64_t first, uint64_t n,
                              double *out, uint32_t flags) {
  int rc = check_engine(e);
  if (rc) return rc;
  LMB_REQUIRE(out || n == 0, "null output");
  LMB_REQUIRE((flags & ~(uint32_t)LMB_BUILD_SYNTH_HEX_FZ) == 0, "unknown flags 0x%x", flags);
  if (n == 0) return LMB_OK;
  double *d = nullptr;
  LMB_CUDA(cudaMalloc(&d, n * 72));
  rc = synth_orient_launch(seed, first, n, d, e->st, flags);
  cudaError_t ce = cudaSuccess;
  if (rc == LMB_OK) ce = cudaMemcpyAsync(out, d, n * 72, cudaMemcpyDeviceToHost, e->st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->st);
  e->bytes_d2h += n * 72;
  cudaFree(d);
  if (ce != cudaSuccess) return cuda_fail(ce, "synthetic orientations", __FILE__, __LINE__);
  return rc;
}

int lmb_db_download(lmb_engine *e, uint64_t first, uint64_t count, uint16_t *out) {
  int rc = check_engine(e);
  if (rc) return rc;
  LMB_REQUIRE(first <= e->n && count <= e->n - first, "record range outside the DB");
  LMB_REQUIRE(out || count == 0, "null output");
  LMB_CUDA(cudaStreamSynchronize(e->st));
  LMB_CUDA(cudaMemcpy(out, e->d_db + first * e->R, (size_t)count * e->R * 2,
                      cudaMemcpyDeviceToHost));
  e->bytes_d2h += (size_t)count * e->R * 2;
  return LMB_OK;
}

int lmb_db_info(lmb_engine *e, uint64_t *n_orient, int32_t *max_nr_spots) {
  LMB_REQUIRE(e, "null engine");
  if (n_orient) *n_orient = e->n;
  if (max_nr_spots) *max_nr_spots = e->S;
  return LMB_OK;
}

int lmb_image_load(lmb_engine *e, int32_t slot, const void *pixels, int32_t dtype,
                   int32_t keep_f64, double *im_scale) {
  int rc = check_engine(e);
  if (rc) return rc;
  LMB_REQUIRE(slot >= 0 && slot < LMB_MAX_SLOTS, "slot %d outside 0..%d", slot,
              LMB_MAX_SLOTS - 1);
  LMB_REQUIRE(pixels, "null pixels");
  LMB_REQUIRE(dtype == LMB_F64 || dtype == LMB_F32 || dtype == 2, "unknown dtype %d", dtype);
  if (keep_f64 && !e->d_f64)
    LMB_CUDA(cudaMalloc(&e->d_f64, e->npx * sizeof(double) * LMB_MAX_SLOTS));
  LMB_CUDA(cudaStreamWaitEvent(e->ld, e->ev_released[slot], 0));
  // A sparse frame (the usual thresholded Laue image) crosses the host link
  // as (index, value) pairs of its positive pixels; a dense one as is.
  bool sparse = false;
  if (!keep_f64 && e->sparse_uploads) {
    rc = dtype == LMB_F64   ? try_sparse(e, static_cast<const double *>(pixels), slot, dtype, &sparse)
         : dtype == LMB_F32 ? try_sparse(e, static_cast<const float *>(pixels), slot, dtype, &sparse)
                            : try_sparse(e, static_cast<const uint8_t *>(pixels), slot, dtype, &sparse);
    if (rc) return rc;
  }
  if (!sparse) {
    LMB_CUDA(cudaMemcpyAsync(e->d_stage, pixels, e->npx * dtype_bytes(dtype),
                             cudaMemcpyHostToDevice, e->ld));
    e->bytes_h2d += e->npx * dtype_bytes(dtype);
    rc = quantize_launch(e->d_stage, dtype, e->npx, e->d_max_bits,
                         e->d_u8 + (size_t)slot * e->npx,
                         keep_f64 ? e->d_f64 + (size_t)slot * e->npx : nullptr, e->d_occ, slot,
                         e->d_scale + slot, e->num_sms, e->ld);
    if (rc) return rc;
  }
  LMB_CUDA(cudaEventRecord(e->ev_loaded[slot], e->ld));
  e->loaded_mask |= 1ull << slot;
  if (keep_f64)
    e->f64_mask |= 1ull << slot;
  else
    e->f64_mask &= ~(1ull << slot);
  if (im_scale) {
    LMB_CUDA(cudaMemcpyAsync(im_scale, e->d_scale + slot, sizeof(double), cudaMemcpyDeviceToHost,
                             e->ld));
    e->bytes_d2h += sizeof(double);
    LMB_CUDA(cudaStreamSynchronize(e->ld));
  }
  return LMB_OK;
}

// Batched sparse upload of n frames of type T (slots already validated).
// One host pass over each frame's memory: tasks of (frame, segment) scan in
// parallel, each writing its positive pixels' (index, value) pairs into its
// own scratch area (capacity capf pairs, the per-frame sparse limit of a
// batch).  Frames whose pairs fit are packed back to back behind a
// descriptor table in a pinned buffer and cross the link in ONE copy; two
// kernels clear their slots and scatter them.  Frames that do not fit go the
// dense way, one frame at a time.
}  // extern "C"

namespace {

// One frame the dense way (copy of the whole frame, max + quantise kernels)
// on the load stream, without a host scan.
int dense_load(lmb_engine *e, int slot, const void *pixels, int dtype) {
  LMB_CUDA(cudaStreamWaitEvent(e->ld, e->ev_released[slot], 0));
  const size_t bytes = e->npx * dtype_bytes(dtype);
  LMB_CUDA(cudaMemcpyAsync(e->d_stage, pixels, bytes, cudaMemcpyHostToDevice, e->ld));
  e->bytes_h2d += bytes;
  const int rc = quantize_launch(e->d_stage, dtype, e->npx, e->d_max_bits,
                                 e->d_u8 + (size_t)slot * e->npx, nullptr, e->d_occ, slot,
                                 e->d_scale + slot, e->num_sms, e->ld);
  if (rc) return rc;
  LMB_CUDA(cudaEventRecord(e->ev_loaded[slot], e->ld));
  e->loaded_mask |= 1ull << slot;
  e->f64_mask &= ~(1ull << slot);
  return LMB_OK;
}

template <typename T>
int load_batch_sparse(lmb_engine *e, const int32_t *slots, const void *const *frames,
                             int n, int dtype) {
  const size_t npx = e->npx, vb = sizeof(T);
  const size_t limit = npx * vb / (2 * (4 + vb));
  const size_t capf = std::max<size_t>(1, std::min(limit, npx / 64 + 1));
  const int nt = std::max(1, std::min(16, omp_get_num_procs()));
  // about four tasks per thread, so the dynamic schedule evens out the threads
  const int nseg = std::max(1, std::min((4 * nt + n - 1) / n, (int)(npx / 4096) + 1));
  const int ntask = n * nseg;
  if (e->bt_idx.size() < (size_t)ntask * capf) e->bt_idx.resize((size_t)ntask * capf);
  if (e->bt_val.size() < (size_t)ntask * capf * vb) e->bt_val.resize((size_t)ntask * capf * vb);
  uint32_t *sidx = e->bt_idx.data();
  T *sval = reinterpret_cast<T *>(e->bt_val.data());
  std::vector<size_t> tcnt((size_t)ntask, 0);
  std::vector<double> tmax((size_t)ntask, 0.0);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (int t = 0; t < ntask; t++) {
    const int f = t / nseg, sg = t % nseg;
    const T *px = static_cast<const T *>(frames[f]);
    const size_t lo = npx * sg / nseg, hi = npx * (sg + 1) / nseg;
    uint32_t *ix = sidx + (size_t)t * capf;
    T *vx = sval + (size_t)t * capf;
    size_t o = 0;
    double m = 0.0;
    for_positive(px, lo, hi, [&](size_t i, T v) {
      if (o < capf) {
        ix[o] = (uint32_t)i;
        vx[o] = v;
      }
      o++;
      if ((double)v > m) m = (double)v;
    });
    tcnt[t] = o;
    tmax[t] = m;
  }
  // frames that fit, their descriptors and packed offsets
  std::vector<SparseFrameDesc> desc;
  std::vector<int> dense;
  std::vector<size_t> toff((size_t)ntask, 0);
  size_t total = 0;
  uint32_t max_nnz = 0;
  for (int f = 0; f < n; f++) {
    size_t nnz = 0;
    double mx = 0.0;
    for (int sg = 0; sg < nseg; sg++) {
      nnz += tcnt[(size_t)f * nseg + sg];
      mx = std::max(mx, tmax[(size_t)f * nseg + sg]);
    }
    if (nnz > capf) {
      dense.push_back(f);
      continue;
    }
    SparseFrameDesc d{};
    d.off = total;
    d.nnz = (uint32_t)nnz;
    d.slot = slots[f];
    d.mx = mx;
    for (int sg = 0; sg < nseg; sg++) {
      toff[(size_t)f * nseg + sg] = total;
      total += tcnt[(size_t)f * nseg + sg];
    }
    max_nnz = std::max(max_nnz, d.nnz);
    desc.push_back(d);
  }
  const int ns = (int)desc.size();
  if (ns) {
    const size_t hdr = (size_t)ns * sizeof(SparseFrameDesc);
    const size_t ioff = ((hdr + 15) / 16) * 16;
    const size_t voff = ioff + ((total * 4 + 15) / 16) * 16;
    const size_t bytes = voff + total * vb;
    const int r = e->bt_next;
    e->bt_next ^= 1;
    if (!e->bt_ev[r]) LMB_CUDA(cudaEventCreateWithFlags(&e->bt_ev[r], cudaEventDisableTiming));
    LMB_CUDA(cudaEventSynchronize(e->bt_ev[r]));  // ring entry free again
    if (e->bt_host_cap[r] < bytes) {
      if (e->bt_host[r]) LMB_CUDA(cudaFreeHost(e->bt_host[r]));
      e->bt_host[r] = nullptr;
      e->bt_host_cap[r] = 0;
      const size_t want = std::max(bytes + bytes / 4, (size_t)1 << 20);
      LMB_CUDA(cudaHostAlloc(&e->bt_host[r], want, cudaHostAllocDefault));
      e->bt_host_cap[r] = want;
    }
    if (e->d_batch_cap < bytes) {
      LMB_CUDA(cudaStreamSynchronize(e->ld));  // the old buffer may still be read
      cudaFree(e->d_batch);
      e->d_batch = nullptr;
      e->d_batch_cap = 0;
      const size_t want = std::max(bytes + bytes / 4, (size_t)1 << 20);
      LMB_CUDA(cudaMalloc(&e->d_batch, want));
      e->d_batch_cap = want;
    }
    char *h = static_cast<char *>(e->bt_host[r]);
    memcpy(h, desc.data(), hdr);
    uint32_t *pidx = reinterpret_cast<uint32_t *>(h + ioff);
    T *pval = reinterpret_cast<T *>(h + voff);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int t = 0; t < ntask; t++) {
      const int f = t / nseg;
      const size_t c = tcnt[t];
      size_t ff = 0;  // is frame f packed?  (dense frames have nnz > capf)
      for (int sg = 0; sg < nseg; sg++) ff += tcnt[(size_t)f * nseg + sg];
      if (ff > capf || c == 0) continue;
      memcpy(pidx + toff[t], sidx + (size_t)t * capf, c * 4);
      memcpy(pval + toff[t], sval + (size_t)t * capf, c * vb);
    }
    for (int i = 0; i < ns; i++)
      LMB_CUDA(cudaStreamWaitEvent(e->ld, e->ev_released[desc[i].slot], 0));
    LMB_CUDA(cudaMemcpyAsync(e->d_batch, h, bytes, cudaMemcpyHostToDevice, e->ld));
    LMB_CUDA(cudaEventRecord(e->bt_ev[r], e->ld));
    e->bytes_h2d += bytes;
    char *d = static_cast<char *>(e->d_batch);
    const int rc = batch_sparse_load_launch(
        reinterpret_cast<const SparseFrameDesc *>(d), ns, max_nnz,
        reinterpret_cast<const uint32_t *>(d + ioff), d + voff, dtype, e->d_u8, e->d_occ,
        e->d_scale, npx, e->num_sms, e->ld);
    if (rc) return rc;
    e->sparse_loads += ns;
    for (int i = 0; i < ns; i++) {
      const int s = desc[i].slot;
      LMB_CUDA(cudaEventRecord(e->ev_loaded[s], e->ld));
      e->loaded_mask |= 1ull << s;
      e->f64_mask &= ~(1ull << s);
    }
  }
  for (int f : dense) {
    const int rc = lmb_image_load(e, slots[f], frames[f], dtype, 0, nullptr);
    if (rc) return rc;
  }
  return LMB_OK;
}

}  // namespace

extern "C" {

int lmb_image_load_batch(lmb_engine *e, const int32_t *slots, const void *const *frames,
                         int32_t n, int32_t dtype, double *im_scales) {
  int rc = check_engine(e);
  if (rc) return rc;
  LMB_REQUIRE(n >= 0 && n <= LMB_MAX_SLOTS, "batch of %d frames (at most %d)", n, LMB_MAX_SLOTS);
  LMB_REQUIRE(n == 0 || (slots && frames), "null slot or frame list");
  LMB_REQUIRE(dtype == LMB_F64 || dtype == LMB_F32 || dtype == LMB_U8, "unknown dtype %d", dtype);
  uint64_t seen = 0;
  for (int i = 0; i < n; i++) {
    LMB_REQUIRE(slots[i] >= 0 && slots[i] < LMB_MAX_SLOTS, "slot %d outside 0..%d", slots[i],
                LMB_MAX_SLOTS - 1);
    LMB_REQUIRE(!(seen >> slots[i] & 1), "slot %d appears twice in the batch", slots[i]);
    LMB_REQUIRE(frames[i], "null frame %d", i);
    seen |= 1ull << slots[i];
  }
  if (!e->sparse_uploads) {
    for (int i = 0; i < n && rc == LMB_OK; i++)
      rc = lmb_image_load(e, slots[i], frames[i], dtype, 0, nullptr);
  } else if (n) {
    // A share of the page-locked frames goes dense over the copy engine
    // (asynchronous: enqueued first, it runs while the host scans the rest),
    // so the host's memory reads and the link work side by side.
    int32_t ss[LMB_MAX_SLOTS];
    const void *sf[LMB_MAX_SLOTS];
    int ns = 0;
    double acc = 0.0;
    for (int i = 0; i < n && rc == LMB_OK; i++) {
      bool dense = false;
      if (e->dense_share > 0.0) {
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, frames[i]) == cudaSuccess &&
            at.type == cudaMemoryTypeHost) {
          acc += e->dense_share;
          if (acc >= 1.0) {
            acc -= 1.0;
            dense = true;
          }
        }
        cudaGetLastError();  // a pageable pointer is not an error here
      }
      if (dense) {
        rc = dense_load(e, slots[i], frames[i], dtype);
      } else {
        ss[ns] = slots[i];
        sf[ns++] = frames[i];
      }
    }
    if (rc == LMB_OK && ns)
      rc = dtype == LMB_F64   ? load_batch_sparse<double>(e, ss, sf, ns, dtype)
           : dtype == LMB_F32 ? load_batch_sparse<float>(e, ss, sf, ns, dtype)
                              : load_batch_sparse<uint8_t>(e, ss, sf, ns, dtype);
  }
  if (rc) return rc;
  if (im_scales && n) {
    double sc[LMB_MAX_SLOTS];
    LMB_CUDA(cudaMemcpyAsync(sc, e->d_scale, sizeof(sc), cudaMemcpyDeviceToHost, e->ld));
    LMB_CUDA(cudaStreamSynchronize(e->ld));
    e->bytes_d2h += sizeof(sc);
    for (int i = 0; i < n; i++) im_scales[i] = sc[slots[i]];
  }
  return LMB_OK;
}

int lmb_match(lmb_engine *e, uint64_t slot_mask, int32_t min_nr_spots, double min_intensity,
              int32_t value_mode) {
  int rc = check_engine(e);
  if (rc) return rc;
  LMB_REQUIRE(e->d_db || e->n == 0, "no DB loaded");
  LMB_REQUIRE((slot_mask & ~e->loaded_mask) == 0, "slot mask names slots with no image");
  LMB_REQUIRE(value_mode == LMB_VALUE_U8 || value_mode == LMB_VALUE_F64, "unknown value mode");
  LMB_REQUIRE(value_mode == LMB_VALUE_U8 || (slot_mask & ~e->f64_mask) == 0,
              "float64 pass needs images loaded with keep_f64");
  CompareTuning tun = e->tuning;
  if (tun.variant >= 2) {  // compact layout: derive it once per DB
    if (e->cl_state == 0) {
      rc = build_compact(e, min_nr_spots);
      if (rc) return rc;
    }
    // variant 3 (automatic): the compact layout alone while the records that
    // can pass hold few spots; beyond that, the compact layout filtered by
    // the batch's cell mask (variant 4) when its hit lists fit a block, the
    // reference records otherwise
    bool compact = e->cl_state == 1;
    if (compact && tun.variant == 3) {
      if (gathered_per_record(e, tun.full_gather ? 0 : min_nr_spots) <= kAutoGather)
        tun.variant = 2;
      else if (!tun.full_gather && min_nr_spots >= 1 && cell_pass_fits(e))
        tun = CompareTuning{kAutoCellVariant, 0, tun.cell_stages, tun.cell_consumers, 1, 1, 0,
                            tun.test_consumer_wait_us, 0, 0, tun.cell_queue};  // cell-mask pass
      else
        compact = false;
    }
    if (!compact)  // warp-specialised over the reference records
      tun = CompareTuning{1, 0, 0, 0, 0, 0, tun.full_gather, tun.test_consumer_wait_us, 0, 0, 0};
  }
  if (tun.variant == 5) {  // its candidate regions, for the filter grid it will launch
    const uint32_t G = (uint32_t)std::min<uint64_t>(e->cl_tiles, (uint64_t)e->num_sms);
    rc = ensure_candidates(e, std::max<uint32_t>(G, 1));
    if (rc) return rc;
  }
  e->last_variant = tun.variant;
  for (int k = 0; k < LMB_MAX_SLOTS; k++)
    if (slot_mask >> k & 1) LMB_CUDA(cudaStreamWaitEvent(e->st, e->ev_loaded[k], 0));
  // The pass (status reset, compare, ordering, status copy-back) replays from
  // a CUDA graph once a configuration has been seen before; the first pass of
  // a configuration runs eagerly (it also sets the kernels' attributes).
  PassKey key;
  key.mask = slot_mask;
  key.min_spots = min_nr_spots;
  key.min_int = min_intensity;
  key.mode = value_mode;
  key.tuning = tun;
  PassGraph *pg = nullptr;
  for (auto &g : e->graphs)
    if (g.key == key) pg = &g;
  if (pg && pg->exec) {
    LMB_CUDA(cudaGraphLaunch(pg->exec, e->st));
  } else if (pg && e->use_graphs) {
    cudaGraph_t graph = nullptr;
    LMB_CUDA(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
    rc = enqueue_pass(e, key, true);
    const cudaError_t ce = cudaStreamEndCapture(e->st, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    LMB_CUDA(ce);
    const cudaError_t ie = cudaGraphInstantiate(&pg->exec, graph, 0);
    cudaGraphDestroy(graph);
    LMB_CUDA(ie);
    LMB_CUDA(cudaGraphLaunch(pg->exec, e->st));
  } else {
    if (!pg) {
      if (e->graphs.size() >= 8) {  // keep the 8 most recent configurations
        if (e->graphs.front().exec) cudaGraphExecDestroy(e->graphs.front().exec);
        e->graphs.erase(e->graphs.begin());
      }
      e->graphs.push_back(PassGraph{key, nullptr});
    }
    rc = enqueue_pass(e, key, false);
    if (rc) return rc;
  }
  for (int k = 0; k < LMB_MAX_SLOTS; k++)
    if (slot_mask >> k & 1) LMB_CUDA(cudaEventRecord(e->ev_released[k], e->st));
  // the pass's status words into the next ring entry
  const int r = (int)(e->pass_seq % kStatusRing);
  LMB_CUDA(cudaMemcpyAsync(e->h_status + (size_t)r * kStatusWords, e->d_status,
                           kStatusWords * sizeof(unsigned int), cudaMemcpyDeviceToHost, e->st));
  LMB_CUDA(cudaEventRecord(e->ev_done[r], e->st));
  e->bytes_d2h += kStatusWords * sizeof(unsigned int);
  for (int k = 0; k < LMB_MAX_SLOTS; k++)
    if (slot_mask >> k & 1) e->slot_ring[k] = r;
  e->done_mask |= slot_mask;
  e->pass_seq++;
  return LMB_OK;
}

}  // extern "C"

namespace {

// Wait for the last pass that included `slot`; its status words.
int slot_status(lmb_engine *e, int slot, const unsigned int **st) {
  LMB_REQUIRE(slot >= 0 && slot < LMB_MAX_SLOTS && (e->done_mask >> slot & 1),
              "slot %d has not been part of a pass", slot);
  const int r = e->slot_ring[slot];
  LMB_CUDA(cudaEventSynchronize(e->ev_done[r]));
  *st = e->h_status + (size_t)r * kStatusWords;
  const int derr = (int)(*st)[2 * LMB_MAX_SLOTS];
  if (derr == DEV_BAD_QUEUE) {
    set_error("compare pass: a compact-layout record longer than the pass's queue entries");
    return LMB_ERR_INVALID;
  }
  if (derr != DEV_OK) {
    set_error("device wait gave up in the compare pass (code %d)", derr);
    return LMB_ERR_TIMEOUT;
  }
  return LMB_OK;
}

}  // namespace

extern "C" {

int lmb_results(lmb_engine *e, int32_t slot, lmb_survivor *out, uint64_t out_capacity,
                uint64_t *n_survivors, uint64_t *n_pass) {
  int rc = check_engine(e);
  if (rc) return rc;
  const unsigned int *sw = nullptr;
  rc = slot_status(e, slot, &sw);
  if (rc) return rc;
  const uint64_t cnt = sw[slot];
  if (n_survivors) *n_survivors = cnt;
  if (n_pass) *n_pass = sw[LMB_MAX_SLOTS + slot];
  if (cnt > e->cap) {
    set_error("slot %d: %llu survivors exceed the engine capacity %u", slot,
              (unsigned long long)cnt, e->cap);
    return LMB_ERR_OVERFLOW;
  }
  if (!out) return LMB_OK;
  if (out_capacity < cnt) {
    set_error("slot %d: %llu survivors exceed the output capacity %llu", slot,
              (unsigned long long)cnt, (unsigned long long)out_capacity);
    return LMB_ERR_OVERFLOW;
  }
  if (cnt)
    LMB_CUDA(cudaMemcpy(out, e->d_sorted + (size_t)slot * e->cap, cnt * sizeof(lmb_survivor),
                        cudaMemcpyDeviceToHost));
  e->bytes_d2h += cnt * sizeof(lmb_survivor);
  return LMB_OK;
}

int lmb_results_batch(lmb_engine *e, const int32_t *slots, int32_t nslots, lmb_survivor *out,
                      uint64_t out_capacity, uint64_t *counts, uint64_t *n_pass) {
  int rc = check_engine(e);
  if (rc) return rc;
  LMB_REQUIRE(nslots >= 0 && (slots || nslots == 0) && counts, "bad slot list");
  uint64_t total = 0;
  bool over = false;
  for (int i = 0; i < nslots; i++) {
    const int k = slots[i];
    const unsigned int *sw = nullptr;
    rc = slot_status(e, k, &sw);
    if (rc) return rc;
    counts[i] = sw[k];
    if (n_pass) n_pass[i] = sw[LMB_MAX_SLOTS + k];
    over |= counts[i] > e->cap;
    total += counts[i];
  }
  if (over) {
    set_error("a slot's survivors exceed the engine capacity %u", e->cap);
    return LMB_ERR_OVERFLOW;
  }
  if (total > out_capacity || (!out && total)) {
    set_error("%llu survivors exceed the output capacity %llu", (unsigned long long)total,
              (unsigned long long)out_capacity);
    return LMB_ERR_OVERFLOW;
  }
  // the survivor lists are final (their passes' events have completed): pack
  // them back to back on the device and copy once, on the download stream so
  // a pass queued meanwhile keeps running
  if (total) {
    if (e->d_gather_cap < total) {
      LMB_CUDA(cudaStreamSynchronize(e->dl));
      cudaFree(e->d_gather);
      e->d_gather = nullptr;
      e->d_gather_cap = 0;
      const uint64_t want = std::max<uint64_t>(total + total / 4, 4096);
      LMB_CUDA(cudaMalloc(&e->d_gather, want * sizeof(lmb_survivor)));
      e->d_gather_cap = want;
    }
    GatherArgs g{};
    g.src = e->d_sorted;
    g.dst = e->d_gather;
    g.cap = e->cap;
    uint64_t off = 0;
    for (int i0 = 0; i0 < nslots; i0 += LMB_MAX_SLOTS) {  // at most 64 lists per launch
      const uint64_t base = off;
      g.dst = e->d_gather + base;
      g.n = std::min(LMB_MAX_SLOTS, nslots - i0);
      g.off[0] = 0;
      for (int i = 0; i < g.n; i++) {
        g.slot[i] = slots[i0 + i];
        g.off[i + 1] = g.off[i] + (uint32_t)counts[i0 + i];
      }
      off = base + g.off[g.n];
      rc = gather_launch(g, e->dl);
      if (rc) return rc;
    }
    LMB_CUDA(cudaMemcpyAsync(out, e->d_gather, total * sizeof(lmb_survivor),
                             cudaMemcpyDeviceToHost, e->dl));
    LMB_CUDA(cudaStreamSynchronize(e->dl));
  }
  e->bytes_d2h += total * sizeof(lmb_survivor);
  return LMB_OK;
}

int lmb_engine_bytes(lmb_engine *e, uint64_t *h2d, uint64_t *d2h) {
  LMB_REQUIRE(e, "null engine");
  if (h2d) *h2d = e->bytes_h2d;
  if (d2h) *d2h = e->bytes_d2h;
  return LMB_OK;
}

int lmb_last_pass_ms(lmb_engine *e, float *compare_ms, float *order_ms) {
  int rc = check_engine(e);
  if (rc) return rc;
  LMB_REQUIRE(e->pass_seq > 0, "no pass has been run");
  LMB_CUDA(cudaEventSynchronize(e->ev[2]));
  float a = 0, b = 0;
  LMB_CUDA(cudaEventElapsedTime(&a, e->ev[0], e->ev[1]));
  LMB_CUDA(cudaEventElapsedTime(&b, e->ev[1], e->ev[2]));
  if (compare_ms) *compare_ms = a;
  if (order_ms) *order_ms = b;
  return LMB_OK;
}

int lmb_engine_set_tuning(lmb_engine *e, const int32_t *fields, int32_t n_fields) {
  LMB_REQUIRE(e && (fields || n_fields == 0), "null argument");
  CompareTuning t{1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  int32_t *dst[11] = {&t.variant,     &t.tile_sub,      &t.stages,
                      &t.consumers,   &t.blocks_per_sm, &t.grid_mult,
                      &t.full_gather, &t.test_consumer_wait_us, &t.cell_consumers,
                      &t.cell_stages, &t.cell_queue};
  for (int i = 0; i < n_fields && i < 11; i++) *dst[i] = fields[i];
  LMB_REQUIRE(t.cell_queue == 0 || t.cell_queue == 1, "cell_queue must be 0 or 1");
  LMB_REQUIRE(t.cell_consumers >= 0 && t.cell_consumers <= 24 && t.cell_stages >= 0 &&
                  t.cell_stages <= 16,
              "cell-mask pass shape (%d consumers, %d stages) out of range", t.cell_consumers,
              t.cell_stages);
  LMB_REQUIRE(t.full_gather == 0 || t.full_gather == 1, "full_gather must be 0 or 1");
  LMB_REQUIRE(t.test_consumer_wait_us >= 0 && t.test_consumer_wait_us <= 1000000,
              "test wait of %d us outside 0..1000000", t.test_consumer_wait_us);
  LMB_REQUIRE(t.variant >= 0 && t.variant <= 5, "unknown compare variant %d", t.variant);
  e->tuning = t;
  return LMB_OK;
}

int lmb_engine_layout_info(lmb_engine *e, int32_t *compact, uint64_t *compact_bytes,
                           int32_t *tiles, int32_t *tile_bytes) {
  LMB_REQUIRE(e, "null engine");
  if (compact) *compact = e->cl_state;
  if (compact_bytes) *compact_bytes = e->cl_bytes;
  if (tiles) *tiles = (int32_t)e->cl_tiles;
  if (tile_bytes) *tile_bytes = (int32_t)e->cl_stage;
  return LMB_OK;
}

int lmb_engine_set_dense_share(lmb_engine *e, double share) {
  LMB_REQUIRE(e, "null engine");
  LMB_REQUIRE(share >= 0.0 && share <= 1.0, "dense share %g outside [0, 1]", share);
  e->dense_share = share;
  return LMB_OK;
}

int lmb_engine_set_sparse_uploads(lmb_engine *e, int32_t enable) {
  LMB_REQUIRE(e, "null engine");
  e->sparse_uploads = enable != 0;
  return LMB_OK;
}

int lmb_engine_get_tuning(lmb_engine *e, int32_t *fields, int32_t n_fields) {
  LMB_REQUIRE(e && (fields || n_fields == 0), "null argument");
  const CompareTuning c = compare_config(e->R, e->tuning);
  const int32_t src[12] = {c.variant,        c.tile_sub,       c.stages,
                           c.consumers,      c.blocks_per_sm,  c.grid_mult,
                           c.full_gather,    e->last_variant,  c.test_consumer_wait_us,
                           c.cell_consumers, c.cell_stages,    c.cell_queue};
  for (int i = 0; i < n_fields && i < 12; i++) fields[i] = src[i];
  return LMB_OK;
}

}  // extern "C"

namespace lmb {

// A frame already in this engine's device memory (written on another stream
// that recorded `ready`) into a slot: the dense quantisation of
// lmb_image_load without any host copy; `consumed` is recorded once the
// frame has been read, so its producer may overwrite it.
int engine_load_device_frame(lmb_engine *e, int slot, const void *d_img, int dtype,
                             int nr_px_y, int nr_px_x, cudaEvent_t ready, cudaEvent_t consumed,
                             double *im_scale) {
  int rc = check_engine(e);
  if (rc) return rc;
  LMB_REQUIRE(slot >= 0 && slot < LMB_MAX_SLOTS, "slot %d outside 0..%d", slot,
              LMB_MAX_SLOTS - 1);
  LMB_REQUIRE(dtype == LMB_F64 || dtype == LMB_F32, "device frame dtype %d", dtype);
  LMB_REQUIRE(nr_px_y == e->geo.nr_px_y && nr_px_x == e->geo.nr_px_x,
              "frame of %d x %d pixels, detector of %d x %d", nr_px_y, nr_px_x, e->geo.nr_px_y,
              e->geo.nr_px_x);
  LMB_CUDA(cudaStreamWaitEvent(e->ld, e->ev_released[slot], 0));
  LMB_CUDA(cudaStreamWaitEvent(e->ld, ready, 0));
  rc = quantize_launch(d_img, dtype, e->npx, e->d_max_bits, e->d_u8 + (size_t)slot * e->npx,
                       nullptr, e->d_occ, slot, e->d_scale + slot, e->num_sms, e->ld);
  if (rc) return rc;
  LMB_CUDA(cudaEventRecord(consumed, e->ld));
  LMB_CUDA(cudaEventRecord(e->ev_loaded[slot], e->ld));
  e->loaded_mask |= 1ull << slot;
  e->f64_mask &= ~(1ull << slot);
  if (im_scale) {
    LMB_CUDA(cudaMemcpyAsync(im_scale, e->d_scale + slot, sizeof(double), cudaMemcpyDeviceToHost,
                             e->ld));
    e->bytes_d2h += sizeof(double);
    LMB_CUDA(cudaStreamSynchronize(e->ld));
  }
  return LMB_OK;
}

int engine_device(const lmb_engine *e) { return e ? e->device : -1; }

}  // namespace lmb

extern "C" {

int lmb_host_alloc(uint64_t bytes, void **out) {
  LMB_REQUIRE(out, "null output");
  *out = nullptr;
  LMB_CUDA(cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocDefault));
  return LMB_OK;
}

int lmb_host_free(void *p) {
  if (p) LMB_CUDA(cudaFreeHost(p));
  return LMB_OK;
}

}  // extern "C"
