// Kernel argument blocks and launchers shared by the translation units of
// liblmb200 (dbbuild.cu, compare.cu, engine.cu).
#pragma once

#include "common.cuh"

namespace lmb {

// A record the cell filter kept: its id and its marked pixels (n of them at
// offset off of its block's pixel region).
struct CandEntry {
  unsigned long long oid;
  uint32_t off;
  uint32_t n;
};
static_assert(sizeof(CandEntry) == 16, "candidate entry layout");

// One batched DB pass (compare.cu).
struct CmpArgs {
  const uint16_t *db;  // n records of R uint16, 16-byte aligned
  uint64_t n;
  int R, S, W, H;
  int qS;  // compact pass: spots per record-queue entry (the layout's largest count)
  const unsigned long long *occ;  // per pixel: bit k = slot k's uint8 pixel > 0
  unsigned long long active;      // slots of this pass
  const uint8_t *u8;              // slot k image at u8 + k*npx
  const double *f64;              // slot k float64 image at f64 + k*npx (value mode F64)
  size_t npx;
  const double *scale;  // imScale per slot
  int mode;             // LMB_VALUE_U8 / LMB_VALUE_F64
  int min_spots;        // MinNrSpots clamped to >= 0
  double min_int;       // MinIntensity
  lmb_survivor *surv;   // slot k list at surv + k*cap, unordered
  uint32_t cap;
  unsigned int *surv_cnt;  // [64] survivors (score != 0)
  unsigned int *pass_cnt;  // [64] orientations passing both thresholds
  int *err;                // device error word
  // compact layout (variant 2): tile t at cl + t * tile_bytes, cl_tiles of them
  const unsigned char *cl;
  uint64_t cl_tiles;
  // 0: a record with fewer spots than MinNrSpots (it cannot pass: its matched
  // count is at most its spot count) is not gathered; 1: every spot is
  int full_gather;
  // variant 4: cell mask of the pass's slots, bit q = some pixel of
  // [q << cm_shift, (q + 1) << cm_shift) is positive in an active slot;
  // cm_bytes (a multiple of 128) of it are copied into each block's shared memory
  const uint32_t *cellmask;
  uint32_t cm_bytes;
  int cm_shift;
  // test only (compact-layout variants): > 0 makes every consumer warp wait
  // this long on a shared-memory barrier nothing arrives at, instead of on its
  // ring slot, so the pass gives up with a timeout (0 in every normal pass)
  uint64_t test_consumer_wait_ns;
  // variant 4: 1 = records that can still pass are copied (their marked
  // spots) into a per-warp queue and counted 32 at a time; 0 = counted in
  // place, chunk by chunk
  int cell_queue;
  // variant 5: records that can still pass after the cell mask, appended by
  // the filter kernel to its block's region (entries at cq_e + cq_ebase[b],
  // their marked pixels at cq_pix + cq_pbase[b]); cq_count[2b], [2b + 1] =
  // entries and pixels the block wrote; the regions hold every record and
  // spot of the block's tiles, so they cannot overflow
  struct CandEntry *cq_e;
  uint32_t *cq_pix;
  const uint64_t *cq_ebase;
  const uint64_t *cq_pbase;
  uint32_t *cq_count;
  uint32_t cq_blocks;  // the filter grid the regions were laid out for
  // filled by compare_launch
  uint64_t full_tiles, ntiles;
  uint32_t tile_bytes;
  uint32_t tile;  // orientations per tile (tile_sub * 32)
  int stages;     // TMA ring depth
  int tile_sub;   // 32-orientation sub-tiles per tile
  int consumers;  // consumer warps (warp-specialised variant)
};

// Launch shape of the compare pass (autotuned; zero fields = defaults).
struct CompareTuning {
  int variant;        // 0 = block-barrier ring, 1 = warp-specialised, 2 = compact layout,
                      // 3 = automatic, 4 = compact layout + the batch's cell mask,
                      // 5 = cell-mask filter kernel + candidate counting kernel
  int tile_sub;       // 32-orientation sub-tiles per tile
  int stages;         // ring depth
  int consumers;      // consumer warps (variant 1)
  int blocks_per_sm;  // resident blocks per SM (variant 0)
  int grid_mult;      // grid = SMs * blocks_per_sm * grid_mult
  int full_gather;    // 1: gather every spot even of records that cannot pass
  int test_consumer_wait_us;  // test only: see CmpArgs::test_consumer_wait_ns
  // shape of the cell-mask pass when the automatic variant picks it
  // (0 = defaults): consumer warps, ring stages
  int cell_consumers;
  int cell_stages;
  int cell_queue;  // variant 4: see CmpArgs::cell_queue
};
CompareTuning compare_config(int R, const CompareTuning &req);

// Ordering of the survivor lists of a pass by orientation ID (compare.cu).
struct OrderArgs {
  const lmb_survivor *surv;
  lmb_survivor *out;
  const unsigned int *surv_cnt;
  uint32_t cap;
  unsigned long long *scratch;  // [64][cap2] keys for lists above the shared-memory size
  uint32_t cap2;                // power of two >= cap
  int slots[LMB_MAX_SLOTS];
};

int dbbuild_launch(const double *d_om, uint64_t n, const int4 *d_hkl, int nh,
                   const lmb_geometry &geo, uint16_t *d_out, cudaStream_t st, bool exact_all);
int synth_orient_launch(uint64_t seed, uint64_t first, uint64_t n, double *d_out,
                        cudaStream_t st, uint32_t flags = 0);
int quantize_launch(const void *d_img, int dtype, size_t npx, unsigned long long *d_max_bits,
                    uint8_t *d_u8, double *d_f64_keep, unsigned long long *d_occ, int slot,
                    double *d_scale_slot, int num_sms, cudaStream_t st);
int engine_load_device_frame(lmb_engine *e, int slot, const void *d_img, int dtype,
                             int nr_px_y, int nr_px_x, cudaEvent_t ready, cudaEvent_t consumed,
                             double *im_scale);
int engine_device(const lmb_engine *e);
int sparse_load_launch(const uint32_t *d_idx, const void *d_val, int dtype, size_t nnz, double mx,
                       uint8_t *d_u8, unsigned long long *d_occ, int slot, double *d_scale_slot,
                       size_t npx, int num_sms, cudaStream_t st);

// One frame of a batched sparse upload: its (pixel index, value) pairs are
// entries [off, off + nnz) of the packed index and value arrays; mx is the
// largest of its values (0 when it has none).
struct SparseFrameDesc {
  uint64_t off;
  uint32_t nnz;
  int32_t slot;
  double mx;
  double reserved;
};
static_assert(sizeof(SparseFrameDesc) == 32, "descriptor layout");

// Clear the frames' slots, then quantise and scatter all frames' pairs: two
// launches for the whole batch (occupancy bits of different slots share a
// word, so both kernels update it atomically).
int batch_sparse_load_launch(const SparseFrameDesc *d_desc, int nframes, uint32_t max_nnz,
                             const uint32_t *d_idx, const void *d_val, int dtype, uint8_t *d_u8,
                             unsigned long long *d_occ, double *d_scale, size_t npx, int num_sms,
                             cudaStream_t st);
int compare_launch(CmpArgs a, const CompareTuning &req, int num_sms, cudaStream_t st);
int order_launch(const OrderArgs &a, int nslots, cudaStream_t st);

// Survivor lists of several slots packed back to back (slot i's list at
// off[i]) for one device-to-host copy.
struct GatherArgs {
  const lmb_survivor *src;  // slot k's sorted list at src + k*cap
  lmb_survivor *dst;
  uint32_t cap;
  int n;
  int slot[LMB_MAX_SLOTS];
  uint32_t off[LMB_MAX_SLOTS + 1];
};
int gather_launch(const GatherArgs &g, cudaStream_t st);

// Duplicate merge on the device (merge.cu).
struct MergeArgs {
  double *quat;        // [n][4] candidates' quaternions, input order
  double *fr;          // [n][4] in the fundamental region
  double *score;
  uint32_t *bits;      // [n][W]: column g, bit l = l merges into g
  uint32_t *unsure;    // [cap][2] (l, g) pairs left to the host
  unsigned *n_unsure;
  unsigned cap_unsure;
  int64_t *out_best;   // per cluster: index of the kept candidate
  int32_t *out_count;  // per cluster: candidates merged (the reference's dArr)
  int *n_clusters;
  int64_t n, W;
  int nsym;
  double sym[24][4];
  double max_angle, rad2deg;
  double mid, window;  // float rounding boundary at max_angle, and the band left to the host
};
int status_reset_launch(unsigned int *d_status, uint64_t mask, cudaStream_t st);

// Compact DB layout (clist.cu): on-detector spots per 32-record chunk, then
// the fixed-size tiles from the host's packing of chunks into tiles.  Byte
// offsets of the parts of a tile of nch chunks (after the 16-byte header and
// the uint8 per-chunk maximum counts).
__host__ __device__ __forceinline__ uint32_t clist_cnt_offset(uint32_t nch) {
  return 16u + ((nch + 15u) / 16u) * 16u;
}
__host__ __device__ __forceinline__ uint32_t clist_base_offset(uint32_t nch) {
  return clist_cnt_offset(nch) + 32u * nch;
}
__host__ __device__ __forceinline__ uint32_t clist_spot_offset(uint32_t nch) {
  return ((clist_base_offset(nch) + 4u * nch + 15u) / 16u) * 16u;
}
// Per consumer warp of the compact pass, a shared-memory queue of 32 records:
// uint64 id[32] | uint32 count[32] | uint32 pixel[32][stride], stride = S
// rounded up to odd (conflict-free lane-strided reads).
__host__ __device__ __forceinline__ uint32_t clist_queue_stride(int S) {
  return (uint32_t)(S < 1 ? 1 : S) | 1u;
}
__host__ __device__ __forceinline__ uint32_t clist_queue_bytes(int S) {
  return 384u + 128u * clist_queue_stride(S);
}
int clist_chunk_launch(const uint16_t *d_db, uint64_t n, int R, int S, int W, int H,
                       uint32_t *d_chunk_spots, unsigned long long *d_hist, cudaStream_t st);

// Cell mask of a pass (variant 4): at most kCellMaskBytes, so it fits a
// block's shared memory beside the ring.  The shift is the smallest that
// makes npx >> shift cells fit; cellmask_bytes is the buffer size used (a
// multiple of 128, words past the last cell stay zero).
constexpr uint32_t kCellMaskBytes = 128u * 1024u;
__host__ __forceinline__ int cellmask_shift(uint64_t npx) {
  int s = 0;
  while (((npx + (1ull << s) - 1) >> s) > 8ull * kCellMaskBytes) s++;
  return s;
}
__host__ __forceinline__ uint32_t cellmask_bytes(uint64_t npx) {
  const int s = cellmask_shift(npx);
  const uint64_t cells = (npx + (1ull << s) - 1) >> s;
  const uint64_t words = (cells + 31) / 32;
  return (uint32_t)(((words * 4 + 127) / 128) * 128);
}
// Per consumer warp of variant 4: the chunk's spots on marked cells (at most
// 32 * qS pixel indices), then per 32-spot window its hit bits and the hits
// before it.
__host__ __device__ __forceinline__ uint32_t cell_warp_bytes(int qS) {
  const uint32_t q = (uint32_t)(qS < 1 ? 1 : qS);
  return ((32u * q + 2u * q) * 4u + 15u) / 16u * 16u;
}
// ... plus, with the candidate queue, a record queue like the compact pass's
__host__ __device__ __forceinline__ uint32_t cell_warp_bytes(int qS, int queue) {
  return cell_warp_bytes(qS) + (queue ? clist_queue_bytes(qS) : 0u);
}
// Variant 5's filter kernel: per consumer warp the hit bits of up to qS
// 32-spot windows.
__host__ __device__ __forceinline__ uint32_t filter_warp_bytes(int qS) {
  const uint32_t q = (uint32_t)(qS < 1 ? 1 : qS);
  return (4u * q + 15u) / 16u * 16u;
}
int cellmask_launch(const unsigned long long *d_occ, uint64_t npx, unsigned long long active,
                    int shift, uint32_t cm_bytes, uint32_t *d_mask, int num_sms, cudaStream_t st);
int clist_fill_launch(const uint16_t *d_db, uint64_t n, int R, int S, int W, int H, uint32_t TB,
                      const uint32_t *d_ctile, const uint32_t *d_cpos, const uint32_t *d_cbase,
                      const uint32_t *d_tnch, unsigned char *d_cl, cudaStream_t st);

}  // namespace lmb
