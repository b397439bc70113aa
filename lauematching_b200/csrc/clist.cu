// Compact device layout of the DB for the compare pass (variant 2).
//
// The reference record (LaueMatchingCPU.c:488-495) is uint16[1 + 2S]: a
// count and S (x, y) pairs, zero padded.  Only the first min(count, S) pairs
// are read by the compare (LaueMatchingGPU.cu:54-55), and a pair off the
// detector never matches (:65).  The compact layout keeps exactly the pairs
// the compare can use, in record order, as pixel indices y*W + x, so a pass
// reads about 1 byte per record plus 4 bytes per on-detector spot instead of
// 2 + 4S bytes.  The reference layout stays resident as the source of truth
// (DB downloads, cache files); the compact one is derived from it.
//
// The layout is a sequence of fixed-size tiles of TB bytes (a multiple of
// 128), each holding whole 32-record chunks, consecutive in ID:
//   uint64 first_record | uint32 nch | uint32 0          (16-byte header)
//   uint8  chunk_max[nch]          (pad to 16)           largest count of a chunk
//   uint8  count[32 * nch]                               on-detector spots
//   uint32 chunk_base[nch]         (pad to 16)           first spot of a chunk
//   uint32 spot[]                                        pixel indices
// Fixed-size tiles let the pass address tile t as t*TB with no table lookup;
// chunk_max lets it pass over, 32 chunks per vote, the chunks none of whose
// records has MinNrSpots spots.
#include "kernels.cuh"

namespace lmb {

// On-detector spots of record i (0 past the end), clamped count like the compare.
__device__ __forceinline__ int clist_count(const uint16_t *db, uint64_t n, int R, int S, int W,
                                           int H, uint64_t i) {
  if (i >= n) return 0;
  const uint16_t *rec = db + i * (uint64_t)R;
  int c = rec[0];
  if (c > S) c = S;
  int k = 0;
  for (int s = 0; s < c; s++) k += (rec[1 + 2 * s] < W && rec[2 + 2 * s] < H) ? 1 : 0;
  return k;
}

// Spots per 32-record chunk (one warp per chunk), and the histogram of the
// records' on-detector spot counts (hist[c], c <= S <= 255).
__global__ void clist_chunk_kernel(const uint16_t *__restrict__ db, uint64_t n, int R, int S, int W,
                                   int H, uint64_t nchunks, uint32_t *__restrict__ chunk_spots,
                                   unsigned long long *__restrict__ hist) {
  __shared__ unsigned int h[256];
  for (int k = threadIdx.x; k < 256; k += blockDim.x) h[k] = 0;
  __syncthreads();
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t ch = i >> 5;
  if (ch < nchunks) {  // whole warps: blockDim is a multiple of 32
    const int c = clist_count(db, n, R, S, W, H, i);
    if (i < n) atomicAdd(&h[c], 1u);
    const int sum = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0) chunk_spots[ch] = (uint32_t)sum;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < 256; k += blockDim.x)
    if (h[k]) atomicAdd(&hist[k], (unsigned long long)h[k]);
}

// Write the tiles from the host's packing: chunk ch goes to tile ctile[ch] at
// position cpos[ch] with first spot cbase[ch]; tile t holds tnch[t] chunks.
__global__ void clist_fill_kernel(const uint16_t *__restrict__ db, uint64_t n, int R, int S, int W,
                                  int H, uint64_t nchunks, uint32_t TB,
                                  const uint32_t *__restrict__ ctile,
                                  const uint32_t *__restrict__ cpos,
                                  const uint32_t *__restrict__ cbase,
                                  const uint32_t *__restrict__ tnch, unsigned char *__restrict__ cl) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t ch = i >> 5;
  if (ch >= nchunks) return;
  const int lane = threadIdx.x & 31;
  const int c = clist_count(db, n, R, S, W, H, i);
  int x = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  const uint32_t t = ctile[ch], pos = cpos[ch], nch = tnch[t];
  unsigned char *tb = cl + (uint64_t)t * TB;
  if (pos == 0 && lane == 0) {
    *reinterpret_cast<uint64_t *>(tb) = ch * 32;
    *reinterpret_cast<uint32_t *>(tb + 8) = nch;
  }
  const int cmax = __reduce_max_sync(0xffffffffu, c);
  tb[clist_cnt_offset(nch) + 32 * pos + lane] = (unsigned char)c;
  if (lane == 0) {
    tb[16 + pos] = (unsigned char)cmax;
    reinterpret_cast<uint32_t *>(tb + clist_base_offset(nch))[pos] = cbase[ch];
  }
  if (c) {
    uint32_t *spots = reinterpret_cast<uint32_t *>(tb + clist_spot_offset(nch));
    const uint16_t *rec = db + i * (uint64_t)R;
    uint32_t o = cbase[ch] + (uint32_t)(x - c);
    int cnt = rec[0];
    if (cnt > S) cnt = S;
    for (int s = 0; s < cnt; s++) {
      const uint32_t px = rec[1 + 2 * s], py = rec[2 + 2 * s];
      if (px < (uint32_t)W && py < (uint32_t)H) spots[o++] = py * (uint32_t)W + px;
    }
  }
}

int clist_chunk_launch(const uint16_t *d_db, uint64_t n, int R, int S, int W, int H,
                       uint32_t *d_chunk_spots, unsigned long long *d_hist, cudaStream_t st) {
  const uint64_t nchunks = (n + 31) / 32;
  if (nchunks == 0) return LMB_OK;
  LMB_REQUIRE(S <= 255, "spot counts above 255 do not fit the histogram");
  const uint64_t threads = nchunks * 32;
  LMB_CUDA(cudaMemsetAsync(d_hist, 0, 256 * sizeof(unsigned long long), st));
  clist_chunk_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
      d_db, n, R, S, W, H, nchunks, d_chunk_spots, d_hist);
  LMB_CUDA(cudaGetLastError());
  return LMB_OK;
}

int clist_fill_launch(const uint16_t *d_db, uint64_t n, int R, int S, int W, int H, uint32_t TB,
                      const uint32_t *d_ctile, const uint32_t *d_cpos, const uint32_t *d_cbase,
                      const uint32_t *d_tnch, unsigned char *d_cl, cudaStream_t st) {
  const uint64_t nchunks = (n + 31) / 32;
  if (nchunks == 0) return LMB_OK;
  const uint64_t threads = nchunks * 32;
  clist_fill_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
      d_db, n, R, S, W, H, nchunks, TB, d_ctile, d_cpos, d_cbase, d_tnch, d_cl);
  LMB_CUDA(cudaGetLastError());
  return LMB_OK;
}

}  // namespace lmb
