// Survivor ordering without allocation.
//
// Same ordering as the pass's order_kernel (ascending orientation id, keys
// id<<24 | index, bitonic), for callers that hand in device buffers they got
// elsewhere and cannot call cudaMalloc themselves -- for example code running
// inside another framework's memory pool, or a thread that must not take the
// implicit device synchronisation of an allocation.  Lists above the
// shared-memory size use a file-scope device array as key scratch instead of
// allocated memory; that array (8 MiB) lives on every GPU that loads the
// library until the process exits.
#include <mutex>

#include "kernels.cuh"

namespace lmb {

static constexpr uint32_t kNoAllocMax = LMB_NOALLOC_ORDER_MAX;
static constexpr uint32_t kNoAllocSmemKeys = 8192;

// Key scratch shared by every call on a device (host code must not use this
// name as a device address: it is the host-side shadow of the symbol).
static __device__ __align__(256) unsigned long long g_order_scratch[kNoAllocMax];

// Key order.  Packed keys (id << 24 | index) compare as integers while every
// id is below 2^40; otherwise keys hold the index alone and compare by
// (id, index) read from the input.  Keys past n sort last either way.
__device__ __forceinline__ bool key_after(unsigned long long x, unsigned long long y,
                                          const lmb_survivor *__restrict__ in, uint32_t n,
                                          bool wide) {
  if (!wide || x >= n || y >= n) return x > y;
  const uint64_t ix = in[x].id, iy = in[y].id;
  return ix != iy ? ix > iy : x > y;
}

__global__ void __launch_bounds__(1024) order_noalloc_kernel(const lmb_survivor *__restrict__ in,
                                                             uint32_t n,
                                                             lmb_survivor *__restrict__ out,
                                                             unsigned long long *scratch) {
  extern __shared__ __align__(16) unsigned long long sk[];
  uint32_t P = 1;
  while (P < n) P <<= 1;
  unsigned long long *keys = (P <= kNoAllocSmemKeys) ? sk : scratch;
  int big = 0;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) big |= (in[i].id >> 40) != 0;
  const bool wide = __syncthreads_or(big) != 0;
  for (uint32_t i = threadIdx.x; i < P; i += blockDim.x)  // every used key rewritten per call
    keys[i] = (i < n) ? (wide ? (unsigned long long)i : ((in[i].id << 24) | i)) : ~0ull;
  __syncthreads();
  for (uint32_t size = 2; size <= P; size <<= 1) {
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t i = threadIdx.x; i < (P >> 1); i += blockDim.x) {
        const uint32_t lo = 2 * i - (i & (stride - 1));
        const uint32_t hi = lo + stride;
        const bool asc = (lo & size) == 0;
        const unsigned long long x = keys[lo], y = keys[hi];
        if (key_after(x, y, in, n, wide) == asc) {
          keys[lo] = y;
          keys[hi] = x;
        }
      }
      __syncthreads();
    }
  }
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) out[i] = in[keys[i] & 0xFFFFFFull];
}

namespace {
std::mutex g_setup_mu;
void *g_scratch_dev[256];  // device address of g_order_scratch per device ordinal
bool g_attr_set[256];

// Once per device, with that device current: resolve the array's device
// address and raise the kernel's shared-memory limit.
int noalloc_setup(int dev, unsigned long long **scratch) {
  LMB_REQUIRE(dev >= 0 && dev < 256, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_dev[dev]) {
    void *p = nullptr;
    LMB_CUDA(cudaGetSymbolAddress(&p, g_order_scratch));
    g_scratch_dev[dev] = p;
  }
  if (!g_attr_set[dev]) {
    LMB_CUDA(cudaFuncSetAttribute(order_noalloc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(kNoAllocSmemKeys * sizeof(unsigned long long))));
    g_attr_set[dev] = true;
  }
  *scratch = static_cast<unsigned long long *>(g_scratch_dev[dev]);
  return LMB_OK;
}
}  // namespace

}  // namespace lmb

using namespace lmb;

extern "C" int lmb_order_survivors_noalloc(const lmb_survivor *d_in, uint64_t n,
                                           lmb_survivor *d_out, void *stream) {
  LMB_REQUIRE(n <= kNoAllocMax,
              "lmb_order_survivors_noalloc: %llu survivors exceed the fixed scratch of %u "
              "entries (LMB_NOALLOC_ORDER_MAX)",
              (unsigned long long)n, kNoAllocMax);
  if (n == 0) return LMB_OK;
  LMB_REQUIRE(d_in && d_out, "null device pointer");
  // the final gather reads the input while it writes the output: no overlap
  LMB_REQUIRE(d_out >= d_in + n || d_in >= d_out + n, "input and output must not overlap");
  int dev = 0;
  LMB_CUDA(cudaGetDevice(&dev));
  unsigned long long *scratch = nullptr;
  const int rc = noalloc_setup(dev, &scratch);
  if (rc) return rc;
  order_noalloc_kernel<<<1, 1024, kNoAllocSmemKeys * sizeof(unsigned long long),
                         static_cast<cudaStream_t>(stream)>>>(d_in, (uint32_t)n, d_out, scratch);
  LMB_CUDA(cudaGetLastError());
  return LMB_OK;
}
