// Allocation-free link list: the ordered compaction of tlbm_link_count +
// tlbm_link_list in one call, with its per-block scratch in a static device
// array instead of a caller-provided buffer.
//
// Who needs it: a host program that reserves all device memory once at start-up
// (a fixed memory budget handed to a solver framework, or a caching allocator
// that owns the rest of the device) and may not call cudaMalloc / cudaFree in
// its time loop, because those calls can fail once the budget is taken and may
// synchronise the device in the middle of an asynchronous pipeline.
#include <mutex>

#include "ops.cuh"

namespace {

// Block counts of the compaction: one int64 per 1024 mask bytes (the total
// goes to the caller's count_out, not here).  kLinkStaticMaxBlocks blocks cover
// masks of up to kLinkStaticMaxBlocks * 1024 bytes (128 Mi entries; 1 MiB of
// device memory, held by every device that loads the library until the process
// exits).
constexpr long long kLinkStaticMaxBlocks = 131072;
static __device__ __align__(256) long long g_link_scratch[kLinkStaticMaxBlocks];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
long long* g_scratch_ptr[kMaxDevices] = {};

// The counting pass (op_link_count) splits the mask into blocks of 1024 bytes
// handled by 256 threads x 4 consecutive bytes; the writing pass below uses
// the same partition, so block b's offset from the scan is its first index.
constexpr int kThreads = 256;
constexpr long long kChunk = 1024;

// Writes the flat indices of the non-zero mask bytes in increasing order,
// keeping only the first `capacity` of them.
__global__ void k_link_list_capped(const uint8_t* mask, long long count, const long long* offsets, long long* out,
                                   long long capacity) {
  __shared__ int sh[kThreads];
  const long long base = (long long)blockIdx.x * kChunk + (long long)threadIdx.x * 4;
  int c = 0;
  bool hit[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const long long i = base + k;
    hit[k] = (i < count) && mask[i];
    c += hit[k];
  }
  sh[threadIdx.x] = c;
  __syncthreads();
  for (int o = 1; o < kThreads; o <<= 1) {
    const int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += t;
    __syncthreads();
  }
  long long pos = offsets[blockIdx.x] + sh[threadIdx.x] - c;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (hit[k]) {
      if (pos < capacity) out[pos] = base + k;
      ++pos;
    }
}

// Device address of g_link_scratch on the current device.  In host code the
// symbol only names a host-side stand-in, so the address is looked up with
// cudaGetSymbolAddress once per device, with that device current.
int scratch_on_current_device(long long** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TLBM_ERR_LAUNCH;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_link_scratch) != cudaSuccess || !p) return TLBM_ERR_LAUNCH;
    g_scratch_ptr[dev] = static_cast<long long*>(p);
  }
  *out = g_scratch_ptr[dev];
  return TLBM_OK;
}

}  // namespace

extern "C" {

TLBM_API int64_t tlbm_link_list_static_capacity(void) { return kLinkStaticMaxBlocks * 1024LL; }

TLBM_API int tlbm_link_list_noalloc(const uint8_t* mask, int64_t count, int64_t* out, int64_t out_capacity,
                                    int64_t* count_out, void* stream) {
  if (count < 0 || out_capacity < 0) return TLBM_ERR_SHAPE;
  // out may be null for a count-only query (out_capacity == 0): nothing is written to it
  if (!count_out || (count > 0 && (!mask || (out_capacity > 0 && !out)))) return TLBM_ERR_ARG;
  const long long nb = tlbm::op_link_blocks(count);
  if (nb > kLinkStaticMaxBlocks) return TLBM_ERR_TOO_LARGE;
  if (tlbm::op_link_blocks(kChunk) != 1 || tlbm::op_link_blocks(kChunk + 1) != 2) return TLBM_ERR_UNSUPPORTED;
  long long* scratch = nullptr;
  int st = scratch_on_current_device(&scratch);
  if (st != TLBM_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // every block count the scan reads is written by this call's count kernel,
  // so nothing of the previous call's contents needs clearing
  st = tlbm::op_link_count(mask, count, scratch, (long long*)count_out, s);
  if (st != TLBM_OK || nb == 0 || out_capacity == 0) return st;
  k_link_list_capped<<<(int)nb, kThreads, 0, s>>>(mask, count, scratch, (long long*)out, out_capacity);
  return cudaGetLastError() == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH;
}

}  // extern "C"
