// Duplicate removal (stage 3) for callers that cannot allocate GPU memory.
//
// Some hosts of this library must not call cudaMalloc once they are running:
// a caller whose memory is all carved out up front by its own allocator or
// memory pool, a real-time loop that may not take the driver's allocation
// locks, or a plugin that is handed pointers and a stream and nothing else.
// rw_tree_run_stage3 needs an rw_tree_im_storage, and creating one allocates.
// rw_tree_unique_noalloc does the same work with its scratch (the device
// status word with the count, and one head count per tile of keys, which the
// one-block tile scan turns into each tile's output offset) in a fixed array
// compiled into this library, so it allocates nothing at all.
//
// The array is sized for RW_NOALLOC_MAX_KEYS keys (about 64 KiB) and lives on
// every GPU that loads the library until the process exits.  Its device
// address is looked up once per device, on that device's first call.  All
// calls share the one array: calls that run at the same time on the GPU (two
// streams, two threads) race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "internal.hpp"

namespace {

constexpr uint32_t kMaxKeys = RW_NOALLOC_MAX_KEYS;
constexpr uint32_t kMaxTiles = (kMaxKeys + rwt::kUniqueTile - 1) / rwt::kUniqueTile;
// [0, 256): DevStatus; from 256: one head count per tile and the total
// (tiles + 1 words), scanned in place into the tiles' output offsets.
constexpr size_t kCountsOffset = 256;
constexpr size_t kScratchBytes = kCountsOffset + (size_t(kMaxTiles) + 1) * 4;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

int fail(const char* what, cudaError_t e);

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};

// Device address of the scratch array on the current device.  A host-side
// reference to g_noalloc_scratch names a host shadow, not device memory, so
// the address must come from cudaGetSymbolAddress.
int scratch_for_current_device(unsigned char** addr, int* num_sms) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return RW_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return fail("cudaGetSymbolAddress", e);
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail("cudaDeviceGetAttribute", e);
    g_num_sms[dev] = sms;
    g_scratch_addr[dev] = p;
  }
  *addr = static_cast<unsigned char*>(g_scratch_addr[dev]);
  *num_sms = g_num_sms[dev];
  return RW_OK;
}

int fail(const char* what, cudaError_t e) {
  rwt::set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
  return RW_ERR_CUDA;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

extern "C" int rw_tree_unique_noalloc(const void* sorted_keys, void* unique_keys,
                                      uint32_t n, int32_t key_bits, uint32_t* n_unique,
                                      rw_stream_t stream) {
  if (!sorted_keys || !unique_keys || !n_unique || n < 1 || n > kMaxKeys ||
      (key_bits != 32 && key_bits != 64))
    return RW_ERR_ARG;
  // the same rules as the allocating entry points: 16-byte aligned key
  // buffers (the kernels read keys as vectors); and separate ones, since tiles
  // write their output while other tiles still read the input.  Both are
  // checked before any device access
  if (!aligned16(sorted_keys) || !aligned16(unique_keys)) return RW_ERR_ARG;
  const uintptr_t in0 = reinterpret_cast<uintptr_t>(sorted_keys);
  const uintptr_t out0 = reinterpret_cast<uintptr_t>(unique_keys);
  const uintptr_t bytes = uintptr_t(n) * (key_bits == 32 ? 4u : 8u);
  if (in0 < out0 + bytes && out0 < in0 + bytes) return RW_ERR_ARG;
  unsigned char* base = nullptr;
  int num_sms = 0;
  if (int rc = scratch_for_current_device(&base, &num_sms)) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  auto* status = reinterpret_cast<rwt::DevStatus*>(base);
  auto* counts = reinterpret_cast<uint32_t*>(base + kCountsOffset);
  const uint32_t tiles = (n + rwt::kUniqueTile - 1) / rwt::kUniqueTile;
  // the array keeps the previous call's words: the status and this call's
  // tile counts must start at zero
  cudaError_t e = cudaMemsetAsync(base, 0, kCountsOffset + (size_t(tiles) + 1) * 4, s);
  if (e != cudaSuccess) return fail("cudaMemsetAsync (scratch)", e);
  e = rwt::launch_unique_raw(sorted_keys, unique_keys, n, key_bits, counts, status, num_sms, s);
  if (e != cudaSuccess) return fail("unique kernels", e);
  rwt::DevStatus host_status;
  e = cudaMemcpyAsync(&host_status, status, sizeof host_status, cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return fail("cudaMemcpyAsync (status)", e);
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail("cudaStreamSynchronize", e);
  if (host_status.err != 0) {
    rwt::set_last_error("device error " + std::to_string(host_status.err) + " in unique");
    return host_status.err;
  }
  *n_unique = host_status.n_unique;
  return RW_OK;
}
