// Duplicate removal (stage 3) for callers that cannot allocate GPU memory.
//
// Some hosts of this library must not call cudaMalloc once they are running:
// a caller whose memory is all carved out up front by its own allocator or
// memory pool, a real-time loop that may not take the driver's allocation
// locks, or a plugin that is handed pointers and a stream and nothing else.
// rw_tree_run_stage3 needs an rw_tree_im_storage, and creating one allocates.
// rw_tree_unique_noalloc does the same work with its scratch (the look-back
// words, the tile ticket and the status word) in a fixed array compiled into
// this library, so it allocates nothing at all.
//
// The array is sized for RW_NOALLOC_MAX_KEYS keys (about 64 KiB) and lives on
// every GPU that loads the library until the process exits.  Its device
// address is looked up once per device, on that device's first call.  All
// calls share the one array: calls that run at the same time on the GPU (two
// streams, two threads) race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "internal.hpp"

namespace {

constexpr uint32_t kMaxKeys = RW_NOALLOC_MAX_KEYS;
constexpr uint32_t kMaxTiles = (kMaxKeys + rwt::kUniqueTile - 1) / rwt::kUniqueTile;
// [0, 256): DevStatus, then the tile ticket at 256; look-back words from 512.
constexpr size_t kTicketOffset = 256;
constexpr size_t kDescOffset = 512;
constexpr size_t kScratchBytes = kDescOffset + (size_t(kMaxTiles) + 1) * 4;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

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
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
      return RW_ERR_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return RW_ERR_CUDA;
    g_num_sms[dev] = sms;
    g_scratch_addr[dev] = p;
  }
  *addr = static_cast<unsigned char*>(g_scratch_addr[dev]);
  *num_sms = g_num_sms[dev];
  return RW_OK;
}

}  // namespace

extern "C" int rw_tree_unique_noalloc(const void* sorted_keys, void* unique_keys,
                                      uint32_t n, int32_t key_bits, uint32_t* n_unique,
                                      rw_stream_t stream) {
  if (!sorted_keys || !unique_keys || !n_unique || n < 1 || n > kMaxKeys ||
      (key_bits != 32 && key_bits != 64))
    return RW_ERR_ARG;
  unsigned char* base = nullptr;
  int num_sms = 0;
  if (int rc = scratch_for_current_device(&base, &num_sms)) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  auto* status = reinterpret_cast<rwt::DevStatus*>(base);
  auto* ticket = reinterpret_cast<uint32_t*>(base + kTicketOffset);
  auto* desc = reinterpret_cast<uint32_t*>(base + kDescOffset);
  const uint32_t tiles = (n + rwt::kUniqueTile - 1) / rwt::kUniqueTile;
  // the array keeps the previous call's words: the ticket, the status and the
  // look-back words of this call's tiles must start at zero
  if (cudaMemsetAsync(base, 0, kDescOffset + (size_t(tiles) + 1) * 4, s) != cudaSuccess)
    return RW_ERR_CUDA;
  if (rwt::launch_unique_raw(sorted_keys, unique_keys, n, key_bits, desc, ticket, status,
                             num_sms, s) != cudaSuccess)
    return RW_ERR_CUDA;
  rwt::DevStatus host_status;
  if (cudaMemcpyAsync(&host_status, status, sizeof host_status, cudaMemcpyDeviceToHost,
                      s) != cudaSuccess)
    return RW_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return RW_ERR_CUDA;
  if (host_status.err != 0) return host_status.err;
  *n_unique = host_status.n_unique;
  return RW_OK;
}
