// Device-side building blocks shared by the tree kernels (sm_100a only).
//
// Single-pass scans use decoupled look-back: every tile publishes a 32-bit
// descriptor (bits 1:0 flag, bits 31:2 value) - first its own aggregate, then
// its inclusive prefix once the predecessors' are known.  Every wait on a
// predecessor is bounded; on timeout the tile records RW_ERR_TIMEOUT in the
// device status word and publishes a (wrong but final) inclusive value so that
// no successor waits on it, and the host reports the error.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rw_tree.h"

namespace rwt {

// Device-resident counts and error word, mirrored to pinned host memory.
struct DevStatus {
  uint32_t n_unique;        // written by the unique kernel's last tile
  uint32_t n_octree_nodes;  // written by the scan's last tile
  int32_t err;              // first rw_status error seen on the device
  uint32_t err_site;        // which kernel reported it
};

enum : uint32_t { kFlagAgg = 1u, kFlagInc = 2u, kFlagMask = 3u };
enum : uint32_t {
  kSiteSort = 1,
  kSiteUnique = 2,
  kSiteScan = 3,
  kSiteTree = 4,
  kSiteOctree = 5
};

// ~1 s of polling with back-off before a wait gives up.
constexpr uint32_t kSpinLimit = 1u << 21;

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Programmatic dependent launch.  Every kernel of the pipeline starts with
// pdl_enter(): it waits until the grid before it in the stream has completed
// and its writes are visible (a no-op when the kernel was launched without
// the attribute), then lets the next grid be scheduled, so that its blocks
// take the SM slots this grid's last wave frees instead of waiting for a
// fresh launch.  Nothing is read or written before the wait.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Launches a kernel that begins with pdl_enter() with programmatic stream
// serialization; errors are reported as by a <<<>>> launch.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t s, Args&&... args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ void report_error(DevStatus* st, int32_t code,
                                             uint32_t site) {
  if (atomicCAS(reinterpret_cast<int*>(&st->err), 0, code) == 0)
    st->err_site = site;
}

__device__ __forceinline__ bool device_failed(const DevStatus* st) {
  return *reinterpret_cast<const volatile int32_t*>(&st->err) != 0;
}

__device__ __forceinline__ void backoff(uint32_t spin) {
  if (spin > 64) __nanosleep(spin > 4096 ? 512 : 64);
}

// ---- bulk copies global -> shared (cp.async.bulk) completed on an mbarrier ----
// One thread arms the barrier with the byte count and issues the copy; every
// thread then waits for the barrier's phase 0.  Source, destination and size
// must be multiples of 16 bytes (the caller checks).

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Initialises the barrier (one arrival per phase) and makes the initialisation
// visible to the copy engine; call from one thread, then __syncthreads().
__device__ __forceinline__ void bulk_barrier_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One thread: expect `bytes` on the barrier and copy them from global memory.
__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_addr(dst_smem)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

// Waits for phase 0 of the barrier, at most `limit` polls (with back-off);
// returns false if the copy did not complete in time.
__device__ __forceinline__ bool bulk_wait(uint64_t* bar, uint32_t limit) {
  const uint32_t a = smem_addr(bar);
  for (uint32_t spin = 0; spin < limit; ++spin) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done) : "r"(a) : "memory");
    if (done) return true;
    backoff(spin);
  }
  return false;
}

// Inclusive warp scan (Kogge-Stone over shuffles).
template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
  const uint32_t lane = lane_id();
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const T u = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= (uint32_t)d) v += u;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  return v;
}

// Block-wide exclusive scan of one value per thread.  `s_warp` needs
// THREADS/32 entries.  Returns the exclusive prefix; *total gets the sum.
template <int THREADS, typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* s_warp, T* total) {
  constexpr int NW = THREADS / 32;
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  const T inc = warp_inclusive_scan(v);
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    T w = lane < (uint32_t)NW ? s_warp[lane] : T(0);
    const T wi = warp_inclusive_scan(w);
    if (lane < (uint32_t)NW) s_warp[lane] = wi - w;
    if (lane == NW - 1) s_warp[NW] = wi;
  }
  __syncthreads();
  const T out = s_warp[warp] + inc - v;
  *total = s_warp[NW];
  __syncthreads();
  return out;
}

// ---------------------------------------------------------------------------
// Segments: a batch of independent point clouds stored back to back.  A plain
// run is one segment.  Every kernel walks a tile map: segment c owns the tiles
// [toff[c], toff[c+1]) of that kernel's tile size.
// ---------------------------------------------------------------------------
struct SegTable {
  uint32_t count;       // segments
  uint32_t total;       // points over all segments
  const uint32_t* off;  // [count + 1] point offsets (device); null when count == 1
};

struct TileMap {
  uint32_t n_tiles;      // tiles over all segments
  const uint32_t* toff;  // [count + 1] tile offsets (device); null when count == 1
};

__device__ __forceinline__ uint32_t seg_begin(const SegTable& s, uint32_t c) {
  return s.off ? s.off[c] : 0u;
}
__device__ __forceinline__ uint32_t seg_size(const SegTable& s, uint32_t c) {
  return s.off ? s.off[c + 1] - s.off[c] : s.total;
}
// Segment of global tile t and its first tile.
__device__ __forceinline__ uint32_t tile_segment(const SegTable& s, const TileMap& m,
                                                 uint32_t t, uint32_t* first_tile) {
  if (!m.toff) {
    *first_tile = 0;
    return 0;
  }
  uint32_t lo = 0, hi = s.count;  // toff[lo] <= t < toff[hi]
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (m.toff[mid] <= t) lo = mid;
    else hi = mid;
  }
  *first_tile = m.toff[lo];
  return lo;
}

}  // namespace rwt
