// Clustering on device digis with no device allocation at all.
//
// Some callers cannot allocate device memory: an event loop whose device memory
// is wholly owned by another allocator, or a trigger path that must not block on
// cudaMalloc/cudaFree (both can synchronise the device). This entry point takes
// device inputs and outputs from the caller and keeps its scratch (per-event
// record, per-chunk module-start counts, cluster module starts, the list of
// modules too large for one warp) in one
// file-scope device array of fixed size, so it calls no cudaMalloc, cudaFree
// or allocating library routine.
//
// The array is a host-side stand-in in host code: its device address is looked
// up with cudaGetSymbolAddress once per device, with that device current, on the
// first call made on that device (so that first call should come before any
// stream capture). Every GPU that loads the library holds the array until exit.
// All calls share it and it keeps the last call's contents: the scratch that
// must start at zero is cleared by each call, and calls that overlap on the GPU
// (different streams, or host threads without ordering) race on it.
//
// Capacity warnings of the chain (more than 2000 module runs, more than 4000 pixels or
// 1024 clusters in a module) stay in the shared scratch and are not returned: a
// module_start[0] of 2000 means that the module list overflowed.
#include <cstdio>
#include <mutex>

#include "../../include/pxl.h"
#include "pxl_internal.cuh"

namespace pxl {

namespace {

constexpr int32_t kNoAllocMaxDigis = 1 << 20;  // 1,048,576 digis per call
constexpr uint32_t kChunk = 256;                // digis per module-start chunk
constexpr int kMaxChunks = int(kNoAllocMaxDigis / kChunk);
constexpr int kMaxDevices = 64;

struct NoAllocScratch {
  EvInfo ev[2];
  uint32_t chunk_nw[kMaxChunks];
  uint32_t chunk_wo[kMaxChunks];
  uint32_t chunk_nmod[kMaxChunks];
  uint32_t clus_module_start[kMaxNumModules + 1];
  uint32_t big_list[kListHeader + kNumLists * kMaxNumModules];
  uint32_t id_seen[64];
  uint32_t status;
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// zero the per-call records, lay out the chunks, clus[i] = i + 1 as count_modules does
__global__ void k_noalloc_init(NoAllocScratch* s, int32_t n, int32_t* clus) {
  const int32_t nchunks = int32_t((uint32_t(n) + kChunk - 1) / kChunk);
  const int32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t stride = gridDim.x * blockDim.x;
  if (tid == 0) {
    s->ev[0] = EvInfo{};
    s->ev[1] = EvInfo{};
    s->ev[0].n_words = uint32_t(n);
    s->status = 0;
  }
  for (int32_t c = tid; c < (nchunks > 0 ? nchunks : 1); c += stride) {  // n = 0 keeps one empty chunk
    s->chunk_wo[c] = uint32_t(c) * kChunk;
    s->chunk_nw[c] = nchunks == 0 ? 0u : ((c + 1 < nchunks) ? kChunk : uint32_t(n) - uint32_t(c) * kChunk);
    s->chunk_nmod[c] = 0;
  }
  for (int32_t i = tid; i < n; i += stride) clus[i] = i + 1;
}

std::mutex g_mu;
NoAllocScratch* g_addr[kMaxDevices] = {};

}  // namespace

}  // namespace pxl

extern "C" int32_t pxl_clusterize_digis_noalloc(const uint16_t* id, const int16_t* x, const int16_t* y,
                                                const int32_t* adc, int32_t n, int32_t apply_charge_cut,
                                                uint32_t* module_start, uint32_t* clus_in_module, uint32_t* module_id,
                                                int32_t* clus, uint16_t* id_out, void* stream) {
  using namespace pxl;
  if (n < 0 || (n > 0 && (!id || !x || !y || !adc || !clus || !id_out)) || !module_start || !clus_in_module ||
      !module_id)
    return PXL_ERR_ARG;
  if (n > kNoAllocMaxDigis) {
    std::fprintf(stderr, "pxl_clusterize_digis_noalloc: %d digis exceed the fixed scratch limit of %d per call\n", n,
                 kNoAllocMaxDigis);
    return PXL_ERR_CAPACITY;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PXL_ERR_CUDA;
  NoAllocScratch* s = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
      void* p = nullptr;
      const cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (err != cudaSuccess || !p) {
        std::fprintf(stderr, "pxl_clusterize_digis_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(err));
        return PXL_ERR_CUDA;
      }
      g_addr[dev] = static_cast<NoAllocScratch*>(p);
    }
    s = g_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the scratch address is the current device's: a stream of another device would run the
  // kernels there with this device's address
  if (st) {
    int sdev = -1;
    if (cudaStreamGetDevice(st, &sdev) != cudaSuccess) return PXL_ERR_CUDA;
    if (sdev != dev) return PXL_ERR_ARG;
  }
  const int32_t nchunks = int32_t((uint32_t(n) + kChunk - 1) / kChunk);
  if (n > 0 && cudaMemcpyAsync(id_out, id, size_t(n) * sizeof(uint16_t), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return PXL_ERR_CUDA;
  k_noalloc_init<<<148, 256, 0, st>>>(s, n, clus);
  Dev d{};
  d.E = 1;
  d.n_fed_slots = nchunks > 0 ? nchunks : 1;
  d.cap_words = kNoAllocMaxDigis;
  d.hits_per_event = 48 * 1024;
  d.apply_charge_cut = apply_charge_cut != 0;
  d.ev = s->ev;
  d.fed_nw = s->chunk_nw;
  d.fed_wo = s->chunk_wo;
  d.fed_nmod = s->chunk_nmod;
  d.status = &s->status;
  d.id_seen = s->id_seen;
  d.mid = reinterpret_cast<int16_t*>(id_out);
  d.xx = const_cast<int16_t*>(x);
  d.yy = const_cast<int16_t*>(y);
  d.adc = const_cast<int32_t*>(adc);
  d.clus = clus;
  d.module_start = module_start;
  d.clus_in_module = clus_in_module;
  d.module_id = module_id;
  d.clus_module_start = s->clus_module_start;
  d.big_list = s->big_list;
  d.cap_big = kMaxNumModules;
  d.bpe = 148 * 4;
  Launch L{st, d.bpe, 256};
  launch_modstart(d, L);
  launch_cluster(d, L);
  return cudaGetLastError() == cudaSuccess ? 0 : PXL_ERR_CUDA;
}
