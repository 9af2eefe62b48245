// Event order and virtual-block plans of the persistent work-queue launches (the
// WorkQueue of pxl_internal.cuh).
#include <cstddef>

#include "pxl_internal.cuh"

namespace pxl {

namespace {

constexpr int kOrderMax = 4096;  // events sorted in one block; larger batches keep event order

// events by decreasing hit count (ties by index): a bitonic sort of (count, index) keys in
// shared memory
__global__ void __launch_bounds__(1024) k_wq_order(const EvInfo* __restrict__ ev, int E, uint32_t* order) {
  __shared__ unsigned long long s_key[kOrderMax];
  if (E > kOrderMax) {
    for (int e = threadIdx.x; e < E; e += blockDim.x) order[e] = uint32_t(e);
    return;
  }
  int n = 1;
  while (n < E) n <<= 1;
  for (int i = threadIdx.x; i < n; i += blockDim.x)  // ascending keys: most hits first, then the lower index
    s_key[i] = i < E ? ((unsigned long long)(0xFFFFFFFFu - ev[i].n_hits) << 32) | uint32_t(i) : ~0ull;
  __syncthreads();
  for (int k = 2; k <= n; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int l = i ^ j;
        if (l > i) {
          const unsigned long long a = s_key[i], b = s_key[l];
          if ((a > b) == ((i & k) == 0)) { s_key[i] = b; s_key[l] = a; }
        }
      }
      __syncthreads();
    }
  for (int i = threadIdx.x; i < E; i += blockDim.x) order[i] = uint32_t(s_key[i] & 0xFFFFFFFFu);
}

// virtual blocks per order slot (ceil(count / units)), their exclusive prefix, and the
// launch's counter cleared; one block
__global__ void __launch_bounds__(1024) k_wq_plan(const EvInfo* __restrict__ ev, int E, const uint32_t* order,
                                                  int count_off, uint32_t units, uint32_t* prefix, uint32_t* head) {
  __shared__ uint32_t sh[33];
  uint32_t carry = 0;
  const char* base = reinterpret_cast<const char*>(ev);
  for (int b = 0; b < E; b += blockDim.x) {
    const int i = b + threadIdx.x;
    uint32_t nb = 0;
    if (i < E) {
      const uint32_t c = *reinterpret_cast<const uint32_t*>(base + size_t(order[i]) * sizeof(EvInfo) + count_off);
      nb = (c + units - 1) / units;
    }
    uint32_t tot;
    const uint32_t ex = block_excl_scan(nb, sh, &tot);
    if (i < E) prefix[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) {
    prefix[E] = carry;
    *head = 0;
  }
}

}  // namespace

void launch_wq_order(const Dev& d, cudaStream_t s) { k_wq_order<<<1, 1024, 0, s>>>(d.ev, d.E, d.wq_order); }

WorkQueue launch_wq_plan(const Dev& d, const Launch& L, int count_off, uint32_t units_per_block) {
  const int slot = L.wq_slot++ % kWqSlots;
  WorkQueue q;
  q.order = d.wq_order;
  q.prefix = d.wq_prefix + size_t(slot) * (size_t(d.E) + 1);
  q.head = d.wq_head + slot;
  q.n = uint32_t(d.E);
  k_wq_plan<<<1, 1024, 0, L.s>>>(d.ev, d.E, d.wq_order, count_off, units_per_block < 1 ? 1u : units_per_block,
                                 const_cast<uint32_t*>(q.prefix), q.head);
  return q;
}

}  // namespace pxl
