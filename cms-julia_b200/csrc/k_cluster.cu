// Per-module clustering fused with the cluster charge cut, and the hit module
// starts. Restates gpu_clustering.jl:94-266 (find_clus),
// gpu_cluster_charge_cut.jl:14-104 and SiPixelRawToClusterGPUKernel.jl:739-752
// (fill_hits_module_start).
//
// find_clus labels 8-connected pixel components by iterated min-propagation,
// which makes every pixel's root the smallest digi index of its component and
// numbers clusters by ascending root. Here each module is one CTA: pixels are
// binned by column in shared memory, components are merged with a lock-free
// union-find that always hooks the larger root under the smaller one (so the
// final root is again the smallest index), and roots are numbered with a
// block scan in index order: the same cluster ids as the reference.
#include "pxl_internal.cuh"

namespace pxl {

namespace {

constexpr int kNPix = 4096;  // >= 4001, the largest range find_clus processes
constexpr int kNBins = 418;

__device__ __forceinline__ int cc_find(volatile int32_t* lab, int x) {
  int p = lab[x];
  while (p != x) { x = p; p = lab[x]; }
  return x;
}

__device__ __forceinline__ void cc_union(int32_t* lab, int a, int b) {
  volatile int32_t* vl = lab;
  while (true) {
    a = cc_find(vl, a);
    b = cc_find(vl, b);
    if (a == b) return;
    if (a < b) { int t = a; a = b; b = t; }
    int old = atomicCAS(&lab[a], a, b);
    if (old == a) return;
    a = old;
  }
}

__global__ void __launch_bounds__(256) k_find_clus(Dev d) {
  const int e = blockIdx.y;
  __shared__ int16_t s_x[kNPix];
  __shared__ int16_t s_y[kNPix];
  __shared__ int32_t s_lab[kNPix];
  __shared__ uint16_t s_sorted[kNPix];
  __shared__ uint32_t s_start[kNBins + 2];
  __shared__ uint32_t s_cur[kNBins + 2];
  __shared__ uint32_t sh[33];
  __shared__ int32_t s_crun;
  __shared__ uint32_t s_warn;
  int32_t* s_charge = reinterpret_cast<int32_t*>(s_x);   // after labelling: [1024]
  uint16_t* s_newc = reinterpret_cast<uint16_t*>(s_y);   // after labelling: [1024]

  const EvInfo& E = d.ev[e];
  const uint32_t nmod = E.n_modules;
  const uint32_t n_el = E.n_words;
  const uint64_t eb = E.word_base;
  if (eb + n_el > uint64_t(d.cap_words)) return;
  const uint32_t* ms = d.module_start + size_t(e) * (kMaxNumModules + 1);

  for (uint32_t m = blockIdx.x; m < nmod; m += gridDim.x) {
    const uint32_t first1 = ms[m + 1];  // 1-based
    const int16_t this_id = d.mid[eb + first1 - 1];
    // msize as the reference derives it (1-based, exclusive end + 1)
    uint32_t msize = (m + 1 < nmod) ? ms[m + 2] : n_el;
    if (first1 < 1 || first1 > n_el || msize < first1 || msize > n_el) continue;  // malformed module list
    if (threadIdx.x == 0) { s_warn = 0; s_crun = 0x7fffffff; }
    if (msize - first1 > uint32_t(kMaxPixInModule)) {
      msize = uint32_t(kMaxPixInModule) + first1;
      if (threadIdx.x == 0) s_warn |= kWarnPixels;
    }
    if (msize == n_el && d.mid[eb + msize - 1] == this_id) msize += 1;
    const int n = int(msize - first1);  // range [first1-1, first1-1+n)
    const uint64_t g0 = eb + first1 - 1;
    for (int b = threadIdx.x; b < kNBins + 2; b += blockDim.x) s_start[b] = 0;
    __syncthreads();
    // load and count by column (bin = (y & 511) + 1)
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const int16_t id = d.mid[g0 + k];
      const int16_t x = d.xx[g0 + k], y = d.yy[g0 + k];
      // a column past the 418-bin histogram makes the reference's histogram assert fail;
      // such a digi is flagged and kept out of the clustering
      const bool in_hist = (uint32_t(uint16_t(y)) & 511u) + 2u <= uint32_t(kNBins);
      if (id != int16_t(kInvId) && !in_hist) atomicOr(&s_warn, kWarnPixels);
      const bool valid = id != int16_t(kInvId) && in_hist;
      s_x[k] = x; s_y[k] = y;
      s_lab[k] = valid ? k : -1;
      if (valid) atomicAdd(&s_start[(uint32_t(uint16_t(y)) & 511u) + 1u], 1u);
      else atomicMin(&s_crun, k);
    }
    __syncthreads();
    // exclusive scan of the bin counts (420 entries, two per thread)
    {
      uint32_t a = 0, b2 = 0;
      int i0 = 2 * threadIdx.x;
      if (i0 < kNBins + 2) a = s_start[i0];
      if (i0 + 1 < kNBins + 2) b2 = s_start[i0 + 1];
      uint32_t tot;
      uint32_t ex = block_excl_scan(a + b2, sh, &tot);
      if (i0 < kNBins + 2) { s_start[i0] = ex; s_cur[i0] = ex; }
      if (i0 + 1 < kNBins + 2) { s_start[i0 + 1] = ex + a; s_cur[i0 + 1] = ex + a; }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      if (s_lab[k] < 0) continue;
      uint32_t bn = (uint32_t(uint16_t(s_y[k])) & 511u) + 1u;
      uint32_t pos = atomicAdd(&s_cur[bn], 1u);
      s_sorted[pos] = uint16_t(k);
    }
    __syncthreads();
    // neighbours: same column (later index) and next column, |dx| <= 1
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      if (s_lab[k] < 0) continue;
      const int16_t xk = s_x[k], yk = s_y[k];
      const uint32_t bn = (uint32_t(uint16_t(yk)) & 511u) + 1u;
      const uint32_t p1 = s_start[bn + 2 <= kNBins + 1 ? bn + 2 : kNBins + 1];
      for (uint32_t p = s_start[bn]; p < p1; ++p) {
        const int mm = s_sorted[p];
        if (mm == k) continue;
        const int16_t ym = s_y[mm];
        if (ym == yk && mm < k) continue;  // each same-column pair once
        const int dx = int(s_x[mm]) - int(xk);
        if (dx > 1 || dx < -1) continue;
        cc_union(s_lab, k, mm);
      }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x)
      if (s_lab[k] >= 0) s_lab[k] = cc_find(s_lab, k);
    __syncthreads();
    // number roots in index order
    uint32_t carry = 0;
    for (int b = 0; b < n; b += blockDim.x) {
      int k = b + threadIdx.x;
      bool root = k < n && s_lab[k] == k;
      uint32_t tot;
      uint32_t ex = block_excl_scan(root ? 1u : 0u, sh, &tot);
      if (root) s_sorted[k] = uint16_t(carry + ex + 1);
      carry += tot;
    }
    __syncthreads();
    const uint32_t nclus = carry;
    const int crun = s_crun < n ? s_crun : n;  // charge sums stop at the first invalid digi
    // cluster_charge_cut
    uint32_t nclus_eff = nclus;
    if (nclus > uint32_t(kMaxClustersPerModule)) {
      nclus_eff = kMaxClustersPerModule;
      if (threadIdx.x == 0) s_warn |= kWarnClusters;
    }
    for (int c = threadIdx.x; c < kMaxClustersPerModule; c += blockDim.x) s_charge[c] = 0;
    __syncthreads();
    if (nclus > 0) {
      for (int k = threadIdx.x; k < crun; k += blockDim.x) {
        uint32_t cl = s_sorted[s_lab[k]];
        if (cl <= nclus_eff) atomicAdd(&s_charge[cl - 1], d.adc[g0 + k]);
      }
    }
    __syncthreads();
    const int32_t cut = this_id < 96 ? 2000 : 4000;
    uint32_t last_new = 0;
    {
      uint32_t c2 = 0;
      for (int b = 0; b < int(nclus_eff); b += blockDim.x) {
        int c = b + threadIdx.x;
        uint32_t ok = (c < int(nclus_eff) && s_charge[c] > cut) ? 1u : 0u;
        uint32_t tot;
        uint32_t ex = block_excl_scan(ok, sh, &tot);
        if (c < int(nclus_eff)) s_newc[c] = ok ? uint16_t(c2 + ex + 1) : uint16_t(kInvId);
        c2 += tot;
      }
      last_new = c2;
    }
    __syncthreads();
    const bool changed = d.apply_charge_cut && nclus_eff > 0 && last_new != nclus_eff;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const uint64_t g = g0 + k;
      if (s_lab[k] < 0) { d.clus[g] = -9999; continue; }
      uint32_t cl = s_sorted[s_lab[k]];
      if (d.apply_charge_cut && nclus > uint32_t(kMaxClustersPerModule) && k < crun && cl > uint32_t(kMaxClustersPerModule)) {
        d.clus[g] = int32_t(kInvId);
        d.mid[g] = int16_t(kInvId);
        continue;
      }
      if (changed && cl <= nclus_eff) {
        uint16_t nc = s_newc[cl - 1];
        d.clus[g] = int32_t(nc);
        if (nc == kInvId) d.mid[g] = int16_t(kInvId);
      } else {
        d.clus[g] = int32_t(cl);
      }
    }
    if (threadIdx.x == 0) {
      d.module_id[size_t(e) * kMaxNumModules + m] = uint32_t(uint16_t(this_id));
      if (uint16_t(this_id) < uint16_t(kMaxNumModules))
        d.clus_in_module[size_t(e) * kMaxNumModules + uint16_t(this_id)] = changed ? last_new : nclus;
      if (s_warn) atomic_or_warn(&d.ev[e], s_warn);
    }
    __syncthreads();
  }
}

// fill_hits_module_start + nClusters, one block per event
__global__ void k_hits_module_start(Dev d) {
  const int e = blockIdx.x;
  __shared__ uint32_t sh[33];
  const uint32_t* cim = d.clus_in_module + size_t(e) * kMaxNumModules;
  uint32_t* cms = d.clus_module_start + size_t(e) * (kMaxNumModules + 1);
  const uint32_t cap = d.hits_per_event;
  uint32_t carry = 0;
  bool clamped = false;
  for (int b = 0; b < kMaxNumModules; b += blockDim.x) {
    int i = b + threadIdx.x;
    uint32_t v = i < kMaxNumModules ? (cim[i] < 1024u ? cim[i] : 1024u) : 0u;
    uint32_t tot;
    uint32_t ex = block_excl_scan(v, sh, &tot);
    if (i < kMaxNumModules) {
      uint32_t inc = carry + ex + v;
      if (inc > cap) { inc = cap; clamped = true; }
      cms[i + 1] = inc;
    }
    carry += tot;
  }
  if (threadIdx.x == 0) cms[0] = 0;
  __syncthreads();
  if (clamped) atomic_or_warn(&d.ev[e], kWarnHitsClamped);
  if (threadIdx.x == 0) {
    uint32_t nc = cms[kMaxNumModules - 1];
    d.ev[e].n_clusters = nc;
    d.ev[e].n_hits = nc;
  }
}

}  // namespace

void launch_cluster(const Dev& d, const Launch& L) {
  dim3 g(L.bpe > 0 ? L.bpe : 64, d.E);
  k_find_clus<<<g, 256, 0, L.s>>>(d);
  L.mark("find_clus_charge_cut");
  k_hits_module_start<<<d.E, 1024, 0, L.s>>>(d);
  L.mark("hits_module_start");
}

}  // namespace pxl
