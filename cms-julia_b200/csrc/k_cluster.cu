// Per-module clustering fused with the cluster charge cut, and the hit module
// starts. Restates gpu_clustering.jl:94-266 (find_clus),
// gpu_cluster_charge_cut.jl:14-104 and SiPixelRawToClusterGPUKernel.jl:739-752
// (fill_hits_module_start).
//
// find_clus labels 8-connected pixel components by iterated min-propagation,
// which makes every pixel's root the smallest digi index of its component and
// numbers clusters by ascending root. Here components are merged with a
// lock-free union-find that always hooks the larger root under the smaller one
// (so the final root is again the smallest index), and roots are numbered by a
// scan in index order: the same cluster ids as the reference.
//
// Three paths share the numbering:
//  * one thread per module for modules of at most 16 digis (about three quarters
//    of them at PU50): neighbour sets as bitmasks, components grown from the
//    smallest digi left, all in registers;
//  * one warp per module for modules of at most kWarpPix digis, from work lists.
//    The warp keeps its digis in registers, finds neighbour pairs by broadcasting
//    every digi (up to 32 digis) or through a column histogram (up to kWarpPix),
//    joins them with the union-find, and scans with ballots;
//  * one CTA per module for larger modules: pixels are binned by column in shared
//    memory and only the same and the next column are searched.
#include <algorithm>

#include "pxl_internal.cuh"

namespace pxl {

namespace {

constexpr int kNPix = 4096;  // >= 4001, the largest range find_clus processes
constexpr int kNBins = 418;
constexpr int kWarpPix = kWarpModulePix;  // digis per module handled by one warp
constexpr int kWarpSlots = kWarpPix / 32;
constexpr int kWarpsPerBlock = 8;

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

// The digi range find_clus assigns to module position m of event e, with the
// reference's msize arithmetic (1-based exclusive end + 1, truncation to
// kMaxPixInModule, +1 for the last module). Returns false for a malformed list.
struct ModRange {
  uint64_t g0;      // first digi (global index)
  int n;            // digis in the range
  int16_t this_id;  // module id of the first digi
  bool truncated;
};

__device__ __forceinline__ bool module_range(const Dev& d, int e, uint32_t m, ModRange& r) {
  const EvInfo& E = d.ev[e];
  const uint32_t nmod = E.n_modules, n_el = E.n_words;
  const uint64_t eb = E.word_base;
  const uint32_t* ms = d.module_start + size_t(e) * (kMaxNumModules + 1);
  const uint32_t first1 = ms[m + 1];  // 1-based
  if (first1 < 1 || first1 > n_el) return false;
  r.this_id = d.mid[eb + first1 - 1];
  uint32_t msize = module_end1(d.mid, eb, ms, m, nmod, n_el, first1, r.this_id);
  if (msize < first1 || msize > n_el) return false;
  r.truncated = false;
  if (msize - first1 > uint32_t(kMaxPixInModule)) {
    msize = uint32_t(kMaxPixInModule) + first1;
    r.truncated = true;
  }
  if (msize == n_el && d.mid[eb + msize - 1] == r.this_id) msize += 1;
  r.n = int(msize - first1);  // range [first1-1, first1-1+n)
  r.g0 = eb + first1 - 1;
  return true;
}

// Module positions are clustered in parallel; a module id seen in several runs of one
// event (only malformed data does that) keeps the count of its last run, as the serial
// loop leaves it: the count is stored with its position as the key of an atomicMax
// ((position + 1) << kCountBits | count, count <= 4000) and k_hits_module_start strips the key.
constexpr uint32_t kCountBits = 13;
constexpr uint32_t kCountMask = (1u << kCountBits) - 1u;
__device__ __forceinline__ void write_module_record(const Dev& d, int e, uint32_t m, int16_t this_id, uint32_t nclus,
                                                    uint32_t warn) {
  d.module_id[size_t(e) * kMaxNumModules + m] = uint32_t(uint16_t(this_id));
  if (uint16_t(this_id) < uint16_t(kMaxNumModules))
    atomicMax(&d.clus_in_module[size_t(e) * kMaxNumModules + uint16_t(this_id)], ((m + 1u) << kCountBits) | nclus);
  if (warn) atomic_or_warn(&d.ev[e], warn);
}

// ------------------------------------------------------------ warp per module
constexpr int kHistWords = 448;  // >= 420 column bins, 14 per lane

template <int kSlots>
struct WarpSmem {
  int32_t lab[32 * kSlots];
  int32_t charge[32 * kSlots];
  uint16_t cid[32 * kSlots];   // cluster number (1-based) of each root
  uint16_t newc[32 * kSlots];  // cluster number after the charge cut
};

// column histogram of one module for the larger warp-clustered modules
struct WarpHist {
  uint32_t start[kHistWords];  // first sorted position of each column bin
  uint32_t cur[kHistWords];
  uint32_t xy[kWarpPix];       // x | column bin << 16 of each digi
  uint8_t sorted[kWarpPix];    // digi indices ordered by column bin
};

// One module of at most 32 * kSlots digis, clustered by one warp with its digis in
// registers (kSlots per lane; shared-memory store for up to 32 * kStore digis).
template <int kSlots, int kStore>
__device__ __forceinline__ void cluster_module_warp(const Dev& d, int e, uint32_t m, const ModRange& r,
                                                    WarpSmem<kStore>& S, WarpHist* H) {
  static_assert(kSlots <= kStore, "slots beyond the shared-memory store");
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt = (1u << lane) - 1u;
  const int n = r.n;
  uint32_t xy[kSlots];  // x (16 bits) | column bin << 16; 0xffffffff when not clustered
  int32_t q[kSlots];
  uint32_t warn = 0;
  int crun = n;
#pragma unroll
  for (int j = 0; j < kSlots; ++j) {
    const int k = int(lane) + 32 * j;
    xy[j] = 0xffffffffu;
    q[j] = 0;
    if (k < n) {
      const uint64_t g = r.g0 + k;
      const int16_t id = d.mid[g];
      const int16_t x = d.xx[g], y = d.yy[g];
      q[j] = d.adc[g];
      const uint32_t yb = uint32_t(uint16_t(y)) & 511u;
      // a column past the 418-bin histogram makes the reference's histogram assert
      // fail; such a digi is flagged and kept out of the clustering
      const bool in_hist = yb + 2u <= uint32_t(kNBins);
      if (id != int16_t(kInvId) && !in_hist) warn |= kWarnPixels;
      const bool valid = id != int16_t(kInvId) && in_hist;
      if (valid) xy[j] = uint32_t(uint16_t(x)) | (yb << 16);
      else crun = crun < k ? crun : k;
      S.lab[k] = valid ? k : -1;
    }
  }
  crun = int(__reduce_min_sync(0xffffffffu, uint32_t(crun)));
  warn = __reduce_or_sync(0xffffffffu, warn);
  __syncwarp();
  // histogram path: neighbour pairs (digi indices < 256) listed in the charge / cluster-number
  // store, which is free until the labels are final; pairs past its capacity are joined at once
  uint16_t* pairs = reinterpret_cast<uint16_t*>(S.charge);
  constexpr uint32_t kPairCap = 32u * kStore * (sizeof(int32_t) + 2 * sizeof(uint16_t)) / sizeof(uint16_t);
  uint32_t np = 0;
  if (H) {
    // neighbour pairs through a column histogram (count, warp scan, scatter); each digi
    // then looks at its own and the next column only, as the CTA path does
    for (int w = int(lane); w < kHistWords; w += 32) H->start[w] = 0;
    __syncwarp();
#pragma unroll
    for (int j = 0; j < kSlots; ++j) {
      const int k = int(lane) + 32 * j;
      if (k < n) H->xy[k] = xy[j];
      if (xy[j] != 0xffffffffu) atomicAdd(&H->start[(xy[j] >> 16) + 1u], 1u);
    }
    __syncwarp();
    constexpr int kPer = kHistWords / 32;
    uint32_t cnt[kPer], tot = 0;
#pragma unroll
    for (int w = 0; w < kPer; ++w) { cnt[w] = H->start[lane * kPer + w]; tot += cnt[w]; }
    uint32_t run = warp_incl_scan(tot) - tot;
#pragma unroll
    for (int w = 0; w < kPer; ++w) {
      H->start[lane * kPer + w] = run;
      H->cur[lane * kPer + w] = run;
      run += cnt[w];
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < kSlots; ++j)
      if (xy[j] != 0xffffffffu) H->sorted[atomicAdd(&H->cur[(xy[j] >> 16) + 1u], 1u)] = uint8_t(lane + 32 * j);
    __syncwarp();
    uint32_t& npairs = H->cur[0];  // the scatter cursors are free again
    if (lane == 0) npairs = 0;
    __syncwarp();
#pragma unroll
    for (int j = 0; j < kSlots; ++j) {
      const int k = int(lane) + 32 * j;
      if (k >= n || xy[j] == 0xffffffffu) continue;
      const int xk = int(int16_t(xy[j] & 0xffffu));
      const uint32_t bn = (xy[j] >> 16) + 1u;
      const uint32_t p1 = H->start[bn + 2u];
      for (uint32_t pp = H->start[bn]; pp < p1; ++pp) {
        const int mm = H->sorted[pp];
        if (mm == k) continue;
        const uint32_t vm = H->xy[mm];
        if ((vm >> 16) == (xy[j] >> 16) && mm < k) continue;  // each same-column pair once
        const int dx = int(int16_t(vm & 0xffffu)) - xk;
        if (dx > 1 || dx < -1) continue;
        const uint32_t slot = atomicAdd(&npairs, 1u);
        if (slot < kPairCap) pairs[slot] = uint16_t(k | (mm << 8));
        else cc_union(S.lab, k, mm);
      }
    }
    __syncwarp();
    np = npairs < kPairCap ? npairs : kPairCap;
  } else {
    // neighbour pairs (|dx| <= 1, |dcolumn| <= 1) by broadcasting every digi, each pair
    // once from its smaller index
#pragma unroll
    for (int jb = 0; jb < kSlots; ++jb) {
      const int base = 32 * jb;
      if (base >= n) break;
      const uint32_t v = xy[jb];
      const int tmax = n - base < 32 ? n - base : 32;
      for (int t = 0; t < tmax; ++t) {
        const uint32_t vm = __shfl_sync(0xffffffffu, v, t);
        if (vm == 0xffffffffu) continue;
        const int mm = base + t;
        const int xm = int(int16_t(vm & 0xffffu)), ym = int(vm >> 16);
#pragma unroll
        for (int j = 0; j <= jb; ++j) {
          const int k = int(lane) + 32 * j;
          if (k >= mm || xy[j] == 0xffffffffu) continue;
          const int dx = int(int16_t(xy[j] & 0xffffu)) - xm;
          const int dy = int(xy[j] >> 16) - ym;
          if (dx <= 1 && dx >= -1 && dy <= 1 && dy >= -1) cc_union(S.lab, k, mm);
        }
      }
    }
  }
  // the neighbour pairs, joined 32 at a time (any order gives the same components, each
  // rooted at its smallest digi index)
  for (uint32_t p = lane; p < np; p += 32) cc_union(S.lab, pairs[p] & 0xff, pairs[p] >> 8);
  __syncwarp();
#pragma unroll
  for (int j = 0; j < kSlots; ++j) {
    const int k = int(lane) + 32 * j;
    if (k < n && xy[j] != 0xffffffffu) S.lab[k] = cc_find(S.lab, k);
  }
  __syncwarp();
  // number the roots in index order
  uint32_t nclus = 0;
#pragma unroll
  for (int j = 0; j < kSlots; ++j) {
    const int k = int(lane) + 32 * j;
    if (32 * j >= n) break;
    const bool root = k < n && S.lab[k] == k;
    const unsigned b = __ballot_sync(0xffffffffu, root);
    if (root) S.cid[k] = uint16_t(nclus + __popc(b & lt) + 1);
    nclus += __popc(b);
  }
  for (uint32_t c = lane; c < nclus; c += 32) S.charge[c] = 0;
  __syncwarp();
  // cluster_charge_cut: charge sums stop at the first invalid digi
#pragma unroll
  for (int j = 0; j < kSlots; ++j) {
    const int k = int(lane) + 32 * j;
    if (k < crun) atomicAdd(&S.charge[S.cid[S.lab[k]] - 1], q[j]);
  }
  __syncwarp();
  const int32_t cut = r.this_id < 96 ? 2000 : 4000;
  uint32_t last_new = 0;
  for (uint32_t base = 0; base < nclus; base += 32) {
    const uint32_t c = base + lane;
    const bool ok = c < nclus && S.charge[c] > cut;
    const unsigned b = __ballot_sync(0xffffffffu, ok);
    if (c < nclus) S.newc[c] = ok ? uint16_t(last_new + __popc(b & lt) + 1) : uint16_t(kInvId);
    last_new += __popc(b);
  }
  __syncwarp();
  const bool changed = d.apply_charge_cut && !d.ev[e].repeated_ids && nclus > 0 && last_new != nclus;
#pragma unroll
  for (int j = 0; j < kSlots; ++j) {
    const int k = int(lane) + 32 * j;
    if (k >= n) continue;
    const uint64_t g = r.g0 + k;
    if (xy[j] == 0xffffffffu) { d.clus[g] = -9999; continue; }
    const uint32_t cl = S.cid[S.lab[k]];
    if (changed) {
      const uint16_t nc = S.newc[cl - 1];
      d.clus[g] = int32_t(nc);
      if (nc == kInvId) d.mid[g] = int16_t(kInvId);
    } else {
      d.clus[g] = int32_t(cl);
    }
  }
  if (lane == 0) write_module_record(d, e, m, r.this_id, changed ? last_new : nclus, warn);
  __syncwarp();
}

// every module position of the batch: modules of <= 32 digis here (one digi per lane),
// larger ones to the mid-size list (<= kWarpPix) or the CTA list
// ------------------------------------------------------------ thread per module
constexpr int kThreadPix = 16;  // modules of at most this many digis: one thread each

// One module of at most kThreadPix digis clustered by one thread, all in registers:
// neighbour sets as bitmasks, each component grown from the smallest digi not yet taken,
// so components come out in the order of their smallest index, which numbers them as the
// reference's min-propagation does; the charge cut keeps that order.
__device__ __forceinline__ void cluster_module_thread(const Dev& d, int e, uint32_t m, const ModRange& r) {
  const int n = r.n;
  uint32_t xy[kThreadPix];  // x (16 bits) | column bin << 16
  int32_t q[kThreadPix];
  uint32_t valid = 0, warn = 0;
  int crun = n;
#pragma unroll
  for (int k = 0; k < kThreadPix; ++k) {
    xy[k] = 0;
    q[k] = 0;
    if (k < n) {
      const uint64_t g = r.g0 + k;
      const int16_t id = d.mid[g];
      q[k] = d.adc[g];
      const uint32_t yb = uint32_t(uint16_t(d.yy[g])) & 511u;
      // a column past the 418-bin histogram makes the reference's histogram assert fail;
      // such a digi is flagged and kept out of the clustering
      const bool in_hist = yb + 2u <= uint32_t(kNBins);
      if (id != int16_t(kInvId) && !in_hist) warn |= kWarnPixels;
      if (id != int16_t(kInvId) && in_hist) {
        xy[k] = uint32_t(uint16_t(d.xx[g])) | (yb << 16);
        valid |= 1u << k;
      } else if (k < crun) {
        crun = k;
      }
    }
  }
  // 8-connected neighbours (|dx| <= 1, |dcolumn| <= 1)
  uint32_t adj[kThreadPix];
#pragma unroll
  for (int a = 0; a < kThreadPix; ++a) adj[a] = 0;
#pragma unroll
  for (int a = 0; a < kThreadPix; ++a) {
#pragma unroll
    for (int b = a + 1; b < kThreadPix; ++b) {
      const int dx = int(int16_t(xy[a] & 0xffffu)) - int(int16_t(xy[b] & 0xffffu));
      const int dy = int(xy[a] >> 16) - int(xy[b] >> 16);
      if (((valid >> a) & (valid >> b) & 1u) && dx <= 1 && dx >= -1 && dy <= 1 && dy >= -1) {
        adj[a] |= 1u << b;
        adj[b] |= 1u << a;
      }
    }
  }
  // components in the order of their smallest digi: cluster number (4 bits per digi, 0-based),
  // charge (digis before the first invalid one) and the number after the charge cut
  const int32_t cut = r.this_id < 96 ? 2000 : 4000;
  uint64_t cl_of = 0, new_of = 0;  // 4 bits per digi
  uint32_t removed = 0;            // digis of clusters the cut removes
  uint32_t nclus = 0, kept = 0;
  for (uint32_t rest = valid; rest;) {
    uint32_t comp = rest & (0u - rest);  // the smallest digi left
    for (;;) {
      uint32_t grown = comp;
#pragma unroll
      for (int k = 0; k < kThreadPix; ++k)
        if ((comp >> k) & 1u) grown |= adj[k];
      if (grown == comp) break;
      comp = grown;
    }
    rest &= ~comp;
    int32_t charge = 0;
#pragma unroll
    for (int k = 0; k < kThreadPix; ++k)
      if (((comp >> k) & 1u) && k < crun) charge += q[k];
    const bool ok = charge > cut;
#pragma unroll
    for (int k = 0; k < kThreadPix; ++k)
      if ((comp >> k) & 1u) {
        cl_of |= uint64_t(nclus) << (4 * k);
        new_of |= uint64_t(ok ? kept : 0u) << (4 * k);
      }
    if (!ok) removed |= comp;
    ++nclus;
    if (ok) ++kept;
  }
  const bool changed = d.apply_charge_cut && !d.ev[e].repeated_ids && nclus > 0 && kept != nclus;
#pragma unroll
  for (int k = 0; k < kThreadPix; ++k) {
    if (k >= n) continue;
    const uint64_t g = r.g0 + k;
    if (!((valid >> k) & 1u)) { d.clus[g] = -9999; continue; }
    if (changed) {
      if ((removed >> k) & 1u) {
        d.clus[g] = int32_t(kInvId);
        d.mid[g] = int16_t(kInvId);
      } else {
        d.clus[g] = int32_t((new_of >> (4 * k)) & 15u) + 1;
      }
    } else {
      d.clus[g] = int32_t((cl_of >> (4 * k)) & 15u) + 1;
    }
  }
  write_module_record(d, e, m, r.this_id, changed ? kept : nclus, warn);
}

// every module position of the batch: modules of <= kThreadPix digis here, one thread
// each; larger ones to the work lists of the warp (<= 32, <= kWarpPix digis) and CTA paths
__global__ void __launch_bounds__(128, 6) k_find_clus_tiny(Dev d) {
  const int e = blockIdx.y;
  const EvInfo& E = d.ev[e];
  const uint32_t nmod = E.n_modules;
  if (E.word_base + uint64_t(E.n_words) > uint64_t(d.cap_words)) return;
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < nmod; m += gridDim.x * blockDim.x) {
    ModRange r;
    if (!module_range(d, e, m, r)) continue;
    if (r.n > kThreadPix) {
      push_module(d, r.n > kWarpPix ? kListClusBig : (r.n > 32 ? kListClusMid : kListClusSmall), e, m);
      continue;
    }
    cluster_module_thread(d, e, m, r);
  }
}

// modules of kThreadPix+1 .. 32 digis (work list), one warp each, one digi per lane
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_find_clus_small(Dev d) {
  __shared__ WarpSmem<1> smem[kWarpsPerBlock];
  const unsigned wib = threadIdx.x >> 5;
  const uint32_t nl = list_size(d, kListClusSmall);
  for (uint32_t i = blockIdx.x * kWarpsPerBlock + wib; i < nl; i += gridDim.x * kWarpsPerBlock) {
    const uint32_t v = list_entry(d, kListClusSmall, i);
    const int e = int(v >> 11);
    ModRange r;
    if (!module_range(d, e, v & 2047u, r)) continue;
    cluster_module_warp<1>(d, e, v & 2047u, r, smem[wib], nullptr);
  }
}

// the mid-size modules (33..256 digis), one warp each, eight digis per lane
constexpr int kMidWarps = 4;  // 7.8 KB of shared memory per warp

__global__ void __launch_bounds__(32 * kMidWarps) k_find_clus_mid(Dev d) {
  __shared__ WarpSmem<kWarpSlots> smem[kMidWarps];
  __shared__ WarpHist hist[kMidWarps];
  const unsigned wib = threadIdx.x >> 5;
  const uint32_t nl = list_size(d, kListClusMid);
  for (uint32_t i = blockIdx.x * kMidWarps + wib; i < nl; i += gridDim.x * kMidWarps) {
    const uint32_t v = list_entry(d, kListClusMid, i);
    const int e = int(v >> 11);
    ModRange r;
    if (!module_range(d, e, v & 2047u, r)) continue;
    cluster_module_warp<kWarpSlots>(d, e, v & 2047u, r, smem[wib], &hist[wib]);
  }
}

// ------------------------------------------------------------ CTA per module
struct BlockSmem {
  int16_t x[kNPix];
  int16_t y[kNPix];
  int32_t lab[kNPix];
  uint16_t sorted[kNPix];
  uint32_t start[kNBins + 2];
  uint32_t cur[kNBins + 2];
  uint32_t sh[33];
  int32_t crun;
  uint32_t warn;
};

__device__ void cluster_module_block(const Dev& d, int e, uint32_t m, BlockSmem& S) {
  int32_t* s_charge = reinterpret_cast<int32_t*>(S.x);  // after labelling: [1024]
  uint16_t* s_newc = reinterpret_cast<uint16_t*>(S.y);  // after labelling: [1024]
  ModRange r;
  if (!module_range(d, e, m, r)) return;
  const int n = r.n;
  const uint64_t g0 = r.g0;
  const int16_t this_id = r.this_id;
  if (threadIdx.x == 0) { S.warn = r.truncated ? kWarnPixels : 0u; S.crun = 0x7fffffff; }
  for (int b = threadIdx.x; b < kNBins + 2; b += blockDim.x) S.start[b] = 0;
  __syncthreads();
  // load and count by column (bin = (y & 511) + 1)
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const int16_t id = d.mid[g0 + k];
    const int16_t x = d.xx[g0 + k], y = d.yy[g0 + k];
    const bool in_hist = (uint32_t(uint16_t(y)) & 511u) + 2u <= uint32_t(kNBins);
    if (id != int16_t(kInvId) && !in_hist) atomicOr(&S.warn, kWarnPixels);
    const bool valid = id != int16_t(kInvId) && in_hist;
    S.x[k] = x; S.y[k] = y;
    S.lab[k] = valid ? k : -1;
    if (valid) atomicAdd(&S.start[(uint32_t(uint16_t(y)) & 511u) + 1u], 1u);
    else atomicMin(&S.crun, k);
  }
  __syncthreads();
  // exclusive scan of the bin counts (420 entries, two per thread)
  {
    uint32_t a = 0, b2 = 0;
    int i0 = 2 * threadIdx.x;
    if (i0 < kNBins + 2) a = S.start[i0];
    if (i0 + 1 < kNBins + 2) b2 = S.start[i0 + 1];
    uint32_t tot;
    uint32_t ex = block_excl_scan(a + b2, S.sh, &tot);
    if (i0 < kNBins + 2) { S.start[i0] = ex; S.cur[i0] = ex; }
    if (i0 + 1 < kNBins + 2) { S.start[i0 + 1] = ex + a; S.cur[i0 + 1] = ex + a; }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    if (S.lab[k] < 0) continue;
    uint32_t bn = (uint32_t(uint16_t(S.y[k])) & 511u) + 1u;
    uint32_t pos = atomicAdd(&S.cur[bn], 1u);
    S.sorted[pos] = uint16_t(k);
  }
  __syncthreads();
  // neighbours: same column (later index) and next column, |dx| <= 1
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    if (S.lab[k] < 0) continue;
    const int16_t xk = S.x[k], yk = S.y[k];
    const uint32_t bn = (uint32_t(uint16_t(yk)) & 511u) + 1u;
    const uint32_t p1 = S.start[bn + 2 <= kNBins + 1 ? bn + 2 : kNBins + 1];
    for (uint32_t p = S.start[bn]; p < p1; ++p) {
      const int mm = S.sorted[p];
      if (mm == k) continue;
      const int16_t ym = S.y[mm];
      if (ym == yk && mm < k) continue;  // each same-column pair once
      const int dx = int(S.x[mm]) - int(xk);
      if (dx > 1 || dx < -1) continue;
      cc_union(S.lab, k, mm);
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x)
    if (S.lab[k] >= 0) S.lab[k] = cc_find(S.lab, k);
  __syncthreads();
  // number roots in index order
  uint32_t carry = 0;
  for (int b = 0; b < n; b += blockDim.x) {
    int k = b + threadIdx.x;
    bool root = k < n && S.lab[k] == k;
    uint32_t tot;
    uint32_t ex = block_excl_scan(root ? 1u : 0u, S.sh, &tot);
    if (root) S.sorted[k] = uint16_t(carry + ex + 1);
    carry += tot;
  }
  __syncthreads();
  const uint32_t nclus = carry;
  const int crun = S.crun < n ? S.crun : n;  // charge sums stop at the first invalid digi
  // cluster_charge_cut
  uint32_t nclus_eff = nclus;
  if (nclus > uint32_t(kMaxClustersPerModule)) {
    nclus_eff = kMaxClustersPerModule;
    if (threadIdx.x == 0) S.warn |= kWarnClusters;
  }
  for (int c = threadIdx.x; c < kMaxClustersPerModule; c += blockDim.x) s_charge[c] = 0;
  __syncthreads();
  if (nclus > 0) {
    for (int k = threadIdx.x; k < crun; k += blockDim.x) {
      uint32_t cl = S.sorted[S.lab[k]];
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
      uint32_t ex = block_excl_scan(ok, S.sh, &tot);
      if (c < int(nclus_eff)) s_newc[c] = ok ? uint16_t(c2 + ex + 1) : uint16_t(kInvId);
      c2 += tot;
    }
    last_new = c2;
  }
  __syncthreads();
  const bool cut_here = d.apply_charge_cut && !d.ev[e].repeated_ids;
  const bool changed = cut_here && nclus_eff > 0 && last_new != nclus_eff;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const uint64_t g = g0 + k;
    if (S.lab[k] < 0) { d.clus[g] = -9999; continue; }
    uint32_t cl = S.sorted[S.lab[k]];
    if (cut_here && nclus > uint32_t(kMaxClustersPerModule) && k < crun && cl > uint32_t(kMaxClustersPerModule)) {
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
  __syncthreads();
  if (threadIdx.x == 0) write_module_record(d, e, m, this_id, changed ? last_new : nclus, S.warn);
  __syncthreads();
}

// the modules the warp path handed over: (event << 11 | module position) entries
__global__ void __launch_bounds__(256) k_find_clus_block(Dev d) {
  __shared__ BlockSmem S;
  const uint32_t n = list_size(d, kListClusBig);
  for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
    const uint32_t v = list_entry(d, kListClusBig, i);
    const int e = int(v >> 11);
    const EvInfo& E = d.ev[e];
    if (E.word_base + uint64_t(E.n_words) > uint64_t(d.cap_words)) continue;
    cluster_module_block(d, e, v & 2047u, S);
  }
}

// cluster_charge_cut (gpu_cluster_charge_cut.jl:14-104) in the reference's serial order, for the
// events where a module id starts more than one run: there a run's cut reads the count the id's
// LAST run left (find_clus writes every count first), as changed by the cuts of its earlier
// runs, and the renumbering of cluster ids beyond that count reads the new numbers of the
// module cut before it (the per-event newclusId buffer is never cleared). One warp per event
// walks the runs in order, 32 digis at a time; the fused kernels left these events uncut.
// A cluster id past 1024 in the sums or the renumbering (the reference indexes out of bounds and
// raises) sets the clusters warning and is skipped.
__global__ void __launch_bounds__(32) k_charge_cut_serial(Dev d) {
  const int e = blockIdx.x;
  const EvInfo& E = d.ev[e];
  if (!d.apply_charge_cut || !E.repeated_ids) return;
  if (E.word_base + uint64_t(E.n_words) > uint64_t(d.cap_words)) return;
  __shared__ int32_t s_charge[kMaxClustersPerModule];
  __shared__ uint16_t s_new[kMaxClustersPerModule];
  __shared__ uint8_t s_ok[kMaxClustersPerModule];
  const unsigned lane = threadIdx.x;
  const unsigned lt = (1u << lane) - 1u;
  for (int c = lane; c < kMaxClustersPerModule; c += 32) s_new[c] = 0;  // one buffer per event
  uint32_t* cim = d.clus_in_module + size_t(e) * kMaxNumModules;
  const uint32_t* ms = d.module_start + size_t(e) * (kMaxNumModules + 1);
  const uint64_t eb = E.word_base;
  const uint32_t n_el = E.n_words, nmod = E.n_modules;
  uint32_t warn = 0;
  __syncwarp();
  // first index >= i0 (0-based) whose digi ends the run: any id but this_id (invalid
  // included, the sums' skip test is always false) or, with skip_inv, a valid other id
  for (uint32_t m = 0; m < nmod; ++m) {
    const uint32_t first = ms[m + 1] - 1u;  // 0-based
    if (first >= n_el) continue;
    const int16_t this_id = d.mid[eb + first];
    if (uint16_t(this_id) >= uint16_t(kMaxNumModules)) continue;
    uint32_t nclus = cim[uint16_t(this_id)] & kCountMask;
    if (nclus == 0) continue;
    if (nclus > uint32_t(kMaxClustersPerModule)) {
      for (uint32_t i0 = first; i0 < n_el; i0 += 32) {
        const uint32_t i = i0 + lane;
        const bool stop = i >= n_el || d.mid[eb + i] != this_id;
        const uint32_t sb = __ballot_sync(0xffffffffu, stop);
        const uint32_t end = sb ? uint32_t(__ffs(sb) - 1) : 32u;
        if (lane < end && d.clus[eb + i] > kMaxClustersPerModule) {
          d.mid[eb + i] = int16_t(kInvId);
          d.clus[eb + i] = int32_t(kInvId);
        }
        __syncwarp();
        if (sb) break;
      }
      nclus = kMaxClustersPerModule;
    }
    for (int c = lane; c < kMaxClustersPerModule; c += 32) s_charge[c] = 0;
    __syncwarp();
    for (uint32_t i0 = first; i0 < n_el; i0 += 32) {
      const uint32_t i = i0 + lane;
      const bool stop = i >= n_el || d.mid[eb + i] != this_id;
      const uint32_t sb = __ballot_sync(0xffffffffu, stop);
      const uint32_t end = sb ? uint32_t(__ffs(sb) - 1) : 32u;
      if (lane < end) {
        const int32_t cl = d.clus[eb + i];
        if (cl >= 1 && cl <= kMaxClustersPerModule) atomicAdd(&s_charge[cl - 1], d.adc[eb + i]);
        else warn |= kWarnClusters;
      }
      if (sb) break;
    }
    __syncwarp();
    const int32_t cut = this_id < 96 ? 2000 : 4000;
    uint32_t carry = 0;
    for (uint32_t c0 = 0; c0 < nclus; c0 += 32) {
      const uint32_t c = c0 + lane;
      const bool ok = c < nclus && s_charge[c] > cut;
      const uint32_t b = __ballot_sync(0xffffffffu, ok);
      if (c < nclus) { s_ok[c] = ok; s_new[c] = uint16_t(carry + __popc(b & ((lt << 1) | 1u))); }
      carry += __popc(b);
    }
    __syncwarp();
    if (carry == nclus) continue;  // nClus == newclusId[nClus]
    if (lane == 0) cim[uint16_t(this_id)] = carry;
    for (uint32_t c = lane; c < nclus; c += 32)
      if (!s_ok[c]) s_new[c] = kInvId;
    __syncwarp();
    for (uint32_t i0 = first; i0 < n_el; i0 += 32) {
      const uint32_t i = i0 + lane;
      const int16_t id = i < n_el ? d.mid[eb + i] : int16_t(0);
      const bool stop = i >= n_el || (id != int16_t(kInvId) && id != this_id);
      const uint32_t sb = __ballot_sync(0xffffffffu, stop);
      const uint32_t end = sb ? uint32_t(__ffs(sb) - 1) : 32u;
      if (lane < end && id != int16_t(kInvId)) {
        const int32_t cl = d.clus[eb + i];
        if (cl >= 1 && cl <= kMaxClustersPerModule) {
          const uint16_t nc = s_new[cl - 1];
          d.clus[eb + i] = int32_t(nc);
          if (nc == kInvId) d.mid[eb + i] = int16_t(kInvId);
        } else {
          warn |= kWarnClusters;
        }
      }
      if (sb) break;
    }
    __syncwarp();
  }
  warn = __reduce_or_sync(0xffffffffu, warn);
  if (lane == 0 && warn) atomic_or_warn(&d.ev[e], warn);
}

// fill_hits_module_start + nClusters, one block per event
__global__ void k_hits_module_start(Dev d) {
  const int e = blockIdx.x;
  __shared__ uint32_t sh[33];
  uint32_t* cim = d.clus_in_module + size_t(e) * kMaxNumModules;
  for (int i = threadIdx.x; i < kMaxNumModules; i += blockDim.x) cim[i] &= kCountMask;  // strip the position key
  __syncthreads();
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

// Blocks of k_find_clus_mid that fit on the current device at once: the kernel takes the
// mid-size modules of the work list in one persistent wave (grid-stride), so that no partial
// last wave of long-running blocks is left (1.48 instead of 1.69 ms per 1000 PU50 events with
// 2.3 waves).
static int mid_wave_ctas() {
  static int cached[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148 * 7;
  if (!cached[dev]) {
    int occ = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_find_clus_mid, 32 * kMidWarps, 0) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || occ < 1 || sms < 1) {
      cudaGetLastError();
      return 148 * 7;
    }
    cached[dev] = occ * sms;
  }
  return cached[dev];
}

void launch_cluster(const Dev& d, const Launch& L) {
  cudaMemsetAsync(d.big_list, 0, kListHeader * sizeof(uint32_t), L.s);
  // enough warps that a few events fill the GPU, at least 8 modules per warp otherwise
  // one thread per module position (at most 2000 per event)
  k_find_clus_tiny<<<dim3(div_up(kMaxNumModules, 128), d.E), 128, 0, L.s>>>(d);
  L.mark("find_clus_tiny");
  k_find_clus_small<<<148 * 64, 32 * kWarpsPerBlock, 0, L.s>>>(d);
  L.mark("find_clus_small");
  k_find_clus_mid<<<mid_wave_ctas(), 32 * kMidWarps, 0, L.s>>>(d);
  L.mark("find_clus_mid");
  k_find_clus_block<<<148 * 2, 256, 0, L.s>>>(d);
  L.mark("find_clus_block");
  k_charge_cut_serial<<<d.E, 32, 0, L.s>>>(d);
  k_hits_module_start<<<d.E, 1024, 0, L.s>>>(d);
  L.mark("hits_module_start");
}

}  // namespace pxl
