// Cellular automaton: doublets, outer-hit lists, cell connection, fishbone,
// ntuplet search, cell -> track lists, early duplicate removal and tuple
// multiplicity. Restates gpu_pixel_doublets.jl:19-360 (doublets_from_histo),
// gpu_ca_cell.jl:130-270, gpu_fishbone.jl:4-63, circle_eq.jl:18-93 and
// ca_hit_ntuplet_generator_kernels_impl.jl:45-211.
//
// Output order equals the serial reference's: doublets are counted per work item
// (inner hit x layer pair), scanned and written in the reference's loop order (so
// doublet ids are the reference's ids); per-key lists (cells ending on a hit,
// neighbours of a cell, tracks of a cell) are filled with atomics at the offsets of a
// shifted scan and then sorted, which restores the reference's push order (ascending
// producer index); tuples are counted per start cell, scanned, and written in the
// reference's depth-first order, so tuple ids match too. The doublet and connection
// tests lay their (item, candidate) and (cell, candidate) pairs end to end over the
// lanes of a warp, so that lanes stay busy whatever the candidate counts; the tuple
// walks run from per-warp queues of the start cells that walk, one tree per lane.
#include <algorithm>
#include <cstddef>

#include "pxl_internal.cuh"

namespace pxl {

namespace {

__constant__ uint8_t c_layer_pairs[2 * kNPairs] = {0, 1, 0, 4, 0, 7, 1, 2, 1, 4, 1, 7, 4, 5, 7, 8, 2, 3, 2, 4,
                                                   2, 7, 5, 6, 8, 9, 0, 2, 1, 3, 0, 5, 0, 8, 4, 6, 7, 9};
__constant__ int16_t c_phi_cuts[kNPairs] = {522, 730, 730, 522, 626, 626, 522, 522, 626, 626,
                                            626, 522, 522, 522, 522, 522, 522, 522, 522};
__constant__ double c_min_z[kNPairs] = {-20., 0., -30., -22., 10., -30., -70., -70., -22., 15.,
                                        -30., -70., -70., -20., -22., 0., -30., -70., -70.};
__constant__ double c_max_z[kNPairs] = {20., 30., 0., 22., 30., -10., 70., 70., 22., 30.,
                                        -15., 70., 70., 20., 22., 30., 0., 70., 70.};
__constant__ float c_max_rf[kNPairs] = {20.f, 9.f, 9.f, 20.f, 7.f, 7.f, 5.f, 5.f, 20.f, 6.f, 6.f,
                                        5.f, 5.f, 20.f, 20.f, 9.f, 9.f, 9.f, 9.f};

// CA parameters (ca_hit_ntuplet_generator.jl:9-30), Float32 as Params stores them
__device__ __forceinline__ float ptmin_f() { return 0.899999976158f; }
constexpr float kThetaBarrel = 0.00200000009499f;
constexpr float kThetaForward = 0.00300000002608f;
constexpr float kHardCurv = 0.0328407224959f;
constexpr float kDcaInner = 0.15000000596f;
constexpr float kDcaOuter = 0.25f;

__device__ __forceinline__ uint32_t phi_bin(int16_t t) { return (uint32_t(int32_t(t >> 9)) & 127u) + 1u; }

struct HitView {
  const float *xg, *yg, *zg, *rg;
  const int16_t *iphi, *ysize, *detind;
};

// ---------------------------------------------------------------- doublets
// per event: cumulative inner-layer sizes over the pairs, number of work items
__global__ void k_items(Dev d, uint32_t* pair_cum) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.E) return;
  const uint32_t* hls = d.hits_layer_start + size_t(e) * 11;
  uint32_t acc = 0;
  for (int p = 0; p < kNPairs; ++p) {
    const int li = c_layer_pairs[2 * p];
    acc += hls[li + 1] - hls[li];
    pair_cum[size_t(e) * kNPairs + p] = acc;
  }
  d.ev[e].n_items = d.ev[e].n_hits ? acc : 0u;
}

// layer pair and event-local 0-based inner hit of work item j
__device__ __forceinline__ int item_pair(uint32_t j, const uint32_t* cum, const uint32_t* hls, uint32_t* hit) {
  int pid = 0;
  while (j >= cum[pid]) ++pid;
  *hit = ((pid == 0) ? j : j - cum[pid - 1]) + hls[c_layer_pairs[2 * pid]];
  return pid;
}

// Inner-hit part of one work item (inner hit x layer pair): the inner-hit cuts and the
// outer-layer candidates of the phi window, the bins kl .. kh-1 (wrapping after 128) in the
// reference's loop order, which are at most two contiguous ranges of the binned hits.
struct ItemHead {
  float z, r;
  int16_t iphi, ysize, cut;
  uint8_t pid, ok;
  uint32_t hit;             // event-local 0-based inner hit
  uint32_t lo0, n0, lo1;    // candidates: [lo0, lo0 + n0) then [lo1, lo1 + n - n0)
  uint32_t n;
};

__device__ __forceinline__ ItemHead item_head(uint32_t j, const uint32_t* cum, const uint32_t* hls, const HitView& hv,
                                              const uint32_t* poff) {
  ItemHead h{};
  uint32_t i;
  const int pid = item_pair(j, cum, hls, &i);
  h.pid = uint8_t(pid);
  h.hit = i;
  const int inner = c_layer_pairs[2 * pid], outer = c_layer_pairs[2 * pid + 1];
  if (hv.detind[i] > 2000) return h;
  const float me_z = hv.zg[i];
  if (double(me_z) < c_min_z[pid] || double(me_z) > c_max_z[pid]) return h;
  const int32_t me_s = hv.ysize[i];  // idealConditions: every ladder is an outer ladder
  if ((inner == 0 && outer > 3) && (me_s > 0 && me_s < 36)) return h;
  if ((inner == 1 && outer > 3) && (me_s > 0 && me_s < 28)) return h;
  h.ok = 1;
  h.z = me_z;
  h.r = hv.rg[i];
  h.iphi = hv.iphi[i];
  h.ysize = int16_t(me_s);
  h.cut = c_phi_cuts[pid];
  const uint32_t h_off = 128u * uint32_t(outer);
  const uint32_t kl = phi_bin(int16_t(h.iphi - h.cut));
  uint32_t kh = phi_bin(int16_t(h.iphi + h.cut)) + 1;
  if (kh == 129) kh = 1;
  if (kl == kh) return h;
  if (kl < kh) {
    h.lo0 = poff[kl + h_off - 1];
    h.n0 = poff[kh - 1 + h_off] - h.lo0;
    h.lo1 = 0;
    h.n = h.n0;
  } else {
    h.lo0 = poff[kl + h_off - 1];
    h.n0 = poff[128 + h_off] - h.lo0;
    h.lo1 = poff[h_off];
    h.n = h.n0 + (poff[kh - 1 + h_off] - h.lo1);
  }
  return h;
}

// The same item for the count pass, over the binned records sorted by iphi (as uint16) within
// each bin: its candidates are exactly the outer hits that pass the reference's dphi cut
// (|int16(iphi_o - iphi_i)| <= cut), i.e. the part of bin kl from iphi - cut on, the bins
// between, and the part of the last bin up to iphi + cut (two binary searches in the edge bins),
// as at most two ranges when the window wraps past bin 128. The window (2 cut + 1 < 2^15) never
// covers all 128 bins, the reference's kl == kh case.
__device__ __forceinline__ ItemHead item_head_s(uint32_t j, const uint32_t* cum, const uint32_t* hls,
                                                const HitView& hv, const uint32_t* poff, const uint16_t* __restrict__ us) {
  ItemHead h = item_head(j, cum, hls, hv, poff);
  if (!h.ok || h.n == 0) return h;
  const int outer = c_layer_pairs[2 * h.pid + 1];
  const uint32_t h_off = 128u * uint32_t(outer);
  const uint16_t lo_u = uint16_t(h.iphi - h.cut), hi_u = uint16_t(h.iphi + h.cut);
  const uint32_t kl = (uint32_t(lo_u) >> 9) + 1u, km = (uint32_t(hi_u) >> 9) + 1u;  // first, last bin
  uint32_t a = poff[kl - 1 + h_off], ae = poff[kl + h_off];
  while (a < ae) {  // first entry of bin kl at or above lo_u
    const uint32_t m = (a + ae) >> 1;
    if (us[m] < lo_u) a = m + 1; else ae = m;
  }
  uint32_t b = poff[km - 1 + h_off], be = poff[km + h_off];
  while (b < be) {  // one past the last entry of bin km at or below hi_u
    const uint32_t m = (b + be) >> 1;
    if (us[m] <= hi_u) b = m + 1; else be = m;
  }
  if (kl <= km) {
    h.lo0 = a;
    h.n0 = b - a;
    h.lo1 = 0;
    h.n = h.n0;
  } else {
    h.lo0 = a;
    h.n0 = poff[128 + h_off] - a;
    h.lo1 = poff[h_off];
    h.n = h.n0 + (b - h.lo1);
  }
  return h;
}

// The outer-hit cuts of one candidate (gpu_pixel_doublets.jl), in the reference's order:
// doublet_pass_a takes the module, z0 and dphi cuts (about a quarter of the candidates pass),
// doublet_pass_b the cluster-size and pt cuts. c_max_r holds small integers, so the float
// comparison with them equals the reference's Float64 one.
__device__ __forceinline__ bool doublet_pass_a(int pid, float me_z, float me_r, int16_t me_p, int16_t cut,
                                               const HitRec& hr) {
  if (hr.det() > 2000) return false;
  const float dr = __fsub_rn(hr.r, me_r);
  if (dr > c_max_rf[pid] || dr < 0 ||
      fabsf(__fsub_rn(__fmul_rn(me_z, hr.r), __fmul_rn(me_r, hr.z))) > __fmul_rn(12.f, dr))
    return false;
  const int16_t dphi = int16_t(hr.iphi - me_p);
  const int16_t i_dphi = int16_t(dphi < 0 ? -dphi : dphi);
  return i_dphi <= cut;
}

__device__ __forceinline__ bool doublet_pass_b(int pid, float me_z, float me_r, int16_t me_p, int32_t me_s,
                                               const HitRec& hr) {
  const int inner = c_layer_pairs[2 * pid], outer = c_layer_pairs[2 * pid + 1];
  const float dz_dr_fact = float(8 * 0.0285 / 0.015);
  const double min_radius = 0.5 * 87.78;
  const double r2t4 = 4. * min_radius * min_radius;
  const float zo = hr.z, ro = hr.r;
  {  // z_size_cut
    if (outer < 4) {
      const int16_t so = hr.ysize;
      const int dy = inner == 0 ? 28 : 20;
      const int16_t ds = int16_t(so - int16_t(me_s));
      if (me_s > 0 && so > 0 && (ds < 0 ? -int(ds) : int(ds)) > dy) return false;
    } else if (inner < 4 && me_s > 0) {
      const float t = __fmul_rn(fabsf(__fdiv_rn(__fsub_rn(me_z, zo), __fsub_rn(me_r, ro))), dz_dr_fact);
      const double tt = __dadd_rn(double(t), 0.5);
      if (!isfinite(tt)) return false;  // the reference raises (InexactError) here
      const long long pred = (long long)trunc(tt);
      const long long df = (long long)me_s - pred;
      if ((df < 0 ? -df : df) > 20) return false;
    }
  }
  {  // pt_cut
    const int16_t dphi = int16_t(hr.iphi - me_p);
    const int16_t i_dphi = int16_t(dphi < 0 ? -dphi : dphi);
    const double dphi_f = __dmul_rn(double(i_dphi), (2 * 3.141592653589793) / double(1 << 16));
    const float rr = __fmul_rn(me_r, ro);
    const float dd = __fsub_rn(ro, me_r);
    if (__dmul_rn(__dmul_rn(dphi_f, dphi_f), __dsub_rn(r2t4, double(rr))) > double(__fmul_rn(dd, dd))) return false;
  }
  return true;
}

// doublet_pass_a without the dphi cut, for candidates that pass it by construction
__device__ __forceinline__ bool doublet_pass_z(int pid, float me_z, float me_r, const HitRec& hr) {
  if (hr.det() > 2000) return false;
  const float dr = __fsub_rn(hr.r, me_r);
  return !(dr > c_max_rf[pid] || dr < 0 ||
           fabsf(__fsub_rn(__fmul_rn(me_z, hr.r), __fmul_rn(me_r, hr.z))) > __fmul_rn(12.f, dr));
}

// Reference order of a passing outer hit among its item's cells: the window's bins in order
// (bin offset from the item's first bin kl), then decreasing hit id within a bin. A window of
// at most 2 * 730 + 1 iphi units touches at most four 512-unit bins, so the bin offset takes
// bits 21-26 and bits 27-31 stay free for the item's slot in its warp group (kOwnerShift).
constexpr uint32_t kOwnerShift = 27;
static_assert(kHitIdBits + 6 <= kOwnerShift, "bin offset bits");
__device__ __forceinline__ uint32_t cell_order_key(int16_t me_p, int16_t cut, const HitRec& hr) {
  const uint32_t kl = (uint32_t(uint16_t(me_p - cut)) >> 9) + 1u;
  const uint32_t bo = (((uint32_t(uint16_t(hr.iphi)) >> 9) + 1u - kl) & 127u);
  return (bo << kHitIdBits) | ((kMaxHitsPerEvent - 1u) - hr.id());
}
__device__ __forceinline__ uint32_t key_hit(uint32_t key) { return (kMaxHitsPerEvent - 1u) - (key & (kMaxHitsPerEvent - 1u)); }

__device__ __forceinline__ bool doublet_pass(const ItemHead& h, const HitRec& hr) {
  return doublet_pass_a(h.pid, h.z, h.r, h.iphi, h.cut, hr) && doublet_pass_b(h.pid, h.z, h.r, h.iphi, h.ysize, hr);
}

__device__ __forceinline__ uint32_t head_candidate(const ItemHead& h, uint32_t k) {
  return k < h.n0 ? h.lo0 + k : h.lo1 + (k - h.n0);
}

// All doublets of one item written from event-local position cell_pos on (the fill of
// groups whose count pass could not keep their outer hits).
__device__ __forceinline__ void write_item_doublets(const Dev& d, const ItemHead& h, const HitRec* __restrict__ hrec,
                                                    uint64_t cell_pos, uint64_t cell_lo, uint32_t cap, uint32_t hb) {
  if (!h.ok) return;
  uint32_t cnt = 0;
  for (uint32_t k = 0; k < h.n; ++k) {
    const HitRec hr = hrec[head_candidate(h, k)];
    if (!doublet_pass(h, hr)) continue;
    const uint64_t local = cell_pos + cnt;
    if (local < cap) {
      const uint64_t g = cell_lo + local;
      d.cell_inner[g] = h.hit;
      d.cell_outer[g] = hr.id();
      atomicAdd(&d.ohc_cur[hb + hr.id()], 1u);
      d.cell_pair[g] = h.pid;
      d.cell_id[g] = int32_t(local + 1);
      d.cell_used[g] = 0;
      d.cn_cur[g] = 0;
      d.ct_cur[g] = 0;
    }
    ++cnt;
  }
}

constexpr uint32_t kNoPool = 0xffffffffu;
constexpr int kGroupCells = 768;  // outer hits one 32-item group stages in shared memory

// Count pass over groups of 32 consecutive items (one warp). The candidates of the group's
// items are laid end to end and take the first cuts 32 at a time on all lanes; the survivors
// (about a quarter) queue in candidate order and take the remaining cuts on full warps, oldest
// first, so passing candidates come out in the order of the cells (item, then the reference's
// candidate order). Their outer hits are staged in shared memory; the group then takes one
// contiguous range of the pool and copies them there. A group with more than kGroupCells
// doublets, or that finds the pool full, records kNoPool and the fill pass searches again.
constexpr int kDblQueue = 64;

template <bool kQ>
__global__ void __launch_bounds__(256) k_doublets_count(Dev d, const uint32_t* __restrict__ pair_cum, WorkQueue q) {
  __shared__ uint32_t s_cum[kNPairs];
  __shared__ uint32_t s_hls[11];
  __shared__ uint4 s_rng[8][32];   // per compacted item: lo0, n0, lo1, first candidate
  __shared__ uint4 s_geo[8][32];   // per compacted item: z, r (float bits), iphi | cut << 16, pid | ysize << 16
  __shared__ uint16_t s_beg[8][32], s_end[8][32];
  __shared__ uint32_t s_over[8][32];
  __shared__ uint32_t s_q[8][kDblQueue];  // owner << kHitIdBits | candidate
  __shared__ uint32_t s_out[8][kGroupCells];  // owner << kOwnerShift | cell_order_key
  for_each_vblock<kQ>(q, [&](int e, uint32_t bx, uint32_t nbx) {
  const EvInfo& E = d.ev[e];
  const uint32_t n = E.n_items;
  if (n == 0) return;
  if (threadIdx.x < kNPairs) s_cum[threadIdx.x] = pair_cum[size_t(e) * kNPairs + threadIdx.x];
  if (threadIdx.x < 11) s_hls[threadIdx.x] = d.hits_layer_start[size_t(e) * 11 + threadIdx.x];
  __syncthreads();
  const uint32_t hb = E.hit_base;
  HitView hv{d.xg + hb, d.yg + hb, d.zg + hb, d.rg + hb, d.iphi + hb, d.ysize + hb, d.detind + hb};
  const uint32_t* poff = d.phi_off + size_t(e) * kPhiTotBins;
  const HitRec* hrec = d.hit_rec_s + hb;  // sorted by iphi within each bin
  const uint16_t* us = d.hit_u_s + hb;
  const uint32_t ib = E.item_base;
  const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  for (uint32_t j0 = bx * blockDim.x + 32u * w; j0 < n; j0 += nbx * blockDim.x) {
    const uint32_t j = j0 + lane;
    ItemHead h{};
    if (j < n) h = item_head_s(j, s_cum, s_hls, hv, poff, us);
    const uint32_t nc = h.ok ? h.n : 0u;
    // items with candidates, compacted (compact index = rank among them); the candidates
    // of compacted item c start at position ctex
    const uint32_t busy = __ballot_sync(0xffffffffu, nc > 0);
    const uint32_t ci = __popc(busy & lt);
    const uint32_t ctex = warp_incl_scan(nc) - nc;
    const uint32_t total = __shfl_sync(0xffffffffu, ctex + nc, 31);
    if (nc > 0) {
      s_rng[w][ci] = make_uint4(h.lo0, h.n0, h.lo1, ctex);
      s_geo[w][ci] = make_uint4(__float_as_uint(h.z), __float_as_uint(h.r),
                                uint32_t(uint16_t(h.iphi)) | (uint32_t(uint16_t(h.cut)) << 16),
                                uint32_t(h.pid) | (uint32_t(uint16_t(h.ysize)) << 16));
    }
    s_beg[w][lane] = 0; s_end[w][lane] = 0; s_over[w][lane] = 0;
    __syncwarp();
    uint32_t nout = 0, qhead = 0, qtail = 0;
    // remaining cuts on queue entries qhead .. qhead + mm - 1, one per lane, in queue order
    auto stage_b = [&](uint32_t mm) {
      bool pass = false;
      uint32_t o = 0, oi = 0;
      if (lane < mm) {
        const uint32_t v = s_q[w][(qhead + lane) % kDblQueue];
        o = v >> kHitIdBits;
        const uint4 g = s_geo[w][o];
        const HitRec hr = hrec[v & (kMaxHitsPerEvent - 1u)];
        pass = doublet_pass_b(int(g.w & 0xffu), __uint_as_float(g.x), __uint_as_float(g.y), int16_t(g.z & 0xffffu),
                              int16_t(g.w >> 16), hr);
        oi = (o << kOwnerShift) | cell_order_key(int16_t(g.z & 0xffffu), int16_t(g.z >> 16), hr);
      }
      const uint32_t bal = __ballot_sync(0xffffffffu, pass);
      if (pass) {
        const uint32_t pos = nout + __popc(bal & lt);
        if (pos < uint32_t(kGroupCells)) s_out[w][pos] = oi;
        else atomicAdd(&s_over[w][o], 1u);
      }
      nout += __popc(bal);
      qhead += mm;
    };
    int cur = -1;  // compacted item owning the candidate before the step
    for (uint32_t t0 = 0; t0 < total; t0 += 32) {
      const uint32_t starts = __reduce_or_sync(0xffffffffu, (nc > 0 && ctex >= t0 && ctex < t0 + 32u) ? (1u << (ctex - t0)) : 0u);
      const uint32_t t = t0 + lane;
      const uint32_t o = uint32_t(cur + int(__popc(starts & ((2u << lane) - 1u))));
      cur += int(__popc(starts));
      bool pass = false;
      uint32_t p = 0;
      if (t < total) {
        const uint4 rg = s_rng[w][o];
        const uint4 g = s_geo[w][o];
        const uint32_t k = t - rg.w;
        p = k < rg.y ? rg.x + k : rg.z + (k - rg.y);
        pass = doublet_pass_z(int(g.w & 0xffu), __uint_as_float(g.x), __uint_as_float(g.y), hrec[p]);
      }
      const uint32_t bal = __ballot_sync(0xffffffffu, pass);
      if (pass) s_q[w][(qtail + __popc(bal & lt)) % kDblQueue] = (o << kHitIdBits) | p;
      qtail += __popc(bal);
      __syncwarp();
      if (qtail - qhead >= 32) {
        stage_b(32);
        __syncwarp();
      }
    }
    stage_b(qtail - qhead);
    __syncwarp();
    // doublets per item: the staged outputs are in item order, so each item's are one run
    const uint32_t nst = nout < uint32_t(kGroupCells) ? nout : uint32_t(kGroupCells);
    for (uint32_t x = lane; x < nst; x += 32) {
      const uint32_t o = s_out[w][x] >> kOwnerShift;
      if (x == 0 || (s_out[w][x - 1] >> kOwnerShift) != o) s_beg[w][o] = uint16_t(x);
      if (x + 1 == nst || (s_out[w][x + 1] >> kOwnerShift) != o) s_end[w][o] = uint16_t(x + 1);
    }
    __syncwarp();
    const uint32_t cnt = nc > 0 ? s_end[w][ci] - s_beg[w][ci] + s_over[w][ci] : 0u;
    if (j < n) d.item_cnt[ib + j] = cnt;
    uint32_t off = kNoPool;
    if (nout > 0 && nout <= uint32_t(kGroupCells)) {
      uint32_t o = 0;
      if (lane == 0) o = atomicAdd(d.dbl_pool_ctr, nout);
      o = __shfl_sync(0xffffffffu, o, 0);
      if (uint64_t(o) + nout <= uint64_t(d.cap_cells)) off = o;
    }
    // each staged outer hit goes to its place in the reference's cell order, its rank by key
    // among its item's (they came in iphi order within each bin)
    if (off != kNoPool)
      for (uint32_t x = lane; x < nout; x += 32) {
        const uint32_t v = s_out[w][x];
        const uint32_t b0 = s_beg[w][v >> kOwnerShift], b1 = s_end[w][v >> kOwnerShift];
        uint32_t rank = 0;
        for (uint32_t y = b0; y < b1; ++y) rank += s_out[w][y] < v;
        d.dbl_pool[off + b0 + rank] = key_hit(v);
      }
    const uint32_t ex = warp_incl_scan(cnt) - cnt;
    if (j < n) d.item_pool[ib + j] = off == kNoPool ? kNoPool : off + ex;
    __syncwarp();
  }
  });
}

// Fill pass over the same 32-item groups: cells of a group are contiguous, so the warp
// writes them with consecutive lanes on consecutive cells, outer hits from the pool and the
// inner hit, pair and inner z / r of each cell's item from shared memory.
template <bool kQ>
__global__ void __launch_bounds__(256) k_doublets_fill(Dev d, const uint32_t* __restrict__ pair_cum, WorkQueue q) {
  __shared__ uint32_t s_cum[kNPairs];
  __shared__ uint32_t s_hls[11];
  __shared__ uint32_t s_pos[8][33];
  __shared__ uint32_t s_hit[8][32];
  __shared__ uint8_t s_pid[8][32];
  for_each_vblock<kQ>(q, [&](int e, uint32_t bx, uint32_t nbx) {
  const EvInfo& E = d.ev[e];
  const uint32_t n = E.n_items;
  if (n == 0) return;
  if (threadIdx.x < kNPairs) s_cum[threadIdx.x] = pair_cum[size_t(e) * kNPairs + threadIdx.x];
  if (threadIdx.x < 11) s_hls[threadIdx.x] = d.hits_layer_start[size_t(e) * 11 + threadIdx.x];
  __syncthreads();
  const uint32_t hb = E.hit_base;
  HitView hv{d.xg + hb, d.yg + hb, d.zg + hb, d.rg + hb, d.iphi + hb, d.ysize + hb, d.detind + hb};
  const uint32_t* poff = d.phi_off + size_t(e) * kPhiTotBins;
  const HitRec* hrec = d.hit_rec + hb;
  const uint32_t ib = E.item_base;
  // raw positions of the count scan are made local to the event; the event keeps its
  // first n_cells doublets, stored from cell_base on
  const uint32_t raw_lo = d.item_cnt[ib];
  const uint64_t cell_lo = E.cell_base;
  const uint32_t keep = E.n_cells;
  const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  for (uint32_t j0 = bx * blockDim.x + 32u * w; j0 < n; j0 += nbx * blockDim.x) {
    const uint32_t j = j0 + lane;
    const bool valid = j < n;
    const uint32_t pos = valid ? d.item_cnt[ib + j] - raw_lo : 0u;
    const uint32_t cnt = valid ? d.item_cnt[ib + j + 1] - d.item_cnt[ib + j] : 0u;
    const uint32_t pool = valid ? d.item_pool[ib + j] : kNoPool;
    if (__any_sync(0xffffffffu, cnt > 0 && pool == kNoPool)) {
      if (cnt > 0) write_item_doublets(d, item_head(j, s_cum, s_hls, hv, poff), hrec, pos, cell_lo, keep, hb);
      continue;
    }
    const uint32_t inc = warp_incl_scan(cnt);
    const uint32_t total = __shfl_sync(0xffffffffu, inc, 31);
    if (total == 0) continue;
    const uint32_t base = __shfl_sync(0xffffffffu, pos, 0);
    const uint32_t pool0 = __shfl_sync(0xffffffffu, pool, 0);
    uint32_t i = 0;
    const int pid = valid ? item_pair(j, s_cum, s_hls, &i) : 0;
    s_pos[w][lane] = inc - cnt;
    if (cnt > 0) {
      s_hit[w][lane] = i;
      s_pid[w][lane] = uint8_t(pid);
    }
    __syncwarp();
    for (uint32_t x = lane; x < total; x += 32) {
      const uint32_t local = base + x;
      if (local >= keep) break;
      uint32_t a = 0, b = 32;
      while (b - a > 1) {
        const uint32_t m = (a + b) >> 1;
        if (s_pos[w][m] <= x) a = m; else b = m;
      }
      const uint64_t g = cell_lo + local;
      d.cell_inner[g] = s_hit[w][a];
      const uint32_t oh = d.dbl_pool[pool0 + x];
      d.cell_outer[g] = oh;
      atomicAdd(&d.ohc_cur[hb + oh], 1u);  // cells ending on each hit
      d.cell_pair[g] = s_pid[w][a];
      d.cell_id[g] = int32_t(local + 1);
      d.cell_used[g] = 0;
      d.cn_cur[g] = 0;
      d.ct_cur[g] = 0;
    }
    __syncwarp();
  }
  });
}

// per event: cell base, raw and capped counts
__global__ void k_cell_bases(Dev d) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.E) return;
  EvInfo& E = d.ev[e];
  const uint32_t lo = d.item_cnt[E.item_base], hi = d.item_cnt[E.item_base + E.n_items];
  E.n_cols_nb = 0;
  E.n_cols_tr = 0;
  uint32_t n = hi - lo;  // doublets found; the reference keeps the first doublets_per_event
  if (n > d.doublets_per_event) { n = d.doublets_per_event; E.warnings |= kWarnDoublets; }
  E.n_cells = n;
}

// after the event scan of n_cells: events past the buffer are emptied, regions fixed
__global__ void k_cell_regions(Dev d) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e > d.E) return;
  d.ev[e].n_cells_raw = d.ev[e].n_cells;
}

// ---------------------------------------------------------------- outer-hit lists
// cells ending on each hit: slots from the shifted scan of the counts the doublet fill took
constexpr int kOhcUnroll = 4;  // cells (list entries) per thread and step, loads independent

__global__ void k_ohc_fill(Dev d) {
  const int e = blockIdx.y;
  const EvInfo& E = d.ev[e];
  const uint64_t cb = E.cell_base;
  const uint32_t hb = E.hit_base;
  const uint32_t n = E.n_cells, stride = gridDim.x * blockDim.x;
  for (uint32_t k0 = blockIdx.x * blockDim.x + threadIdx.x; k0 < n; k0 += kOhcUnroll * stride) {
    uint32_t o[kOhcUnroll], slot[kOhcUnroll];
#pragma unroll
    for (int u = 0; u < kOhcUnroll; ++u) o[u] = k0 + u * stride < n ? d.cell_outer[cb + k0 + u * stride] : 0xffffffffu;
#pragma unroll
    for (int u = 0; u < kOhcUnroll; ++u)
      if (o[u] != 0xffffffffu) slot[u] = atomicAdd(&d.ohc_cnt[hb + o[u] + 1], 1u);
#pragma unroll
    for (int u = 0; u < kOhcUnroll; ++u)
      if (o[u] != 0xffffffffu) d.ohc_list[slot[u]] = uint32_t(cb + k0 + u * stride);
  }
}

// bitonic sorting network over N values held in registers (indices are compile-time)
template <int N>
__device__ __forceinline__ void bitonic_regs(uint32_t (&v)[N]) {
#pragma unroll
  for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
      for (int i = 0; i < N; ++i) {
        const int l = i ^ j;
        if (l > i) {
          const uint32_t lo = min(v[i], v[l]), hi = max(v[i], v[l]);
          if ((i & k) == 0) { v[i] = lo; v[l] = hi; } else { v[i] = hi; v[l] = lo; }
        }
      }
    }
  }
}

template <int N>
__device__ __forceinline__ void sort_regs(uint32_t* a, uint32_t n) {
  uint32_t v[N];
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = uint32_t(i) < n ? a[i] : 0xffffffffu;  // padding sorts last
  bitonic_regs<N>(v);
#pragma unroll
  for (int i = 0; i < N; ++i)
    if (uint32_t(i) < n) a[i] = v[i];
}

// Sorts a list of at most kMax entries in place with a register network and returns true;
// longer lists are left to k_sort_long (a list kernel keeps the few registers of its largest
// network, which sets its occupancy).
template <int kMax>
__device__ __forceinline__ bool sort_short(uint32_t* a, uint32_t n) {
  if (n < 2) return true;
  if (n <= 4) { sort_regs<4>(a, n); return true; }
  if (n <= 8) { sort_regs<8>(a, n); return true; }
  return false;
}

// sort a short list in place (ascending; entries are ids below 0xffffffff): one load and
// one store per entry through a register network up to 32 entries, insertion sort above
__device__ __forceinline__ void sort_list(uint32_t* a, uint32_t n) {
  if (n < 2) return;
  if (n <= 4) { sort_regs<4>(a, n); return; }
  if (n <= 8) { sort_regs<8>(a, n); return; }
  if (n <= 16) { sort_regs<16>(a, n); return; }
  if (n <= 32) { sort_regs<32>(a, n); return; }
  for (uint32_t p = 1; p < n; ++p) {
    const uint32_t v = a[p];
    uint32_t q = p;
    while (q > 0 && a[q - 1] > v) { a[q] = a[q - 1]; --q; }
    a[q] = v;
  }
}

// per-hit lists (kind 0: cells ending on the hit; 2: tuples through the hit, descending)
// lists above the short-sort limit, sorted afterwards by k_sort_long (a list of n entries
// needs n > 8, so the buffer of cap_long = entries / 9 entries cannot overflow)
__device__ __forceinline__ void push_long_list(const Dev& d, uint32_t lo, uint32_t n) {
  const uint32_t slot = atomicAdd(d.long_ctr, 1u);
  if (slot < uint32_t(d.cap_long)) d.long_lists[slot] = make_uint2(lo, n);
  else atomicOr(d.status, kWarnBuffer);
}

__global__ void __launch_bounds__(256) k_sort_long(Dev d, uint32_t* list) {
  uint32_t nl = *d.long_ctr;
  if (nl > uint32_t(d.cap_long)) nl = uint32_t(d.cap_long);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nl; i += gridDim.x * blockDim.x) {
    const uint2 l = d.long_lists[i];
    sort_list(list + l.x, l.y);
  }
}

template <int kKind>
__global__ void k_sort_hit_lists(Dev d) {
  const int e = blockIdx.y;
  const EvInfo& E = d.ev[e];
  const uint32_t hb = E.hit_base;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < E.n_hits; k += gridDim.x * blockDim.x) {
    const uint32_t h = hb + k;
    if (kKind == 0) {
      const uint32_t lo = d.ohc_cnt[h], hi = d.ohc_cnt[h + 1];
      sort_list(d.ohc_list + lo, hi - lo);
      if (hi - lo > uint32_t(kMaxCellsPerHit)) atomic_or_warn(&d.ev[e], kWarnLists);
    }
  }
}

// ---------------------------------------------------------------- connect
struct CircleEq {
  float xp, yp, c, alpha, beta;
  __device__ CircleEq(float x1, float y1, float x2, float y2, float x3, float y3) {
    const bool no_flip = fabsf(__fsub_rn(x3, x1)) < fabsf(__fsub_rn(y3, y1));
    const float x1p = no_flip ? __fsub_rn(x1, x2) : __fsub_rn(y1, y2);
    const float y1p = no_flip ? __fsub_rn(y1, y2) : __fsub_rn(x1, x2);
    const float d12 = __fadd_rn(__fmul_rn(x1p, x1p), __fmul_rn(y1p, y1p));
    const float x3p = no_flip ? __fsub_rn(x3, x2) : __fsub_rn(y3, y2);
    const float y3p = no_flip ? __fsub_rn(y3, y2) : __fsub_rn(x3, x2);
    const float d32 = __fadd_rn(__fmul_rn(x3p, x3p), __fmul_rn(y3p, y3p));
    const float num = __fsub_rn(__fmul_rn(x1p, y3p), __fmul_rn(y1p, x3p));
    const float det = __fsub_rn(__fmul_rn(d12, y3p), __fmul_rn(d32, y1p));
    const float st2 = __fsub_rn(__fmul_rn(d12, x3p), __fmul_rn(d32, x1p));
    const float seq = __fadd_rn(__fmul_rn(det, det), __fmul_rn(st2, st2));
    float al2 = __fdiv_rn(1.0f, __fsqrt_rn(seq));
    const float be2 = __fmul_rn(-st2, al2);
    const float ct = __fmul_rn(__fmul_rn(2.0f, num), al2);
    al2 = __fmul_rn(al2, det);
    xp = x2; yp = y2;
    c = no_flip ? ct : -ct;
    alpha = no_flip ? al2 : -be2;
    beta = no_flip ? be2 : -al2;
  }
  __device__ float dca0() const {
    const float x = __fadd_rn(__fmul_rn(c, xp), alpha);
    const float y = __fadd_rn(__fmul_rn(c, yp), beta);
    return __fsub_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y))), 1.0f);
  }
};

__device__ __forceinline__ bool are_aligned(float r1, float z1, float ri, float zi, float ro, float zo, float ptmin,
                                            float theta_cut) {
  const float radius_diff = fabsf(__fsub_rn(r1, ro));
  const float dz = __fsub_rn(z1, zo);
  const float d13 = __fadd_rn(__fmul_rn(radius_diff, radius_diff), __fmul_rn(dz, dz));
  const float p_min = __fmul_rn(ptmin, __fsqrt_rn(d13));
  const float t = fabsf(__fadd_rn(__fadd_rn(__fmul_rn(z1, __fsub_rn(ri, ro)), __fmul_rn(zi, __fsub_rn(ro, r1))),
                                  __fmul_rn(zo, __fsub_rn(r1, ri))));
  return __fmul_rn(t, p_min) <= __fmul_rn(__fmul_rn(theta_cut, d13), radius_diff);
}

// connect's candidates of each outer-hit list entry, gathered once per entry
__global__ void __launch_bounds__(256) k_ohc_records(Dev d) {
  const int e = blockIdx.y;
  const EvInfo& E = d.ev[e];
  const uint32_t hb = E.hit_base;
  const uint32_t lo = d.ohc_cnt[hb], hi = d.ohc_cnt[uint64_t(hb) + E.n_hits];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t p0 = lo + blockIdx.x * blockDim.x + threadIdx.x; p0 < hi; p0 += kOhcUnroll * stride) {
    uint32_t ih[kOhcUnroll];
#pragma unroll
    for (int u = 0; u < kOhcUnroll; ++u) ih[u] = p0 + u * stride < hi ? d.ohc_list[p0 + u * stride] : 0xffffffffu;
#pragma unroll
    for (int u = 0; u < kOhcUnroll; ++u)
      if (ih[u] != 0xffffffffu) ih[u] = d.cell_inner[ih[u]];
    float4 h[kOhcUnroll];
    int16_t det[kOhcUnroll];
#pragma unroll
    for (int u = 0; u < kOhcUnroll; ++u)
      if (p0 + u * stride < hi) {
        h[u] = d.hit_xyzr[hb + ih[u]];
        det[u] = d.detind[hb + ih[u]];
      }
#pragma unroll
    for (int u = 0; u < kOhcUnroll; ++u)
      if (p0 + u * stride < hi) d.ohc_rec[p0 + u * stride] = make_float2(det[u] < 96 ? -h[u].w : h[u].w, h[u].z);
  }
}

// Connection test of every cell with the cells ending on its inner hit (the outer-hit list,
// at most kMaxCellsPerHit entries). A warp takes 32 cells and spreads their (cell, candidate)
// pairs over its lanes, 32 pairs per step; the cheap alignment test runs on every pair, and the
// pairs that pass it (a few percent) queue in shared memory for the circle / DCA test, which
// then runs on full warps. A passing pair counts one neighbour of the candidate (cn_cur), sets
// both used flags and goes to the pair list that k_connect_fill turns into neighbour lists; none
// of these depends on the evaluation order.
constexpr int kConnWarps = 8;
constexpr int kConnQueue = 64;

template <bool kQ>
__global__ void __launch_bounds__(256) k_connect_test(Dev d, WorkQueue q) {
  __shared__ float4 s_rz[kConnWarps][32];  // inner r, z and outer r, z of each cell
  __shared__ float4 s_xy[kConnWarps][32];  // inner x, y and outer x, y
  __shared__ uint32_t s_lo[kConnWarps][32];
  __shared__ uint32_t s_ex[kConnWarps][32];
  __shared__ uint8_t s_barrel[kConnWarps][32];
  __shared__ uint16_t s_queue[kConnWarps][kConnQueue];  // pair: owner lane << 8 | candidate
  for_each_vblock<kQ>(q, [&](int e, uint32_t bx, uint32_t nbx) {
  const EvInfo& E = d.ev[e];
  const uint64_t cb = E.cell_base;
  const uint32_t hb = E.hit_base;
  const float4* hxyzr = d.hit_xyzr + hb;
  const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  uint64_t c0 = 0;
  // circle / DCA test of the queued pairs q0 .. q0+31 (lanes past qn idle)
  auto circle_step = [&](uint32_t q0, uint32_t qn) {
    bool cut = false;
    uint32_t o = 0, c = 0;
    if (q0 + lane < qn) {
      const uint32_t v = s_queue[w][q0 + lane];
      const uint32_t a = v >> 8, j = v & 0xffu;
      const uint32_t p = s_lo[w][a] + j;
      const float4 xy = s_xy[w][a];
      const float region = signbit(d.ohc_rec[p].x) ? kDcaInner : kDcaOuter;
      const float4 h1 = hxyzr[d.cell_inner[d.ohc_list[p]]];  // the candidate's inner hit
      const CircleEq eq(h1.x, h1.y, xy.x, xy.y, xy.z, xy.w);
      if (eq.c > kHardCurv) cut = false;
      else cut = fabsf(eq.dca0()) < __fmul_rn(region, fabsf(eq.c));
      if (cut) {
        o = d.ohc_list[p];
        c = uint32_t(c0 + a);
      }
    }
    const uint32_t bal = __ballot_sync(0xffffffffu, cut);
    if (bal) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(d.cn_pair_ctr, uint32_t(__popc(bal)));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (cut) {
        const uint32_t slot = base + __popc(bal & lt);
        d.cell_used[o] = 1;
        d.cell_used[c] = 1;
        if (slot < uint32_t(d.cap_pairs)) {
          d.cn_pairs[slot] = make_uint2(o, c);
          atomicAdd(&d.cn_cur[o], 1u);
        } else {
          atomicOr(d.status, kWarnBuffer);
        }
      }
    }
  };
  for (uint32_t k0 = bx * blockDim.x + 32u * w; k0 < E.n_cells; k0 += nbx * blockDim.x) {
    const uint32_t k = k0 + lane;
    c0 = cb + k0;
    const uint64_t c = cb + k;
    uint32_t n = 0;
    if (k < E.n_cells) {
      const uint32_t ih = d.cell_inner[c];
      const uint32_t lo = d.ohc_cnt[hb + ih];
      n = d.ohc_cnt[hb + ih + 1] - lo;
      if (n > uint32_t(kMaxCellsPerHit)) n = kMaxCellsPerHit;
      if (n > 0) {  // geometry only for cells with candidates
        const uint32_t oh = d.cell_outer[c];
        const float4 hi = hxyzr[ih], ho = hxyzr[oh];
        s_lo[w][lane] = lo;
        s_rz[w][lane] = make_float4(hi.w, hi.z, ho.w, ho.z);
        s_xy[w][lane] = make_float4(hi.x, hi.y, ho.x, ho.y);
        s_barrel[w][lane] = d.detind[hb + ih] < 1184 ? 1 : 0;
      }
    }
    const uint32_t inc = warp_incl_scan(n);
    const uint32_t total = __shfl_sync(0xffffffffu, inc, 31);
    s_ex[w][lane] = inc - n;
    __syncwarp();
    uint32_t qn = 0;
    uint32_t a = 0;  // owner of this lane's pair, non-decreasing over the steps
    for (uint32_t x0 = 0; x0 < total; x0 += 32) {
      const uint32_t x = x0 + lane;
      bool al = false;
      uint32_t j = 0;
      if (x < total) {
        while (a < 31 && s_ex[w][a + 1] <= x) ++a;
        j = x - s_ex[w][a];
        const float2 rec = d.ohc_rec[s_lo[w][a] + j];  // the candidate's inner hit: r (sign: inner barrel), z
        const float4 rz = s_rz[w][a];
        al = are_aligned(fabsf(rec.x), rec.y, rz.x, rz.y, rz.z, rz.w, ptmin_f(), s_barrel[w][a] ? kThetaBarrel : kThetaForward);
      }
      const uint32_t bal = __ballot_sync(0xffffffffu, al);
      if (al) s_queue[w][qn + __popc(bal & lt)] = uint16_t((a << 8) | j);
      qn += __popc(bal);
      __syncwarp();
      if (qn >= 32) {
        qn -= 32;
        circle_step(qn, qn + 32);
        __syncwarp();
      }
    }
    circle_step(0, qn);
    __syncwarp();
  }
  });
}

// neighbour lists from the pair list: each passing (candidate o, cell c) appends c to o's list
__global__ void __launch_bounds__(256) k_connect_fill(Dev d) {
  uint32_t np = *d.cn_pair_ctr;
  if (np > uint32_t(d.cap_pairs)) np = uint32_t(d.cap_pairs);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    const uint2 pc = d.cn_pairs[i];
    d.cn_list[atomicAdd(&d.cn_cnt[pc.x + 1], 1u)] = pc.y;
  }
}

// per-cell lists: neighbours (kind 0) or tracks (kind 1), sorted ascending; flags overflow
template <int kKind>
__global__ void k_sort_cell_lists(Dev d) {
  const int e = blockIdx.y;
  const EvInfo& E = d.ev[e];
  const uint64_t cb = E.cell_base;
  __shared__ uint32_t s_cols;
  if (threadIdx.x == 0) s_cols = 0;
  __syncthreads();
  uint32_t cols = 0;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < E.n_cells; k += gridDim.x * blockDim.x) {
    const uint64_t c = cb + k;
    const uint32_t* cnt = kKind == 0 ? d.cn_cnt : d.ct_cnt;
    uint32_t* list = kKind == 0 ? d.cn_list : d.ct_list;
    const uint32_t lo = cnt[c];
    uint32_t hi = cnt[c + 1];
    const uint64_t lcap = uint64_t(kKind == 0 ? d.cap_pairs : d.cap_tuple_hits);
    if (uint64_t(hi) > lcap) hi = uint32_t(lcap);
    if (hi > lo) {
      ++cols;
      if (!sort_short<8>(list + lo, hi - lo)) push_long_list(d, lo, hi - lo);
      if (hi - lo > uint32_t(kCellRows)) atomic_or_warn(&d.ev[e], kWarnLists);
    }
    // cells with two or more tracks, for the duplicate remover
    if (kKind == 1 && cnt[c + 1] - cnt[c] >= 2) atomicOr(&d.dup_bits[c >> 5], 1u << (c & 31));
  }
  if (cols) atomicAdd(&s_cols, cols);
  __syncthreads();
  if (threadIdx.x == 0 && s_cols) {
    // columns of the fixed column store: one per cell with a non-empty list plus the reserved one
    uint32_t* counter = kKind == 0 ? &d.ev[e].n_cols_nb : &d.ev[e].n_cols_tr;
    const uint32_t before = atomicAdd(counter, s_cols);
    if (before + s_cols + 1 > d.columns_per_event) atomic_or_warn(&d.ev[e], kWarnColumns);
  }
}

// ---------------------------------------------------------------- fishbone
template <bool kQ>
__global__ void __launch_bounds__(128) k_fishbone(Dev d, WorkQueue q) {
  for_each_vblock<kQ>(q, [&](int e, uint32_t bx, uint32_t nbx) {
  const EvInfo& E = d.ev[e];
  if (E.n_hits <= 1) return;
  const uint32_t hb = E.hit_base;
  const float* xg = d.xg + hb;
  const float* yg = d.yg + hb;
  const float* zg = d.zg + hb;
  const int16_t* det = d.detind + hb;
  for (uint32_t k = bx * blockDim.x + threadIdx.x; k < E.n_hits; k += nbx * blockDim.x) {
    const uint32_t lo = d.ohc_cnt[hb + k];
    uint32_t n = d.ohc_cnt[hb + k + 1] - lo;
    if (n < 2) continue;
    if (n > uint32_t(kMaxCellsPerHit)) n = kMaxCellsPerHit;
    const uint32_t* L = d.ohc_list + lo;
    const float xo = xg[k], yo = yg[k], zo = zg[k];
    // the cells that carry a neighbour relation, in list order
    float dx[kMaxCellsPerHit], dy[kMaxCellsPerHit], dz[kMaxCellsPerHit], nrm[kMaxCellsPerHit];
    uint16_t idet[kMaxCellsPerHit];
    uint8_t idx[kMaxCellsPerHit];
    // gathered kFishBatch entries at a time: each stage's loads are independent of one
    // another, so a batch waits for four load latencies rather than four per entry
    constexpr int kFishBatch = 8;
    uint32_t curr = 0;
    for (uint32_t j0 = 0; j0 < n; j0 += kFishBatch) {
      uint32_t cb8[kFishBatch], ih8[kFishBatch];
      bool used[kFishBatch];
#pragma unroll
      for (int i = 0; i < kFishBatch; ++i) cb8[i] = j0 + i < n ? L[j0 + i] : 0u;
#pragma unroll
      for (int i = 0; i < kFishBatch; ++i) used[i] = j0 + i < n && d.cell_used[cb8[i]] != 0;
#pragma unroll
      for (int i = 0; i < kFishBatch; ++i) ih8[i] = used[i] ? d.cell_inner[cb8[i]] : 0u;
#pragma unroll
      for (int i = 0; i < kFishBatch; ++i) {
        if (!used[i]) continue;
        const float4 hi = d.hit_xyzr[hb + ih8[i]];
        idx[curr] = uint8_t(j0 + i);
        idet[curr] = uint16_t(det[ih8[i]]);
        dx[curr] = __fsub_rn(hi.x, xo);
        dy[curr] = __fsub_rn(hi.y, yo);
        dz[curr] = __fsub_rn(hi.z, zo);
        nrm[curr] = __fadd_rn(__fadd_rn(__fmul_rn(dx[curr], dx[curr]), __fmul_rn(dy[curr], dy[curr])),
                              __fmul_rn(dz[curr], dz[curr]));
        ++curr;
      }
    }
    if (curr < 2) continue;
    for (uint32_t ic = 0; ic + 1 < curr; ++ic) {
      for (uint32_t jc = ic + 1; jc < curr; ++jc) {
        const float cos12 = __fadd_rn(__fadd_rn(__fmul_rn(dx[ic], dx[jc]), __fmul_rn(dy[ic], dy[jc])),
                                      __fmul_rn(dz[ic], dz[jc]));
        if (idet[ic] != idet[jc] &&
            __fmul_rn(cos12, cos12) >= __fmul_rn(__fmul_rn(0.99999f, nrm[ic]), nrm[jc])) {
          if (nrm[ic] > nrm[jc]) { d.cell_id[L[idx[ic]]] = -1; break; }
          d.cell_id[L[idx[jc]]] = -1;
        }
      }
    }
  }
  });
}

// ---------------------------------------------------------------- ntuplets
constexpr int kMaxDepth = 8;

// Depth-first walk of find_ntuplets from one start cell. kFill == false counts tuples and
// hits and appends each tuple's record (its doublets, and its ordinal and hit offset among the
// start cell's tuples) to part `part` of the record pool; kFill == true writes the tuples from
// the given global tuple / hit positions (run only when the pool overflowed).
template <bool kFill>
__device__ void walk(const Dev& d, uint64_t cb, uint64_t start, uint64_t* tuple_pos, uint64_t* hit_pos,
                     uint32_t* ntup, uint32_t* nhit, uint64_t tuple_lo, uint32_t tcap, int e, uint32_t part) {
  uint32_t stack_c[kMaxDepth];
  uint32_t stack_k[kMaxDepth];
  int depth = 0;
  stack_c[0] = uint32_t(start);
  stack_k[0] = 0;
  bool descended = false;  // whether the current top has an alive neighbour
  bool alive_child[kMaxDepth];
  alive_child[0] = false;
  (void)descended;
  while (depth >= 0) {
    const uint32_t c = stack_c[depth];
    const uint32_t lo = d.cn_cnt[c];
    uint32_t nn = d.cn_cnt[c + 1] - lo;
    if (nn > uint32_t(kCellRows)) nn = kCellRows;
    // entries past the pair buffer were not stored (buffer warning raised by the fill)
    if (uint64_t(lo) + nn > uint64_t(d.cap_pairs)) nn = uint64_t(lo) < uint64_t(d.cap_pairs) ? uint32_t(d.cap_pairs - lo) : 0u;
    bool pushed = false;
    while (stack_k[depth] < nn) {
      const uint32_t o = d.cn_list[lo + stack_k[depth]];
      stack_k[depth]++;
      if (d.cell_id[o] < 0) continue;  // killed by the fishbone
      alive_child[depth] = true;
      if (depth + 1 >= kMaxDepth) { atomic_or_warn(&d.ev[e], kWarnTuples); continue; }
      ++depth;
      stack_c[depth] = o;
      stack_k[depth] = 0;
      alive_child[depth] = false;
      pushed = true;
      break;
    }
    if (pushed) continue;
    // all neighbours of the top visited
    if (!alive_child[depth] && depth >= 1) {
      const uint32_t nh = uint32_t(depth) + 2;  // doublets on the stack + 1
      if (kFill) {
        const uint64_t g = *tuple_pos;
        const uint64_t hp = *hit_pos;
        if (g < uint64_t(d.cap_tuples) && hp + nh <= uint64_t(d.cap_tuple_hits)) {
          d.tuple_off[g] = uint32_t(hp);
          const uint32_t hbase = d.ev[e].hit_base;
          for (int k = 0; k <= depth; ++k) {
            const uint32_t ih = d.cell_inner[stack_c[k]];
            d.tuple_hits[hp + k] = ih;
            d.tuple_det[hp + k] = uint16_t(d.detind[hbase + ih]);
          }
          const uint32_t oh = d.cell_outer[stack_c[depth]];
          d.tuple_hits[hp + depth + 1] = oh;
          d.tuple_det[hp + depth + 1] = uint16_t(d.detind[hbase + oh]);
          d.quality[g] = 0;
          // cell -> track pairs, only for the tuples kept (the event's n_tuples: the
          // reference's cap, or none when the event is past the batch buffers), so that
          // the counts equal the entries k_cell_tracks_fill writes
          if (g - tuple_lo < tcap) {
            const uint64_t pp = hp - g;  // sum over earlier tuples of (hits - 1)
            for (int k = 0; k <= depth; ++k) {
              d.tuple_cell[pp + k] = stack_c[k];
              atomicAdd(&d.ct_cur[stack_c[k]], 1u);
            }
          }
        }
        *tuple_pos = g + 1;
        *hit_pos = hp + nh;
      } else {
        // the tuple's record, appended to the warp's part of the pool
        const uint32_t slot = atomicAdd(&d.tp_ctr[part * kTpStride], 1u);
        if (slot < d.tp_part) {
          const uint64_t r = uint64_t(part) * d.tp_part + slot;
          uint32_t cc[kMaxDepth];
#pragma unroll
          for (int k = 0; k < kMaxDepth; ++k) cc[k] = k <= depth ? stack_c[k] : 0u;
          d.tp_hdr[r] = make_uint4(uint32_t(start), *ntup, *nhit, (uint32_t(e) << 4) | nh);
          d.tp_cells[2 * r] = make_uint4(cc[0], cc[1], cc[2], cc[3]);
          d.tp_cells[2 * r + 1] = make_uint4(cc[4], cc[5], cc[6], cc[7]);
        } else {
          d.tp_ctr[kTpParts * kTpStride] = 1u;  // the fill walks again
        }
        *ntup += 1;
        *nhit += nh;
      }
    }
    --depth;
  }
  (void)cb;
}

__device__ __forceinline__ bool is_start(const Dev& d, uint64_t c) {
  if (d.cell_id[c] < 0) return false;
  const int p = d.cell_pair[c];
  return p < 8 || p > 12;  // minHitsPerNtuplet = 3 (…_impl.jl:125)
}

// Thread per walk: a warp looks at 32 cells at a time and queues in shared memory the
// ones that start a walk (count pass: start cells with at least one neighbour; fill pass:
// start cells the count pass gave tuples), then walks 32 queued cells at once, so that
// every lane of a walking warp has a tree to walk. The count pass writes zero for the
// cells it does not walk; the fill takes each walk's positions from the scanned counts,
// so the order of the walks does not matter.
constexpr int kNtupWarps = 4;
constexpr int kNtupQueue = 64;

template <bool kFill, bool kQ>
__global__ void __launch_bounds__(32 * kNtupWarps) k_ntuplets(Dev d, WorkQueue q) {
  __shared__ uint32_t s_queue[kNtupWarps][kNtupQueue];
  // the fill walks only when the count pass could not keep every tuple's record
  if (kFill && d.tp_ctr[kTpParts * kTpStride] == 0) return;
  const uint32_t part = ((blockIdx.y * gridDim.x + blockIdx.x) * kNtupWarps + (threadIdx.x >> 5)) % kTpParts;
  for_each_vblock<kQ>(q, [&](int e, uint32_t bx, uint32_t nbx) {
  const EvInfo& E = d.ev[e];
  const uint64_t cb = E.cell_base;
  const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const uint32_t ncell = E.n_cells;
  const uint64_t tuple_lo = kFill && ncell > 0 ? d.tstart_cnt[cb] >> 32 : 0;
  // walks the queued cells q0 .. qn (at most 32; lanes past qn idle)
  auto walk_queued = [&](uint32_t q0, uint32_t qn) {
    if (q0 + lane >= qn) return;
    const uint64_t c = cb + s_queue[w][q0 + lane];
    if (!kFill) {
      uint32_t nt = 0, nh = 0;
      walk<false>(d, cb, c, nullptr, nullptr, &nt, &nh, 0, 0, e, part);
      d.tstart_cnt[c] = (uint64_t(nt) << 32) | nh;
    } else {
      const uint64_t v = d.tstart_cnt[c];
      uint64_t tp = v >> 32, hp = v & 0xFFFFFFFFull;
      walk<true>(d, cb, c, &tp, &hp, nullptr, nullptr, tuple_lo, E.n_tuples, e, 0u);
    }
  };
  uint32_t qn = 0;
  for (uint32_t k0 = bx * blockDim.x + 32u * w; k0 < ncell; k0 += nbx * blockDim.x) {
    const uint32_t k = k0 + lane;
    bool walker = false;
    if (k < ncell) {
      const uint64_t c = cb + k;
      if (is_start(d, c)) {
        if (!kFill) walker = d.cn_cnt[c + 1] > d.cn_cnt[c];
        else walker = (d.tstart_cnt[c + 1] >> 32) != (d.tstart_cnt[c] >> 32);
      }
      if (!kFill && !walker) d.tstart_cnt[c] = 0;
    }
    const unsigned b = __ballot_sync(0xffffffffu, walker);
    if (walker) s_queue[w][qn + __popc(b & lt)] = k;
    qn += __popc(b);
    __syncwarp();
    if (qn >= 32) {
      qn -= 32;
      walk_queued(qn, qn + 32);
      __syncwarp();
    }
  }
  walk_queued(0, qn);
  __syncwarp();
  });
}

// The fill from the pool: two blocks per part r move its records to their tuple and hit
// positions (the start cell's scanned positions plus the record's ordinal and hit offset) and
// write what the walking fill writes at a leaf. Independent records, one thread each, so the
// gathers of the tuples' hits overlap; nothing is walked again.
constexpr int kPoolBlocksPerPart = 2;  // measured faster than one (1000 PU50 events: 1.01 / 1.05 ms)

__global__ void __launch_bounds__(256) k_tuples_from_pool(Dev d) {
  if (d.tp_ctr[kTpParts * kTpStride]) return;  // a part overflowed: k_ntuplets<true> walks
  const uint32_t r = blockIdx.x / kPoolBlocksPerPart;
  uint32_t n = d.tp_ctr[r * kTpStride];
  if (n > d.tp_part) n = d.tp_part;
  for (uint32_t i = threadIdx.x + (blockIdx.x % kPoolBlocksPerPart) * blockDim.x; i < n;
       i += kPoolBlocksPerPart * blockDim.x) {
    const uint64_t s = uint64_t(r) * d.tp_part + i;
    const uint4 h = d.tp_hdr[s];
    const uint4 c0 = d.tp_cells[2 * s], c1 = d.tp_cells[2 * s + 1];
    const uint32_t cells[kMaxDepth] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
    const int e = int(h.w >> 4);
    const uint32_t nh = h.w & 15u;
    const int depth = int(nh) - 2;  // index of the tuple's last doublet
    const uint64_t v = d.tstart_cnt[h.x];
    const uint64_t g = (v >> 32) + h.y;
    const uint64_t hp = (v & 0xFFFFFFFFull) + h.z;
    if (!(g < uint64_t(d.cap_tuples) && hp + nh <= uint64_t(d.cap_tuple_hits))) continue;
    const EvInfo& E = d.ev[e];
    const uint32_t hbase = E.hit_base;
    uint32_t ih[kMaxDepth];
    uint32_t top = 0;
#pragma unroll
    for (int k = 0; k < kMaxDepth; ++k) {
      ih[k] = k <= depth ? d.cell_inner[cells[k]] : 0u;
      if (k == depth) top = cells[k];
    }
    const uint32_t oh = d.cell_outer[top];
    int16_t det[kMaxDepth];
#pragma unroll
    for (int k = 0; k < kMaxDepth; ++k)
      if (k <= depth) det[k] = d.detind[hbase + ih[k]];
    const int16_t det_o = d.detind[hbase + oh];
    d.tuple_off[g] = uint32_t(hp);
#pragma unroll
    for (int k = 0; k < kMaxDepth; ++k)
      if (k <= depth) {
        d.tuple_hits[hp + k] = ih[k];
        d.tuple_det[hp + k] = uint16_t(det[k]);
      }
    d.tuple_hits[hp + depth + 1] = oh;
    d.tuple_det[hp + depth + 1] = uint16_t(det_o);
    d.quality[g] = 0;
    // cell -> track pairs only for the tuples the event keeps (as the walking fill)
    if (g - E.tuple_base < E.n_tuples) {
      const uint64_t pp = hp - g;
#pragma unroll
      for (int k = 0; k < kMaxDepth; ++k)
        if (k <= depth) {
          d.tuple_cell[pp + k] = cells[k];
          atomicAdd(&d.ct_cur[cells[k]], 1u);
        }
    }
  }
}

__global__ void k_tuple_bases(Dev d) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e > d.E) return;
  if (e == d.E) {
    const uint64_t v = d.tstart_cnt[d.ev[d.E].n_cells_raw];
    d.ev[e].n_tuples_raw = uint32_t(v >> 32);
    d.ev[e].n_tuple_hits_raw = uint32_t(v);
    d.ev[e].tuple_base = uint32_t(v >> 32);
    d.ev[e].tuple_hit_base = uint32_t(v);
    // the pair list (cell, tuple) holds hits - tuples entries
    d.ev[e].n_dup_cells = 0;
    return;
  }
  EvInfo& E = d.ev[e];
  const uint64_t lo = d.tstart_cnt[E.cell_base], hi = d.tstart_cnt[uint64_t(E.cell_base) + E.n_cells_raw];
  E.tuple_base = uint32_t(lo >> 32);
  E.tuple_hit_base = uint32_t(lo);
  E.n_tuples_raw = uint32_t(hi >> 32) - uint32_t(lo >> 32);
  E.n_tuple_hits_raw = uint32_t(hi) - uint32_t(lo);
  uint32_t nt = E.n_tuples_raw;
  if (nt > d.tuples_per_event) { nt = d.tuples_per_event; E.warnings |= kWarnTuples; }
  if (uint64_t(E.tuple_base) + E.n_tuples_raw > uint64_t(d.cap_tuples) ||
      uint64_t(E.tuple_hit_base) + E.n_tuple_hits_raw > uint64_t(d.cap_tuple_hits)) {
    E.warnings |= kWarnBuffer;
    nt = 0;
  }
  E.n_tuples = nt;
  E.n_dup_cells = 0;
  E.dup_cell_base = 0;
}

// Tuple hit offsets end markers and the live sizes for the per-tuple loops. An event with more
// tuples than it keeps ends as the reference's bulk_finalize_fill leaves an overflowing
// container (hist_to_container.jl:150-161): the offset after the last kept tuple is set to that
// tuple's start, so the last kept tuple shows no hits (its doublets still list it).
__global__ void k_tuple_ends(Dev d) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.E) return;
  EvInfo& E = d.ev[e];
  E.n_tuple_hits = 0;
  E.last_tuple_end = 0;
  const uint64_t tb = E.tuple_base;
  if (tb + E.n_tuples_raw <= uint64_t(d.cap_tuples)) {
    d.tuple_off[tb + E.n_tuples_raw] = E.tuple_hit_base + E.n_tuple_hits_raw;
    const uint32_t nt = E.n_tuples;
    if (nt > 0 && nt < E.n_tuples_raw) {
      E.last_tuple_end = d.tuple_off[tb + nt];
      d.tuple_off[tb + nt] = d.tuple_off[tb + nt - 1];
    }
    // hits of the tuples kept (the first n_tuples)
    E.n_tuple_hits = d.tuple_off[tb + nt] - E.tuple_hit_base;
  }
}

// cell -> tuple lists: fill from the (cell, tuple) pairs of the kept tuples
__global__ void k_cell_tracks_fill(Dev d) {
  const int e = blockIdx.y;
  const EvInfo& E = d.ev[e];
  const uint64_t tb = E.tuple_base;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < E.n_tuples; t += gridDim.x * blockDim.x) {
    const uint64_t g = tb + t;
    // the walk registered every doublet of the last kept tuple, also when its visible size is 0
    const uint32_t h0 = d.tuple_off[g];
    const uint32_t h1 = (t + 1 == E.n_tuples && E.last_tuple_end) ? E.last_tuple_end : d.tuple_off[g + 1];
    const uint64_t pp = uint64_t(h0) - g;
    for (uint32_t k = 0; k + 1 < h1 - h0; ++k) {
      const uint32_t c = d.tuple_cell[pp + k];
      d.ct_list[atomicAdd(&d.ct_cnt[c + 1], 1u)] = uint32_t(g);
    }
  }
}

// kernel_early_duplicate_remover (…_impl.jl:143-166)
__global__ void k_early_dup(Dev d) {
  const int e = blockIdx.y;
  const EvInfo& E = d.ev[e];
  if (E.n_cells == 0) return;
  // only cells with two or more tracks act: walk their bitmap
  const uint64_t c_lo = E.cell_base, c_hi = c_lo + E.n_cells;
  for (uint64_t wi = (c_lo >> 5) + blockIdx.x * blockDim.x + threadIdx.x; wi <= (c_hi - 1) >> 5;
       wi += uint64_t(gridDim.x) * blockDim.x) {
    for (uint32_t bits = dup_word(d, wi, c_lo, c_hi); bits; bits &= bits - 1) {
      const uint64_t c = 32 * wi + uint32_t(__ffs(bits) - 1);
      const uint32_t lo = d.ct_cnt[c];
      uint32_t n = d.ct_cnt[c + 1] - lo;
      if (n > uint32_t(kCellRows)) n = kCellRows;
      uint32_t maxn = 0;
      for (uint32_t j = 0; j < n; ++j) {
        const uint32_t t = d.ct_list[lo + j];
        const uint32_t s = d.tuple_off[t + 1] - d.tuple_off[t];
        maxn = s > maxn ? s : maxn;
      }
      for (uint32_t j = 0; j < n; ++j) {
        const uint32_t t = d.ct_list[lo + j];
        if (d.tuple_off[t + 1] - d.tuple_off[t] != maxn) d.quality[t] = 1;
      }
    }
  }
}

// tuple multiplicity counts (kernel_countMultiplicity + finalize!) per event: offsets after
// kernel_fillMultiplicity are the exclusive prefix over bins 1..8
__global__ void k_multiplicity(Dev d) {
  const int e = blockIdx.x;
  EvInfo& E = d.ev[e];
  __shared__ uint32_t s_cnt[9];
  if (threadIdx.x < 9) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t tb = E.tuple_base;
  for (uint32_t t = threadIdx.x; t < E.n_tuples; t += blockDim.x) {
    const uint64_t g = tb + t;
    const uint32_t n = d.tuple_off[g + 1] - d.tuple_off[g];
    if (n < 3 || d.quality[g] == 1) continue;
    if (n < 9) atomicAdd(&s_cnt[n - 1], 1u);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int b = 0; b < 9; ++b) { E.tm_off[b] = acc; acc += s_cnt[b]; }
    for (int n = 3; n <= 5; ++n)
      if (s_cnt[n - 1] > d.fits_per_mult) E.warnings |= kWarnFitsCapped;
  }
}

}  // namespace

// CTAs of one persistent wave per tunable stage (SMs x resident CTAs of the stage's
// work-queue kernels, the smaller where a stage has two); 0 for the stages without one
int prepare_ca_kernels(int ctas[kTuneCount]) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return -1;
  auto occ = [&](auto kernel, int threads) {
    int n = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, 0) == cudaSuccess ? n : 0;
  };
  for (int s = 0; s < kTuneCount; ++s) ctas[s] = 0;
  ctas[kTuneDoublets] = sms * std::min(occ(k_doublets_count<true>, 256), occ(k_doublets_fill<true>, 256));
  ctas[kTuneConnect] = sms * occ(k_connect_test<true>, 256);
  ctas[kTuneFishbone] = sms * occ(k_fishbone<true>, 128);
  ctas[kTuneNtuplets] = sms * std::min(occ(k_ntuplets<false, true>, 32 * kNtupWarps),
                                       occ(k_ntuplets<true, true>, 32 * kNtupWarps));
  return 0;
}

// a list-sorting kernel followed by the sort of the lists it left long
template <class F>
void launch_sorted(const Dev& d, const Launch& L, uint32_t* list, F&& sort_kernel) {
  cudaMemsetAsync(d.long_ctr, 0, sizeof(uint32_t), L.s);
  sort_kernel(L.s);
  k_sort_long<<<148 * 4, 256, 0, L.s>>>(d, list);
}

void launch_ca(const Dev& d, const Launch& L) {
  auto g = [&](int seg) { return dim3(L.bpe_of(seg), d.E); };
  const int eb = div_up(d.E + 1, 128);
  uint32_t* pair_cum = d.pair_cum;
  // counters of the cells ending on each hit (the per-cell counters are cleared by the
  // doublet fill that writes the cells)
  cudaMemsetAsync(d.ohc_cur, 0, size_t(d.cap_hits) * sizeof(uint32_t), L.s);
  k_items<<<div_up(d.E, 128), 128, 0, L.s>>>(d, pair_cum);
  launch_ev_scan(d, L.s, int(offsetof(EvInfo, n_items)), int(offsetof(EvInfo, item_base)));
  L.mark("doublet_items");
  cudaMemsetAsync(d.dbl_pool_ctr, 0, sizeof(uint32_t), L.s);
  // the per-event stages run on their static grid or from a work queue (Launch::queue_of):
  // virtual blocks of (strides x block size) work units, events by decreasing hit count
  launch_wq_order(d, L.s);
  auto plan = [&](int seg, int count_off, int threads) {
    return launch_wq_plan(d, L, count_off, uint32_t(L.queue_of(seg)) * uint32_t(threads));
  };
  const int ctas_dbl = L.queue_of(kTuneDoublets) ? L.wq_ctas[kTuneDoublets] : 0;
  if (ctas_dbl) {
    const WorkQueue q = plan(kTuneDoublets, int(offsetof(EvInfo, n_items)), 256);
    k_doublets_count<true><<<ctas_dbl, 256, 0, L.s>>>(d, pair_cum, q);
  } else {
    k_doublets_count<false><<<g(kTuneDoublets), 256, 0, L.s>>>(d, pair_cum, WorkQueue{});
  }
  L.mark("doublets_count");
  excl_scan_u32(d.item_cnt, d.cap_items, &d.ev[d.E].n_items, d.scan_tmp, L.s);
  k_cell_bases<<<eb, 128, 0, L.s>>>(d);
  launch_ev_scan(d, L.s, int(offsetof(EvInfo, n_cells)), int(offsetof(EvInfo, cell_base)));
  launch_ev_clamp(d, L.s, int(offsetof(EvInfo, n_cells)), int(offsetof(EvInfo, cell_base)), d.cap_cells);
  k_cell_regions<<<eb, 128, 0, L.s>>>(d);
  L.mark("doublets_scan");
  if (ctas_dbl) {
    const WorkQueue q = plan(kTuneDoublets, int(offsetof(EvInfo, n_items)), 256);
    k_doublets_fill<true><<<ctas_dbl, 256, 0, L.s>>>(d, pair_cum, q);
  } else {
    k_doublets_fill<false><<<g(kTuneDoublets), 256, 0, L.s>>>(d, pair_cum, WorkQueue{});
  }
  L.mark("doublets_fill");
  // cells ending on each hit (counted by the doublet fill)
  excl_scan_shift_u32(d.ohc_cur, d.ohc_cnt, d.cap_hits, &d.ev[d.E].n_hits, d.scan_tmp, L.s);
  k_ohc_fill<<<g(kTuneHitLists), 256, 0, L.s>>>(d);
  k_sort_hit_lists<0><<<g(kTuneHitLists), 256, 0, L.s>>>(d);
  k_ohc_records<<<g(kTuneHitLists), 256, 0, L.s>>>(d);
  L.mark("outer_hit_lists");
  // connection and neighbour lists
  cudaMemsetAsync(d.cn_pair_ctr, 0, sizeof(uint32_t), L.s);
  if (L.queue_of(kTuneConnect)) {
    const WorkQueue q = plan(kTuneConnect, int(offsetof(EvInfo, n_cells)), 256);
    k_connect_test<true><<<L.wq_ctas[kTuneConnect], 256, 0, L.s>>>(d, q);
  } else {
    k_connect_test<false><<<g(kTuneConnect), 256, 0, L.s>>>(d, WorkQueue{});
  }
  L.mark("connect");
  excl_scan_shift_u32(d.cn_cur, d.cn_cnt, d.cap_cells, &d.ev[d.E].n_cells_raw, d.scan_tmp, L.s);
  k_connect_fill<<<148 * 8, 256, 0, L.s>>>(d);
  launch_sorted(d, L, d.cn_list, [&](cudaStream_t s) { k_sort_cell_lists<0><<<g(kTuneCellLists), 256, 0, s>>>(d); });
  L.mark("neighbour_lists");
  if (L.queue_of(kTuneFishbone)) {
    const WorkQueue q = plan(kTuneFishbone, int(offsetof(EvInfo, n_hits)), 128);
    k_fishbone<true><<<L.wq_ctas[kTuneFishbone], 128, 0, L.s>>>(d, q);
  } else {
    k_fishbone<false><<<g(kTuneFishbone), 128, 0, L.s>>>(d, WorkQueue{});
  }
  L.mark("fishbone");
  // ntuplets: the count pass keeps each tuple's record in the pool; the fill moves the records
  // into place, or walks again when the pool overflowed
  cudaMemsetAsync(d.tp_ctr, 0, size_t(kTpParts * kTpStride + 1) * sizeof(uint32_t), L.s);
  const int ctas_nt = L.queue_of(kTuneNtuplets) ? L.wq_ctas[kTuneNtuplets] : 0;
  if (ctas_nt) {
    const WorkQueue q = plan(kTuneNtuplets, int(offsetof(EvInfo, n_cells)), 32 * kNtupWarps);
    k_ntuplets<false, true><<<ctas_nt, 32 * kNtupWarps, 0, L.s>>>(d, q);
  } else {
    k_ntuplets<false, false><<<g(kTuneNtuplets), 32 * kNtupWarps, 0, L.s>>>(d, WorkQueue{});
  }
  L.mark("ntuplets_count");
  excl_scan_u64(d.tstart_cnt, d.cap_cells, &d.ev[d.E].n_cells_raw, d.scan_tmp64, L.s);
  k_tuple_bases<<<eb, 128, 0, L.s>>>(d);
  k_tuples_from_pool<<<kTpParts * kPoolBlocksPerPart, 256, 0, L.s>>>(d);
  if (ctas_nt) {
    const WorkQueue q = plan(kTuneNtuplets, int(offsetof(EvInfo, n_cells)), 32 * kNtupWarps);
    k_ntuplets<true, true><<<ctas_nt, 32 * kNtupWarps, 0, L.s>>>(d, q);
  } else {
    // the walking fill returns at once unless the pool overflowed: a few blocks per event
    k_ntuplets<true, false><<<dim3(std::min(L.bpe_of(kTuneNtuplets), 8), d.E), 32 * kNtupWarps, 0, L.s>>>(
        d, WorkQueue{});
  }
  k_tuple_ends<<<div_up(d.E, 128), 128, 0, L.s>>>(d);
  L.mark("ntuplets_fill");
  excl_scan_shift_u32(d.ct_cur, d.ct_cnt, d.cap_cells, &d.ev[d.E].n_cells_raw, d.scan_tmp, L.s);
  k_cell_tracks_fill<<<g(kTuneCellTracks), 256, 0, L.s>>>(d);
  cudaMemsetAsync(d.dup_bits, 0, size_t(d.cap_cells / 32 + 2) * sizeof(uint32_t), L.s);
  launch_sorted(d, L, d.ct_list, [&](cudaStream_t s) { k_sort_cell_lists<1><<<g(kTuneCellTracks), 256, 0, s>>>(d); });
  L.mark("cell_tracks");
  k_early_dup<<<g(kTuneEarlyDup), 256, 0, L.s>>>(d);
  k_multiplicity<<<d.E, 256, 0, L.s>>>(d);
  L.mark("dup_multiplicity");
}

}  // namespace pxl
