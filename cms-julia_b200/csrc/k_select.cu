// Track classification, duplicate cleaning and vertex finding. Restates
// ca_hit_ntuplet_generator_kernels_impl.jl:213-362 (kernel_classify_tracks,
// kernel_fast_duplicate_remover, kernel_count/fill_hit_in_tracks,
// kernel_triplet_cleaner) with the cuts of ca_hit_ntuplet_generator_kernels.jl:79-87,
// and plugin-PixelVertexFinding/gpu_vertex_finder.jl:51-436.
//
// kernel_fast_duplicate_remover is order dependent (a cell sees the marks of the
// cells before it), so it walks the cells in order within an event, one warp per
// event, taking 32 cells at once when they share no track. The triplet cleaner only
// ever writes "dup" and tests "!= bad", so its hits run in parallel. Vertex sums keep
// the reference's track order (one thread per vertex walks its tracks in order).
#include <cstddef>

#include "pxl_internal.cuh"

namespace pxl {

namespace {

constexpr float kChi2Coeff[4] = {0.68177776f, 0.74609577f, -0.08035491f, 0.00315399f};

// kernel_classify_tracks
__global__ void k_classify(Dev d) {
  const int e = blockIdx.y;
  const EvInfo& E = d.ev[e];
  const uint64_t tb = E.tuple_base;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < E.n_tuples; t += gridDim.x * blockDim.x) {
    const uint64_t g = tb + t;
    const uint32_t n = d.tuple_off[g + 1] - d.tuple_off[g];
    if (d.quality[g] == 1) continue;
    if (n < 3) continue;
    const float* st = d.t_state + 5 * g;
    bool nan = false;
    for (int k = 0; k < 5; ++k) nan |= isnan(st[k]);
    if (nan) continue;
    const float ptv = d.t_pt[g];
    const float pt = ptv < 10.0f ? ptv : 10.0f;
    const float cut = __fmul_rn(30.0f, __fadd_rn(kChi2Coeff[0], __fmul_rn(pt, __fadd_rn(kChi2Coeff[1],
                      __fmul_rn(pt, __fadd_rn(kChi2Coeff[2], __fmul_rn(pt, kChi2Coeff[3])))))));
    if (__fmul_rn(3.0f, d.t_chi2[g]) >= cut) continue;
    const bool quad = n > 3;
    const float max_tip = quad ? 0.5f : 0.3f, min_pt = quad ? 0.3f : 0.5f, max_zip = 12.0f;
    if (fabsf(st[1]) < max_tip && ptv > min_pt && fabsf(st[4]) < max_zip) d.quality[g] = 2;
  }
}


// kernel_fast_duplicate_remover: one warp per event, cells in order, qualities in global
// memory; for the events above min_tuples tuples, which the shared-memory form cannot hold
__global__ void k_fast_dup(Dev d, uint32_t min_tuples) {
  const int e = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (e >= d.E) return;
  const unsigned lane = threadIdx.x & 31u;
  const EvInfo& E = d.ev[e];
  if (E.n_cells == 0 || E.n_tuples <= min_tuples) return;
  const uint64_t c_lo = E.cell_base, c_hi = c_lo + E.n_cells;
  for (uint64_t wi = c_lo >> 5; wi <= (c_hi - 1) >> 5; ++wi) {
   uint32_t bits = dup_word(d, wi, c_lo, c_hi);
   while (bits) {
    const uint32_t c = uint32_t(32 * wi) + uint32_t(__ffs(bits) - 1);
    bits &= bits - 1;
    const uint32_t l0 = d.ct_cnt[c];
    uint32_t n = d.ct_cnt[c + 1] - l0;
    if (n > uint32_t(kCellRows)) n = kCellRows;
    // argmin |tip| over the loose tracks, first in list order on ties (strict <, mc = 10000)
    float best = 10000.f;
    uint32_t best_pos = 0xFFFFFFFFu;
    for (uint32_t j = lane; j < n; j += 32) {
      const uint32_t t = d.ct_list[l0 + j];
      if (d.quality[t] == 2) {
        const float s = fabsf(d.t_state[5 * size_t(t) + 1]);
        if (s < best) { best = s; best_pos = j; }
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const float ob = __shfl_down_sync(0xffffffffu, best, o);
      const uint32_t op = __shfl_down_sync(0xffffffffu, best_pos, o);
      if (ob < best || (ob == best && op < best_pos)) { best = ob; best_pos = op; }
    }
    best_pos = __shfl_sync(0xffffffffu, best_pos, 0);
    const uint32_t im = best_pos == 0xFFFFFFFFu ? 0xFFFFFFFFu : d.ct_list[l0 + best_pos];
    __syncwarp();
    for (uint32_t j = lane; j < n; j += 32) {
      const uint32_t t = d.ct_list[l0 + j];
      if (d.quality[t] != 0 && t != im) d.quality[t] = 1;
    }
    __syncwarp();
   }
  }
}

// The same remover with the event's qualities in shared memory: one warp per event
// stages the static part of 32 dup cells at a time (track lists and |tip|) into
// shared memory, then walks the cells in order with shared-memory reads only. The
// argmin takes the smallest |tip| bit pattern (|tip| >= 0 orders as its bits) and,
// among equal ones, the first position: the reference's strict < in list order.
constexpr int kDupMaxTuples = 32768;        // qualities of one event in shared memory (the reference's cap)
constexpr int kDupLargeTuples = 256 * 1024;  // the same for extended-capacity events, 104 KB of shared memory
constexpr int kDupStage = 1024;             // staged track entries per batch of cells

template <int kMaxT>
constexpr size_t dup_smem_bytes() { return 4 * (size_t(kMaxT) / 16 + size_t(kMaxT) / 32 + 2 * kDupStage + 33); }

// qualities (0 bad, 1 dup, 2 loose) packed 2 bits per track, 16 per word
__device__ __forceinline__ uint32_t q_get(const uint32_t* w, uint32_t t) { return (w[t >> 4] >> (2 * (t & 15))) & 3u; }
__device__ __forceinline__ void q_set_dup(uint32_t* w, uint32_t t) {  // any non-bad quality -> dup
  const uint32_t sh = 2 * (t & 15);
  atomicAnd(&w[t >> 4], ~(2u << sh));
  atomicOr(&w[t >> 4], 1u << sh);
}

// The inputs of the ordered walk, gathered with a whole CTA per event: the cells with two
// or more tracks in cell order (from the bitmap), and for each its track entries (at most
// kCellRows) as (event-local tuple id, |tip| bits), laid end to end with offsets.
__global__ void __launch_bounds__(256) k_dup_prep(Dev d) {
  const int e = blockIdx.x;
  EvInfo& E = d.ev[e];
  __shared__ uint32_t sh[33];
  if (E.n_cells == 0 || E.n_tuples > uint32_t(kDupLargeTuples)) {
    if (threadIdx.x == 0) E.n_dup_cells = 0;
    return;
  }
  const uint64_t tb = E.tuple_base;
  const uint64_t c_lo = E.cell_base, c_hi = c_lo + E.n_cells;
  uint32_t* list = d.dup_list + c_lo;
  // cells, in order
  uint32_t ndup = 0;
  for (uint64_t w0 = c_lo >> 5; w0 <= (c_hi - 1) >> 5; w0 += blockDim.x) {
    const uint64_t wi = w0 + threadIdx.x;
    uint32_t bits = wi <= (c_hi - 1) >> 5 ? dup_word(d, wi, c_lo, c_hi) : 0u;
    uint32_t tot;
    uint32_t pos = ndup + block_excl_scan(__popc(bits), sh, &tot);
    for (; bits; bits &= bits - 1) list[pos++] = uint32_t(32 * wi) + uint32_t(__ffs(bits) - 1);
    ndup += tot;
  }
  __syncthreads();
  // entries
  uint32_t* eoff = d.dup_eoff + c_lo + e;
  uint32_t* et = d.dup_et + E.tuple_hit_base;
  uint32_t* ek = d.dup_ek + E.tuple_hit_base;
  uint32_t base = 0;
  for (uint32_t q0 = 0; q0 < ndup; q0 += blockDim.x) {
    const uint32_t q = q0 + threadIdx.x;
    uint32_t n = 0, l0 = 0;
    if (q < ndup) {
      const uint32_t c = list[q];
      l0 = d.ct_cnt[c];
      n = d.ct_cnt[c + 1] - l0;
      if (n > uint32_t(kCellRows)) n = kCellRows;
    }
    uint32_t tot;
    const uint32_t o = base + block_excl_scan(n, sh, &tot);
    if (q < ndup) {
      eoff[q] = o;
      for (uint32_t j = 0; j < n; ++j) {
        const uint32_t t = d.ct_list[l0 + j];
        et[o + j] = uint32_t(t - tb);
        ek[o + j] = __float_as_uint(fabsf(d.t_state[5 * size_t(t) + 1]));
      }
    }
    base += tot;
  }
  if (threadIdx.x == 0) {
    eoff[ndup] = base;
    E.n_dup_cells = ndup;
  }
}

// Events of kMinT < n_tuples <= kMaxT tuples (dynamic shared memory of dup_smem_bytes<kMaxT>()).
template <int kMaxT, int kMinT>
__global__ void __launch_bounds__(32) k_fast_dup_smem(Dev d) {
  extern __shared__ uint32_t s_dup[];
  uint32_t* s_q = s_dup;                          // [kMaxT / 16]
  uint32_t* s_seen = s_q + kMaxT / 16;            // [kMaxT / 32]
  uint32_t* s_t = s_seen + kMaxT / 32;            // [kDupStage]
  uint32_t* s_tip = s_t + kDupStage;              // [kDupStage]
  uint32_t* s_off = s_tip + kDupStage;            // [33]
  const int e = blockIdx.x;
  const unsigned lane = threadIdx.x;
  const EvInfo& E = d.ev[e];
  const uint64_t tb = E.tuple_base;
  const uint32_t nt = E.n_tuples;
  if (nt > uint32_t(kMaxT) || nt <= uint32_t(kMinT)) return;  // another form handles such events
  if (E.n_dup_cells == 0) return;
  const uint32_t nw = (nt + 15) / 16;
  for (uint32_t w = lane; w < nw; w += 32) {
    uint32_t v = 0;
    for (uint32_t k = 0; k < 16; ++k) {
      const uint32_t t = 16 * w + k;
      if (t < nt) v |= uint32_t(d.quality[tb + t] & 3u) << (2 * k);
    }
    s_q[w] = v;
  }
  for (uint32_t w = lane; w < uint32_t(kMaxT / 32); w += 32) s_seen[w] = 0;
  __syncwarp();
  // the event's cells with two or more tracks, in order, and their track entries as
  // k_dup_prep laid them out: offsets (ndup + 1) and (tuple, |tip| bits) per entry
  const uint32_t ndup = E.n_dup_cells;
  const uint32_t* eoff = d.dup_eoff + E.cell_base + e;
  const uint32_t* et = d.dup_et + E.tuple_hit_base;
  const uint32_t* ek = d.dup_ek + E.tuple_hit_base;
  for (uint32_t q0 = 0; q0 < ndup;) {
    // stage up to 32 cells whose entries fit kDupStage
    const uint32_t q = q0 + lane;
    const uint32_t o_lo = eoff[q0];
    const uint32_t o = q <= ndup ? eoff[q] : 0xffffffffu;
    const uint32_t o_next = __shfl_down_sync(0xffffffffu, o, 1);
    const uint32_t o_last = q0 + 32 <= ndup ? eoff[q0 + 32] : 0xffffffffu;
    const uint32_t end = lane == 31 ? o_last : o_next;  // end of cell q's entries
    const bool fits = q < ndup && end - o_lo <= uint32_t(kDupStage);
    const uint32_t ncell = __popc(__ballot_sync(0xffffffffu, fits));
    const uint32_t total = __shfl_sync(0xffffffffu, end, ncell - 1) - o_lo;
    if (lane < ncell) s_off[lane] = o - o_lo;
    if (lane == 0) s_off[ncell] = total;
    for (uint32_t x = lane; x < total; x += 32) {
      s_t[x] = et[o_lo + x];
      s_tip[x] = ek[o_lo + x];
    }
    __syncwarp();
    // cells that share no track are independent: when no track is listed twice in the
    // stage, each lane takes one cell (same result as the ordered walk)
    bool twice = false;
    for (uint32_t x = lane; x < total; x += 32) {
      const uint32_t t = s_t[x], bit = 1u << (t & 31);
      twice |= (atomicOr(&s_seen[t >> 5], bit) & bit) != 0;
    }
    __syncwarp();
    for (uint32_t x = lane; x < total; x += 32) s_seen[s_t[x] >> 5] = 0;
    __syncwarp();
    // |tip| < 10000 as the reference's initial best (mc = 10000, strict <)
    const uint32_t lim = __float_as_uint(10000.f);
    if (!__any_sync(0xffffffffu, twice)) {
      if (lane < ncell) {
        const uint32_t o = s_off[lane], nk = s_off[lane + 1] - o;
        uint32_t best = lim, im = 0xffffffffu;
        for (uint32_t j = 0; j < nk; ++j) {
          const uint32_t t = s_t[o + j];
          const uint32_t key = s_tip[o + j];
          if (key < best && q_get(s_q, t) == 2) { best = key; im = t; }
        }
        for (uint32_t j = 0; j < nk; ++j) {
          const uint32_t t = s_t[o + j];
          if (t != im && q_get(s_q, t) != 0) q_set_dup(s_q, t);
        }
      }
      __syncwarp();
      q0 += ncell;
      continue;
    }
    for (uint32_t k = 0; k < ncell; ++k) {
      const uint32_t o = s_off[k], nk = s_off[k + 1] - o;
      uint32_t key0 = 0xffffffffu, key1 = 0xffffffffu, q0v = 0, q1v = 0;
      uint32_t t0 = 0, t1 = 0;
      if (lane < nk) {
        t0 = s_t[o + lane];
        q0v = q_get(s_q, t0);
        if (q0v == 2) key0 = s_tip[o + lane];
      }
      if (lane + 32 < nk) {
        t1 = s_t[o + lane + 32];
        q1v = q_get(s_q, t1);
        if (q1v == 2) key1 = s_tip[o + lane + 32];
      }
      if (key0 >= lim) key0 = 0xffffffffu;
      if (key1 >= lim) key1 = 0xffffffffu;
      const uint32_t kmin = __reduce_min_sync(0xffffffffu, key0 < key1 ? key0 : key1);
      uint32_t im = 0xffffffffu;
      if (kmin != 0xffffffffu) {
        const uint32_t pos = __reduce_min_sync(0xffffffffu, key0 == kmin ? lane : (key1 == kmin ? lane + 32 : 0xffffffffu));
        im = s_t[o + pos];
      }
      if (lane < nk && q0v != 0 && t0 != im) q_set_dup(s_q, t0);
      if (lane + 32 < nk && q1v != 0 && t1 != im) q_set_dup(s_q, t1);
      __syncwarp();
    }
    q0 += ncell;
  }
  __syncwarp();
  for (uint32_t t = lane; t < nt; t += 32) d.quality[tb + t] = uint8_t(q_get(s_q, t));
}

// hit -> loose tuple lists
template <int kPass>
__global__ void k_hit_to_tuple(Dev d) {
  const int e = blockIdx.y;
  const EvInfo& E = d.ev[e];
  const uint64_t tb = E.tuple_base;
  const uint32_t hb = E.hit_base;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < E.n_tuples; t += gridDim.x * blockDim.x) {
    const uint64_t g = tb + t;
    if (d.quality[g] != 2) continue;
    const uint32_t h0 = d.tuple_off[g], h1 = d.tuple_off[g + 1];
    for (uint32_t p = h0; p < h1; ++p) {
      const uint32_t h = hb + d.tuple_hits[p];
      if (kPass == 0) atomicAdd(&d.htt_cur[h], 1u);
      else d.htt_list[atomicAdd(&d.htt_cnt[h + 1], 1u)] = uint32_t(g);
    }
  }
}

// kernel_triplet_cleaner over hits; lists ordered by decreasing tuple id as the reference fills them
__global__ void k_triplet_cleaner(Dev d) {
  const int e = blockIdx.y;
  const EvInfo& E = d.ev[e];
  const uint32_t hb = E.hit_base;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < E.n_hits; k += gridDim.x * blockDim.x) {
    const uint32_t lo = d.htt_cnt[hb + k], hi = d.htt_cnt[hb + k + 1];
    const uint32_t n = hi - lo;
    uint32_t* L = d.htt_list + lo;
    for (uint32_t p = 1; p < n; ++p) {  // decreasing id
      const uint32_t v = L[p];
      uint32_t q = p;
      while (q > 0 && L[q - 1] < v) { L[q] = L[q - 1]; --q; }
      L[q] = v;
    }
    if (n < 2) continue;
    uint32_t maxnh = 0;
    for (uint32_t j = 0; j < n; ++j) {
      const uint32_t t = L[j];
      const uint32_t s = d.tuple_off[t + 1] - d.tuple_off[t];
      maxnh = s > maxnh ? s : maxnh;
    }
    for (uint32_t j = 0; j < n; ++j) {
      const uint32_t t = L[j];
      if (d.tuple_off[t + 1] - d.tuple_off[t] != maxnh) d.quality[t] = 1;
    }
    if (maxnh > 3) continue;
    float mc = 10000.f;
    uint32_t im = 0xFFFFFFFFu;
    for (uint32_t j = 0; j < n; ++j) {
      const uint32_t t = L[j];
      const float s = fabsf(d.t_state[5 * size_t(t) + 1]);
      if (d.quality[t] != 0 && s < mc) { mc = s; im = t; }
    }
    for (uint32_t j = 0; j < n; ++j) {
      const uint32_t t = L[j];
      if (d.quality[t] != 0 && t != im) d.quality[t] = 1;
    }
  }
}

// ---------------------------------------------------------------- vertices
constexpr int kVtxThreads = 256;
constexpr int kMaxVtx = 1024;
constexpr int kVtxSmemTracks = 2048;  // selected tracks whose vertex arrays fit shared memory

struct VtxShared {
  uint32_t sh[33];
  uint32_t off[257];
  uint32_t cur[256];
  uint32_t nv, nvi, warn;
  uint32_t vcnt[kMaxVtx], voff[kMaxVtx + 1];
  uint16_t parent[kMaxVtx];
};

// cluster_tracks_by_density, fit_vertices, split_vertices and sort_by_pt2 on the selected
// tracks of one event (one CTA). TI / TB: types of the per-track vertex ids and neighbour
// counts and of the histogram / list entries; the arrays are in shared memory for events of
// up to kVtxSmemTracks selected tracks (16-bit entries) and in global memory above.
template <typename TI, typename TB>
__device__ __forceinline__ void vertex_core(Dev& d, EvInfo& E, int e, uint32_t nt, const float* __restrict__ zt,
                                            const float* __restrict__ ezt2, const float* ptt2, const uint32_t* itrk,
                                            TI* iv, TI* nn, uint8_t* izt, TB* B, float* zv, float* wv, float* vchi2,
                                            float* ptv2, uint16_t* sort_ind, VtxShared& S) {
  const uint64_t tb = E.tuple_base;
  uint32_t* sh = S.sh;
  uint32_t* s_off = S.off;
  uint32_t* s_cur = S.cur;
  uint32_t& s_nv = S.nv;
  uint32_t& s_nvi = S.nvi;
  uint32_t& s_warn = S.warn;
  uint32_t* s_vcnt = S.vcnt;
  uint32_t* s_voff = S.voff;
  uint16_t* s_parent = S.parent;
  // cluster_tracks_by_density (:84-206), HisToContainer{UInt8,256,16000,8,UInt16}
  for (int b = threadIdx.x; b < 257; b += blockDim.x) s_off[b] = 0;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) {
    int32_t iz = int32_t(trunc(__dmul_rn(double(zt[i]), 10.)));
    iz = iz < -128 ? -128 : (iz > 127 ? 127 : iz);
    izt[i] = uint8_t(iz + 128);
    atomicAdd(&s_off[izt[i]], 1u);
    iv[i] = TI(i + 1);
  }
  __syncthreads();
  {  // exclusive starts of the 256 bins
    const uint32_t v = threadIdx.x < 256 ? s_off[threadIdx.x] : 0u;
    uint32_t tot;
    const uint32_t ex = block_excl_scan(v, sh, &tot);
    if (threadIdx.x < 256) { s_off[threadIdx.x] = ex; s_cur[threadIdx.x] = ex; }
    if (threadIdx.x == 0) s_off[256] = tot;
  }
  __syncthreads();
  // histogram contents (1-based track indices), decreasing track index within a bin: one
  // warp walks the tracks from the last down, 32 at a time, ranking equal bins by lane
  if (threadIdx.x < 32) {
    const unsigned lane = threadIdx.x, lt = (1u << lane) - 1u;
    for (uint32_t b0 = 0; b0 < nt; b0 += 32) {
      const bool ok = b0 + lane < nt;
      const uint32_t i = ok ? nt - 1 - (b0 + lane) : 0u;
      const uint32_t bin = ok ? uint32_t(izt[i]) : 0xffffffffu;
      const uint32_t peers = __match_any_sync(0xffffffffu, bin);
      const uint32_t start = ok ? s_cur[bin] : 0u;
      __syncwarp();
      if (ok) {
        const uint32_t rank = __popc(peers & lt);
        B[start + rank] = TB(i + 1);
        if (rank == uint32_t(__popc(peers)) - 1u) s_cur[bin] = start + rank + 1;
      }
      __syncwarp();
    }
  }
  __syncthreads();
  const float eps = 0.07f, err2_max = __fmul_rn(0.01f, 0.01f), chi2_max = 9.0f;
  for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) {
    if (ezt2[i] > err2_max) continue;
    const int bs0 = int(izt[i]) + 1;
    const int be = bs0 + 1 < 256 ? bs0 + 1 : 256;
    const int bs = bs0 - 1 > 1 ? bs0 - 1 : 1;
    int32_t cnt = 0;
    for (uint32_t p = s_off[bs - 1]; p < s_off[be]; ++p) {
      const uint32_t j = B[p] - 1;
      if (j == i) continue;
      const float dist = fabsf(__fsub_rn(zt[i], zt[j]));
      if (dist > eps) continue;
      if (__fmul_rn(dist, dist) > __fmul_rn(chi2_max, __fadd_rn(ezt2[i], ezt2[j]))) continue;
      ++cnt;
    }
    nn[i] = TI(cnt);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) {
    float mdist = eps;
    const int bs0 = int(izt[i]) + 1;
    const int be = bs0 + 1 < 256 ? bs0 + 1 : 256;
    const int bs = bs0 - 1 > 1 ? bs0 - 1 : 1;
    int32_t a = int32_t(i + 1);
    for (uint32_t p = s_off[bs - 1]; p < s_off[be]; ++p) {
      const uint32_t j = B[p] - 1;
      if (nn[j] < nn[i]) continue;
      if (nn[j] == nn[i] && zt[j] >= zt[i]) continue;
      const float dist = fabsf(__fsub_rn(zt[i], zt[j]));
      if (dist > mdist) continue;
      if (__fmul_rn(dist, dist) > __fmul_rn(chi2_max, __fadd_rn(ezt2[i], ezt2[j]))) continue;
      mdist = dist;
      a = int32_t(j + 1);
    }
    iv[i] = TI(a);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) {
    int32_t m = iv[i];
    while (m != int32_t(iv[m - 1])) m = iv[m - 1];
    iv[i] = TI(m);
  }
  __syncthreads();
  uint32_t found = 0;
  for (uint32_t b = 0; b < nt; b += blockDim.x) {
    const uint32_t i = b + threadIdx.x;
    const bool root = i < nt && iv[i] == int32_t(i + 1);
    const bool seed = root && nn[i] >= 2;
    uint32_t tot;
    const uint32_t ex = block_excl_scan(seed ? 1u : 0u, sh, &tot);
    if (root) iv[i] = TI(seed ? -int32_t(found + ex + 1) : -9998);
    found += tot;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x)
    if (iv[i] >= 0) iv[i] = iv[iv[i] - 1];
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) iv[i] = TI(-iv[i]);
  if (threadIdx.x == 0) {
    if (found >= uint32_t(kMaxVtx)) { s_warn |= kWarnVertex; found = kMaxVtx - 1; }
    s_nv = found;
    s_nvi = found;
  }
  __syncthreads();
  // per-vertex track lists in ascending track order (the order of the reference's loops over
  // all tracks); B (the z histogram) is free again. A vertex made by a split keeps its parent's
  // list and selects its own tracks by id, as the loops over all tracks do.
  const uint32_t nv0 = s_nv;
  for (uint32_t v = threadIdx.x; v < uint32_t(kMaxVtx); v += blockDim.x) { s_vcnt[v] = 0; s_parent[v] = uint16_t(v); }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x)
    if (iv[i] >= 1 && uint32_t(iv[i]) <= nv0) atomicAdd(&s_vcnt[iv[i] - 1], 1u);
  __syncthreads();
  {
    uint32_t base = 0;
    for (uint32_t b = 0; b < nv0; b += blockDim.x) {
      const uint32_t v = b + threadIdx.x;
      const uint32_t c = v < nv0 ? s_vcnt[v] : 0u;
      uint32_t tot;
      const uint32_t ex = block_excl_scan(c, sh, &tot);
      if (v < nv0) { s_voff[v] = base + ex; s_vcnt[v] = base + ex; }
      base += tot;
    }
    if (threadIdx.x == 0) s_voff[nv0] = base;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x)
    if (iv[i] >= 1 && uint32_t(iv[i]) <= nv0) B[atomicAdd(&s_vcnt[iv[i] - 1], 1u)] = TB(i);
  __syncthreads();
  for (uint32_t v = threadIdx.x; v < nv0; v += blockDim.x) {
    const uint32_t lo = s_voff[v], hi = s_voff[v + 1];
    for (uint32_t p = lo + 1; p < hi; ++p) {
      const uint32_t x = B[p];
      uint32_t q = p;
      while (q > lo && B[q - 1] > x) { B[q] = B[q - 1]; --q; }
      B[q] = TB(x);
    }
  }
  __syncthreads();
  // fit_vertices, :228-286 (one thread per vertex keeps the track order of the sums)
  auto fit = [&](double chi2max) {
    const uint32_t nvf = s_nvi;
    for (uint32_t v = threadIdx.x; v < nvf; v += blockDim.x) {
      const uint32_t pv = s_parent[v], lo = s_voff[pv], hi = s_voff[pv + 1];
      float z = 0, w = 0;
      for (uint32_t p = lo; p < hi; ++p) {
        const uint32_t i = B[p];
        if (iv[i] != int32_t(v + 1)) continue;
        const float wi = __fdiv_rn(1.0f, ezt2[i]);
        z = __fadd_rn(z, __fmul_rn(zt[i], wi));
        w = __fadd_rn(w, wi);
      }
      if (!(w > 0)) atomicOr(&s_warn, kWarnVertex);
      z = __fdiv_rn(z, w);
      float c2s = 0;
      int32_t cnt = -1;
      for (uint32_t p = lo; p < hi; ++p) {
        const uint32_t i = B[p];
        if (iv[i] != int32_t(v + 1)) continue;
        float c2 = __fsub_rn(z, zt[i]);
        c2 = __fmul_rn(c2, __fdiv_rn(c2, ezt2[i]));
        if (double(c2) > chi2max) { iv[i] = 9999; continue; }
        c2s = __fadd_rn(c2s, c2);
        cnt += 1;
      }
      if (cnt > 0) w = __fmul_rn(w, __fdiv_rn(float(cnt), c2s));
      zv[v] = z; wv[v] = w; vchi2[v] = c2s; nn[v] = TI(cnt);
    }
    __syncthreads();
    if (threadIdx.x == 0) s_nv = nvf;
    __syncthreads();
  };
  fit(50.);
  // split_vertices, :288-371: each vertex decides alone; new ids follow the vertex order
  {
    const uint32_t nvf = s_nv;
    for (uint32_t b = 0; b < nvf; b += blockDim.x) {
      const uint32_t kv = b + threadIdx.x;
      bool split = false;
      float znew0 = 0, znew1 = 0;
      const uint32_t lo = kv < nvf ? s_voff[kv] : 0u, hi = kv < nvf ? s_voff[kv + 1] : 0u;
      if (kv < nvf && nn[kv] >= 4 && !(vchi2[kv] < __fmul_rn(9.0f, float(nn[kv])))) {
        if (nn[kv] >= 512) {
          atomicOr(&s_warn, kWarnVertex);
        } else {
          // 2-means in the vertex's tracks (zz = zt - zv, weights 1/ezt2), at most 20 iterations
          uint32_t nq = 0;
          const float zc = zv[kv];
          for (uint32_t p = lo; p < hi; ++p) if (iv[B[p]] == int32_t(kv + 1)) ++nq;
          if (nq != uint32_t(nn[kv] + 1)) atomicOr(&s_warn, kWarnVertex);
          bool more = true;
          int iter = 20;
          // first assignment: zz < 0 -> 1 else 2, kept per track in izt
          for (uint32_t p = lo; p < hi; ++p) {
            const uint32_t i = B[p];
            if (iv[i] == int32_t(kv + 1)) izt[i] = __fsub_rn(zt[i], zc) < 0 ? 1 : 2;
          }
          float w0 = 0, w1 = 0;
          while (more) {
            more = false;
            znew0 = znew1 = 0; w0 = w1 = 0;
            for (uint32_t p = lo; p < hi; ++p) {
              const uint32_t i = B[p];
              if (iv[i] != int32_t(kv + 1)) continue;
              const float zz = __fsub_rn(zt[i], zc), ww = __fdiv_rn(1.0f, ezt2[i]);
              if (izt[i] == 1) { znew0 = __fadd_rn(znew0, __fmul_rn(zz, ww)); w0 = __fadd_rn(w0, ww); }
              else { znew1 = __fadd_rn(znew1, __fmul_rn(zz, ww)); w1 = __fadd_rn(w1, ww); }
            }
            znew0 = __fdiv_rn(znew0, w0);
            znew1 = __fdiv_rn(znew1, w1);
            for (uint32_t p = lo; p < hi; ++p) {
              const uint32_t i = B[p];
              if (iv[i] != int32_t(kv + 1)) continue;
              const float zz = __fsub_rn(zt[i], zc);
              const float d0 = fabsf(__fsub_rn(znew0, zz)), d1 = fabsf(__fsub_rn(znew1, zz));
              const uint8_t newer = d0 < d1 ? 1 : 2;
              more |= newer != izt[i];
              izt[i] = newer;
            }
            if (--iter <= 0) more = false;
          }
          if (!(w0 == 0 || w1 == 0)) {
            const float dd = __fsub_rn(znew0, znew1);
            const float dist2 = __fmul_rn(dd, dd);
            const float chi2_dist = __fdiv_rn(dist2, __fadd_rn(__fdiv_rn(1.0f, w0), __fdiv_rn(1.0f, w1)));
            split = !(chi2_dist < 4);
          }
        }
      }
      uint32_t tot;
      const uint32_t ex = block_excl_scan(split ? 1u : 0u, sh, &tot);
      if (split) {
        const uint32_t slot = s_nvi + ex;  // 0-based id of the new vertex
        const int32_t newv = int32_t(slot + 1);
        if (slot < uint32_t(kMaxVtx)) s_parent[slot] = uint16_t(kv);
        for (uint32_t p = lo; p < hi; ++p) {
          const uint32_t i = B[p];
          if (iv[i] == int32_t(kv + 1) && izt[i] == 2) iv[i] = TI(newv);
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) s_nvi += tot;
      __syncthreads();
    }
    if (threadIdx.x == 0 && s_nvi >= uint32_t(kMaxVtx)) { s_warn |= kWarnVertex; s_nvi = kMaxVtx - 1; }
    __syncthreads();
  }
  fit(5000.);
  // sort_by_pt2, :391-436 (the sorted order itself is dropped by the reference)
  const uint32_t nvf = s_nv;
  if (nvf >= 1) {
    for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) d.idv[tb + itrk[i]] = int16_t(iv[i]);
    for (uint32_t v = threadIdx.x; v < nvf; v += blockDim.x) {
      const uint32_t pv = s_parent[v], lo = s_voff[pv], hi = s_voff[pv + 1];
      float s = 0;
      for (uint32_t p = lo; p < hi; ++p) {
        const uint32_t i = B[p];
        if (iv[i] == int32_t(v + 1)) s = __fadd_rn(s, ptt2[i]);
      }
      ptv2[v] = s;
    }
    if (threadIdx.x == 0 && nvf == 1) sort_ind[0] = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    E.n_vtx = nvf;
    if (s_warn) E.warnings |= s_warn;
  }
}

__global__ void __launch_bounds__(kVtxThreads) k_vertices(Dev d) {
  const int e = blockIdx.x;
  EvInfo& E = d.ev[e];
  const uint64_t tb = E.tuple_base;
  const uint32_t ntu = E.n_tuples;
  float* zv = d.zv + size_t(e) * kMaxVtx;
  float* wv = d.wv + size_t(e) * kMaxVtx;
  float* vchi2 = d.vchi2 + size_t(e) * kMaxVtx;
  float* ptv2 = d.ptv2 + size_t(e) * kMaxVtx;
  uint16_t* sort_ind = d.sort_ind + size_t(e) * kMaxVtx;
  int32_t* nn = d.ndof + tb + size_t(e) * kMaxVtx;  // length n_tuples + 1024
  float* zt = d.vws_zt + tb;
  float* ezt2 = d.vws_ezt2 + tb;
  float* ptt2 = d.vws_ptt2 + tb;
  int32_t* iv = d.vws_iv + tb;     // 1-based values as the reference stores them
  uint32_t* itrk = d.vws_itrk + tb;
  uint8_t* izt = d.vws_izt + tb;
  __shared__ VtxShared S;
  __shared__ float s_zt[kVtxSmemTracks], s_ezt2[kVtxSmemTracks];
  __shared__ int16_t s_iv[kVtxSmemTracks], s_nn[kVtxSmemTracks];
  __shared__ uint16_t s_b[kVtxSmemTracks];
  __shared__ uint8_t s_izt[kVtxSmemTracks];
  uint32_t* sh = S.sh;
  for (int v = threadIdx.x; v < kMaxVtx; v += blockDim.x) { zv[v] = 0; wv[v] = 0; vchi2[v] = 0; ptv2[v] = 0; sort_ind[v] = 0; }
  for (uint32_t t = threadIdx.x; t < ntu + kMaxVtx; t += blockDim.x) nn[t] = 0;
  for (uint32_t t = threadIdx.x; t < ntu; t += blockDim.x) d.idv[tb + t] = -1;
  if (threadIdx.x == 0) S.warn = 0;
  // load_tracks (:51-82): >= 4 hits, loose, pt >= 0.5, in tuple order
  uint32_t nt = 0;
  for (uint32_t b = 0; b < ntu; b += blockDim.x) {
    const uint32_t t = b + threadIdx.x;
    bool sel = false;
    if (t < ntu) {
      const uint64_t g = tb + t;
      const uint32_t n = d.tuple_off[g + 1] - d.tuple_off[g];
      sel = n >= 4 && d.quality[g] == 2 && !(d.t_pt[g] < 0.5f);
    }
    uint32_t tot;
    const uint32_t ex = block_excl_scan(sel ? 1u : 0u, sh, &tot);
    if (sel) {
      const uint64_t g = tb + t;
      const uint32_t i = nt + ex;
      const float pt = d.t_pt[g];
      itrk[i] = t;
      zt[i] = d.t_state[5 * g + 4];
      ezt2[i] = d.t_cov[15 * g + 14];
      ptt2[i] = __fmul_rn(pt, pt);
    }
    nt += tot;
  }
  if (threadIdx.x == 0) E.n_vtx_tracks = nt;
  __syncthreads();
  if (nt <= uint32_t(kVtxSmemTracks)) {
    for (uint32_t i = threadIdx.x; i < nt; i += blockDim.x) { s_zt[i] = zt[i]; s_ezt2[i] = ezt2[i]; }
    for (uint32_t i = threadIdx.x; i < uint32_t(kVtxSmemTracks); i += blockDim.x) s_nn[i] = 0;
    __syncthreads();
    vertex_core<int16_t, uint16_t>(d, E, e, nt, s_zt, s_ezt2, ptt2, itrk, s_iv, s_nn, s_izt, s_b, zv, wv, vchi2, ptv2,
                                   sort_ind, S);
    // neighbour counts of the tracks, then ndof of the vertices: the reference's nn array
    const uint32_t nw = nt > S.nv ? nt : S.nv;
    for (uint32_t i = threadIdx.x; i < nw; i += blockDim.x) nn[i] = s_nn[i];
  } else {
    vertex_core<int32_t, uint32_t>(d, E, e, nt, zt, ezt2, ptt2, itrk, iv, nn, izt, d.vws_bins + tb, zv, wv, vchi2,
                                   ptv2, sort_ind, S);
  }
}

}  // namespace

void launch_classify(const Dev& d, const Launch& L) {
  auto g = [&](int seg) { return dim3(L.bpe_of(seg), d.E); };
  k_classify<<<g(kTuneClassify), 256, 0, L.s>>>(d);
  L.mark("classify");
  // events by tuple count: shared-memory qualities up to 32K tuples (every event at the
  // reference's capacities), a 104 KB form up to 256K, global memory above
  k_dup_prep<<<d.E, 256, 0, L.s>>>(d);
  k_fast_dup_smem<kDupMaxTuples, 0><<<d.E, 32, dup_smem_bytes<kDupMaxTuples>(), L.s>>>(d);
  if (d.tuples_per_event > uint32_t(kDupMaxTuples)) {
    k_fast_dup_smem<kDupLargeTuples, kDupMaxTuples><<<d.E, 32, dup_smem_bytes<kDupLargeTuples>(), L.s>>>(d);
  }
  if (d.tuples_per_event > uint32_t(kDupLargeTuples)) k_fast_dup<<<div_up(d.E, 4), 128, 0, L.s>>>(d, kDupLargeTuples);
  L.mark("fast_duplicate_remover");
  cudaMemsetAsync(d.htt_cur, 0, size_t(d.cap_hits) * sizeof(uint32_t), L.s);
  k_hit_to_tuple<0><<<g(kTuneHitToTuple), 256, 0, L.s>>>(d);
  excl_scan_shift_u32(d.htt_cur, d.htt_cnt, d.cap_hits, &d.ev[d.E].n_hits, d.scan_tmp, L.s);
  k_hit_to_tuple<1><<<g(kTuneHitToTuple), 256, 0, L.s>>>(d);
  L.mark("hit_to_tuple");
  k_triplet_cleaner<<<g(kTuneHitToTuple), 256, 0, L.s>>>(d);
  L.mark("triplet_cleaner");
}

int prepare_select_kernels() {
  const cudaError_t err = cudaFuncSetAttribute(k_fast_dup_smem<kDupLargeTuples, kDupMaxTuples>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               int(dup_smem_bytes<kDupLargeTuples>()));
  return err == cudaSuccess ? 0 : -1;
}

void launch_vertices(const Dev& d, const Launch& L) {
  k_vertices<<<d.E, kVtxThreads, 0, L.s>>>(d);
  L.mark("vertices");
}

}  // namespace pxl
