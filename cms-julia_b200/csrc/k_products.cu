// Copy-out of the CA, fit and vertex products in the reference's layouts
// (TrackSOA stride 32768, or the extended per-event tuple capacity when larger, 1-based ids,
// PreAllocMatrix columns as CSR lists).
// The device keeps compact per-event arrays; the fixed-stride views the
// reference exposes are rebuilt here on the host.
#include <algorithm>
#include <cstring>
#include <vector>

#include "pxl_ctx.h"

using namespace pxl;

namespace {

// device -> host on the context's stream (which the caller has ordered after the context's work)
template <class T>
std::vector<T> dvec(cudaStream_t s, const T* src, int64_t n) {
  std::vector<T> v(size_t(std::max<int64_t>(n, 0)));
  if (n > 0) {
    cudaMemcpyAsync(v.data(), src, size_t(n) * sizeof(T), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
  }
  return v;
}

template <class T>
int64_t out(const std::vector<T>& v, void* dst, int64_t max_bytes) {
  if (dst && max_bytes > 0 && !v.empty())
    std::memcpy(dst, v.data(), size_t(std::min<int64_t>(int64_t(v.size() * sizeof(T)), max_bytes)));
  return int64_t(v.size());
}

// CSR of per-key lists truncated to `rows` entries, values mapped to 1-based event-local ids
std::vector<uint32_t> csr(const std::vector<uint32_t>& cnt, const std::vector<uint32_t>& list, uint32_t list_base,
                          uint32_t rows, uint32_t id_base) {
  const size_t n = cnt.size() - 1;
  std::vector<uint32_t> v(n + 1, 0);
  std::vector<uint32_t> ent;
  for (size_t k = 0; k < n; ++k) {
    uint32_t lo = cnt[k], hi = cnt[k + 1];
    uint32_t len = std::min(hi - lo, rows);
    for (uint32_t j = 0; j < len; ++j) ent.push_back(list[lo + j - list_base] - id_base + 1);
    v[k + 1] = uint32_t(ent.size());
  }
  v.insert(v.end(), ent.begin(), ent.end());
  return v;
}

}  // namespace

int64_t copy_ca_product(PxlCtx* ctx, int32_t e, int32_t product, void* dst, int64_t max_bytes) {
  const Dev& d = ctx->d;
  const cudaStream_t s = ctx->stream;
  const EvInfo& E = ctx->ev_host[size_t(e)];
  const bool ca = (ctx->done_mask & PXL_STAGE_TUPLES) != 0;
  const bool fit = (ctx->done_mask & PXL_STAGE_FIT) != 0;
  const bool vtx = (ctx->done_mask & PXL_STAGE_VERTICES) != 0;
  const uint64_t cb = E.cell_base, tb = E.tuple_base;
  const uint32_t nc = E.n_cells, nt = E.n_tuples, nh = E.n_hits;
  // TrackSOA / ZVertexSoA stride: the reference's 32768, or the extended per-event tuple capacity
  const uint32_t stride = std::max(uint32_t(kTupleStride), d.tuples_per_event);
  switch (product) {
    case PXL_P_CELLS: {
      if (!ca) return PXL_ERR_STATE;
      auto in = dvec(s, d.cell_inner + cb, nc);
      auto ou = dvec(s, d.cell_outer + cb, nc);
      auto pr = dvec(s, d.cell_pair + cb, nc);
      auto id = dvec(s, d.cell_id + cb, nc);
      auto us = dvec(s, d.cell_used + cb, nc);
      std::vector<int32_t> v(size_t(nc) * 5);
      for (uint32_t k = 0; k < nc; ++k) {
        v[5 * k] = int32_t(in[k] + 1); v[5 * k + 1] = int32_t(ou[k] + 1); v[5 * k + 2] = int32_t(pr[k]) + 1;
        v[5 * k + 3] = id[k]; v[5 * k + 4] = us[k];
      }
      return out(v, dst, max_bytes);
    }
    case PXL_P_CELL_NEIGHBORS:
    case PXL_P_CELL_TRACKS: {
      if (!ca) return PXL_ERR_STATE;
      const bool nb = product == PXL_P_CELL_NEIGHBORS;
      auto cnt = dvec(s, (nb ? d.cn_cnt : d.ct_cnt) + cb, int64_t(nc) + 1);
      if (nc == 0) return out(std::vector<uint32_t>(1, 0), dst, max_bytes);
      uint32_t lo = cnt[0], hi = cnt[nc];
      auto list = dvec(s, (nb ? d.cn_list : d.ct_list) + lo, int64_t(hi - lo));
      return out(csr(cnt, list, lo, uint32_t(kCellRows), nb ? uint32_t(cb) : uint32_t(tb)), dst, max_bytes);
    }
    case PXL_P_OUTER_HIT_OF_CELL: {
      if (!ca) return PXL_ERR_STATE;
      auto cnt = dvec(s, d.ohc_cnt + E.hit_base, int64_t(nh) + 1);
      if (nh == 0) return out(std::vector<uint32_t>(1, 0), dst, max_bytes);
      uint32_t lo = cnt[0], hi = cnt[nh];
      auto list = dvec(s, d.ohc_list + lo, int64_t(hi - lo));
      return out(csr(cnt, list, lo, uint32_t(kMaxCellsPerHit), uint32_t(cb)), dst, max_bytes);
    }
    case PXL_P_TUPLE_MULTIPLICITY: {
      if (!ca) return PXL_ERR_STATE;
      // bins 1..8 hold the non-duplicate tuples by hit count; the reference's fill leaves each
      // bin in decreasing tuple id
      auto off = dvec(s, d.tuple_off + tb, int64_t(nt) + 1);
      auto q = dvec(s, d.quality + tb, nt);
      std::vector<uint32_t> v(E.tm_off, E.tm_off + 9);
      std::vector<std::vector<uint32_t>> bins(9);
      for (uint32_t t = 0; t < nt; ++t) {
        uint32_t n = off[t + 1] - off[t];
        if (n < 3 || n >= 9 || q[t] == 1) continue;
        bins[n - 1].push_back(t + 1);
      }
      for (auto& b : bins) for (auto it = b.rbegin(); it != b.rend(); ++it) v.push_back(*it);
      return out(v, dst, max_bytes);
    }
    case PXL_P_HIT_INDICES_OFF: {
      if (!ca) return PXL_ERR_STATE;
      auto off = dvec(s, d.tuple_off + tb, int64_t(nt) + 1);
      std::vector<uint32_t> v(stride + 1);
      const uint32_t base = nt ? off[0] : 0u;
      const uint32_t total = nt ? off[nt] - base : 0u;
      for (uint32_t t = 0; t <= stride; ++t) v[t] = t < nt ? off[t] - base + 1 : total + 1;
      return out(v, dst, max_bytes);
    }
    case PXL_P_HIT_INDICES:
    case PXL_P_HIT_INDICES32:
    case PXL_P_DET_INDICES: {
      if (!ca) return PXL_ERR_STATE;
      if (nt == 0) return 0;
      auto off = dvec(s, d.tuple_off + tb, int64_t(nt) + 1);
      const uint32_t lo = off[0], n = off[nt] - off[0];
      if (product == PXL_P_DET_INDICES) return out(dvec(s, d.tuple_det + lo, n), dst, max_bytes);
      auto h = dvec(s, d.tuple_hits + lo, n);
      for (auto& x : h) x += 1;  // 1-based hit ids
      if (product == PXL_P_HIT_INDICES32) return out(h, dst, max_bytes);
      std::vector<uint16_t> v(n);
      for (uint32_t k = 0; k < n; ++k) {
        if (h[k] > 0xFFFFu) return PXL_ERR_CAPACITY;  // an extended-capacity event above 65535 hits
        v[k] = uint16_t(h[k]);
      }
      return out(v, dst, max_bytes);
    }
    case PXL_P_QUALITY:
    case PXL_P_FITTED: {
      if (!ca || (product == PXL_P_FITTED && !fit)) return PXL_ERR_STATE;
      std::vector<uint8_t> v(stride, 0);
      auto q = dvec(s, (product == PXL_P_QUALITY ? d.quality : d.t_fitted) + tb, nt);
      std::copy(q.begin(), q.end(), v.begin());
      return out(v, dst, max_bytes);
    }
    case PXL_P_CHI2:
    case PXL_P_ETA:
    case PXL_P_PT:
    case PXL_P_STATE:
    case PXL_P_COVARIANCE: {
      if (!fit) return PXL_ERR_STATE;
      int w = product == PXL_P_STATE ? 5 : (product == PXL_P_COVARIANCE ? 15 : 1);
      const float* src = product == PXL_P_CHI2 ? d.t_chi2 : product == PXL_P_ETA ? d.t_eta
                         : product == PXL_P_PT ? d.t_pt : product == PXL_P_STATE ? d.t_state : d.t_cov;
      std::vector<float> v(size_t(stride) * w, 0.f);
      auto a = dvec(s, src + tb * w, int64_t(nt) * w);
      std::copy(a.begin(), a.end(), v.begin());
      return out(v, dst, max_bytes);
    }
    case PXL_P_IDV: {
      if (!vtx) return PXL_ERR_STATE;
      std::vector<int16_t> v(stride, int16_t(-1));
      auto a = dvec(s, d.idv + tb, nt);
      std::copy(a.begin(), a.end(), v.begin());
      return out(v, dst, max_bytes);
    }
    case PXL_P_ZV:
    case PXL_P_WV:
    case PXL_P_VCHI2:
    case PXL_P_PTV2: {
      if (!vtx) return PXL_ERR_STATE;
      const float* src = product == PXL_P_ZV ? d.zv : product == PXL_P_WV ? d.wv : product == PXL_P_VCHI2 ? d.vchi2 : d.ptv2;
      return out(dvec(s, src + size_t(e) * 1024, 1024), dst, max_bytes);
    }
    case PXL_P_NDOF: {
      if (!vtx) return PXL_ERR_STATE;
      std::vector<int32_t> v(stride, 0);
      const uint32_t len = std::max(E.n_vtx_tracks, E.n_vtx);
      auto a = dvec(s, d.ndof + tb + size_t(e) * 1024, len);
      std::copy(a.begin(), a.end(), v.begin());
      return out(v, dst, max_bytes);
    }
    case PXL_P_SORT_IND: {
      if (!vtx) return PXL_ERR_STATE;
      return out(dvec(s, d.sort_ind + size_t(e) * 1024, 1024), dst, max_bytes);
    }
    default:
      return PXL_ERR_ARG;
  }
}
