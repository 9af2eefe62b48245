// Context, conditions upload, batch buffers, launch sequence, CUDA graph and
// the C ABI declared in include/pxl.h.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pxl.h"
#include "pxl_ctx.h"
#include "pxl_internal.cuh"

using namespace pxl;


namespace {

#define CK(x)                                                                     \
  do {                                                                            \
    cudaError_t err__ = (x);                                                      \
    if (err__ != cudaSuccess) {                                                   \
      std::fprintf(stderr, "pxl: %s failed: %s\n", #x, cudaGetErrorString(err__)); \
      return PXL_ERR_CUDA;                                                        \
    }                                                                             \
  } while (0)

template <class T>
int dalloc(PxlCtx* c, T** p, int64_t n) {
  size_t bytes = size_t(std::max<int64_t>(n, 1)) * sizeof(T);
  void* q = nullptr;
  cudaError_t err = cudaMalloc(&q, bytes);
  if (err != cudaSuccess) {
    std::fprintf(stderr, "pxl: cudaMalloc(%zu) failed: %s\n", bytes, cudaGetErrorString(err));
    return PXL_ERR_CUDA;
  }
  c->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return 0;
}

template <class T>
int upload(PxlCtx* c, const T** dst, const std::vector<T>& v) {
  T* q = nullptr;
  int rc = dalloc(c, &q, int64_t(v.size()));
  if (rc) return rc;
  if (!v.empty()) CK(cudaMemcpy(q, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  *dst = q;
  return 0;
}

struct Rd {
  const uint8_t* p;
  size_t n, off = 0;
  bool ok = true;
  template <class T> T get() {
    T v{};
    if (off + sizeof(T) > n) { ok = false; return v; }
    std::memcpy(&v, p + off, sizeof(T));
    off += sizeof(T);
    return v;
  }
  template <class T> void get_n(T* dst, size_t k) {
    if (off + k * sizeof(T) > n) { ok = false; return; }
    std::memcpy(dst, p + off, k * sizeof(T));
    off += k * sizeof(T);
  }
  void skip(size_t k) { if (off + k > n) ok = false; else off += k; }
};

// ES products -> device conditions (layouts: SiPixelFedCablingMapGPUWrapperESProducer.jl:27-57,
// SiPixelGainCalibrationForHLTGPUESProducer.jl:14-46, PixelCPEFastESProducer.jl:16-103,
// BeamSpotESProducer.jl:11-28)
int load_conditions(PxlCtx* ctx, const PxlConditions* cd) {
  Conditions& c = ctx->d.c;
  {
    Rd r{cd->cabling_map, cd->cabling_map_bytes};
    std::vector<uint32_t> a[6];
    for (auto& v : a) { v.resize(kCablingSize); r.get_n(v.data(), kCablingSize); }
    std::vector<uint8_t> bad(kCablingSize);
    r.get_n(bad.data(), kCablingSize);
    if (!r.ok) return PXL_ERR_CONDITIONS;
    std::vector<uint64_t> cab(kCablingSize);
    for (uint32_t i = 0; i < kCablingSize; ++i) {
      uint64_t raw = a[3][i], mod = a[5][i] & 0xFFFFu, rd = std::min<uint32_t>(a[4][i], 255u);
      cab[i] = raw | (mod << 32) | (rd << 48) | (uint64_t(bad[i] != 0) << 56);
    }
    int rc = upload(ctx, &c.cab, cab);
    if (rc) return rc;
  }
  {
    Rd r{cd->fed_ids, cd->fed_ids_bytes};
    uint32_t n = r.get<uint32_t>();
    std::vector<uint32_t> ids(n);
    r.get_n(ids.data(), n);
    if (!r.ok || n > uint32_t(kMaxFedSlots)) return PXL_ERR_CONDITIONS;
    // slots follow the fedIds order, skipping FED 40 (SiPixelRawToClusterCUDA.jl:75-81)
    std::vector<uint32_t> slots;
    std::vector<int16_t> slot_of(4096, -1);
    for (uint32_t id : ids) {
      if (id == 40 || id < 1200 || id >= 4096) continue;
      slot_of[id] = int16_t(slots.size());
      slots.push_back(id);
    }
    c.n_fed_ids = int32_t(slots.size());
    ctx->d.n_fed_slots = int32_t(slots.size());
    int rc = upload(ctx, &c.fed_ids, slots);
    if (rc) return rc;
    const int16_t* q;
    rc = upload(ctx, &q, slot_of);
    if (rc) return rc;
    ctx->fed_slot_of = const_cast<int16_t*>(q);
  }
  {
    Rd r{cd->gain, cd->gain_bytes};
    r.skip(8);
    std::vector<uint32_t> first(2000), lcd(2000);
    for (int i = 0; i < 2000; ++i) {
      uint32_t f = r.get<uint32_t>(), l = r.get<uint32_t>();
      int32_t cols = r.get<int32_t>();
      first[i] = f;
      lcd[i] = cols != 0 ? (l - f) / uint32_t(cols) : 0u;
    }
    float fv[6];
    r.get_n(fv, 6);
    uint32_t uv[4];
    r.get_n(uv, 4);
    uint32_t nbytes = r.get<uint32_t>();
    uint32_t n = nbytes / 2;
    std::vector<uint16_t> pairs(n);
    for (uint32_t i = 0; i < n; ++i) { uint8_t g = r.get<uint8_t>(), p = r.get<uint8_t>(); pairs[i] = uint16_t(g | (p << 8)); }
    if (!r.ok) return PXL_ERR_CONDITIONS;
    c.min_ped = fv[0]; c.min_gain = fv[2]; c.ped_prec = fv[4]; c.gain_prec = fv[5];
    c.rows_avg = uv[0]; c.dead_flag = uv[2]; c.noisy_flag = uv[3];
    c.n_gain_pairs = n;
    int rc = upload(ctx, &c.gain_first, first);
    if (!rc) rc = upload(ctx, &c.gain_lcd, lcd);
    if (!rc) rc = upload(ctx, &c.gain_pairs, pairs);
    if (rc) return rc;
  }
  float bsv[11];
  {
    Rd r{cd->beamspot, cd->beamspot_bytes};
    r.get_n(bsv, 11);
    if (!r.ok) return PXL_ERR_CONDITIONS;
    c.bs_x = bsv[0]; c.bs_y = bsv[1]; c.bs_z = bsv[2];
  }
  {
    Rd r{cd->cpe, cd->cpe_bytes};
    c.thick_b = r.get<float>(); c.thick_e = r.get<float>(); c.pitch_x = r.get<float>(); c.pitch_y = r.get<float>();
    uint32_t n = r.get<uint32_t>();
    std::vector<DetParamsD> det(n);
    for (uint32_t i = 0; i < n; ++i) {
      DetParamsD& dp = det[i];
      dp.is_barrel = r.get<uint8_t>() != 0;
      r.get<uint8_t>(); r.get<uint16_t>(); r.get<uint16_t>(); r.skip(2); r.get<uint32_t>();
      dp.shift_x = r.get<float>(); dp.shift_y = r.get<float>(); dp.cw_x = r.get<float>(); dp.cw_y = r.get<float>();
      dp.x0 = r.get<float>(); dp.y0 = r.get<float>(); dp.z0 = r.get<float>();
      r.get_n(dp.sx, 3); r.get_n(dp.sy, 3);
      dp.px = r.get<float>(); dp.py = r.get<float>(); dp.pz = r.get<float>();
      r.get_n(dp.R, 9);
    }
    float lad[6][kLadders];
    for (int k = 0; k < 6; ++k) r.get_n(lad[k], kLadders);  // Z, X, Y, R, MinZ, MaxZ
    float ecz[2];
    r.get_n(ecz, 2);
    r.get_n(c.layer_start, 11);
    if (!r.ok) return PXL_ERR_CONDITIONS;
    c.n_det = int32_t(n);
    int rc = upload(ctx, &c.det, det);
    if (rc) return rc;
    // average geometry shifted by the beam spot (gpuPixelRecHits.jl:45-67), Float32
    std::vector<float> ag(6 * kLadders + 2);
    for (int il = 0; il < kLadders; ++il) {
      float z = lad[0][il] - c.bs_z, x = lad[1][il] - c.bs_x, y = lad[2][il] - c.bs_y;
      ag[il] = z;
      ag[kLadders + il] = x;
      ag[2 * kLadders + il] = y;
      ag[3 * kLadders + il] = std::sqrt(x * x + y * y);
      ag[4 * kLadders + il] = lad[4][il] - c.bs_z;
      ag[5 * kLadders + il] = lad[5][il] - c.bs_z;
    }
    ag[6 * kLadders] = ecz[0] - c.bs_z;
    ag[6 * kLadders + 1] = ecz[1] - c.bs_z;
    ctx->avg_geom = ag;
    rc = upload(ctx, &c.avg_geom, ag);
    if (rc) return rc;
  }
  c.b_field = float(0.0114256972711507);
  return 0;
}

int alloc_batch(PxlCtx* ctx) {
  Dev& d = ctx->d;
  const PxlParams& p = ctx->p;
  const int64_t E = p.max_events;
  d.cap_words = p.max_words;
  d.cap_hits = p.max_hits;
  d.cap_cells = p.max_doublets;
  d.cap_tuples = p.max_tuples;
  d.cap_tuple_hits = 5 * p.max_tuples;
  d.cap_items = 8 * p.max_hits;  // inner-hit items over 19 layer pairs: each hit is inner in at most 6 pairs
  d.cap_pairs = 2 * p.max_doublets;
  d.hits_per_event = uint32_t(p.hits_per_event);
  d.doublets_per_event = uint32_t(p.doublets_per_event);
  d.tuples_per_event = uint32_t(p.tuples_per_event);
  d.fits_per_mult = uint32_t(p.fits_per_multiplicity);
  d.columns_per_event = uint32_t(p.columns_per_event);
  d.fit_precision = p.fit_precision;
  d.include_errors = p.include_errors;
  d.use_quality = p.use_quality;
  d.apply_charge_cut = 1;
  const int64_t NF = std::max(d.n_fed_slots, 1);
  int rc = 0;
#define A(ptr, n) do { rc = dalloc(ctx, &d.ptr, (n)); if (rc) return rc; } while (0)
  A(ev, E + 1);
  A(fed_src, E * NF); A(fed_nw, E * NF); A(fed_wo, E * NF); A(fed_nmod, E * NF);
  A(xx, d.cap_words); A(yy, d.cap_words); A(adc, d.cap_words); A(mid, d.cap_words); A(clus, d.cap_words);
  A(pdigi, d.cap_words); A(rawid, d.cap_words);
  A(err, 5 * d.cap_words); A(err_count, 1); A(id_seen, E * 64);
  A(wq_order, E); A(wq_head, kWqSlots); A(wq_prefix, kWqSlots * (E + 1));
  A(module_start, E * (kMaxNumModules + 1)); A(clus_in_module, E * kMaxNumModules); A(module_id, E * kMaxNumModules);
  A(clus_module_start, E * (kMaxNumModules + 1));
  A(xl, d.cap_hits); A(yl, d.cap_hits); A(xerr, d.cap_hits); A(yerr, d.cap_hits);
  A(xg, d.cap_hits); A(yg, d.cap_hits); A(zg, d.cap_hits); A(rg, d.cap_hits);
  A(iphi, d.cap_hits); A(xsize, d.cap_hits); A(ysize, d.cap_hits); A(detind, d.cap_hits); A(charge, d.cap_hits);
  A(hits_layer_start, E * 11); A(phi_off, E * kPhiTotBins); A(phi_bins, d.cap_hits); A(hit_rec, d.cap_hits); A(hit_rec_s, d.cap_hits); A(hit_u_s, d.cap_hits); A(hit_sum, d.cap_hits); A(hit_me, d.cap_hits); A(hit_xyzr, d.cap_hits);
  A(pair_cum, E * kNPairs);
  A(item_cnt, d.cap_items + 1);
  A(item_pool, d.cap_items); A(dbl_pool, d.cap_cells); A(dbl_pool_ctr, 1);
  A(tuple_det, d.cap_tuple_hits);
  A(cell_inner, d.cap_cells); A(cell_outer, d.cap_cells); A(cell_pair, d.cap_cells); A(cell_id, d.cap_cells);
  A(cell_used, d.cap_cells);
  A(ohc_cnt, d.cap_hits + 1); A(ohc_cur, d.cap_hits); A(ohc_list, d.cap_cells); A(ohc_rec, d.cap_cells);
  A(cn_pairs, d.cap_pairs); A(cn_pair_ctr, 1); d.cap_long = std::max({d.cap_cells, d.cap_pairs, d.cap_tuple_hits}) / 9 + 1;
  A(long_lists, d.cap_long); A(long_ctr, 1); A(cn_cnt, d.cap_cells + 1); A(cn_cur, d.cap_cells); A(cn_list, d.cap_pairs);
  A(tstart_cnt, d.cap_cells + 1);
  // tuple record pool: the batch's tuples plus a quarter for uneven parts
  d.tp_part = uint32_t((d.cap_tuples + d.cap_tuples / 4) / kTpParts + 64);
  // PXL_TUPLE_POOL_PART (records per part) shrinks the pool, so that tests can make it overflow
  // and check the walking fill that then runs
  if (const char* v = std::getenv("PXL_TUPLE_POOL_PART")) d.tp_part = uint32_t(std::max(1, std::atoi(v)));
  A(tp_hdr, int64_t(kTpParts) * d.tp_part); A(tp_cells, 2 * int64_t(kTpParts) * d.tp_part);
  A(tp_ctr, kTpParts * kTpStride + 1);
  A(tuple_off, d.cap_tuples + 1); A(tuple_hits, d.cap_tuple_hits); A(quality, d.cap_tuples);
  A(tuple_cell, d.cap_tuple_hits);
  A(ct_cnt, d.cap_cells + 1); A(ct_cur, d.cap_cells); A(ct_list, d.cap_tuple_hits);
  A(tm_bins, d.cap_tuples);
  A(t_state, 5 * d.cap_tuples); A(t_cov, 15 * d.cap_tuples); A(t_pt, d.cap_tuples); A(t_eta, d.cap_tuples);
  A(t_chi2, d.cap_tuples); A(t_fitted, d.cap_tuples);
  A(fit_list, d.cap_tuples); A(refit_list, d.cap_tuples);
  A(htt_cnt, d.cap_hits + 1); A(htt_cur, d.cap_hits); A(htt_list, d.cap_tuple_hits);
  A(dup_bits, d.cap_cells / 32 + 2); A(dup_list, d.cap_cells); A(dup_eoff, d.cap_cells + E + 1);
  A(dup_et, d.cap_tuple_hits); A(dup_ek, d.cap_tuple_hits);
  A(vws_zt, d.cap_tuples); A(vws_ezt2, d.cap_tuples); A(vws_ptt2, d.cap_tuples); A(vws_iv, d.cap_tuples);
  A(vws_itrk, d.cap_tuples); A(vws_izt, d.cap_tuples); A(vws_bins, d.cap_tuples);
  A(idv, d.cap_tuples); A(zv, E * 1024); A(wv, E * 1024); A(vchi2, E * 1024); A(ptv2, E * 1024);
  A(ndof, d.cap_tuples + E * 1024); A(sort_ind, E * 1024);
  int64_t st = scan_tmp_elems(std::max({d.cap_words, d.cap_items, d.cap_cells, d.cap_hits, d.cap_tuples}) + 1);
  A(scan_tmp, st); A(scan_tmp64, st);
  A(status, 1);
  d.cap_big = E * kMaxNumModules;
  A(big_list, kListHeader + kNumLists * d.cap_big);
#undef A
  // input staging
  ctx->raw_cap = size_t(d.cap_words) * 4 + size_t(E) * (4 + 16 * 4 + size_t(d.n_fed_slots + 8) * 24) + 4096;
  for (int k = 0; k < PxlCtx::kSlots; ++k) {
    rc = dalloc(ctx, &ctx->d_raw[k], int64_t(ctx->raw_cap));
    if (rc) return rc;
    rc = dalloc(ctx, &ctx->d_ev_off[k], E + 1);
    if (rc) return rc;
    CK(cudaMallocHost(&ctx->h_off[k], size_t(E + 1) * sizeof(uint64_t)));
    CK(cudaEventCreateWithFlags(&ctx->ev_staged[k], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ctx->ev_consumed[k], cudaEventDisableTiming));
  }
  return 0;
}

int run_chain(PxlCtx* ctx, uint32_t mask, cudaStream_t s) {
  Dev& d = ctx->d;
  if (d.E <= 0) return 0;
  Launch L{s, d.bpe, 256, (ctx->prof.on && !ctx->capturing) ? &ctx->prof : nullptr};
  L.tune = ctx->tune;
  L.wq_ctas = ctx->wq_ctas;
  if ((mask & PXL_STAGE_DIGIS) && L.prof) ctx->prof.n = 0;
  // stages run in chain order; a producer boundary may stop after any of them and a
  // later call (pxl_event_continue) resumes from the products already on the device
  // a direct (non-graph) run over the context's slot-0 input orders itself after that slot's
  // copy and marks the slot free once the raw data has been unpacked
  const bool own_slot0 = (mask & PXL_STAGE_DIGIS) && !ctx->capturing && d.raw == ctx->d_raw[0];
  if (own_slot0) CK(cudaStreamWaitEvent(s, ctx->ev_staged[0], 0));
  if (mask & PXL_STAGE_DIGIS) {
    CK(cudaMemsetAsync(d.err_count, 0, sizeof(uint32_t), s));
    CK(cudaMemsetAsync(d.status, 0, sizeof(uint32_t), s));
    launch_raw(d, L, ctx->fed_slot_of);
    if (own_slot0) CK(cudaEventRecord(ctx->ev_consumed[0], s));
    launch_cluster(d, L);
    launch_ev_scan(d, s, int(offsetof(EvInfo, n_hits)), int(offsetof(EvInfo, hit_base)));
    launch_ev_clamp(d, s, int(offsetof(EvInfo, n_hits)), int(offsetof(EvInfo, hit_base)), d.cap_hits);
  }
  if (mask & PXL_STAGE_HITS) launch_rechits(d, L);
  if (mask & PXL_STAGE_TUPLES) launch_ca(d, L);
  if (mask & PXL_STAGE_FIT) launch_fit(d, L);
  if (mask & PXL_STAGE_CLASSIFY) launch_classify(d, L);
  if (mask & PXL_STAGE_VERTICES) launch_vertices(d, L);
  CK(cudaGetLastError());
  ctx->done_mask = (mask & PXL_STAGE_DIGIS) ? mask : (ctx->done_mask | mask);
  return 0;
}

// Records that the context's last work went to stream s.
int note_done(PxlCtx* ctx, cudaStream_t s) {
  CK(cudaEventRecord(ctx->last_done, s));
  if (s != ctx->stream) CK(cudaStreamWaitEvent(ctx->stream, ctx->last_done, 0));
  return 0;
}

int fetch_ev_impl(PxlCtx* ctx) {
  if (ctx->ev_host_valid) return 0;
  ctx->ev_host.resize(size_t(ctx->last_E) + 1);
  CK(cudaMemcpyAsync(ctx->ev_host.data(), ctx->d.ev, ctx->ev_host.size() * sizeof(EvInfo), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->ev_host_valid = true;
  return 0;
}

// Device -> host copy on the context's stream (ordered after its work, waiting for nothing else).
template <class T>
int64_t copy_dev(cudaStream_t s, const T* src, int64_t n, void* dst, int64_t max_bytes) {
  if (n < 0) return -1;
  if (dst && max_bytes > 0 && n > 0) {
    size_t nb = size_t(std::min<int64_t>(n * int64_t(sizeof(T)), max_bytes));
    if (cudaMemcpyAsync(dst, src, nb, cudaMemcpyDeviceToHost, s) != cudaSuccess) return PXL_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PXL_ERR_CUDA;
  }
  return n;
}

// 32-bit hit ids as the reference's 16-bit hindex_type; PXL_ERR_CAPACITY when an id does not fit
// (an extended-capacity event above 65535 hits)
int64_t copy_dev_u16(cudaStream_t s, const uint32_t* src, int64_t n, uint32_t add, void* dst, int64_t max_bytes) {
  if (n < 0) return -1;
  if (dst && max_bytes > 0 && n > 0) {
    std::vector<uint32_t> v(static_cast<size_t>(n));
    if (copy_dev(s, src, n, v.data(), n * 4) < 0) return PXL_ERR_CUDA;
    std::vector<uint16_t> w(static_cast<size_t>(n));
    for (int64_t k = 0; k < n; ++k) {
      const uint32_t x = v[size_t(k)] + add;
      if (x > 0xFFFFu) return PXL_ERR_CAPACITY;
      w[size_t(k)] = uint16_t(x);
    }
    std::memcpy(dst, w.data(), size_t(std::min<int64_t>(2 * n, max_bytes)));
  }
  return n;
}

template <class T>
int64_t copy_host(const std::vector<T>& v, void* dst, int64_t max_bytes) {
  if (dst && max_bytes > 0 && !v.empty())
    std::memcpy(dst, v.data(), size_t(std::min<int64_t>(int64_t(v.size() * sizeof(T)), max_bytes)));
  return int64_t(v.size());
}

template <class T>
std::vector<T> dvec(cudaStream_t s, const T* src, int64_t n) {
  std::vector<T> v(size_t(std::max<int64_t>(n, 0)));
  if (n > 0) copy_dev(s, src, n, v.data(), n * int64_t(sizeof(T)));
  return v;
}

// Host -> device copy of a batch into input slot k on stream s, ordered after the last chain
// that read the slot; the slot's pinned offsets are reused only once their previous copy ended.
int stage_slot(PxlCtx* ctx, int k, const uint8_t* blob, const uint64_t* offs, int32_t n, cudaStream_t s) {
  if (n <= 0 || n > ctx->p.max_events) return PXL_ERR_ARG;
  uint64_t base = offs[0], nbytes = offs[n] - offs[0];
  if (offs[n] < offs[0] || nbytes > ctx->raw_cap) return PXL_ERR_CAPACITY;
  CK(cudaEventSynchronize(ctx->ev_staged[k]));
  for (int32_t e = 0; e <= n; ++e) ctx->h_off[k][e] = offs[e] - base;
  CK(cudaStreamWaitEvent(s, ctx->ev_consumed[k], 0));
  CK(cudaMemcpyAsync(ctx->d_raw[k], blob + base, nbytes, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(ctx->d_ev_off[k], ctx->h_off[k], size_t(n + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
  CK(cudaEventRecord(ctx->ev_staged[k], s));
  ctx->slot_E[k] = n;
  return 0;
}

int stage_input(PxlCtx* ctx, const uint8_t* blob, const uint64_t* offs, int32_t n, bool on_device, cudaStream_t s) {
  if (n <= 0 || n > ctx->p.max_events) return PXL_ERR_ARG;
  if (on_device) {
    ctx->d.raw = blob;
    ctx->d.ev_off = offs;
  } else {
    int rc = stage_slot(ctx, 0, blob, offs, n, s);
    if (rc) return rc;
    ctx->d.raw = ctx->d_raw[0];
    ctx->d.ev_off = ctx->d_ev_off[0];
  }
  ctx->d.E = n;
  ctx->last_E = n;
  ctx->ev_host_valid = false;
  return 0;
}

int choose_shape(PxlCtx* ctx) {
  Dev& d = ctx->d;
  if (ctx->p.blocks_per_event > 0) { d.bpe = ctx->p.blocks_per_event; return 0; }
  // modules-per-event CTAs: enough CTAs to fill 148 SMs x 8 resident CTAs with few events,
  // at least one wave of modules per event otherwise
  int target = 148 * 8;
  int bpe = std::max(1, std::min(256, target / std::max(1, d.E)));
  d.bpe = std::max(bpe, 4);
  return 0;
}

// Captures run_chain(mask) over the current input pointers into slot k's graph.
int capture_slot(PxlCtx* ctx, int k, uint32_t mask) {
  if (ctx->graph_exec[k]) { cudaGraphExecDestroy(ctx->graph_exec[k]); ctx->graph_exec[k] = nullptr; }
  if (ctx->graph[k]) { cudaGraphDestroy(ctx->graph[k]); ctx->graph[k] = nullptr; }
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  ctx->capturing = true;
  int rc = run_chain(ctx, mask, ctx->stream);
  ctx->capturing = false;
  cudaGraph_t g = nullptr;
  cudaError_t err = cudaStreamEndCapture(ctx->stream, &g);
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  if (err != cudaSuccess) { std::fprintf(stderr, "pxl: capture failed: %s\n", cudaGetErrorString(err)); return PXL_ERR_CUDA; }
  ctx->graph[k] = g;
  CK(cudaGraphInstantiate(&ctx->graph_exec[k], g, 0));
  return 0;
}

int launch_slot(PxlCtx* ctx, int k, cudaStream_t s) {
  CK(cudaStreamWaitEvent(s, ctx->ev_staged[k], 0));
  CK(cudaGraphLaunch(ctx->graph_exec[k], s));
  CK(cudaEventRecord(ctx->ev_consumed[k], s));
  if (int rc = note_done(ctx, s)) return rc;
  ctx->ev_host_valid = false;
  ctx->last_E = ctx->graph_E;
  ctx->last_mask = ctx->graph_mask;
  return 0;
}
}  // namespace

int pxl_fetch_ev(PxlCtx* ctx) { return fetch_ev_impl(ctx); }
static int fetch_ev(PxlCtx* ctx) { return fetch_ev_impl(ctx); }

extern "C" {

int32_t pxl_version(void) { return PXL_ABI_VERSION; }

int32_t pxl_params_default(PxlParams* p) {
  if (!p) return PXL_ERR_ARG;
  std::memset(p, 0, sizeof(*p));
  p->device = 0;
  p->max_events = 1;
  p->max_words = 300000;  // MAX_FED_WORDS = 150 * 2000 (SiPixelRawToClusterGPUKernel.jl:193)
  p->max_hits = 48 * 1024;
  p->max_doublets = 458752;
  p->max_tuples = 32 * 1024;
  p->hits_per_event = 48 * 1024;
  p->doublets_per_event = 458752;
  p->tuples_per_event = 32 * 1024;
  p->fits_per_multiplicity = 24 * 1024;
  p->include_errors = 1;
  p->use_quality = 1;
  p->blocks_per_event = 0;
  p->threads_per_block = 0;
  p->columns_per_event = kMaxActiveColumns;
  return 0;
}

int32_t pxl_params_extended(PxlParams* p) {
  const int32_t rc = pxl_params_default(p);
  if (rc) return rc;
  p->hits_per_event = 256 * 1024;
  p->doublets_per_event = 4 * 1024 * 1024;
  p->tuples_per_event = 256 * 1024;
  p->fits_per_multiplicity = 256 * 1024;
  p->columns_per_event = 4 * 1024 * 1024;
  return 0;
}

int32_t pxl_ctx_create(const PxlConditions* cond, const PxlParams* params, PxlCtx** out) {
  if (!cond || !out) return PXL_ERR_ARG;
  *out = nullptr;
  PxlCtx* ctx = new PxlCtx();
  if (params) ctx->p = *params;
  else pxl_params_default(&ctx->p);
  // event-local hit ids take kHitIdBits bits in the doublet search's hit records
  const PxlParams& q = ctx->p;
  if (q.max_events <= 0 || q.hits_per_event <= 0 || uint32_t(q.hits_per_event) > kMaxHitsPerEvent ||
      q.doublets_per_event <= 0 || q.tuples_per_event <= 0 || q.fits_per_multiplicity <= 0 ||
      q.columns_per_event <= 0 || q.fit_precision < 0 || q.fit_precision > 1) {
    delete ctx;
    return PXL_ERR_ARG;
  }
  if (cudaSetDevice(ctx->p.device) != cudaSuccess) { delete ctx; return PXL_ERR_CUDA; }
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) { delete ctx; return PXL_ERR_CUDA; }
  if (cudaEventCreateWithFlags(&ctx->last_done, cudaEventDisableTiming) != cudaSuccess) {
    pxl_ctx_destroy(ctx);
    return PXL_ERR_CUDA;
  }
  int rc = (prepare_select_kernels() || prepare_ca_kernels(ctx->wq_ctas)) ? PXL_ERR_CUDA : 0;
  if (!rc) rc = load_conditions(ctx, cond);
  if (!rc) rc = alloc_batch(ctx);
  if (rc) { pxl_ctx_destroy(ctx); return rc; }
  *out = ctx;
  return 0;
}

int32_t pxl_ctx_destroy(PxlCtx* ctx) {
  if (!ctx) return PXL_ERR_ARG;
  cudaSetDevice(ctx->p.device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (int k = 0; k < PxlCtx::kSlots; ++k) {
    if (ctx->ev_staged[k]) cudaEventSynchronize(ctx->ev_staged[k]);
    if (ctx->ev_consumed[k]) cudaEventSynchronize(ctx->ev_consumed[k]);
    if (ctx->graph_exec[k]) cudaGraphExecDestroy(ctx->graph_exec[k]);
    if (ctx->graph[k]) cudaGraphDestroy(ctx->graph[k]);
    if (ctx->h_off[k]) cudaFreeHost(ctx->h_off[k]);
    if (ctx->ev_staged[k]) cudaEventDestroy(ctx->ev_staged[k]);
    if (ctx->ev_consumed[k]) cudaEventDestroy(ctx->ev_consumed[k]);
  }
  if (ctx->last_done) { cudaEventSynchronize(ctx->last_done); cudaEventDestroy(ctx->last_done); }
  for (auto& x : ctx->exp) {
    if (x.copied) { cudaEventSynchronize(x.copied); cudaEventDestroy(x.copied); }
    if (x.ready) cudaEventDestroy(x.ready);
  }
  for (void* q : ctx->allocs) cudaFree(q);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return 0;
}

int32_t pxl_batch_stage(PxlCtx* ctx, const uint8_t* blob, const uint64_t* offs, int32_t n, void* stream) {
  if (!ctx || !blob || !offs) return PXL_ERR_ARG;
  cudaSetDevice(ctx->p.device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  return stage_input(ctx, blob, offs, n, false, s);
}

int32_t pxl_batch_run(PxlCtx* ctx, const uint8_t* blob, const uint64_t* offs, int32_t n, int32_t on_device,
                      uint32_t mask, void* stream) {
  if (!ctx || !blob || !offs) return PXL_ERR_ARG;
  cudaSetDevice(ctx->p.device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  int rc = stage_input(ctx, blob, offs, n, on_device != 0, s);
  if (rc) return rc;
  choose_shape(ctx);
  ctx->last_mask = mask;
  rc = run_chain(ctx, mask, s);
  if (rc) return rc;
  return note_done(ctx, s);
}

int32_t pxl_event_run(PxlCtx* ctx, const uint8_t* raw_event, size_t nbytes, uint32_t mask, void* stream) {
  if (!ctx || !raw_event) return PXL_ERR_ARG;
  uint64_t offs[2] = {0, nbytes};
  return pxl_batch_run(ctx, raw_event, offs, 1, 0, mask | PXL_STAGE_DIGIS, stream);
}

int32_t pxl_event_continue(PxlCtx* ctx, uint32_t mask, void* stream) {
  if (!ctx || ctx->d.E <= 0 || (mask & PXL_STAGE_DIGIS)) return PXL_ERR_ARG;
  if (!(ctx->done_mask & PXL_STAGE_DIGIS)) return PXL_ERR_STATE;
  // every stage needs the one before it
  for (uint32_t b = PXL_STAGE_HITS; b <= PXL_STAGE_VERTICES; b <<= 1)
    if ((mask & b) && !((ctx->done_mask | mask) & (b >> 1))) return PXL_ERR_STATE;
  cudaSetDevice(ctx->p.device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  ctx->ev_host_valid = false;
  int rc = run_chain(ctx, mask, s);
  ctx->last_mask |= mask;
  if (rc) return rc;
  return note_done(ctx, s);
}

int32_t pxl_graph_capture(PxlCtx* ctx, uint32_t mask) {
  if (!ctx || ctx->d.E <= 0) return PXL_ERR_STATE;
  cudaSetDevice(ctx->p.device);
  choose_shape(ctx);
  CK(cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < PxlCtx::kSlots; ++k) {
    if (ctx->graph_exec[k]) { cudaGraphExecDestroy(ctx->graph_exec[k]); ctx->graph_exec[k] = nullptr; }
    if (ctx->graph[k]) { cudaGraphDestroy(ctx->graph[k]); ctx->graph[k] = nullptr; }
  }
  // slot 0 replays the current input (the context's own slot-0 buffer or a device batch)
  int rc = capture_slot(ctx, 0, mask);
  if (rc) return rc;
  // the other slots exist when the input is the context's own buffer
  if (ctx->d.raw == ctx->d_raw[0]) {
    const uint8_t* raw0 = ctx->d.raw;
    const uint64_t* off0 = ctx->d.ev_off;
    for (int k = 1; k < PxlCtx::kSlots && !rc; ++k) {
      ctx->d.raw = ctx->d_raw[k];
      ctx->d.ev_off = ctx->d_ev_off[k];
      rc = capture_slot(ctx, k, mask);
    }
    ctx->d.raw = raw0;
    ctx->d.ev_off = off0;
    if (rc) return rc;
  }
  ctx->graph_mask = mask;
  ctx->graph_E = ctx->d.E;
  ctx->last_mask = mask;
  return 0;
}

int32_t pxl_graph_launch(PxlCtx* ctx, void* stream) {
  if (!ctx || !ctx->graph_exec[0]) return PXL_ERR_STATE;
  cudaSetDevice(ctx->p.device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  return launch_slot(ctx, 0, s);
}

int32_t pxl_slot_stage(PxlCtx* ctx, int32_t slot, const uint8_t* blob, const uint64_t* offs, int32_t n,
                       void* copy_stream) {
  if (!ctx || !blob || !offs || slot < 0 || slot >= PxlCtx::kSlots) return PXL_ERR_ARG;
  cudaSetDevice(ctx->p.device);
  cudaStream_t s = copy_stream ? static_cast<cudaStream_t>(copy_stream) : ctx->stream;
  return stage_slot(ctx, slot, blob, offs, n, s);
}

int32_t pxl_slot_launch(PxlCtx* ctx, int32_t slot, void* stream) {
  if (!ctx || slot < 0 || slot >= PxlCtx::kSlots) return PXL_ERR_ARG;
  if (!ctx->graph_exec[slot] || ctx->slot_E[slot] != ctx->graph_E) return PXL_ERR_STATE;
  cudaSetDevice(ctx->p.device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  return launch_slot(ctx, slot, s);
}

int64_t pxl_results_async(PxlCtx* ctx, uint32_t* host_dst, int64_t max_events, void* stream) {
  if (!ctx || !host_dst) return PXL_ERR_ARG;
  cudaSetDevice(ctx->p.device);
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  const int64_t n = std::min<int64_t>(max_events, ctx->last_E);
  if (n <= 0) return 0;
  // one uint32 (n_vtx) per event, gathered from the per-event records
  CK(cudaStreamWaitEvent(s, ctx->last_done, 0));
  CK(cudaMemcpy2DAsync(host_dst, sizeof(uint32_t), &ctx->d.ev[0].n_vtx, sizeof(EvInfo), sizeof(uint32_t), size_t(n),
                       cudaMemcpyDeviceToHost, s));
  return n;
}

int32_t pxl_graph_kernel_nodes(PxlCtx* ctx) {
  if (!ctx || !ctx->graph[0]) return PXL_ERR_STATE;
  size_t n = 0;
  CK(cudaGraphGetNodes(ctx->graph[0], nullptr, &n));
  std::vector<cudaGraphNode_t> nodes(n);
  CK(cudaGraphGetNodes(ctx->graph[0], nodes.data(), &n));
  int32_t k = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    CK(cudaGraphNodeGetType(nd, &t));
    if (t == cudaGraphNodeTypeKernel) ++k;
  }
  return k;
}

int32_t pxl_profile_enable(PxlCtx* ctx, int32_t on) {
  if (!ctx) return PXL_ERR_ARG;
  cudaSetDevice(ctx->p.device);
  if (on && !ctx->prof.ev[0])
    for (int i = 0; i < Prof::kMax; ++i) CK(cudaEventCreate(&ctx->prof.ev[i]));
  ctx->prof.on = on != 0;
  ctx->prof.n = 0;
  return 0;
}

int32_t pxl_profile_read(PxlCtx* ctx, float* ms, const char** names, int32_t max) {
  if (!ctx || !ms) return PXL_ERR_ARG;
  cudaSetDevice(ctx->p.device);
  CK(cudaStreamSynchronize(ctx->stream));
  int32_t k = 0;
  for (int i = 1; i < ctx->prof.n && k < max; ++i, ++k) {
    CK(cudaEventElapsedTime(&ms[k], ctx->prof.ev[i - 1], ctx->prof.ev[i]));
    if (names) names[k] = ctx->prof.name[i];
  }
  return k;
}

int32_t pxl_autotune(PxlCtx* ctx, const int32_t* candidates, int32_t n_candidates, int32_t reps, int32_t* chosen) {
  if (!ctx || !candidates || n_candidates <= 0 || n_candidates > 32 || reps <= 0) return PXL_ERR_ARG;
  if (ctx->d.E <= 0) return PXL_ERR_STATE;
  for (int i = 0; i < n_candidates; ++i)
    if (candidates[i] == 0 || candidates[i] > 4096 || candidates[i] < -64) return PXL_ERR_ARG;
  // timed segments (names given by the launchers) and the stage each one tunes
  static const struct { const char* name; int seg; } kMap[] = {
      {"doublets_count", kTuneDoublets}, {"doublets_fill", kTuneDoublets}, {"outer_hit_lists", kTuneHitLists},
      {"connect", kTuneConnect}, {"neighbour_lists", kTuneCellLists}, {"fishbone", kTuneFishbone},
      {"ntuplets_count", kTuneNtuplets}, {"ntuplets_fill", kTuneNtuplets}, {"cell_tracks", kTuneCellTracks},
      {"dup_multiplicity", kTuneEarlyDup}, {"classify", kTuneClassify},
      {"hit_to_tuple", kTuneHitToTuple}, {"triplet_cleaner", kTuneHitToTuple},
      {"broken_line_fit_3", kTuneFitTuples}, {"broken_line_fit_4", kTuneFitTuples}};
  cudaSetDevice(ctx->p.device);
  const bool prof_was = ctx->prof.on;
  int rc = pxl_profile_enable(ctx, 1);
  if (rc) return rc;
  double best_t[kTuneCount];
  int best_b[kTuneCount];
  for (int s = 0; s < kTuneCount; ++s) { best_t[s] = 1e300; best_b[s] = 0; }
  for (int c = 0; c < n_candidates; ++c) {
    for (int s = 0; s < kTuneCount; ++s) ctx->tune[s] = candidates[c];
    double acc[kTuneCount] = {};
    for (int r = 0; r <= reps; ++r) {  // the first run of each shape is a warm-up
      rc = run_chain(ctx, 0x3F, ctx->stream);
      if (rc) break;
      CK(cudaStreamSynchronize(ctx->stream));
      CK(cudaGetLastError());
      if (r == 0) continue;
      for (int i = 1; i < ctx->prof.n; ++i) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ctx->prof.ev[i - 1], ctx->prof.ev[i]));
        for (const auto& m : kMap)
          if (std::strcmp(m.name, ctx->prof.name[i]) == 0) acc[m.seg] += ms;
      }
    }
    if (rc) break;
    for (int s = 0; s < kTuneCount; ++s)
      if (acc[s] < best_t[s]) { best_t[s] = acc[s]; best_b[s] = candidates[c]; }
  }
  for (int s = 0; s < kTuneCount; ++s) {
    ctx->tune[s] = rc ? 0 : best_b[s];
    if (chosen) chosen[s] = ctx->tune[s];
  }
  ctx->last_mask = 0x3F;
  ctx->done_mask = 0x3F;
  ctx->ev_host_valid = false;
  pxl_profile_enable(ctx, prof_was ? 1 : 0);
  return rc;
}

int32_t pxl_sync(PxlCtx* ctx) {
  if (!ctx) return PXL_ERR_ARG;
  cudaSetDevice(ctx->p.device);
  // waits for this context's work only (its stream is ordered after the last work it enqueued)
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaGetLastError());
  ctx->ev_host_valid = false;
  int rc = fetch_ev(ctx);
  if (rc) return rc;
  uint32_t w = 0;
  for (int e = 0; e < ctx->last_E; ++e) w |= ctx->ev_host[e].warnings;
  uint32_t st = 0;
  if (copy_dev(ctx->stream, ctx->d.status, 1, &st, 4) < 0) return PXL_ERR_CUDA;
  return int32_t(w | st);
}

int32_t pxl_event_counts(PxlCtx* ctx, int32_t e, PxlEventCounts* out) {
  if (!ctx || !out || e < 0 || e >= ctx->last_E) return PXL_ERR_ARG;
  cudaSetDevice(ctx->p.device);
  int rc = fetch_ev(ctx);
  if (rc) return rc;
  const EvInfo& E = ctx->ev_host[e];
  out->n_words = E.n_words;
  out->n_modules = E.n_modules;
  out->n_clusters = E.n_clusters;
  out->n_hits = E.n_hits;
  out->n_doublets = E.n_cells;
  out->n_tuples = E.n_tuples;
  out->n_tuple_hits = E.n_tuple_hits;
  out->n_vertices = E.n_vtx;
  out->n_vertex_tracks = E.n_vtx_tracks;
  out->warnings = E.warnings;
  out->n_errors = E.n_errors;
  out->n_fits_fp64 = E.n_refit3 + E.n_refit4;
  return 0;
}

int64_t pxl_copy_product(PxlCtx* ctx, int32_t e, int32_t product, void* dst, int64_t max_bytes) {
  if (!ctx || e < 0 || e >= ctx->last_E) return PXL_ERR_ARG;
  cudaSetDevice(ctx->p.device);
  if (fetch_ev(ctx)) return PXL_ERR_CUDA;
  const Dev& d = ctx->d;
  const cudaStream_t s = ctx->stream;
  const EvInfo& E = ctx->ev_host[e];
  const uint64_t wb = E.word_base, hb = E.hit_base;
  const int64_t nw = E.n_words, nh = E.n_hits;
  const size_t M1 = kMaxNumModules + 1;
  switch (product) {
    case PXL_P_XX: return copy_dev(s, d.xx + wb, nw, dst, max_bytes);
    case PXL_P_YY: return copy_dev(s, d.yy + wb, nw, dst, max_bytes);
    case PXL_P_ADC: return copy_dev(s, d.adc + wb, nw, dst, max_bytes);
    case PXL_P_MODULE_IND: return copy_dev(s, d.mid + wb, nw, dst, max_bytes);
    case PXL_P_CLUS: return copy_dev(s, d.clus + wb, nw, dst, max_bytes);
    case PXL_P_PDIGI: return copy_dev(s, d.pdigi + wb, nw, dst, max_bytes);
    case PXL_P_RAW_ID: return copy_dev(s, d.rawid + wb, nw, dst, max_bytes);
    case PXL_P_MODULE_START: return copy_dev(s, d.module_start + size_t(e) * M1, int64_t(M1), dst, max_bytes);
    case PXL_P_CLUS_IN_MODULE: return copy_dev(s, d.clus_in_module + size_t(e) * kMaxNumModules, kMaxNumModules, dst, max_bytes);
    case PXL_P_MODULE_ID: return copy_dev(s, d.module_id + size_t(e) * kMaxNumModules, kMaxNumModules, dst, max_bytes);
    case PXL_P_CLUS_MODULE_START: return copy_dev(s, d.clus_module_start + size_t(e) * M1, int64_t(M1), dst, max_bytes);
    case PXL_P_XL: return copy_dev(s, d.xl + hb, nh, dst, max_bytes);
    case PXL_P_YL: return copy_dev(s, d.yl + hb, nh, dst, max_bytes);
    case PXL_P_XERR: return copy_dev(s, d.xerr + hb, nh, dst, max_bytes);
    case PXL_P_YERR: return copy_dev(s, d.yerr + hb, nh, dst, max_bytes);
    case PXL_P_XG: return copy_dev(s, d.xg + hb, nh, dst, max_bytes);
    case PXL_P_YG: return copy_dev(s, d.yg + hb, nh, dst, max_bytes);
    case PXL_P_ZG: return copy_dev(s, d.zg + hb, nh, dst, max_bytes);
    case PXL_P_RG: return copy_dev(s, d.rg + hb, nh, dst, max_bytes);
    case PXL_P_IPHI: return copy_dev(s, d.iphi + hb, nh, dst, max_bytes);
    case PXL_P_CHARGE: return copy_dev(s, d.charge + hb, nh, dst, max_bytes);
    case PXL_P_XSIZE: return copy_dev(s, d.xsize + hb, nh, dst, max_bytes);
    case PXL_P_YSIZE: return copy_dev(s, d.ysize + hb, nh, dst, max_bytes);
    case PXL_P_DET_IND: return copy_dev(s, d.detind + hb, nh, dst, max_bytes);
    case PXL_P_HITS_LAYER_START: return copy_dev(s, d.hits_layer_start + size_t(e) * 11, 11, dst, max_bytes);
    case PXL_P_PHI_OFF: return copy_dev(s, d.phi_off + size_t(e) * kPhiTotBins, kPhiTotBins, dst, max_bytes);
    case PXL_P_PHI_BINS: return copy_dev_u16(s, d.phi_bins + hb, nh, 0, dst, max_bytes);
    case PXL_P_PHI_BINS32: return copy_dev(s, d.phi_bins + hb, nh, dst, max_bytes);
    case PXL_P_AVERAGE_GEOMETRY: return copy_host(ctx->avg_geom, dst, max_bytes);
    case PXL_P_ERRORS: {
      uint32_t total = 0;
      if (copy_dev(s, d.err_count, 1, &total, 4) < 0) return PXL_ERR_CUDA;
      total = std::min<uint32_t>(total, uint32_t(d.cap_words));
      std::vector<uint32_t> all = dvec(s, d.err, int64_t(total) * 5);
      std::vector<std::pair<uint32_t, std::array<uint32_t, 4>>> mine;
      for (uint32_t k = 0; k < total; ++k)
        if (all[5 * k] == uint32_t(e))
          mine.push_back({all[5 * k + 1], {all[5 * k + 2], all[5 * k + 3], all[5 * k + 4] & 0xFFu, all[5 * k + 4] >> 8}});
      std::sort(mine.begin(), mine.end(), [](auto& a, auto& b) { return a.first < b.first; });
      std::vector<uint32_t> v;
      for (auto& m : mine) v.insert(v.end(), m.second.begin(), m.second.end());
      return copy_host(v, dst, max_bytes);
    }
    default:
      break;
  }
  return copy_ca_product(ctx, e, product, dst, max_bytes);
}

int32_t pxl_clusterize_digis(PxlCtx* ctx, const uint16_t* id, const int16_t* x, const int16_t* y, const int32_t* adc,
                             int32_t n, int32_t apply_charge_cut, uint32_t* module_start, uint32_t* clus_in_module,
                             uint32_t* module_id, int32_t* clus, uint16_t* id_out) {
  if (!ctx || !id || !x || !y || !adc || n < 0 || n > ctx->d.cap_words) return PXL_ERR_ARG;
  cudaSetDevice(ctx->p.device);
  cudaStream_t s = ctx->stream;
  Dev d = ctx->d;
  d.E = 1;
  d.n_fed_slots = 1;
  d.apply_charge_cut = apply_charge_cut != 0;
  d.bpe = 148 * 4;
  EvInfo ev{};
  ev.n_words = uint32_t(n);
  CK(cudaMemcpyAsync(d.ev, &ev, sizeof(EvInfo), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d.mid, id, size_t(n) * 2, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d.xx, x, size_t(n) * 2, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d.yy, y, size_t(n) * 2, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d.adc, adc, size_t(n) * 4, cudaMemcpyHostToDevice, s));
  std::vector<int32_t> ci(size_t(std::max(n, 1)));
  for (int32_t i = 0; i < n; ++i) ci[size_t(i)] = i + 1;  // count_modules: clus[i] = i
  CK(cudaMemcpyAsync(d.clus, ci.data(), size_t(n) * 4, cudaMemcpyHostToDevice, s));
  uint32_t nw = uint32_t(n), zero = 0;
  CK(cudaMemcpyAsync(d.fed_nw, &nw, 4, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d.fed_wo, &zero, 4, cudaMemcpyHostToDevice, s));
  Launch L{s, d.bpe, 256};
  launch_modstart(d, L);
  launch_cluster(d, L);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(module_start, d.module_start, (kMaxNumModules + 1) * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(clus_in_module, d.clus_in_module, kMaxNumModules * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(module_id, d.module_id, kMaxNumModules * 4, cudaMemcpyDeviceToHost, s));
  if (n > 0) {
    CK(cudaMemcpyAsync(clus, d.clus, size_t(n) * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(id_out, d.mid, size_t(n) * 2, cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(s));
  ctx->ev_host_valid = false;
  ctx->last_E = 0;
  return 0;
}

}  // extern "C"
