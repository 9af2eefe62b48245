// Test infrastructure (CPU oracle): C-ABI used by tests/, smoke() and the
// cpu_baseline leg of bench.py to drive the oracle and read its products.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <thread>

#include "oracle.h"

using namespace orc;

struct OrcCtx {
  Conditions cond;
  EventOut ev;
  Options opt;
};

namespace {

template <class T>
int64_t put(const std::vector<T>& v, void* dst, int64_t max_bytes) {
  int64_t nb = int64_t(v.size() * sizeof(T));
  if (dst && max_bytes > 0) std::memcpy(dst, v.data(), size_t(std::min(nb, max_bytes)));
  return int64_t(v.size());
}
template <class T>
int64_t put_arr(const T* v, size_t n, void* dst, int64_t max_bytes) {
  int64_t nb = int64_t(n * sizeof(T));
  if (dst && max_bytes > 0) std::memcpy(dst, v, size_t(std::min(nb, max_bytes)));
  return int64_t(n);
}

// The per-event counts: the tuples are those the container keeps (at most the capacity, the
// last one of an overflowing container holding no hits), not the raw counter.
// The last count is the CountValidator's N(track): the TrackSOA's tuples with hits
// (count_to_validator.jl:50-55).
void event_counts(const EventOut& e, uint32_t* v) {
  const uint32_t nt = std::min(e.n_tuples, e.caps.tuples);
  const uint32_t nth = e.tuple_off.empty() ? 0u : e.tuple_off[nt] - 1;
  uint32_t with_hits = 0;
  for (uint32_t t = 0; t < nt; ++t) with_hits += e.tuple_off[t + 1] > e.tuple_off[t];
  const uint32_t c[12] = {e.word_counter, e.n_modules, e.n_clusters, e.n_hits, e.n_cells, nt, nth,
                          e.nv_final, e.n_vtx_tracks, e.flags, uint32_t(e.errors.size()), with_hits};
  std::memcpy(v, c, sizeof(c));
}

void run_event(const Conditions& c, const Options& o, const uint8_t* raw, size_t n, EventOut& ev) {
  ev.flags = 0;
  ev.caps = o.caps;
  raw_to_clusters(c, raw, n, o, ev);
  if (o.stage_mask & 2) make_hits(c, ev);
  if (o.stage_mask & 4) ca_tuples(c, ev);
  if (o.stage_mask & 8) fit_tuples(c, ev);
  if (o.stage_mask & 16) classify_tuples(c, ev);
  if (o.stage_mask & 32) make_vertices(c, ev);
}

}  // namespace

extern "C" {

OrcCtx* orc_ctx_create(const uint8_t* cab, size_t ncab, const uint8_t* fed, size_t nfed, const uint8_t* gain, size_t ngain,
                       const uint8_t* cpe, size_t ncpe, const uint8_t* bs, size_t nbs) {
  OrcCtx* c = new OrcCtx();
  if (parse_conditions(cab, ncab, fed, nfed, gain, ngain, cpe, ncpe, bs, nbs, &c->cond) != 0) { delete c; return nullptr; }
  return c;
}

void orc_ctx_destroy(OrcCtx* c) { delete c; }

// Per-event capacities (0 keeps a value): the reference's by default, larger ones for the
// extended mode. The tuple-hit, multiplicity and hit-to-tuple capacities follow the tuples.
void orc_set_caps(OrcCtx* c, uint32_t hits, uint32_t doublets, uint32_t tuples, uint32_t fits_per_mult,
                  uint32_t columns) {
  Caps& k = c->opt.caps;
  if (hits) k.hits = hits;
  if (doublets) k.doublets = doublets;
  if (tuples) {
    k.tuples = tuples;
    k.tuple_hits = 5 * tuples;
    k.multiplicity = std::max<uint32_t>(tuples, 48 * 1024);
    k.hit_to_tuple = 4 * k.multiplicity;
  }
  if (fits_per_mult) k.fits_per_mult = fits_per_mult;
  if (columns) k.columns = columns;
}

int32_t orc_run_event(OrcCtx* c, const uint8_t* raw, size_t nbytes, int32_t stage_mask) {
  c->opt.stage_mask = stage_mask;
  run_event(c->cond, c->opt, raw, nbytes, c->ev);
  return int32_t(c->ev.flags);
}

// counts: word_counter, n_modules, n_clusters, n_hits, n_cells, n_tuples, n_tuple_hits,
// nv_final, n_vtx_tracks, flags, n_errors, n_tracks
int32_t orc_counts(OrcCtx* c, uint32_t* out) {
  event_counts(c->ev, out);
  return 12;
}

// Copies a named product into dst (at most max_bytes); returns the element count, or -1.
int64_t orc_get(OrcCtx* c, const char* name, void* dst, int64_t max_bytes) {
  const EventOut& e = c->ev;
  std::string n(name);
  if (n == "words") return put(e.words, dst, max_bytes);
  if (n == "xx") return put(e.xx, dst, max_bytes);
  if (n == "yy") return put(e.yy, dst, max_bytes);
  if (n == "adc") return put(e.adc, dst, max_bytes);
  if (n == "module_ind") return put(e.module_ind, dst, max_bytes);
  if (n == "clus") return put(e.clus, dst, max_bytes);
  if (n == "pdigi") return put(e.pdigi, dst, max_bytes);
  if (n == "raw_id_arr") return put(e.raw_id_arr, dst, max_bytes);
  if (n == "module_start") return put_arr(e.module_start, kMaxNumModules + 1, dst, max_bytes);
  if (n == "clus_in_module") return put_arr(e.clus_in_module, kMaxNumModules, dst, max_bytes);
  if (n == "module_id") return put_arr(e.module_id, kMaxNumModules, dst, max_bytes);
  if (n == "clus_module_start") return put_arr(e.clus_module_start, kMaxNumModules + 1, dst, max_bytes);
  if (n == "xl") return put(e.xl, dst, max_bytes);
  if (n == "yl") return put(e.yl, dst, max_bytes);
  if (n == "xerr") return put(e.xerr, dst, max_bytes);
  if (n == "yerr") return put(e.yerr, dst, max_bytes);
  if (n == "xg") return put(e.xg, dst, max_bytes);
  if (n == "yg") return put(e.yg, dst, max_bytes);
  if (n == "zg") return put(e.zg, dst, max_bytes);
  if (n == "rg") return put(e.rg, dst, max_bytes);
  if (n == "iphi") return put(e.iphi, dst, max_bytes);
  if (n == "charge") return put(e.charge, dst, max_bytes);
  if (n == "xsize") return put(e.xsize, dst, max_bytes);
  if (n == "ysize") return put(e.ysize, dst, max_bytes);
  if (n == "det_ind") return put(e.det_ind, dst, max_bytes);
  if (n == "hits_layer_start") return put_arr(e.hits_layer_start, 11, dst, max_bytes);
  if (n == "phi_off") return put_arr(e.phi_off, kPhiTotBins, dst, max_bytes);
  if (n == "phi_bins") return put(e.phi_bins, dst, max_bytes);
  if (n == "agc") {
    std::vector<float> v;
    for (int k = 0; k < 6; ++k) v.insert(v.end(), e.agc_ladder[k], e.agc_ladder[k] + kLadders);
    v.push_back(e.agc_endcap_z[0]); v.push_back(e.agc_endcap_z[1]);
    return put(v, dst, max_bytes);
  }
  if (n == "cells") {  // per cell: inner, outer, layer_pair, doublet_id, used (int32 x 5)
    std::vector<int32_t> v;
    v.reserve(e.cells.size() * 5);
    for (auto& cc : e.cells) {
      v.push_back(cc.inner_hit); v.push_back(cc.outer_hit); v.push_back(cc.layer_pair_id); v.push_back(cc.doublet_id);
      v.push_back(cc.used);
    }
    return put(v, dst, max_bytes);
  }
  if (n == "cell_neighbors") {  // CSR over cells: n_cells+1 offsets then entries
    std::vector<uint32_t> v(e.cells.size() + 1, 0);
    std::vector<uint32_t> ent;
    for (size_t i = 0; i < e.cells.size(); ++i) {
      uint32_t col = e.cells[i].outer_neighbors;
      uint32_t l = e.cell_neighbors.length(col);
      for (uint32_t k = 0; k < l; ++k) ent.push_back(e.cell_neighbors.at(col, k));
      v[i + 1] = uint32_t(ent.size());
    }
    v.insert(v.end(), ent.begin(), ent.end());
    return put(v, dst, max_bytes);
  }
  if (n == "cell_tracks") {
    std::vector<uint32_t> v(e.cells.size() + 1, 0);
    std::vector<uint32_t> ent;
    for (size_t i = 0; i < e.cells.size(); ++i) {
      uint32_t col = e.cells[i].tracks;
      uint32_t l = e.cell_tracks.length(col);
      for (uint32_t k = 0; k < l; ++k) ent.push_back(e.cell_tracks.at(col, k));
      v[i + 1] = uint32_t(ent.size());
    }
    v.insert(v.end(), ent.begin(), ent.end());
    return put(v, dst, max_bytes);
  }
  if (n == "outer_hit_of_cell") {  // CSR over hits 1..n_hits
    std::vector<uint32_t> v(e.n_hits + 1, 0);
    std::vector<uint32_t> ent;
    for (uint32_t h = 1; h <= e.n_hits; ++h) {
      uint32_t l = e.outer_hit_of_cell.length(h);
      for (uint32_t k = 0; k < l; ++k) ent.push_back(e.outer_hit_of_cell.at(h, k));
      v[h] = uint32_t(ent.size());
    }
    v.insert(v.end(), ent.begin(), ent.end());
    return put(v, dst, max_bytes);
  }
  if (n == "tuple_off") return put(e.tuple_off, dst, max_bytes);
  if (n == "tuple_hits") return put(e.tuple_hits, dst, max_bytes);
  if (n == "det_hits") return put(e.det_hits, dst, max_bytes);
  if (n == "quality") return put(e.quality, dst, max_bytes);
  if (n == "tm_off") return put_arr(e.tm_off, 9, dst, max_bytes);
  if (n == "tm_bins") return put(e.tm_bins, dst, max_bytes);
  if (n == "pt") return put(e.pt, dst, max_bytes);
  if (n == "eta") return put(e.eta, dst, max_bytes);
  if (n == "chi2") return put(e.chi2, dst, max_bytes);
  if (n == "state") return put(e.state, dst, max_bytes);
  if (n == "cov") return put(e.cov, dst, max_bytes);
  if (n == "fitted") return put(e.fitted, dst, max_bytes);
  if (n == "hit_to_tuple_off") return put(e.hit_to_tuple_off, dst, max_bytes);
  if (n == "hit_to_tuple_bins") return put(e.hit_to_tuple_bins, dst, max_bytes);
  if (n == "idv") return put(e.idv, dst, max_bytes);
  if (n == "zv") return put(e.zv, dst, max_bytes);
  if (n == "wv") return put(e.wv, dst, max_bytes);
  if (n == "vchi2") return put(e.vchi2, dst, max_bytes);
  if (n == "ptv2") return put(e.ptv2, dst, max_bytes);
  if (n == "ndof") return put(e.ndof, dst, max_bytes);
  if (n == "sort_ind") return put(e.sort_ind, dst, max_bytes);
  if (n == "errors") {
    std::vector<uint32_t> v;
    for (auto& er : e.errors) { v.push_back(er.raw_id); v.push_back(er.word); v.push_back(er.error_type); v.push_back(er.fed_id); }
    return put(v, dst, max_bytes);
  }
  return -1;
}

// Clustering on digis alone, as the reference's clustering test drives it.
int32_t orc_clusterize_digis(const uint16_t* id, const int16_t* x, const int16_t* y, const int32_t* adc, int32_t n,
                             uint32_t* module_start, uint32_t* clus_in_module, uint32_t* module_id, int32_t* clus,
                             uint16_t* id_out, int32_t apply_charge_cut) {
  for (int i = 0; i < kMaxNumModules; ++i) clus_in_module[i] = 0;
  clusterize_digis(id, x, y, adc, n, module_start, clus_in_module, module_id, clus, id_out, apply_charge_cut);
  return 0;
}

// One broken-line fit in FP64 (see orc::bl_fit_track).
int32_t orc_bl_fit(const double* hits, const float* ge, int32_t n, double B, double* state5, double* cov15, double* chi2,
                   double* pt, double* eta, double* fast4) {
  double cl, cc;
  int rc = bl_fit_track(hits, ge, n, B, state5, cov15, &cl, &cc, pt, eta, fast4);
  chi2[0] = cl; chi2[1] = cc;
  return rc;
}

// Runs the full chain over events with n_threads host threads (event-parallel, like the
// reference's stream threads). Returns elapsed seconds; per-event counts go to
// counts[n_events * 12] when non-null.
double orc_run_batch(OrcCtx* c, const uint8_t* blob, const uint64_t* offsets, int32_t n_events, int32_t n_threads,
                     int32_t stage_mask, uint32_t* counts) {
  int nt = n_threads > 0 ? n_threads : 1;
  Options o = c->opt;
  o.stage_mask = stage_mask;
  auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) {
    th.emplace_back([&, t] {
      EventOut ev;
      for (int e = t; e < n_events; e += nt) {
        run_event(c->cond, o, blob + offsets[e], size_t(offsets[e + 1] - offsets[e]), ev);
        if (counts) event_counts(ev, counts + size_t(e) * 12);
      }
    });
  }
  for (auto& x : th) x.join();
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

// Riemann fit of one track
int32_t orc_riemann_fit(const double* hits, const float* ge, int32_t n, double B, double* state5, double* chi2,
                        double* pt) {
  return riemann_fit_track(hits, ge, n, B, state5, chi2, chi2 + 1, pt);
}

// forward-mode gradient of one track's chi2 (chi2_line + chi2_circle) w.r.t. its hits
double orc_bl_chi2_grad_fwd(const double* hits, const float* ge, int32_t n, double B, double* grad) {
  return bl_chi2_grad_fwd(hits, ge, n, B, grad);
}

// FP64 broken-line fits of n tracks (hits row-major per hit, offsets[n+1]) with n_threads
// host threads; state5[5n] and pt[n] (may be null) receive the results. Returns seconds.
double orc_bl_fit_batch(const double* hits, const float* ge, const int32_t* offsets, int32_t n, double B,
                        int32_t n_threads, double* state5, double* pt) {
  int nt = n_threads > 0 ? n_threads : 1;
  auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) {
    th.emplace_back([&, t] {
      for (int32_t k = t; k < n; k += nt) {
        const int32_t a = offsets[k], m = offsets[k + 1] - offsets[k];
        double st[5], cv[15], cl, cc, p, eta;
        bl_fit_track(hits + 3 * size_t(a), ge + 6 * size_t(a), m, B, st, cv, &cl, &cc, &p, &eta, nullptr);
        if (state5) for (int j = 0; j < 5; ++j) state5[5 * size_t(k) + j] = st[j];
        if (pt) pt[k] = p;
      }
    });
  }
  for (auto& x : th) x.join();
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // extern "C"
