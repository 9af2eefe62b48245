// Test infrastructure (CPU oracle): cellular-automaton doublets, connection,
// fishbone, ntuplet search, multiplicity and track classification, restated
// from the reference (plugin-PixelTriplets/gpu_pixel_doublets.jl:19-360,
// gpu_ca_cell.jl:28-270, gpu_fishbone.jl:4-63, circle_eq.jl:18-93,
// ca_hit_ntuplet_generator.jl:9-97, ca_hit_ntuplet_generator_kernels.jl:141-231,
// ca_hit_ntuplet_generator_kernels_impl.jl:25-362, CUDACore/hist_to_container.jl).
#include <algorithm>
#include <cmath>
#include <functional>

#include "oracle.h"

namespace orc {

namespace {

const int kNPairs = 19;
const uint8_t kLayerPairs[2 * kNPairs] = {0, 1, 0, 4, 0, 7, 1, 2, 1, 4, 1, 7, 4, 5, 7, 8, 2, 3, 2, 4,
                                          2, 7, 5, 6, 8, 9, 0, 2, 1, 3, 0, 5, 0, 8, 4, 6, 7, 9};
const int16_t kPhiCuts[kNPairs] = {522, 730, 730, 522, 626, 626, 522, 522, 626, 626, 626, 522, 522, 522, 522, 522, 522, 522, 522};
const double kMinZ[kNPairs] = {-20., 0., -30., -22., 10., -30., -70., -70., -22., 15., -30, -70., -70., -20., -22., 0, -30., -70., -70.};
const double kMaxZ[kNPairs] = {20., 30., 0., 22., 30., -10., 70., 70., 22., 30., -15., 70., 70., 20., 22., 30., 0., 70., 70.};
const double kMaxR[kNPairs] = {20., 9., 9., 20., 7., 7., 5., 5., 20., 6., 6., 5., 5., 20., 20., 9., 9., 9., 9.};

// CA parameters (ca_hit_ntuplet_generator.jl:9-30), stored as Float32 by Params.
const float kPtMin = float(0.899999976158);
const float kThetaBarrel = float(0.00200000009499);
const float kThetaForward = float(0.00300000002608);
const float kHardCurv = float(0.0328407224959);
const float kDcaInner = float(0.15000000596);
const float kDcaOuter = float(0.25);

// CircleEq{Float32}, circle_eq.jl:18-47 and dca0 :287-291
struct CircleEq {
  float xp, yp, c, alpha, beta;
  CircleEq(float x1, float y1, float x2, float y2, float x3, float y3) {
    bool no_flip = std::fabs(x3 - x1) < std::fabs(y3 - y1);
    float x1p = no_flip ? x1 - x2 : y1 - y2;
    float y1p = no_flip ? y1 - y2 : x1 - x2;
    float d12 = x1p * x1p + y1p * y1p;
    float x3p = no_flip ? x3 - x2 : y3 - y2;
    float y3p = no_flip ? y3 - y2 : x3 - x2;
    float d32 = x3p * x3p + y3p * y3p;
    float num = x1p * y3p - y1p * x3p;
    float det = d12 * y3p - d32 * y1p;
    float st2 = d12 * x3p - d32 * x1p;
    float seq = det * det + st2 * st2;
    float al2 = 1.0f / std::sqrt(seq);
    float be2 = -st2 * al2;
    float ct = 2.0f * num * al2;
    al2 *= det;
    xp = x2; yp = y2;
    c = no_flip ? ct : -ct;
    alpha = no_flip ? al2 : -be2;
    beta = no_flip ? be2 : -al2;
  }
  float dca0() const {
    float x = c * xp + alpha;
    float y = c * yp + beta;
    return std::sqrt(x * x + y * y) - 1.0f;
  }
};

// are_aligned, gpu_ca_cell.jl:130-136
bool are_aligned(float r1, float z1, float ri, float zi, float ro, float zo, float ptmin, float theta_cut) {
  float radius_diff = std::fabs(r1 - ro);
  float d13 = radius_diff * radius_diff + (z1 - zo) * (z1 - zo);
  float p_min = ptmin * std::sqrt(d13);
  float t = std::fabs(z1 * (ri - ro) + zi * (ro - r1) + zo * (r1 - ri));
  return t * p_min <= theta_cut * d13 * radius_diff;
}

inline uint32_t phi_bin(int16_t t) { return (uint32_t(int32_t(t >> 9)) & 127u) + 1u; }

}  // namespace

void ca_tuples(const Conditions&, EventOut& ev) {
  const uint32_t nh = ev.n_hits;
  const Caps& caps = ev.caps;
  // reset (resetCAHitNTupletGeneratorKernels, init_doublets)
  ev.cell_neighbors.init_lazy(kCellNeighborsRows, int(caps.columns));
  ev.cell_tracks.init_lazy(kCellTracksRows, int(caps.columns));
  ev.cell_neighbors.extend();
  ev.cell_tracks.extend();
  ev.outer_hit_of_cell.init(kMaxCellsPerHit, std::max<uint32_t>(nh, 1));
  ev.cells.clear();
  ev.n_cells = 0;
  ev.tuple_off.assign(caps.tuples + 1, 0);
  ev.tuple_hits.assign(caps.tuple_hits, 0);
  ev.quality.assign(caps.tuples, 0);
  ev.n_tuples = 0;
  ev.n_tuple_hits = 0;
  std::fill(ev.tm_off, ev.tm_off + 9, 0u);
  ev.tm_bins.assign(caps.multiplicity, 0);

  if (nh != 0) {
    // ---- doublets_from_histo, gpu_pixel_doublets.jl:121-360
    const uint32_t* offsets = ev.hits_layer_start;
    auto layer_size = [&](int li) { return offsets[li + 1] - offsets[li]; };  // li 0-based
    uint32_t ilcs[kNPairs];
    ilcs[0] = layer_size(kLayerPairs[0]);
    for (int i = 1; i < kNPairs; ++i) ilcs[i] = ilcs[i - 1] + layer_size(kLayerPairs[2 * i]);
    uint32_t n_tot = ilcs[kNPairs - 1];
    const int min_y_size_b1 = 36, min_y_size_b2 = 28, max_dy_size_12 = 28, max_dy_size = 20, max_dy_pred = 20;
    const float dz_dr_fact = float(8 * 0.0285 / 0.015);
    const float z0_cut = 12.f;
    const double min_radius = 0.5 * 87.78;
    const double min_radius_2t4 = 4. * min_radius * min_radius;
    int pid = 0;  // 0-based pair index
    for (uint32_t j = 0; j < n_tot; ++j) {
      while (j >= ilcs[pid]) ++pid;
      int inner = kLayerPairs[2 * pid], outer = kLayerPairs[2 * pid + 1];
      uint32_t h_off = 128u * uint32_t(outer);
      uint32_t i = (pid == 0) ? j : j - ilcs[pid - 1];
      i += offsets[inner];
      i += 1;  // 1-based hit id
      int16_t mi = ev.det_ind[i - 1];
      if (mi > 2000) continue;
      float me_z = ev.zg[i - 1];
      if (double(me_z) < kMinZ[pid] || double(me_z) > kMaxZ[pid]) continue;
      int32_t me_s = ev.ysize[i - 1];  // idealConditions: every ladder counts as outer
      if ((inner == 0 && outer > 3) && (me_s > 0 && me_s < min_y_size_b1)) continue;
      if ((inner == 1 && outer > 3) && (me_s > 0 && me_s < min_y_size_b2)) continue;
      int16_t me_p = ev.iphi[i - 1];
      float me_r = ev.rg[i - 1];
      int16_t cut = kPhiCuts[pid];
      uint32_t kl = phi_bin(int16_t(me_p - cut));
      uint32_t kh = phi_bin(int16_t(me_p + cut)) + 1;
      if (kh == 129) kh = 1;
      for (uint32_t cb = kl; cb != kh;) {
        uint32_t p = ev.phi_off[cb + h_off - 1] + 1;
        uint32_t e = ev.phi_off[cb + h_off] + 1;
        bool capped = false;
        for (; p < e; ++p) {
          uint32_t oi = ev.phi_bins[p - 1];
          if (!(oi > offsets[outer] && oi <= offsets[outer + 1])) ev.flags |= kFlagNeighbourOverflow;
          int16_t mo = ev.det_ind[oi - 1];
          if (mo > 2000) continue;
          {  // z0_cut_off, :69-74
            float zo = ev.zg[oi - 1], ro = ev.rg[oi - 1];
            float dr = ro - me_r;
            if (double(dr) > kMaxR[pid] || dr < 0 || std::fabs(me_z * ro - me_r * zo) > z0_cut * dr) continue;
          }
          int16_t mo_p = ev.iphi[oi - 1];
          int16_t dphi = int16_t(mo_p - me_p);
          int16_t i_dphi = int16_t(dphi < 0 ? -dphi : dphi);
          if (i_dphi > cut) continue;
          {  // z_size_cut, :79-88
            bool only_barrel = outer < 4;
            int16_t so = ev.ysize[oi - 1];
            int dy = inner == 0 ? max_dy_size_12 : max_dy_size;
            float zo = ev.zg[oi - 1], ro = ev.rg[oi - 1];
            bool kill;
            if (only_barrel) {
              kill = me_s > 0 && so > 0 && std::abs(int(int16_t(so - int16_t(me_s)))) > dy;
            } else {
              kill = false;
              if (inner < 4 && me_s > 0) {
                float t = std::fabs((me_z - zo) / (me_r - ro)) * dz_dr_fact;
                double tt = double(t) + 0.5;
                if (!std::isfinite(tt)) { ev.flags |= kFlagFitDomain; continue; }
                int64_t pred = int64_t(std::trunc(tt));
                kill = std::llabs(int64_t(me_s) - pred) > max_dy_pred;
              }
            }
            if (kill) continue;
          }
          {  // pt_cut, :61-65
            float ro = ev.rg[oi - 1];
            double dphi_f = double(i_dphi) * ((2 * M_PI) / double(1 << 16));
            float rr = me_r * ro;
            float dd = ro - me_r;
            if (dphi_f * dphi_f * (min_radius_2t4 - double(rr)) > double(dd * dd)) continue;
          }
          ev.n_cells += 1;
          if (ev.n_cells > caps.doublets) { ev.n_cells -= 1; ev.flags |= kFlagDoubletsCapped; capped = true; break; }
          Cell c;
          c.outer_neighbors = 1; c.tracks = 1; c.doublet_id = int32_t(ev.n_cells); c.layer_pair_id = int16_t(pid + 1);
          c.used = 0; c.inner_z = ev.zg[i - 1]; c.inner_r = ev.rg[i - 1]; c.inner_hit = i; c.outer_hit = oi;
          ev.cells.push_back(c);
          ev.outer_hit_of_cell.push(oi, ev.n_cells);
        }
        (void)capped;
        cb = cb + 1;
        if (cb == 129) cb = 1;
      }
    }
  }

  // ---- launch_kernels, ca_hit_ntuplet_generator_kernels.jl:265-317
  std::vector<Cell>& cells = ev.cells;
  if (ev.n_cells && true) {
    // kernel_connect, …_impl.jl:45-114
    for (uint32_t idx = 1; idx <= ev.n_cells; ++idx) {
      Cell tc = cells[idx - 1];
      uint32_t ih = tc.inner_hit;
      uint32_t nposs = ev.outer_hit_of_cell.length(ih);
      float ri = tc.inner_r, zi = tc.inner_z;
      float ro = ev.rg[tc.outer_hit - 1], zo = ev.zg[tc.outer_hit - 1];
      bool is_barrel = ev.det_ind[tc.inner_hit - 1] < 1184;
      for (uint32_t k = 0; k < nposs; ++k) {
        uint32_t oc = ev.outer_hit_of_cell.at(ih, k);
        const Cell& o = cells[oc - 1];
        float r1 = o.inner_r, z1 = o.inner_z;
        bool aligned = are_aligned(r1, z1, ri, zi, ro, zo, kPtMin, is_barrel ? kThetaBarrel : kThetaForward);
        float region = ev.det_ind[o.inner_hit - 1] < 96 ? kDcaInner : kDcaOuter;
        CircleEq eq(ev.xg[o.inner_hit - 1], ev.yg[o.inner_hit - 1], ev.xg[tc.inner_hit - 1], ev.yg[tc.inner_hit - 1],
                    ev.xg[tc.outer_hit - 1], ev.yg[tc.outer_hit - 1]);
        bool cut;
        if (eq.c > kHardCurv) cut = false;
        else cut = std::fabs(eq.dca0()) < region * std::fabs(eq.c);
        if (aligned && cut) {
          Cell& oo = cells[oc - 1];
          if (oo.outer_neighbors == 1) {
            uint32_t col = ev.cell_neighbors.extend();
            if (col == caps.columns) ev.flags |= kFlagColumnsFull;
            if (col > 1) oo.outer_neighbors = col;
          }
          if (oo.outer_neighbors > 1) {
            if (ev.cell_neighbors.length(oo.outer_neighbors) == uint32_t(kCellNeighborsRows)) ev.flags |= kFlagNeighbourOverflow;
            ev.cell_neighbors.push(oo.outer_neighbors, idx);
          }
          cells[idx - 1].used |= 1;
          oo.used |= 1;
        }
      }
    }
    // fish_bone (early), gpu_fishbone.jl:4-63
    if (nh > 1) {
      float dx[kMaxCellsPerHit], dy[kMaxCellsPerHit], dz[kMaxCellsPerHit], norms[kMaxCellsPerHit];
      uint16_t idet[kMaxCellsPerHit];
      uint32_t cidx[kMaxCellsPerHit];
      for (uint32_t idy = 1; idy <= nh; ++idy) {
        uint32_t nout = ev.outer_hit_of_cell.length(idy);
        if (nout < 2) continue;
        const Cell& fc = cells[ev.outer_hit_of_cell.at(idy, 0) - 1];
        float xo = ev.xg[fc.outer_hit - 1], yo = ev.yg[fc.outer_hit - 1], zo = ev.zg[fc.outer_hit - 1];
        uint32_t curr = 0;
        for (uint32_t ic = 0; ic < nout; ++ic) {
          uint32_t ci = ev.outer_hit_of_cell.at(idy, ic);
          const Cell& c = cells[ci - 1];
          if (c.used == 0) continue;
          cidx[curr] = ci;
          idet[curr] = uint16_t(ev.det_ind[c.inner_hit - 1]);
          dx[curr] = ev.xg[c.inner_hit - 1] - xo;
          dy[curr] = ev.yg[c.inner_hit - 1] - yo;
          dz[curr] = c.inner_z - zo;
          norms[curr] = dx[curr] * dx[curr] + dy[curr] * dy[curr] + dz[curr] * dz[curr];
          ++curr;
        }
        if (curr < 2) continue;
        for (uint32_t ic = 0; ic + 1 < curr; ++ic) {
          for (uint32_t jc = ic + 1; jc < curr; ++jc) {
            float cos12 = dx[ic] * dx[jc] + dy[ic] * dy[jc] + dz[ic] * dz[jc];
            if (idet[ic] != idet[jc] && cos12 * cos12 >= 0.99999f * norms[ic] * norms[jc]) {
              if (norms[ic] > norms[jc]) { cells[cidx[ic] - 1].doublet_id = -1; break; }
              cells[cidx[jc] - 1].doublet_id = -1;
            }
          }
        }
      }
    }
    // kernel_find_ntuplets, …_impl.jl:116-132 with find_ntuplets, gpu_ca_cell.jl:232-270.
    // The temporary ntuplet is a Stack whose iteration runs from the top, so the reversed
    // fill puts the innermost hit first.
    uint32_t tmp[8];
    int depth = 0;
    auto emit = [&](const Cell& self) {
      uint32_t hits[6];
      int len = depth;
      for (int k = 0; k < len; ++k) hits[k] = cells[tmp[k] - 1].inner_hit;
      hits[len] = self.outer_hit;
      uint32_t n = uint32_t(len + 1);
      uint32_t c0 = ev.n_tuples, c1 = ev.n_tuple_hits;
      ev.n_tuples += 1;
      ev.n_tuple_hits += n;
      if (ev.n_tuples > caps.tuples) { ev.flags |= kFlagTuplesOverflow; return; }
      if (c1 + n > caps.tuple_hits) { ev.flags |= kFlagTuplesOverflow; return; }
      uint32_t it = ev.n_tuples;
      ev.tuple_off[it - 1] = c1 + 1;
      for (uint32_t k = 0; k < n; ++k) ev.tuple_hits[c1 + k] = hits[k];
      (void)c0;
      for (int k = len - 1; k >= 0; --k) {  // add_track over the stack, top first
        Cell& c = cells[tmp[k] - 1];
        if (c.tracks == 1) {
          uint32_t col = ev.cell_tracks.extend();
          if (col == caps.columns) ev.flags |= kFlagColumnsFull;
          if (col > 1) c.tracks = col;
        }
        if (c.tracks > 1) ev.cell_tracks.push(c.tracks, it);
      }
      ev.quality[it - 1] = 0;
    };
    std::function<void(const Cell&)> find;
    find = [&](const Cell& self) {
      tmp[depth++] = uint32_t(self.doublet_id);
      bool last = true;
      uint32_t col = self.outer_neighbors;
      uint32_t nn = ev.cell_neighbors.length(col);
      for (uint32_t k = 0; k < nn; ++k) {
        uint32_t other = ev.cell_neighbors.at(col, k);
        if (cells[other - 1].doublet_id < 0) continue;
        last = false;
        Cell oc = cells[other - 1];
        find(oc);
      }
      if (last && depth >= 2) emit(self);
      --depth;
    };
    for (uint32_t idx = 1; idx <= ev.n_cells; ++idx) {
      Cell tc = cells[idx - 1];
      if (tc.doublet_id < 0) continue;
      int p = tc.layer_pair_id - 1;
      bool do_it = (p < 8 || p > 12);  // minHitsPerNtuplet = 3
      if (do_it) find(tc);
    }
  }
  // bulk_finalize_fill, hist_to_container.jl:246-257
  {
    uint32_t m = ev.n_tuples, n = ev.n_tuple_hits;
    if (m > caps.tuples) ev.tuple_off[caps.tuples] = ev.tuple_off[caps.tuples - 1];
    else for (uint32_t i = m + 1; i <= caps.tuples + 1; ++i) ev.tuple_off[i - 1] = n + 1;
  }
  auto tsize = [&](uint32_t it) { return ev.tuple_off[it] - ev.tuple_off[it - 1]; };  // it 1-based
  // kernel_early_duplicate_remover, …_impl.jl:143-166
  for (uint32_t idx = 1; idx <= ev.n_cells; ++idx) {
    uint32_t col = cells[idx - 1].tracks;
    uint32_t nt = ev.cell_tracks.length(col);
    if (nt < 2) continue;
    uint32_t maxn = 0;
    for (uint32_t k = 0; k < nt; ++k) maxn = std::max(maxn, tsize(ev.cell_tracks.at(col, k)));
    for (uint32_t k = 0; k < nt; ++k) {
      uint32_t it = ev.cell_tracks.at(col, k);
      if (tsize(it) != maxn) ev.quality[it - 1] = 1;
    }
  }
  // kernel_countMultiplicity / finalize! / kernel_fillMultiplicity, :174-211
  uint32_t ntb = std::min<uint32_t>(ev.n_tuples, caps.tuples);
  for (uint32_t it = 1; it <= ntb; ++it) {
    uint32_t n = tsize(it);
    if (n < 3 || ev.quality[it - 1] == 1) continue;
    if (n < 9) ev.tm_off[n - 1] += 1;
  }
  for (int b = 1; b < 9; ++b) ev.tm_off[b] += ev.tm_off[b - 1];
  for (uint32_t it = 1; it <= ntb; ++it) {
    uint32_t n = tsize(it);
    if (n < 3 || ev.quality[it - 1] == 1) continue;
    if (n >= 9) continue;
    uint32_t w = ev.tm_off[n - 1];
    ev.tm_off[n - 1] -= 1;
    if (w >= 1 && w <= caps.multiplicity) ev.tm_bins[w - 1] = it;
  }
  // kernel_fill_hit_indices, :25-38
  ev.det_hits.assign(caps.tuple_hits, 0);
  uint32_t sz = std::min<uint32_t>(ev.tuple_off[caps.tuples] - 1, caps.tuple_hits);
  for (uint32_t k = 0; k < sz; ++k) ev.det_hits[k] = uint16_t(ev.det_ind[ev.tuple_hits[k] - 1]);
}

// classify_tuples, ca_hit_ntuplet_generator_kernels.jl:319-328
void classify_tuples(const Conditions&, EventOut& ev) {
  const Caps& caps = ev.caps;
  const uint32_t kNone = 0xFFFFFFFFu;  // no tuple (the reference's sentinel 60000 is above its 32K tuple ids)
  const float chi2_coeff[4] = {0.68177776f, 0.74609577f, -0.08035491f, 0.00315399f};
  const float chi2_max_pt = 10.0f, chi2_scale = 30.0f;
  const float trip_tip = 0.3f, trip_pt = 0.5f, trip_zip = 12.0f;
  const float quad_tip = 0.5f, quad_pt = 0.3f, quad_zip = 12.0f;
  auto tsize = [&](uint32_t it) { return ev.tuple_off[it] - ev.tuple_off[it - 1]; };
  auto tip = [&](uint32_t it) { return ev.state[size_t(it - 1) * 5 + 1]; };
  auto zip = [&](uint32_t it) { return ev.state[size_t(it - 1) * 5 + 4]; };
  // kernel_classify_tracks, …_impl.jl:213-247
  for (uint32_t it = 1; it <= caps.tuples; ++it) {
    uint32_t n = tsize(it);
    if (n == 0) break;
    if (ev.quality[it - 1] == 1) continue;
    if (n < 3) continue;
    bool isnan_ = false;
    for (int k = 0; k < 5; ++k) isnan_ |= std::isnan(ev.state[size_t(it - 1) * 5 + k]);
    if (isnan_) continue;
    float pt = std::min(ev.pt[it - 1], chi2_max_pt);
    float chi2_cut = chi2_scale * (chi2_coeff[0] + pt * (chi2_coeff[1] + pt * (chi2_coeff[2] + pt * chi2_coeff[3])));
    if (3.0f * ev.chi2[it - 1] >= chi2_cut) continue;
    bool quad = n > 3;
    float mtip = quad ? quad_tip : trip_tip, mpt = quad ? quad_pt : trip_pt, mzip = quad ? quad_zip : trip_zip;
    bool ok = (std::fabs(tip(it)) < mtip) && (ev.pt[it - 1] > mpt) && (std::fabs(zip(it)) < mzip);
    if (ok) ev.quality[it - 1] = 2;
  }
  // kernel_fast_duplicate_remover, :250-279 (cells in order; later cells see earlier marks)
  for (uint32_t idx = 1; idx <= ev.n_cells; ++idx) {
    uint32_t col = ev.cells[idx - 1].tracks;
    uint32_t nt = ev.cell_tracks.length(col);
    if (nt < 2) continue;
    float mc = 10000.f;
    uint32_t im = kNone;
    for (uint32_t k = 0; k < nt; ++k) {
      uint32_t it = ev.cell_tracks.at(col, k);
      if (ev.quality[it - 1] == 2 && std::fabs(tip(it)) < mc) { mc = std::fabs(tip(it)); im = it; }
    }
    for (uint32_t k = 0; k < nt; ++k) {
      uint32_t it = ev.cell_tracks.at(col, k);
      if (ev.quality[it - 1] != 0 && it != im) ev.quality[it - 1] = 1;
    }
  }
  // kernel_count_hit_in_tracks / finalize! / kernel_fill_hit_in_tracks, :281-311
  const uint32_t nbins = caps.hits;  // HitToTuple bins, one per hit id
  ev.hit_to_tuple_off.assign(nbins + 1, 0);
  ev.hit_to_tuple_bins.assign(caps.hit_to_tuple, 0);
  for (uint32_t it = 1; it <= caps.tuples; ++it) {
    if (tsize(it) == 0) break;
    if (ev.quality[it - 1] != 2) continue;
    for (uint32_t h = ev.tuple_off[it - 1]; h <= ev.tuple_off[it] - 1; ++h) ev.hit_to_tuple_off[ev.tuple_hits[h - 1] - 1] += 1;
  }
  for (uint32_t b = 1; b <= nbins; ++b) ev.hit_to_tuple_off[b] += ev.hit_to_tuple_off[b - 1];
  for (uint32_t it = 1; it <= caps.tuples; ++it) {
    if (tsize(it) == 0) break;
    if (ev.quality[it - 1] != 2) continue;
    for (uint32_t h = ev.tuple_off[it - 1]; h <= ev.tuple_off[it] - 1; ++h) {
      uint32_t b = ev.tuple_hits[h - 1];
      uint32_t w = ev.hit_to_tuple_off[b - 1];
      ev.hit_to_tuple_off[b - 1] -= 1;
      if (w >= 1 && w <= caps.hit_to_tuple) ev.hit_to_tuple_bins[w - 1] = it;
    }
  }
  // kernel_triplet_cleaner, :313-362
  for (uint32_t idx = 1; idx <= nbins; ++idx) {
    uint32_t b0 = ev.hit_to_tuple_off[idx - 1], b1 = ev.hit_to_tuple_off[idx];
    if (b1 - b0 < 2) continue;
    float mc = 10000.f;
    uint32_t im = kNone, maxnh = 0;
    for (uint32_t p = b0; p < b1; ++p) maxnh = std::max(maxnh, tsize(ev.hit_to_tuple_bins[p]));
    for (uint32_t p = b0; p < b1; ++p) {
      uint32_t it = ev.hit_to_tuple_bins[p];
      if (maxnh != tsize(it)) ev.quality[it - 1] = 1;
    }
    if (maxnh > 3) continue;
    for (uint32_t p = b0; p < b1; ++p) {
      uint32_t it = ev.hit_to_tuple_bins[p];
      if (ev.quality[it - 1] != 0 && std::fabs(tip(it)) < mc) { mc = std::fabs(tip(it)); im = it; }
    }
    for (uint32_t p = b0; p < b1; ++p) {
      uint32_t it = ev.hit_to_tuple_bins[p];
      if (ev.quality[it - 1] != 0 && it != im) ev.quality[it - 1] = 1;
    }
  }
}

}  // namespace orc
