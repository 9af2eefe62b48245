// Test infrastructure (CPU oracle): CPE rechits and the phi binner, restated
// from the reference (plugin-SiPixelRecHits/gpuPixelRecHits.jl:31-338,
// PixelRecHits.jl:20-82, CondFormats/pixelCPEforGPU.jl:246-577,
// Geometry/phase1PixelTopology.jl:249-296, DataFormats/SOARotation.jl:126-136,
// DataFormats/approx_atan2.jl:159-184, CUDACore/hist_to_container.jl:217-270).
// Arithmetic follows the reference's types: FP32 without contraction, one FP64
// expression in the charge-unbalance term.
#include <algorithm>
#include <cmath>

#include "oracle.h"

namespace orc {

namespace {

inline uint16_t local_x(uint16_t px) {
  int shift = 0;
  if (px > 79) shift += 1;
  if (px > 80) shift += 1;
  return uint16_t(px + shift);
}
inline uint16_t local_y(uint16_t py) {
  int roc = py / 52;
  int shift = 2 * roc;
  int yin = py - 52 * roc;
  if (yin > 0) shift += 1;
  return uint16_t(py + shift);
}
inline bool is_big_pix_x(uint32_t px) { return px == 79 || px == 80; }
inline bool is_big_pix_y(uint32_t py) { uint32_t ly = py - 52 * (py / 52); return ly == 0 || ly == 51; }

// approx_atan2s_P and unsafe_atan2s_impl, approx_atan2.jl:159-180
inline int16_t unsafe_atan2s(float y, float x) {
  const int16_t pi4 = 8192, pi34 = 24576;
  float r = (std::fabs(x) - std::fabs(y)) / (std::fabs(x) + std::fabs(y));
  if (x < 0) r = -r;
  int16_t angle = (x >= 0) ? pi4 : pi34;
  float z = r * r;
  float p = r * (-10422.177734375f + z * (3349.97412109375f + z * (-1525.589599609375f + z * 406.64190673828125f)));
  angle = int16_t(angle + int16_t(std::trunc(p)));
  return (y < 0) ? int16_t(-angle) : angle;
}

// correction, pixelCPEforGPU.jl:277-305
float correction(uint32_t sizeM1, int32_t q_f, int32_t q_l, uint16_t upper_edge_first_pix, uint16_t lower_edge_last_pix,
                 float lorentz_shift, float thickness, float cot_angle, float pitch, bool first_is_big, bool last_is_big) {
  if (sizeM1 == 0) return 0.0f;
  float w_eff = 0.0f;
  bool simple = true;
  if (sizeM1 == 1) {
    float w_inner = pitch * float(uint16_t(lower_edge_last_pix - upper_edge_first_pix));
    float w_pred = thickness * cot_angle - lorentz_shift;
    w_eff = std::fabs(w_pred) - w_inner;
    simple = (w_eff < 0.0f) || (w_eff > pitch);
  }
  if (simple) {
    float sum_of_edge = 2.0f;
    sum_of_edge += first_is_big ? 1.0f : 0.0f;
    sum_of_edge += last_is_big ? 1.0f : 0.0f;
    w_eff = pitch * 0.5f * sum_of_edge;
  }
  float qdiff = float(q_l - q_f);
  float qsum = float(q_l + q_f);
  qsum = qsum == 0.0f ? 1.0f : qsum;
  return 0.5f * (qdiff / qsum) * w_eff;
}

struct Clus {
  uint32_t min_row, max_row, min_col, max_col;
  int32_t q_f_x, q_l_x, q_f_y, q_l_y, charge;
  float xpos, ypos, xerr, yerr;
  int16_t xsize, ysize;
};

// position_corr, pixelCPEforGPU.jl:321-461
void position_corr(const CpeParams& cp, const DetParams& d, Clus& c) {
  uint16_t llx = uint16_t(c.min_row + 1), lly = uint16_t(c.min_col + 1);
  uint16_t urx = uint16_t(c.max_row), ury = uint16_t(c.max_col);
  uint16_t llxl = local_x(llx), llyl = local_y(lly), urxl = local_x(urx), uryl = local_y(ury);
  uint16_t mx = uint16_t(llxl + urxl), my = uint16_t(llyl + uryl);
  int64_t xsize = int64_t(urxl) + 2 - int64_t(llxl);
  int64_t ysize = int64_t(uryl) + 2 - int64_t(llyl);
  if (is_big_pix_x(c.min_row)) xsize += 1;
  if (is_big_pix_x(c.max_row)) xsize += 1;
  if (is_big_pix_y(c.min_col)) ysize += 1;
  if (is_big_pix_y(c.max_col)) ysize += 1;
  int32_t unb_x = int32_t(std::trunc(8.0 * double(std::fabs(float(c.q_f_x - c.q_l_x))) / double(float(c.q_f_x + c.q_l_x))));
  int32_t unb_y = int32_t(std::trunc(8.0 * double(std::fabs(float(c.q_f_y - c.q_l_y))) / double(float(c.q_f_y + c.q_l_y))));
  xsize = 8 * xsize - unb_x;
  ysize = 8 * ysize - unb_y;
  c.xsize = int16_t(uint32_t(std::min<int64_t>(xsize, 1023)));
  c.ysize = int16_t(uint32_t(std::min<int64_t>(ysize, 1023)));
  if (c.min_row == 0 || c.max_row == 159) c.xsize = int16_t(-c.xsize);
  if (c.min_col == 0 || c.max_col == 415) c.ysize = int16_t(-c.ysize);
  float xpos = d.shift_x + cp.pitch_x * (0.5f * float(mx) + float(int16_t(-81)));
  float ypos = d.shift_y + cp.pitch_y * (0.5f * float(my) + float(int16_t(-216)));
  float gvx = xpos - d.x0, gvy = ypos - d.y0, gvz = -1.0f / d.z0;
  float cotalpha = gvx * gvz, cotbeta = gvy * gvz;
  float thickness = d.is_barrel ? cp.thickness_b : cp.thickness_e;
  float xcorr = correction(c.max_row - c.min_row, c.q_f_x, c.q_l_x, llxl, urxl, d.charge_width_x, thickness, cotalpha,
                           cp.pitch_x, is_big_pix_x(c.min_row), is_big_pix_x(c.max_row));
  float ycorr = correction(c.max_col - c.min_col, c.q_f_y, c.q_l_y, llyl, uryl, d.charge_width_y, thickness, cotbeta,
                           cp.pitch_y, is_big_pix_y(c.min_col), is_big_pix_y(c.max_col));
  c.xpos = xpos + xcorr;
  c.ypos = ypos + ycorr;
}

// errorFromDB, pixelCPEforGPU.jl:542-577
void error_from_db(const DetParams& d, Clus& c) {
  c.xerr = 0.0050f;
  c.yerr = 0.0085f;
  uint32_t sx = c.max_row - c.min_row, sy = c.max_col - c.min_col;
  bool edge_x = c.min_row == 0 || c.max_row == 159;
  bool edge_y = c.min_col == 0 || c.max_col == 415;
  int ix = sx == 0 ? 1 : 0, iy = sy == 0 ? 1 : 0;
  ix += (sx == 0 && is_big_pix_x(c.min_row)) ? 1 : 0;
  iy += (sy == 0 && is_big_pix_y(c.min_col)) ? 1 : 0;
  if (!edge_x) c.xerr = d.sx[ix];
  if (!edge_y) c.yerr = d.sy[iy];
}

}  // namespace

void make_hits(const Conditions& cond, EventOut& ev) {
  const CpeParams& cp = cond.cpe;
  const BeamSpot& bs = cond.bs;
  // average geometry shifted by the beam spot, gpuPixelRecHits.jl:45-67
  for (int il = 0; il < kLadders; ++il) {
    ev.agc_ladder[0][il] = cp.ladder_z[il] - bs.z;
    ev.agc_ladder[1][il] = cp.ladder_x[il] - bs.x;
    ev.agc_ladder[2][il] = cp.ladder_y[il] - bs.y;
    ev.agc_ladder[3][il] = std::sqrt(ev.agc_ladder[1][il] * ev.agc_ladder[1][il] + ev.agc_ladder[2][il] * ev.agc_ladder[2][il]);
    ev.agc_ladder[4][il] = cp.ladder_minz[il] - bs.z;
    ev.agc_ladder[5][il] = cp.ladder_maxz[il] - bs.z;
  }
  ev.agc_endcap_z[0] = cp.endcap_z[0] - bs.z;
  ev.agc_endcap_z[1] = cp.endcap_z[1] - bs.z;

  uint32_t nh = ev.n_clusters;
  ev.n_hits = nh;
  ev.xl.assign(nh, 0.f); ev.yl.assign(nh, 0.f); ev.xerr.assign(nh, 0.f); ev.yerr.assign(nh, 0.f);
  ev.xg.assign(nh, 0.f); ev.yg.assign(nh, 0.f); ev.zg.assign(nh, 0.f); ev.rg.assign(nh, 0.f);
  ev.iphi.assign(nh, 0); ev.xsize.assign(nh, 0); ev.ysize.assign(nh, 0); ev.det_ind.assign(nh, 0);
  ev.charge.assign(nh, 0);
  const uint32_t n = ev.word_counter;
  const int max_iter = 160;  // MaxHitsInIter
  std::vector<Clus> cl(max_iter);
  if (ev.n_modules != 0) {
    for (uint32_t mod = 1; mod <= ev.module_start[0]; ++mod) {
      uint32_t me = ev.module_id[mod - 1];
      uint32_t nclus = ev.clus_in_module[me];
      if (nclus == 0) continue;
      const DetParams& d = cp.det[me];
      for (uint32_t start = 1; start <= nclus; start += max_iter) {
        uint32_t first = ev.module_start[mod];  // 1-based digi index
        uint32_t nin = std::min<uint32_t>(max_iter, nclus - start + 1);
        uint32_t last = start - 1 + nin;
        for (uint32_t ic = 0; ic < nin; ++ic) {
          cl[ic].min_row = 0xFFFFFFFFu; cl[ic].max_row = 0; cl[ic].min_col = 0xFFFFFFFFu; cl[ic].max_col = 0;
          cl[ic].charge = 0; cl[ic].q_f_x = cl[ic].q_l_x = cl[ic].q_f_y = cl[ic].q_l_y = 0;
        }
        for (uint32_t i = first; i <= n; ++i) {
          int16_t id = ev.module_ind[i - 1];
          if (id == int16_t(kInvId)) continue;
          if (uint32_t(int32_t(id)) != me) break;
          int32_t c = ev.clus[i - 1];
          if (c < int32_t(start) || c > int32_t(last)) continue;
          uint32_t x = uint32_t(int32_t(ev.xx[i - 1])), y = uint32_t(int32_t(ev.yy[i - 1]));
          Clus& k = cl[c - start];
          if (k.min_row > x) k.min_row = x;
          if (k.max_row < x) k.max_row = x;
          if (k.min_col > y) k.min_col = y;
          if (k.max_col < y) k.max_col = y;
        }
        for (uint32_t i = first; i <= n; ++i) {
          int16_t id = ev.module_ind[i - 1];
          if (id == int16_t(kInvId)) continue;
          if (uint32_t(int32_t(id)) != me) break;
          int32_t c = ev.clus[i - 1];
          if (c < int32_t(start) || c > int32_t(last)) continue;
          Clus& k = cl[c - start];
          uint32_t x = uint32_t(int32_t(ev.xx[i - 1])), y = uint32_t(int32_t(ev.yy[i - 1]));
          int32_t ch = std::min<int32_t>(ev.adc[i - 1], 65535);
          k.charge += ch;
          if (k.min_row == x) k.q_f_x += ch;
          if (k.max_row == x) k.q_l_x += ch;
          if (k.min_col == y) k.q_f_y += ch;
          if (k.max_col == y) k.q_l_y += ch;
        }
        uint32_t hfirst = ev.clus_module_start[me] + start;  // 1-based
        for (uint32_t ic = 0; ic < nin; ++ic) {
          uint32_t h = hfirst - 1 + ic + 1;  // 1-based hit index
          if (h > ev.caps.hits) break;
          Clus& k = cl[ic];
          position_corr(cp, d, k);
          error_from_db(d, k);
          uint32_t h0 = h - 1;
          if (h0 >= nh) { ev.flags |= kFlagHitsClamped; break; }
          ev.charge[h0] = uint32_t(k.charge);
          ev.det_ind[h0] = int16_t(me);
          ev.xl[h0] = k.xpos;
          ev.yl[h0] = k.ypos;
          ev.xsize[h0] = k.xsize;
          ev.ysize[h0] = k.ysize;
          ev.xerr[h0] = k.xerr * k.xerr;
          ev.yerr[h0] = k.yerr * k.yerr;
          // toGlobal_Special: multiplyInverse(R, xl, yl) + p, then minus the beam spot
          float vx = k.xpos, vy = k.ypos;
          float ux = d.R[0] * vx + d.R[3] * vy;
          float uy = d.R[1] * vx + d.R[4] * vy;
          float uz = d.R[2] * vx + d.R[5] * vy;
          ux += d.px; uy += d.py; uz += d.pz;
          float xg = ux - bs.x, yg = uy - bs.y, zg = uz - bs.z;
          ev.xg[h0] = xg; ev.yg[h0] = yg; ev.zg[h0] = zg;
          ev.rg[h0] = std::sqrt(xg * xg + yg * yg);
          ev.iphi[h0] = unsafe_atan2s(yg, xg);
        }
      }
    }
  }
  // setHitsLayerStart, PixelRecHits.jl:20-28
  for (int i = 0; i < 11; ++i) ev.hits_layer_start[i] = ev.clus_module_start[cp.layer_start[i]];
  // fill_many_from_vector(Hist{Int16,128,…,16,UInt16,10}), hist_to_container.jl:217-270
  std::fill(ev.phi_off, ev.phi_off + kPhiTotBins, 0u);
  ev.phi_bins.assign(nh, 0);
  if (nh == 0) return;
  const uint32_t* offs = ev.hits_layer_start;
  auto layer_of = [&](uint32_t i) -> int {
    int k = 0;
    while (k < 11 && offs[k] < i) ++k;  // searchsortedfirst (first offset >= i)
    return (k < 11 && offs[k] == i) ? k : k - 1;
  };
  auto binof = [](int16_t t) -> uint32_t { return (uint32_t(int32_t(t >> 9)) & 127u) + 1u; };
  uint32_t ntot = offs[10];
  for (uint32_t i = 0; i < ntot; ++i) {
    int ih = layer_of(i);
    uint32_t b = binof(ev.iphi[i]) + 128u * uint32_t(ih);
    ev.phi_off[b - 1] += 1;
  }
  for (int b = 1; b < kPhiTotBins; ++b) ev.phi_off[b] += ev.phi_off[b - 1];
  for (uint32_t i = 0; i < ntot; ++i) {
    int ih = layer_of(i);
    uint32_t b = binof(ev.iphi[i]) + 128u * uint32_t(ih);
    uint32_t w = ev.phi_off[b - 1];
    ev.phi_off[b - 1] -= 1;
    if (w >= 1 && w <= nh) ev.phi_bins[w - 1] = i + 1;
  }
}

}  // namespace orc
