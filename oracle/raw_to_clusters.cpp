// Test infrastructure (CPU oracle): conditions parsing and the raw -> digis ->
// clusters stage, restated from the reference (Maya-Ali0/CMS-Julia,
// src/julia-serial). See oracle.h for the oracle's role and its pinning.
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "oracle.h"

namespace orc {

namespace {

struct Reader {
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

}  // namespace

// SiPixelFedCablingMapGPUWrapperESProducer.jl:27-57, SiPixelGainCalibrationForHLTGPUESProducer.jl:14-46,
// PixelCPEFastESProducer.jl:16-103, BeamSpotESProducer.jl:11-28.
int parse_conditions(const uint8_t* cabling, size_t ncab, const uint8_t* fedids, size_t nfed, const uint8_t* gain,
                     size_t ngain, const uint8_t* cpe, size_t ncpe, const uint8_t* bs, size_t nbs, Conditions* out) {
  Conditions& c = *out;
  {
    Reader r{cabling, ncab};
    auto rd = [&](std::vector<uint32_t>& v) { v.resize(kCablingSize); r.get_n(v.data(), kCablingSize); };
    rd(c.cabling.fed); rd(c.cabling.link); rd(c.cabling.roc); rd(c.cabling.raw_id); rd(c.cabling.roc_in_det);
    rd(c.cabling.module_id);
    c.cabling.bad_rocs.resize(kCablingSize);
    r.get_n(c.cabling.bad_rocs.data(), kCablingSize);
    c.cabling.size = 0;
    if (!r.ok) return -1;
  }
  {
    Reader r{fedids, nfed};
    uint32_t n = r.get<uint32_t>();
    c.fed_ids.resize(n);
    r.get_n(c.fed_ids.data(), n);
    if (!r.ok) return -2;
  }
  {
    Reader r{gain, ngain};
    Gains& g = c.gains;
    r.skip(8);
    for (int i = 0; i < 2000; ++i) { g.rc[i].first = r.get<uint32_t>(); g.rc[i].last = r.get<uint32_t>(); g.rc[i].cols = r.get<int32_t>(); }
    g.min_ped = r.get<float>(); g.max_ped = r.get<float>(); g.min_gain = r.get<float>(); g.max_gain = r.get<float>();
    g.ped_precision = r.get<float>(); g.gain_precision = r.get<float>();
    g.rows_averaged = r.get<uint32_t>(); g.nbins_encoding = r.get<uint32_t>();
    g.dead_flag = r.get<uint32_t>(); g.noisy_flag = r.get<uint32_t>();
    uint32_t nbytes = r.get<uint32_t>();
    uint32_t n = nbytes / 2;
    g.gain.resize(n); g.ped.resize(n);
    for (uint32_t i = 0; i < n; ++i) { g.gain[i] = r.get<uint8_t>(); g.ped[i] = r.get<uint8_t>(); }
    if (!r.ok) return -3;
  }
  {
    Reader r{cpe, ncpe};
    CpeParams& p = c.cpe;
    p.thickness_b = r.get<float>(); p.thickness_e = r.get<float>(); p.pitch_x = r.get<float>(); p.pitch_y = r.get<float>();
    uint32_t n = r.get<uint32_t>();
    p.det.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
      DetParams& d = p.det[i];
      d.is_barrel = r.get<uint8_t>() != 0; d.is_pos_z = r.get<uint8_t>() != 0;
      d.layer = r.get<uint16_t>(); d.index = r.get<uint16_t>(); r.skip(2); d.raw_id = r.get<uint32_t>();
      d.shift_x = r.get<float>(); d.shift_y = r.get<float>(); d.charge_width_x = r.get<float>(); d.charge_width_y = r.get<float>();
      d.x0 = r.get<float>(); d.y0 = r.get<float>(); d.z0 = r.get<float>();
      for (int k = 0; k < 3; ++k) d.sx[k] = r.get<float>();
      for (int k = 0; k < 3; ++k) d.sy[k] = r.get<float>();
      d.px = r.get<float>(); d.py = r.get<float>(); d.pz = r.get<float>();
      for (int k = 0; k < 9; ++k) d.R[k] = r.get<float>();
    }
    r.get_n(p.ladder_z, kLadders); r.get_n(p.ladder_x, kLadders); r.get_n(p.ladder_y, kLadders);
    r.get_n(p.ladder_r, kLadders); r.get_n(p.ladder_minz, kLadders); r.get_n(p.ladder_maxz, kLadders);
    p.endcap_z[0] = r.get<float>(); p.endcap_z[1] = r.get<float>();
    r.get_n(p.layer_start, 11);
    r.get_n(p.layer, 116);
    if (!r.ok) return -4;
  }
  {
    Reader r{bs, nbs};
    float v[11];
    r.get_n(v, 11);
    if (!r.ok) return -5;
    c.bs = {v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8], v[9], v[10]};
  }
  return 0;
}

namespace {

struct DetIdGPU { uint32_t raw_id, roc_in_det, module_id; bool ok; };

// get_raw_id, SiPixelRawToClusterGPUKernel.jl:266-269 (UInt32 index arithmetic wraps)
DetIdGPU get_raw_id(const Cabling& cm, uint8_t fed, uint32_t link, uint32_t roc) {
  uint32_t index = uint32_t(fed) * kMaxLink * kMaxRoc + (link - 1u) * kMaxRoc + roc + 1u;  // 1-based
  if (index < 1 || index > kCablingSize) return {0, 0, 0, false};
  return {cm.raw_id[index - 1], cm.roc_in_det[index - 1], cm.module_id[index - 1], true};
}

// check_roc, SiPixelRawToClusterGPUKernel.jl:394-468. The later branches compare
// error_found (a Bool) with the codes, so only code 25 can be reported; the map size is 0,
// so the cabling test in the 25 branch never clears it.
uint8_t check_roc(uint32_t w, uint8_t fed, uint32_t link, const Cabling& cm) {
  uint8_t error_type = uint8_t((w >> 21) & 0x1F);
  if (error_type < 25) return 0;
  if (error_type == 25) {
    uint32_t index = uint32_t(fed) * kMaxLink * kMaxRoc + (link - 1u) * kMaxRoc + 1u;
    bool found = true;
    if (index > 1 && index <= cm.size) {
      if (!(link == cm.link[index - 1] && 1 == cm.roc[index - 1])) found = false;
    }
    return found ? error_type : 0;
  }
  return 0;
}

// frame_conversion, SiPixelRawToClusterGPUKernel.jl:271-350
bool frame_conversion(bool bpix, int side, uint32_t layer, uint32_t roc_in_det, int64_t lrow, int64_t lcol,
                      int64_t* grow, int64_t* gcol) {
  int64_t sr, sc, ro, co;
  if (bpix) {
    if (side == -1 && layer != 1) {
      if (roc_in_det < 8) { sr = 1; sc = -1; ro = 0; co = (8 - int64_t(roc_in_det)) * 52 - 1; }
      else { sr = -1; sc = 1; ro = 2 * 80 - 1; co = (int64_t(roc_in_det) - 8) * 52; }
    } else {
      if (roc_in_det < 8) { sr = -1; sc = 1; ro = 2 * 80 - 1; co = int64_t(roc_in_det) * 52; }
      else { sr = 1; sc = -1; ro = 0; co = (16 - int64_t(roc_in_det)) * 52 - 1; }
    }
  } else {
    if (roc_in_det < 8) { sr = 1; sc = -1; ro = 0; co = (8 - int64_t(roc_in_det)) * 52 - 1; }
    else { sr = -1; sc = 1; ro = 2 * 80 - 1; co = (int64_t(roc_in_det) - 8) * 52; }
  }
  *grow = sr * lrow + ro;
  *gcol = sc * lcol + co;
  // UInt32 conversions of the reference throw on negative values
  return *grow >= 0 && *gcol >= 0 && *gcol <= 0xFFFFFFFFll;
}

}  // namespace

void raw_to_clusters(const Conditions& c, const uint8_t* raw, size_t nbytes, const Options& o, EventOut& ev) {
  // ---- a1: FedRawDataCollection (bin/ReadRAW.jl:23-31) and the payload walk
  // (SiPixelRawToClusterCUDA.jl:75-131, initialize_word_fed SiPixelRawToClusterGPUKernel.jl:217-226)
  std::vector<std::pair<size_t, int32_t>> fed_data(4096, {0, 0});  // fedid -> (byte offset, size)
  {
    Reader r{raw, nbytes};
    int32_t nfeds = r.get<int32_t>();
    for (int32_t i = 0; i < nfeds && r.ok; ++i) {
      int32_t fid = r.get<int32_t>(), sz = r.get<int32_t>();
      if (fid >= 0 && fid < 4096) fed_data[fid] = {r.off, sz};
      r.skip(size_t(sz));
    }
  }
  ev.words.clear();
  ev.fed_id_pairs.clear();
  ev.errors.clear();
  uint32_t wc = 0;
  for (uint32_t fed_id : c.fed_ids) {
    if (fed_id == 40) continue;
    if (fed_id >= 4096) continue;
    auto fd = fed_data[fed_id];
    int32_t len = fd.second;
    uint32_t n_words = uint32_t(len) / 8;
    if (n_words == 0) continue;
    const uint8_t* d = raw + fd.first;
    // Header and trailer checks, SiPixelRawToClusterCUDA.jl:90-128 with ErrorChecker.jl:82-137.
    // The reference's ErrorChecker is built with _includeErrors = false (ErrorChecker.jl:30-35),
    // so these checks store no error record. A header that fails check() (event_id >> 28 != 0x5,
    // fed_header.jl:182) ends the header loop silently; a source id other than the FED's only
    // prints (ErrorChecker.jl:90). The other failures make the reference raise: a header announcing
    // more headers or a trailer announcing more trailers indexes the undefined name rawData
    // (SiPixelRawToClusterCUDA.jl:110, :120); a trailer failing check() (event_size >> 28 != 0xA,
    // fed_trailer.jl:214) or whose fragment_length (event_size & 0xFFFFFF) differs from the FED's
    // 64-bit word count prints the undefined name fedId (ErrorChecker.jl:125, :129); a FED size
    // that is not a whole number of 64-bit words fails the payload assertions
    // (SiPixelRawToClusterCUDA.jl:126-128). Those raise conditions are flagged and the payload
    // [8, size - 8) is unpacked as on the valid path.
    uint32_t h0, h1, t0, t1;
    std::memcpy(&h0, d, 4); std::memcpy(&h1, d + 4, 4);
    std::memcpy(&t0, d + len - 8, 4); std::memcpy(&t1, d + len - 4, 4);
    {
      bool raise = len % 8 != 0 || len < 16;
      if ((h1 >> 28) == 0x5u && ((h0 >> 3) & 1u)) raise = true;  // more_headers
      if ((t1 >> 28) != 0xAu) raise = true;                        // trailer check()
      else if ((t1 & 0xFFFFFFu) != n_words) raise = true;          // fragment_length
      else if ((t0 >> 3) & 1u) raise = true;                       // more_trailers
      if (raise) ev.flags |= kFlagFedFormat;
    }
    uint32_t num_word32 = len >= 16 ? uint32_t(len - 16) / 4 : 0u;
    size_t base = ev.words.size();
    ev.words.resize(base + num_word32);
    std::memcpy(ev.words.data() + base, d + 8, size_t(num_word32) * 4);
    uint32_t p0 = wc / 2, p1 = (wc + num_word32) / 2;
    if (ev.fed_id_pairs.size() < p1) ev.fed_id_pairs.resize(p1);
    for (uint32_t k = p0; k < p1; ++k) ev.fed_id_pairs[k] = uint8_t(fed_id - 1200);
    wc += num_word32;
    (void)h0; (void)h1; (void)t0; (void)t1;
  }
  ev.word_counter = wc;
  // a pair no FED writes (after a last FED with an odd word count, a size on which the reference
  // raises) reads as id 0 here; the reference reads what an earlier event left there
  if (ev.fed_id_pairs.size() < (wc + 1) / 2) ev.fed_id_pairs.resize((wc + 1) / 2, 0);
  uint32_t n = wc;
  ev.xx.assign(n, 0); ev.yy.assign(n, 0); ev.adc.assign(n, 0); ev.pdigi.assign(n, 0); ev.raw_id_arr.assign(n, 0);
  ev.module_ind.assign(n, int16_t(kInvId)); ev.clus.assign(n, 0);

  // ---- a2: raw_to_digi_kernal, SiPixelRawToClusterGPUKernel.jl:537-658
  for (uint32_t g = 0; g < n; ++g) {
    uint8_t fed = ev.fed_id_pairs[g / 2];
    uint32_t ww = ev.words[g];
    if (ww == 0) continue;
    uint32_t link = (ww >> 26) & 0x3F, roc = (ww >> 21) & 0x1F;
    DetIdGPU det = get_raw_id(c.cabling, fed, link, roc);
    uint8_t error_type = check_roc(ww, fed, link, c.cabling);
    bool skip_roc = (roc < 8) ? false : (error_type != 0);
    if (o.include_errors && skip_roc) {
      ev.errors.push_back({0xffffffffu, ww, error_type, fed});
      continue;
    }
    if (!det.ok) { ev.flags |= kFlagModuleOverflow; continue; }
    uint32_t raw_id = det.raw_id;
    bool barrel = ((raw_id >> 25) & 0x7) == 1;
    uint32_t index = uint32_t(fed) * kMaxLink * kMaxRoc + (link - 1u) * kMaxRoc + roc + 1u;
    if (o.use_quality) {
      if (index >= 1 && index <= kCablingSize && c.cabling.bad_rocs[index - 1]) continue;
    }
    uint32_t layer = barrel ? ((raw_id >> 20) & 0xF) : 0;
    uint32_t the_module = barrel ? ((raw_id >> 2) & 0x3FF) : 0;
    uint32_t panel = barrel ? 0 : (raw_id >> 10) & 0x3;
    int side = barrel ? ((the_module < 5) ? -1 : 1) : ((panel == 1) ? -1 : 1);
    int64_t row, col;
    if (layer == 1) {
      col = (ww >> 15) & 0x3F;
      row = (ww >> 8) & 0x7F;
      if (o.include_errors && !(row < 80 && col < 52)) {
        ev.errors.push_back({raw_id, ww, 37, fed});
        continue;
      }
    } else {
      int32_t dcol = int32_t((ww >> 16) & 0x1F), pxid = int32_t((ww >> 8) & 0xFF);
      row = 80 - pxid / 2;
      col = int64_t(dcol) * 2 + pxid % 2;
      if (row < 0) { ev.flags |= kFlagModuleOverflow; continue; }  // the reference raises here (UInt32 field)
      if (o.include_errors && !((dcol < 26) & (2 <= pxid) & (pxid < 162))) {
        ev.errors.push_back({raw_id, ww, 37, fed});
        continue;
      }
    }
    int64_t grow, gcol;
    if (!frame_conversion(barrel, side, layer, det.roc_in_det, row, col, &grow, &gcol)) {
      ev.flags |= kFlagModuleOverflow;
      continue;
    }
    ev.xx[g] = int16_t(grow);
    ev.yy[g] = int16_t(gcol);
    ev.adc[g] = int32_t(ww & 0xFF);
    uint32_t a = std::min<uint32_t>(uint32_t(ev.adc[g]), 1023u);
    ev.pdigi[g] = (uint32_t(grow) << 0) | (uint32_t(gcol) << 11) | (a << 22);
    ev.module_ind[g] = int16_t(det.module_id);
    ev.raw_id_arr[g] = raw_id;
  }

  // ---- a3: calib_digis, gpu_calib_pixel.jl:28-71 with get_ped_and_gain,
  // CondFormats/si_pixel_gain_for_hlt_on_gpu.jl:47-75
  ev.clus_module_start[0] = 0;
  ev.module_start[0] = 0;
  for (int i = 0; i < kMaxNumModules; ++i) ev.clus_in_module[i] = 0;
  const Gains& gn = c.gains;
  for (uint32_t i = 0; i < n; ++i) {
    int16_t id = ev.module_ind[i];
    if (id == int16_t(kInvId)) continue;
    float cf = id < 96 ? 50.f : 47.f;
    float off = id < 96 ? -670.f : -60.f;
    int16_t row = ev.xx[i], col = ev.yy[i];
    const Gains::RangeAndCols& rc = gn.rc[id];
    uint32_t lcd = (rc.last - rc.first) / uint32_t(rc.cols);
    uint32_t offset = rc.first + uint32_t(int32_t(col)) * lcd + 2u * (uint32_t(int32_t(row)) / gn.rows_averaged);
    uint32_t k = offset / 2;
    if (k >= gn.ped.size()) { ev.flags |= kFlagModuleOverflow; continue; }
    uint8_t sp = gn.ped[k], sg = gn.gain[k];
    bool dead = (uint32_t(sp) & 0xFF) == gn.dead_flag, noisy = (uint32_t(sp) & 0xFF) == gn.noisy_flag;
    float ped = float(sp) * gn.ped_precision + gn.min_ped;
    float gain = float(sg) * gn.gain_precision + gn.min_gain;
    if (dead || noisy) {
      ev.module_ind[i] = int16_t(kInvId);
      ev.adc[i] = 0;
    } else {
      float vcal = float(ev.adc[i]) * gain - ped * gain;
      float v = vcal * cf + off;
      ev.adc[i] = std::max<int32_t>(100, int32_t(std::trunc(v)));
    }
  }

  // ---- a4-a6 clustering
  std::vector<uint16_t> idv(n);
  for (uint32_t i = 0; i < n; ++i) idv[i] = uint16_t(ev.module_ind[i]);
  clusterize_digis(idv.data(), ev.xx.data(), ev.yy.data(), ev.adc.data(), int(n), ev.module_start, ev.clus_in_module,
                   ev.module_id, ev.clus.data(), idv.data(), 1, &ev.flags);
  for (uint32_t i = 0; i < n; ++i) ev.module_ind[i] = int16_t(idv[i]);
  ev.n_modules = ev.module_start[0];

  // ---- a7: fill_hits_module_start, SiPixelRawToClusterGPUKernel.jl:739-752
  uint32_t* ms = ev.clus_module_start;
  ms[0] = 0;
  for (int i = 0; i < kMaxNumModules; ++i) ms[i + 1] = std::min(kMaxHitsInModule, ev.clus_in_module[i]);
  for (int i = 2; i <= kMaxNumModules; ++i) ms[i] += ms[i - 1];
  for (int i = 0; i <= kMaxNumModules; ++i)
    if (ms[i] > ev.caps.hits) { ms[i] = ev.caps.hits; ev.flags |= kFlagHitsClamped; }
  ev.n_clusters = ms[kMaxNumModules - 1];  // setNClusters!(…, clus_module_start_d[MAX_NUM_MODULES]) (1-based)
}

// count_modules (gpu_clustering.jl:52-74), find_clus (:94-266) and cluster_charge_cut
// (gpu_cluster_charge_cut.jl:14-104), on 0-based arrays; module_start/clus values keep the
// reference's 1-based meaning (digi index i+1, cluster numbers from 1).
void clusterize_digis(const uint16_t* id_in, const int16_t* x, const int16_t* y, const int32_t* adc, int n,
                      uint32_t* module_start, uint32_t* clus_in_module, uint32_t* module_id, int32_t* clus,
                      uint16_t* id, int apply_charge_cut, uint32_t* flags) {
  if (id != id_in) std::memcpy(id, id_in, sizeof(uint16_t) * size_t(n));
  // count_modules
  module_start[0] = 0;
  for (int i = 0; i < n; ++i) {
    clus[i] = i + 1;
    if (id[i] == kInvId) continue;
    int j = i - 1;
    while (j >= 0 && id[j] == kInvId) --j;
    if (j < 0 || id[j] != id[i]) {
      module_start[0] = std::min<uint32_t>(module_start[0] + 1, kMaxNumModules);
      uint32_t loc = module_start[0];  // 0-based slot loc = 1-based loc-1+1
      module_start[loc] = uint32_t(i + 1);
    }
  }
  // find_clus
  const int nbins = 418;  // HisToContainer{Int16,418,4000,9,UInt16,1}: bin = (y & 511) + 1
  std::vector<uint32_t> off(nbins + 1);
  std::vector<uint16_t> bins(4000 + 8);
  std::vector<uint16_t> nn(size_t(4001) * 10);
  std::vector<uint8_t> nnn(4001);
  for (uint32_t mod = 1; mod <= module_start[0]; ++mod) {
    int first_pixel = int(module_start[mod]);  // 1-based
    uint16_t this_module_id = id[first_pixel - 1];
    int first = first_pixel;
    int msize = n;
    for (int i = first; i <= n; ++i) {
      if (id[i - 1] == kInvId) continue;
      if (id[i - 1] != this_module_id) { msize = std::min(msize, i); break; }
    }
    std::fill(off.begin(), off.end(), 0u);
    if (msize - first_pixel > 4000) msize = 4000 + first_pixel;
    if (msize == n && id[msize - 1] == this_module_id) msize += 1;
    auto binof = [](int16_t t) -> uint32_t { return uint32_t((uint32_t(uint16_t(t)) >> 0) & 511u) + 1u; };
    for (int i = first; i <= msize - 1; ++i) {
      if (id[i - 1] == kInvId) continue;
      off[binof(y[i - 1]) - 1] += 1;
    }
    // finalize!: inclusive prefix scan over the nbins+1 counters
    for (int b = 1; b <= nbins; ++b) off[b] += off[b - 1];
    for (int i = first; i <= msize - 1; ++i) {
      if (id[i - 1] == kInvId) continue;
      uint32_t b = binof(y[i - 1]);
      uint32_t w = off[b - 1];
      off[b - 1] -= 1;
      bins[w - 1] = uint16_t(i - first_pixel);
    }
    uint32_t hsize = off[nbins];
    std::fill(nnn.begin(), nnn.begin() + hsize + 1, uint8_t(0));
    for (uint32_t j = 0; j < hsize; ++j) {
      uint32_t k = j + 1;
      uint32_t p = 1 + j;  // begin_h(hist) = 1
      int i = int(bins[p - 1]) + first_pixel;
      uint32_t be = binof(int16_t(y[i - 1] + 1));
      uint32_t e = off[be] + 1;  // end_h(hist, be) = off[be+1] + 1 (1-based off)
      p += 1;
      while (p < e) {
        int m = int(bins[p - 1]) + first_pixel;
        if (y[m - 1] - y[i - 1] > 1) break;
        if (std::abs(int(x[m - 1]) - int(x[i - 1])) > 1) { p += 1; continue; }
        nnn[k] += 1;
        if (nnn[k] > 10) { nnn[k] = 10; break; }
        nn[size_t(k) * 10 + nnn[k] - 1] = bins[p - 1];
        p += 1;
      }
    }
    bool more = true;
    int n_loops = 0;
    while (more) {
      if (n_loops % 2 == 1) {
        for (uint32_t j = 0; j < hsize; ++j) {
          int i = int(bins[j]) + first_pixel;
          int m = clus[i - 1];
          while (m != clus[m - 1]) m = clus[m - 1];
          clus[i - 1] = m;
        }
      } else {
        more = false;
        for (uint32_t j = 0; j < hsize; ++j) {
          uint32_t k = j + 1;
          int i = int(bins[j]) + first_pixel;
          for (uint32_t kk = 1; kk <= nnn[k]; ++kk) {
            int m = int(nn[size_t(k) * 10 + kk - 1]) + first_pixel;
            int32_t old = clus[m - 1];
            clus[m - 1] = std::min(clus[m - 1], clus[i - 1]);
            if (old != clus[i - 1]) more = true;
            clus[i - 1] = std::min(clus[i - 1], old);
          }
        }
      }
      ++n_loops;
    }
    int found = 0;
    for (int i = first; i <= msize - 1; ++i) {
      if (id[i - 1] == kInvId) continue;
      if (clus[i - 1] == i) { int old = found; ++found; clus[i - 1] = -(old + 1); }
    }
    for (int i = first; i <= msize - 1; ++i) {
      if (id[i - 1] == kInvId) continue;
      if (clus[i - 1] > 0) clus[i - 1] = clus[clus[i - 1] - 1];
    }
    for (int i = first; i <= msize - 1; ++i) {
      if (id[i - 1] == kInvId) { clus[i - 1] = -9999; continue; }
      clus[i - 1] = -clus[i - 1];
    }
    clus_in_module[this_module_id] = uint32_t(found);
    module_id[mod - 1] = this_module_id;
  }
  if (!apply_charge_cut) return;
  // cluster_charge_cut. The skip test there, `id[i] == INV_ID | id[i] == -INV_ID`, parses as a
  // chained comparison that is always false, so the charge sums stop at the first invalid
  // digi of the module; the renumbering loop skips invalid digis correctly.
  std::vector<int32_t> charge(kMaxClustersPerModule);
  std::vector<uint16_t> newclus(kMaxClustersPerModule);
  std::vector<uint8_t> ok(kMaxClustersPerModule);
  for (uint32_t mod = 1; mod <= module_start[0]; ++mod) {
    int first_pixel = int(module_start[mod]);
    uint16_t this_id = id[first_pixel - 1];
    uint32_t nclus = clus_in_module[this_id];
    if (nclus == 0) continue;
    if (nclus > uint32_t(kMaxClustersPerModule)) {
      for (int i = first_pixel; i <= n; ++i) {
        if (id[i - 1] != this_id) break;
        if (clus[i - 1] > kMaxClustersPerModule) { id[i - 1] = kInvId; clus[i - 1] = kInvId; }
      }
      nclus = kMaxClustersPerModule;
    }
    std::fill(charge.begin(), charge.end(), 0);
    for (int i = first_pixel; i <= n; ++i) {
      if (id[i - 1] != this_id) break;
      int32_t cl = clus[i - 1];
      // an id past 1024 (a run with more clusters than the count its id's last run left)
      // indexes the reference's charge buffer out of bounds: it raises
      if (cl >= 1 && cl <= kMaxClustersPerModule) charge[cl - 1] += adc[i - 1];
      else if (flags) *flags |= kFlagClustersPerModule;
    }
    int32_t cut = this_id < 96 ? 2000 : 4000;
    for (uint32_t i = 0; i < nclus; ++i) { ok[i] = charge[i] > cut ? 1 : 0; newclus[i] = ok[i]; }
    for (uint32_t i = 1; i < nclus; ++i) newclus[i] = uint16_t(newclus[i] + newclus[i - 1]);
    if (nclus == newclus[nclus - 1]) continue;
    clus_in_module[this_id] = newclus[nclus - 1];
    for (uint32_t i = 0; i < nclus; ++i) if (ok[i] == 0) newclus[i] = kInvId;
    for (int i = first_pixel; i <= n; ++i) {
      if (id[i - 1] == kInvId) continue;
      if (id[i - 1] != this_id) break;
      int32_t cl = clus[i - 1];
      // newclus keeps the numbers of the module cut before this one beyond nclus: a run whose
      // own clusters outnumber the count its id's last run left reads them, as the reference
      // reads its per-event newclusId buffer; past 1024 the reference raises
      if (cl < 1 || cl > kMaxClustersPerModule) {
        if (flags) *flags |= kFlagClustersPerModule;
        continue;
      }
      clus[i - 1] = newclus[cl - 1];
      if (clus[i - 1] == kInvId) id[i - 1] = kInvId;
    }
  }
}

}  // namespace orc
