// Test infrastructure (CPU oracle): pixel vertex finding, restated from the
// reference (plugin-PixelVertexFinding/gpu_vertex_finder.jl:51-436,
// pixel_vertex_producer_cuda.jl:3-30, CUDADataFormats/z_vertex_soa.jl:4-26).
#include <algorithm>
#include <cmath>

#include "oracle.h"

namespace orc {

void make_vertices(const Conditions&, EventOut& ev) {
  const int32_t min_T = 2;
  const float eps = 0.07f, err_max = 0.01f, chi2_max = 9.0f;
  const float pt_min = 0.5f;
  const uint32_t ntb = ev.caps.tuples;  // ZVertexSoA track stride (the TrackSOA's)
  ev.idv.assign(ntb, -1);
  ev.zv.assign(kMaxVtx, 0.f); ev.wv.assign(kMaxVtx, 0.f); ev.vchi2.assign(kMaxVtx, 0.f); ev.ptv2.assign(kMaxVtx, 0.f);
  ev.ndof.assign(ntb, 0);
  ev.sort_ind.assign(kMaxVtx, 0);
  ev.nv_final = 0;
  // WorkSpace
  std::vector<uint32_t> itrk;
  std::vector<float> zt, ezt2, ptt2;
  // load_tracks, :51-82
  auto tsize = [&](uint32_t it) { return ev.tuple_off[it] - ev.tuple_off[it - 1]; };
  for (uint32_t idx = 1; idx <= ntb; ++idx) {
    uint32_t nh = tsize(idx);
    if (nh == 0) break;
    if (nh < 4) continue;
    if (ev.quality[idx - 1] != 2) continue;
    float pt = ev.pt[idx - 1];
    if (pt < pt_min) continue;
    itrk.push_back(idx);
    zt.push_back(ev.state[size_t(idx - 1) * 5 + 4]);
    ezt2.push_back(ev.cov[size_t(idx - 1) * 15 + 14]);
    ptt2.push_back(pt * pt);
  }
  uint32_t nt = uint32_t(itrk.size());
  ev.n_vtx_tracks = nt;
  std::vector<uint8_t> izt(nt);
  std::vector<int32_t> iv(nt);
  std::vector<int32_t>& nn = ev.ndof;
  // cluster_tracks_by_density, :84-206 with HisToContainer{UInt8,256,16000,8,UInt16}
  const float err2_max = err_max * err_max;
  uint32_t off[257] = {};
  std::vector<uint32_t> bins(std::max<uint32_t>(nt, 1));
  for (uint32_t i = 0; i < nt; ++i) {
    double zz = double(zt[i]) * 10.;
    int32_t iz = int32_t(std::trunc(zz));
    iz = std::min(std::max(iz, int32_t(-128)), int32_t(127));
    izt[i] = uint8_t(iz + 128);
    off[izt[i]] += 1;  // bin(t) = t + 1 (1-based) -> slot t
    iv[i] = int32_t(i + 1);
  }
  for (int b = 1; b < 257; ++b) off[b] += off[b - 1];
  for (uint32_t i = 0; i < nt; ++i) {
    uint32_t w = off[izt[i]];
    off[izt[i]] -= 1;
    bins[w - 1] = i + 1;
  }
  // for_each_in_bins(hist, izt[i], 1, f): bins max(1,b-1)..min(256,b+1) (1-based bins)
  auto for_each = [&](uint8_t v, auto&& f) {
    int bs = int(v) + 1;
    int be = std::min(256, bs + 1);
    bs = std::max(1, bs - 1);
    for (uint32_t pj = off[bs - 1] + 1; pj <= off[be]; ++pj) f(uint32_t(bins[pj - 1]));
  };
  for (uint32_t i = 1; i <= nt; ++i) {
    if (ezt2[i - 1] > err2_max) continue;
    for_each(izt[i - 1], [&](uint32_t j) {
      if (i == j) return;
      float dist = std::fabs(zt[i - 1] - zt[j - 1]);
      if (dist > eps) return;
      if (dist * dist > chi2_max * (ezt2[i - 1] + ezt2[j - 1])) return;
      nn[i - 1] += 1;
    });
  }
  for (uint32_t i = 1; i <= nt; ++i) {
    float mdist = eps;
    for_each(izt[i - 1], [&](uint32_t j) {
      if (nn[j - 1] < nn[i - 1]) return;
      if (nn[j - 1] == nn[i - 1] && zt[j - 1] >= zt[i - 1]) return;
      float dist = std::fabs(zt[i - 1] - zt[j - 1]);
      if (dist > mdist) return;
      if (dist * dist > chi2_max * (ezt2[i - 1] + ezt2[j - 1])) return;
      mdist = dist;
      iv[i - 1] = int32_t(j);
    });
  }
  for (uint32_t i = 1; i <= nt; ++i) {
    int32_t m = iv[i - 1];
    while (m != iv[m - 1]) m = iv[m - 1];
    iv[i - 1] = m;
  }
  int32_t found = 0;
  for (uint32_t i = 1; i <= nt; ++i) {
    if (iv[i - 1] == int32_t(i)) {
      if (nn[i - 1] >= min_T) { found += 1; iv[i - 1] = -found; }
      else iv[i - 1] = -9998;
    }
  }
  if (found >= kMaxVtx) { ev.flags |= kFlagVertexAssert; found = kMaxVtx - 1; }
  for (uint32_t i = 1; i <= nt; ++i)
    if (iv[i - 1] >= 0) iv[i - 1] = iv[iv[i - 1] - 1];
  for (uint32_t i = 1; i <= nt; ++i) iv[i - 1] = -iv[i - 1];
  uint32_t nv_intermediate = uint32_t(found);
  ev.nv_final = uint32_t(found);

  // fit_vertices, :228-286
  auto fit = [&](double chi2max) {
    uint32_t nvf = nv_intermediate;
    ev.nv_final = nvf;
    for (uint32_t i = 0; i < nvf; ++i) { ev.zv[i] = 0; ev.wv[i] = 0; ev.vchi2[i] = 0; }
    for (uint32_t i = 0; i < nt; ++i) {
      if (iv[i] > 9990) continue;
      if (iv[i] < 1 || uint32_t(iv[i]) > nvf) { ev.flags |= kFlagVertexAssert; continue; }
      float w = 1 / ezt2[i];
      ev.zv[iv[i] - 1] += zt[i] * w;
      ev.wv[iv[i] - 1] += w;
    }
    for (uint32_t i = 0; i < nvf; ++i) {
      if (!(ev.wv[i] > 0)) ev.flags |= kFlagVertexAssert;
      ev.zv[i] /= ev.wv[i];
      nn[i] = -1;
    }
    for (uint32_t i = 0; i < nt; ++i) {
      if (iv[i] > 9990) continue;
      float c2 = ev.zv[iv[i] - 1] - zt[i];
      c2 *= c2 / ezt2[i];
      if (double(c2) > chi2max) { iv[i] = 9999; continue; }
      ev.vchi2[iv[i] - 1] += c2;
      nn[iv[i] - 1] += 1;
    }
    for (uint32_t i = 0; i < nvf; ++i)
      if (nn[i] > 0) ev.wv[i] *= (float(nn[i]) / ev.vchi2[i]);
  };
  fit(50.);
  // split_vertices, :288-371
  {
    uint32_t nvf = ev.nv_final;
    const float split_chi2 = 9.f;
    std::vector<uint32_t> it(512);
    std::vector<float> zz(512), ww(512);
    std::vector<uint8_t> nv(512);
    for (uint32_t kv = 1; kv <= nvf; ++kv) {
      if (nn[kv - 1] < 4) continue;
      if (ev.vchi2[kv - 1] < split_chi2 * float(nn[kv - 1])) continue;
      if (nn[kv - 1] >= 512) { ev.flags |= kFlagVertexAssert; continue; }
      uint32_t nq = 0;
      for (uint32_t k = 1; k <= nt; ++k) {
        if (iv[k - 1] == int32_t(kv)) {
          nq += 1;
          zz[nq - 1] = zt[k - 1] - ev.zv[kv - 1];
          nv[nq - 1] = zz[nq - 1] < 0 ? 1 : 2;
          ww[nq - 1] = 1 / ezt2[k - 1];
          it[nq - 1] = k;
        }
      }
      float znew[2], wnew[2];
      if (nq != uint32_t(nn[kv - 1] + 1)) ev.flags |= kFlagVertexAssert;
      int max_iter = 20;
      bool more = true;
      while (more) {
        more = false;
        znew[0] = znew[1] = 0; wnew[0] = wnew[1] = 0;
        for (uint32_t k = 0; k < nq; ++k) {
          int i = nv[k] - 1;
          znew[i] += zz[k] * ww[k];
          wnew[i] += ww[k];
        }
        znew[0] /= wnew[0];
        znew[1] /= wnew[1];
        for (uint32_t k = 0; k < nq; ++k) {
          float d0 = std::fabs(znew[0] - zz[k]), d1 = std::fabs(znew[1] - zz[k]);
          uint8_t newer = d0 < d1 ? 1 : 2;
          more |= newer != nv[k];
          nv[k] = newer;
        }
        max_iter -= 1;
        if (max_iter <= 0) more = false;
      }
      if (wnew[0] == 0 || wnew[1] == 0) continue;
      float dist2 = (znew[0] - znew[1]) * (znew[0] - znew[1]);
      float chi2_dist = dist2 / ((1 / wnew[0]) + (1 / wnew[1]));
      if (chi2_dist < 4) continue;
      nv_intermediate += 1;
      uint32_t newv = nv_intermediate;
      for (uint32_t k = 0; k < nq; ++k)
        if (nv[k] == 2) iv[it[k] - 1] = int32_t(newv);
    }
  }
  if (nv_intermediate >= uint32_t(kMaxVtx)) { ev.flags |= kFlagVertexAssert; nv_intermediate = kMaxVtx - 1; }
  fit(5000.);
  // sort_by_pt2, :391-436 (the sorted order is computed into a local and dropped)
  uint32_t nvf = ev.nv_final;
  if (nvf >= 1) {
    for (uint32_t i = 0; i < nt; ++i) ev.idv[itrk[i] - 1] = int16_t(iv[i]);
    for (uint32_t i = 0; i < nt; ++i) {
      if (iv[i] > 9990) continue;
      ev.ptv2[iv[i] - 1] += ptt2[i];
    }
    if (nvf == 1) ev.sort_ind[0] = 1;
  }
}

}  // namespace orc
