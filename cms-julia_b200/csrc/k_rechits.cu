// CPE rechits and the phi binner. Restates gpuPixelRecHits.jl:31-338
// (getHits), pixelCPEforGPU.jl:246-577 (position_corr, correction,
// errorFromDB), phase1PixelTopology.jl:249-296, SOARotation.jl:126-136,
// approx_atan2.jl:159-184 (unsafe_atan2s), PixelRecHits.jl:20-82 and
// hist_to_container.jl:217-270 (fill_many_from_vector).
// One warp per module (a CTA for the few modules above 256 digis or 128
// clusters, handed over through a device work list); per-cluster reductions
// use shared-memory integer atomics (order independent) and are recorded per hit;
// k_cpe then evaluates the CPE one hit per thread in FP32 with round-to-nearest and
// no contraction, as the reference does.
#include <algorithm>

#include "pxl_internal.cuh"

namespace pxl {

namespace {

__device__ __forceinline__ uint16_t local_x(uint16_t px) {
  int shift = 0;
  if (px > 79) shift += 1;
  if (px > 80) shift += 1;
  return uint16_t(px + shift);
}
__device__ __forceinline__ uint16_t local_y(uint16_t py) {
  int roc = py / 52;
  int shift = 2 * roc;
  int yin = py - 52 * roc;
  if (yin > 0) shift += 1;
  return uint16_t(py + shift);
}
__device__ __forceinline__ bool big_x(uint32_t px) { return px == 79 || px == 80; }
__device__ __forceinline__ bool big_y(uint32_t py) { uint32_t ly = py - 52 * (py / 52); return ly == 0 || ly == 51; }

__device__ __forceinline__ int16_t atan2s(float y, float x) {
  const int16_t pi4 = 8192, pi34 = 24576;
  float r = __fdiv_rn(__fsub_rn(fabsf(x), fabsf(y)), __fadd_rn(fabsf(x), fabsf(y)));
  if (x < 0) r = -r;
  int16_t angle = (x >= 0) ? pi4 : pi34;
  float z = __fmul_rn(r, r);
  float p = __fmul_rn(r, __fadd_rn(-10422.177734375f,
                     __fmul_rn(z, __fadd_rn(3349.97412109375f,
                     __fmul_rn(z, __fadd_rn(-1525.589599609375f, __fmul_rn(z, 406.64190673828125f)))))));
  angle = int16_t(angle + int16_t(truncf(p)));
  return (y < 0) ? int16_t(-angle) : angle;
}

__device__ float correction(uint32_t sizeM1, int32_t q_f, int32_t q_l, uint16_t upper, uint16_t lower, float lorentz,
                            float thick, float cot, float pitch, bool first_big, bool last_big) {
  if (sizeM1 == 0) return 0.0f;
  float w_eff = 0.0f;
  bool simple = true;
  if (sizeM1 == 1) {
    float w_inner = __fmul_rn(pitch, float(uint16_t(lower - upper)));
    float w_pred = __fsub_rn(__fmul_rn(thick, cot), lorentz);
    w_eff = __fsub_rn(fabsf(w_pred), w_inner);
    simple = (w_eff < 0.0f) || (w_eff > pitch);
  }
  if (simple) {
    float s = 2.0f;
    s = __fadd_rn(s, first_big ? 1.0f : 0.0f);
    s = __fadd_rn(s, last_big ? 1.0f : 0.0f);
    w_eff = __fmul_rn(__fmul_rn(pitch, 0.5f), s);
  }
  float qdiff = float(q_l - q_f);
  float qsum = float(q_l + q_f);
  qsum = qsum == 0.0f ? 1.0f : qsum;
  return __fmul_rn(__fmul_rn(0.5f, __fdiv_rn(qdiff, qsum)), w_eff);
}

constexpr int kMaxClus = 1024;
constexpr int kWarpClus = 128;  // clusters per module handled by one warp
constexpr int kWarpSlots = kWarpModulePix / 32;
constexpr int kWarpsPerBlock = 8;

// per-cluster reductions of getHits: bounding box and charges (total, first/last row and column)
struct ClusSum {
  uint32_t minr, maxr, minc, maxc;
  int32_t q, qfx, qlx, qfy, qly;
};

// CPE of one cluster and its hit record at event-local hit index h (gpuPixelRecHits.jl:266-333)
__device__ void write_hit(const Dev& d, int e, uint32_t me, uint32_t h, const ClusSum& s) {
  const Conditions& c = d.c;
  const uint32_t hb = d.ev[e].hit_base;
  if (h >= d.hits_per_event) return;
  if (uint64_t(hb) + h >= uint64_t(d.cap_hits)) { atomic_or_warn(&d.ev[e], kWarnBuffer); return; }
  const DetParamsD& dp = c.det[me];
  const uint32_t min_row = s.minr, max_row = s.maxr, min_col = s.minc, max_col = s.maxc;
  const int32_t qfx = s.qfx, qlx = s.qlx, qfy = s.qfy, qly = s.qly;
  // position_corr
  const uint16_t llx = uint16_t(min_row + 1), lly = uint16_t(min_col + 1), urx = uint16_t(max_row), ury = uint16_t(max_col);
  const uint16_t llxl = local_x(llx), llyl = local_y(lly), urxl = local_x(urx), uryl = local_y(ury);
  const uint16_t mx = uint16_t(llxl + urxl), my = uint16_t(llyl + uryl);
  int32_t xsize = int32_t(urxl) + 2 - int32_t(llxl);
  int32_t ysize = int32_t(uryl) + 2 - int32_t(llyl);
  if (big_x(min_row)) xsize += 1;
  if (big_x(max_row)) xsize += 1;
  if (big_y(min_col)) ysize += 1;
  if (big_y(max_col)) ysize += 1;
  const int32_t unb_x = int32_t(trunc(__ddiv_rn(__dmul_rn(8.0, double(fabsf(float(qfx - qlx)))), double(float(qfx + qlx)))));
  const int32_t unb_y = int32_t(trunc(__ddiv_rn(__dmul_rn(8.0, double(fabsf(float(qfy - qly)))), double(float(qfy + qly)))));
  xsize = 8 * xsize - unb_x;
  ysize = 8 * ysize - unb_y;
  int16_t sxs = int16_t(xsize < 1023 ? xsize : 1023);
  int16_t sys = int16_t(ysize < 1023 ? ysize : 1023);
  if (min_row == 0 || max_row == 159) sxs = int16_t(-sxs);
  if (min_col == 0 || max_col == 415) sys = int16_t(-sys);
  float xpos = __fadd_rn(dp.shift_x, __fmul_rn(c.pitch_x, __fadd_rn(__fmul_rn(0.5f, float(mx)), -81.0f)));
  float ypos = __fadd_rn(dp.shift_y, __fmul_rn(c.pitch_y, __fadd_rn(__fmul_rn(0.5f, float(my)), -216.0f)));
  const float gvz = __fdiv_rn(-1.0f, dp.z0);
  const float cota = __fmul_rn(__fsub_rn(xpos, dp.x0), gvz);
  const float cotb = __fmul_rn(__fsub_rn(ypos, dp.y0), gvz);
  const float thick = dp.is_barrel ? c.thick_b : c.thick_e;
  const float xcorr = correction(max_row - min_row, qfx, qlx, llxl, urxl, dp.cw_x, thick, cota, c.pitch_x, big_x(min_row), big_x(max_row));
  const float ycorr = correction(max_col - min_col, qfy, qly, llyl, uryl, dp.cw_y, thick, cotb, c.pitch_y, big_y(min_col), big_y(max_col));
  xpos = __fadd_rn(xpos, xcorr);
  ypos = __fadd_rn(ypos, ycorr);
  // errorFromDB
  float xerr = 0.0050f, yerr = 0.0085f;
  {
    const uint32_t sx = max_row - min_row, sy = max_col - min_col;
    const bool edge_x = min_row == 0 || max_row == 159, edge_y = min_col == 0 || max_col == 415;
    int ix = sx == 0 ? 1 : 0, iy = sy == 0 ? 1 : 0;
    ix += (sx == 0 && big_x(min_row)) ? 1 : 0;
    iy += (sy == 0 && big_y(min_col)) ? 1 : 0;
    if (!edge_x) xerr = dp.sx[ix];
    if (!edge_y) yerr = dp.sy[iy];
  }
  // toGlobal_Special and beam spot
  float ux = __fadd_rn(__fmul_rn(dp.R[0], xpos), __fmul_rn(dp.R[3], ypos));
  float uy = __fadd_rn(__fmul_rn(dp.R[1], xpos), __fmul_rn(dp.R[4], ypos));
  float uz = __fadd_rn(__fmul_rn(dp.R[2], xpos), __fmul_rn(dp.R[5], ypos));
  ux = __fadd_rn(ux, dp.px); uy = __fadd_rn(uy, dp.py); uz = __fadd_rn(uz, dp.pz);
  const float xg = __fsub_rn(ux, c.bs_x), yg = __fsub_rn(uy, c.bs_y), zg = __fsub_rn(uz, c.bs_z);
  const size_t o = size_t(hb) + h;
  d.charge[o] = uint32_t(s.q);
  d.detind[o] = int16_t(me);
  d.xl[o] = xpos; d.yl[o] = ypos;
  d.xsize[o] = sxs; d.ysize[o] = sys;
  d.xerr[o] = __fmul_rn(xerr, xerr); d.yerr[o] = __fmul_rn(yerr, yerr);
  d.xg[o] = xg; d.yg[o] = yg; d.zg[o] = zg;
  const float rg = __fsqrt_rn(__fadd_rn(__fmul_rn(xg, xg), __fmul_rn(yg, yg)));
  d.rg[o] = rg;
  d.hit_xyzr[o] = make_float4(xg, yg, zg, rg);
  d.iphi[o] = atan2s(yg, xg);
}

// The module at position m of event e as getHits reads it: detector index, cluster count
// (capped at kMaxClus) and digi range [first0, end0). Returns false when there is nothing to do.
struct HitModule {
  uint32_t me, nclus, first0, end0;
};

__device__ __forceinline__ bool hit_module(const Dev& d, int e, uint32_t m, HitModule& hm) {
  const EvInfo& E = d.ev[e];
  const uint32_t nmod = E.n_modules, n_el = E.n_words;
  const uint32_t* ms = d.module_start + size_t(e) * (kMaxNumModules + 1);
  hm.me = d.module_id[size_t(e) * kMaxNumModules + m];
  if (hm.me >= uint32_t(kMaxNumModules) || int32_t(hm.me) >= d.c.n_det) return false;
  hm.nclus = d.clus_in_module[size_t(e) * kMaxNumModules + hm.me];
  if (hm.nclus == 0) return false;
  if (hm.nclus > uint32_t(kMaxClus)) hm.nclus = kMaxClus;
  if (ms[m + 1] < 1 || ms[m + 1] > n_el) return false;
  hm.first0 = ms[m + 1] - 1;
  const uint64_t eb = E.word_base;
  // the module's first digi may have been invalidated by the charge cut: compare with its id
  const uint32_t e1 = module_end1(d.mid, eb, ms, m, nmod, n_el, ms[m + 1], int16_t(hm.me));
  hm.end0 = (m + 1 < nmod) ? e1 - 1 : n_el;
  if (hm.end0 < hm.first0 || hm.end0 > n_el) return false;
  // A module id with several runs (corrupt or repeated FED data): the reference's serial
  // getHits writes the same nclus hit slots once per run, so the last run's values are the
  // ones left. Only that run writes here; the others would race with it.
  if (E.repeated_ids) {
    const uint32_t* mid = d.module_id + size_t(e) * kMaxNumModules;
    for (uint32_t k = m + 1; k < nmod; ++k)
      if (mid[k] == hm.me) return false;
  }
  return true;
}

// ------------------------------------------------------------ warp per module
struct WarpHitSmem {
  uint32_t minr[kWarpClus], maxr[kWarpClus], minc[kWarpClus], maxc[kWarpClus];
  int32_t q[kWarpClus], qfx[kWarpClus], qlx[kWarpClus], qfy[kWarpClus], qly[kWarpClus];
};

// Per-cluster sums of one module with its digis in registers, kS per lane (the module's
// digi count rounded up to a power-of-two number of warp slots). The sums go to the hit's
// record; the CPE of all records then runs one hit per thread in k_cpe.
template <int kS>
__device__ __forceinline__ void module_sums(const Dev& d, int e, const HitModule& hm, const uint32_t* cms,
                                            WarpHitSmem& S) {
  const unsigned lane = threadIdx.x & 31u;
  const EvInfo& E = d.ev[e];
  const uint64_t eb = E.word_base;
  const uint32_t hb = E.hit_base;
  const uint32_t nclus = hm.nclus;
  for (uint32_t k = lane; k < nclus; k += 32) {
    S.minr[k] = 0xFFFFFFFFu; S.maxr[k] = 0; S.minc[k] = 0xFFFFFFFFu; S.maxc[k] = 0;
    S.q[k] = 0; S.qfx[k] = 0; S.qlx[k] = 0; S.qfy[k] = 0; S.qly[k] = 0;
  }
  __syncwarp();
  // digis of this module's range that belong to it, kept in registers
  uint32_t xs[kS], ys[kS];
  int32_t cls[kS], chs[kS];
#pragma unroll
  for (int j = 0; j < kS; ++j) {
    const uint32_t i = hm.first0 + lane + 32u * j;
    cls[j] = 0;
    if (i < hm.end0) {
      const uint64_t g = eb + i;
      const int16_t id = d.mid[g];
      const int32_t cl = d.clus[g];
      if (id != int16_t(kInvId) && uint32_t(int32_t(id)) == hm.me && cl >= 1 && uint32_t(cl) <= nclus) {
        cls[j] = cl;
        xs[j] = uint32_t(int32_t(d.xx[g]));
        ys[j] = uint32_t(int32_t(d.yy[g]));
        const int32_t a = d.adc[g];
        chs[j] = a < 65535 ? a : 65535;
        atomicMin(&S.minr[cl - 1], xs[j]); atomicMax(&S.maxr[cl - 1], xs[j]);
        atomicMin(&S.minc[cl - 1], ys[j]); atomicMax(&S.maxc[cl - 1], ys[j]);
      }
    }
  }
  __syncwarp();
#pragma unroll
  for (int j = 0; j < kS; ++j) {
    if (cls[j] == 0) continue;
    const int k = cls[j] - 1;
    atomicAdd(&S.q[k], chs[j]);
    if (S.minr[k] == xs[j]) atomicAdd(&S.qfx[k], chs[j]);
    if (S.maxr[k] == xs[j]) atomicAdd(&S.qlx[k], chs[j]);
    if (S.minc[k] == ys[j]) atomicAdd(&S.qfy[k], chs[j]);
    if (S.maxc[k] == ys[j]) atomicAdd(&S.qly[k], chs[j]);
  }
  __syncwarp();
  for (uint32_t k = lane; k < nclus; k += 32) {
    const uint32_t h = cms[hm.me] + k;
    if (h >= d.hits_per_event) continue;
    if (uint64_t(hb) + h >= uint64_t(d.cap_hits)) { atomic_or_warn(&d.ev[e], kWarnBuffer); continue; }
    const size_t o = size_t(hb) + h;
    d.hit_sum[o] = ClusSumRec{S.minr[k], S.maxr[k], S.minc[k], S.maxc[k], S.q[k], S.qfx[k], S.qlx[k], S.qfy[k], S.qly[k]};
    d.hit_me[o] = hm.me;
  }
  __syncwarp();
}

// Six blocks per SM (the most its 37 KB of shared memory allows): 40 registers and about
// 130 bytes of spills, faster than four blocks without the cap; the kernel waits on its
// digi gathers, and more warps in flight hide more of them.
__global__ void __launch_bounds__(32 * kWarpsPerBlock, 6) k_get_hits_warp(Dev d) {
  __shared__ WarpHitSmem smem[kWarpsPerBlock];
  const int e = blockIdx.y;
  const unsigned lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
  WarpHitSmem& S = smem[wib];
  const EvInfo& E = d.ev[e];
  const uint32_t nmod = E.n_modules;
  if (E.word_base + uint64_t(E.n_words) > uint64_t(d.cap_words)) return;
  const uint32_t* cms = d.clus_module_start + size_t(e) * (kMaxNumModules + 1);
  for (uint32_t m = blockIdx.x * kWarpsPerBlock + wib; m < nmod; m += gridDim.x * kWarpsPerBlock) {
    HitModule hm;
    if (!hit_module(d, e, m, hm)) continue;
    const uint32_t nd = hm.end0 - hm.first0;
    if (nd > uint32_t(kWarpModulePix) || hm.nclus > uint32_t(kWarpClus)) {
      if (lane == 0) push_module(d, kListHitsBig, e, m);
      continue;
    }
    if (nd <= 32) module_sums<1>(d, e, hm, cms, S);
    else if (nd <= 64) module_sums<2>(d, e, hm, cms, S);
    else if (nd <= 128) module_sums<4>(d, e, hm, cms, S);
    else module_sums<kWarpSlots>(d, e, hm, cms, S);
  }
}

// CPE of the hits whose cluster sums k_get_hits_warp recorded, one hit per thread
__global__ void __launch_bounds__(256) k_cpe(Dev d) {
  const int e = blockIdx.y;
  const EvInfo& E = d.ev[e];
  const uint32_t hb = E.hit_base;
  for (uint32_t h = blockIdx.x * blockDim.x + threadIdx.x; h < E.n_hits; h += gridDim.x * blockDim.x) {
    const size_t o = size_t(hb) + h;
    const uint32_t me = d.hit_me[o];
    if (me == 0xFFFFFFFFu) continue;
    const ClusSumRec r = d.hit_sum[o];
    write_hit(d, e, me, h, ClusSum{r.minr, r.maxr, r.minc, r.maxc, r.q, r.qfx, r.qlx, r.qfy, r.qly});
  }
}

// ------------------------------------------------------------ CTA per module
struct BlockHitSmem {
  uint32_t minr[kMaxClus], maxr[kMaxClus], minc[kMaxClus], maxc[kMaxClus];
  int32_t q[kMaxClus], qfx[kMaxClus], qlx[kMaxClus], qfy[kMaxClus], qly[kMaxClus];
};

__global__ void __launch_bounds__(256) k_get_hits_block(Dev d) {
  __shared__ BlockHitSmem S;
  const uint32_t nbig = list_size(d, kListHitsBig);
  for (uint32_t bi = blockIdx.x; bi < nbig; bi += gridDim.x) {
    const uint32_t v = list_entry(d, kListHitsBig, bi);
    const int e = int(v >> 11);
    const uint32_t m = v & 2047u;
    const EvInfo& E = d.ev[e];
    if (E.word_base + uint64_t(E.n_words) > uint64_t(d.cap_words)) continue;
    const uint64_t eb = E.word_base;
    const uint32_t* cms = d.clus_module_start + size_t(e) * (kMaxNumModules + 1);
    HitModule hm;
    if (!hit_module(d, e, m, hm)) continue;
    const uint32_t nclus = hm.nclus;
    for (uint32_t k = threadIdx.x; k < nclus; k += blockDim.x) {
      S.minr[k] = 0xFFFFFFFFu; S.maxr[k] = 0; S.minc[k] = 0xFFFFFFFFu; S.maxc[k] = 0;
      S.q[k] = 0; S.qfx[k] = 0; S.qlx[k] = 0; S.qfy[k] = 0; S.qly[k] = 0;
    }
    __syncthreads();
    for (uint32_t i = hm.first0 + threadIdx.x; i < hm.end0; i += blockDim.x) {
      const uint64_t g = eb + i;
      const int16_t id = d.mid[g];
      if (id == int16_t(kInvId) || uint32_t(int32_t(id)) != hm.me) continue;
      const int32_t cl = d.clus[g];
      if (cl < 1 || uint32_t(cl) > nclus) continue;
      const uint32_t x = uint32_t(int32_t(d.xx[g])), y = uint32_t(int32_t(d.yy[g]));
      atomicMin(&S.minr[cl - 1], x); atomicMax(&S.maxr[cl - 1], x);
      atomicMin(&S.minc[cl - 1], y); atomicMax(&S.maxc[cl - 1], y);
    }
    __syncthreads();
    for (uint32_t i = hm.first0 + threadIdx.x; i < hm.end0; i += blockDim.x) {
      const uint64_t g = eb + i;
      const int16_t id = d.mid[g];
      if (id == int16_t(kInvId) || uint32_t(int32_t(id)) != hm.me) continue;
      const int32_t cl = d.clus[g];
      if (cl < 1 || uint32_t(cl) > nclus) continue;
      const uint32_t x = uint32_t(int32_t(d.xx[g])), y = uint32_t(int32_t(d.yy[g]));
      const int32_t a = d.adc[g];
      const int32_t ch = a < 65535 ? a : 65535;
      const int k = cl - 1;
      atomicAdd(&S.q[k], ch);
      if (S.minr[k] == x) atomicAdd(&S.qfx[k], ch);
      if (S.maxr[k] == x) atomicAdd(&S.qlx[k], ch);
      if (S.minc[k] == y) atomicAdd(&S.qfy[k], ch);
      if (S.maxc[k] == y) atomicAdd(&S.qly[k], ch);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < nclus; k += blockDim.x) {
      const ClusSum s{S.minr[k], S.maxr[k], S.minc[k], S.maxc[k], S.q[k], S.qfx[k], S.qlx[k], S.qfy[k], S.qly[k]};
      write_hit(d, e, hm.me, cms[hm.me] + k, s);
    }
    __syncthreads();
  }
}

// setHitsLayerStart + fill_many_from_vector for the 10x128 phi histogram, one block per event.
// Bins end up holding hit ids in decreasing order (the reference fill decrements the bin cursor).
__global__ void __launch_bounds__(1024) k_phi_binner(Dev d) {
  const int e = blockIdx.x;
  __shared__ uint32_t s_off[kPhiTotBins + 3];
  __shared__ uint32_t s_hls[11];
  __shared__ uint32_t sh[33];
  const EvInfo& E = d.ev[e];
  const uint32_t hb = E.hit_base;
  const uint32_t nh = E.n_hits;
  const uint32_t* cms = d.clus_module_start + size_t(e) * (kMaxNumModules + 1);
  if (threadIdx.x < 11) {
    const uint32_t ls = d.c.layer_start[threadIdx.x];
    s_hls[threadIdx.x] = cms[ls <= uint32_t(kMaxNumModules) ? ls : uint32_t(kMaxNumModules)];
  }
  for (int b = threadIdx.x; b < kPhiTotBins + 3; b += blockDim.x) s_off[b] = 0;
  __syncthreads();
  if (threadIdx.x < 11) d.hits_layer_start[size_t(e) * 11 + threadIdx.x] = s_hls[threadIdx.x];
  uint32_t* poff = d.phi_off + size_t(e) * kPhiTotBins;
  if (nh == 0 || uint64_t(hb) + nh > uint64_t(d.cap_hits)) {
    for (int b = threadIdx.x; b < kPhiTotBins; b += blockDim.x) poff[b] = 0;
    return;
  }
  const uint32_t ntot = s_hls[10];
  auto layer_of = [&](uint32_t i) -> int {
    int k = 0;
    while (k < 11 && s_hls[k] < i) ++k;  // searchsortedfirst
    return (k < 11 && s_hls[k] == i) ? k : k - 1;
  };
  auto bin_of = [&](uint32_t i) -> uint32_t {
    const int16_t t = d.iphi[hb + i];
    return ((uint32_t(int32_t(t >> 9)) & 127u) + 1u) + 128u * uint32_t(layer_of(i));
  };
  for (uint32_t i = threadIdx.x; i < ntot; i += blockDim.x) atomicAdd(&s_off[bin_of(i) - 1], 1u);
  __syncthreads();
  // inclusive scan of 1281 counters
  {
    uint32_t carry = 0;
    for (int b = 0; b < kPhiTotBins; b += blockDim.x) {
      int k = b + threadIdx.x;
      uint32_t v = k < kPhiTotBins ? s_off[k] : 0u;
      uint32_t tot;
      uint32_t ex = block_excl_scan(v, sh, &tot);
      if (k < kPhiTotBins) s_off[k] = carry + ex + v;
      carry += tot;
    }
  }
  __syncthreads();
  uint32_t* bins = d.phi_bins + hb;
  for (uint32_t i = threadIdx.x; i < ntot; i += blockDim.x) {
    uint32_t w = atomicSub(&s_off[bin_of(i) - 1], 1u);
    bins[w - 1] = i + 1;
  }
  __syncthreads();
  for (int b = threadIdx.x; b < kPhiTotBins; b += blockDim.x) poff[b] = s_off[b];
  // Each binned hit's place in two orders of its bin, by its rank among the bin's hits (a
  // bin holds a few tens of hits): decreasing hit id, the reference's order (its fill
  // decrements the bin cursor), for the doublet records and the bins; and increasing iphi
  // (as uint16, ties by decreasing id) for the records of the doublet search's exact phi
  // windows.
  HitRec* rec = d.hit_rec + hb;
  HitRec* rs = d.hit_rec_s + hb;
  uint16_t* us = d.hit_u_s + hb;
  for (uint32_t p = threadIdx.x; p < ntot; p += blockDim.x) {
    const uint32_t v = bins[p], i = v - 1u;
    const uint32_t b = bin_of(i) - 1u;
    const uint32_t lo = s_off[b], hi = s_off[b + 1];
    const uint16_t u = uint16_t(d.iphi[hb + i]);
    uint32_t rid = 0, ru = 0;
    for (uint32_t q = lo; q < hi; ++q) {
      const uint32_t w = bins[q];
      const uint16_t uq = uint16_t(d.iphi[hb + w - 1u]);
      rid += w > v;
      ru += uq < u || (uq == u && w > v);
    }
    HitRec r;
    r.z = d.zg[hb + i];
    r.r = d.rg[hb + i];
    r.iphi = int16_t(u);
    r.ysize = d.ysize[hb + i];
    // hits sit on modules below 2000, so the detector index fits the record's 11 bits
    r.det_id = (uint32_t(d.detind[hb + i]) << kHitIdBits) | i;
    rec[lo + rid] = r;
    rs[lo + ru] = r;
    us[lo + ru] = u;
  }
  __syncthreads();
  for (uint32_t p = threadIdx.x; p < ntot; p += blockDim.x) bins[p] = (rec[p].det_id & (kMaxHitsPerEvent - 1u)) + 1u;
}

}  // namespace

void launch_rechits(const Dev& d, const Launch& L) {
  // at least 16 blocks per event: short blocks (a dozen modules per warp) keep the tail of
  // the launch short (1.10 instead of 1.17 ms per 1000 PU50 events with 4)
  const int bx = std::max(16, std::min(250, (148 * 8 * 4) / std::max(1, int(d.E))));
  // records of the warp-handled modules' clusters; hits of other modules keep 0xFFFFFFFF
  cudaMemsetAsync(d.hit_me, 0xFF, size_t(d.cap_hits) * sizeof(uint32_t), L.s);
  k_get_hits_warp<<<dim3(bx, d.E), 32 * kWarpsPerBlock, 0, L.s>>>(d);
  L.mark("get_hits_warp");
  k_cpe<<<dim3(std::max(1, std::min(64, (148 * 8 * 2) / std::max(1, int(d.E)))), d.E), 256, 0, L.s>>>(d);
  L.mark("cpe");
  k_get_hits_block<<<148 * 2, 256, 0, L.s>>>(d);
  L.mark("get_hits_block");
  k_phi_binner<<<d.E, 1024, 0, L.s>>>(d);
  L.mark("phi_binner");
}

}  // namespace pxl
