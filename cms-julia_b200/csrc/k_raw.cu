// FED payload walk, raw -> digi unpacking with gain calibration, and module
// starts. Restates SiPixelRawToClusterCUDA.jl:75-131 (payload walk),
// SiPixelRawToClusterGPUKernel.jl:537-658 (raw_to_digi_kernal),
// gpu_calib_pixel.jl:28-71 (calib_digis) and gpu_clustering.jl:52-74
// (count_modules) for a batch of events.
#include <cstddef>

#include "pxl_internal.cuh"

namespace pxl {

namespace {

// Single-block scan of one EvInfo count field into a base field over E events;
// ev[E] receives the batch total in both fields.
__global__ void k_ev_scan(EvInfo* ev, int E, int count_off, int base_off) {
  __shared__ uint32_t sh[33];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  char* base = reinterpret_cast<char*>(ev);
  for (int b = 0; b < E; b += blockDim.x) {
    int e = b + threadIdx.x;
    uint32_t v = e < E ? *reinterpret_cast<uint32_t*>(base + size_t(e) * sizeof(EvInfo) + count_off) : 0u;
    uint32_t tot;
    uint32_t ex = block_excl_scan(v, sh, &tot);
    if (e < E) *reinterpret_cast<uint32_t*>(base + size_t(e) * sizeof(EvInfo) + base_off) = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *reinterpret_cast<uint32_t*>(base + size_t(E) * sizeof(EvInfo) + base_off) = carry;
    *reinterpret_cast<uint32_t*>(base + size_t(E) * sizeof(EvInfo) + count_off) = carry;
  }
}

__device__ __forceinline__ int32_t ld_i32(const uint8_t* p) {
  // records sit on 4-byte boundaries when the blob does; read bytewise to stay safe otherwise
  uint32_t v = uint32_t(p[0]) | (uint32_t(p[1]) << 8) | (uint32_t(p[2]) << 16) | (uint32_t(p[3]) << 24);
  return int32_t(v);
}

// One block per event: FedRawDataCollection directory (bin/ReadRAW.jl:23-31), then the
// payload word counts in fedIds order (SiPixelRawToClusterCUDA.jl:75-131: skip FED 40,
// skip empty FEDs, payload = bytes [8, size-8)). The directory is a chain of records whose
// positions depend on every earlier size, so one thread follows it; the FED header and
// trailer checks then run one FED per thread.
__global__ void k_fed_table(Dev d, const int16_t* __restrict__ fed_slot_of) {
  const int e = blockIdx.x;
  const int NF = d.n_fed_slots;
  __shared__ uint64_t s_src[kMaxFedSlots];
  __shared__ uint32_t s_nw[kMaxFedSlots];
  __shared__ int32_t s_len[kMaxFedSlots];
  __shared__ uint32_t sh[33];
  __shared__ uint32_t s_warn;
  for (int f = threadIdx.x; f < NF; f += blockDim.x) { s_nw[f] = 0; s_src[f] = 0; s_len[f] = 0; }
  if (threadIdx.x == 0) s_warn = 0;
  __syncthreads();
  const uint64_t off0 = d.ev_off[e], off1 = d.ev_off[e + 1];
  const uint8_t* ev = d.raw + off0;
  const uint64_t nbytes = off1 - off0;
  if (threadIdx.x == 0) {
    if (nbytes >= 4) {
      int32_t nfeds = ld_i32(ev);
      uint64_t p = 4;
      for (int32_t k = 0; k < nfeds; ++k) {
        if (p + 8 > nbytes) { s_warn |= kWarnBuffer; break; }
        int32_t fid = ld_i32(ev + p), size = ld_i32(ev + p + 4);
        if (size < 0 || p + 8 + uint64_t(size) > nbytes) { s_warn |= kWarnBuffer; break; }
        if (fid >= 0 && fid < 4096) {
          int slot = fed_slot_of[fid];
          if (slot >= 0) {
            uint32_t nw64 = uint32_t(size) / 8;
            uint32_t nw32 = nw64 == 0 ? 0u : (size >= 16 ? uint32_t(size - 16) / 4 : 0u);
            s_nw[slot] = nw32;
            s_src[slot] = off0 + p + 8 + 8;
            s_len[slot] = size;
          }
        }
        p += 8 + uint64_t(size);
      }
    }
  }
  __syncthreads();
  // Header and trailer checks (SiPixelRawToClusterCUDA.jl:90-128, ErrorChecker.jl:82-137). The
  // reference's checker stores no error record (_includeErrors = false, ErrorChecker.jl:30-35):
  // a header failing check() ends its loop silently and a foreign source id only prints. A header
  // announcing more headers, a trailer failing check() or announcing more trailers, a
  // fragment_length other than the FED's 64-bit word count, or a size that is not a whole
  // number of 64-bit words make the reference raise; they set PXL_WARN_FED_FORMAT here and the
  // payload [8, size - 8) is unpacked as on the valid path.
  for (int f = threadIdx.x; f < NF; f += blockDim.x) {
    const int32_t len = s_len[f];
    if (len < 8) continue;  // empty FEDs are skipped (n_words == 0)
    const uint8_t* fd = d.raw + s_src[f] - 8;  // the FED's data: header, payload, trailer
    const uint32_t h0 = uint32_t(ld_i32(fd)), h1 = uint32_t(ld_i32(fd + 4));
    const uint32_t t0 = uint32_t(ld_i32(fd + len - 8)), t1 = uint32_t(ld_i32(fd + len - 4));
    bool raise = (len & 7) != 0 || len < 16;
    if ((h1 >> 28) == 0x5u && ((h0 >> 3) & 1u)) raise = true;   // more_headers (fed_header.jl:177)
    if ((t1 >> 28) != 0xAu) raise = true;                         // trailer check() (fed_trailer.jl:214)
    else if ((t1 & 0xFFFFFFu) != uint32_t(len) / 8u) raise = true;  // fragment_length (fed_trailer.jl:193)
    else if ((t0 >> 3) & 1u) raise = true;                        // more_trailers (fed_trailer.jl:201)
    if (raise) atomicOr(&s_warn, kWarnFedFormat);
  }
  uint32_t carry = 0;
  for (int b = 0; b < NF; b += blockDim.x) {
    int f = b + threadIdx.x;
    uint32_t v = f < NF ? s_nw[f] : 0u;
    uint32_t tot;
    uint32_t ex = block_excl_scan(v, sh, &tot);
    if (f < NF) {
      d.fed_src[size_t(e) * NF + f] = s_src[f];
      d.fed_nw[size_t(e) * NF + f] = v;
      d.fed_wo[size_t(e) * NF + f] = carry + ex;
    }
    carry += tot;
  }
  if (threadIdx.x == 0) {
    EvInfo& E = d.ev[e];
    E.raw_off = off0;
    E.n_words = carry;
    E.warnings = s_warn;
    E.n_errors = 0;
  }
}

// raw_to_digi_kernal + calib_digis of one FED word ww: event-local word index local, global
// digi index g, FED id fed + 1200.
__device__ __forceinline__ void unpack_word(const Dev& d, int e, uint32_t local, uint64_t g, uint8_t fed, uint32_t ww) {
  const Conditions& c = d.c;
  int16_t xx = 0, yy = 0, mid = int16_t(kInvId);
  int32_t adc = 0;
  uint32_t pdigi = 0, rawid = 0;
  d.clus[g] = int32_t(local + 1);  // count_modules: clus[i] = i
  if (ww != 0) {
    const uint32_t link = (ww >> 26) & 0x3Fu, roc = (ww >> 21) & 0x1Fu;
    const uint32_t index = uint32_t(fed) * kMaxLink * kMaxRoc + (link - 1u) * kMaxRoc + roc + 1u;  // 1-based
    // check_roc: only code 25 survives the reference's comparisons (SiPixelRawToClusterGPUKernel.jl:394-468)
    const uint8_t etype = (roc == 25u) ? 25 : 0;
    const bool skip_roc = roc < 8u ? false : (etype != 0);
    bool keep = true;
    if (d.include_errors && skip_roc) {
      uint32_t pos = atomicAdd(&d.ev[e].n_errors, 1u);
      uint32_t gp = atomicAdd(d.err_count, 1u);
      if (gp < uint32_t(d.cap_words)) {
        d.err[5 * size_t(gp) + 0] = uint32_t(e);
        d.err[5 * size_t(gp) + 1] = local;
        d.err[5 * size_t(gp) + 2] = 0xffffffffu;
        d.err[5 * size_t(gp) + 3] = ww;
        d.err[5 * size_t(gp) + 4] = 25u | (uint32_t(fed) << 8);
      }
      (void)pos;
      keep = false;
    }
    uint64_t cab = 0;
    if (keep) {
      if (index < 1u || index > kCablingSize) { atomic_or_warn(&d.ev[e], kWarnModules); keep = false; }
      else cab = c.cab[index - 1];
    }
    if (keep && d.use_quality && ((cab >> 56) & 1u)) keep = false;
    if (keep) {
      const uint32_t raw_id = uint32_t(cab);
      const bool barrel = ((raw_id >> 25) & 0x7u) == 1u;
      const uint32_t layer = barrel ? ((raw_id >> 20) & 0xFu) : 0u;
      const uint32_t the_module = barrel ? ((raw_id >> 2) & 0x3FFu) : 0u;
      const uint32_t panel = barrel ? 0u : ((raw_id >> 10) & 0x3u);
      const int side = barrel ? ((the_module < 5u) ? -1 : 1) : ((panel == 1u) ? -1 : 1);
      const uint32_t roc_in_det = uint32_t((cab >> 48) & 0xFFu);
      int32_t row, col;
      bool conv_err = false;
      if (layer == 1u) {
        col = int32_t((ww >> 15) & 0x3Fu);
        row = int32_t((ww >> 8) & 0x7Fu);
        if (d.include_errors && !(row < 80 && col < 52)) conv_err = true;
      } else {
        const int32_t dcol = int32_t((ww >> 16) & 0x1Fu), pxid = int32_t((ww >> 8) & 0xFFu);
        row = 80 - pxid / 2;
        col = dcol * 2 + pxid % 2;
        if (row < 0) { atomic_or_warn(&d.ev[e], kWarnModules); keep = false; }
        else if (d.include_errors && !((dcol < 26) & (2 <= pxid) & (pxid < 162))) conv_err = true;
      }
      if (keep && conv_err) {
        atomicAdd(&d.ev[e].n_errors, 1u);
        uint32_t gp = atomicAdd(d.err_count, 1u);
        if (gp < uint32_t(d.cap_words)) {
          d.err[5 * size_t(gp) + 0] = uint32_t(e);
          d.err[5 * size_t(gp) + 1] = local;
          d.err[5 * size_t(gp) + 2] = raw_id;
          d.err[5 * size_t(gp) + 3] = ww;
          d.err[5 * size_t(gp) + 4] = 37u | (uint32_t(fed) << 8);
        }
        keep = false;
      }
      if (keep) {
        // frame_conversion, SiPixelRawToClusterGPUKernel.jl:271-350
        int32_t sr, sc, ro, co;
        const bool flip = barrel ? (side == -1 && layer != 1u) : true;
        if (flip) {
          if (roc_in_det < 8u) { sr = 1; sc = -1; ro = 0; co = (8 - int32_t(roc_in_det)) * 52 - 1; }
          else { sr = -1; sc = 1; ro = 159; co = (int32_t(roc_in_det) - 8) * 52; }
        } else {
          if (roc_in_det < 8u) { sr = -1; sc = 1; ro = 159; co = int32_t(roc_in_det) * 52; }
          else { sr = 1; sc = -1; ro = 0; co = (16 - int32_t(roc_in_det)) * 52 - 1; }
        }
        const int32_t grow = sr * row + ro, gcol = sc * col + co;
        if (grow < 0 || gcol < 0) {
          atomic_or_warn(&d.ev[e], kWarnModules);
        } else {
          xx = int16_t(grow);
          yy = int16_t(gcol);
          adc = int32_t(ww & 0xFFu);
          const uint32_t a = uint32_t(adc) < 1023u ? uint32_t(adc) : 1023u;
          pdigi = uint32_t(grow) | (uint32_t(gcol) << 11) | (a << 22);
          mid = int16_t(uint32_t(cab >> 32) & 0xFFFFu);
          rawid = raw_id;
          // calib_digis, gpu_calib_pixel.jl:41-70, with get_ped_and_gain
          if (mid != int16_t(kInvId) && (mid < 0 || mid >= kMaxNumModules)) {
            atomic_or_warn(&d.ev[e], kWarnModules);  // the reference indexes its 2000-entry gain table out of range
            mid = int16_t(kInvId);
          }
          if (mid != int16_t(kInvId)) {
            const float cf = mid < 96 ? 50.f : 47.f;
            const float off = mid < 96 ? -670.f : -60.f;
            const int m = mid;
            const uint32_t offset = c.gain_first[m] + uint32_t(int32_t(yy)) * c.gain_lcd[m] +
                                    2u * (uint32_t(int32_t(xx)) / c.rows_avg);
            const uint32_t kk = offset / 2;
            if (kk >= c.n_gain_pairs) {
              atomic_or_warn(&d.ev[e], kWarnModules);
            } else {
              const uint16_t pr = c.gain_pairs[kk];
              const uint32_t sg = pr & 0xFFu, sp = pr >> 8;
              const bool bad = sp == c.dead_flag || sp == c.noisy_flag;
              const float ped = __fadd_rn(__fmul_rn(float(sp), c.ped_prec), c.min_ped);
              const float gain = __fadd_rn(__fmul_rn(float(sg), c.gain_prec), c.min_gain);
              if (bad) {
                mid = int16_t(kInvId);
                adc = 0;
              } else {
                const float vcal = __fsub_rn(__fmul_rn(float(adc), gain), __fmul_rn(ped, gain));
                const float v = __fadd_rn(__fmul_rn(vcal, cf), off);
                const int32_t t = int32_t(truncf(v));
                adc = t > 100 ? t : 100;
              }
            }
          }
        }
      }
    }
  }
  d.xx[g] = xx; d.yy[g] = yy; d.adc[g] = adc; d.mid[g] = mid; d.pdigi[g] = pdigi; d.rawid[g] = rawid;
}

// raw_to_digi_kernal + calib_digis for the words of one FED slot per warp (kUnpackWarps slots
// per block: a FED holds a few hundred words, which one warp decodes in a few steps). The payload
// is read with 128-bit loads where it sits on 4-byte boundaries (always, for FED sizes in whole
// 64-bit words): the words before the first 16-byte boundary and after the last one are read
// singly, the rest as 16-byte vectors.
constexpr int kUnpackWarps = 8;

__global__ void __launch_bounds__(32 * kUnpackWarps) k_unpack(Dev d) {
  __shared__ __align__(16) uint32_t s_words[kUnpackWarps][128];
  const unsigned lane = threadIdx.x & 31u, wq = threadIdx.x >> 5;
  const int f = blockIdx.x * kUnpackWarps + int(wq), e = blockIdx.y;
  const int NF = d.n_fed_slots;
  if (f >= NF) return;
  const size_t fs = size_t(e) * NF + f;
  const uint32_t nw = d.fed_nw[fs];
  if (nw == 0) return;
  const EvInfo& E = d.ev[e];
  const uint32_t wo = d.fed_wo[fs];
  const uint64_t gbase = uint64_t(E.word_base) + wo;
  if (gbase + nw > uint64_t(d.cap_words)) {
    if (lane == 0) { atomic_or_warn(&d.ev[e], kWarnBuffer); atomicOr(d.status, kWarnBuffer); }
    return;
  }
  const uint8_t* src = d.raw + d.fed_src[fs];
  const uint8_t fed = uint8_t(d.c.fed_ids[f] - 1200u);
  // The reference stores one FED id per word pair (initialize_word_fed,
  // SiPixelRawToClusterGPUKernel.jl:217-226): a FED ending on an odd word leaves its last word in
  // a pair that the next non-empty FED writes (or none: id 0). Only FED sizes that are not whole
  // 64-bit words, on which the reference raises, give odd word counts.
  uint8_t fed_last = fed;
  if ((wo + nw) & 1u) {
    fed_last = 0;
    for (int f2 = f + 1; f2 < NF; ++f2)
      if (d.fed_nw[size_t(e) * NF + f2] > 0) { fed_last = uint8_t(d.c.fed_ids[f2] - 1200u); break; }
  }
  auto word = [&](uint32_t k, uint32_t ww) {
    unpack_word(d, e, wo + k, gbase + k, k + 1 == nw ? fed_last : fed, ww);
  };
  if ((reinterpret_cast<uintptr_t>(src) & 3u) == 0) {
    const uint32_t* src32 = reinterpret_cast<const uint32_t*>(src);
    uint32_t head = uint32_t((16u - (reinterpret_cast<uintptr_t>(src) & 15u)) & 15u) >> 2;
    head = head < nw ? head : nw;
    if (lane < head) word(lane, __ldg(src32 + lane));
    const uint32_t nvec = (nw - head) >> 2;
    const uint4* v = reinterpret_cast<const uint4*>(src32 + head);
    // the warp loads 32 aligned 16-byte vectors (128 words) and decodes them word by word through
    // shared memory, lane l taking words l, l + 32, l + 64, l + 96, so that the per-digi stores
    // of consecutive lanes stay consecutive
    uint32_t* sw = s_words[wq];
    for (uint32_t j0 = 0; j0 < nvec; j0 += 32) {
      if (j0 + lane < nvec) reinterpret_cast<uint4*>(sw)[lane] = __ldg(v + j0 + lane);
      __syncwarp();
      const uint32_t nwords = 4u * min(32u, nvec - j0);
#pragma unroll
      for (uint32_t i = 0; i < 4; ++i) {
        const uint32_t wi = 32u * i + lane;
        if (wi < nwords) word(head + 4u * j0 + wi, sw[wi]);
      }
      __syncwarp();
    }
    for (uint32_t k = head + 4 * nvec + lane; k < nw; k += 32) word(k, __ldg(src32 + k));
  } else {
    for (uint32_t k = lane; k < nw; k += 32) {
      uint32_t ww;
      memcpy(&ww, src + 4ull * k, 4);
      word(k, ww);
    }
  }
}

// count_modules flag: a valid digi whose previous valid digi (in the event) has another id.
__device__ __forceinline__ bool module_start_flag(const Dev& d, uint64_t ebase, uint32_t i) {
  const int16_t id = d.mid[ebase + i];
  if (id == int16_t(kInvId)) return false;
  int64_t j = int64_t(i) - 1;
  while (j >= 0 && d.mid[ebase + j] == int16_t(kInvId)) --j;
  return j < 0 || d.mid[ebase + j] != id;
}

// Module starts per FED slot, one warp per slot (kModWarps slots per block): the flags of 32
// words per step, counted with a ballot.
constexpr int kModWarps = 8;

__global__ void __launch_bounds__(32 * kModWarps) k_modstart_count(Dev d) {
  const int f = blockIdx.x * kModWarps + int(threadIdx.x >> 5), e = blockIdx.y;
  const int NF = d.n_fed_slots;
  if (f >= NF) return;
  const unsigned lane = threadIdx.x & 31u;
  const size_t fs = size_t(e) * NF + f;
  const uint32_t nw = d.fed_nw[fs], wo = d.fed_wo[fs];
  uint32_t cnt = 0;
  const uint64_t ebase = d.ev[e].word_base;
  if (ebase + wo + nw <= uint64_t(d.cap_words))
    for (uint32_t k0 = 0; k0 < nw; k0 += 32) {
      const uint32_t k = k0 + lane;
      cnt += __popc(__ballot_sync(0xffffffffu, k < nw && module_start_flag(d, ebase, wo + k)));
    }
  if (lane == 0) d.fed_nmod[fs] = cnt;
}

// per event: module-start offsets per FED slot, n_modules; zero the cluster counters
__global__ void k_modstart_scan(Dev d) {
  const int e = blockIdx.x;
  const int NF = d.n_fed_slots;
  __shared__ uint32_t sh[33];
  uint32_t carry = 0;
  for (int b = 0; b < NF; b += blockDim.x) {
    int f = b + threadIdx.x;
    uint32_t v = f < NF ? d.fed_nmod[size_t(e) * NF + f] : 0u;
    uint32_t tot;
    uint32_t ex = block_excl_scan(v, sh, &tot);
    if (f < NF) d.fed_nmod[size_t(e) * NF + f] = carry + ex;
    carry += tot;
  }
  uint32_t* cim = d.clus_in_module + size_t(e) * kMaxNumModules;
  for (int i = threadIdx.x; i < kMaxNumModules; i += blockDim.x) cim[i] = 0;
  for (int i = threadIdx.x; i < 64; i += blockDim.x) d.id_seen[size_t(e) * 64 + i] = 0;
  if (threadIdx.x == 0) {
    d.ev[e].repeated_ids = 0;
    uint32_t nm = carry < uint32_t(kMaxNumModules) ? carry : uint32_t(kMaxNumModules);
    d.ev[e].n_modules = nm;
    d.module_start[size_t(e) * (kMaxNumModules + 1)] = nm;
    d.module_start[size_t(e) * (kMaxNumModules + 1) + kMaxNumModules] = 0;
    d.clus_module_start[size_t(e) * (kMaxNumModules + 1)] = 0;
    if (carry > uint32_t(kMaxNumModules)) atomic_or_warn(&d.ev[e], kWarnModules);
  }
}

// The module starts of each FED slot at the slot's offset, one warp per slot, in word order
// (rank of a flag = flags of the earlier lanes plus those of the earlier steps).
__global__ void __launch_bounds__(32 * kModWarps) k_modstart_fill(Dev d) {
  const int f = blockIdx.x * kModWarps + int(threadIdx.x >> 5), e = blockIdx.y;
  const int NF = d.n_fed_slots;
  if (f >= NF) return;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt = (1u << lane) - 1u;
  const size_t fs = size_t(e) * NF + f;
  const uint32_t nw = d.fed_nw[fs], wo = d.fed_wo[fs];
  const uint64_t ebase = d.ev[e].word_base;
  if (ebase + wo + nw > uint64_t(d.cap_words)) return;
  uint32_t carry = d.fed_nmod[fs];
  uint32_t* ms = d.module_start + size_t(e) * (kMaxNumModules + 1);
  for (uint32_t k0 = 0; k0 < nw; k0 += 32) {
    const uint32_t k = k0 + lane;
    const bool fl = k < nw && module_start_flag(d, ebase, wo + k);
    const uint32_t bal = __ballot_sync(0xffffffffu, fl);
    if (fl) {
      const uint32_t r = carry + __popc(bal & lt);
      const uint32_t i1 = wo + k + 1;  // 1-based digi index
      // a module id starting a second run: the event's charge cut runs in serial order
      const uint16_t id = uint16_t(d.mid[ebase + wo + k]);
      if (id < 2048u) {
        const uint32_t bit = 1u << (id & 31u);
        if (atomicOr(&d.id_seen[size_t(e) * 64 + (id >> 5)], bit) & bit) d.ev[e].repeated_ids = 1;
      }
      if (r < uint32_t(kMaxNumModules - 1)) ms[r + 1] = i1;
      else atomicMax(&ms[kMaxNumModules], i1);
    }
    carry += __popc(bal);
  }
}

}  // namespace

void launch_raw(const Dev& d, const Launch& L, const int16_t* fed_slot_of) {
  const int NF = d.n_fed_slots;
  L.mark("start");
  k_fed_table<<<d.E, 256, 0, L.s>>>(d, fed_slot_of);
  k_ev_scan<<<1, 1024, 0, L.s>>>(d.ev, d.E, int(offsetof(EvInfo, n_words)), int(offsetof(EvInfo, word_base)));
  launch_ev_clamp(d, L.s, int(offsetof(EvInfo, n_words)), int(offsetof(EvInfo, word_base)), d.cap_words);
  L.mark("fed_table");
  k_unpack<<<dim3(div_up(NF, kUnpackWarps), d.E), 32 * kUnpackWarps, 0, L.s>>>(d);
  L.mark("unpack_calib");
  const dim3 gm(div_up(NF, kModWarps), d.E);
  k_modstart_count<<<gm, 32 * kModWarps, 0, L.s>>>(d);
  k_modstart_scan<<<d.E, 256, 0, L.s>>>(d);
  k_modstart_fill<<<gm, 32 * kModWarps, 0, L.s>>>(d);
  L.mark("module_starts");
}

void launch_modstart(const Dev& d, const Launch& L) {
  const dim3 gm(div_up(d.n_fed_slots, kModWarps), d.E);
  k_modstart_count<<<gm, 32 * kModWarps, 0, L.s>>>(d);
  k_modstart_scan<<<d.E, 256, 0, L.s>>>(d);
  k_modstart_fill<<<gm, 32 * kModWarps, 0, L.s>>>(d);
}

void launch_ev_scan(const Dev& d, cudaStream_t s, int count_off, int base_off) {
  k_ev_scan<<<1, 1024, 0, s>>>(d.ev, d.E, count_off, base_off);
}

// Events whose region [base, base + count) would pass the buffer capacity are
// emptied (count = 0, buffer warning) and the batch total is capped, so that no
// later kernel indexes past the buffer.
__global__ void k_ev_clamp(EvInfo* ev, int E, int count_off, int base_off, int64_t cap, uint32_t* status) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e > E) return;
  char* b = reinterpret_cast<char*>(ev) + size_t(e) * sizeof(EvInfo);
  uint32_t& cnt = *reinterpret_cast<uint32_t*>(b + count_off);
  const uint32_t base = *reinterpret_cast<const uint32_t*>(b + base_off);
  if (e == E) {
    if (int64_t(cnt) > cap) cnt = uint32_t(cap);
    return;
  }
  if (int64_t(base) + int64_t(cnt) > cap) {
    cnt = 0;
    atomicOr(&ev[e].warnings, kWarnBuffer);
    atomicOr(status, kWarnBuffer);
  }
}

void launch_ev_clamp(const Dev& d, cudaStream_t s, int count_off, int base_off, int64_t cap) {
  k_ev_clamp<<<div_up(d.E + 1, 128), 128, 0, s>>>(d.ev, d.E, count_off, base_off, cap, d.status);
}

}  // namespace pxl
