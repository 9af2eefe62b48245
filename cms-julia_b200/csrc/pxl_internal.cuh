// Internal definitions shared by the kernels of libpxl_b200.so.
//
// Batched layout: a batch of E events is processed by every kernel at once.
// Per-event variable-length data (digis, hits, doublets, tuples) are packed
// back to back; per-event counts and prefix offsets live in EvInfo[E] on the
// device and are produced by the kernels themselves, so the launch sequence
// has no host synchronisation and can be captured in one CUDA graph.
// Per-event work uses 2D grids: blockIdx.y = event, the x dimension strides
// over that event's work items (launch shape from the autotuner).
// Every stage writes its output in the order the serial reference produces it
// (count -> scan -> fill passes, then sorting of short per-key lists), so the
// integer products match the reference element by element.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pxl {

constexpr int kMaxNumModules = 2000;
constexpr uint32_t kMaxLink = 48, kMaxRoc = 8, kMaxFed = 150;
constexpr uint32_t kCablingSize = kMaxFed * kMaxLink * kMaxRoc;  // 57600
constexpr uint16_t kInvId = 9999;
constexpr int kMaxClustersPerModule = 1024;
constexpr int kMaxPixInModule = 4000;
constexpr int kLadders = 148;
constexpr int kPhiTotBins = 1281;
constexpr int kNPairs = 19;
constexpr int kTupleStride = 32 * 1024;
constexpr int kMaxCellsPerHit = 128;
constexpr int kCellRows = 64;
constexpr int kTpParts = 4096;  // parts of the tuple record pool
constexpr int kTpStride = 32;   // words between the parts' counters
constexpr int kMaxActiveColumns = 512 * 1024 / 8;  // MAX_NUM_OF_ACTIVE_DOUBLETS, the default column cap
constexpr uint32_t kHitIdBits = 21;                // event-local hit ids are below 2^21
constexpr uint32_t kMaxHitsPerEvent = 1u << kHitIdBits;
constexpr int kMaxFedSlots = 160;
constexpr int kWarpModulePix = 256;  // modules up to this many digis are clustered by one warp

// per-event warning bits (same values as PXL_WARN_* in include/pxl.h)
enum : uint32_t {
  kWarnModules = 0x1u, kWarnPixels = 0x2u, kWarnClusters = 0x4u, kWarnHitsClamped = 0x8u,
  kWarnDoublets = 0x10u, kWarnColumns = 0x20u, kWarnTuples = 0x40u, kWarnFitDomain = 0x80u,
  kWarnFitsCapped = 0x100u, kWarnVertex = 0x200u, kWarnLists = 0x400u, kWarnBuffer = 0x800u,
  kWarnFedFormat = 0x1000u,
};

struct DetParamsD {
  float shift_x, shift_y, cw_x, cw_y;
  float x0, y0, z0;
  float sx[3], sy[3];
  float px, py, pz;
  float R[9];
  uint8_t is_barrel;
};

struct Conditions {
  // cabling, one 64-bit word per (fed, link, roc) entry:
  // raw_id | module_id << 32 | roc_in_det << 48 | bad_roc << 56 | barrel << 57 | layer << 58 | side(-1) << 62
  const uint64_t* cab;
  const uint32_t* fed_ids;
  int32_t n_fed_ids;
  // gains
  const uint32_t* gain_first;  // [2000]
  const uint32_t* gain_lcd;    // [2000], (last - first) / cols
  const uint16_t* gain_pairs;  // gain | ped << 8 per entry
  uint32_t n_gain_pairs;
  float min_ped, ped_prec, min_gain, gain_prec;
  uint32_t rows_avg, dead_flag, noisy_flag;
  // CPE
  const DetParamsD* det;
  int32_t n_det;
  float thick_b, thick_e, pitch_x, pitch_y;
  uint32_t layer_start[11];
  const float* avg_geom;  // 6*148 + 2, already shifted by the beam spot
  float bs_x, bs_y, bs_z;
  float b_field;  // 1/(pT R) as the CA producer passes it, stored Float32
};

struct EvInfo {
  uint64_t raw_off;  // byte offset of the event in the raw blob
  uint32_t n_words, word_base;
  uint32_t n_modules, n_clusters;
  uint32_t n_hits, hit_base;
  uint32_t n_items, item_base;      // doublet work items (inner hits over the layer pairs)
  uint32_t n_cells, cell_base;
  uint32_t n_cells_raw;             // length of the event's cell region (= n_cells)
  uint32_t n_tuples, tuple_base;
  uint32_t n_tuple_hits, tuple_hit_base;
  uint32_t n_tuples_raw, n_tuple_hits_raw;
  uint32_t n_vtx, n_vtx_tracks;
  uint32_t n_errors, error_base;
  uint32_t warnings;
  uint32_t tm_off[9];               // tuple multiplicity offsets (bins 1..8, reference layout)
  uint32_t n_dup_cells, dup_cell_base;
  uint32_t n_cols_nb, n_cols_tr;    // non-empty neighbour / track lists (column store use)
  uint32_t n_fit3, n_fit4;          // tuples fitted with 3 and with 4 hits (fit5as4 included)
  uint32_t n_refit3, n_refit4;      // of those, mixed-precision fits redone in FP64
  // 1 when a module id starts more than one module run (only corrupted data does that): the
  // charge cut of such an event runs in the reference's serial order (k_charge_cut_serial)
  uint32_t repeated_ids;
  // when the event found more tuples than it keeps: the hit offset where the last kept tuple's
  // hits really end (its visible size is 0, as the reference's overflowing bulk_finalize_fill
  // leaves it); 0 otherwise
  uint32_t last_tuple_end;
};

// The fields the doublet search reads of an outer-hit candidate, packed in phi-bin order
// so that the search loads one 16-byte record per candidate.
// bounding box and charges (total, first / last row and column) of one cluster
struct ClusSumRec {
  uint32_t minr, maxr, minc, maxc;
  int32_t q, qfx, qlx, qfy, qly;
};

struct alignas(16) HitRec {
  float z, r;
  int16_t iphi, ysize;
  uint32_t det_id;  // detector index (below 2048) << kHitIdBits | event-local 0-based hit index
  __host__ __device__ int det() const { return int(det_id >> kHitIdBits); }
  __host__ __device__ uint32_t id() const { return det_id & (kMaxHitsPerEvent - 1u); }
};

// Everything a kernel may need, passed by value.
struct Dev {
  Conditions c;
  int32_t E;
  int32_t n_fed_slots;
  // limits
  int64_t cap_words, cap_hits, cap_cells, cap_tuples, cap_tuple_hits, cap_items, cap_pairs, cap_long;
  uint32_t hits_per_event, doublets_per_event, tuples_per_event, fits_per_mult, columns_per_event;
  int32_t include_errors, use_quality;
  int32_t fit_precision;     // 0 FP64 (the reference), 1 mixed precision
  int32_t apply_charge_cut;  // 1 in the chain; 0 only for the stand-alone clustering entry
  // inputs
  const uint8_t* raw;
  const uint64_t* ev_off;
  EvInfo* ev;
  // FED table, [E][n_fed_slots]
  uint64_t* fed_src;
  uint32_t* fed_nw;
  uint32_t* fed_wo;
  uint32_t* fed_nmod;  // module starts found per FED slot
  // digis [cap_words]
  int16_t* xx; int16_t* yy; int32_t* adc; int16_t* mid; int32_t* clus; uint32_t* pdigi; uint32_t* rawid;
  // FED error records [cap_words]: raw_id, word, type | fed << 8
  uint32_t* err;
  uint32_t* err_count;  // per event
  uint32_t* id_seen;    // [E][64] module ids that start a run (bit per id below 2048)
  // clusters, per event
  uint32_t* module_start;       // [E][2001]
  uint32_t* clus_in_module;     // [E][2000]
  uint32_t* module_id;          // [E][2000]
  uint32_t* clus_module_start;  // [E][2001]
  // hits [cap_hits]
  float* xl; float* yl; float* xerr; float* yerr; float* xg; float* yg; float* zg; float* rg;
  int16_t* iphi; int16_t* xsize; int16_t* ysize; int16_t* detind; uint32_t* charge;
  uint32_t* hits_layer_start;  // [E][11]
  uint32_t* phi_off;           // [E][1281]
  uint32_t* phi_bins;          // [cap_hits], 1-based hit ids
  struct HitRec* hit_rec;      // [cap_hits] the binned hits' doublet fields, in bin order
  struct HitRec* hit_rec_s;    // [cap_hits] the same, sorted by iphi (as uint16) within each bin
  uint16_t* hit_u_s;           // [cap_hits] their iphi (as uint16), for the phi-window searches
  struct ClusSumRec* hit_sum;  // [cap_hits] per-cluster sums of getHits, input of the CPE
  uint32_t* hit_me;            // [cap_hits] module of the hit's record, 0xFFFFFFFF when none
  float4* hit_xyzr;            // [cap_hits] global x, y, z, r of each hit
  // doublets: work items and cells
  uint32_t* pair_cum;      // [E][19] cumulative inner-layer sizes over the layer pairs
  uint32_t* item_cnt;      // [cap_items] doublets per inner hit item, then exclusive positions
  uint32_t* item_pool;     // [cap_items] first pool entry of the item's outer hits (kNoPool: none)
  uint32_t* dbl_pool;      // [cap_cells] outer hits found by the count pass, 32-item groups in item order
  uint32_t* dbl_pool_ctr;  // [1] entries taken from dbl_pool
  uint32_t* cell_inner;    // [cap_cells] event-local 0-based hit index
  uint32_t* cell_outer;
  uint8_t* cell_pair;      // 0-based layer pair
  int32_t* cell_id;        // reference doublet id: 1-based, -1 when killed
  uint8_t* cell_used;
  // outer-hit-of-cell lists (CSR over hits)
  uint32_t* ohc_cnt;       // [cap_hits + 1] counts -> offsets
  uint32_t* ohc_cur;       // [cap_hits] fill cursors
  uint32_t* ohc_list;      // [cap_cells] global cell indices
  float2* ohc_rec;         // [cap_cells] per list entry: r, z of the cell's inner hit (connect's candidate);
                           // r negative when that hit is on an inner-barrel module
  // cell neighbours (CSR over cells)
  uint2* cn_pairs;         // [cap_pairs] passing (candidate, cell) pairs of the connection test
  uint32_t* cn_pair_ctr;   // [1] entries of cn_pairs
  uint32_t* cn_cnt;        // [cap_cells + 1]
  uint32_t* cn_cur;        // [cap_cells]
  uint32_t* cn_list;       // [cap_pairs] global cell indices
  uint2* long_lists;       // [cap_long] (first entry, length) of the lists left to k_sort_long
  uint32_t* long_ctr;      // [1]
  // tuples
  uint64_t* tstart_cnt;    // [cap_cells + 1] (tuples << 32 | hits) per start cell -> exclusive positions
  // tuples found by the count pass, in kTpParts parts of tp_part records each (a warp appends to
  // part (warp id mod kTpParts)): header (start cell, tuple ordinal and hit offset within the start
  // cell's tuples, event << 4 | hits) and the tuple's doublets (two uint4, unused entries 0)
  uint4* tp_hdr;           // [kTpParts * tp_part]
  uint4* tp_cells;         // [2 * kTpParts * tp_part]
  uint32_t* tp_ctr;        // [kTpParts * kTpStride + 1] records per part; last word: a part overflowed
  uint32_t tp_part;
  uint32_t* tuple_off;     // [cap_tuples + 1] global hit offsets (0-based, packed)
  uint32_t* tuple_hits;    // [cap_tuple_hits] event-local 0-based hit index
  uint16_t* tuple_det;     // [cap_tuple_hits] detector index of each tuple hit (det_indices)
  uint8_t* quality;        // [cap_tuples] 0 bad 1 dup 2 loose
  uint32_t* tuple_cell;    // [cap_tuple_hits] (cell of each doublet of a tuple) for the cell -> track lists
  uint32_t* ct_cnt;        // [cap_cells + 1] tracks per cell -> offsets
  uint32_t* ct_cur;        // [cap_cells]
  uint32_t* ct_list;       // [cap_tuple_hits] global tuple indices
  uint32_t* tm_bins;       // [cap_tuples] tuple multiplicity, global tuple indices, bins ascending by id
  // fit results [cap_tuples]
  float* t_state; float* t_cov; float* t_pt; float* t_eta; float* t_chi2; uint8_t* t_fitted;
  uint32_t* fit_list;      // [cap_tuples] per event: 3-hit fits from the front, 4-hit fits from the back
  uint32_t* refit_list;    // [cap_tuples] per event, the same way: mixed-precision fits redone in FP64
  // hit -> tuple lists
  uint32_t* htt_cnt;       // [cap_hits + 1]
  uint32_t* htt_cur;
  uint32_t* htt_list;      // [cap_tuple_hits]
  // cells with >= 2 tracks, compacted per event
  uint32_t* dup_bits;      // [cap_cells / 32 + 2] cells with two or more tracks, one bit each
  uint32_t* dup_list;      // [cap_cells] those cells in order, at the event's cell base
  uint32_t* dup_eoff;      // [cap_cells + E + 1] their entry offsets, at cell base + event index
  uint32_t* dup_et;        // [cap_tuple_hits] entries: event-local tuple id, at the tuple-hit base
  uint32_t* dup_ek;        // [cap_tuple_hits] entries: |tip| bits
  // vertices, per event
  int16_t* idv;            // [cap_tuples] per tuple (global tuple index), -1 when unused
  float* vws_zt; float* vws_ezt2; float* vws_ptt2;  // [cap_tuples] vertex-finder workspace per selected track
  int32_t* vws_iv; uint32_t* vws_itrk; uint8_t* vws_izt; uint32_t* vws_bins;
  float* zv; float* wv; float* vchi2; float* ptv2;  // [E][1024]
  int32_t* ndof;           // [cap_tuples] per event slot region (same packing as tuples)
  uint16_t* sort_ind;      // [E][1024]
  // scratch for scans
  uint32_t* scan_tmp;      // [scan tile sums]
  uint64_t* scan_tmp64;
  uint32_t* status;        // [1] global status bits (buffer overflow)
  // module work lists (event << 11 | module position): a header of kListHeader counters,
  // then cap_big entries per list (kListClus*, kListHitsBig)
  uint32_t* big_list;
  int64_t cap_big;
  // launch shape
  int32_t bpe;             // blocks per event for per-event kernels
  // persistent work-queue launches (workqueue.cu): events by decreasing hit count, and per
  // launch slot a pulled-block counter and the virtual-block prefix over that order
  uint32_t* wq_order;      // [E]
  uint32_t* wq_head;       // [kWqSlots]
  uint32_t* wq_prefix;     // [kWqSlots][E + 1]
};

// One set of device export buffers of pxl_export_async: the batch's loose tracks and vertices
// packed event after event (index rows: first track, tracks, first vertex, vertices).
struct ExportSet {
  uint32_t* index = nullptr;
  float* state = nullptr; float* cov = nullptr; float* pt = nullptr; float* eta = nullptr; float* chi2 = nullptr;
  uint8_t* n_hits = nullptr; int16_t* vertex = nullptr; uint32_t* tuple = nullptr;
  float* zv = nullptr; float* wv = nullptr; float* vchi2 = nullptr; float* ptv2 = nullptr; int32_t* ndof = nullptr;
  uint32_t cap_tracks = 0, cap_vertices = 0;
  cudaEvent_t ready = nullptr, copied = nullptr;  // kernels done (compute stream), copies done (copy stream)
};

// ---------------------------------------------------------------- persistent work queues
// A per-event kernel runs either on a static grid (blocks per event x events; the hardware
// hands the blocks out in event order) or as a persistent grid of one wave of CTAs that pull
// virtual blocks from a device counter. An event gets as many virtual blocks as its work needs
// (its count of the stage's work units over the units one block takes), and the events come
// most work first, so that the longest events start early and the short ones fill the tail.
// Either way the kernel body sees (event, block, blocks of the event).
constexpr int kWqSlots = 16;  // persistent launches per chain run (each its own counter)

struct WorkQueue {
  const uint32_t* order = nullptr;   // [n] events, most work first
  const uint32_t* prefix = nullptr;  // [n + 1] virtual blocks before each order slot
  uint32_t* head = nullptr;          // pulled virtual blocks
  uint32_t n = 0;
};

template <bool kQ, class F>
__device__ __forceinline__ void for_each_vblock(const WorkQueue& q, F&& body) {
  if constexpr (!kQ) {
    body(int(blockIdx.y), uint32_t(blockIdx.x), uint32_t(gridDim.x));
  } else {
    __shared__ uint32_t s_v;
    const uint32_t total = q.prefix[q.n];
    for (;;) {
      __syncthreads();  // the previous block's shared memory and s_v are free again
      if (threadIdx.x == 0) s_v = atomicAdd(q.head, 1u);
      __syncthreads();
      const uint32_t v = s_v;
      if (v >= total) return;
      // the order slot i with prefix[i] <= v < prefix[i + 1] (slots without work are skipped)
      uint32_t lo = 0, hi = q.n;
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (q.prefix[mid] <= v) lo = mid; else hi = mid;
      }
      body(int(q.order[lo]), v - q.prefix[lo], q.prefix[lo + 1] - q.prefix[lo]);
    }
  }
}

// Track lists by hit count for the stand-alone fits (workspace layout).
constexpr int kFitMaxN = 8;
struct FitPlan {
  uint32_t count[kFitMaxN + 1];   // tracks with n hits, n = 3..8
  uint32_t cursor[kFitMaxN + 1];
  uint32_t base[kFitMaxN + 1];    // first list entry of each hit count
  uint32_t pad;
  int32_t list[1];                // track indices grouped by hit count (n_tracks entries)
  __host__ __device__ uint32_t base_of(int n) const { return base[n]; }
};
int64_t fit_plan_bytes(int32_t n_tracks);
int fit_plan_build(const int32_t* offs, int32_t n, FitPlan* plan, int32_t* status, cudaStream_t s);

// Two side streams of the current device with a fork event and two join events, created on
// first use; side_streams_lock returns them held by the caller until side_streams_unlock
// (nullptr, and nothing held, when they could not be created).
struct SideStreams {
  cudaStream_t st[2];
  cudaEvent_t fork, join[2];
};
SideStreams* side_streams_lock();
void side_streams_unlock();

// Enqueues launch(k, stream) for k = 0 .. n-1 round robin on s and the two side streams,
// forked from s and joined back into it: the per-hit-count fit kernels then overlap where an
// earlier one's last blocks leave SMs idle. Without side streams every launch goes on s.
template <class F>
int fan_out(cudaStream_t s, int n, F&& launch) {
  SideStreams* ss = side_streams_lock();
  if (!ss) {
    for (int k = 0; k < n; ++k) launch(k, s);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
  }
  bool ok = cudaEventRecord(ss->fork, s) == cudaSuccess && cudaStreamWaitEvent(ss->st[0], ss->fork, 0) == cudaSuccess &&
            cudaStreamWaitEvent(ss->st[1], ss->fork, 0) == cudaSuccess;
  for (int k = 0; ok && k < n; ++k) launch(k, k % 3 == 0 ? s : ss->st[k % 3 - 1]);
  for (int j = 0; ok && j < 2; ++j)
    ok = cudaEventRecord(ss->join[j], ss->st[j]) == cudaSuccess && cudaStreamWaitEvent(s, ss->join[j], 0) == cudaSuccess;
  side_streams_unlock();
  return ok && cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
  const unsigned lane = threadIdx.x & 31u;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= unsigned(o)) v += t;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread (blockDim.x <= 1024, multiple of 32).
// `sh` needs 33 uint32 of shared memory. Returns the exclusive prefix; *total gets the sum.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t* total) {
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  const unsigned nw = (blockDim.x + 31) >> 5;
  uint32_t inc = warp_incl_scan(v);
  if (lane == 31) sh[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    uint32_t s = lane < nw ? sh[lane] : 0u;
    uint32_t si = warp_incl_scan(s);
    if (lane < nw) sh[lane] = si - s;
    if (lane == nw - 1) sh[32] = si;
  }
  __syncthreads();
  uint32_t r = sh[wid] + inc - v;
  if (total) *total = sh[32];
  __syncthreads();
  return r;
}

__device__ __forceinline__ void atomic_or_warn(EvInfo* ev, uint32_t bits) { atomicOr(&ev->warnings, bits); }

// module work lists between the per-module kernels
enum : int { kListClusBig = 0, kListHitsBig = 1, kListClusMid = 2, kListClusSmall = 3, kNumLists = 4, kListHeader = 4 };

__device__ __forceinline__ void push_module(const Dev& d, int list, int e, uint32_t m) {
  const uint32_t slot = atomicAdd(&d.big_list[list], 1u);
  if (slot < uint32_t(d.cap_big)) d.big_list[kListHeader + size_t(list) * d.cap_big + slot] = (uint32_t(e) << 11) | m;
}
__device__ __forceinline__ uint32_t list_size(const Dev& d, int list) {
  const uint32_t c = d.big_list[list];
  return c < uint32_t(d.cap_big) ? c : uint32_t(d.cap_big);
}
__device__ __forceinline__ uint32_t list_entry(const Dev& d, int list, uint32_t i) {
  return d.big_list[kListHeader + size_t(list) * d.cap_big + i];
}

// End of a module's digi range as find_clus and getHits bound it: the 1-based index of the
// first valid digi with another module id after first1, or n_el if none. The next entry
// of the module-start list holds exactly this, except when more than 2000 module runs
// overflowed the list: its last slot then holds the last run, and the module before it
// must scan (gpu_clustering.jl:106-114, gpuPixelRecHits.jl:149-156).
__device__ __forceinline__ uint32_t module_end1(const int16_t* mid, uint64_t eb, const uint32_t* ms, uint32_t m,
                                                uint32_t nmod, uint32_t n_el, uint32_t first1, int16_t this_id) {
  if (m + 1 >= nmod) return n_el;
  if (!(nmod == uint32_t(kMaxNumModules) && m + 2 == nmod)) return ms[m + 2];
  for (uint32_t i1 = first1; i1 <= n_el; ++i1) {
    const int16_t id = mid[eb + i1 - 1];
    if (id != int16_t(kInvId) && id != this_id) return i1;
  }
  return n_el;
}

// Bits of the event's cells [c_lo, c_hi) in word wi of the two-or-more-tracks bitmap
// (set by k_sort_cell_lists<1> in k_ca.cu): walking the words in order walks those cells in order.
__device__ __forceinline__ uint32_t dup_word(const Dev& d, uint64_t wi, uint64_t c_lo, uint64_t c_hi) {
  uint32_t m = d.dup_bits[wi];
  if (wi == (c_lo >> 5)) m &= ~0u << (c_lo & 31);
  if (wi == ((c_hi - 1) >> 5) && (c_hi & 31)) m &= (1u << (c_hi & 31)) - 1u;
  return m;
}

inline int div_up(int64_t a, int64_t b) { return int((a + b - 1) / b); }

// ---------------------------------------------------------------- launchers (per stage file)
// Optional per-kernel timing: when enabled, the launchers record a CUDA event after
// every kernel; segment i lasts from event i-1 to event i.
struct Prof {
  static constexpr int kMax = 128;
  bool on = false;
  int n = 0;
  cudaEvent_t ev[kMax] = {};
  const char* name[kMax] = {};
};

// Stages whose launch shape (blocks per event) the autotuner chooses.
enum TuneSeg : int {
  kTuneDoublets, kTuneHitLists, kTuneConnect, kTuneCellLists, kTuneFishbone, kTuneNtuplets, kTuneCellTracks,
  kTuneEarlyDup, kTuneClassify, kTuneHitToTuple, kTuneFitTuples, kTuneCount
};

struct Launch {
  cudaStream_t s;
  int bpe;        // blocks per event
  int tpb;        // threads per block
  Prof* prof = nullptr;
  // [kTuneCount] launch shape per stage: > 0 blocks per event (static grid), < 0 persistent
  // work queue with -value loop strides per virtual block, 0 the default
  const int* tune = nullptr;
  const int* wq_ctas = nullptr;  // [kTuneCount] CTAs of one persistent wave per stage (0: none)
  mutable int wq_slot = 0;       // next work-queue slot of the run
  int bpe_of(int seg) const {
    const int b = (tune && tune[seg] > 0) ? tune[seg] : bpe;
    return b > 0 ? b : 64;
  }
  // loop strides per virtual block when the stage runs from a work queue, else 0
  int queue_of(int seg) const { return (tune && tune[seg] < 0 && wq_ctas && wq_ctas[seg] > 0) ? -tune[seg] : 0; }
  void mark(const char* nm) const {
    if (prof && prof->on && prof->n < Prof::kMax) {
      cudaEventRecord(prof->ev[prof->n], s);
      prof->name[prof->n] = nm;
      ++prof->n;
    }
  }
};

// workqueue.cu: the event order of the run (most hits first, once the hits are known), and the
// plan of one persistent launch: virtual blocks per event = ceil(count / units_per_block) with
// count the EvInfo field at count_off
void launch_wq_order(const Dev& d, cudaStream_t s);
WorkQueue launch_wq_plan(const Dev& d, const Launch& L, int count_off, uint32_t units_per_block);

void launch_raw(const Dev& d, const Launch& L, const int16_t* fed_slot_of);  // a1-a4
void launch_modstart(const Dev& d, const Launch& L);  // a4 only (digis already in place)
void launch_ev_scan(const Dev& d, cudaStream_t s, int count_off, int base_off);
void launch_ev_clamp(const Dev& d, cudaStream_t s, int count_off, int base_off, int64_t cap);
void launch_cluster(const Dev& d, const Launch& L);   // a5-a7
void launch_rechits(const Dev& d, const Launch& L);   // a8-a9
void launch_ca(const Dev& d, const Launch& L);        // a10-a14
int prepare_ca_kernels(int ctas[kTuneCount]);         // CTAs of one persistent wave per stage (current device)
void launch_fit(const Dev& d, const Launch& L);       // a15-a16
void launch_classify(const Dev& d, const Launch& L);  // a17
int prepare_select_kernels();  // kernel attributes (dynamic shared memory) on the current device
void launch_vertices(const Dev& d, const Launch& L);  // a18-a20

// global scans over packed arrays (scan.cu)
// In place exclusive scan of data[0..n), n = min(ncap, *n_dev) (n_dev may be null); data[n] = total.
void excl_scan_u32(uint32_t* data, int64_t ncap, const uint32_t* n_dev, uint32_t* tmp, cudaStream_t s);
void excl_scan_u64(uint64_t* data, int64_t ncap, const uint32_t* n_dev, uint64_t* tmp, cudaStream_t s);
// out[0] = 0, out[i + 1] = exclusive prefix of in[i]: offsets of lists filled by
// atomicAdd(&out[key + 1], 1) (scan.cu)
void excl_scan_shift_u32(const uint32_t* in, uint32_t* out, int64_t ncap, const uint32_t* n_dev, uint32_t* tmp,
                         cudaStream_t s);
int64_t scan_tmp_elems(int64_t n);

}  // namespace pxl

struct PxlCtx;
// copy-out of the CA / fit / vertex products in the reference's layout (k_products.cu)
int64_t copy_ca_product(PxlCtx* ctx, int32_t e, int32_t product, void* dst, int64_t max_bytes);
