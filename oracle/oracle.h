// Test infrastructure: CPU oracle for the pixel reconstruction chain.
//
// A serial restatement of the reference's algorithm (Maya-Ali0/CMS-Julia,
// src/julia-serial) in C++, used only by tests/, __graft_entry__.smoke() and
// bench.py's cpu_baseline leg as the checker. It follows the reference's
// operation order, integer widths (Int16/UInt16 wrap), FP32/FP64 promotions and
// iteration order; each function names the reference file:line it restates.
// Parity pinning: the clustering stage is pinned against the reference's own
// known-answer tests (test/gpu_clustering_t.jl, plugin-SiPixelClusterizer/
// testClustering.jl) and the histogram container against test/
// his_to_container_cpu.jl invariants. The rest of the chain is pinned only by
// this restatement: the reference cannot run here (no Julia) and its golden
// data files are not distributed, so stages after clustering are
// "parity unpinned" beyond their restated semantics.
#pragma once
#include <cstdint>
#include <algorithm>
#include <cstring>
#include <vector>

namespace orc {

constexpr int kMaxNumModules = 2000;
constexpr int kNumModules = 1856;
constexpr uint32_t kMaxFed = 150, kMaxLink = 48, kMaxRoc = 8;
constexpr uint32_t kCablingSize = kMaxFed * kMaxLink * kMaxRoc;
constexpr uint16_t kInvId = 9999;
constexpr int kMaxClustersPerModule = 1024;
constexpr uint32_t kMaxHitsInModule = 1024;
constexpr uint32_t kMaxNumClusters = 48 * 1024;  // also the hit capacity
constexpr int kLadders = 148;
constexpr int kPhiBins = 128, kPhiHists = 10, kPhiTotBins = kPhiBins * kPhiHists + 1;
constexpr int kTupleBins = 32 * 1024;            // TrackSOA stride
constexpr int kTupleHitCap = 5 * 32 * 1024;
constexpr int kMaxCellsPerHit = 128;
constexpr int kCellNeighborsRows = 64, kCellTracksRows = 64;
constexpr int kMaxActiveDoublets = 512 * 1024 / 8;
constexpr int kMaxFitsPerMultiplicity = 24 * 1024;
constexpr int kMaxVtx = 1024, kMaxVtxTracks = 32 * 1024;

struct Cabling {
  std::vector<uint32_t> fed, link, roc, raw_id, roc_in_det, module_id;
  std::vector<uint8_t> bad_rocs;
  uint32_t size = 0;  // the reference builds the map with size 0 (SiPixelFedCablingMapGPUWrapperESProducer.jl:38)
};

struct Gains {
  struct RangeAndCols { uint32_t first, last; int32_t cols; };
  std::vector<uint8_t> gain, ped;  // decoding structure {gain, ped} per entry
  RangeAndCols rc[2000];
  float min_ped, max_ped, min_gain, max_gain, ped_precision, gain_precision;
  uint32_t rows_averaged, nbins_encoding, dead_flag, noisy_flag;
};

struct DetParams {
  bool is_barrel, is_pos_z;
  uint16_t layer, index;
  uint32_t raw_id;
  float shift_x, shift_y, charge_width_x, charge_width_y;
  float x0, y0, z0;
  float sx[3], sy[3];
  float px, py, pz;
  float R[9];  // R11 R12 R13 R21 R22 R23 R31 R32 R33
};

struct CpeParams {
  float thickness_b, thickness_e, pitch_x, pitch_y;
  std::vector<DetParams> det;
  float ladder_z[kLadders], ladder_x[kLadders], ladder_y[kLadders], ladder_r[kLadders], ladder_minz[kLadders],
      ladder_maxz[kLadders];
  float endcap_z[2];
  uint32_t layer_start[11];
  uint8_t layer[116];
};

struct BeamSpot { float x, y, z, sigma_z, width_x, width_y, dxdz, dydz, emit_x, emit_y, beta_star; };

struct Conditions {
  Cabling cabling;
  std::vector<uint32_t> fed_ids;
  Gains gains;
  CpeParams cpe;
  BeamSpot bs;
};

// Parses the five conditions blobs; returns 0 or a negative code.
int parse_conditions(const uint8_t* cabling, size_t ncab, const uint8_t* fedids, size_t nfed, const uint8_t* gain,
                     size_t ngain, const uint8_t* cpe, size_t ncpe, const uint8_t* bs, size_t nbs, Conditions* out);

struct PixelError { uint32_t raw_id, word; uint8_t error_type, fed_id; };

struct Cell {
  uint32_t outer_neighbors;  // column in the neighbours matrix (1 = empty column)
  uint32_t tracks;           // column in the tracks matrix (1 = empty column)
  int32_t doublet_id;        // 1-based; -1 once killed by the fishbone
  int16_t layer_pair_id;     // 1-based pair index
  uint16_t used;
  float inner_z, inner_r;
  // 1-based hit ids: the reference's UInt16 (hindex_type, ca_constants.jl:19) never wraps at
  // its 48K hit capacity, so 32 bits give the same values there and room for the extended mode
  uint32_t inner_hit, outer_hit;
};

// Per-event capacities. The defaults are the reference's; the extended mode raises them so
// that high-pileup events are not truncated (hit ids, tuple ids and list entries are 32-bit).
struct Caps {
  uint32_t hits = kMaxNumClusters;              // MAX_NUMBER_OF_HITS clamp of clusModuleStart
  uint32_t doublets = 458752;                   // maxNumberOfDoublets
  uint32_t tuples = kTupleBins;                 // TrackSOA stride
  uint32_t tuple_hits = kTupleHitCap;           // 5 hits per tuple slot
  uint32_t fits_per_mult = kMaxFitsPerMultiplicity;
  uint32_t columns = kMaxActiveDoublets;        // PreAllocMatrix columns (neighbours, tracks)
  uint32_t multiplicity = 48 * 1024;            // TupleMultiplicity entries (MAX_TUPLES)
  uint32_t hit_to_tuple = 4 * 48 * 1024;        // HitToTuple entries (4 * MAX_TUPLES)
  bool extended() const { return hits != kMaxNumClusters || doublets != 458752u || tuples != uint32_t(kTupleBins); }
};

// Fixed-row column store (PreAllocMatrix, CUDACore/simple_matrix.jl:1-58). init() makes every
// column addressable (columns indexed directly, as outer_hit_of_cell is by hit id);
// init_lazy() leaves the columns to extend(), which hands them out in order and backs only
// the ones handed out (the reference preallocates them all; the contents are the same).
struct ColumnStore {
  int rows = 0, cols = 0;
  uint32_t ncol = 0;
  std::vector<uint32_t> data, len;
  void init(int r, int c) {
    if (rows != r || cols != c || len.size() != size_t(c)) { rows = r; cols = c; data.assign(size_t(r) * c, 0); len.assign(c, 0); }
    ncol = 0;
    std::fill(len.begin(), len.end(), 0u);
  }
  void init_lazy(int r, int c) {
    rows = r; cols = c; ncol = 0;
    len.clear();
  }
  uint32_t extend() {
    if (ncol == uint32_t(cols)) return uint32_t(cols);
    ++ncol;
    if (len.size() < ncol) {
      len.resize(ncol, 0);
      if (data.size() < size_t(ncol) * rows) data.resize(std::max(size_t(ncol) * rows, 2 * data.size()));
    }
    return ncol;
  }
  void push(uint32_t col, uint32_t v) {  // 1-based column
    uint32_t& l = len[col - 1];
    if (l == uint32_t(rows)) return;
    data[size_t(col - 1) * rows + l] = v;
    ++l;
  }
  uint32_t length(uint32_t col) const { return len[col - 1]; }
  uint32_t at(uint32_t col, uint32_t k) const { return data[size_t(col - 1) * rows + k]; }  // k 0-based
  void reset() { ncol = 0; std::fill(len.begin(), len.end(), 0u); }
};

struct EventOut {
  // a1-a2
  uint32_t word_counter = 0;
  std::vector<uint32_t> words;
  std::vector<uint8_t> fed_id_pairs;
  std::vector<int16_t> xx, yy, module_ind;
  std::vector<int32_t> adc, clus;
  std::vector<uint32_t> pdigi, raw_id_arr;
  std::vector<PixelError> errors;
  uint32_t n_modules = 0;
  // a3-a7
  uint32_t module_start[kMaxNumModules + 1];
  uint32_t clus_in_module[kMaxNumModules];
  uint32_t module_id[kMaxNumModules];
  uint32_t clus_module_start[kMaxNumModules + 1];
  uint32_t n_clusters = 0;
  // a8-a9
  uint32_t n_hits = 0;
  std::vector<float> xl, yl, xerr, yerr, xg, yg, zg, rg;
  std::vector<int16_t> iphi, xsize, ysize, det_ind;
  std::vector<uint32_t> charge;
  uint32_t hits_layer_start[11];
  uint32_t phi_off[kPhiTotBins];
  std::vector<uint32_t> phi_bins;     // 1-based hit ids
  float agc_ladder[6][kLadders], agc_endcap_z[2];
  // a10-a14
  uint32_t n_cells = 0;
  std::vector<Cell> cells;
  ColumnStore cell_neighbors, cell_tracks, outer_hit_of_cell;
  uint32_t n_tuples = 0, n_tuple_hits = 0;
  std::vector<uint32_t> tuple_off;   // kTupleBins + 1, 1-based starts as the reference stores them
  std::vector<uint32_t> tuple_hits;  // 1-based hit ids
  std::vector<uint16_t> det_hits;    // det_indices bins
  std::vector<uint8_t> quality;      // 0 bad, 1 dup, 2 loose
  uint32_t tm_off[9];                // TupleMultiplicity offsets
  std::vector<uint32_t> tm_bins;     // tuple ids
  // a15-a16
  std::vector<float> pt, eta, chi2;  // kTupleBins
  std::vector<float> state, cov;     // kTupleBins x 5, kTupleBins x 15 (row per tuple)
  std::vector<uint8_t> fitted;       // 1 if the tuple went through the broken-line fit
  // a17
  std::vector<uint32_t> hit_to_tuple_off;
  std::vector<uint32_t> hit_to_tuple_bins;
  // a18-a20
  uint32_t nv_final = 0, n_vtx_tracks = 0;
  std::vector<int16_t> idv;
  std::vector<float> zv, wv, vchi2, ptv2;
  std::vector<int32_t> ndof;
  std::vector<uint16_t> sort_ind;
  // flags for conditions where the reference would raise (assertion or domain error)
  uint32_t flags = 0;
  Caps caps;  // capacities of the last run (from Options)
};

enum Flags : uint32_t {
  kFlagModuleOverflow = 1u << 0,
  kFlagPixelsPerModule = 1u << 1,
  kFlagClustersPerModule = 1u << 2,
  kFlagHitsClamped = 1u << 3,
  kFlagDoubletsCapped = 1u << 4,
  kFlagColumnsFull = 1u << 5,
  kFlagTuplesOverflow = 1u << 6,
  kFlagFitDomain = 1u << 7,
  kFlagFitsCapped = 1u << 8,
  kFlagVertexAssert = 1u << 9,
  kFlagNeighbourOverflow = 1u << 10,
  kFlagFedFormat = 1u << 12,  // a FED header / trailer condition on which the reference raises
};

struct Options {
  bool include_errors = true, use_quality = true, is_run2 = true;
  int stage_mask = 0x3F;  // 1 raw2digi+clusters, 2 rechits, 4 CA, 8 fit, 16 classify, 32 vertices
  Caps caps;
};

void raw_to_clusters(const Conditions& c, const uint8_t* raw_event, size_t nbytes, const Options& o, EventOut& ev);
// Clustering entry on digis alone (count_modules + find_clus + cluster_charge_cut), as the
// reference's clustering test drives them (test/gpu_clustering_t.jl:245-280).
void clusterize_digis(const uint16_t* id, const int16_t* x, const int16_t* y, const int32_t* adc, int n,
                      uint32_t* module_start, uint32_t* clus_in_module, uint32_t* module_id, int32_t* clus,
                      uint16_t* id_out, int apply_charge_cut, uint32_t* flags = nullptr);
void make_hits(const Conditions& c, EventOut& ev);
void ca_tuples(const Conditions& c, EventOut& ev);
void fit_tuples(const Conditions& c, EventOut& ev);
void classify_tuples(const Conditions& c, EventOut& ev);
void make_vertices(const Conditions& c, EventOut& ev);

// Standalone broken-line fit of one track in FP64, N hits (3..8), hits 3xN column-major,
// covariance 6xN column-major; out: par[5] = (phi, tip, 1/pt signed via q*kappa/B-> as
// copyFromCircle!), cov[15], chi2_line, chi2_circle, pt, eta. Returns 0, or nonzero
// when the reference would raise.
int bl_fit_track(const double* hits, const float* ge, int n, double B, double* state5, double* cov15,
                 double* chi2_line, double* chi2_circle, double* pt, double* eta, double* fast_fit4);
// chi2_line + chi2_circle of one track and its gradient with respect to the hit
// coordinates (grad[3n], hit-major) by forward-mode dual numbers (brokenline_fwd.cpp)
double bl_chi2_grad_fwd(const double* hits, const float* ge, int n, double B, double* grad);

// Riemann helix fit of one track (riemann.cpp): state5 = (phi, d0, q/pT, cot(theta), zip),
// the circle and line chi2 and pT; hits row-major per hit, ge 6 per hit. Returns 0 or 1
// (non-finite result), -1 for a hit count outside 3..8.
int riemann_fit_track(const double* hits, const float* ge, int n, double B, double* state5, double* chi2_circle,
                      double* chi2_line, double* pt);

}  // namespace orc
