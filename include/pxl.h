/*
 * pxl.h - C ABI of the B200 pixel reconstruction chain (libpxl_b200.so).
 *
 * Drop-in boundary for the five producers of Maya-Ali0/CMS-Julia's serial
 * chain (paths relative to src/julia-serial/):
 *   BeamSpotToPOD            plugin-BeamSpotProducer/BeamSpotToPOD.jl:4-16
 *   SiPixelRawToClusterCUDA  plugin-SiPixelClusterizer/SiPixelRawToClusterCUDA.jl:27-152
 *   SiPixelRecHitCUDA        plugin-SiPixelRecHits/SiPixelRecHitCUDA.jl:25-45
 *   CAHitNtupletCUDA         plugin-PixelTriplets/ca_hit_ntuplet.jl:10-19
 *   PixelVertexProducerCUDA  plugin-PixelVertexFinding/pixel_vertex_producer_cuda.jl:3-30
 * and of the ES producers that feed them with conditions.
 *
 * Every function returns an int32 status: 0 ok, > 0 capacity or data warning
 * (PXL_WARN_* bits, the products are valid up to the reference's truncation
 * rules), < 0 fatal (PXL_ERR_*). No C++ exception crosses this boundary.
 * Pointers are plain host pointers unless a parameter says "device".
 * A context is not reentrant: one context per host thread / stream.
 */
#ifndef PXL_H
#define PXL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PXL_ABI_VERSION 3  /* 3: PxlEventCounts.n_fits_fp64 */

/* fatal status codes */
#define PXL_ERR_ARG (-1)
#define PXL_ERR_CUDA (-2)
#define PXL_ERR_CONDITIONS (-3)
#define PXL_ERR_CAPACITY (-4)
#define PXL_ERR_STATE (-5)

/* per-event warning bits, the places where the reference truncates or raises */
#define PXL_WARN_MODULES 0x1u          /* more than 2000 module starts (gpu_clustering.jl:141) */
#define PXL_WARN_PIXELS_PER_MODULE 0x2u /* > 4000 pixels in a module (gpu_clustering.jl:204-207) */
#define PXL_WARN_CLUSTERS_PER_MODULE 0x4u /* > 1024 clusters (gpu_cluster_charge_cut.jl:111-135) */
#define PXL_WARN_HITS_CLAMPED 0x8u     /* clusModuleStart clamped to the hit capacity */
#define PXL_WARN_DOUBLETS 0x10u        /* doublet capacity reached (gpu_pixel_doublets.jl:342-346) */
#define PXL_WARN_COLUMNS 0x20u         /* neighbour / track column store full */
#define PXL_WARN_TUPLES 0x40u          /* tuple capacity reached (hist_to_container.jl:234-236) */
#define PXL_WARN_FIT_DOMAIN 0x80u      /* a fit met a condition on which the reference raises */
#define PXL_WARN_FITS_CAPPED 0x100u    /* > 24576 tuples of one multiplicity (broken_line_fit_on_gpu.jl:46-50) */
#define PXL_WARN_VERTEX 0x200u         /* vertex finder assertion condition */
#define PXL_WARN_LISTS 0x400u          /* a per-hit / per-cell list exceeded its row capacity */
#define PXL_WARN_BUFFER 0x800u         /* batch buffer capacity exceeded: products incomplete */
#define PXL_WARN_FED_FORMAT 0x1000u    /* a FED header / trailer / size on which the reference raises
                                          (SiPixelRawToClusterCUDA.jl:104-128, ErrorChecker.jl:116-137) */

/* stage mask for the producer boundary */
#define PXL_STAGE_DIGIS 0x1u     /* SiPixelRawToClusterCUDA: digis + clusters */
#define PXL_STAGE_HITS 0x2u      /* SiPixelRecHitCUDA */
#define PXL_STAGE_TUPLES 0x4u    /* CAHitNtupletCUDA: doublets, ntuplets */
#define PXL_STAGE_FIT 0x8u       /* CAHitNtupletCUDA: broken-line fit */
#define PXL_STAGE_CLASSIFY 0x10u /* CAHitNtupletCUDA: classify_tuples */
#define PXL_STAGE_VERTICES 0x20u /* PixelVertexProducerCUDA */
#define PXL_STAGE_ALL 0x3Fu

typedef struct PxlCtx PxlCtx;

/* The five ES products, each in the reference's binary layout. Replaces
 * SiPixelFedCablingMapGPUWrapperESProducer.jl:27-67 (cablingMap.bin, fedIds.bin),
 * SiPixelGainCalibrationForHLTGPUESProducer.jl:14-57 (gain.bin),
 * PixelCPEFastESProducer.jl:16-113 (cpefast.bin), BeamSpotESProducer.jl:11-41 (beamspot.bin). */
typedef struct PxlConditions {
  const uint8_t* cabling_map; size_t cabling_map_bytes;
  const uint8_t* fed_ids; size_t fed_ids_bytes;
  const uint8_t* gain; size_t gain_bytes;
  const uint8_t* cpe; size_t cpe_bytes;
  const uint8_t* beamspot; size_t beamspot_bytes;
} PxlConditions;

/* Hard-coded parameters of the reference (SiPixelRawToClusterCUDA.jl:40-44,
 * ca_hit_ntuplet_generator.jl:9-30, pixel_vertex_producer_cuda.jl:11-19) and the
 * batch buffer sizes. Capacities at their defaults reproduce the reference's
 * truncation rules; larger values give the extended-capacity mode. */
typedef struct PxlParams {
  int32_t device;
  int32_t max_events;                /* events per batch */
  int64_t max_words;                 /* FED words per batch (sum over events) */
  int64_t max_hits;                  /* hits per batch */
  int64_t max_doublets;              /* doublets per batch */
  int64_t max_tuples;                /* tuples per batch */
  int32_t hits_per_event;            /* 49152 (MAX_NUMBER_OF_HITS); at most 2097152 (2^21) */
  int32_t doublets_per_event;        /* 458752 (maxNumberOfDoublets) */
  int32_t tuples_per_event;          /* 32768 (TrackSOA stride) */
  int32_t fits_per_multiplicity;     /* 24576 (MAX_NUM_OF_CONCURRENT_FITS) */
  int32_t include_errors;            /* 1 */
  int32_t use_quality;               /* 1 */
  int32_t blocks_per_event;          /* launch shape; 0 = chosen by the autotuner */
  int32_t threads_per_block;         /* launch shape; 0 = chosen by the autotuner */
  int32_t columns_per_event;         /* 65536 (MAX_NUM_OF_ACTIVE_DOUBLETS): cells with a neighbour or
                                        track list; a warning (PXL_WARN_COLUMNS) above it */
  int32_t fit_precision;             /* broken-line fits of the chain: 0 = FP64 as the reference
                                        (broken_line_fit_on_gpu.jl:28-30); 1 = FP32 arithmetic with
                                        the band solve, transport and covariance in FP64 (pxl_bl_fit
                                        precision 1); a tuple whose FP32 fit gives pT >= 50 GeV (or
                                        no finite pT) is fitted again in FP64 (n_fits_fp64) */
} PxlParams;

typedef struct PxlEventCounts {
  uint32_t n_words;      /* digis = 32-bit FED words (word_counter) */
  uint32_t n_modules;    /* moduleStart[1] */
  uint32_t n_clusters;   /* clusModuleStart[2000] */
  uint32_t n_hits;
  uint32_t n_doublets;
  uint32_t n_tuples;
  uint32_t n_tuple_hits;
  uint32_t n_vertices;   /* nvFinal */
  uint32_t n_vertex_tracks;
  uint32_t warnings;     /* PXL_WARN_* */
  uint32_t n_errors;     /* FED error records */
  uint32_t n_fits_fp64;  /* fit_precision 1: tuples fitted again in FP64 (stiff tracks) */
} PxlEventCounts;

/* Products in the reference's layout, for pxl_copy_product (element type in brackets,
 * length per event). Values are those the reference stores, 1-based where it is. */
enum PxlProduct {
  /* SiPixelDigisSoA (CUDADataFormats/SiPixelDigisSoA.jl:15-49), length n_words */
  PXL_P_XX = 1,         /* int16 */
  PXL_P_YY = 2,         /* int16 */
  PXL_P_ADC = 3,        /* int32 */
  PXL_P_MODULE_IND = 4, /* int16 */
  PXL_P_CLUS = 5,       /* int32 */
  PXL_P_PDIGI = 6,      /* uint32 */
  PXL_P_RAW_ID = 7,     /* uint32 */
  /* SiPixelClustersSoA (CUDADataFormats/SiPixelClusterSoA.jl:64-92) */
  PXL_P_MODULE_START = 10,      /* uint32[2001] */
  PXL_P_CLUS_IN_MODULE = 11,    /* uint32[2000] */
  PXL_P_MODULE_ID = 12,         /* uint32[2000] */
  PXL_P_CLUS_MODULE_START = 13, /* uint32[2001] */
  /* TrackingRecHit2DSOAView (CUDADataFormats/TrackingRecHit2DSOAView.jl:35-55), length n_hits */
  PXL_P_XL = 20, PXL_P_YL = 21, PXL_P_XERR = 22, PXL_P_YERR = 23, /* float */
  PXL_P_XG = 24, PXL_P_YG = 25, PXL_P_ZG = 26, PXL_P_RG = 27,     /* float */
  PXL_P_IPHI = 28,            /* int16 */
  PXL_P_CHARGE = 29,          /* uint32 */
  PXL_P_XSIZE = 30, PXL_P_YSIZE = 31, PXL_P_DET_IND = 32, /* int16 */
  PXL_P_HITS_LAYER_START = 33, /* uint32[11] */
  PXL_P_PHI_OFF = 34,          /* uint32[1281] */
  PXL_P_PHI_BINS = 35,         /* uint16[n_hits], 1-based hit ids (PXL_ERR_CAPACITY above 65535 hits) */
  PXL_P_AVERAGE_GEOMETRY = 36, /* float[6*148+2], beam-spot shifted */
  PXL_P_PHI_BINS32 = 37,       /* uint32[n_hits], 1-based hit ids (any hit count) */
  /* CA internals, for parity tests */
  PXL_P_CELLS = 40,            /* int32[5*n_doublets]: inner, outer (1-based), layer pair (1-based), doublet id, used */
  PXL_P_CELL_NEIGHBORS = 41,   /* uint32 CSR: n_doublets+1 offsets, then 1-based cell ids */
  PXL_P_CELL_TRACKS = 42,      /* uint32 CSR: n_doublets+1 offsets, then tuple ids */
  PXL_P_OUTER_HIT_OF_CELL = 43,/* uint32 CSR: n_hits+1 offsets, then 1-based cell ids */
  PXL_P_TUPLE_MULTIPLICITY = 44, /* uint32[9] offsets then uint32 tuple ids (bin order) */
  /* TrackSOA (CUDADataFormats/PixelTrackHeterogeneous.jl:10-62), stride 32768, or the context's
   * tuples_per_event when larger (extended capacity); the same stride for the ZVertexSoA's
   * per-track arrays (idv, ndof) */
  PXL_P_HIT_INDICES_OFF = 50,  /* uint32[32769], 1-based starts as bulk_fill stores them */
  PXL_P_HIT_INDICES = 51,      /* uint16[n_tuple_hits], 1-based hit ids (PXL_ERR_CAPACITY above 65535 hits) */
  PXL_P_HIT_INDICES32 = 67,    /* uint32[n_tuple_hits], 1-based hit ids (any hit count) */
  PXL_P_DET_INDICES = 52,      /* uint16[n_tuple_hits] */
  PXL_P_QUALITY = 53,          /* uint8[32768]: 0 bad, 1 dup, 2 loose */
  PXL_P_CHI2 = 54, PXL_P_ETA = 55, PXL_P_PT = 56, /* float[32768] */
  PXL_P_STATE = 57,            /* float[32768*5], row per track */
  PXL_P_COVARIANCE = 58,       /* float[32768*15], row per track */
  PXL_P_FITTED = 59,           /* uint8[32768]: 1 where the broken-line fit wrote the track */
  /* ZVertexSoA (CUDADataFormats/z_vertex_soa.jl:4-26) */
  PXL_P_IDV = 60,              /* int16[32768] */
  PXL_P_ZV = 61, PXL_P_WV = 62, PXL_P_VCHI2 = 63, PXL_P_PTV2 = 64, /* float[1024] */
  PXL_P_NDOF = 65,             /* int32[32768] */
  PXL_P_SORT_IND = 66,         /* uint16[1024] */
  PXL_P_ERRORS = 70            /* uint32[4*n_errors]: rawId, word, errorType, fedId */
};

/* Returns PXL_ABI_VERSION. */
int32_t pxl_version(void);

/* Fills the reference's parameters and default batch sizes. */
int32_t pxl_params_default(PxlParams* params);

/* The defaults with the extended per-event capacities: 262144 hits, 4194304 doublets,
 * 262144 tuples and fits per multiplicity, 4194304 list columns. High-pileup events
 * (pileup 200 gives about 31K hits, 0.8M doublets and 70K tuples) then run whole where the
 * reference's capacities (ca_hit_ntuplet_generator.jl:40, PixelTrackHeterogeneous.jl:55,
 * gpu_clustering_constants.jl:14) truncate them. Hit ids are 32-bit throughout. Batch sizes
 * (max_*) stay the caller's to set. No counterpart in the reference. */
int32_t pxl_params_extended(PxlParams* params);

/* Uploads the conditions and allocates every device buffer of a batch.
 * Replaces the ES producers' produce() and the producers' constructors.
 * Testing aid: the environment variable PXL_TUPLE_POOL_PART, when set at this call, sets the
 * records per part of the tuple record pool (normally sized from max_tuples); a pool too small
 * for a batch makes the tuple fill walk the trees again, with the same products. */
int32_t pxl_ctx_create(const PxlConditions* conditions, const PxlParams* params, PxlCtx** ctx);
int32_t pxl_ctx_destroy(PxlCtx* ctx);

/* Plain per-event API: one raw event (bin/ReadRAW.jl:23-31 layout: int32 nFeds, then
 * per FED int32 fedId, int32 size, size bytes) from host memory, run through the stages
 * in stage_mask with one launch sequence. Replaces the five producers' produce()
 * (SiPixelRawToClusterCUDA.jl:54-148, SiPixelRecHitCUDA.jl:25-42, ca_hit_ntuplet.jl:10-16,
 * pixel_vertex_producer_cuda.jl:24-28). stream: a cudaStream_t or NULL for the ctx stream.
 * Returns after the work is enqueued; pxl_sync waits and returns the warnings. */
int32_t pxl_event_run(PxlCtx* ctx, const uint8_t* raw_event, size_t nbytes, uint32_t stage_mask, void* stream);

/* Runs further stages (no PXL_STAGE_DIGIS bit) on the event or batch already on the
 * device, so each producer of the chain can run its own stage in turn: stage_mask =
 * PXL_STAGE_HITS for SiPixelRecHitCUDA, PXL_STAGE_TUPLES|PXL_STAGE_FIT|PXL_STAGE_CLASSIFY
 * for CAHitNtupletCUDA (ca_hit_ntuplet_generator.jl:65-97), PXL_STAGE_VERTICES for
 * PixelVertexProducerCUDA. Returns PXL_ERR_STATE when a needed stage has not run. */
int32_t pxl_event_continue(PxlCtx* ctx, uint32_t stage_mask, void* stream);

/* Batched API: n_events raw events back to back in `blob`, event e at
 * [event_offsets[e], event_offsets[e+1]). blob/event_offsets are host pointers
 * (input_on_device = 0) or device pointers (1). All events go through each stage in
 * one launch per kernel over a prefix-offset packed layout. */
int32_t pxl_batch_run(PxlCtx* ctx, const uint8_t* blob, const uint64_t* event_offsets, int32_t n_events,
                      int32_t input_on_device, uint32_t stage_mask, void* stream);

/* Stages a batch into the context's device input buffer (host -> device copies on the
 * stream), for pxl_graph_launch. */
int32_t pxl_batch_stage(PxlCtx* ctx, const uint8_t* blob, const uint64_t* event_offsets, int32_t n_events,
                        void* stream);

/* Captures the whole chain for the staged batch shape into one CUDA graph per input slot
 * (no host synchronisation inside), and replays slot 0's graph. Slot 0 is the input that
 * pxl_batch_stage / pxl_batch_run staged; when that is the context's own buffer, a graph is
 * also captured for every other slot. */
int32_t pxl_graph_capture(PxlCtx* ctx, uint32_t stage_mask);
int32_t pxl_graph_launch(PxlCtx* ctx, void* stream);

/* Double-buffered input for streaming batches. The context holds PXL_INPUT_SLOTS device
 * input buffers. pxl_slot_stage enqueues on copy_stream the host -> device copy of a batch
 * into `slot`, after the last chain that read that slot (blob must stay valid until the copy
 * ends: pinned memory for an asynchronous copy). pxl_slot_launch makes `stream` wait for that
 * copy and replays the slot's graph (pxl_graph_capture first; the staged event count must be
 * the captured one, else PXL_ERR_STATE). Staging batch i+1 into one slot while batch i runs
 * from the other overlaps the input copy with the chain. Products and results are those of
 * the last launch, as for pxl_graph_launch. */
#define PXL_INPUT_SLOTS 2
int32_t pxl_slot_stage(PxlCtx* ctx, int32_t slot, const uint8_t* blob, const uint64_t* event_offsets,
                       int32_t n_events, void* copy_stream);
int32_t pxl_slot_launch(PxlCtx* ctx, int32_t slot, void* stream);

/* Enqueues on `stream` the copy of the per-event vertex counts (nvFinal) of the last run into
 * host memory (pinned for an asynchronous copy), one uint32 per event; returns the count. */
int64_t pxl_results_async(PxlCtx* ctx, uint32_t* host_dst, int64_t max_events, void* stream);

/* Compacted track and vertex collections of the last run, for a consumer of a whole batch:
 * the tracks of quality loose (TrackSOA, CUDADataFormats/PixelTrackHeterogeneous.jl:10-62,
 * the ones the vertex finder takes) and the vertices (ZVertexSoA, z_vertex_soa.jl:4-26) of all
 * events, packed event after event (tracks in tuple order), each array copied to host memory
 * in ONE device->host copy. The compaction kernels go on `stream` (ordered after the context's
 * last run), the copies on `copy_stream` (NULL: the same stream); nothing synchronises the
 * host. Two device export sets alternate, so the copies of one batch overlap the next chain;
 * the host arrays must stay untouched until copy_stream reaches the copies (pinned memory for
 * a truly asynchronous copy). The first call allocates the export sets (about 100 bytes per
 * tuple of the batch capacity, twice). Every pointer may be NULL (not copied). A batch with
 * more tracks (vertices) than max_tracks (max_vertices) copies only the first ones; index row
 * n_events holds the totals, so the caller can tell. No counterpart in the reference, which
 * hands one event at a time to its consumers. */
typedef struct PxlExport {
  int64_t max_tracks;    /* capacity of the per-track host arrays */
  int64_t max_vertices;  /* capacity of the per-vertex host arrays */
  uint32_t* index;       /* [n_events + 1][4]: first track, tracks, first vertex, vertices; last row: totals */
  float* state;          /* [max_tracks][5]: phi, tip, q/pT, cot(theta), zip (TrackSOA stateAtBS) */
  float* cov;            /* [max_tracks][15] */
  float* pt;             /* [max_tracks] */
  float* eta;            /* [max_tracks] */
  float* chi2;           /* [max_tracks] */
  uint8_t* n_hits;       /* [max_tracks] hits of the track's tuple */
  int16_t* vertex;       /* [max_tracks] the track's vertex as ZVertexSoA's idv holds it (-1: none) */
  uint32_t* tuple;       /* [max_tracks] the track's 1-based tuple slot in its event's TrackSOA */
  float* zv;             /* [max_vertices] */
  float* wv;             /* [max_vertices] */
  float* vchi2;          /* [max_vertices] */
  float* ptv2;           /* [max_vertices] */
  int32_t* ndof;         /* [max_vertices] */
} PxlExport;
int32_t pxl_export_async(PxlCtx* ctx, const PxlExport* out, void* stream, void* copy_stream);
/* Bytes that pxl_export_async copies for `out` and a batch of n_events. */
int64_t pxl_export_bytes(const PxlExport* out, int32_t n_events);

/* CountValidator (plugin-Validation/count_to_validator.jl:18-84) on the device, over every
 * event of the last run. expected[5 * n_events]: per event n_modules, n_digis, n_clusters
 * (digicluster.bin), n_tracks (tracks.bin) and n_vertices (vertices.bin), the count files
 * bin/ReadRAW.jl:47-59 reads. An event is good when its modules, digis and clusters are equal,
 * its N(track) (tuples with hits, the TrackSOA loop of :50-55) is within a relative 0.012 and its
 * vertex count is equal. status[n_events] (may be NULL) receives per event the failed checks (bit 0
 * modules, 1 digis, 2 clusters, 3 tracks, 4 vertices) | N(track) << 8. Returns the number of good
 * events, or < 0; synchronises. n_events must be the last run's event count. */
int32_t pxl_validate_counts(PxlCtx* ctx, const uint32_t* expected, int32_t n_events, uint32_t* status);

/* Number of kernel nodes in the captured graph (the kernels one replay launches). */
int32_t pxl_graph_kernel_nodes(PxlCtx* ctx);

/* Per-kernel timing of non-graph runs: when enabled, a CUDA event is recorded after
 * each kernel group; pxl_profile_read returns the milliseconds of each segment of the last
 * run and its name (static strings), at most max entries. */
int32_t pxl_profile_enable(PxlCtx* ctx, int32_t on);
int32_t pxl_profile_read(PxlCtx* ctx, float* ms, const char** names, int32_t max);

/* Launch-shape autotuner. Runs the whole chain on the batch staged last (pxl_batch_stage or
 * pxl_batch_run) once per candidate shape (each shape warmed up once, then timed reps times
 * with per-stage CUDA events) and keeps, for each tunable stage (doublets, hit lists, connect,
 * cell lists, fishbone, ntuplets, cell tracks, early duplicates, classification, hit-to-tuple,
 * fits), the fastest. A candidate c > 0 (at most 4096) is a static grid of c blocks per event;
 * c < 0 (at least -64) a persistent work queue: the doublet, connect, fishbone and ntuplet
 * stages run as one wave of CTAs that pull virtual blocks of -c loop strides, events with the
 * most hits first (the other stages run their default grid for it). The choice holds for later
 * runs and graph captures of this context. chosen[PXL_TUNE_STAGES] (may be NULL) receives it.
 * Products of the staged batch are recomputed. No counterpart in the reference, whose
 * serial loops have no launch shape. */
#define PXL_TUNE_STAGES 11
int32_t pxl_autotune(PxlCtx* ctx, const int32_t* candidates, int32_t n_candidates, int32_t reps, int32_t* chosen);

/* Waits for the context's work; returns 0, the OR of the events' PXL_WARN_* bits, or < 0. */
int32_t pxl_sync(PxlCtx* ctx);

/* Reads the counts of event `event` of the last run (synchronises). */
int32_t pxl_event_counts(PxlCtx* ctx, int32_t event, PxlEventCounts* counts);

/* Copies product `product` (enum PxlProduct) of event `event` in the reference's layout to
 * host memory (at most max_bytes). Returns the element count, or < 0. */
int64_t pxl_copy_product(PxlCtx* ctx, int32_t event, int32_t product, void* host_dst, int64_t max_bytes);

/* Clustering on digis alone: count_modules, find_clus and (apply_charge_cut != 0)
 * cluster_charge_cut on one module-ordered digi stream, as test/gpu_clustering_t.jl:245-280
 * drives gpu_clustering.jl:52-266 and gpu_cluster_charge_cut.jl:14-104. Host arrays of
 * length n; module_start[2001], clus_in_module[2000], module_id[2000] outputs. */
int32_t pxl_clusterize_digis(PxlCtx* ctx, const uint16_t* id, const int16_t* x, const int16_t* y, const int32_t* adc,
                             int32_t n, int32_t apply_charge_cut, uint32_t* module_start, uint32_t* clus_in_module,
                             uint32_t* module_id, int32_t* clus, uint16_t* id_out);

/* Same clustering as pxl_clusterize_digis, on DEVICE arrays, for callers that cannot
 * allocate device memory (an event loop whose device memory belongs to another allocator,
 * or a path that must not block on cudaMalloc/cudaFree). It allocates nothing: inputs
 * (id, x, y, adc; n digis) and outputs (module_start[2001], clus_in_module[2000],
 * module_id[2000], clus[n], id_out[n]) are the caller's device buffers, and the scratch
 * is a fixed file-scope device array of the library (about 90 KB on every GPU that loads
 * it, held until exit). At most 1,048,576 digis per call; larger n returns
 * PXL_ERR_CAPACITY. The first call on a device looks the array up on that device, so make
 * it before any stream capture. Calls share the array: calls that overlap on the GPU race.
 * Enqueued on `stream` (a cudaStream_t of the current device, or NULL; a stream of another
 * device returns PXL_ERR_ARG); the caller synchronises. Capacity warnings are not returned
 * (the status is 0 or an error): module_start[0] == 2000 means the module list overflowed.
 * No counterpart in the reference: it adds an allocation-free form of the clustering. */
int32_t pxl_clusterize_digis_noalloc(const uint16_t* id, const int16_t* x, const int16_t* y, const int32_t* adc,
                                     int32_t n, int32_t apply_charge_cut, uint32_t* module_start,
                                     uint32_t* clus_in_module, uint32_t* module_id, int32_t* clus, uint16_t* id_out,
                                     void* stream);

/* Standalone broken-line fits of n_tracks tracks (broken_line.jl:275-696, driven as
 * broken_line_fit_on_gpu.jl:24-163 does). Device pointers: hits[3*H] (x,y,z per hit,
 * float64), hits_ge[6*H] (global covariance per hit, float32), hit_offsets[n_tracks+1]
 * (3..8 hits per track, any order). precision: 0 = FP64 throughout, 1 = FP32 arithmetic
 * with the band-matrix LDL^T solve, the parameter transport and the covariance in FP64.
 * workspace: device scratch of at least pxl_fit_workspace_bytes(n_tracks) bytes, used
 * to group the tracks by hit count (contents need not be initialised).
 * Outputs (device): state[5*n] (phi, tip, q/pt, cot(theta), zip as copyFromCircle! stores
 * them), cov[15*n], chi2[n], pt[n], eta[n], status[n] (0 ok, 1 domain, -1 bad hit count). */
int64_t pxl_fit_workspace_bytes(int32_t n_tracks);
int32_t pxl_bl_fit(const double* hits, const float* hits_ge, const int32_t* hit_offsets, int32_t n_tracks, double b_field,
                   int32_t precision, float* state, float* cov, float* chi2, float* pt, float* eta, int32_t* status,
                   void* workspace, int64_t workspace_bytes, void* stream);

/* Stand-alone Riemann helix fits (plugin-PixelTriplets/riemann_fit.jl: fast_fit, the
 * Riemann-Chernov circle_fit with multiple scattering, line_fit in the rotated s-z plane),
 * parameters and chi2 (no covariance propagation). Same track inputs and workspace as
 * pxl_bl_fit; precision 0 = FP64, 1 = FP32 per-hit geometry and covariance models with
 * FP64 Cholesky inverses, scatter matrix, 3x3 eigenproblem and final parameters.
 * Outputs (device): state[5*n] (phi, d0, q/pT, cot(theta), zip), chi2[2*n] (circle, line),
 * pt[n], status[n] (0 ok, 1 non-finite result, -1 bad hit count). */
int32_t pxl_riemann_fit(const double* hits, const float* hits_ge, const int32_t* hit_offsets, int32_t n_tracks,
                        double b_field, int32_t precision, float* state, float* chi2, float* pt, int32_t* status,
                        void* workspace, int64_t workspace_bytes, void* stream);

/* Adjoint of the broken-line fit: per track the FP64 chi2 = chi2_line + chi2_circle and
 * its gradient with respect to the hit coordinates, the fit being recomputed in the
 * backward pass (nothing stored between passes). Same track inputs as pxl_bl_fit.
 * Alignment (optional, all of hit_module[H], module_pos[3*n_modules] (module centres,
 * FP64) and n_modules > 0): when align[6*n_modules] (tx, ty, tz, wx, wy, wz per module;
 * float) is given, each hit h on module m (hit_module >= 0) is first moved to
 * h + t_m + w_m x (h - c_m). Outputs (device, each may be NULL): chi2[n] (float),
 * grad_hits[3*H] (float, gradient w.r.t. the moved hits), grad_align[6*n_modules]
 * (float) and grad_align64[6*n_modules] (FP64) = d(sum chi2)/d(alignment), accumulated
 * in FP64. workspace: pxl_adjoint_workspace_bytes(n_tracks, n_modules) bytes.
 * The reference has no gradient path: this extends the fit of broken_line.jl. */
int64_t pxl_adjoint_workspace_bytes(int32_t n_tracks, int32_t n_modules);
int32_t pxl_bl_fit_adjoint(const double* hits, const float* hits_ge, const int32_t* hit_offsets, int32_t n_tracks,
                           double b_field, const int16_t* hit_module, const double* module_pos, const float* align,
                           int32_t n_modules, float* chi2, float* grad_hits, float* grad_align, double* grad_align64,
                           void* workspace, int64_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PXL_H */
