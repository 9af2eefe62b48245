// Host-side context object behind the PxlCtx handle of include/pxl.h.
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/pxl.h"
#include "pxl_internal.cuh"

struct PxlCtx {
  PxlParams p{};
  int device = 0;
  cudaStream_t stream = nullptr;
  // recorded after the last work this context enqueued, on whichever stream it went: the
  // context's reads (sync, counts, copy-out) order themselves after it and wait for nothing else
  cudaEvent_t last_done = nullptr;
  pxl::Dev d{};
  std::vector<void*> allocs;
  int16_t* fed_slot_of = nullptr;
  // host copy of the conditions needed at copy-out
  std::vector<float> avg_geom;
  // input slots: each has its own device raw buffer, offsets and captured graph, so the
  // copy of one batch overlaps the chain running on the other
  static constexpr int kSlots = PXL_INPUT_SLOTS;
  cudaGraph_t graph[kSlots] = {};
  cudaGraphExec_t graph_exec[kSlots] = {};
  uint32_t graph_mask = 0;
  int graph_E = -1;
  // last run
  int32_t last_E = 0;
  uint32_t last_mask = 0;
  uint32_t done_mask = 0;
  std::vector<pxl::EvInfo> ev_host;
  bool ev_host_valid = false;
  // per slot: pinned staging of the rebased offsets, device input, events staged in it,
  // an event after its copies and one after the last chain that read it
  uint64_t* h_off[kSlots] = {};
  size_t raw_cap = 0;
  uint64_t* d_ev_off[kSlots] = {};
  uint8_t* d_raw[kSlots] = {};
  int32_t slot_E[kSlots] = {};
  cudaEvent_t ev_staged[kSlots] = {};
  cudaEvent_t ev_consumed[kSlots] = {};
  // per-kernel timing of non-graph runs
  pxl::Prof prof;
  bool capturing = false;
  // blocks per event of the tunable stages (0 = the default shape), set by pxl_autotune
  int tune[pxl::kTuneCount] = {};
  // CTAs of one persistent work-queue wave per stage (0: the stage has no work-queue form)
  int wq_ctas[pxl::kTuneCount] = {};
  // pxl_export_async: two alternating device export sets (allocated by the first call)
  pxl::ExportSet exp[2];
  int exp_next = 0;
  // pxl_validate_counts: expected counts and per-event status (allocated by the first call)
  uint32_t* val_expected = nullptr;
  uint32_t* val_status = nullptr;
};

// reads the events' counters back (synchronises the context stream)
int pxl_fetch_ev(PxlCtx* ctx);
