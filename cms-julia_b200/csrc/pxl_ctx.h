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
  pxl::Dev d{};
  std::vector<void*> allocs;
  int16_t* fed_slot_of = nullptr;
  // host copy of the conditions needed at copy-out
  std::vector<float> avg_geom;
  // graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  uint32_t graph_mask = 0;
  int graph_E = -1;
  // last run
  int32_t last_E = 0;
  uint32_t last_mask = 0;
  uint32_t done_mask = 0;
  std::vector<pxl::EvInfo> ev_host;
  bool ev_host_valid = false;
  // pinned staging for offsets
  uint64_t* h_off = nullptr;
  size_t raw_cap = 0;
  uint64_t* d_ev_off = nullptr;
  uint8_t* d_raw = nullptr;
  // per-kernel timing of non-graph runs
  pxl::Prof prof;
  bool capturing = false;
  // blocks per event of the tunable stages (0 = the default shape), set by pxl_autotune
  int tune[pxl::kTuneCount] = {};
};

// reads the events' counters back (synchronises the context stream)
int pxl_fetch_ev(PxlCtx* ctx);
