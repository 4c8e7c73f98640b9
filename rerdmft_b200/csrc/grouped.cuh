// Grouped execution for batches of uneven problems (the geometry scan): one persistent launch runs
// the tiles of many independent FP64 GEMMs of different shapes, and a small autotuner picks each
// shape's tile configuration and split-K count by measured throughput, with a persisted cache.
#pragma once

#include <string>
#include <vector>

#include "gemm_f64.cuh"

namespace rr {

// Tile configuration of the grouped DMMA GEMM (an index into the configuration table of
// gemm_grouped.cu) and the split-K count, chosen per problem shape.
struct GemmChoice {
  int cfg = 0;
  int splits = 1;
};

// Small per-launch tables (problem descriptors, tile offsets) staged through a pinned host buffer
// into a linear device buffer.  Space is handed out in order and recycled by reset(), which the
// owner calls only after the stream has passed every launch that read earlier tables (a full wait);
// when the buffer runs out, put() continues in a larger one and keeps the full one until reset().
// Side streams of a caller's grouped launches: tile launches of different configurations run beside
// each other, joined before the reductions (created on first use, on the device current then).
struct SideStreams {
  static constexpr int kCount = 4;
  cudaStream_t st[kCount] = {};
  cudaEvent_t fork = nullptr, done[kCount] = {};
  SideStreams() = default;
  SideStreams(const SideStreams&) = delete;
  SideStreams& operator=(const SideStreams&) = delete;
  ~SideStreams();
  void make();
};

struct TableRing {
  DevBuf<char> dev;
  char* host = nullptr;
  size_t cap = 0, used = 0;
  SideStreams side;  // the grouped launches that take their tables from this ring run their tiles here
  // buffers that filled up since the last reset(): kept until then, since tables in them may still
  // be read by queued launches
  std::vector<std::pair<DevBuf<char>, char*>> retired;
  TableRing() = default;
  TableRing(const TableRing&) = delete;
  TableRing& operator=(const TableRing&) = delete;
  ~TableRing();
  void reserve(size_t bytes);
  void reset();
  // Copies `bytes` from src into the table space (asynchronously, ordered on s); returns the device
  // address (16-byte aligned), valid until the next reset().
  const void* put(const void* src, size_t bytes, cudaStream_t s);
};

// Every product of `descs` in as few launches as the chosen tile configurations allow (one
// persistent launch per configuration present, problems of one configuration sharing it tile by
// tile), then one fixed-order split-K reduction and one mirror launch per element kind that needs
// them.  Each problem's choice comes from autotune_choice, so its result does not depend on which
// other problems share the launch.  work: split-K scratch (grown after a full wait of s when short).
// launches (optional) is incremented by the number of kernels launched.
void gemm_grouped(const std::vector<GemmDesc>& descs, cudaStream_t s, TableRing& ring, DevBuf<double>& work,
                  int64_t* launches);

// A built grouped launch sequence: its tables live in the TableRing it was built with and its split-K
// scratch in `work`, so it may be executed again (on the same stream) until the ring's next reset() or
// the next growth of that scratch.  For loops that repeat the same products (SP2 steps).
struct GroupedLaunch {
  int kind;  // 0 GEMM tiles, 1 split-K reduction, 2 mirror
  int cfg, pl;
  bool cplx, AK, BKM, vec2;
  const void* probs;
  const int64_t* off;
  int n;
  int64_t total;
  int blocks;
};
struct GroupedPlan {
  std::vector<GroupedLaunch> launches;
  SideStreams* side = nullptr;  // of the ring the plan was built with
};
void gemm_grouped_plan(const std::vector<GemmDesc>& descs, cudaStream_t s, TableRing& ring, DevBuf<double>& work,
                       GroupedPlan& plan);
void gemm_grouped_exec(const GroupedPlan& plan, cudaStream_t s, int64_t* launches);

// The tuned choice for this problem shape: looked up in the cache, else measured on the spot (each
// candidate configuration and split count timed as a grouped launch of enough copies of the problem
// to fill the GPU, CUDA events, the fastest per problem kept).  The first call loads the file named by
// RR_AUTOTUNE_CACHE when that variable is set.
GemmChoice autotune_choice(const GemmDesc& d);
// The same for every problem of descs (one lock for all; empty problems get the default).
void autotune_choices(const std::vector<GemmDesc>& descs, std::vector<GemmChoice>& out);
// Cache file: one line per shape, "<key> <cfg> <splits> <microseconds per problem>".
void autotune_load(const std::string& path);
void autotune_save(const std::string& path);
// Saves to RR_AUTOTUNE_CACHE when it is set and entries were added since the last save.
void autotune_flush();
void autotune_clear();
int64_t autotune_entries();
// Totals over the process: seconds spent timing candidates and kernels they launched.
void autotune_totals(double* seconds, int64_t* launches);

}  // namespace rr
