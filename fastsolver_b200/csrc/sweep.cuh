// sweep.cuh -- persistent level walk of a refinement sweep (sweep.cu).
#pragma once
#include "common.cuh"
#include "util.cuh"

namespace hodlr {

// One tree level of an FP32 apply path: its reduce, slot-sum, node-apply and
// broadcast work, with the unit counts of each step (device array, one
// entry per level, deepest first).
struct SweepLevel {
  const GemmItem<float, float> *red_items;
  const GemmSeg<float> *red_segs;
  const SumTask<float> *sums;
  const GemmItem<float, float> *ap_items;
  const GemmSeg<float> *ap_segs;
  const GemmItem<float, float> *bc_items;
  const GemmSeg<float> *bc_segs;
  int n_red, red_mt, red_nt;  // items, 64-row and 16-column blocks per item
  int n_sums, sum_units;      // tasks, kSweepSumChunk-element chunks per task
  int sum_max_slots;          // most partial slots of one task
  int n_ap, ap_rb;            // items, 128-row blocks per item
  int n_bc, bc_rb;
};

// Slot-sum elements per work unit of the persistent kernel.
constexpr int kSweepSumChunk = 32;
// Words of the grid barrier: arrival counter, release word and abort flag,
// each on its own 128-byte line.
constexpr int kSweepBarWords = 96;

// True unless the environment sets HODLR_PERSISTENT_SWEEP=0 (one launch per
// step instead).
bool sweep_persistent_enabled();

// All levels in one cooperative launch; max_n bounds the apply / broadcast
// items' column count (<= 32); bar: kSweepBarWords unsigned words of device
// memory (the grid barrier, cleared by the launch).
void launch_sweep_levels(const SweepLevel *levels, int nlevels, int max_n, unsigned *bar,
                         cudaStream_t s);

// The device flag raised by a grid-barrier wait that ran out (1), 0, or -1.
int sweep_error_flag(bool reset);

// Test hook of the timeout path: barrier waits give up after `polls` tries
// (<= 0: the default, 2^22), and with skip_one_arrival CTA 0 of the next
// sweep launch leaves before its first arrival.  Synchronous.
void sweep_set_wait_hook(long long polls, int skip_one_arrival);

}  // namespace hodlr
