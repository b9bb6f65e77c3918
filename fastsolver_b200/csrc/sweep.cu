// sweep.cu -- the tree levels of a refinement sweep in one persistent kernel.
//
// A sweep applies the FP32 factors to m right-hand-side columns: after the
// leaf solves, every level from the deepest up runs the reduce V_c^T d_c
// (split-K partial slots), the fixed-order slot sums, the node apply
// [eta0; eta1] = M [W0; W1] and the broadcast d_c -= u_c eta_c (the per-node
// unit of fast_solver.cc:203-254).  Each step moves only tens of MB, so one
// launch per step (four per level) spends most of its time ramping up and
// draining.  sweep_levels_kernel runs all of them: one cooperative launch of
// as many 128-thread CTAs as fit on the GPU, every CTA taking work units of a
// step by grid stride (a 64 x 16 block of a reduce item, 32 elements of a
// slot sum, 128 rows of an apply or broadcast item -- the same CTA units as
// the one-step kernels, skinny_units.cuh), and a grid barrier between steps.
//
// The grid barrier is a counter in global memory: each CTA adds one, and the
// CTA whose arrival completes the barrier publishes it in a release word that
// the others poll with backoff.  Every wait is bounded
// (g_sweep_spin_limit polls with a sleep); on timeout the CTA raises
// g_sweep_error and an abort flag, and every CTA leaves at its next barrier,
// so the kernel always ends.  The host reports the flag as
// HODLR_ERR_TIMEOUT.  The launch is cooperative, so all CTAs are resident.
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>

#include "common.cuh"
#include "skinny_units.cuh"
#include "sweep.cuh"

namespace hodlr {

__device__ int g_sweep_error = 0;
// test hooks (hodlr_debug_sweep_barrier_hook): the bound of a barrier wait,
// and a one-shot request that CTA 0 of the next sweep kernel leave before
// its first arrival, so that every other CTA's wait runs out
__device__ long long g_sweep_spin_limit = 1LL << 22;
__device__ int g_sweep_skip_arrival = 0;

namespace {

using namespace sk;
constexpr int kThreads = 128;
constexpr long long kSweepSpinDefault = 1LL << 22;
constexpr int kSweepWarpSlots = 32;  // slot counts summed by one warp per unit

// Grid barrier; false when the kernel is being abandoned (a wait ran out).
// bar[0] counts arrivals; the CTA whose arrival completes barrier k publishes
// k + 1 in bar[32] (its own 128-byte line, so the waiting CTAs poll a line
// that no atomic touches) and bar[64] is the abort flag.  Waiters back off
// exponentially up to ~1 us between polls, which keeps hundreds of polling
// CTAs from saturating the L2 slice that holds the flag.
__device__ bool grid_sync(unsigned *bar, unsigned &gen, long long limit) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned *release = bar + 32;
    volatile unsigned *abort = bar + 64;
    ++gen;
    __threadfence();  // this CTA's results before its arrival
    const unsigned old = atomicAdd(bar, 1u);
    int ok = 1;
    if (old == gen * gridDim.x - 1) {
      __threadfence();
      *release = gen;  // the last arrival opens the barrier
    } else {
      unsigned sleep = 32;
      for (long long it = 0;; ++it) {
        if (*release >= gen) break;
        if (*abort) { ok = 0; break; }
        if (it >= limit) {
          atomicExch(bar + 64, 1u);
          atomicExch(&g_sweep_error, 1);
          ok = 0;
          break;
        }
        __nanosleep(sleep);
        if (sleep < 1024) sleep <<= 1;
      }
    }
    __threadfence();  // the other CTAs' results after the barrier
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// 3 CTAs (12 warps) per SM: the units keep a chunk of A, their share of B
// and a row's Cin values in registers (up to 168 per thread); measured at
// N = 262144 (m = 16) the same sweep time as 4 CTAs per SM, where the
// 128-register bound makes them spill
template <int NC>
__global__ void __launch_bounds__(kThreads, 3)
    sweep_levels_kernel(const SweepLevel *__restrict__ levels, int nlevels, unsigned *bar) {
  extern __shared__ __align__(16) unsigned char smem[];
  const long long limit = g_sweep_spin_limit > 0 ? g_sweep_spin_limit : kSweepSpinDefault;
  if (blockIdx.x == 0) {
    __shared__ int s_skip;
    if (threadIdx.x == 0) s_skip = atomicExch(&g_sweep_skip_arrival, 0);
    __syncthreads();
    if (s_skip) return;  // test hook: this CTA never arrives
  }
  unsigned gen = 0;
  const int tid = threadIdx.x;
  for (int l = 0; l < nlevels; ++l) {
    const SweepLevel L = levels[l];
    // reduce: partial slots of V_c^T d_c
    {
      const int per = L.red_mt * L.red_nt;
      const int nu = L.n_red * per;
      for (int u = blockIdx.x; u < nu; u += gridDim.x) {
        const int item = u / per, rem = u - item * per;
        tn2_unit<float, true>(L.red_items, L.red_segs, 1.f, 0.f, item, rem / L.red_nt,
                              rem % L.red_nt, smem);
      }
    }
    if (!grid_sync(bar, gen, limit)) return;
    // slot sums in a fixed order (the REDOP_ADD of gemm.cc:74-133,
    // deterministic); a unit is 32 elements of one task.  Levels whose tasks
    // have at most kSweepWarpSlots slots (the deepest ones: thousands of
    // small tasks): every warp takes a unit of its own and adds its slots in
    // order, with no barrier.  Otherwise warp w of the CTA adds slots w,
    // w + 4, ... of a unit, then warp 0 adds the four partial sums in order.
    {
      const int lane = tid & 31, w = tid >> 5;
      const int nu = L.n_sums * L.sum_units;
      if (L.sum_max_slots <= kSweepWarpSlots) {
        constexpr int kWarps = kThreads / 32;
        for (int u = blockIdx.x * kWarps + w; u < nu; u += gridDim.x * kWarps) {
          const SumTask<float> tk = L.sums[u / L.sum_units];
          const long long e = (long long)(u % L.sum_units) * kSweepSumChunk + lane;
          if (e < tk.len) {
            double acc = 0.0;
#pragma unroll 4
            for (int q = 0; q < tk.nslots; ++q) acc += double(__ldcg(tk.src + e + (long long)q * tk.stride));
            tk.dst[e] = float(acc);
          }
        }
      } else {
        double *part = reinterpret_cast<double *>(smem);  // [4][32]
        for (int u = blockIdx.x; u < nu; u += gridDim.x) {
          const SumTask<float> tk = L.sums[u / L.sum_units];
          const long long e = (long long)(u % L.sum_units) * kSweepSumChunk + lane;
          double acc = 0.0;
          if (e < tk.len) {
#pragma unroll 8
            for (int q = w; q < tk.nslots; q += kThreads / 32)
              acc += double(__ldcg(tk.src + e + (long long)q * tk.stride));
          }
          part[w * 32 + lane] = acc;
          __syncthreads();
          if (w == 0 && e < tk.len)
            tk.dst[e] = float(((part[lane] + part[32 + lane]) + part[64 + lane]) + part[96 + lane]);
          __syncthreads();
        }
      }
    }
    if (!grid_sync(bar, gen, limit)) return;
    // node apply [eta0; eta1] = M [W0; W1]
    {
      float *Bs = reinterpret_cast<float *>(smem);
      const int nu = L.n_ap * L.ap_rb;
      for (int u = blockIdx.x; u < nu; u += gridDim.x)
        nn_rows_unit<NC, true>(L.ap_items, L.ap_segs, 1.f, 0.f, u / L.ap_rb, u % L.ap_rb, Bs);
    }
    if (!grid_sync(bar, gen, limit)) return;
    // broadcast d_c -= u_c eta_c
    {
      float *Bs = reinterpret_cast<float *>(smem);
      const int nu = L.n_bc * L.bc_rb;
      for (int u = blockIdx.x; u < nu; u += gridDim.x)
        nn_rows_unit<NC, true>(L.bc_items, L.bc_segs, -1.f, 1.f, u / L.bc_rb, u % L.bc_rb, Bs);
    }
    if (l + 1 < nlevels && !grid_sync(bar, gen, limit)) return;
  }
}

size_t sweep_smem() {
  const size_t rows_b = std::max({nn_rows_kc<8>() * 8, nn_rows_kc<16>() * 16, nn_rows_kc<32>() * 32}) *
                       sizeof(float);
  return std::max(tn2_smem_bytes<float>(), rows_b);
}

template <int NC>
void launch_nc(const SweepLevel *levels, int nlevels, unsigned *bar, cudaStream_t s) {
  const size_t smem = sweep_smem();
  auto kern = sweep_levels_kernel<NC>;
  raise_smem_limit(reinterpret_cast<const void *>(kern), smem);
  // co-resident CTAs (cached per device: the occupancy query is not a stream
  // operation, but keep it out of captured regions after the first call)
  static std::mutex mu;
  static std::map<int, int> grid_of;
  int dev = 0;
  HODLR_CUDA_TRY(cudaGetDevice(&dev));
  int grid = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto f = grid_of.find(dev);
    if (f == grid_of.end()) {
      int per_sm = 0, sms = 0;
      HODLR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem));
      HODLR_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      grid = std::max(1, per_sm) * sms;
      grid_of[dev] = grid;
    } else {
      grid = f->second;
    }
  }
  HODLR_CUDA_TRY(cudaMemsetAsync(bar, 0, kSweepBarWords * sizeof(unsigned), s));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  HODLR_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, levels, nlevels, bar));
  HODLR_LAUNCH_CHECK();
}

}  // namespace

bool sweep_persistent_enabled() {
  static const bool on = [] {
    const char *e = std::getenv("HODLR_PERSISTENT_SWEEP");
    return !(e && e[0] == '0');
  }();
  return on;
}

void launch_sweep_levels(const SweepLevel *levels, int nlevels, int max_n, unsigned *bar,
                         cudaStream_t s) {
  if (nlevels <= 0) return;
  if (max_n <= 8) launch_nc<8>(levels, nlevels, bar, s);
  else if (max_n <= 16) launch_nc<16>(levels, nlevels, bar, s);
  else launch_nc<32>(levels, nlevels, bar, s);
}

int sweep_error_flag(bool reset) {
  int h = 0;
  if (cudaMemcpyFromSymbol(&h, g_sweep_error, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  if (reset && h) {
    int z = 0;
    cudaMemcpyToSymbol(g_sweep_error, &z, sizeof(int));
  }
  return h;
}

void sweep_set_wait_hook(long long polls, int skip_one_arrival) {
  const long long lim = polls > 0 ? polls : kSweepSpinDefault;
  const int skip = skip_one_arrival ? 1 : 0;
  HODLR_CUDA_TRY(cudaMemcpyToSymbol(g_sweep_spin_limit, &lim, sizeof(lim)));
  HODLR_CUDA_TRY(cudaMemcpyToSymbol(g_sweep_skip_arrival, &skip, sizeof(skip)));
}

}  // namespace hodlr
