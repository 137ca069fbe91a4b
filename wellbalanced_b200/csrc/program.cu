// Op programs: the small-op phases between two stage kernels of a refined step — reflux,
// restriction and the halo fill of every level, and the stable time step — in ONE launch
// instead of one launch per level and op list (carafe/mhd.py:889-994: the patchwork halo
// exchanges, refluxes and restrictions of a step, and stable_step). The flux register's
// face fluxes (HLLD per interface face, ~160 registers a thread) keep their own launch, so
// that the program's blocks stay small and several per SM for the latency-bound copies.
//
// A program is a list of segments (an op list of one kind on one pool), grouped into
// phases that run in order; the segments of a phase run together (their ops touch
// disjoint points, as in the standalone launches). The work items of all segments — runs
// of consecutive ops, about two per block and phase, so that a block pays the hand-out
// cost once per run and not per op — are numbered in program order and handed out by one
// ticket counter: a block takes the next ticket, and before it runs an item of phase p it
// waits until every item of phase p - 1 has finished (a per-phase completion counter).
// The halo, interpolation and restriction ops of an item go to the block's four warps,
// one op per warp at a time (most of them are a few dozen points). Tickets go out in order, so a block only
// ever waits for items that running blocks hold: the launch needs no co-residency of its
// blocks (no cooperative launch, no grid barrier), and every wait is bounded (a second);
// a wait that runs out sets the program's error word, and the blocks skip their remaining
// items and return. The last block to leave resets the counters, so consecutive launches
// and graph replays need no host work between them.
//
// Each item runs the device body of the standalone kernel of its kind (ops.cuh,
// ratecell.cuh) on 128 threads, with the same arithmetic per point: a step through
// programs equals, bit for bit, the step through the standalone launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "halo.cuh"
#include "layout.cuh"
#include "ops.cuh"
#include "ratecell.cuh"
#include "stage.cuh"
#include "wb_internal.cuh"
#include "wellbalanced_b200.h"

namespace wb {

constexpr int kProgramThreads = 128;
constexpr int kProgramWarps = kProgramThreads / 32;
constexpr int kProgramMaxRun = 64;  // ops per item at most
// launch bounds: 128 registers a thread (the interpolation's unrolled weights)
constexpr int kProgramBlocksPerSM = 4;
constexpr unsigned long long kProgramWaitNs = 1000000000ull;  // a second

template <typename S>
struct ProgramArgs {
  S* pools[2];
  const PatchDesc* patches;
  unsigned* counters;  // [0] ticket, [1] blocks left, [2] error bits, [3 + p] items of phase p done
  int nsegments, nphases, total;
  wb_program_params p;
  int phase_total[WB_PROGRAM_MAX_SEGMENTS];
  wb_program_segment seg[WB_PROGRAM_MAX_SEGMENTS];
};

__device__ __forceinline__ unsigned load_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Thread 0 of a block: wait until *done reaches `target`, the error word is set, or a
// second passes (then the error word gets bit 2). Returns whether the phase completed.
__device__ bool wait_phase(const unsigned* done, unsigned target, unsigned* error) {
  if (load_acquire(done) >= target) return true;
  const unsigned long long start = global_ns();
  while (true) {
    __nanosleep(128);
    if (load_acquire(done) >= target) return true;
    if (load_acquire(error)) return false;
    if (global_ns() - start > kProgramWaitNs) {
      atomicOr(error, 2u);
      return false;
    }
  }
}

template <typename S>
__global__ void __launch_bounds__(kProgramThreads, kProgramBlocksPerSM)
    program_kernel(const __grid_constant__ ProgramArgs<S> a) {
  __shared__ int s_ticket, s_go;
  const int tid = threadIdx.x;
  unsigned* ticket = a.counters;
  unsigned* left = a.counters + 1;
  unsigned* error = a.counters + 2;
  unsigned* done = a.counters + 3;
  const wb_program_params& p = a.p;
  while (true) {
    if (tid == 0) s_ticket = int(atomicAdd(ticket, 1u));
    __syncthreads();
    const int t = s_ticket;
    if (t >= a.total) break;  // uniform over the block
    int k = 0;
    while (k + 1 < a.nsegments && a.seg[k + 1].first <= t) ++k;
    const wb_program_segment& sg = a.seg[k];
    const int item = t - sg.first;
    const int phase = sg.phase;
    const int run = sg.pad;  // ops per item
    const int op0 = item * run, op1 = min(sg.count, op0 + run);
    const int warp = tid / 32;
    if (tid == 0) {
      const bool go = phase == 0 || wait_phase(done + phase - 1, unsigned(a.phase_total[phase - 1]), error);
      s_go = go && !load_acquire(error);
    }
    __syncthreads();
    if (s_go) {
      S* pool = a.pools[sg.pool];
      switch (sg.kind) {
        case WB_SEG_COPY:
          for (int o = op0 + warp; o < op1; o += kProgramWarps)
            copy_op<S, 32>(pool, a.patches, static_cast<const CopyOp*>(sg.ops)[o]);
          break;
        case WB_SEG_INTERP:
          for (int o = op0 + warp; o < op1; o += kProgramWarps)
            interp_op<S, 32>(pool, a.patches, static_cast<const InterpOp*>(sg.ops)[o]);
          break;
        case WB_SEG_RESTRICT:
          for (int o = op0 + warp; o < op1; o += kProgramWarps)
            restrict_op<S, 32>(pool, a.patches, static_cast<const RestrictOp*>(sg.ops)[o]);
          break;
        case WB_SEG_REFLUX:
          // the ops of a reflux segment touch disjoint cells: the block's threads over each op
          for (int o = op0; o < op1; ++o)
            reflux_op<S, kProgramThreads>(pool, a.patches, static_cast<const RefluxOp*>(sg.ops)[o], p.reg, p.dt);
          break;
        case WB_SEG_INIT_KEYS:
          for (int i = tid; i < p.ninstances; i += kProgramThreads) {
            p.keys[2 * i] = double_to_key(0.0);
            p.keys[2 * i + 1] = rate_min_identity();
          }
          if (p.level_keys)
            for (int i = tid; i < p.ninstances * p.nlevels; i += kProgramThreads) p.level_keys[i] = rate_min_identity();
          break;
        case WB_SEG_RATE: {
          const RateSlots slots{p.keys, p.ninstances, p.level_keys, p.nlevels, error};
          for (int o = op0; o < op1; ++o) {
            const int patch = static_cast<const int*>(sg.ops)[o];
            const int start = static_cast<const int*>(sg.aux)[o];
            if (p.ndim == 2)
              rate_chunk2d<S, kProgramThreads>(pool, a.patches, patch, start, p.b0[0], p.b0[1], p.gamma, slots);
            else
              rate_chunk3d<S, kProgramThreads>(pool, a.patches, patch, start, p.b0[0], p.b0[1], p.b0[2], p.gamma,
                                               slots);
          }
          break;
        }
        case WB_SEG_FINALIZE_DT:
          for (int i = tid; i < p.ninstances; i += kProgramThreads)
            finalize_dt_one(i, p.keys, p.cfl, p.dt_eta, p.dt_kappa, p.gamma, p.inv_dx2_sum, p.level_keys,
                            p.inv_dx2_levels, p.nlevels, p.time, p.end, p.dt, p.advance);
          break;
        case WB_SEG_ADVANCE_TIME:
          for (int i = tid; i < p.ninstances; i += kProgramThreads) p.time[i] += p.dt[i];
          break;
        default:
          break;
      }
    }
    __syncthreads();  // every thread's stores of the item, and its reads of s_ticket / s_go
    if (tid == 0) {
      __threadfence();
      atomicAdd(done + phase, 1u);
    }
  }
  // the last block to leave resets the counters (every other block has taken its final
  // ticket by then); the error word stays for the host
  if (tid == 0) {
    __threadfence();
    if (atomicAdd(left, 1u) == gridDim.x - 1) {
      *ticket = 0u;
      *left = 0u;
      for (int q = 0; q < a.nphases; ++q) done[q] = 0u;
      __threadfence();
    }
  }
}

namespace {

// Blocks per SM the kernel's registers allow (queried once per instantiation and
// device), times the SMs; no more blocks than items.
template <typename S>
int program_grid(int items, int capacity_only) {
  static std::mutex mutex;
  static int cached[64] = {};
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) return 0;
  std::lock_guard<std::mutex> lock(mutex);
  if (!cached[device]) {
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, program_kernel<S>, kProgramThreads, 0) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || per_sm <= 0)
      return 0;
    cached[device] = per_sm * sms;
  }
  if (capacity_only) return cached[device];
  return items < cached[device] ? items : cached[device];
}

template <typename S>
int launch_program(const ProgramArgs<S>& a, cudaStream_t stream) {
  const int grid = program_grid<S>(a.total, 0);
  if (grid <= 0) {
    set_error("run_program: occupancy query failed");
    return kCudaError;
  }
  program_kernel<S><<<grid, kProgramThreads, 0, stream>>>(a);
  return check_launch("run_program");
}

// Host checks of a program: kinds, pools, phases in order with no empty phase, the
// pointers each kind needs; fills in the items' numbering and the phase totals.
template <typename S>
int prepare(ProgramArgs<S>& a, const wb_program_segment* segments, int nsegments, const wb_program_params* params) {
  if (nsegments <= 0 || nsegments > WB_PROGRAM_MAX_SEGMENTS) {
    set_error("run_program: %d segments (1..%d)", nsegments, WB_PROGRAM_MAX_SEGMENTS);
    return kBadArgument;
  }
  std::memcpy(&a.p, params, sizeof(wb_program_params));
  const wb_program_params& p = a.p;
  if (p.ninstances <= 0 || (p.level_keys && p.nlevels <= 0) || (p.ndim != 2 && p.ndim != 3) || !(p.gamma > 1.0)) {
    set_error("run_program: bad ninstances / nlevels / ndim / gamma");
    return kBadArgument;
  }
  int64_t total = 0;
  int phase = 0;
  for (int k = 0; k < nsegments; ++k) {
    wb_program_segment sg = segments[k];
    if (sg.kind < WB_SEG_COPY || sg.kind > WB_SEG_ADVANCE_TIME || (sg.pool != 0 && sg.pool != 1) || sg.count <= 0) {
      set_error("run_program: segment %d: bad kind %d, pool %d or count %d", k, sg.kind, sg.pool, sg.count);
      return kBadArgument;
    }
    if (k == 0 ? sg.phase != 0 : (sg.phase != phase && sg.phase != phase + 1)) {
      set_error("run_program: segment %d: phase %d after phase %d (phases run 0, 1, ... without gaps)", k, sg.phase,
                phase);
      return kBadArgument;
    }
    phase = sg.phase;
    const bool needs_ops = sg.kind <= WB_SEG_REFLUX || sg.kind == WB_SEG_RATE;
    const bool one_item = sg.kind == WB_SEG_INIT_KEYS || sg.kind == WB_SEG_FINALIZE_DT || sg.kind == WB_SEG_ADVANCE_TIME;
    const bool spacings = p.level_keys ? p.inv_dx2_levels != nullptr : p.inv_dx2_sum != nullptr;
    if ((needs_ops && !sg.ops) || (sg.kind == WB_SEG_RATE && !sg.aux) || (one_item && sg.count != 1) ||
        (sg.kind == WB_SEG_REFLUX && !p.reg) ||
        ((sg.kind == WB_SEG_REFLUX || sg.kind == WB_SEG_FINALIZE_DT || sg.kind == WB_SEG_ADVANCE_TIME) && !p.dt) ||
        ((sg.kind == WB_SEG_INIT_KEYS || sg.kind == WB_SEG_RATE || sg.kind == WB_SEG_FINALIZE_DT) && !p.keys) ||
        (sg.kind == WB_SEG_ADVANCE_TIME && !p.time) ||
        (sg.kind == WB_SEG_FINALIZE_DT && (((p.end || p.advance) && !p.time) || !spacings))) {
      set_error("run_program: segment %d (kind %d) lacks an operand (ops, work list, register, dt, keys, time or "
                "spacings) or has more than one item",
                k, sg.kind);
      return kBadArgument;
    }
    // runs of ops: about two items per block of the grid, at most kProgramMaxRun ops each
    const int capacity = program_grid<S>(0, 1);
    if (capacity <= 0) {
      set_error("run_program: occupancy query failed");
      return kCudaError;
    }
    const bool runs = sg.kind <= WB_SEG_REFLUX || sg.kind == WB_SEG_RATE;
    sg.pad = runs ? std::max(1, std::min(kProgramMaxRun, (sg.count + 2 * capacity - 1) / (2 * capacity))) : 1;
    sg.first = int(total);
    total += (sg.count + sg.pad - 1) / sg.pad;
    if (total >= (int64_t(1) << 31) - (int64_t(1) << 20)) {
      set_error("run_program: too many items");
      return kTooLarge;
    }
    a.seg[k] = sg;
  }
  a.nsegments = nsegments;
  a.nphases = phase + 1;
  a.total = int(total);
  for (int q = 0; q < a.nphases; ++q) a.phase_total[q] = 0;
  for (int k = 0; k < nsegments; ++k) a.phase_total[a.seg[k].phase] += (a.seg[k].count + a.seg[k].pad - 1) / a.seg[k].pad;
  return kOk;
}

}  // namespace
}  // namespace wb

extern "C" int wb_run_program(int precision, void* pool0, void* pool1, const void* patches,
                              const wb_program_segment* segments, int nsegments, const wb_program_params* params,
                              unsigned* counters, void* stream) {
  using namespace wb;
  set_error("");
  if (precision != 32 && precision != 64 && precision != kMath32State64) {
    set_error("run_program: precision must be 32, 64 or %d, got %d", kMath32State64, precision);
    return kBadArgument;
  }
  if (!pool0 || !patches || !segments || !params || !counters) {
    set_error("run_program: a required pointer is NULL");
    return kBadArgument;
  }
  for (int k = 0; k < nsegments && k < WB_PROGRAM_MAX_SEGMENTS; ++k)
    if (segments[k].pool == 1 && !pool1) {
      set_error("run_program: segment %d uses the second pool, which is NULL", k);
      return kBadArgument;
    }
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (precision == 32) {
    ProgramArgs<float> a{};
    a.pools[0] = static_cast<float*>(pool0), a.pools[1] = static_cast<float*>(pool1);
    a.patches = static_cast<const PatchDesc*>(patches), a.counters = counters;
    const int status = prepare(a, segments, nsegments, params);
    return status != kOk ? status : launch_program<float>(a, s);
  }
  ProgramArgs<double> a{};  // float64 and the float64 state of the mixed precision
  a.pools[0] = static_cast<double*>(pool0), a.pools[1] = static_cast<double*>(pool1);
  a.patches = static_cast<const PatchDesc*>(patches), a.counters = counters;
  const int status = prepare(a, segments, nsegments, params);
  return status != kOk ? status : launch_program<double>(a, s);
}
