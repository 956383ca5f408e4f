// batched.cu -- the batched form: many independent solves of uneven grid sizes and orders
// advanced together by SSPRK33 (kernel/kernel_time_integrator.cl:224-303), with every stage
// of every solve processed by one persistent kernel.
//
// Each solve is an ieq_ctx (its settings, SBP tables and SoA state).  A stage is a queue of
// tiles -- bricks of tx*ty*tz = 256 nodes of one solve, the brick shape chosen per solve by
// the autotuner -- that the resident blocks take round-robin; stages are separated by a
// software grid barrier whose wait is bounded (on time-out the kernel sets an error flag
// and returns, the host reports IEQ_ERR_TIMEOUT).  The last block to arrive at a barrier
// also does the stage-time bookkeeping of all solves (SSPRK33_2a/_3a, calc_time_3_args).
// The whole num_steps launch is captured in a CUDA graph.
#include <cstring>
#include <vector>

#include "ieq_host.h"
#include "stage_kernel.cuh"

namespace ieq {

struct BatchSolveDesc {
  StageArgs<double, SoA<double>> st[3];   // the three SSPRK33 stages
  int op_id, periodic;
  int tx, ty, tz;
  int tiles_x, tiles_y, tiles_z;
  long long tile_begin;
  double *time;
  double dt;
};

// the grid barrier's state, reset before every run: arrival count, generation, error flag,
// and its wait parameters -- arrivals the barrier expects beyond the grid (0; a test sets 1
// to make every wait run out) and the spin limit of a wait
struct BatchSync {
  unsigned count;
  unsigned generation;
  int error;
  int extra;
  long long spin_limit;
};

// resident blocks of 256 threads per SM the batched kernels are compiled for
#ifndef IEQ_BATCH_MIN_BLOCKS
#define IEQ_BATCH_MIN_BLOCKS 2
#endif

constexpr long long kBarrierSpinLimit = 20000000;   // x 64 ns nanosleep: about 1.3 s

// bounded grid barrier; the last block to arrive runs `last` before releasing the others
template <typename Last>
__device__ bool grid_barrier(BatchSync *sync, Last last) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned *gen = &sync->generation;
    const unsigned g = *gen;
    __threadfence();
    const long long limit = sync->spin_limit;
    if (atomicAdd(&sync->count, 1u) == gridDim.x - 1 + (unsigned)sync->extra) {
      last();
      sync->count = 0;
      __threadfence();
      atomicAdd(&sync->generation, 1u);
    } else {
      long long it = 0;
      while (*gen == g) {
        if (++it > limit) {
          atomicExch(&sync->error, 1);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    ok = *((volatile int *)&sync->error) == 0;
  }
  __syncthreads();
  return ok != 0;
}

// F selects the load path: SoA (read-only cache; separate launches per stage) or SoAcg
// (L2 only; the persistent kernel).  Both have the SoA descriptor's memory layout.
template <typename F>
__device__ __forceinline__ void run_tile(const BatchSolveDesc *descs, int ns, long long tile, int stage,
                                         int &cur_solve, StageArgs<double, F> &sa, BatchSolveDesc &sd) {
  static_assert(sizeof(StageArgs<double, F>) == sizeof(StageArgs<double, SoA<double>>), "layout");
  // the solve owning this tile (descs are ordered by tile_begin)
  int lo = 0, hi = ns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (descs[mid].tile_begin <= tile) lo = mid;
    else hi = mid - 1;
  }
  const int s = lo;
  if (s != cur_solve) {
    __syncthreads();
    // block-cooperative copy of the solve's stage arguments into shared memory
    const int nw = (int)(sizeof(StageArgs<double, F>) / 8);
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(&descs[s].st[stage]);
    unsigned long long *dst = reinterpret_cast<unsigned long long *>(&sa);
    for (int i = threadIdx.x; i < nw; i += blockDim.x) dst[i] = src[i];
    if (threadIdx.x == 0) sd = descs[s];
    __syncthreads();
    cur_solve = s;
  }
  const long long lt = tile - sd.tile_begin;
  const int bx = (int)(lt % sd.tiles_x);
  const int by = (int)((lt / sd.tiles_x) % sd.tiles_y);
  const int bz = (int)(lt / ((long long)sd.tiles_x * sd.tiles_y));
  const int t = threadIdx.x;
  const int ix = bx * sd.tx + t % sd.tx;
  const int iy = by * sd.ty + (t / sd.tx) % sd.ty;
  const int iz = bz * sd.tz + t / (sd.tx * sd.ty);
  if (ix >= sa.m.nx || iy >= sa.m.ny || iz >= sa.m.nz) return;
  switch (sd.op_id * 2 + sd.periodic) {
    case 0: stage_node<double, F, 0, false, false, DISS_NONE, 1>(sa, ix, iy, iz); break;
    case 1: stage_node<double, F, 0, true, false, DISS_NONE, 1>(sa, ix, iy, iz); break;
    case 2: stage_node<double, F, 1, false, false, DISS_NONE, 1>(sa, ix, iy, iz); break;
    case 3: stage_node<double, F, 1, true, false, DISS_NONE, 1>(sa, ix, iy, iz); break;
    case 4: stage_node<double, F, 2, false, false, DISS_NONE, 1>(sa, ix, iy, iz); break;
    case 5: stage_node<double, F, 2, true, false, DISS_NONE, 1>(sa, ix, iy, iz); break;
  }
}

// stage-time bookkeeping of all solves after stage `stage` (0, 1, 2) of SSPRK33
__device__ void batch_times(const BatchSolveDesc *descs, int ns, int stage) {
  for (int s = 0; s < ns; ++s) {
    double *t = descs[s].time;
    const double dt = descs[s].dt;
    if (stage == 0) {
      t[1] = t[0] + dt;                 // SSPRK33_2a
    } else if (stage == 1) {
      t[1] = t[0] + 0.5 * dt;           // SSPRK33_3a: (REAL)(0.5*DT)
    } else {
      const double t0 = t[0] + dt;      // calc_time_3_args
      t[0] = t0;
      t[1] = t0;
    }
  }
  __threadfence();
}

__global__ void __launch_bounds__(256, IEQ_BATCH_MIN_BLOCKS) k_batch_persistent(const BatchSolveDesc *descs, int ns, long long ntiles,
                                                          int nsteps, BatchSync *sync) {
  __shared__ StageArgs<double, SoAcg<double>> sa;
  __shared__ BatchSolveDesc sd;
  for (int step = 0; step < nsteps; ++step) {
    for (int stage = 0; stage < 3; ++stage) {
      int cur = -1;
      for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
        run_tile<SoAcg<double>>(descs, ns, tile, stage, cur, sa, sd);
      if (!grid_barrier(sync, [&] { batch_times(descs, ns, stage); })) return;
    }
  }
}

// the same stage as an ordinary launch (one block per tile); the last block does the times
__global__ void __launch_bounds__(256, IEQ_BATCH_MIN_BLOCKS) k_batch_stage(const BatchSolveDesc *descs, int ns, long long ntiles, int stage,
                                                     BatchSync *sync) {
  __shared__ StageArgs<double, SoA<double>> sa;
  __shared__ BatchSolveDesc sd;
  int cur = -1;
  run_tile<SoA<double>>(descs, ns, blockIdx.x, stage, cur, sa, sd);
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&sync->count, 1u) == gridDim.x - 1) {
      batch_times(descs, ns, stage);
      sync->count = 0;
    }
  }
}

}  // namespace ieq

using namespace ieq;

struct ieq_batch {
  std::vector<ieq_ctx *> solves;
  std::vector<BatchSolveDesc> host;
  BatchSolveDesc *d_desc = nullptr;
  BatchSync *d_sync = nullptr;
  long long ntiles = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  std::vector<int> tiles;   // tx, ty, tz per solve
  cudaGraphExec_t graph = nullptr;
  int graph_steps = -1, graph_persistent = -1;   // graph_persistent: the mode of the graph
  int grid = 0;
  std::vector<void *> bound;
  cudaEvent_t fork = nullptr;          // IEQ_BATCH_BRANCHES: fork/join of the solves' streams
  std::vector<cudaEvent_t> join;
  BatchSync sync_init{0u, 0u, 0, 0, kBarrierSpinLimit};   // copied to d_sync before every run
};

// from api.cu / api_fused.inc
namespace ieq {
template <typename R, typename F>
StageArgs<R, F> stage_args_for_batch(ieq_ctx *c);
ieq_status batch_enter(ieq_ctx *c, void *b, void *b2, void *b3, void *u, double **soa_base, long long *stride);
ieq_status batch_leave(ieq_ctx *c, void *b, void *b2, void *b3);
ieq_status batch_enqueue_steps(ieq_ctx *c, int steps, double *time);
}  // namespace ieq

static ieq_status bfail(ieq_batch *b, ieq_status st, const std::string &m) {
  b->err = m;
  return st;
}

extern "C" {

ieq_status ieq_batch_create(ieq_batch **out, ieq_ctx *const *solves, int n) {
  if (!out || !solves || n <= 0) return IEQ_ERR_ARG;
  *out = nullptr;
  ieq_batch *b = new ieq_batch();
  for (int i = 0; i < n; ++i) {
    ieq_ctx *c = solves[i];
    const ieq::Settings &s = c->s;
    std::string why;
    if (s.real_float) why = "REAL must be double";
    else if (s.integrator != "SSPRK33") why = "the integrator must be SSPRK33";
    else if (s.hall) why = "Hall solves are not batched";
    else if (s.dissipation) why = "solves with dissipation are not batched";
    else if (s.extended) why = "the extended operators are not batched";
    else if (s.variable_u) why = "variable velocity is not batched";
    else if (s.uibj < 0 || s.source < 0 || s.ujbi < 0) why = "no flux forms";
    else if (i > 0 && c->device != solves[0]->device) why = "all solves must use one device";
    if (!why.empty()) {
      b->err = "solve " + std::to_string(i) + ": " + why;
      *out = b;
      return IEQ_ERR_SETTINGS;
    }
    b->solves.push_back(c);
    b->tiles.insert(b->tiles.end(), {32, 4, 2});
  }
  b->device = solves[0]->device;
  cudaSetDevice(b->device);
  b->join.assign(n, nullptr);
  bool ev = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; i < n && ev; ++i) ev = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ev || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&b->d_desc, n * sizeof(BatchSolveDesc)) != cudaSuccess ||
      cudaMalloc(&b->d_sync, sizeof(BatchSync)) != cudaSuccess ||
      cudaMemset(b->d_sync, 0, sizeof(BatchSync)) != cudaSuccess) {
    b->err = "CUDA allocation failed";
    *out = b;
    return IEQ_ERR_CUDA;
  }
  *out = b;
  return IEQ_OK;
}

void ieq_batch_destroy(ieq_batch *b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->d_desc) cudaFree(b->d_desc);
  if (b->d_sync) cudaFree(b->d_sync);
  if (b->stream) cudaStreamDestroy(b->stream);
  if (b->fork) cudaEventDestroy(b->fork);
  for (cudaEvent_t e : b->join)
    if (e) cudaEventDestroy(e);
  delete b;
}

const char *ieq_batch_last_error(const ieq_batch *b) { return b ? b->err.c_str() : ""; }

void *ieq_batch_stream(ieq_batch *b) { return b ? (void *)b->stream : nullptr; }

ieq_status ieq_batch_set_tile(ieq_batch *b, int solve, int tx, int ty, int tz) {
  if (!b || solve < 0 || solve >= (int)b->solves.size()) return IEQ_ERR_ARG;
  if (tx < 1 || ty < 1 || tz < 1 || tx * ty * tz != 256) return bfail(b, IEQ_ERR_ARG, "tile must hold 256 nodes");
  b->tiles[3 * solve] = tx;
  b->tiles[3 * solve + 1] = ty;
  b->tiles[3 * solve + 2] = tz;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return IEQ_OK;
}

// Bind the solves' fields: fields[5*i + k] holds solve i's b, b2, b3, u and time (device
// pointers in the reference layout; rho is 1 and not read).  The state is copied into each
// context's SoA buffers and the tile queue is built.
ieq_status ieq_batch_bind(ieq_batch *b, void *const *fields) {
  if (!b || !fields) return IEQ_ERR_ARG;
  if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, IEQ_ERR_CUDA, "cudaSetDevice");
  const int n = (int)b->solves.size();
  b->host.assign(n, BatchSolveDesc{});
  b->bound.assign(fields, fields + 5 * n);
  long long tiles = 0;
  for (int i = 0; i < n; ++i) {
    ieq_ctx *c = b->solves[i];
    void *bb = fields[5 * i], *b2 = fields[5 * i + 1], *b3 = fields[5 * i + 2], *u = fields[5 * i + 3],
         *tm = fields[5 * i + 4];
    if (!bb || !b2 || !b3 || !u || !tm) return bfail(b, IEQ_ERR_ARG, "null field");
    double *base = nullptr;
    long long s = 0;
    ieq_status st = batch_enter(c, bb, b2, b3, u, &base, &s);
    if (st != IEQ_OK) return bfail(b, st, c->err);
    BatchSolveDesc &d = b->host[i];
    // u is never written during a run: it may use the read-only cached path
    const SoA<double> b1s{base, s, 0}, b2s{base + 6 * s, s, 0}, b3s{base + 9 * s, s, 0}, us{base + 15 * s, s, 1};
    for (int k = 0; k < 3; ++k) {
      StageArgs<double, SoA<double>> a = stage_args_for_batch<double, SoA<double>>(c);
      a.u = us;
      a.time = (double *)tm;
      a.h = (double)c->s.dt;
      if (k == 0) {
        a.bk = b1s; a.X = b1s; a.out = b2s; a.mode = EP_X_PLUS_HF;
      } else if (k == 1) {
        a.bk = b2s; a.X = b1s; a.Y = b2s; a.out = b3s; a.mode = EP_PX_QYHF; a.p = 0.75; a.q = 0.25;
      } else {
        a.bk = b3s; a.X = b1s; a.Y = b3s; a.out = b1s; a.mode = EP_PX_QYHF; a.p = 1.0 / 3.0; a.q = 2.0 / 3.0;
      }
      d.st[k] = a;
    }
    d.op_id = c->op_id;
    d.periodic = c->s.periodic ? 1 : 0;
    d.tx = b->tiles[3 * i];
    d.ty = b->tiles[3 * i + 1];
    d.tz = b->tiles[3 * i + 2];
    d.tiles_x = (c->s.nodes[0] + d.tx - 1) / d.tx;
    d.tiles_y = (c->s.nodes[1] + d.ty - 1) / d.ty;
    d.tiles_z = (c->s.nodes[2] + d.tz - 1) / d.tz;
    d.tile_begin = tiles;
    tiles += (long long)d.tiles_x * d.tiles_y * d.tiles_z;
    d.time = (double *)tm;
    d.dt = c->s.dt;
  }
  b->ntiles = tiles;
  // the inputs were converted on the solves' streams; order them before the batch stream
  for (ieq_ctx *c : b->solves)
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bfail(b, IEQ_ERR_CUDA, "conversion");
  if (cudaMemcpyAsync(b->d_desc, b->host.data(), n * sizeof(BatchSolveDesc), cudaMemcpyHostToDevice, b->stream) !=
          cudaSuccess ||
      cudaMemsetAsync(b->d_sync, 0, sizeof(BatchSync), b->stream) != cudaSuccess)
    return bfail(b, IEQ_ERR_CUDA, "descriptor upload");
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return IEQ_OK;
}

// num_steps SSPRK33 steps of every bound solve on the batch stream.  persistent = 1: one
// persistent launch (stages separated by the bounded grid barrier); 0: one launch per stage.
// Either is captured once into a CUDA graph and replayed.  Returns IEQ_ERR_TIMEOUT if a
// grid barrier gave up (blocks not co-resident).  Synchronises.
ieq_status ieq_batch_run(ieq_batch *b, int num_steps, int mode) {
  if (!b || num_steps < 0 || b->ntiles == 0 || mode < 0 || mode > 2) return IEQ_ERR_ARG;
  if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, IEQ_ERR_CUDA, "cudaSetDevice");
  const int n = (int)b->solves.size();
  if (!b->graph || b->graph_steps != num_steps || b->graph_persistent != mode) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    int per_sm = 0, nsm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_persistent, 256, 0);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device);
    const long long resident = (long long)per_sm * nsm;
    b->grid = (int)(resident < b->ntiles ? resident : b->ntiles);
    if (b->grid < 1) return bfail(b, IEQ_ERR_CUDA, "no resident blocks for the persistent kernel");
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      return bfail(b, IEQ_ERR_CUDA, "capture");
    if (mode == IEQ_BATCH_BRANCHES) {
      // one branch per solve: fork onto the solves' streams, join back
      ieq_status st = IEQ_OK;
      if (cudaEventRecord(b->fork, b->stream) != cudaSuccess) st = IEQ_ERR_CUDA;
      for (int i = 0; i < n && st == IEQ_OK; ++i) {
        ieq_ctx *c = b->solves[i];
        if (cudaStreamWaitEvent(c->stream, b->fork, 0) != cudaSuccess) st = IEQ_ERR_CUDA;
        if (st == IEQ_OK) st = batch_enqueue_steps(c, num_steps, b->host[i].time);
        if (st == IEQ_OK && (cudaEventRecord(b->join[i], c->stream) != cudaSuccess ||
                             cudaStreamWaitEvent(b->stream, b->join[i], 0) != cudaSuccess))
          st = IEQ_ERR_CUDA;
      }
      cudaStreamEndCapture(b->stream, &g);
      if (st != IEQ_OK) {
        if (g) cudaGraphDestroy(g);
        return bfail(b, st, "branch capture");
      }
      if (cudaGraphInstantiate(&b->graph, g, 0) != cudaSuccess) return bfail(b, IEQ_ERR_CUDA, "instantiate");
      cudaGraphDestroy(g);
      b->graph_steps = num_steps;
      b->graph_persistent = mode;
    } else if (mode == IEQ_BATCH_PERSISTENT) {
      k_batch_persistent<<<b->grid, 256, 0, b->stream>>>(b->d_desc, n, b->ntiles, num_steps, b->d_sync);
    } else {
      for (int step = 0; step < num_steps; ++step)
        for (int k = 0; k < 3; ++k)
          k_batch_stage<<<(unsigned)b->ntiles, 256, 0, b->stream>>>(b->d_desc, n, b->ntiles, k, b->d_sync);
    }
    if (mode != IEQ_BATCH_BRANCHES) {
      if (cudaStreamEndCapture(b->stream, &g) != cudaSuccess) return bfail(b, IEQ_ERR_CUDA, "capture end");
      if (cudaGraphInstantiate(&b->graph, g, 0) != cudaSuccess) return bfail(b, IEQ_ERR_CUDA, "instantiate");
      cudaGraphDestroy(g);
      b->graph_steps = num_steps;
      b->graph_persistent = mode;
    }
  }
  // a fresh barrier state for every run: a run after a time-out starts from a zero count
  // and a clear error flag
  if (cudaMemcpyAsync(b->d_sync, &b->sync_init, sizeof(BatchSync), cudaMemcpyHostToDevice, b->stream) != cudaSuccess)
    return bfail(b, IEQ_ERR_CUDA, "barrier reset");
  if (num_steps > 0 && cudaGraphLaunch(b->graph, b->stream) != cudaSuccess) return bfail(b, IEQ_ERR_CUDA, "launch");
  BatchSync hs{};
  if (cudaMemcpyAsync(&hs, b->d_sync, sizeof(hs), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess ||
      cudaStreamSynchronize(b->stream) != cudaSuccess)
    return bfail(b, IEQ_ERR_CUDA, std::string("batch run: ") + cudaGetErrorString(cudaGetLastError()));
  if (hs.error) return bfail(b, IEQ_ERR_TIMEOUT, "grid barrier timed out (blocks not co-resident)");
  return IEQ_OK;
}

// copy the solves' state back into the bound fields (b, b2, b3)
ieq_status ieq_batch_unbind(ieq_batch *b) {
  if (!b || b->bound.empty()) return IEQ_ERR_ARG;
  for (size_t i = 0; i < b->solves.size(); ++i) {
    ieq_status st = batch_leave(b->solves[i], b->bound[5 * i], b->bound[5 * i + 1], b->bound[5 * i + 2]);
    if (st != IEQ_OK) return bfail(b, st, b->solves[i]->err);
  }
  for (ieq_ctx *c : b->solves)
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bfail(b, IEQ_ERR_CUDA, "conversion");
  return IEQ_OK;
}

int ieq_batch_grid(const ieq_batch *b) { return b ? b->grid : 0; }

// Test hook of the persistent mode's grid barrier: the barrier then waits for `extra_arrivals`
// blocks beyond the grid (1: a block that never comes, so every wait runs out) with a spin
// limit of `spin_limit` 64-ns sleeps (<= 0: the default, about 1.3 s).  (0, 0) restores the
// production barrier.
ieq_status ieq_batch_test_barrier(ieq_batch *b, int extra_arrivals, long long spin_limit) {
  if (!b || extra_arrivals < 0 || extra_arrivals > 1) return IEQ_ERR_ARG;
  b->sync_init.extra = extra_arrivals;
  b->sync_init.spin_limit = spin_limit > 0 ? spin_limit : kBarrierSpinLimit;
  return IEQ_OK;
}

long long ieq_batch_total_tiles(const ieq_batch *b) { return b ? b->ntiles : 0; }

}  // extern "C"
