// Batching form: frequency sweeps over several geometries of uneven N.
//
// A job is one (geometry, omega): assemble the complex128 VIE matrix, LU
// factor it (FP64 tensor-core path), solve one plane-wave right-hand side
// and reduce the absorbed power of every object (overlap method) -- the
// per-frequency work of a sweep such as a heat-transfer spectrum.  No
// reference counterpart: the reference runs such sweeps one frequency at a
// time through SWGGeometry::AssembleVIEMatrix / HMatrix::LUFactorize.
//
// Execution:
//  * every job's launch sequence is the same for a given geometry, and the
//    frequency enters only through a device word (the kernels' fq argument),
//    so the sequence is captured once per (geometry, slot) into a CUDA graph
//    and replayed per frequency: one graph launch per job instead of the
//    thousands of launches of the recursive LU;
//  * a geometry's jobs are spread over S slots, each with its own stream,
//    matrix and buffers, so that small factorisations run concurrently;
//  * an online autotuner picks, per size class (N rounded up to 1024), the
//    LU panel slice height (rows per CTA of the cooperative panel kernel:
//    16, 32 or 64), the CTA tile of the complex128 tensor-core GEMM (64 x 64,
//    128 x 64 or 64 x 128) and the number of concurrent slots (1, 2, 4, ... up
//    to the caller's maximum) by
//    timing the sweep's own first jobs (their results are kept), and
//    remembers the choice for later geometries of the same class.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "internal.h"

namespace bg {

#define BATCH_MAXOBJ 4       // objects per geometry (absorbed-power outputs)

__global__ void k_batch_status(const int *info, const int *solve_err, int *acc) {
  if (threadIdx.x == 0) {
    if (*info) atomicMax(acc, *info);
    if (*solve_err) atomicMax(acc + 1, 1);
  }
}

struct Slot {
  cudaStream_t s = nullptr;
  bg_matrix *M = nullptr;
  void *rhs = nullptr, *T = nullptr;
  double *fq = nullptr, *part = nullptr, *out = nullptr;
  int *status = nullptr;     // [max LAPACK info, solve error]
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

static void slot_free(Slot &S) {
  if (S.exec) cudaGraphExecDestroy(S.exec);
  if (S.graph) cudaGraphDestroy(S.graph);
  if (S.M) bg_matrix_destroy(S.M);
  void *ps[] = {S.rhs, S.T, S.fq, S.part, S.out, S.status};
  for (void *p : ps)
    if (p) cudaFree(p);
  if (S.s) cudaStreamDestroy(S.s);
  S = Slot();
}

// one job's launch sequence on the calling thread's stream
static int enqueue_job(bg_geometry *g, Slot &S, const double *E0, const double *nhat) {
  int N = g->N, st;
  // the placeholder omega (1, 0) is never used: every kernel reads S.fq
  if ((st = assemble_far(g, 1.0, 0.0, S.M->d, S.M->ld, S.fq))) return st;
  if ((st = assemble_near(g, 1.0, 0.0, S.M->d, S.M->ld, S.fq))) return st;
  if ((st = assemble_gram(g, 1.0, 0.0, S.M->d, S.M->ld, S.fq))) return st;
  if ((st = lu_factor_enqueue(S.M))) return st;
  if ((st = rhs_planewave(g, 1.0, 0.0, E0, nhat, S.rhs, S.fq))) return st;
  if ((st = lu_solve_enqueue(S.M, S.rhs, N, 1, S.T))) return st;
  k_batch_status<<<1, 32, 0, stream()>>>(lu_capture_info_ptr(S.M), lu_capture_solve_err_ptr(S.M), S.status);
  BG_LAUNCHED();
  return opft_enqueue(g, 1.0, 0.0, S.rhs, S.fq, S.part, S.out);
}

static bool s_warm = false;          // lazily set kernel attributes and tables are in place
static bool s_capture_failed = false;

static int slot_init(bg_geometry *g, Slot &S, const double *E0, const double *nhat, bool use_graph) {
  int N = g->N, NO = (int)g->objs.size();
  BG_CUDA_TRY(cudaStreamCreateWithFlags(&S.s, cudaStreamNonBlocking));
  int st = bg_matrix_create(g, BG_C128, &S.M);
  if (st) return st;
  BG_CUDA_TRY(cudaMalloc(&S.rhs, 16 * (size_t)N));
  BG_CUDA_TRY(cudaMalloc(&S.T, 16 * (size_t)N));
  BG_CUDA_TRY(cudaMalloc(&S.fq, 4 * sizeof(double)));
  BG_CUDA_TRY(cudaMalloc(&S.part, sizeof(double) * (size_t)((N + 127) / 128) * NO));
  BG_CUDA_TRY(cudaMalloc(&S.out, sizeof(double) * BATCH_MAXOBJ));
  BG_CUDA_TRY(cudaMalloc(&S.status, 2 * sizeof(int)));
  BG_CUDA_TRY(cudaMemset(S.status, 0, 2 * sizeof(int)));
  BG_CUDA_TRY(cudaMemset(S.out, 0, sizeof(double) * BATCH_MAXOBJ));
  const double one[2] = {1.0, 0.0};
  BG_CUDA_TRY(cudaMemcpy(S.fq, one, sizeof one, cudaMemcpyHostToDevice));
  set_thread_stream(S.s);
  st = lu_capture_prepare(S.M);
  if (!st && use_graph && !s_warm) {
    // one uncaptured pass per process: tables and kernel attributes that the
    // library sets on first use are then in place before any capture
    st = enqueue_job(g, S, E0, nhat);
    if (!st) {
      cudaError_t e = cudaStreamSynchronize(S.s);
      if (e != cudaSuccess) { set_error("batch warm-up: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
    }
    if (!st) s_warm = true;
  }
  if (!st && use_graph) {
    cudaError_t e = cudaStreamBeginCapture(S.s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      int cst = enqueue_job(g, S, E0, nhat);
      cudaGraph_t graph = nullptr;
      e = cudaStreamEndCapture(S.s, &graph);
      if (!cst && e == cudaSuccess) {
        S.graph = graph;
        e = cudaGraphInstantiate(&S.exec, S.graph, 0);
      } else if (graph) {
        cudaGraphDestroy(graph);
      }
      if (cst || e != cudaSuccess) {
        // the sequence could not be recorded: run this slot's jobs as direct launches
        if (S.exec) cudaGraphExecDestroy(S.exec);
        if (S.graph) cudaGraphDestroy(S.graph);
        S.exec = nullptr;
        S.graph = nullptr;
        s_capture_failed = true;
      }
    } else {
      s_capture_failed = true;
    }
    cudaGetLastError();
  }
  set_thread_stream(nullptr);
  return st;
}

// launches job (omega) on slot S and copies its absorbed powers to dst (device)
// w: pinned host {Re, Im}, so that the copy does not wait for the stream
static int run_job(bg_geometry *g, Slot &S, const double *w, const double *E0, const double *nhat, double *dst) {
  BG_CUDA_TRY(cudaMemcpyAsync(S.fq, w, 2 * sizeof(double), cudaMemcpyHostToDevice, S.s));
  if (S.exec) {
    BG_CUDA_TRY(cudaGraphLaunch(S.exec, S.s));
    g_launches++;
  } else {
    set_thread_stream(S.s);
    int st = enqueue_job(g, S, E0, nhat);
    set_thread_stream(nullptr);
    if (st) return st;
  }
  BG_CUDA_TRY(cudaMemcpyAsync(dst, S.out, sizeof(double) * BATCH_MAXOBJ, cudaMemcpyDeviceToDevice, S.s));
  return BG_OK;
}

// autotuner memory: size class -> (panel rows, slots)
struct Tuned { int rows = 0, slots = 0, tile = 0; double s_per_job = 0; };
static std::map<int, Tuned> s_tuned;
static std::mutex s_tune_mu;
static int size_class(int N) { return (N + 1023) / 1024; }

static double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static int sync_slots(std::vector<Slot> &slots) {
  for (auto &S : slots) BG_CUDA_TRY(cudaStreamSynchronize(S.s));
  return BG_OK;
}

// Runs jobs [j0, j1) of geometry g round-robin over the slots; returns seconds.
static int run_range(bg_geometry *g, std::vector<Slot> &slots, const double *omega, int j0, int j1,
                     const double *E0, const double *nhat, double *d_out, double *secs) {
  double t0 = now();
  for (int j = j0; j < j1; j++) {
    Slot &S = slots[(j - j0) % slots.size()];
    int st = run_job(g, S, omega + 2 * j, E0, nhat, d_out + (size_t)j * BATCH_MAXOBJ);
    if (st) return st;
  }
  int st = sync_slots(slots);
  *secs = now() - t0;
  return st;
}

// factorisation / solve status accumulated by the slots' jobs
static int check_slots(std::vector<Slot> &slots) {
  for (auto &S : slots) {
    int acc[2] = {0, 0};
    if (!S.status) continue;
    BG_CUDA_TRY(cudaMemcpy(acc, S.status, sizeof acc, cudaMemcpyDeviceToHost));
    if (acc[1]) { set_error("batched triangular solve timed out"); return BG_ERR_CUDA; }
    if (acc[0]) { set_error("batched LU: singular matrix (info %d)", acc[0]); return BG_ERR_NUMERIC; }
  }
  return BG_OK;
}

static void free_slots(std::vector<Slot> &slots) {
  for (auto &S : slots) slot_free(S);
  slots.clear();
}

// whole sweep of one geometry: tuning (when the size class is new) and the rest
static int sweep_geometry(bg_geometry *g, const double *omega, int nw, const double *E0, const double *nhat,
                          int max_slots, bool use_graph, double *d_out, double *tuning) {
  int st = bg_geometry_precompute(g);
  if (st) return st;
  int cls = size_class(g->N);
  Tuned tn;
  {
    std::lock_guard<std::mutex> lk(s_tune_mu);
    auto it = s_tuned.find(cls);
    if (it != s_tuned.end()) tn = it->second;
  }
  int j = 0;
  std::vector<Slot> slots;
  const int saved_rows = lu_get_panel_rows(), saved_tile = lu_get_gemm_tile();
  const bool tuned_now = tn.rows == 0;
  if (tuned_now) {
    // panel slice height, one slot, one job each (the first is also the warm-up)
    double best = 1e30;
    int best_rows = saved_rows;
    const int cand_rows[3] = {32, 16, 64};
    for (int c = 0; c < 3 && j < nw; c++) {
      lu_set_panel_rows(cand_rows[c]);
      slots.resize(1);
      if ((st = slot_init(g, slots[0], E0, nhat, use_graph))) break;
      double t = 0;
      if ((st = run_range(g, slots, omega, j, j + 1, E0, nhat, d_out, &t))) break;
      j++;
      if (j < nw) {   // time a replay, not the first launch of the graph
        if ((st = run_range(g, slots, omega, j, j + 1, E0, nhat, d_out, &t))) break;
        j++;
      }
      if (t < best) { best = t; best_rows = cand_rows[c]; }
      st = check_slots(slots);
      free_slots(slots);
      if (st) break;
    }
    if (st) { free_slots(slots); lu_set_panel_rows(saved_rows); return st; }
    lu_set_panel_rows(best_rows);
    // GEMM tile: the 64 x 64 default was timed above; one job each for the others
    int best_tile = saved_tile;
    for (int tile = 1; tile <= 2 && j < nw && !st; tile++) {
      lu_set_gemm_tile(tile);
      slots.resize(1);
      if ((st = slot_init(g, slots[0], E0, nhat, use_graph))) break;
      double t = 0;
      if ((st = run_range(g, slots, omega, j, j + 1, E0, nhat, d_out, &t))) break;
      j++;
      if (j < nw) {
        if ((st = run_range(g, slots, omega, j, j + 1, E0, nhat, d_out, &t))) break;
        j++;
      }
      if (t < best) { best = t; best_tile = tile; }
      st = check_slots(slots);
      free_slots(slots);
    }
    if (st) { free_slots(slots); lu_set_panel_rows(saved_rows); lu_set_gemm_tile(saved_tile); return st; }
    lu_set_gemm_tile(best_tile);
    // concurrent slots: time two jobs per slot for each count
    double best_rate = best;
    int best_slots = 1;
    for (int ns = 2; ns <= std::max(1, max_slots) && j < nw; ns *= 2) {
      slots.resize(ns);
      for (auto &S : slots)
        if ((st = slot_init(g, S, E0, nhat, use_graph))) break;
      if (st) break;
      double t = 0;
      int jn = std::min(nw, j + ns);   // first launch of each graph
      if ((st = run_range(g, slots, omega, j, jn, E0, nhat, d_out, &t))) break;
      j = jn;
      jn = std::min(nw, j + 2 * ns);
      if (jn > j) {
        if ((st = run_range(g, slots, omega, j, jn, E0, nhat, d_out, &t))) break;
        double rate = t / (jn - j);
        if (rate < best_rate) { best_rate = rate; best_slots = ns; }
        j = jn;
      }
      st = check_slots(slots);
      free_slots(slots);
      if (st) break;
    }
    if (st) { free_slots(slots); lu_set_panel_rows(saved_rows); lu_set_gemm_tile(saved_tile); return st; }
    tn.rows = best_rows;
    tn.tile = best_tile;
    tn.slots = best_slots;
    tn.s_per_job = best_rate;
    std::lock_guard<std::mutex> lk(s_tune_mu);
    s_tuned[cls] = tn;
  }
  lu_set_panel_rows(tn.rows);
  lu_set_gemm_tile(tn.tile);
  double t = 0;
  if (j < nw) {
    slots.resize(std::min(tn.slots, nw - j));
    for (auto &S : slots)
      if ((st = slot_init(g, S, E0, nhat, use_graph))) break;
    if (!st) st = run_range(g, slots, omega, j, nw, E0, nhat, d_out, &t);
  }
  if (!st) st = check_slots(slots);
  free_slots(slots);
  lu_set_panel_rows(saved_rows);
  lu_set_gemm_tile(saved_tile);
  if (tuning) {
    tuning[0] = tn.rows;
    tuning[1] = tn.slots;
    tuning[2] = tuned_now ? tn.s_per_job : 0.0;
    tuning[3] = tn.tile;
  }
  return st;
}

}  // namespace bg

using namespace bg;

extern "C" {

int bg_batch_sweep(bg_geometry *const *geoms, int ngeom, const double *omega, int nomega, const double *E0,
                   const double *nhat, int max_streams, int flags, double *pabs, double *stats) {
  if (!geoms || ngeom <= 0 || !omega || nomega <= 0 || !E0 || !nhat || !pabs || max_streams < 1) {
    set_error("bg_batch_sweep: bad arguments");
    return BG_ERR_ARG;
  }
  for (int i = 0; i < ngeom; i++) {
    if (!geoms[i]) { set_error("bg_batch_sweep: geometry %d is NULL", i); return BG_ERR_ARG; }
    if ((int)geoms[i]->objs.size() > BATCH_MAXOBJ) {
      set_error("bg_batch_sweep: at most %d objects per geometry", BATCH_MAXOBJ);
      return BG_ERR_ARG;
    }
    if (geoms[i]->dispersive) {
      set_error("bg_batch_sweep: geometry %d has a frequency-dependent MATERIAL; sweep it with bg_assemble", i);
      return BG_ERR_ARG;
    }
  }
  for (int j = 0; j < nomega; j++)
    if (omega[2 * j] == 0.0 && omega[2 * j + 1] == 0.0) { set_error("bg_batch_sweep: omega must be nonzero"); return BG_ERR_ARG; }
  int st = ensure_device();
  if (st) return st;
  bool use_graph = !(flags & BG_BATCH_NO_GRAPHS);
  double *d_out = nullptr, *h_w = nullptr;
  BG_CUDA_TRY(cudaMallocHost(&h_w, sizeof(double) * 2 * (size_t)nomega));
  memcpy(h_w, omega, sizeof(double) * 2 * (size_t)nomega);
  cudaError_t ea = cudaMalloc(&d_out, sizeof(double) * BATCH_MAXOBJ * (size_t)nomega);
  if (ea != cudaSuccess) { cudaFreeHost(h_w); set_error("bg_batch_sweep: %s", cudaGetErrorString(ea)); return BG_ERR_NOMEM; }
  double t0 = std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
  for (int i = 0; i < ngeom && !st; i++) {
    double tun[4] = {0, 0, 0, 0};
    cudaError_t e0 = cudaMemset(d_out, 0, sizeof(double) * BATCH_MAXOBJ * (size_t)nomega);
    if (e0 != cudaSuccess) { set_error("bg_batch_sweep: %s", cudaGetErrorString(e0)); st = BG_ERR_CUDA; break; }
    st = sweep_geometry(geoms[i], h_w, nomega, E0, nhat, max_streams, use_graph, d_out, tun);
    if (!st) {
      cudaError_t e = cudaMemcpy(pabs + (size_t)i * nomega * BATCH_MAXOBJ, d_out,
                                 sizeof(double) * BATCH_MAXOBJ * (size_t)nomega, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) { set_error("bg_batch_sweep: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
    }
    if (stats) {
      stats[4 + 4 * i] = tun[0];
      stats[5 + 4 * i] = tun[1];
      stats[6 + 4 * i] = tun[2];
      stats[7 + 4 * i] = tun[3];
    }
  }
  double t1 = std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
  cudaFree(d_out);
  cudaFreeHost(h_w);
  if (stats) {
    stats[0] = t1 - t0;
    stats[1] = (double)ngeom * nomega;
    stats[2] = use_graph ? 1.0 : 0.0;
    stats[3] = s_capture_failed ? 1.0 : 0.0;
  }
  return st;
}

}  // extern "C"
