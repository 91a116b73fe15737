// Context of the west_b200 library (shared by the translation units that
// drive it).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/west_b200.h"
#include "wb_internal.h"

namespace wb {

// Records the message of a failed call (wb_last_error) and returns code.
int fail(int code, const std::string& msg);

#define WB_CU(call)                                                                            \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return ::wb::fail(WB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Grow-only device buffer.
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int ensure(size_t b) {
    if (b <= bytes) return 0;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    if (cudaMalloc(&p, b) != cudaSuccess) {
      cudaGetLastError();
      return -1;
    }
    bytes = b;
    return 0;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

}  // namespace wb

// The opaque handle of the C ABI.
struct wb_ctx {
  using DBuf = wb::DBuf;
  int device = 0;
  cudaStream_t stream = nullptr;
  int npw = 0, nr = 0, nnr = 0, nocc = 0, nkb = 0, nproj = 0, npv = 0;
  int maxiter = 0, kinetic_only = 0, precision = WB_PRECISION_FP64, batch_cap = 0;
  int nfull = 0;             // fully occupied bands (nbnd_occ_full); nocc - nfull fractional ones
  int nz = 0;                // stick length (box edge along z)
  int rt = 0;                // 1: runtime-size FFT path (no compiled kernels for this box)
  wb::RtGeo geo{};           // its geometry (radix plans, active columns, twiddle tables)
  DBuf rt_colx, twx, twy, twz, twx32, twy32, twz32;
  double omega = 0, wk = 0, alpha = 0;
  wb::StickTab st{};
  wb::FftArgs fa{};
  // constant device data
  DBuf perm, gqz, spg, stpos, tw, g2kin, sqvc, vs, evc, W, D, eprec, et, occ, evcr, iprec;
  // per-call workspace
  DBuf dvg_in, dng_out, aux, dvbox, B, X, G, T, sticks, sticks2, acc, part, C, rho, conv, act, items, nact,
      ecol, epcol, unconv, items_pp, items_pk, iota_items, fcoef;
  int* nact_host = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  wb_stats stats{};
  // stage profiling: event pairs recorded on the stream, resolved after the call
  int prof = 0;
  std::vector<cudaEvent_t> evpool;
  size_t evused = 0;
  struct Mark { int stage, e0, e1; };
  std::vector<Mark> marks;
  // mixed form: FP32 constants (made on first use) and workspace
  int have32 = 0;
  wb::FftArgs32 fa32{};
  DBuf W32, D32, g2kin32, vs32, tw32, g32, P32, T32, d32, sticks32, part32, C32, ecol32, rho0, rho_in, conv_in,
      act_in, items_in, nact_in;
  // CUDA graphs of the PCG loops: one conditional WHILE node whose body is one
  // masked PCG pass; rebuilt when a buffer, the batch or tr2 changes
  struct LoopGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<const void*> key;
    double tr2 = 0.0;
    void release() {
      if (exec) cudaGraphExecDestroy(exec);
      if (graph) cudaGraphDestroy(graph);
      exec = nullptr;
      graph = nullptr;
      key.clear();
    }
  };
  // two graphs per form: a Davidson alternates tr2 (1e-4 in its extra starting
  // step, tr2_dfpt in its iterations), and re-instantiating the graph at each
  // change cost tens of ms per solve
  struct LoopCache {
    LoopGraph slot[2];
    int last = 0;  // the slot of the latest capture or hit
    cudaGraphExec_t cur() const { return slot[last].exec; }
    void release() {
      slot[0].release();
      slot[1].release();
    }
  };
  LoopCache loop64, loop32;
  int use_graphs = 1;
  int cap_nsys = 0;          // systems the per-call workspace is sized for (grow-only)
  // autotuned launch shapes (set on the first batch of each form, then fixed)
  struct Tune {
    int on = 1, done64 = 0, done32 = 0;
    int dmma_ctas = 2, dmma_pf = 1, umma_ctas = 2, update_nj = 0, unfused64 = 0, unfused32 = 0;
    float ms = 0.f;
  } tune;
  cudaEvent_t tev0 = nullptr, tev1 = nullptr;
  cudaEvent_t wait_ev = nullptr;  // blocking-sync event of the calls' waits (wb_wait)
  // pinned staging of a batch's small host transfers (unconverged counts, item
  // tables): copies from or to pageable memory would wait for the stream by
  // spinning, ahead of the blocking wait
  unsigned char* pin = nullptr;
  size_t pin_bytes = 0;
  int ensure_pin(size_t b) {
    if (b <= pin_bytes) return 0;
    if (pin) cudaFreeHost(pin);
    pin = nullptr;
    pin_bytes = 0;
    if (cudaMallocHost(&pin, b) != cudaSuccess) {
      cudaGetLastError();
      return -1;
    }
    pin_bytes = b;
    return 0;
  }
  DBuf loopst;               // int[8] loop state (wb_la.cu loop_init / loop_ctl)
  int* loop_host = nullptr;  // pinned copy of it
  int loop_pending = 0;      // launches per pass of a graph run whose counters await the batch's wait
  // tensor-core GEMMs of the mixed form: W split into bf16 hi/lo tiles, and the
  // error word their bounded waits write
  int umma = 0, umma_M = 0;
  DBuf umma_braket_w, umma_update_w, umma_err;
  // PDEP Davidson state (wb_davidson)
  DBuf dav_dvg, dav_dng, dav_tmp, dav_hr, dav_vr, dav_A, dav_V, dav_w, dav_part, dav_coef, dav_dots, dav_bj;
  wb_apply_fn dav_apply = nullptr;  // operator hook of the Davidson (wb_davidson_set_apply)
  void* dav_apply_user = nullptr;
  // the Davidson's dense steps as CUDA graphs, one executable per phase, basis
  // size, batch size and buffer set, most recently used first; dav_st holds the
  // iteration's device state (unconverged count, conv flags, eigenvalues) and
  // dav_host its pinned copy
  struct DavGraph {
    std::vector<long long> key;
    cudaGraphExec_t exec = nullptr;
  };
  std::vector<DavGraph> dav_graphs;
  DBuf dav_st;
  cudaStream_t dav_aux = nullptr;  // second stream for captures that add conditional nodes
  cudaEvent_t dav_ev[2] = {nullptr, nullptr};  // timing of a deferred operator call
  void* dav_host = nullptr;
  size_t dav_host_bytes = 0;
  void dav_graphs_release() {
    for (DavGraph& g : dav_graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    dav_graphs.clear();
  }
  // device address of the allocation-free entry point's scratch array, looked
  // up on this context's first such call (null until then)
  void* noalloc_base = nullptr;
  int ev_get() {
    if (evused == evpool.size()) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return -1;
      evpool.push_back(e);
    }
    return (int)evused++;
  }
};

// Waits for the context's stream through a blocking-sync event: the calling
// thread sleeps until the GPU signals instead of spinning on a core.  A thread
// that spins through a wait on a host whose cores other processes keep busy
// loses its time slices, and every slice it waits for leaves the GPU idle
// before the next launch: c1 Davidson solves beside 32 busy processes took
// 72-108 ms (medians of two runs) with spinning waits, 45-54 ms with sleeping
// ones; on an idle host the wake-ups cost 1-5 ms of a 40 ms solve.  (Polling the
// event for half a millisecond before sleeping did worse under load.)
inline cudaError_t wb_wait(wb_ctx* c) {
  if (!c->wait_ev) return cudaStreamSynchronize(c->stream);
  const cudaError_t e = cudaEventRecord(c->wait_ev, c->stream);
  return e == cudaSuccess ? cudaEventSynchronize(c->wait_ev) : e;
}

namespace wb {
// apply_operator on device buffers for the Davidson: when *deferred comes back
// true the batch is only enqueued and the caller, after waiting on ctx's
// stream, calls apply_settle; otherwise the call completed as usual.
int apply_deferred(wb_ctx* c, int m, const double* dvg, int ld_dvg, double* dng, int ld_dng, double tr2,
                   bool* deferred);
void apply_settle(wb_ctx* c);
}  // namespace wb
