// The early-exit iteration loop as one CUDA graph.
//
// A conditional WHILE node holds the body: every launch of one iteration
// followed by a one-thread step kernel that advances the device iteration
// counter and sets the loop condition to (changed != 0 && it < stop).  The
// kernels read their buffer parity and changed-counter slot from the device
// counter, so one captured body serves every iteration and every run; it is
// rebuilt only when the dispatch plan changes.
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "runtime.h"

namespace {

__global__ void k_loop_step(uint32_t *loop, const unsigned long long *changed, cudaGraphConditionalHandle cond) {
  // loop[0]: iteration counter, loop[1]: stop value, loop[2]: stop when nothing changed
  const uint32_t it = loop[0] + 1u;
  loop[0] = it;
  const bool go = (loop[2] == 0u || changed[it - 1] != 0ull) && it < loop[1];
  cudaGraphSetConditional(cond, go ? 1u : 0u);
}

void destroy_graph(lpa_handle *h) {
  if (h->graph_exec) cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(h->graph_exec));
  if (h->graph) cudaGraphDestroy(static_cast<cudaGraph_t>(h->graph));
  h->graph_exec = nullptr;
  h->graph = nullptr;
}

cudaError_t build_graph(lpa_handle *h) {
  destroy_graph(h);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e != cudaSuccess) return e;
  cudaGraphConditionalHandle cond;
  e = cudaGraphConditionalHandleCreate(&cond, g, 1u, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return e;
  }
  cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = cond;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  e = cudaGraphAddNode(&node, g, nullptr, 0, &p);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return e;
  }
  cudaGraph_t body = p.conditional.phGraph_out[0];
  e = cudaStreamBeginCaptureToGraph(h->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return e;
  }
  const int saved_cur = h->cur;
  const int saved_timings = h->opts.record_timings;
  h->cur = 0;
  h->opts.record_timings = 0;
  h->loop_it = h->d_loop_it;
  const uint64_t launches = h->launches;
  lpa_rt_enqueue_iteration(h, h->d_changed, h->d_work);
  h->launches_per_graph_iteration = h->launches - launches + 1;
  h->launches = launches;
  k_loop_step<<<1, 1, 0, h->stream>>>(h->d_loop_it, h->d_changed, cond);
  h->loop_it = nullptr;
  h->cur = saved_cur;
  h->opts.record_timings = saved_timings;
  cudaGraph_t captured = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(h->stream, &captured);
  if (e2 != cudaSuccess) {
    cudaGraphDestroy(g);
    return e2;
  }
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiate(&exec, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return e;
  }
  h->graph = g;
  h->graph_exec = exec;
  h->graph_plan_version = h->plan_version;
  return cudaSuccess;
}

}  // namespace

void lpa_rt_destroy_graph(lpa_handle *h) { destroy_graph(h); }

lpa_status lpa_run_graph(lpa_handle *h, int max_iter, bool early_exit, int *iters_done) {
  if (max_iter == 0) return LPA_OK;
  if (max_iter + 2 > h->changed_slots) {
    h->last_error = "max_iter exceeds the changed-counter slots";
    return LPA_ERR_INVALID_ARG;
  }
  auto fail = [&](cudaError_t e, const char *where) {
    h->last_error = std::string(where) + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? LPA_ERR_OOM : LPA_ERR_CUDA;
  };
  cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess) return fail(e, "cudaSetDevice");
  if (!h->d_loop_it) {
    e = cudaMalloc(&h->d_loop_it, 4 * sizeof(uint32_t));
    if (e != cudaSuccess) return fail(e, "loop counter");
    h->allocations.push_back(h->d_loop_it);
  }
  if (!h->graph_exec || h->graph_plan_version != h->plan_version) {
    e = build_graph(h);
    if (e != cudaSuccess) return fail(e, "build iteration graph");
  }
  const uint32_t start = uint32_t(h->cur);
  uint32_t *ctl = reinterpret_cast<uint32_t *>(h->h_pinned);
  ctl[0] = start;
  ctl[1] = start + uint32_t(max_iter);
  ctl[2] = early_exit ? 1u : 0u;
  e = cudaMemsetAsync(h->d_changed, 0, size_t(max_iter + 2) * sizeof(unsigned long long), h->stream);
  if (e != cudaSuccess) return fail(e, "clear counters");
  e = cudaMemsetAsync(h->d_work, 0, size_t(lpa_dev::kWorkCounters) * size_t(max_iter + 2) * sizeof(uint32_t), h->stream);
  if (e != cudaSuccess) return fail(e, "clear work counters");
  e = cudaMemcpyAsync(h->d_loop_it, ctl, 3 * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream);
  if (e != cudaSuccess) return fail(e, "loop control");
  e = cudaGraphLaunch(static_cast<cudaGraphExec_t>(h->graph_exec), h->stream);
  if (e != cudaSuccess) return fail(e, "graph launch");
  uint32_t it_end = 0;
  e = cudaMemcpyAsync(&it_end, h->d_loop_it, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream);
  if (e != cudaSuccess) return fail(e, "read loop counter");
  std::vector<unsigned long long> hist(size_t(max_iter) + 2);
  e = cudaMemcpyAsync(hist.data(), h->d_changed, hist.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                      h->stream);
  if (e != cudaSuccess) return fail(e, "read counters");
  lpa_status st = lpa_rt_take_error(h);  // synchronises
  if (st != LPA_OK) return st;
  const uint32_t done = it_end - start;
  for (uint32_t i = 0; i < done; i++) h->history.push_back(hist[start + i]);
  h->iterations += done;
  h->launches += uint64_t(done) * h->launches_per_graph_iteration;
  if (done) h->last_changed = hist[start + done - 1];
  h->cur = int(it_end & 1u);
  if (iters_done) *iters_done = int(done);
  return LPA_OK;
}
