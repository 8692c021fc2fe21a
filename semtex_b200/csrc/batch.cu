// Many independent direct solves replayed as one CUDA graph.
//
// The reference runs one problem per `elliptic` process (elliptic/drive.cpp:
// 61-96, one Field::solve each).  Problems of a few hundred to a few thousand
// unknowns each leave a B200 nearly idle, and issuing their kernels one call
// at a time leaves it waiting on the host.  stx_batch_create captures the
// whole set once -- each system's Field::solve on its own context stream,
// forked from and joined back into the batch stream -- and stx_batch_launch
// replays it with a single graph launch: every problem's kernels are nodes of
// one graph, independent problems are parallel branches.
#include <cuda_runtime.h>

#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/semtex_b200.h"
#include "stx_internal.hpp"

struct stx_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int nsystems = 0;
  int kernel_nodes = 0;
};

namespace {

struct BatchError : std::runtime_error {
  int code;
  BatchError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw BatchError(STX_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class F>
int batch_guarded(F&& f) {
  try {
    f();
    stx::set_last_error("");
    return STX_OK;
  } catch (const BatchError& e) {
    stx::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    stx::set_last_error(e.what());
    return STX_ECUDA;
  }
}

void release(stx_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  b->exec = nullptr;
  b->graph = nullptr;
  b->stream = nullptr;
}

}  // namespace

extern "C" {

int stx_batch_create(stx_modal* const* systems, const double* const* d_forcing, double* const* d_unknown,
                     int n, void* stream, stx_batch** out) {
  stx_batch* b = nullptr;
  std::vector<cudaEvent_t> ev;
  bool capturing = false;
  const int rc = batch_guarded([&] {
    if (!systems || !d_forcing || !d_unknown || !out || n < 1) throw BatchError(STX_EINVAL, "bad argument");
    *out = nullptr;
    const int device = systems[0] ? systems[0]->ctx->device : 0;
    for (int i = 0; i < n; ++i) {
      if (!systems[i] || !d_forcing[i] || !d_unknown[i]) throw BatchError(STX_EINVAL, "null system or buffer");
      if (systems[i]->method == STX_JACPCG) throw BatchError(STX_EINVAL, "batched solves are DIRECT or MIXED");
      if (systems[i]->ctx->device != device) throw BatchError(STX_EINVAL, "systems on different devices");
    }
    ck(cudaSetDevice(device), "cudaSetDevice");
    // one solve of each outside the capture: workspaces and one-time kernel
    // attributes are set up here, so that the capture only records work
    std::set<cudaStream_t> streams;
    for (int i = 0; i < n; ++i) {
      const int r = stx_field_solve(systems[i], d_forcing[i], d_unknown[i], 0.0, 0, nullptr);
      if (r != STX_OK) throw BatchError(r, std::string("warm-up solve: ") + stx_last_error());
      streams.insert(systems[i]->ctx->stream);
    }
    for (cudaStream_t s : streams) ck(cudaStreamSynchronize(s), "warm-up sync");
    b = new stx_batch();
    b->device = device;
    b->nsystems = n;
    if (stream) {
      b->stream = static_cast<cudaStream_t>(stream);
    } else {
      ck(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream");
      b->own_stream = true;
    }
    ev.resize(n + 1);
    for (auto& e : ev) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    ck(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    capturing = true;
    ck(cudaEventRecord(ev[0], b->stream), "fork");
    for (int i = 0; i < n; ++i) {
      cudaStream_t s = systems[i]->ctx->stream;
      ck(cudaStreamWaitEvent(s, ev[0], 0), "fork wait");
      const int r = stx_field_solve(systems[i], d_forcing[i], d_unknown[i], 0.0, 0, nullptr);
      if (r != STX_OK) throw BatchError(r, std::string("captured solve: ") + stx_last_error());
      ck(cudaEventRecord(ev[i + 1], s), "join");
      ck(cudaStreamWaitEvent(b->stream, ev[i + 1], 0), "join wait");
    }
    capturing = false;
    ck(cudaStreamEndCapture(b->stream, &b->graph), "end capture");
    ck(cudaGraphInstantiate(&b->exec, b->graph, 0), "instantiate");
    size_t nn = 0;
    ck(cudaGraphGetNodes(b->graph, nullptr, &nn), "graph nodes");
    std::vector<cudaGraphNode_t> nodes(nn);
    ck(cudaGraphGetNodes(b->graph, nodes.data(), &nn), "graph nodes");
    for (auto nd : nodes) {
      cudaGraphNodeType t;
      ck(cudaGraphNodeGetType(nd, &t), "node type");
      if (t == cudaGraphNodeTypeKernel) ++b->kernel_nodes;
    }
    *out = b;
  });
  if (capturing && b) {  // leave no stream in capture mode after a failure
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(b->stream, &g);
    if (g) cudaGraphDestroy(g);
  }
  for (auto e : ev)
    if (e) cudaEventDestroy(e);
  if (rc != STX_OK && b) {
    release(b);
    delete b;
  }
  return rc;
}

int stx_batch_launch(stx_batch* b) {
  return batch_guarded([&] {
    if (!b || !b->exec) throw BatchError(STX_EINVAL, "null batch");
    ck(cudaSetDevice(b->device), "cudaSetDevice");
    ck(cudaGraphLaunch(b->exec, b->stream), "graph launch");
  });
}

int stx_batch_info(const stx_batch* b, int* nsystems, int* kernel_nodes, void** stream) {
  return batch_guarded([&] {
    if (!b) throw BatchError(STX_EINVAL, "null batch");
    if (nsystems) *nsystems = b->nsystems;
    if (kernel_nodes) *kernel_nodes = b->kernel_nodes;
    if (stream) *stream = b->stream;
  });
}

int stx_batch_destroy(stx_batch* b) {
  return batch_guarded([&] {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    release(b);
    delete b;
  });
}

}  // extern "C"
