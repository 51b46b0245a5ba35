// Device scratch owned by one context.  Buffers only grow; growth is refused while a CUDA
// graph is being captured (the first, eager call of a step sizes everything).
#pragma once
#include <utility>
#include <vector>

#include "common.cuh"

namespace mpsb {

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

struct Workspace {
  DevBuf splitk;          // split-K partial tiles
  DevBuf qr;              // QR: reflectors, tau, V^H V and T V1^H
  DevBuf svd;             // SVD: the Jacobi working matrix, V, norms, flags
  DevBuf oz;              // sliced tensor-core GEMM: int8 slices of both operands, row exponents
  DevBuf named[16];       // per-sweep temporaries (see engine.cu)
  bool capturing = false;
  // batched calls: a GEMM's split-K partition is chosen from one problem's shape alone (not
  // from the batch's grid), so every copy of a batch computes exactly what the same problem
  // computes in a batch of one
  bool per_problem = false;
  int64_t launches = 0;   // kernel launches issued (eager) or recorded (capture)
  // when set (and not capturing), the sliced GEMM brackets its tensor-core kernel with a pair of
  // CUDA events appended here, so its device time can be read apart from the slicing kernels
  struct TimedLaunch {
    cudaEvent_t start, stop;
    double ops;   // int8 operations of the launch
  };
  std::vector<TimedLaunch>* prof = nullptr;
  // look-ahead lane of the blocked QR (created by its first eager call): a stream, the two events
  // of its fork / join, and the lane's own workspace (its GEMMs' split-K partials)
  cudaStream_t qr_side = nullptr;
  cudaEvent_t qr_ev[2] = {nullptr, nullptr};
  Workspace* qr_side_ws = nullptr;
};

inline void count_launch(Workspace* ws) {
  if (ws) ws->launches++;
}

inline int devbuf_ensure(Workspace* ws, DevBuf& b, size_t bytes) {
  if (bytes <= b.cap) return MPSB_OK;
  if (ws && ws->capturing) {
    set_last_message("workspace growth (%zu bytes) requested during graph capture", bytes);
    return MPSB_ERR_UNSUPPORTED;
  }
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
  size_t want = bytes + bytes / 4 + 4096;
  cudaError_t e = cudaMalloc(&b.p, want);
  if (e != cudaSuccess) {
    set_last_error(e, "cudaMalloc(workspace)", __FILE__, __LINE__);
    return MPSB_ERR_OUT_OF_MEMORY;
  }
  b.cap = want;
  return MPSB_OK;
}

// every device buffer of a workspace, and its QR look-ahead lane (context teardown)
inline void ws_free(Workspace& w) {
  if (w.qr_side) {
    cudaStreamSynchronize(w.qr_side);
    cudaStreamDestroy(w.qr_side);
    w.qr_side = nullptr;
  }
  for (cudaEvent_t& e : w.qr_ev)
    if (e) {
      cudaEventDestroy(e);
      e = nullptr;
    }
  if (w.qr_side_ws) {
    ws_free(*w.qr_side_ws);
    delete w.qr_side_ws;
    w.qr_side_ws = nullptr;
  }
  DevBuf* all[] = {&w.splitk, &w.qr, &w.svd, &w.oz};
  for (DevBuf* b : all) {
    if (b->p) cudaFree(b->p);
    b->p = nullptr;
    b->cap = 0;
  }
  for (DevBuf& b : w.named) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
  }
}

inline int ws_splitk(Workspace* ws, size_t bytes, cd** out) {
  if (!ws) return MPSB_ERR_INVALID_ARG;
  MPSB_TRY(devbuf_ensure(ws, ws->splitk, bytes));
  *out = static_cast<cd*>(ws->splitk.p);
  return MPSB_OK;
}

}  // namespace mpsb
