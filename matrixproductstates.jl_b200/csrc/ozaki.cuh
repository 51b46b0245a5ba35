// Split-precision (int8-sliced, exact int32 accumulation) complex GEMM on tcgen05.
#pragma once
#include "common.cuh"

namespace mpsb {

constexpr int OZ_MIN_SLICES = 3;
constexpr int OZ_MAX_SLICES = 7;

// true when g can run on the sliced tensor-core path with `slices` int8 slices per operand
bool ozgemm_supported(const Gemm& g, int slices);
// device scratch the launch needs (slices of both operands and their row exponents)
size_t ozgemm_scratch_bytes(const Gemm& g, int slices);
// one thread waits `seconds` on an mbarrier nothing arrives on, then sets bit 2 of *err
int wait_probe_launch(double seconds, int* err, cudaStream_t s);
// C = alpha op(A) op(B) + beta C with each operand split into `slices` int8 slices; `err`
// (device word, may be null) gets bit 1 when a bounded wait inside the kernel runs out
int ozgemm_launch(const Gemm& g, int slices, void* scratch, size_t scratch_bytes, int* err, Workspace* ws,
                  cudaStream_t s);

}  // namespace mpsb
