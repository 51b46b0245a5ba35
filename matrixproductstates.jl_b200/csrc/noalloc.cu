// prod_AOR without any device allocation.
//
// Who needs this: callers whose device memory is owned by their own pool allocator (a
// Julia CUDA.jl or PyTorch caching allocator that has already reserved nearly all of the
// GPU's memory), or hosts that must not call cudaMalloc / cudaFree inside their time loop
// because those calls synchronise the whole device and can fail under such a pool.  The
// regular entry points keep their scratch in context-owned buffers that grow with
// cudaMalloc; this one keeps the only scratch prod_AOR needs -- the intermediate
// T = A * R -- in a fixed array compiled into the library, and takes a plain CUDA stream
// instead of a context.  The caller still passes every input and the output.
#include <mutex>

#include "common.cuh"
#include "misc.cuh"

namespace mpsb {
namespace {

// Fixed scratch: 16 MiB per device.  Every GPU that loads this library holds it until the
// process exits.  It holds T[chiL*d, wR*chiR0] (complex128), so chiL*d*wR*chiR0 <= 1 Mi elements.
constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(16) << 20;
constexpr int64_t NOALLOC_SCRATCH_ELEMS = NOALLOC_SCRATCH_BYTES / sizeof(cd);
static __device__ __align__(256) cd g_prod_aor_scratch[NOALLOC_SCRATCH_ELEMS];

constexpr int MAX_DEVICES = 128;
std::mutex g_scratch_mu;
cd* g_scratch_addr[MAX_DEVICES] = {};

// The host-side name g_prod_aor_scratch is only a stand-in for the device array; the device
// address is looked up once per device (with that device current) and cached.
int scratch_for_current_device(cd** out) {
  int dev = 0;
  MPSB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= MAX_DEVICES) {
    set_last_message("device ordinal %d outside the no-alloc scratch table", dev);
    return MPSB_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    MPSB_CUDA_TRY(cudaGetSymbolAddress(&p, g_prod_aor_scratch));
    g_scratch_addr[dev] = static_cast<cd*>(p);
  }
  *out = g_scratch_addr[dev];
  return MPSB_OK;
}

}  // namespace
}  // namespace mpsb

using namespace mpsb;

extern "C" int mpsb_op_prod_AOR_noalloc(void* stream, const void* A, const void* O, const void* R, void* AOR,
                                        int chiL, int d, int chiR, int wL, int wR, int chiR0) {
  if (!A || !O || !R || !AOR) return MPSB_ERR_INVALID_ARG;
  if (chiL < 1 || d < 1 || chiR < 1 || wL < 1 || wR < 1 || chiR0 < 1) return MPSB_ERR_DIMENSION;
  const int64_t t_elems = (int64_t)chiL * d * wR * chiR0;
  if (t_elems > NOALLOC_SCRATCH_ELEMS) {
    set_last_message("prod_AOR needs %lld complex elements of scratch (chiL*d*wR*chiR0); the fixed no-alloc "
                     "scratch holds %lld (16 MiB)", (long long)t_elems, (long long)NOALLOC_SCRATCH_ELEMS);
    return MPSB_ERR_UNSUPPORTED;
  }
  cd* T = nullptr;
  MPSB_TRY(scratch_for_current_device(&T));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // T = A(chiL*d x chiR) * R(chiR x wR*chiR0); every element of T is written (beta = 0),
  // so nothing left in the shared array by an earlier call is read
  Gemm g;
  g.M = chiL * d; g.N = wR * chiR0; g.K = chiR;
  g.A = static_cast<const cd*>(A); g.a_m = 1; g.a_k = (int64_t)chiL * d;
  g.B = static_cast<const cd*>(R); g.b_k = 1; g.b_n = chiR;
  g.C = T; g.c_m = 1; g.c_n = (int64_t)chiL * d;
  MPSB_TRY(gemm_launch(g, nullptr, s));
  MpoApply a;
  a.X = chiL; a.Y = chiR0; a.K1 = d; a.K2 = wR; a.M1 = wL; a.M2 = d;
  a.in = T; a.in_x = 1; a.in_k1 = chiL; a.in_k2 = (int64_t)chiL * d; a.in_y = (int64_t)chiL * d * wR;
  a.op = static_cast<const cd*>(O);
  a.out = static_cast<cd*>(AOR); a.out_x = 1; a.out_m1 = chiL; a.out_m2 = (int64_t)chiL * wL;
  a.out_y = (int64_t)chiL * wL * d;
  return mpo_apply_launch_strided(a, (int64_t)wL * d * wR, (int64_t)wL * d, 1, wL, s);
}
