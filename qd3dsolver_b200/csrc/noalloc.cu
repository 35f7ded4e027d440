// Allocation-free folded apply: Y = (H - sigma)^2 X with the intermediate (H - sigma) X kept
// in a fixed device array compiled into the library instead of a caller workspace.
//
// Who needs this: code that must not allocate device memory at the moment it applies the
// operator -- a host language binding with no device allocator of its own (a C or Fortran
// caller handing over only X and Y), a real-time or callback context where cudaMalloc's
// implicit device synchronisation is not allowed, or a caller whose allocator is owned by
// another runtime. qdkp_apply needs the caller to provide n*m scratch elements for the folded
// mode; this entry point needs nothing beyond X and Y.
//
// Cost: every GPU that loads libqdkp.so holds the array (QDKP_NOALLOC_SCRATCH_BYTES) until the
// process exits, whether or not this entry point is used.
#include <mutex>

#include "qdkp_common.cuh"

namespace qdkp {

int launch_apply(const qdkp_operator* op, const void* X, int64_t ldx, void* Y, int64_t ldy,
                 int m, double sigma, int shifted, int precision, cudaStream_t st);

// The scratch: one folded intermediate of at most QDKP_NOALLOC_SCRATCH_BYTES.
static __device__ __align__(256) unsigned char g_fold_scratch[QDKP_NOALLOC_SCRATCH_BYTES];

// In host code `g_fold_scratch` names a host-side shadow, not device memory; its device
// address is looked up once per device with that device current and cached here.
static std::mutex g_scratch_mu;
static void* g_scratch_ptr[64] = {nullptr};

static int scratch_address(int device, void** out) {
  if (device < 0 || device >= 64) { set_error("device ordinal out of range"); return QDKP_ERR_ARG; }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    QDKP_CUDA_TRY(cudaGetSymbolAddress(&p, g_fold_scratch));
    g_scratch_ptr[device] = p;
  }
  *out = g_scratch_ptr[device];
  return QDKP_OK;
}

}  // namespace qdkp

using namespace qdkp;

extern "C" {

size_t qdkp_apply_folded_noalloc_max_elems(int precision) {
  if (precision == QDKP_C128) return QDKP_NOALLOC_SCRATCH_BYTES / 16;
  if (precision == QDKP_C64) return QDKP_NOALLOC_SCRATCH_BYTES / 8;
  return 0;
}

int qdkp_apply_folded_noalloc(const qdkp_operator* op, const void* X, int64_t ldx, void* Y,
                              int64_t ldy, int m, double sigma, int precision, void* stream) {
  QDKP_CHECK_ARG(op != nullptr && X != nullptr && Y != nullptr, "NULL operator or block");
  QDKP_CHECK_ARG(m > 0 && ldx >= m && ldy >= m, "need m > 0 and leading dimensions >= m");
  QDKP_CHECK_ARG(precision == QDKP_C128 || precision == QDKP_C64, "bad precision");
  const int64_t n = (int64_t)op->n_bands * op->n_sites;
  const size_t need = (size_t)n * (size_t)m;
  if (need > qdkp_apply_folded_noalloc_max_elems(precision)) {
    set_error("qdkp_apply_folded_noalloc: n * m = " + std::to_string(need) +
              " complex elements exceed the fixed scratch of " +
              std::to_string((unsigned long long)QDKP_NOALLOC_SCRATCH_BYTES) +
              " bytes; use qdkp_apply with a caller workspace");
    return QDKP_ERR_WORKSPACE;
  }
  // the operator's device is made current for the call and the caller's current device is
  // restored on every return path
  int prev = -1;
  QDKP_CUDA_TRY(cudaGetDevice(&prev));
  if (prev != op->device) QDKP_CUDA_TRY(cudaSetDevice(op->device));
  void* T = nullptr;
  int rc = scratch_address(op->device, &T);
  if (rc == QDKP_OK) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // Every element of T that the second launch reads is written by the first one in this
    // call, so nothing left over from an earlier call is ever read and nothing needs clearing.
    rc = launch_apply(op, X, ldx, T, m, m, sigma, 1, precision, st);
    if (rc == QDKP_OK) rc = launch_apply(op, T, m, Y, ldy, m, sigma, 1, precision, st);
  }
  if (prev != op->device) cudaSetDevice(prev);
  return rc;
}

}  // extern "C"
