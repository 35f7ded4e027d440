// LOBPCG on the device (filled in below the stubs as the solver lands).
#include "qdkp_common.cuh"

using namespace qdkp;

extern "C" {

size_t qdkp_lobpcg_workspace_size(const qdkp_operator* op, const qdkp_lobpcg_params* prm) {
  (void)op; (void)prm;
  return 0;
}

int qdkp_lobpcg_solve(const qdkp_operator* op, const qdkp_lobpcg_params* prm, const void* X0,
                      double* lambda, void* V, double* resid_history, qdkp_lobpcg_info* info,
                      void* ws, size_t ws_bytes, void* stream) {
  set_error("qdkp_lobpcg_solve: not built yet");
  return QDKP_ERR_UNSUPPORTED;
}

size_t qdkp_residuals_workspace_size(const qdkp_operator* op, int k) { return 0; }

int qdkp_residuals(const qdkp_operator* op, const void* V, int64_t ldv, int k,
                   const double* E_in, double* rq, double* res, void* ws, size_t ws_bytes,
                   void* stream) {
  set_error("qdkp_residuals: not built yet");
  return QDKP_ERR_UNSUPPORTED;
}

}  // extern "C"
