// Shared device/host helpers for the qdkp library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/qdkp.h"

struct qdkp_operator;

namespace qdkp {

// ---------------------------------------------------------------------------------------------
// Complex arithmetic on the CUDA vector types (interleaved re, im: the numpy complex layout).
// ---------------------------------------------------------------------------------------------
template <typename T> struct cvec;
template <> struct cvec<double> { typedef double2 type; };
template <> struct cvec<float> { typedef float2 type; };
template <typename T> using cplx = typename cvec<T>::type;

template <typename T> __host__ __device__ __forceinline__ cplx<T> mk(T re, T im) {
  cplx<T> z; z.x = re; z.y = im; return z;
}
template <typename T> __host__ __device__ __forceinline__ cplx<T> czero() { return mk<T>(T(0), T(0)); }

// Overloads for double2 / float2 (cplx<T> is a non-deduced alias, so these are not templates).
#define QDKP_CPLX_OPS(C, R)                                                                    \
  __host__ __device__ __forceinline__ C cadd(C a, C b) { C z; z.x = a.x + b.x; z.y = a.y + b.y; return z; } \
  __host__ __device__ __forceinline__ C csub(C a, C b) { C z; z.x = a.x - b.x; z.y = a.y - b.y; return z; } \
  __host__ __device__ __forceinline__ C cmul(C a, C b) {                                        \
    C z; z.x = a.x * b.x - a.y * b.y; z.y = a.x * b.y + a.y * b.x; return z; }                 \
  /* conj(a) * b */                                                                           \
  __host__ __device__ __forceinline__ C cmulc(C a, C b) {                                       \
    C z; z.x = a.x * b.x + a.y * b.y; z.y = a.x * b.y - a.y * b.x; return z; }                 \
  __host__ __device__ __forceinline__ C cscale(R s, C a) { C z; z.x = s * a.x; z.y = s * a.y; return z; } \
  /* acc += s a (s real) */                                                                   \
  __host__ __device__ __forceinline__ void caxpy(C& acc, R s, C a) {                            \
    acc.x = fma(s, a.x, acc.x); acc.y = fma(s, a.y, acc.y); }                                  \
  /* acc += i s a */                                                                          \
  __host__ __device__ __forceinline__ void caxpy_i(C& acc, R s, C a) {                          \
    acc.x = fma(-s, a.y, acc.x); acc.y = fma(s, a.x, acc.y); }                                 \
  /* acc += c a */                                                                            \
  __host__ __device__ __forceinline__ void cfma(C& acc, C c, C a) {                             \
    acc.x = fma(c.x, a.x, acc.x); acc.x = fma(-c.y, a.y, acc.x);                               \
    acc.y = fma(c.x, a.y, acc.y); acc.y = fma(c.y, a.x, acc.y); }                              \
  /* acc += conj(c) a */                                                                      \
  __host__ __device__ __forceinline__ void cfmac(C& acc, C c, C a) {                            \
    acc.x = fma(c.x, a.x, acc.x); acc.x = fma(c.y, a.y, acc.x);                                \
    acc.y = fma(c.x, a.y, acc.y); acc.y = fma(-c.y, a.x, acc.y); }
QDKP_CPLX_OPS(double2, double)
QDKP_CPLX_OPS(float2, float)
#undef QDKP_CPLX_OPS

// ---------------------------------------------------------------------------------------------
// Error handling: every entry point returns an int status and records a message.
// ---------------------------------------------------------------------------------------------
void set_error(const std::string& msg);
// Counts kernel launches made by this library (qdkp_kernel_launches).
void count_launch(int n = 1);
long long launches_so_far();

#define QDKP_CUDA_TRY(expr)                                                              \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess) {                                                             \
      ::qdkp::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));              \
      return QDKP_ERR_CUDA;                                                              \
    }                                                                                    \
  } while (0)

#define QDKP_CHECK_ARG(cond, msg)                                                        \
  do {                                                                                   \
    if (!(cond)) { ::qdkp::set_error(msg); return QDKP_ERR_ARG; }                        \
  } while (0)

// Per-site coefficient fields, structure of arrays: field f of site s at fields[f * N + s].
enum FieldIndex {
  F_G1 = 0, F_G2, F_G3, F_P0, F_EC, F_EV, F_DSO, F_B, F_D,
  F_EXX, F_EYY, F_EZZ, F_EXY, F_EYZ, F_EZX, F_COUNT
};

constexpr double kG = 0.0380998;   // hbar^2 / 2 m0 in eV nm^2 (qdsolver_core.py:19)

// One operator/block pair of a multi-slot H.X launch (eight bands).
struct HXSlot {
  const void* rec;        // operator record in the launch precision
  const unsigned* msk;    // neighbour masks of the operator's sites
  const void* X;
  void* Y;
  int N, ldx, ldy;        // sites; leading dimensions (unused when ld_same)
  int sx, sy;             // site strides of x and y (ny nz, nz)
  int tile0;              // first CTA of this slot in the launch
  int m;                  // column count if m_dev is NULL
  const int* m_dev;       // device column count (active width), or NULL
  const int* skip;        // nonzero: slot idle this tick
  int ld_same;            // leading dimensions equal the column count
  int nzp, NP;            // padded z extent of the record and its entry stride
  int shifted;
  double sigma;
  double cb;              // conduction-band face weight (apply_cb_weight)
};

int launch_apply_multi(const HXSlot* slots_dev, int nslots, int total_tiles, int precision,
                       cudaStream_t st);
// CTAs one H.X launch uses for n_sites x m items
int apply_tiles(int64_t n_sites, int m);
double apply_cb_weight(const qdkp_operator* op);
// (re)build the per-site stencil record and neighbour masks from fields64
int build_records(qdkp_operator* op);
size_t record_doubles(int nx, int ny, int nzp);

}  // namespace qdkp

// The operator handle (opaque to C callers).
struct qdkp_operator {
  int nx, ny, nz;
  int64_t n_sites;
  double h;
  int n_bands;            // 8, 6 or 4
  int flags;              // QDKP_* flags
  int device;
  double* fields64;       // device, F_COUNT * n_sites doubles (library-owned)
  int nzp;                // nz rounded up to a multiple of 4 (record rows)
  double* rec64;          // device, per-site stencil record (FP64), record_doubles(nx, ny, nzp)
  float* rec32;           // the same record in FP32
  unsigned* nbmask;       // device, per-site neighbour mask
  int staged_cfg[2];      // staged H.X tile shape per precision (c128, c64); -1 = by heuristic
  int64_t nnz_equiv;      // CSR nonzero count of the equivalent assembled matrix
};
