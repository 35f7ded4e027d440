// Tall-skinny block kernels (norms, residual gather, Gram, block update) and one-CTA FP64
// small dense kernels (Cholesky + triangular inverse, Hermitian generalized eigensolver by
// Householder reduction and implicit QL) for the LOBPCG driver.
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>
#include <cstdlib>
#include <cstring>

#include "dense_dev.cuh"
#include "umma_dev.cuh"

namespace qdkp {

// ------------------------------------------------------------------------------------------------
// Column norms: out[j] = sum_r |A[r, j] - lambda_j B[r, j]|^2 (B may be NULL).
// ------------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kTallThreads)
colnorm2_partial(const cplx<T>* __restrict__ A, long long lda, const cplx<T>* __restrict__ B,
                 long long ldb, const double* __restrict__ lam, int m, long long n,
                 double* __restrict__ partial) {
  double acc[kMaxBlock];
#pragma unroll
  for (int j = 0; j < kMaxBlock; ++j) acc[j] = 0.0;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int j = 0; j < kMaxBlock; ++j) {
      if (j < m) {
        const cplx<T> av = A[r * lda + j];
        double2 a = make_double2((double)av.x, (double)av.y);
        if (B) {
          const cplx<T> b = B[r * ldb + j];
          a.x -= lam[j] * (double)b.x;
          a.y -= lam[j] * (double)b.y;
        }
        acc[j] = fma(a.x, a.x, fma(a.y, a.y, acc[j]));
      }
    }
  }
  __shared__ double red[kTallThreads / 32][kMaxBlock];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < kMaxBlock; ++j) {
    if (j < m) {
      double v = acc[j];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp][j] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x < m) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][threadIdx.x];
    partial[(long long)blockIdx.x * m + threadIdx.x] = s;
  }
}

__global__ void reduce_partials(const double* __restrict__ partial, int nparts, int m,
                                double* __restrict__ out) {
  const int j = threadIdx.x;
  if (j < m) {
    double s = 0.0;
    for (int b = 0; b < nparts; ++b) s += partial[(long long)b * m + j];
    out[j] = s;
  }
}

template <typename T>
int launch_colnorm2(const cplx<T>* A, long long lda, const cplx<T>* B, long long ldb,
                    const double* lambda, int m, long long n, double* partial, int nparts,
                    double* out, cudaStream_t st) {
  if (m > kMaxBlock) { set_error("block wider than kMaxBlock"); return QDKP_ERR_ARG; }
  colnorm2_partial<T><<<nparts, kTallThreads, 0, st>>>(A, lda, B, ldb, lambda, m, n, partial);
  count_launch();
  reduce_partials<<<1, 32, 0, st>>>(partial, nparts, m, out);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

// ------------------------------------------------------------------------------------------------
// R[:, c] = AX[:, idx[c]] - lambda[idx[c]] X[:, idx[c]]   (active residual columns, compacted)
// ------------------------------------------------------------------------------------------------
__global__ void resid_gather_kernel(const double2* __restrict__ AX, long long ldax,
                                    const double2* __restrict__ X, long long ldx,
                                    const double* __restrict__ lam, const int* __restrict__ idx,
                                    int ma, long long n, double2* __restrict__ R, long long ldr) {
  const long long total = n * ma;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / ma;
    const int c = (int)(e - r * ma);
    const int j = idx[c];
    const double l = lam[j];
    const double2 a = AX[r * ldax + j], x = X[r * ldx + j];
    R[r * ldr + c] = make_double2(a.x - l * x.x, a.y - l * x.y);
  }
}

int launch_resid_gather(const double2* AX, long long ldax, const double2* X, long long ldx,
                        const double* lambda, const int* idx, int ma, long long n, double2* R,
                        long long ldr, cudaStream_t st) {
  resid_gather_kernel<<<1184, 256, 0, st>>>(AX, ldax, X, ldx, lambda, idx, ma, n, R, ldr);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

template <typename TS, typename TD>
__global__ void gather_kernel(const cplx<TS>* __restrict__ src, long long lds,
                              const int* __restrict__ idx, int ma, long long n,
                              cplx<TD>* __restrict__ dst, long long ldd) {
  const long long total = n * ma;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / ma;
    const int c = (int)(e - r * ma);
    const cplx<TS> v = src[r * lds + (idx ? idx[c] : c)];
    dst[r * ldd + c] = mk<TD>((TD)v.x, (TD)v.y);
  }
}

template <typename TS, typename TD>
int launch_gather(const cplx<TS>* src, long long lds, const int* idx, int ma, long long n,
                  cplx<TD>* dst, long long ldd, cudaStream_t st) {
  gather_kernel<TS, TD><<<1184, 256, 0, st>>>(src, lds, idx, ma, n, dst, ldd);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

template <typename TS, typename TD>
int launch_copy(const cplx<TS>* src, long long lds, int cols, long long n, cplx<TD>* dst,
                long long ldd, cudaStream_t st) {
  if (std::is_same<TS, TD>::value && lds == cols && ldd == cols) {
    QDKP_CUDA_TRY(cudaMemcpyAsync(dst, src, (size_t)n * cols * sizeof(cplx<TD>),
                                  cudaMemcpyDeviceToDevice, st));
    return QDKP_OK;
  }
  return launch_gather<TS, TD>(src, lds, nullptr, cols, n, dst, ldd, st);
}

// ------------------------------------------------------------------------------------------------
// Gram: out = A^H B over concatenated column lists, FP64 accumulation, deterministic.
// ------------------------------------------------------------------------------------------------
constexpr int kGramParts = 296;

// The complex product A^H B is one real GEMM over the interleaved (re, im) view: with
// A' (n x 2P) and B' (n x 2Q) the real views, C' = A'^T B' and
//   Re G_ij = C'_{2i,2j} + C'_{2i+1,2j+1},   Im G_ij = C'_{2i,2j+1} - C'_{2i+1,2j}.
// C' is accumulated on the FP64 tensor cores (mma.sync.m8n8k4.f64; the tcgen05 family has no
// f64 kind). A CTA of 3 x 3 warps owns all 8x8 tiles of C' for its slice of rows; each warp
// owns a rectangle of up to 6 x 6 tiles and keeps them in registers across the slice.

constexpr int kGramSplit = 16;

// A CTA per (row part, column panel): its partial of C', then the last CTAs reduce the
// partials into `result` (gram_finish_last; `counters`: kGramSplit + 1 zeroed ints)
template <int MR, int MC, typename T>
__global__ void __launch_bounds__(512)
gram_partial_kernel(const BlockList<T> A, const BlockList<T> B, long long n,
                    long long rows_per_part, double* __restrict__ partial, int ptc,
                    int* __restrict__ counters, double2* __restrict__ result) {
  extern __shared__ __align__(16) unsigned char gsm_d[];
  const int RP = (2 * A.total() + 7) / 8 * 8, RQ = (2 * B.total() + 7) / 8 * 8;
  const long long r0 = blockIdx.x * rows_per_part;
  double* out = partial + (long long)blockIdx.x * RP * RQ;
  bool done = false;
  if constexpr (std::is_same<T, float>::value) {
    if (gridDim.y == 1 && gram_tf32_rects(A.total(), B.total()) <= (int)(blockDim.x >> 5)) {
      gram_core_tf32(A, B, r0, min(n, r0 + rows_per_part), out, gsm_d);
      done = true;
    }
  }
  if (!done)
    gram_core<MR, MC>(A, B, r0, min(n, r0 + rows_per_part), out, gsm_d, blockIdx.y * ptc, ptc);
  gram_finish_last(partial, (int)gridDim.x, kGramSplit, counters, A.total(), B.total(),
                   (int)blockIdx.x, result);
}

size_t gram_partial_elems(int P, int Q) {
  const size_t RP = (2 * P + 7) / 8 * 8, RQ = (2 * Q + 7) / 8 * 8;
  // the partials, the group sums, then the kGramSplit + 1 counters
  return (size_t)(kGramParts + kGramSplit) * RP * RQ / 2 + 1 + (kGramSplit + 1 + 3) / 4;
}

template <typename T>
int launch_gram(const BlockList<T>& A, const BlockList<T>& B, long long n,
                double2* partial, size_t partial_elems, double2* out, cudaStream_t st) {
  const int P = A.total(), Q = B.total();
  if (P > kMaxSmall || Q > kMaxSmall || P <= 0 || Q <= 0) {
    set_error("gram dimensions out of range");
    return QDKP_ERR_ARG;
  }
  const int RP = (2 * P + 7) / 8 * 8, RQ = (2 * Q + 7) / 8 * 8;
  long long parts = (n + 255) / 256;
  if (parts > kGramParts) parts = kGramParts;
  if (parts < 1) parts = 1;
  long long rpp = (n + parts - 1) / parts;
  rpp = (rpp + 3) / 4 * 4;
  parts = (n + rpp - 1) / rpp;
  const size_t counter_at = ((size_t)(parts + kGramSplit) * RP * RQ + 1) / 2 + 1;   // double2 units
  if (counter_at + (kGramSplit + 1 + 3) / 4 > partial_elems) {
    set_error("gram partial buffer too small");
    return QDKP_ERR_WORKSPACE;
  }
  int* counters = reinterpret_cast<int*>(partial + counter_at);
  QDKP_CUDA_TRY(cudaMemsetAsync(counters, 0, (kGramSplit + 1) * sizeof(int), st));
  const size_t smem = gram_smem_bytes(P, Q, (int)sizeof(cplx<T>));
  static bool attr = false;
  if (!attr) {
    const int big = 200 * 1024;
    cudaFuncSetAttribute(gram_partial_kernel<3, 3, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    attr = true;
  }
  const GramPlan gp = gram_plan(P, Q);
  int threads = gp.threads;
  if (std::is_same<T, float>::value && gp.panels == 1) {   // the TF32 core: a warp per rectangle
    const int G = gram_tf32_rects(P, Q);
    if (G > threads / 32 && G <= 16) threads = 512;
  }
  double* pd = reinterpret_cast<double*>(partial);
  gram_partial_kernel<3, 3, T><<<dim3((unsigned)parts, gp.panels), threads, smem, st>>>(
      A, B, n, rpp, pd, gp.ptc, counters, out);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

// ------------------------------------------------------------------------------------------------
// Block update: Y = beta Y + sum_k A_k C_k  (C_k row-major cols_k x q)
// ------------------------------------------------------------------------------------------------
struct CoefList {
  const double2* c[3];
};

template <typename T>
__global__ void __launch_bounds__(kUpdThreads, 2)
update_kernel(const BlockList<T> A, const CoefList C, int q, long long n, cplx<T>* Y,
              long long ldy, int accumulate) {
  extern __shared__ __align__(16) unsigned char usm[];
  const double2* Cf[3] = {C.c[0], C.c[1], C.c[2]};
  constexpr int chunk = std::is_same<T, float>::value ? kTfUpdChunk : kUpdChunk;
  const long long per = ((n + gridDim.x - 1) / gridDim.x + chunk - 1) / chunk * chunk;
  const long long r0 = (long long)blockIdx.x * per;
  if (r0 >= n) return;
  if constexpr (std::is_same<T, float>::value)
    update_rows_tf32(A, Cf, q, r0, min(n, r0 + per), Y, ldy, accumulate, 0, usm);
  else
    update_rows(A, Cf, q, r0, min(n, r0 + per), Y, ldy, accumulate, 0, usm);
}

// complex64 blocks on the tcgen05 tensor cores (umma_dev.cuh): one CTA per SM at most, each a
// contiguous range of 128-row tiles run as one pipeline
__global__ void __launch_bounds__(kUmmaThreads, 1)
update_umma_kernel(const BlockList<float> A, const CoefList C, int q, long long n, float2* Y,
                   long long ldy, int accumulate, int cmax, int ldmax) {
  extern __shared__ __align__(128) unsigned char usm_u[];
  const double2* Cf[3] = {C.c[0], C.c[1], C.c[2]};
  const UmmaPlan pl = umma_plan(A.total(), q, 1, cmax, ldmax);
  const long long tiles = (n + kUmmaRows - 1) / kUmmaRows;
  const long long per = (tiles + gridDim.x - 1) / gridDim.x * kUmmaRows;
  const long long r0 = (long long)blockIdx.x * per;
  if (r0 >= n) return;
  UmmaCtx cx;
  umma_ctx_init(cx, pl);
  update_rows_umma(pl, cx, A, Cf, q, r0, min(n, r0 + per), Y, ldy, accumulate, 0, usm_u);
  umma_ctx_free(cx);
}

bool c64_update_tcgen05() {
  static const bool on = [] {
    const char* v = std::getenv("QDKP_C64_UPDATE");
    if (v && std::strcmp(v, "mma") == 0) return false;
    if (v && std::strcmp(v, "tcgen05") == 0) return true;
    return kC64UpdateTcgen05Default;
  }();
  return on;
}

template <typename T>
int launch_update(const BlockList<T>& A, const double2* const* C, int q, long long n,
                  cplx<T>* Y, long long ldy, int accumulate, cudaStream_t st) {
  if (q > kMaxBlock || A.total() > kMaxSmall || q < 1) { set_error("update dimensions out of range"); return QDKP_ERR_ARG; }
  CoefList cl;
  for (int b = 0; b < 3; ++b) cl.c[b] = b < A.nblk ? C[b] : nullptr;
  const int P = A.total();
  if constexpr (std::is_same<T, float>::value) if (c64_update_tcgen05()) {
    static bool uattr = false;
    if (!uattr) {
      QDKP_CUDA_TRY(cudaFuncSetAttribute(update_umma_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kUmmaSmemLimit));
      uattr = true;
    }
    // blocks are split into sub-blocks of at most kMaxBlock columns (the operand buffers' width),
    // three to a launch; a list that needs more sub-blocks is formed by launches that accumulate
    // (there Y must not alias an input). Raw stages hold rows of up to 32 complex values; a
    // block with a longer row is read directly.
    struct Sub { const float2* p; long long ld; int cols; const double2* c; };
    std::vector<Sub> subs;
    for (int b = 0; b < A.nblk; ++b)
      for (int c0 = 0; c0 < A.cols[b]; c0 += kMaxBlock)
        subs.push_back({A.p[b] + c0, A.ld[b], std::min(kMaxBlock, A.cols[b] - c0),
                        C[b] ? C[b] + (size_t)c0 * q : nullptr});
    int nsm = 148;
    QDKP_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0));
    long long ublocks = (n + kUmmaRows - 1) / kUmmaRows;
    if (ublocks > nsm) ublocks = nsm;
    for (size_t s0 = 0; s0 < subs.size(); s0 += 3) {
      BlockList<float> L;
      CoefList cs;
      L.nblk = (int)std::min<size_t>(3, subs.size() - s0);
      int cmax = 1, ldmax = 1, Ps = 0;
      for (int b = 0; b < 3; ++b) cs.c[b] = nullptr;
      for (int b = 0; b < L.nblk; ++b) {
        const Sub& u = subs[s0 + b];
        L.p[b] = u.p; L.ld[b] = u.ld; L.cols[b] = u.cols; cs.c[b] = u.c;
        cmax = std::max(cmax, u.cols);
        if (u.ld <= 32) ldmax = std::max(ldmax, (int)u.ld);
        Ps += u.cols;
      }
      ldmax = std::max(ldmax, cmax);
      const UmmaPlan pl = umma_plan(Ps, q, 1, cmax, ldmax);
      if (!pl.nout_pass) { set_error("tcgen05 update plan does not fit shared memory"); return QDKP_ERR_ARG; }
      update_umma_kernel<<<(unsigned)ublocks, kUmmaThreads, pl.bytes, st>>>(
          L, cs, q, n, Y, ldy, s0 == 0 ? accumulate : 1, cmax, ldmax);
      count_launch();
      QDKP_CUDA_TRY(cudaGetLastError());
    }
    return QDKP_OK;
  }
  const size_t smem = std::is_same<T, float>::value ? update_tf32_smem_bytes(P, q)
                                                    : update_smem_bytes(P, q);
  static bool attr = false;
  if (!attr) {
    QDKP_CUDA_TRY(cudaFuncSetAttribute(update_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       200 * 1024));
    attr = true;
  }
  long long blocks = (n + kUpdChunk - 1) / kUpdChunk;
  if (blocks > 148 * 4) blocks = 148 * 4;
  update_kernel<T><<<(unsigned)blocks, kUpdThreads, smem, st>>>(A, cl, q, n, Y, ldy, accumulate);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

// ------------------------------------------------------------------------------------------------
// Small dense FP64 (one CTA).
// ------------------------------------------------------------------------------------------------

__global__ void __launch_bounds__(kSmallThreads)
chol_inv_kernel(const double2* __restrict__ G, int n, double2* __restrict__ Uinv,
                int* __restrict__ status) {
  extern __shared__ double2 ssm[];
  double2* S1 = ssm + n * n;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) ssm[e] = G[e];
  __syncthreads();
  const int fail = block_cholesky_upper(ssm, n);
  if (threadIdx.x == 0) *status = fail;
  if (fail) return;
  block_upper_inverse(ssm, n, S1);
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) Uinv[e] = S1[e];
}

int launch_chol_inv(const double2* G, int n, double2* Uinv, int* status, cudaStream_t st) {
  if (n < 1 || n > kMaxSmall) { set_error("chol_inv dimension out of range"); return QDKP_ERR_ARG; }
  const size_t smem = 2 * (size_t)n * n * sizeof(double2);
  QDKP_CUDA_TRY(cudaFuncSetAttribute(chol_inv_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  chol_inv_kernel<<<1, kSmallThreads, smem, st>>>(G, n, Uinv, status);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

// w ascending, V columns permuted accordingly; generalized problem through B = U^H U (with
// 0 < nwant < n only the first nwant pairs are computed).
__global__ void __launch_bounds__(kSmallThreads)
eigh_kernel(const double2* __restrict__ A, const double2* __restrict__ B, int n,
            double* __restrict__ w, double2* __restrict__ Vout, double2* __restrict__ scratch,
            int* __restrict__ status, int nwant) {
  extern __shared__ double2 esm[];
  const int st = block_eigh(A, B, n, w, Vout, scratch, esm, esm + n * n, nwant);
  if (threadIdx.x == 0) *status = st;
}

int launch_eigh(const double2* A, const double2* B, int n, double* w, double2* V,
                double2* scratch, int* status, cudaStream_t st, int nwant) {
  if (n < 1 || n > kMaxSmall) { set_error("eigh dimension out of range"); return QDKP_ERR_ARG; }
  const size_t smem = 2 * (size_t)n * n * sizeof(double2);
  QDKP_CUDA_TRY(cudaFuncSetAttribute(eigh_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  eigh_kernel<<<1, kSmallThreads, smem, st>>>(A, B, n, w, V, scratch, status, nwant);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

// complex128 (plain form, refinement) and complex64 (mixed-precision search) blocks
#define QDKP_BLOCKOPS_INST(T)                                                                      \
  template int launch_colnorm2<T>(const cplx<T>*, long long, const cplx<T>*, long long,          \
                                  const double*, int, long long, double*, int, double*,          \
                                  cudaStream_t);                                                 \
  template int launch_gram<T>(const BlockList<T>&, const BlockList<T>&, long long, double2*,     \
                              size_t, double2*, cudaStream_t);                                   \
  template int launch_update<T>(const BlockList<T>&, const double2* const*, int, long long,       \
                                cplx<T>*, long long, int, cudaStream_t);
QDKP_BLOCKOPS_INST(double)
QDKP_BLOCKOPS_INST(float)
#undef QDKP_BLOCKOPS_INST
template int launch_gather<double, double>(const double2*, long long, const int*, int, long long,
                                           double2*, long long, cudaStream_t);
template int launch_gather<float, float>(const float2*, long long, const int*, int, long long,
                                         float2*, long long, cudaStream_t);
template int launch_copy<double, double>(const double2*, long long, int, long long, double2*,
                                         long long, cudaStream_t);
template int launch_copy<float, float>(const float2*, long long, int, long long, float2*,
                                       long long, cudaStream_t);
template int launch_copy<double, float>(const double2*, long long, int, long long, float2*,
                                        long long, cudaStream_t);
template int launch_copy<float, double>(const float2*, long long, int, long long, double2*,
                                        long long, cudaStream_t);

}  // namespace qdkp

using namespace qdkp;

extern "C" {

size_t qdkp_block_gram_workspace_size(int P, int Q) {
  if (P < 1 || Q < 1 || P > kMaxSmall || Q > kMaxSmall) return 0;
  return gram_partial_elems(P, Q) * sizeof(double2) + (size_t)P * Q * sizeof(double2) + 256;
}

int qdkp_block_gram(const void* A, int64_t lda, int P, const void* B, int64_t ldb, int Q,
                    int64_t n, int precision, double* out, void* ws, size_t ws_bytes,
                    void* stream) {
  QDKP_CHECK_ARG(A && B && out && ws, "NULL argument");
  QDKP_CHECK_ARG(P >= 1 && Q >= 1 && P <= kMaxSmall && Q <= kMaxSmall && n >= 1 && lda >= P &&
                 ldb >= Q, "bad block shapes");
  QDKP_CHECK_ARG(precision == QDKP_C128 || precision == QDKP_C64, "bad precision");
  if (ws_bytes < qdkp_block_gram_workspace_size(P, Q)) {
    set_error("qdkp_block_gram: workspace too small");
    return QDKP_ERR_WORKSPACE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t pe = gram_partial_elems(P, Q);
  double2* part = static_cast<double2*>(ws);
  double2* dout = part + pe;
  int rc;
  if (precision == QDKP_C64) {
    BlockList<float> La, Lb;
    La.nblk = 1; La.p[0] = static_cast<const float2*>(A); La.ld[0] = lda; La.cols[0] = P;
    Lb.nblk = 1; Lb.p[0] = static_cast<const float2*>(B); Lb.ld[0] = ldb; Lb.cols[0] = Q;
    rc = launch_gram(La, Lb, n, part, pe, dout, st);
  } else {
    BlockList<double> La, Lb;
    La.nblk = 1; La.p[0] = static_cast<const double2*>(A); La.ld[0] = lda; La.cols[0] = P;
    Lb.nblk = 1; Lb.p[0] = static_cast<const double2*>(B); Lb.ld[0] = ldb; Lb.cols[0] = Q;
    rc = launch_gram(La, Lb, n, part, pe, dout, st);
  }
  if (rc != QDKP_OK) return rc;
  QDKP_CUDA_TRY(cudaMemcpyAsync(out, dout, (size_t)P * Q * sizeof(double2), cudaMemcpyDeviceToHost, st));
  QDKP_CUDA_TRY(cudaStreamSynchronize(st));
  return QDKP_OK;
}

size_t qdkp_block_eigh_workspace_size(int n) {
  if (n < 1 || n > kMaxSmall) return 0;
  const size_t mat = ((size_t)n * n * sizeof(double2) + 255) / 256 * 256;
  return 5 * mat + ((size_t)n * sizeof(double) + 255) / 256 * 256 + 256;
}

int qdkp_block_eigh(const double* A, const double* B, int n, int nwant, double* w, double* V,
                    void* ws, size_t ws_bytes, void* stream) {
  QDKP_CHECK_ARG(A && w && V && ws, "NULL argument");
  QDKP_CHECK_ARG(n >= 1 && n <= kMaxSmall, "n must be in [1, 72]");
  QDKP_CHECK_ARG(nwant >= 1 && nwant <= n, "nwant must be in [1, n]");
  if (ws_bytes < qdkp_block_eigh_workspace_size(n)) {
    set_error("qdkp_block_eigh: workspace too small");
    return QDKP_ERR_WORKSPACE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t mb = (size_t)n * n * sizeof(double2);
  const size_t mat = (mb + 255) / 256 * 256;
  char* p = static_cast<char*>(ws);
  double2* dA = reinterpret_cast<double2*>(p);
  double2* dB = reinterpret_cast<double2*>(p + mat);
  double2* dV = reinterpret_cast<double2*>(p + 2 * mat);
  double2* scr = reinterpret_cast<double2*>(p + 3 * mat);     // 2 n^2
  double* dw = reinterpret_cast<double*>(p + 5 * mat);
  int* dstat = reinterpret_cast<int*>(p + 5 * mat + ((size_t)n * sizeof(double) + 255) / 256 * 256);
  QDKP_CUDA_TRY(cudaMemcpyAsync(dA, A, mb, cudaMemcpyHostToDevice, st));
  if (B) QDKP_CUDA_TRY(cudaMemcpyAsync(dB, B, mb, cudaMemcpyHostToDevice, st));
  const int rc = launch_eigh(dA, B ? dB : nullptr, n, dw, dV, scr, dstat, st, nwant < n ? nwant : 0);
  if (rc != QDKP_OK) return rc;
  int hstat = 0;
  QDKP_CUDA_TRY(cudaMemcpyAsync(w, dw, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
  QDKP_CUDA_TRY(cudaMemcpyAsync(V, dV, mb, cudaMemcpyDeviceToHost, st));
  QDKP_CUDA_TRY(cudaMemcpyAsync(&hstat, dstat, sizeof(int), cudaMemcpyDeviceToHost, st));
  QDKP_CUDA_TRY(cudaStreamSynchronize(st));
  if (hstat != 0) {
    set_error(hstat == 1 ? "qdkp_block_eigh: B is not positive definite"
                         : "qdkp_block_eigh: non-finite spectrum");
    return QDKP_ERR_NUMERIC;
  }
  return QDKP_OK;
}

size_t qdkp_block_update_workspace_size(int P, int q) {
  if (P < 1 || q < 1 || P > kMaxSmall || q > kMaxBlock) return 0;
  return (size_t)P * q * sizeof(double2) + 256;
}

int qdkp_block_update(const void* A, int64_t lda, int P, const double* C, int q, int64_t n,
                      void* Y, int64_t ldy, int precision, void* ws, size_t ws_bytes,
                      void* stream) {
  QDKP_CHECK_ARG(A && C && Y && ws, "NULL argument");
  QDKP_CHECK_ARG(P >= 1 && q >= 1 && P <= kMaxSmall && q <= kMaxBlock && n >= 1 && lda >= P &&
                 ldy >= q, "bad block shapes");
  QDKP_CHECK_ARG(precision == QDKP_C128 || precision == QDKP_C64, "bad precision");
  if (ws_bytes < qdkp_block_update_workspace_size(P, q)) {
    set_error("qdkp_block_update: workspace too small");
    return QDKP_ERR_WORKSPACE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double2* dC = static_cast<double2*>(ws);
  QDKP_CUDA_TRY(cudaMemcpyAsync(dC, C, (size_t)P * q * sizeof(double2), cudaMemcpyHostToDevice, st));
  const double2* Cs[1] = {dC};
  int rc;
  if (precision == QDKP_C64) {
    BlockList<float> La;
    La.nblk = 1; La.p[0] = static_cast<const float2*>(A); La.ld[0] = lda; La.cols[0] = P;
    rc = launch_update(La, Cs, q, n, static_cast<float2*>(Y), ldy, 0, st);
  } else {
    BlockList<double> La;
    La.nblk = 1; La.p[0] = static_cast<const double2*>(A); La.ld[0] = lda; La.cols[0] = P;
    rc = launch_update(La, Cs, q, n, static_cast<double2*>(Y), ldy, 0, st);
  }
  if (rc != QDKP_OK) return rc;
  QDKP_CUDA_TRY(cudaStreamSynchronize(st));
  return QDKP_OK;
}

}  // extern "C"
