// Tall-skinny block kernels and one-CTA small dense FP64 kernels used by the LOBPCG driver.
//
// Blocks are row-major (n, cols) complex arrays with a leading dimension (elements). Every
// reduction over the long dimension is two-stage and deterministic: each CTA writes a partial,
// a second kernel sums the partials in a fixed order.
#pragma once
#include "qdkp_common.cuh"

namespace qdkp {

constexpr int kMaxBlock = 24;          // largest LOBPCG block width (columns) supported
constexpr int kMaxSmall = 3 * kMaxBlock;  // largest Rayleigh-Ritz dimension
constexpr int kTallThreads = 256;
constexpr int kSmallThreads = 512;
// Gram kernels: 3 x 3 warps, each owning up to kGramMaxT x kGramMaxT 8x8 tiles of the real
// product, rows staged kGramChunk at a time.
constexpr int kGramWarpsR = 3, kGramWarpsC = 3;
constexpr int kGramThreads = 32 * kGramWarpsR * kGramWarpsC;
constexpr int kGramMaxT = 6;                        // tiles per warp per dimension
constexpr int kGramChunk = 32;                      // rows staged per step

// A group of up to three column blocks concatenated along the columns: [B0 | B1 | B2].
template <typename T>
struct BlockList {
  const cplx<T>* p[3];
  long long ld[3];
  int cols[3];
  int nblk;
  __host__ __device__ int total() const {
    int t = 0;
    for (int i = 0; i < nblk; ++i) t += cols[i];
    return t;
  }
};

// Which kernel forms complex64 block updates: the tcgen05 pipeline (umma_dev.cuh) or the
// split-TF32 mma.sync kernel (dense_dev.cuh). QDKP_C64_UPDATE=tcgen05 or =mma in the environment
// chooses; read once per process.
bool c64_update_tcgen05();

// Tall block kernels, for complex128 (T = double) and complex64 (T = float) blocks; sums and
// the Gram / coefficient matrices are FP64 either way.
template <typename T>
int launch_colnorm2(const cplx<T>* A, long long lda, const cplx<T>* B, long long ldb,
                    const double* lambda, int m, long long n, double* partial, int nparts,
                    double* out, cudaStream_t st);
int launch_resid_gather(const double2* AX, long long ldax, const double2* X, long long ldx,
                        const double* lambda, const int* idx, int ma, long long n, double2* R,
                        long long ldr, cudaStream_t st);
template <typename TS, typename TD>
int launch_gather(const cplx<TS>* src, long long lds, const int* idx, int ma, long long n,
                  cplx<TD>* dst, long long ldd, cudaStream_t st);
// dst = src (columns [0, cols)), converting the precision when TS != TD
template <typename TS, typename TD>
int launch_copy(const cplx<TS>* src, long long lds, int cols, long long n, cplx<TD>* dst,
                long long ldd, cudaStream_t st);
// overloads that spell the precision through the vector type (cplx<T> is not deducible)
#define QDKP_TALL_OVERLOADS(C, R)                                                                \
  inline int launch_colnorm2(const C* A, long long lda, const C* B, long long ldb,            \
                             const double* lambda, int m, long long n, double* partial,       \
                             int nparts, double* out, cudaStream_t st) {                      \
    return launch_colnorm2<R>(A, lda, B, ldb, lambda, m, n, partial, nparts, out, st);        \
  }                                                                                           \
  inline int launch_gather(const C* src, long long lds, const int* idx, int ma, long long n,  \
                           C* dst, long long ldd, cudaStream_t st) {                          \
    return launch_gather<R, R>(src, lds, idx, ma, n, dst, ldd, st);                           \
  }                                                                                           \
  inline int launch_copy(const C* src, long long lds, int cols, long long n, C* dst,          \
                         long long ldd, cudaStream_t st) {                                    \
    return launch_copy<R, R>(src, lds, cols, n, dst, ldd, st);                                \
  }
QDKP_TALL_OVERLOADS(double2, double)
QDKP_TALL_OVERLOADS(float2, float)
#undef QDKP_TALL_OVERLOADS
// out (P x Q, row-major, ld Q) = A^H B for concatenated column lists.
template <typename T>
int launch_gram(const BlockList<T>& A, const BlockList<T>& B, long long n,
                double2* partial, size_t partial_elems, double2* out, cudaStream_t st);
size_t gram_partial_elems(int P, int Q);
// Y = beta * Y + sum_k A_k C_k; C_k (cols_k x q, row-major, ld q) in device memory.
template <typename T>
int launch_update(const BlockList<T>& A, const double2* const* C, int q, long long n,
                  cplx<T>* Y, long long ldy, int accumulate, cudaStream_t st);

// Small dense (one CTA). Matrices row-major with ld = n. status: 0 ok, 1 failure.
int launch_chol_inv(const double2* G, int n, double2* Uinv, int* status, cudaStream_t st);
// nwant > 0: only the nwant smallest eigenpairs are needed (w[0..nwant), V's first columns)
int launch_eigh(const double2* A, const double2* B, int n, double* w, double2* V,
                double2* scratch, int* status, cudaStream_t st, int nwant = 0);

}  // namespace qdkp
