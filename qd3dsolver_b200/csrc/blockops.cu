// Tall-skinny block kernels (norms, residual gather, Gram, block update) and one-CTA FP64
// small dense kernels (Cholesky + triangular inverse, Hermitian generalized eigensolver by
// parallel cyclic Jacobi) for the LOBPCG driver.
#include <algorithm>
#include <cmath>

#include "blockops.cuh"

namespace qdkp {

// ------------------------------------------------------------------------------------------------
// Column norms: out[j] = sum_r |A[r, j] - lambda_j B[r, j]|^2 (B may be NULL).
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kTallThreads)
colnorm2_partial(const double2* __restrict__ A, long long lda, const double2* __restrict__ B,
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
        double2 a = A[r * lda + j];
        if (B) {
          const double2 b = B[r * ldb + j];
          a.x -= lam[j] * b.x;
          a.y -= lam[j] * b.y;
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

int launch_colnorm2(const double2* A, long long lda, const double2* B, long long ldb,
                    const double* lambda, int m, long long n, double* partial, int nparts,
                    double* out, cudaStream_t st) {
  if (m > kMaxBlock) { set_error("block wider than kMaxBlock"); return QDKP_ERR_ARG; }
  colnorm2_partial<<<nparts, kTallThreads, 0, st>>>(A, lda, B, ldb, lambda, m, n, partial);
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

__global__ void gather_kernel(const double2* __restrict__ src, long long lds,
                              const int* __restrict__ idx, int ma, long long n,
                              double2* __restrict__ dst, long long ldd) {
  const long long total = n * ma;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / ma;
    const int c = (int)(e - r * ma);
    dst[r * ldd + c] = src[r * lds + (idx ? idx[c] : c)];
  }
}

int launch_gather(const double2* src, long long lds, const int* idx, int ma, long long n,
                  double2* dst, long long ldd, cudaStream_t st) {
  gather_kernel<<<1184, 256, 0, st>>>(src, lds, idx, ma, n, dst, ldd);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

int launch_copy(const double2* src, long long lds, int cols, long long n, double2* dst,
                long long ldd, cudaStream_t st) {
  if (lds == cols && ldd == cols) {
    QDKP_CUDA_TRY(cudaMemcpyAsync(dst, src, (size_t)n * cols * sizeof(double2),
                                  cudaMemcpyDeviceToDevice, st));
    return QDKP_OK;
  }
  return launch_gather(src, lds, nullptr, cols, n, dst, ldd, st);
}

// ------------------------------------------------------------------------------------------------
// Gram: out = A^H B over concatenated column lists, FP64 accumulation, deterministic.
// ------------------------------------------------------------------------------------------------
constexpr int kGramParts = 296;

__device__ __forceinline__ double2 list_elem(const BlockList<double>& L, long long r, int c) {
  int b = 0;
  while (b < L.nblk - 1 && c >= L.cols[b]) { c -= L.cols[b]; ++b; }
  return L.p[b][r * L.ld[b] + c];
}

// The complex product A^H B is one real GEMM over the interleaved (re, im) view: with
// A' (n x 2P) and B' (n x 2Q) the real views, C' = A'^T B' and
//   Re G_ij = C'_{2i,2j} + C'_{2i+1,2j+1},   Im G_ij = C'_{2i,2j+1} - C'_{2i+1,2j}.
// C' is accumulated on the FP64 tensor cores (mma.sync.m8n8k4.f64; the tcgen05 family has no
// f64 kind). A CTA of 3 x 3 warps owns all 8x8 tiles of C' for its slice of rows; each warp
// owns a rectangle of up to 6 x 6 tiles and keeps them in registers across the slice.
constexpr int kGramWarpsR = 3, kGramWarpsC = 3;
constexpr int kGramThreads = 32 * kGramWarpsR * kGramWarpsC;
constexpr int kGramMaxT = 6;                        // tiles per warp per dimension
constexpr int kGramChunk = 32;                      // rows staged per step

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

template <int MAXT>
__global__ void __launch_bounds__(kGramThreads)
gram_partial_kernel(const BlockList<double> A, const BlockList<double> B, long long n,
                    long long rows_per_part, double* __restrict__ partial) {
  extern __shared__ double gsm_d[];
  const int P = A.total(), Q = B.total();
  const int RP = (2 * P + 7) / 8 * 8, RQ = (2 * Q + 7) / 8 * 8;   // padded real widths
  double* sA = gsm_d;                        // [kGramChunk][RP]
  double* sB = gsm_d + kGramChunk * RP;      // [kGramChunk][RQ]
  const long long r0 = blockIdx.x * rows_per_part;
  const long long r1 = min(n, r0 + rows_per_part);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int TR = RP / 8, TC = RQ / 8;
  const int wr = warp / kGramWarpsC, wc = warp % kGramWarpsC;
  const int tr_per = (TR + kGramWarpsR - 1) / kGramWarpsR, tc_per = (TC + kGramWarpsC - 1) / kGramWarpsC;
  const int tr0 = wr * tr_per, tc0 = wc * tc_per;
  double acc[MAXT][MAXT][2];
#pragma unroll
  for (int i = 0; i < MAXT; ++i)
#pragma unroll
    for (int j = 0; j < MAXT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  for (long long rt = r0; rt < r1; rt += kGramChunk) {
    // stage rows [rt, rt + chunk) of A' and B' (zero padded)
    for (int e = threadIdx.x; e < kGramChunk * (RP / 2); e += blockDim.x) {
      const int row = e / (RP / 2), c = e - row * (RP / 2);
      double2 z = make_double2(0.0, 0.0);
      if (rt + row < r1 && c < P) z = list_elem(A, rt + row, c);
      *reinterpret_cast<double2*>(&sA[row * RP + 2 * c]) = z;
    }
    for (int e = threadIdx.x; e < kGramChunk * (RQ / 2); e += blockDim.x) {
      const int row = e / (RQ / 2), c = e - row * (RQ / 2);
      double2 z = make_double2(0.0, 0.0);
      if (rt + row < r1 && c < Q) z = list_elem(B, rt + row, c);
      *reinterpret_cast<double2*>(&sB[row * RQ + 2 * c]) = z;
    }
    __syncthreads();
#pragma unroll 2
    for (int k0 = 0; k0 < kGramChunk; k0 += 4) {
      double a[MAXT], b[MAXT];
#pragma unroll
      for (int i = 0; i < MAXT; ++i) {
        const int ti = tr0 + i;
        a[i] = (i < tr_per && ti < TR) ? sA[(k0 + t4) * RP + ti * 8 + g] : 0.0;
      }
#pragma unroll
      for (int j = 0; j < MAXT; ++j) {
        const int tj = tc0 + j;
        b[j] = (j < tc_per && tj < TC) ? sB[(k0 + t4) * RQ + tj * 8 + g] : 0.0;
      }
#pragma unroll
      for (int i = 0; i < MAXT; ++i)
#pragma unroll
        for (int j = 0; j < MAXT; ++j)
          if (i < tr_per && j < tc_per) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
    __syncthreads();
  }
  // partial C' (RP x RQ, row-major) for this slice
  double* out = partial + (long long)blockIdx.x * RP * RQ;
#pragma unroll
  for (int i = 0; i < MAXT; ++i)
#pragma unroll
    for (int j = 0; j < MAXT; ++j) {
      const int ti = tr0 + i, tj = tc0 + j;
      if (i < tr_per && j < tc_per && ti < TR && tj < TC) {
        const int row = ti * 8 + g, col = tj * 8 + 2 * t4;
        out[(long long)row * RQ + col] = acc[i][j][0];
        out[(long long)row * RQ + col + 1] = acc[i][j][1];
      }
    }
}

// Stage 1: column-block sums of the partial C' slices (coalesced over the RP x RQ elements);
// stage 2: the remaining per-split sums folded into the complex Gram matrix.
constexpr int kGramSplit = 16;

__global__ void gram_reduce1_kernel(const double* __restrict__ partial, int nparts, int elems,
                                    double* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int sp = blockIdx.y;
  if (e >= elems) return;
  const int per = (nparts + kGramSplit - 1) / kGramSplit;
  const int b0 = sp * per, b1 = min(nparts, b0 + per);
  double s = 0.0;
  for (int b = b0; b < b1; ++b) s += partial[(long long)b * elems + e];
  out[(long long)sp * elems + e] = s;
}

__global__ void gram_reduce2_kernel(const double* __restrict__ part2, int P, int Q, int RQ,
                                    int elems, double2* __restrict__ out) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= P * Q) return;
  const int i = o / Q, j = o - i * Q;
  const long long rr = (long long)(2 * i) * RQ + 2 * j;   // C'_{2i,2j}
  double re = 0.0, im = 0.0;
  for (int sp = 0; sp < kGramSplit; ++sp) {
    const double* c = part2 + (long long)sp * elems;
    re += c[rr] + c[rr + RQ + 1];
    im += c[rr + 1] - c[rr + RQ];
  }
  out[o] = make_double2(re, im);
}

size_t gram_partial_elems(int P, int Q) {
  const size_t RP = (2 * P + 7) / 8 * 8, RQ = (2 * Q + 7) / 8 * 8;
  return (size_t)(kGramParts + kGramSplit) * RP * RQ / 2 + 1;   // in double2 units
}

int launch_gram(const BlockList<double>& A, const BlockList<double>& B, long long n,
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
  rpp = (rpp + kGramChunk - 1) / kGramChunk * kGramChunk;
  parts = (n + rpp - 1) / rpp;
  if ((size_t)(parts + kGramSplit) * RP * RQ > 2 * partial_elems) {
    set_error("gram partial buffer too small");
    return QDKP_ERR_WORKSPACE;
  }
  const size_t smem = (size_t)kGramChunk * (RP + RQ) * sizeof(double);
  const int TR = RP / 8, TC = RQ / 8;
  const int tmax = std::max((TR + kGramWarpsR - 1) / kGramWarpsR, (TC + kGramWarpsC - 1) / kGramWarpsC);
  double* pd = reinterpret_cast<double*>(partial);
  const unsigned grid = (unsigned)parts;
  if (tmax <= 2) gram_partial_kernel<2><<<grid, kGramThreads, smem, st>>>(A, B, n, rpp, pd);
  else if (tmax <= 3) gram_partial_kernel<3><<<grid, kGramThreads, smem, st>>>(A, B, n, rpp, pd);
  else if (tmax <= 4) gram_partial_kernel<4><<<grid, kGramThreads, smem, st>>>(A, B, n, rpp, pd);
  else gram_partial_kernel<6><<<grid, kGramThreads, smem, st>>>(A, B, n, rpp, pd);
  count_launch();
  const int elems = RP * RQ;
  double* part2 = pd + (size_t)parts * elems;
  gram_reduce1_kernel<<<dim3((elems + 255) / 256, kGramSplit), 256, 0, st>>>(pd, (int)parts, elems, part2);
  count_launch();
  gram_reduce2_kernel<<<(P * Q + 127) / 128, 128, 0, st>>>(part2, P, Q, RQ, elems, out);
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

// Y' = A' C'' on the FP64 tensor cores, with A' (rows x 2P) the real view of [A_0 | A_1 | A_2]
// and C'' (2P x 2q) the real representation of the stacked complex coefficients:
//   C''_{2i,2j} = Re C_ij, C''_{2i,2j+1} = Im C_ij, C''_{2i+1,2j} = -Im C_ij,
//   C''_{2i+1,2j+1} = Re C_ij.
// An MMA accumulator pair (d0, d1) of a lane is exactly one complex output (re, im).
// A CTA stages 32 rows of every input block before it writes the same rows of Y, so Y may
// alias one of the inputs.
constexpr int kUpdRows = 32;
constexpr int kUpdThreads = 256;

__global__ void __launch_bounds__(kUpdThreads)
update_kernel(const BlockList<double> A, const CoefList C, int q, long long n, double2* Y,
              long long ldy, int accumulate) {
  extern __shared__ double usm[];
  const int P = A.total();
  const int KP = 2 * P;                       // real K
  const int KPp = (KP + 3) / 4 * 4;           // padded to the MMA k step
  const int NQ = (2 * q + 7) / 8 * 8;         // padded real N
  double* sC = usm;                           // [KPp][NQ]
  double* sA = usm + KPp * NQ;                // [kUpdRows][KPp + 1]
  const int lda_s = KPp + 1;
  int off[3];
  int tot = 0;
  for (int b = 0; b < A.nblk; ++b) { off[b] = tot; tot += A.cols[b]; }
  for (int e = threadIdx.x; e < KPp * NQ; e += blockDim.x) sC[e] = 0.0;
  __syncthreads();
  for (int e = threadIdx.x; e < P * q; e += blockDim.x) {
    const int i = e / q, j = e - i * q;
    int b = 0;
    while (b < A.nblk - 1 && i >= off[b] + A.cols[b]) ++b;
    const double2 c = C.c[b][(i - off[b]) * q + j];
    sC[(2 * i) * NQ + 2 * j] = c.x;
    sC[(2 * i) * NQ + 2 * j + 1] = c.y;
    sC[(2 * i + 1) * NQ + 2 * j] = -c.y;
    sC[(2 * i + 1) * NQ + 2 * j + 1] = c.x;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int mt = warp & 3;                   // 8-row tile within the 32-row slice
  const int nhalf = warp >> 2;               // which half of the n tiles
  const int NT = NQ / 8;
  const int nt_per = (NT + 1) / 2;
  const int nt0 = nhalf * nt_per;
  for (long long r0 = (long long)blockIdx.x * kUpdRows; r0 < n; r0 += (long long)gridDim.x * kUpdRows) {
    __syncthreads();
    // stage rows [r0, r0 + 32) of every input (complex elements, coalesced per block)
    for (int b = 0; b < A.nblk; ++b) {
      const int cb = A.cols[b];
      for (int e = threadIdx.x; e < kUpdRows * cb; e += blockDim.x) {
        const int row = e / cb, c = e - row * cb;
        double2 z = make_double2(0.0, 0.0);
        if (r0 + row < n) z = A.p[b][(r0 + row) * A.ld[b] + c];
        sA[row * lda_s + 2 * (off[b] + c)] = z.x;
        sA[row * lda_s + 2 * (off[b] + c) + 1] = z.y;
      }
    }
    for (int e = threadIdx.x; e < kUpdRows * (KPp - KP); e += blockDim.x) {
      const int row = e / (KPp - KP), c = e - row * (KPp - KP);
      sA[row * lda_s + KP + c] = 0.0;
    }
    __syncthreads();
    double acc[3][2];
    const long long rowg = r0 + mt * 8 + g;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int col = (nt0 + j) * 4 + t4;     // complex output column
      double2 y0 = make_double2(0.0, 0.0);
      if (accumulate && j < nt_per && nt0 + j < NT && col < q && rowg < n) y0 = Y[rowg * ldy + col];
      acc[j][0] = y0.x; acc[j][1] = y0.y;
    }
    for (int k0 = 0; k0 < KPp; k0 += 4) {
      const double a = sA[(mt * 8 + g) * lda_s + k0 + t4];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        if (j < nt_per && nt0 + j < NT) {
          const double bb = sC[(k0 + t4) * NQ + (nt0 + j) * 8 + g];
          dmma(acc[j][0], acc[j][1], a, bb);
        }
      }
    }
    __syncthreads();   // every warp has read the staged rows before any row of Y is written
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int col = (nt0 + j) * 4 + t4;
      if (j < nt_per && nt0 + j < NT && col < q && rowg < n)
        Y[rowg * ldy + col] = make_double2(acc[j][0], acc[j][1]);
    }
  }
}

int launch_update(const BlockList<double>& A, const double2* const* C, int q, long long n,
                  double2* Y, long long ldy, int accumulate, cudaStream_t st) {
  if (q > kMaxBlock || A.total() > kMaxSmall || q < 1) { set_error("update dimensions out of range"); return QDKP_ERR_ARG; }
  CoefList cl;
  for (int b = 0; b < 3; ++b) cl.c[b] = b < A.nblk ? C[b] : nullptr;
  const int P = A.total();
  const int KPp = (2 * P + 3) / 4 * 4, NQ = (2 * q + 7) / 8 * 8;
  const size_t smem = ((size_t)KPp * NQ + (size_t)kUpdRows * (KPp + 1)) * sizeof(double);
  static bool attr = false;
  if (!attr) {
    QDKP_CUDA_TRY(cudaFuncSetAttribute(update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       120 * 1024));
    attr = true;
  }
  long long blocks = (n + kUpdRows - 1) / kUpdRows;
  if (blocks > 148 * 4) blocks = 148 * 4;
  update_kernel<<<(unsigned)blocks, kUpdThreads, smem, st>>>(A, cl, q, n, Y, ldy, accumulate);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

// ------------------------------------------------------------------------------------------------
// Small dense FP64 (one CTA).
// ------------------------------------------------------------------------------------------------

// In-place upper Cholesky of the Hermitian matrix in S (n x n, ld n): S = U^H U, U in the upper
// triangle. Returns nonzero (block-uniform) if a pivot is not positive and finite.
__device__ int block_cholesky_upper(double2* S, int n) {
  __shared__ int fail;
  if (threadIdx.x == 0) fail = 0;
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    if (threadIdx.x == 0) {
      const double d = S[k * n + k].x;
      if (!(d > 0.0) || !isfinite(d)) fail = 1;
      else S[k * n + k] = make_double2(sqrt(d), 0.0);
    }
    __syncthreads();
    if (fail) break;
    const double piv = S[k * n + k].x;
    for (int j = k + 1 + threadIdx.x; j < n; j += blockDim.x) {
      S[k * n + j].x /= piv;
      S[k * n + j].y /= piv;
    }
    __syncthreads();
    const int w = n - k - 1;
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
      const int i = k + 1 + e / w, j = k + 1 + e % w;
      if (j >= i) {
        const double2 a = S[k * n + i], b = S[k * n + j];
        // S[i][j] -= conj(a) * b
        S[i * n + j].x -= a.x * b.x + a.y * b.y;
        S[i * n + j].y -= a.x * b.y - a.y * b.x;
      }
    }
    __syncthreads();
  }
  __syncthreads();
  return fail;
}

// Uinv = inv(U) for the upper triangle of S; written to `out` (ld n), one column per thread.
__device__ void block_upper_inverse(const double2* S, int n, double2* out) {
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    for (int i = n - 1; i > j; --i) out[i * n + j] = make_double2(0.0, 0.0);
    const double2 ujj = S[j * n + j];
    out[j * n + j] = make_double2(1.0 / ujj.x, 0.0);
    for (int i = j - 1; i >= 0; --i) {
      double2 s = make_double2(0.0, 0.0);
      for (int k = i + 1; k <= j; ++k) cfma(s, S[i * n + k], out[k * n + j]);
      const double d = S[i * n + i].x;
      out[i * n + j] = make_double2(-s.x / d, -s.y / d);
    }
  }
  __syncthreads();
}

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

// Parallel cyclic Jacobi on the Hermitian C (smem, n x n); V (smem) accumulates rotations.
// Round-robin ordering gives n/2 disjoint (p, q) pairs per round. A pair is rotated while
// |C_pq| > eps sqrt(|C_pp C_qq|) (the relative-accuracy threshold, so eigenvalues far below
// ||C|| -- the wanted end of a folded spectrum -- are resolved to working precision); the
// iteration stops after a sweep without rotations.
__device__ void block_jacobi(double2* C, double2* V, int n) {
  __shared__ double rcs[kMaxSmall / 2 + 1], rsn[kMaxSmall / 2 + 1];
  __shared__ double2 re[kMaxSmall / 2 + 1];
  __shared__ int rp[kMaxSmall / 2 + 1], rq[kMaxSmall / 2 + 1];
  __shared__ int rotated;
  __shared__ double fro_red[kSmallThreads / 32];
  __shared__ double floor_abs;
  const int n2 = n + (n & 1);
  const int npair = n2 / 2;
  {
    // absolute floor eps ||C||_F: off-diagonals below it are rounding noise (the accuracy
    // LAPACK's Hermitian solvers deliver), so chasing them only adds sweeps
    double f = 0.0;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) f += C[e].x * C[e].x + C[e].y * C[e].y;
    for (int o = 16; o > 0; o >>= 1) f += __shfl_xor_sync(0xffffffffu, f, o);
    if ((threadIdx.x & 31) == 0) fro_red[threadIdx.x >> 5] = f;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += fro_red[w];
      floor_abs = 2.2e-16 * sqrt(t);
    }
    __syncthreads();
  }
  for (int sweep = 0; sweep < 30; ++sweep) {
    if (threadIdx.x == 0) rotated = 0;
    __syncthreads();
    for (int r = 0; r < n2 - 1; ++r) {
      if (threadIdx.x < npair) {
        const int k = threadIdx.x;
        int p, q;
        if (k == 0) { p = r; q = n2 - 1; }
        else { p = (r + k) % (n2 - 1); q = (r - k + n2 - 1) % (n2 - 1); }
        if (p > q) { const int t = p; p = q; q = t; }
        double cs = 1.0, sn = 0.0;
        double2 e = make_double2(1.0, 0.0);
        if (q < n) {
          const double2 c = C[p * n + q];
          const double ac = hypot(c.x, c.y);
          const double a = C[p * n + p].x, b = C[q * n + q].x;
          if (ac > floor_abs && ac > 2.2e-16 * sqrt(fabs(a) * fabs(b))) {
            const double tau = (b - a) / (2.0 * ac);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            cs = 1.0 / sqrt(1.0 + t * t);
            sn = t * cs;
            e = make_double2(c.x / ac, c.y / ac);
            if (sn != 0.0) rotated = 1;
          }
        }
        rp[k] = p; rq[k] = q; rcs[k] = cs; rsn[k] = sn; re[k] = e;
      }
      __syncthreads();
      // columns: C <- C J, V <- V J with J = [[cs, sn e], [-sn conj(e), cs]] on (p, q)
      for (int t = threadIdx.x; t < n * npair; t += blockDim.x) {
        const int k = t / n, i = t - k * n;
        const int p = rp[k], q = rq[k];
        if (q >= n || rsn[k] == 0.0) continue;
        const double cs = rcs[k], sn = rsn[k];
        const double2 e = re[k];
        const double2 m10 = make_double2(-sn * e.x, sn * e.y);   // -sn conj(e)
        const double2 m01 = make_double2(sn * e.x, sn * e.y);    //  sn e
        double2 x = C[i * n + p], y = C[i * n + q];
        double2 np = cscale(cs, x); cfma(np, m10, y);
        double2 nq = cscale(cs, y); cfma(nq, m01, x);
        C[i * n + p] = np; C[i * n + q] = nq;
        x = V[i * n + p]; y = V[i * n + q];
        np = cscale(cs, x); cfma(np, m10, y);
        nq = cscale(cs, y); cfma(nq, m01, x);
        V[i * n + p] = np; V[i * n + q] = nq;
      }
      __syncthreads();
      // rows: C <- J^H C, J^H = [[cs, -sn e], [sn conj(e), cs]]
      for (int t = threadIdx.x; t < n * npair; t += blockDim.x) {
        const int k = t / n, j = t - k * n;
        const int p = rp[k], q = rq[k];
        if (q >= n || rsn[k] == 0.0) continue;
        const double cs = rcs[k], sn = rsn[k];
        const double2 e = re[k];
        const double2 a01 = make_double2(-sn * e.x, -sn * e.y);
        const double2 a10 = make_double2(sn * e.x, -sn * e.y);
        const double2 x = C[p * n + j], y = C[q * n + j];
        double2 np = cscale(cs, x); cfma(np, a01, y);
        double2 nq = cscale(cs, y); cfma(nq, a10, x);
        C[p * n + j] = np; C[q * n + j] = nq;
      }
      __syncthreads();
      if (threadIdx.x < npair) {
        const int k = threadIdx.x, p = rp[k], q = rq[k];
        if (q < n && rsn[k] != 0.0) {
          C[p * n + q] = make_double2(0.0, 0.0);
          C[q * n + p] = make_double2(0.0, 0.0);
          C[p * n + p].y = 0.0;
          C[q * n + q].y = 0.0;
        }
      }
      __syncthreads();
    }
    if (!rotated) break;
    __syncthreads();
  }
}

// w ascending, V columns permuted accordingly; generalized problem through B = U^H U.
__global__ void __launch_bounds__(kSmallThreads)
eigh_kernel(const double2* __restrict__ A, const double2* __restrict__ B, int n,
            double* __restrict__ w, double2* __restrict__ Vout, double2* __restrict__ scratch,
            int* __restrict__ status) {
  extern __shared__ double2 esm[];
  double2* S0 = esm;
  double2* S1 = esm + n * n;
  double2* Ug = scratch;           // Uinv (global)
  double2* Tg = scratch + n * n;   // A Uinv (global)
  __shared__ int rank[kMaxSmall];
  __shared__ double wd[kMaxSmall];
  if (B) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) S0[e] = B[e];
    __syncthreads();
    const int fail = block_cholesky_upper(S0, n);
    if (fail) { if (threadIdx.x == 0) *status = 1; return; }
    block_upper_inverse(S0, n, S1);             // Uinv in shared memory
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) Ug[e] = S1[e];
    // T = A Uinv  (Uinv upper: k <= j), A staged into S0
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) S0[e] = A[e];
    __syncthreads();
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e / n, j = e % n;
      double2 s = make_double2(0.0, 0.0);
      for (int k = 0; k <= j; ++k) cfma(s, S0[i * n + k], S1[k * n + j]);
      Tg[e] = s;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) S0[e] = Tg[e];
    __syncthreads();
    // C = Uinv^H T (k <= i) into Tg, then Hermitised into S0
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e / n, j = e % n;
      double2 s = make_double2(0.0, 0.0);
      for (int k = 0; k <= i; ++k) cfmac(s, S1[k * n + i], S0[k * n + j]);
      Tg[e] = s;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) S1[e] = Tg[e];
    __syncthreads();
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e / n, j = e % n;
      const double2 a = S1[i * n + j], b = S1[j * n + i];
      S0[e] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
    }
    __syncthreads();
  } else {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e / n, j = e % n;
      const double2 a = A[i * n + j], b = A[j * n + i];
      S0[e] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < n * n; e += blockDim.x)
    S1[e] = make_double2((e / n == e % n) ? 1.0 : 0.0, 0.0);
  __syncthreads();
  block_jacobi(S0, S1, n);
  for (int i = threadIdx.x; i < n; i += blockDim.x) wd[i] = S0[i * n + i].x;
  __syncthreads();
  int bad = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    int r = 0;
    const double wi = wd[i];
    if (!isfinite(wi)) bad = 1;
    for (int j = 0; j < n; ++j) {
      const double wj = wd[j];
      r += (wj < wi) || (wj == wi && j < i);
    }
    rank[i] = r;
    w[r] = wi;
  }
  bad = __syncthreads_or(bad);
  // Vout[:, rank[j]] = (Uinv) W[:, j]
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    double2 s;
    if (B) {
      s = make_double2(0.0, 0.0);
      for (int k = i; k < n; ++k) cfma(s, Ug[i * n + k], S1[k * n + j]);
    } else {
      s = S1[i * n + j];
    }
    Vout[i * n + rank[j]] = s;
  }
  if (threadIdx.x == 0) *status = bad ? 2 : 0;
}

int launch_eigh(const double2* A, const double2* B, int n, double* w, double2* V,
                double2* scratch, int* status, cudaStream_t st) {
  if (n < 1 || n > kMaxSmall) { set_error("eigh dimension out of range"); return QDKP_ERR_ARG; }
  const size_t smem = 2 * (size_t)n * n * sizeof(double2);
  QDKP_CUDA_TRY(cudaFuncSetAttribute(eigh_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  eigh_kernel<<<1, kSmallThreads, smem, st>>>(A, B, n, w, V, scratch, status);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

}  // namespace qdkp
