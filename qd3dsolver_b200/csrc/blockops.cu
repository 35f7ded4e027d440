// Tall-skinny block kernels (norms, residual gather, Gram, block update) and one-CTA FP64
// small dense kernels (Cholesky + triangular inverse, Hermitian generalized eigensolver by
// parallel cyclic Jacobi) for the LOBPCG driver.
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
  reduce_partials<<<1, 32, 0, st>>>(partial, nparts, m, out);
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
constexpr int kGramRows = 8;
constexpr int kGramMaxOut = (kMaxSmall * kMaxSmall + kTallThreads - 1) / kTallThreads;
constexpr int kGramParts = 592;

__device__ __forceinline__ double2 list_elem(const BlockList<double>& L, long long r, int c) {
  int b = 0;
  while (b < L.nblk - 1 && c >= L.cols[b]) { c -= L.cols[b]; ++b; }
  return L.p[b][r * L.ld[b] + c];
}

__global__ void __launch_bounds__(kTallThreads)
gram_partial_kernel(const BlockList<double> A, const BlockList<double> B, long long n,
                    long long rows_per_part, double2* __restrict__ partial) {
  extern __shared__ double2 gsm[];
  const int P = A.total(), Q = B.total();
  double2* sA = gsm;
  double2* sB = gsm + kGramRows * P;
  const long long r0 = blockIdx.x * rows_per_part;
  const long long r1 = min(n, r0 + rows_per_part);
  const int PQ = P * Q;
  double2 acc[kGramMaxOut];
#pragma unroll
  for (int k = 0; k < kGramMaxOut; ++k) acc[k] = make_double2(0.0, 0.0);
  for (long long rt = r0; rt < r1; rt += kGramRows) {
    for (int e = threadIdx.x; e < kGramRows * P; e += blockDim.x) {
      const int row = e / P, col = e - row * P;
      sA[e] = rt + row < r1 ? list_elem(A, rt + row, col) : make_double2(0.0, 0.0);
    }
    for (int e = threadIdx.x; e < kGramRows * Q; e += blockDim.x) {
      const int row = e / Q, col = e - row * Q;
      sB[e] = rt + row < r1 ? list_elem(B, rt + row, col) : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kGramMaxOut; ++k) {
      const int o = threadIdx.x + k * kTallThreads;
      if (o < PQ) {
        const int i = o / Q, j = o - i * Q;
#pragma unroll
        for (int row = 0; row < kGramRows; ++row) cfmac(acc[k], sA[row * P + i], sB[row * Q + j]);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < kGramMaxOut; ++k) {
    const int o = threadIdx.x + k * kTallThreads;
    if (o < PQ) partial[(long long)blockIdx.x * PQ + o] = acc[k];
  }
}

__global__ void gram_reduce_kernel(const double2* __restrict__ partial, int nparts, int PQ,
                                   double2* __restrict__ out) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o < PQ) {
    double2 s = make_double2(0.0, 0.0);
    for (int b = 0; b < nparts; ++b) {
      const double2 v = partial[(long long)b * PQ + o];
      s.x += v.x; s.y += v.y;
    }
    out[o] = s;
  }
}

size_t gram_partial_elems(int P, int Q) { return (size_t)kGramParts * P * Q; }

int launch_gram(const BlockList<double>& A, const BlockList<double>& B, long long n,
                double2* partial, size_t partial_elems, double2* out, cudaStream_t st) {
  const int P = A.total(), Q = B.total();
  if (P > kMaxSmall || Q > kMaxSmall || P <= 0 || Q <= 0) {
    set_error("gram dimensions out of range");
    return QDKP_ERR_ARG;
  }
  long long parts = (n + 63) / 64;
  if (parts > kGramParts) parts = kGramParts;
  if (parts < 1) parts = 1;
  long long rpp = (n + parts - 1) / parts;
  rpp = (rpp + kGramRows - 1) / kGramRows * kGramRows;
  parts = (n + rpp - 1) / rpp;
  if ((size_t)parts * P * Q > partial_elems) { set_error("gram partial buffer too small"); return QDKP_ERR_WORKSPACE; }
  const size_t smem = (size_t)kGramRows * (P + Q) * sizeof(double2);
  gram_partial_kernel<<<(unsigned)parts, kTallThreads, smem, st>>>(A, B, n, rpp, partial);
  gram_reduce_kernel<<<(P * Q + 255) / 256, 256, 0, st>>>(partial, (int)parts, P * Q, out);
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

// ------------------------------------------------------------------------------------------------
// Block update: Y = beta Y + sum_k A_k C_k  (C_k row-major cols_k x q)
// ------------------------------------------------------------------------------------------------
struct CoefList {
  const double2* c[3];
};

__global__ void __launch_bounds__(kTallThreads)
update_kernel(const BlockList<double> A, const CoefList C, int q, long long n,
              double2* Y, long long ldy, int accumulate) {
  extern __shared__ double2 csm[];
  int off[3];
  int tot = 0;
  for (int b = 0; b < A.nblk; ++b) { off[b] = tot; tot += A.cols[b]; }
  for (int e = threadIdx.x; e < tot * q; e += blockDim.x) {
    const int row = e / q;
    int b = 0;
    while (b < A.nblk - 1 && row >= off[b] + A.cols[b]) ++b;
    csm[e] = C.c[b][(row - off[b]) * q + (e - row * q)];
  }
  __syncthreads();
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    double2 acc[kMaxBlock];
#pragma unroll
    for (int c = 0; c < kMaxBlock; ++c)
      acc[c] = (accumulate && c < q) ? Y[r * ldy + c] : make_double2(0.0, 0.0);
    for (int b = 0; b < A.nblk; ++b) {
      const double2* __restrict__ a = A.p[b] + r * A.ld[b];
      for (int i = 0; i < A.cols[b]; ++i) {
        const double2 v = a[i];
        const double2* crow = csm + (off[b] + i) * q;
#pragma unroll
        for (int c = 0; c < kMaxBlock; ++c)
          if (c < q) cfma(acc[c], crow[c], v);
      }
    }
#pragma unroll
    for (int c = 0; c < kMaxBlock; ++c)
      if (c < q) Y[r * ldy + c] = acc[c];
  }
}

int launch_update(const BlockList<double>& A, const double2* const* C, int q, long long n,
                  double2* Y, long long ldy, int accumulate, cudaStream_t st) {
  if (q > kMaxBlock || A.total() > kMaxSmall) { set_error("update dimensions out of range"); return QDKP_ERR_ARG; }
  CoefList cl;
  for (int b = 0; b < 3; ++b) cl.c[b] = b < A.nblk ? C[b] : nullptr;
  const size_t smem = (size_t)A.total() * q * sizeof(double2);
  long long blocks = (n + kTallThreads - 1) / kTallThreads;
  if (blocks > 148 * 8) blocks = 148 * 8;
  update_kernel<<<(unsigned)blocks, kTallThreads, smem, st>>>(A, cl, q, n, Y, ldy, accumulate);
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
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) ssm[e] = G[e];
  __syncthreads();
  const int fail = block_cholesky_upper(ssm, n);
  if (threadIdx.x == 0) *status = fail;
  if (fail) return;
  block_upper_inverse(ssm, n, Uinv);
}

int launch_chol_inv(const double2* G, int n, double2* Uinv, int* status, cudaStream_t st) {
  if (n < 1 || n > kMaxSmall) { set_error("chol_inv dimension out of range"); return QDKP_ERR_ARG; }
  const size_t smem = (size_t)n * n * sizeof(double2);
  QDKP_CUDA_TRY(cudaFuncSetAttribute(chol_inv_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  chol_inv_kernel<<<1, kSmallThreads, smem, st>>>(G, n, Uinv, status);
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
  const int n2 = n + (n & 1);
  const int npair = n2 / 2;
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
          if (ac > 1e-300 && ac > 2.2e-16 * sqrt(fabs(a) * fabs(b))) {
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
    block_upper_inverse(S0, n, Ug);
    __threadfence_block();
    __syncthreads();
    // T = A Uinv  (Uinv upper: k <= j)
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e / n, j = e % n;
      double2 s = make_double2(0.0, 0.0);
      for (int k = 0; k <= j; ++k) cfma(s, A[i * n + k], Ug[k * n + j]);
      Tg[e] = s;
    }
    __threadfence_block();
    __syncthreads();
    // C = Uinv^H T (k <= i), Hermitised
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e / n, j = e % n;
      double2 s = make_double2(0.0, 0.0);
      for (int k = 0; k <= i; ++k) cfmac(s, Ug[k * n + i], Tg[k * n + j]);
      S1[e] = s;
    }
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
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

}  // namespace qdkp
