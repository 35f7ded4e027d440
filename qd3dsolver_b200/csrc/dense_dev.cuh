// Device building blocks shared by the single-solve and batched LOBPCG kernels: FP64 MMA,
// block-list element access, and the one-CTA Cholesky / triangular inverse / Hermitian
// eigensolver routines.
#pragma once
#include "blockops.cuh"

namespace qdkp {

static __device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}


constexpr int kStageBudget = 64 * 1024;    // shared memory for the row stages of one CTA

// Stages in flight: as many (2..4) as fit the budget, so that a CTA keeps several chunk loads
// outstanding while it works on one (the kernels are latency- or bandwidth-bound otherwise).
__host__ __device__ __forceinline__ int stage_count(size_t stage_bytes) {
  const int ns = (int)(kStageBudget / stage_bytes);
  return ns < 2 ? 2 : (ns > 4 ? 4 : ns);
}

// Dynamic shared memory this launch was given (the %dynamic_smem_size special register). The
// staged kernels fit their stage count and chunk size into it, so a product narrower than the
// one the launch was sized for can never over-run its allocation.
__device__ __forceinline__ unsigned dyn_smem_bytes() {
  unsigned r;
  asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(r));
  return r;
}

// Stages (2..4) of `stage_bytes` that fit both the budget and `avail` bytes.
__device__ __forceinline__ int stage_count_fit(size_t stage_bytes, size_t avail) {
  int ns = stage_count(stage_bytes);
  while (ns > 2 && (size_t)ns * stage_bytes > avail) --ns;
  return ns;
}

// cp.async.wait_group takes an immediate: wait until at most n (0..3) groups are pending
__device__ __forceinline__ void cp_async_wait_pending(int n) {
  if (n >= 3) asm volatile("cp.async.wait_group 3;\n" ::: "memory");
  else if (n == 2) asm volatile("cp.async.wait_group 2;\n" ::: "memory");
  else if (n == 1) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
  else asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

template <typename T>
static __device__ __forceinline__ double2 list_elem(const BlockList<T>& L, long long r, int c) {
  int b = 0;
  while (b < L.nblk - 1 && c >= L.cols[b]) { c -= L.cols[b]; ++b; }
  const cplx<T> v = L.p[b][r * L.ld[b] + c];
  return make_double2((double)v.x, (double)v.y);
}


// In-place upper Cholesky of the Hermitian matrix in S (n x n, ld n): S = U^H U, U in the upper
// triangle. Returns nonzero (block-uniform) if a pivot is not positive and finite.
static __device__ int block_cholesky_upper(double2* S, int n) {
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
static __device__ void block_upper_inverse(const double2* S, int n, double2* out) {
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


// Eigen-decomposition of the Hermitian C in S0 (n x n, shared memory), with S1 = I on entry:
// Householder reduction to tridiagonal form (C <- H C H, Q <- Q H, H = I - tau v v^H, one column
// per step), a diagonal phase that makes the sub-diagonal real, and the implicit QL iteration
// with shifts of Bowdler, Martin, Reinsch and Wilkinson (the tql2 scheme) on the real symmetric
// tridiagonal matrix. One thread runs the QL recurrences and records each sweep's plane
// rotations; then every row of the eigenvector matrix Z applies them, so the rotations stay
// exactly orthogonal even inside clusters of (near-)equal eigenvalues. On return S0's diagonal
// holds the eigenvalues (unsorted) and S1 the eigenvectors of C (columns). gtmp: n * n global
// double2 of scratch. Returns nonzero (block-uniform) if an eigenvalue needed more than 60 QL
// iterations (only non-finite input gets there).
static __device__ int block_tql(double2* S0, double2* S1, int n, double2* gtmp) {
  __shared__ double2 hv[kMaxSmall], hp[kMaxSmall], hq[kMaxSmall], ph[kMaxSmall];
  __shared__ double td[kMaxSmall], tb[kMaxSmall], rc[kMaxSmall], rs[kMaxSmall];
  __shared__ int ri[kMaxSmall];
  __shared__ double s_tau, s_K;
  __shared__ int s_nrot, s_state;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  // ---- Householder reduction ----
  for (int k = 0; k + 2 < n; ++k) {
    if (warp == 0) {
      double nx2 = 0.0;
      for (int i = k + 1 + lane; i < n; i += 32) {
        const double2 x = S0[i * n + k];
        nx2 += x.x * x.x + x.y * x.y;
      }
      for (int o = 16; o > 0; o >>= 1) nx2 += __shfl_xor_sync(0xffffffffu, nx2, o);
      const double2 x0 = S0[(k + 1) * n + k];
      const double ax0 = sqrt(x0.x * x0.x + x0.y * x0.y);
      const double nx = sqrt(nx2);
      // alpha = -phase(x0) |x|; v = x - alpha e_1; v^H v = 2 |x| (|x| + |x0|)
      const double2 phs = ax0 > 0.0 ? make_double2(x0.x / ax0, x0.y / ax0) : make_double2(1.0, 0.0);
      for (int i = lane; i < n; i += 32) {
        double2 v = make_double2(0.0, 0.0);
        if (i == k + 1) v = make_double2(x0.x + phs.x * nx, x0.y + phs.y * nx);
        else if (i > k + 1) v = S0[i * n + k];
        hv[i] = v;
      }
      // a column whose |x| (|x| + |x0|) is below the smallest normal double is left as it is
      // (entries of that size do not change a tridiagonal of a matrix of ordinary scale; 1 / it
      // would overflow)
      const double den = nx * (nx + ax0);
      if (lane == 0) s_tau = den >= 2.2250738585072014e-308 ? 1.0 / den : 0.0;
    }
    __syncthreads();
    const double tau = s_tau;
    // every thread has read tau before warp 0 can move on to the next column and rewrite it
    __syncthreads();
    if (tau == 0.0) continue;                      // column already reduced (uniform)
    // p = tau C v and q = Q v, a warp per row
    for (int i = warp; i < n; i += nwarps) {
      double2 sp = make_double2(0.0, 0.0), sq = make_double2(0.0, 0.0);
      for (int j = k + 1 + lane; j < n; j += 32) {
        const double2 v = hv[j];
        cfma(sp, S0[i * n + j], v);
        cfma(sq, S1[i * n + j], v);
      }
      for (int o = 16; o > 0; o >>= 1) {
        sp.x += __shfl_xor_sync(0xffffffffu, sp.x, o); sp.y += __shfl_xor_sync(0xffffffffu, sp.y, o);
        sq.x += __shfl_xor_sync(0xffffffffu, sq.x, o); sq.y += __shfl_xor_sync(0xffffffffu, sq.y, o);
      }
      if (lane == 0) { hp[i] = make_double2(tau * sp.x, tau * sp.y); hq[i] = sq; }
    }
    __syncthreads();
    if (warp == 0) {                               // K = tau / 2 v^H p
      double2 s = make_double2(0.0, 0.0);
      for (int i = k + 1 + lane; i < n; i += 32) cfmac(s, hv[i], hp[i]);
      for (int o = 16; o > 0; o >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, o); s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
      }
      // v^H C v is real for Hermitian C; its rounding residue in s.y is dropped
      if (lane == 0) s_K = 0.5 * tau * s.x;
    }
    __syncthreads();
    const double K = s_K;
    // C <- C - v w^H - w v^H with w = p - K v;  Q <- Q - tau q v^H
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e / n, j = e - i * n;
      const double2 vi = hv[i], vj = hv[j];
      const double2 wi = make_double2(hp[i].x - K * vi.x, hp[i].y - K * vi.y);
      const double2 wj = make_double2(hp[j].x - K * vj.x, hp[j].y - K * vj.y);
      double2 c = S0[e];
      // c -= vi conj(wj) + wi conj(vj)
      c.x -= vi.x * wj.x + vi.y * wj.y + wi.x * vj.x + wi.y * vj.y;
      c.y -= vi.y * wj.x - vi.x * wj.y + wi.y * vj.x - wi.x * vj.y;
      S0[e] = c;
      const double2 qi = hq[i];
      double2 q = S1[e];
      q.x -= tau * (qi.x * vj.x + qi.y * vj.y);
      q.y -= tau * (qi.y * vj.x - qi.x * vj.y);
      S1[e] = q;
    }
    __syncthreads();
  }
  // ---- real tridiagonal form: D^H T D with D = diag(ph), ph_{i+1} = ph_i e_i / |e_i| ----
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    td[i] = S0[i * n + i].x;
    hv[i] = i + 1 < n ? S0[(i + 1) * n + i] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double2 p = make_double2(1.0, 0.0);
    for (int i = 0; i < n; ++i) {
      ph[i] = p;
      const double2 e = hv[i];
      const double ae = sqrt(e.x * e.x + e.y * e.y);
      tb[i] = ae;
      if (ae > 0.0) p = cmul(p, make_double2(e.x / ae, e.y / ae));
    }
    tb[n - 1] = 0.0;
  }
  __syncthreads();
  double* Z = reinterpret_cast<double*>(S0);       // S0 is free now: n x n real
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e - i * n;
    S1[e] = cmul(S1[e], ph[j]);
    Z[e] = i == j ? 1.0 : 0.0;
  }
  // ---- implicit QL; thread 0 carries the iteration state across sweeps ----
  int l = 0, it = 0, fail = 0;
  for (;;) {
    if (threadIdx.x == 0) {
      int nrot = 0, state = 0;                     // 0: a sweep to apply, 1: finished
      for (;;) {
        if (l >= n) { state = 1; break; }
        int m = l;
        for (; m < n - 1; ++m) {
          const double dd = fabs(td[m]) + fabs(td[m + 1]);
          if (fabs(tb[m]) <= 2.220446049250313e-16 * dd || fabs(tb[m]) < 1e-300) break;
        }
        if (m == l) { ++l; it = 0; continue; }
        if (++it > 60) { fail = 1; state = 1; break; }
        double g = (td[l + 1] - td[l]) / (2.0 * tb[l]);
        double r = sqrt(g * g + 1.0);
        g = td[m] - td[l] + tb[l] / (g + (g >= 0.0 ? r : -r));
        double s = 1.0, c = 1.0, p = 0.0;
        bool early = false;
        for (int i = m - 1; i >= l; --i) {
          const double f = s * tb[i], bb = c * tb[i];
          const double h2 = f * f + g * g;
          if (h2 == 0.0) { td[i + 1] -= p; tb[i + 1] = 0.0; tb[m] = 0.0; early = true; break; }
          const double inv = rsqrt(h2);
          tb[i + 1] = h2 * inv;
          s = f * inv; c = g * inv;
          g = td[i + 1] - p;
          r = (td[i] - g) * s + 2.0 * c * bb;
          p = s * r;
          td[i + 1] = g + p;
          g = c * r - bb;
          ri[nrot] = i; rc[nrot] = c; rs[nrot] = s; ++nrot;
        }
        if (!early) { td[l] -= p; tb[l] = g; tb[m] = 0.0; }
        break;
      }
      s_nrot = nrot; s_state = state | (fail << 1);
    }
    __syncthreads();
    const int nrot = s_nrot, state = s_state;
    for (int row = threadIdx.x; row < n; row += blockDim.x) {
      double* z = Z + row * n;
      for (int u = 0; u < nrot; ++u) {
        const int i = ri[u];
        const double c = rc[u], s = rs[u];
        const double f = z[i + 1];
        z[i + 1] = s * z[i] + c * f;
        z[i] = c * z[i] - s * f;
      }
    }
    __syncthreads();
    if (state & 1) { fail = state >> 1; break; }
  }
  // ---- V = (Q D) Z into S1, eigenvalues onto S0's diagonal ----
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e - i * n;
    double2 v = make_double2(0.0, 0.0);
    for (int k = 0; k < n; ++k) caxpy(v, Z[k * n + j], S1[i * n + k]);
    gtmp[e] = v;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) S1[e] = gtmp[e];
  for (int i = threadIdx.x; i < n; i += blockDim.x) S0[i * n + i] = make_double2(td[i], 0.0);
  __syncthreads();
  return fail;
}


// Partial Gram sums reduced by the CTAs that finish last, with no waiting. The partials
// (RP x RQ real each, one per part, `parts` of them) form `split` groups of consecutive parts;
// every CTA of the launch (all parts, all column panels on blockIdx.y) counts itself in its
// group's counter once its partial is written; the last of a group sums the group's partials
// in part order into the group's slot after the partials, and the last group to finish folds
// the group sums, in group order, into the complex P x Q result. The CTA that completes a count
// resets it to zero. Sums and their order are those of a two-pass reduction.
static __device__ void gram_finish_last(double* __restrict__ partial, int parts, int split,
                                        int* __restrict__ counters, int P, int Q, int part,
                                        double2* __restrict__ out) {
  __shared__ int s_last;
  const int RP = (2 * P + 7) / 8 * 8, RQ = (2 * Q + 7) / 8 * 8;
  const int elems = RP * RQ;
  const int per = (parts + split - 1) / split;
  const int ngroups = (parts + per - 1) / per;
  const int grp = part / per;
  const int b0 = grp * per, b1 = min(parts, b0 + per);
  __threadfence();                                   // this CTA's partial, device-wide
  __syncthreads();
  if (threadIdx.x == 0) {
    const int members = (b1 - b0) * (int)gridDim.y;
    s_last = atomicAdd(&counters[grp], 1) == members - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double* sums = partial + (long long)(parts + grp) * elems;
  for (int e = threadIdx.x; e < elems; e += blockDim.x) {
    double acc = 0.0;
    for (int b = b0; b < b1; ++b) acc += __ldcg(partial + (long long)b * elems + e);
    sums[e] = acc;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    counters[grp] = 0;
    s_last = atomicAdd(&counters[split], 1) == ngroups - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  for (int o = threadIdx.x; o < P * Q; o += blockDim.x) {
    const int i = o / Q, j = o - i * Q;
    const long long rr = (long long)(2 * i) * RQ + 2 * j;   // C'_{2i,2j}
    double re = 0.0, im = 0.0;
    for (int g = 0; g < ngroups; ++g) {
      const double* c = partial + (long long)(parts + g) * elems;
      re += __ldcg(c + rr) + __ldcg(c + rr + RQ + 1);
      im += __ldcg(c + rr + 1) - __ldcg(c + rr + RQ);
    }
    out[o] = make_double2(re, im);
  }
  if (threadIdx.x == 0) counters[split] = 0;
}

// =============================================================================================
// Rayleigh-Ritz eigensolve for the wanted eigenpairs only: LOBPCG keeps the m smallest of the
// 3m Ritz pairs, so the tridiagonal problem is solved for those alone, by multisection with
// Sturm counts and inverse iteration, which run in parallel where the QL recurrence is serial.
// Every routine is CTA-wide for 512 threads (16 warps); block-uniform return codes.
// =============================================================================================
constexpr int kRrWarps = 16;

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// integer mixing (xorshift-multiply) for deterministic pseudo-random start vectors
__device__ __forceinline__ unsigned mix32(unsigned x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}
__device__ __forceinline__ double start_value(int i, int j) {
  return (double)(mix32((unsigned)(i * 131 + j * 7919 + 17)) >> 8) * (1.0 / 8388608.0) - 1.0;
}

struct RrShared {
  double td[kMaxSmall], tb[kMaxSmall], e2[kMaxSmall], tau[kMaxSmall], rinv[kMaxSmall];
  double lam[kMaxSmall];
  double2 esub[kMaxSmall], ph[kMaxSmall], xcol[kMaxSmall], psm[kMaxSmall];
  double G[kMaxBlock * kMaxBlock];
  double lo, hi;
  int bad;
};

// Upper Cholesky B = U^H U in place (S, ld n), one barrier per column: step k subtracts
// conj(S_ki) S_kj / S_kk from S_ij (k < i <= j) with the unscaled pivot row; the rows are scaled
// by 1 / sqrt(S_kk) at the end. rinv = 1 / U_kk. Returns nonzero on a bad pivot.
static __device__ int rr_cholesky(double2* __restrict__ S, int n, double* __restrict__ rinv) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwp = blockDim.x >> 5;
  for (int k = 0; k < n; ++k) {
    const double d = S[k * n + k].x;
    if (!(d > 0.0) || !isfinite(d)) { __syncthreads(); return 1; }
    const double inv = 1.0 / d;
    for (int i = k + 1 + warp; i < n; i += nwp) {
      const double2 a = S[k * n + i];
      for (int j = i + lane; j < n; j += 32) {
        const double2 b = S[k * n + j];
        double2 t = S[i * n + j];
        t.x -= (a.x * b.x + a.y * b.y) * inv;
        t.y -= (a.x * b.y - a.y * b.x) * inv;
        S[i * n + j] = t;
      }
    }
    __syncthreads();
  }
  for (int k = threadIdx.x; k < n; k += blockDim.x) rinv[k] = 1.0 / sqrt(S[k * n + k].x);
  __syncthreads();
  for (int i = warp; i < n; i += nwp)
    for (int j = i + lane; j < n; j += 32) {
      const double r = rinv[i];
      if (j == i) S[i * n + j] = make_double2(1.0 / r, 0.0);
      else { S[i * n + j].x *= r; S[i * n + j].y *= r; }
    }
  __syncthreads();
  return 0;
}

// Rows of A (ld n) times U^-1 (U upper, pivots as reciprocals rinv): a warp per row (rows
// warp + 16 r), the row in registers (lane l holds columns l + 32 q), w_k = a_k / U_kk broadcast
// by a shuffle, then a_j -= w_k U_kj. Written conjugate-transposed (row i into column i) when
// `trans`, in place otherwise; every row is read before any is written.
template <int R, int CC>
static __device__ void rr_rows_solve(double2* __restrict__ A, const double2* __restrict__ U,
                                     int n, const double* __restrict__ rinv, bool trans) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double2 a[R][CC];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int q = 0; q < CC; ++q) {
      const int i = warp + kRrWarps * r, j = lane + 32 * q;
      a[r][q] = (i < n && j < n) ? A[i * n + j] : make_double2(0.0, 0.0);
    }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    const int kl = k & 31, kq = k >> 5;
    const double rk = rinv[k];
    double2 u[CC];
#pragma unroll
    for (int q = 0; q < CC; ++q) {
      const int j = lane + 32 * q;
      u[q] = (j > k && j < n) ? U[k * n + j] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      double2 ak = a[r][0];
#pragma unroll
      for (int q = 1; q < CC; ++q) if (kq == q) ak = a[r][q];
      ak.x = __shfl_sync(0xffffffffu, ak.x, kl) * rk;
      ak.y = __shfl_sync(0xffffffffu, ak.y, kl) * rk;
#pragma unroll
      for (int q = 0; q < CC; ++q) {
        if (lane + 32 * q == k) a[r][q] = ak;
        a[r][q].x -= ak.x * u[q].x - ak.y * u[q].y;
        a[r][q].y -= ak.x * u[q].y + ak.y * u[q].x;
      }
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int q = 0; q < CC; ++q) {
      const int i = warp + kRrWarps * r, j = lane + 32 * q;
      if (i < n && j < n) {
        if (trans) A[j * n + i] = make_double2(a[r][q].x, -a[r][q].y);
        else A[i * n + j] = a[r][q];
      }
    }
  __syncthreads();
}

// Householder tridiagonalisation of the Hermitian part of Csm (read once), held in registers:
// warp w owns rows w + 16 r, lane l columns l + 32 q. Step k forms the reflector
// H = I - tau v v^H (v^H v = 2 / tau) from column k in every warp (identical butterfly sums),
// p = tau C v row-wise, K = tau / 2 v^H p, w = p - K v and C <- C - v w^H - w v^H; two barriers
// per column. Reflector k (v_j, j > k) is stored in row n - 1 - k of Rf's strict lower triangle
// (v_j at column j - k - 1), tau_k in sh.tau. On return sh.td / sh.tb / sh.e2 hold the real
// tridiagonal T = D^H (Q^H C Q) D, sh.ph the phases D (the off-diagonal made real and >= 0).
template <int R, int CC>
static __device__ void rr_tridiag(const double2* __restrict__ Csm, int n,
                                  double2* __restrict__ Rf, RrShared& sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double2 c[R][CC];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int q = 0; q < CC; ++q) {
      const int i = warp + kRrWarps * r, j = lane + 32 * q;
      if (i < n && j < n) {
        const double2 a = Csm[i * n + j], b = Csm[j * n + i];
        c[r][q] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
      } else {
        c[r][q] = make_double2(0.0, 0.0);
      }
    }
  if (warp == 0)                                   // column 0 is row 0 conjugated
#pragma unroll
    for (int q = 0; q < CC; ++q) {
      const int j = lane + 32 * q;
      if (j < n) sh.xcol[j] = j > 0 ? make_double2(c[0][q].x, -c[0][q].y) : make_double2(0.0, 0.0);
    }
  __syncthreads();
  for (int k = 0; k + 2 < n; ++k) {
    const int j0 = k + 1;
    double2 vs[CC];
    double nx2 = 0.0;
#pragma unroll
    for (int q = 0; q < CC; ++q) {
      const int j = lane + 32 * q;
      vs[q] = (j > k && j < n) ? sh.xcol[j] : make_double2(0.0, 0.0);
      nx2 += vs[q].x * vs[q].x + vs[q].y * vs[q].y;
    }
    nx2 = warp_sum(nx2);
    const double2 x0 = sh.xcol[j0];
    const double ax0 = sqrt(x0.x * x0.x + x0.y * x0.y);
    const double nx = sqrt(nx2);
    // alpha = -phase(x0) |x|, v = x - alpha e_1
    const double2 phs = ax0 > 0.0 ? make_double2(x0.x / ax0, x0.y / ax0) : make_double2(1.0, 0.0);
    // below the smallest normal double the column is left as it is (1 / den would overflow)
    const double den = nx * (nx + ax0);
    const double tau = den >= 2.2250738585072014e-308 ? 1.0 / den : 0.0;
    const double2 v0 = make_double2(x0.x + phs.x * nx, x0.y + phs.y * nx);
#pragma unroll
    for (int q = 0; q < CC; ++q)
      if (lane + 32 * q == j0) vs[q] = v0;
    double2 vr[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = warp + kRrWarps * r;
      vr[r] = (i > j0 && i < n) ? sh.xcol[i] : (i == j0 ? v0 : make_double2(0.0, 0.0));
    }
    if (warp == 0) {
#pragma unroll
      for (int q = 0; q < CC; ++q) {
        const int j = lane + 32 * q;
        if (j > k && j < n) Rf[(n - 1 - k) * n + (j - k - 1)] = vs[q];
      }
      if (lane == 0) sh.tau[k] = tau;
    }
    double2 pr[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      double sx = 0.0, sy = 0.0;
      if (warp + kRrWarps * r >= k)                // rows above k are reduced already
#pragma unroll
        for (int q = 0; q < CC; ++q) {
          sx += c[r][q].x * vs[q].x - c[r][q].y * vs[q].y;
          sy += c[r][q].x * vs[q].y + c[r][q].y * vs[q].x;
        }
      pr[r] = make_double2(sx, sy);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      pr[r].x = tau * warp_sum(pr[r].x);
      pr[r].y = tau * warp_sum(pr[r].y);
    }
    if (lane == 0)
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = warp + kRrWarps * r;
        if (i < n) sh.psm[i] = pr[r];
      }
    __syncthreads();
    double2 pc[CC];
    double s = 0.0;                                // Re v^H p (v^H C v is real)
#pragma unroll
    for (int q = 0; q < CC; ++q) {
      const int j = lane + 32 * q;
      pc[q] = j < n ? sh.psm[j] : make_double2(0.0, 0.0);
      s += vs[q].x * pc[q].x + vs[q].y * pc[q].y;
    }
    const double K = 0.5 * tau * warp_sum(s);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (warp + kRrWarps * r < k) continue;
      const double2 wi = make_double2(pr[r].x - K * vr[r].x, pr[r].y - K * vr[r].y);
      const double2 vi = vr[r];
#pragma unroll
      for (int q = 0; q < CC; ++q) {
        const double2 vj = vs[q];
        const double2 wj = make_double2(pc[q].x - K * vj.x, pc[q].y - K * vj.y);
        c[r][q].x -= vi.x * wj.x + vi.y * wj.y + wi.x * vj.x + wi.y * vj.y;
        c[r][q].y -= vi.y * wj.x - vi.x * wj.y + wi.y * vj.x - wi.x * vj.y;
      }
    }
    // row k is final (diagonal and sub-diagonal); row k + 1, conjugated, is the next column
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = warp + kRrWarps * r;
      if (i == k) {
#pragma unroll
        for (int q = 0; q < CC; ++q) {
          const int j = lane + 32 * q;
          if (j == k) sh.td[k] = c[r][q].x;
          if (j == k + 1) sh.esub[k] = make_double2(c[r][q].x, -c[r][q].y);
        }
      }
      if (i == k + 1) {
#pragma unroll
        for (int q = 0; q < CC; ++q) {
          const int j = lane + 32 * q;
          if (j < n) sh.xcol[j] = j > k + 1 ? make_double2(c[r][q].x, -c[r][q].y) : make_double2(0.0, 0.0);
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {                    // the last two rows
    const int i = warp + kRrWarps * r;
#pragma unroll
    for (int q = 0; q < CC; ++q) {
      const int j = lane + 32 * q;
      if (n >= 2 && i == n - 2) {
        if (j == n - 2) sh.td[n - 2] = c[r][q].x;
        if (j == n - 1) sh.esub[n - 2] = make_double2(c[r][q].x, -c[r][q].y);
      }
      if (i == n - 1 && j == n - 1) sh.td[n - 1] = c[r][q].x;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double2 p = make_double2(1.0, 0.0);
    for (int i = 0; i < n; ++i) {
      sh.ph[i] = p;
      if (i + 1 < n) {
        const double2 e = sh.esub[i];
        const double ae = sqrt(e.x * e.x + e.y * e.y);
        sh.tb[i] = ae;
        sh.e2[i] = ae * ae;
        if (ae > 0.0) p = cmul(p, make_double2(e.x / ae, e.y / ae));
      }
    }
    sh.tb[n - 1] = 0.0;
    sh.e2[n - 1] = 0.0;
  }
  __syncthreads();
}

// Eigenvalues of the tridiagonal below x: sign changes of the leading-minor determinants
// p_{i+1} = (d_i - x) p_i - e_{i-1}^2 p_{i-1} (the Sturm sequence; an FMA per step where the
// ratio form needs a division), both kept in [2^-600, 2^600] by a common power-of-two scale; a
// zero is replaced by -2^-300 times its predecessor (a zero pivot counts as negative).
static __device__ __forceinline__ int rr_sturm(const double* __restrict__ td,
                                               const double* __restrict__ e2, int n, double x) {
  const double big = 0x1p600, small = 0x1p-600;
  double pm = 1.0, p = td[0] - x;
  if (p == 0.0) p = -0x1p-300;
  bool neg = p < 0.0;
  int c = neg;
#pragma unroll 4
  for (int i = 1; i < n; ++i) {
    double pn = fma(td[i] - x, p, -e2[i - 1] * pm);
    pn = pn == 0.0 ? -0x1p-300 * p : pn;
    const double m = fmax(fabs(pn), fabs(p));
    const double f = m > big ? small : (m < small ? big : 1.0);
    pm = p * f; p = pn * f;
    const bool ng = p < 0.0;
    c += ng != neg;
    neg = ng;
  }
  return c;
}

// The nwant smallest eigenpairs of A x = lambda B x (B = nullptr: the identity), A and B n x n
// Hermitian (global, ld n): w[0..nwant) ascending and Vout[:, 0..nwant) (ld n; the other columns
// are zeroed). Steps: B = U^H U (rr_cholesky); C^H = (U^-H A U^-1)^H by two row solves
// (rr_rows_solve); Householder to the real tridiagonal T (rr_tridiag); eigenvalues by
// multisection (G lanes per eigenvalue, Sturm counts, G + 1 sub-intervals per round, down to
// 2 eps ||T||); eigenvectors by two inverse-iteration steps (a thread per eigenvalue, LU of
// T - lambda I with partial pivoting, pseudo-random start), orthonormalised by two Cholesky-QR
// passes; V = U^-1 Q D Z with the reflectors applied in reverse order. Returns 0, 1 (B not
// positive definite), 2 (non-finite T) or 3 (inverse-iteration vectors not independent: the
// caller then solves the full problem). S0 / S1: n x n shared matrices.
template <int R, int CC>
static __device__ int rr_wanted(const double2* __restrict__ A, const double2* __restrict__ B,
                                int n, int nwant, double* __restrict__ w,
                                double2* __restrict__ Vout, double2* S0, double2* S1,
                                RrShared& sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwp = blockDim.x >> 5;
  const double eps = 1.1102230246251565e-16;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) S1[e] = A[e];
  if (B) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) S0[e] = B[e];
    __syncthreads();
    if (rr_cholesky(S0, n, sh.rinv)) return 1;
    rr_rows_solve<R, CC>(S1, S0, n, sh.rinv, true);      // W^H with W = A U^-1
    rr_rows_solve<R, CC>(S1, S0, n, sh.rinv, false);     // W^H U^-1 = C^H
  } else {
    __syncthreads();
  }
  rr_tridiag<R, CC>(S1, n, S0, sh);     // reflectors below S0's diagonal, U above it
  // ---- Gershgorin bounds ----
  if (warp == 0) {
    double lo = INFINITY, hi = -INFINITY;
    for (int i = lane; i < n; i += 32) {
      const double r = (i > 0 ? sh.tb[i - 1] : 0.0) + (i + 1 < n ? sh.tb[i] : 0.0);
      lo = fmin(lo, sh.td[i] - r);
      hi = fmax(hi, sh.td[i] + r);
    }
    lo = warp_min(lo);
    hi = warp_max(hi);
    if (lane == 0) {
      const double tn = fmax(fabs(lo), fabs(hi));
      sh.lo = lo - 4.0 * eps * tn * n - 1e-300;
      sh.hi = hi + 4.0 * eps * tn * n + 1e-300;
      sh.bad = !(isfinite(lo) && isfinite(hi));
    }
  }
  __syncthreads();
  if (sh.bad) return 2;
  const double tn = fmax(fabs(sh.lo), fabs(sh.hi));
  // ---- multisection: lanes t of group g evaluate a + (b - a)(t + 1) / (G + 1) ----
  int G = 32;
  while (G > 1 && nwant * G > (int)blockDim.x) G >>= 1;
  {
    const int g = threadIdx.x / G, t = threadIdx.x % G;
    const int base = lane / G * G;
    const unsigned gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u) << base);
    const bool act = g < nwant;
    double a = sh.lo, b = sh.hi;
    for (int round = 0; round < 64; ++round) {
      const bool conv = !act || (b - a) <= fmax(2.0 * eps * tn, 4.0 * eps * fmax(fabs(a), fabs(b)));
      if (__all_sync(0xffffffffu, conv)) break;
      const double x = a + (b - a) * ((double)(t + 1) / (double)(G + 1));
      const int cnt = rr_sturm(sh.td, sh.e2, n, x);
      const unsigned below = __ballot_sync(0xffffffffu, cnt <= g) & gmask;   // x below lambda_g
      const int hiT = below ? 31 - __clz(below) - base : -1;
      const unsigned above = ~below & gmask;
      const int loT = above ? __ffs(above) - 1 - base : G;
      const double na = hiT >= 0 ? a + (b - a) * ((double)(hiT + 1) / (double)(G + 1)) : a;
      const double nb = loT < G ? a + (b - a) * ((double)(loT + 1) / (double)(G + 1)) : b;
      a = conv ? a : na;
      b = conv ? b : nb;
    }
    if (act && t == 0) sh.lam[g] = 0.5 * (a + b);
  }
  __syncthreads();
  // ---- inverse iteration: arrays interleaved [i][j] in S1 (free after the tridiagonalisation) ----
  const int zs = (n * nwant + 1) & ~1;
  double* Z = reinterpret_cast<double*>(S1);
  double* ur = Z + zs;                  // 1 / pivot of U's row i
  double* u1 = ur + n * nwant;          // U_{i,i+1}
  double* u2 = u1 + n * nwant;          // U_{i,i+2} (from row exchanges)
  const double tiny = eps * tn + 1e-300;
  if ((int)threadIdx.x < nwant) {
    const int j = threadIdx.x;
    const double mu = sh.lam[j];
    for (int i = 0; i < n; ++i) Z[i * nwant + j] = start_value(i, j);
    for (int step = 0; step < 2; ++step) {
      // forward: factor T - mu I row by row, exchanging rows when the sub-diagonal is larger,
      // and eliminate the right-hand side alongside
      double a = sh.td[0] - mu, bcur = n > 1 ? sh.tb[0] : 0.0;
      double y = Z[j];
      for (int i = 0; i + 1 < n; ++i) {
        const double cc = sh.tb[i];
        const double an = sh.td[i + 1] - mu;
        const double bn = i + 2 < n ? sh.tb[i + 1] : 0.0;
        const double yn = Z[(i + 1) * nwant + j];
        const bool sw = fabs(a) < fabs(cc);
        const double ap = fabs(a) < tiny ? (a < 0.0 ? -tiny : tiny) : a;
        const double ri = 1.0 / (sw ? cc : ap);
        const double l = (sw ? a : cc) * ri;
        ur[i * nwant + j] = ri;
        u1[i * nwant + j] = sw ? an : bcur;
        u2[i * nwant + j] = sw ? bn : 0.0;
        Z[i * nwant + j] = sw ? yn : y;
        const double na = sw ? bcur - l * an : an - l * bcur;
        const double ny = sw ? y - l * yn : yn - l * y;
        bcur = sw ? -l * bn : bn;
        a = na;
        y = ny;
      }
      const double ap = fabs(a) < tiny ? (a < 0.0 ? -tiny : tiny) : a;
      ur[(n - 1) * nwant + j] = 1.0 / ap;
      u1[(n - 1) * nwant + j] = 0.0;
      u2[(n - 1) * nwant + j] = 0.0;
      Z[(n - 1) * nwant + j] = y;
      double x1 = 0.0, x2 = 0.0, mx = 0.0;          // back substitution
      for (int i = n - 1; i >= 0; --i) {
        const double x = (Z[i * nwant + j] - u1[i * nwant + j] * x1 - u2[i * nwant + j] * x2) * ur[i * nwant + j];
        Z[i * nwant + j] = x;
        x2 = x1;
        x1 = x;
        mx = fmax(mx, fabs(x));
      }
      const double sc = mx > 0.0 && isfinite(mx) ? 1.0 / mx : 0.0;
      for (int i = 0; i < n; ++i) Z[i * nwant + j] *= sc;
    }
  }
  __syncthreads();
  // ---- Cholesky-QR, twice: G = Z^T Z (a thread per entry), G = R^T R (warp 0; the diagonal
  //      holds 1 / R_kk), Z <- Z R^-1 (a thread per row, the row in registers) ----
  const int ng = nwant * (nwant + 1) / 2;
  for (int pass = 0; pass < 2; ++pass) {
    for (int e = threadIdx.x; e < ng; e += blockDim.x) {
      int a = 0, rem = e;
      while (rem >= nwant - a) { rem -= nwant - a; ++a; }
      const int b = a + rem;
      double d = 0.0;
      for (int i = 0; i < n; ++i) d = fma(Z[i * nwant + a], Z[i * nwant + b], d);
      sh.G[a * nwant + b] = d;
      sh.G[b * nwant + a] = d;
    }
    __syncthreads();
    if (warp == 0) {
      int bad = 0;
      for (int k = 0; k < nwant; ++k) {
        const double d0 = sh.G[k * nwant + k];
        __syncwarp();
        // the vectors have max-abs 1 (first pass) or unit norm (second): a pivot this small means
        // a vector (nearly) in the span of the previous ones
        if (!(d0 > 1e-10) || !isfinite(d0)) bad = 1;
        const double ri = bad ? 0.0 : 1.0 / sqrt(d0);
        for (int j = k + lane; j < nwant; j += 32) sh.G[k * nwant + j] = j == k ? ri : sh.G[k * nwant + j] * ri;
        __syncwarp();
        for (int j = k + 1 + lane; j < nwant; j += 32) {
          const double gkj = sh.G[k * nwant + j];
          for (int i = k + 1; i <= j; ++i) sh.G[i * nwant + j] -= sh.G[k * nwant + i] * gkj;
        }
        __syncwarp();
      }
      if (lane == 0) sh.bad = bad;
    }
    __syncthreads();
    if (sh.bad) return 3;
    if ((int)threadIdx.x < n) {
      const int i = threadIdx.x;
      double z[kMaxBlock];
#pragma unroll
      for (int k = 0; k < kMaxBlock; ++k) z[k] = k < nwant ? Z[i * nwant + k] : 0.0;
#pragma unroll
      for (int k = 0; k < kMaxBlock; ++k) {
        if (k < nwant) {
          z[k] *= sh.G[k * nwant + k];
#pragma unroll
          for (int jj = k + 1; jj < kMaxBlock; ++jj)
            if (jj < nwant) z[jj] -= z[k] * sh.G[k * nwant + jj];
        }
      }
#pragma unroll
      for (int k = 0; k < kMaxBlock; ++k) if (k < nwant) Z[i * nwant + k] = z[k];
    }
    __syncthreads();
  }
  // ---- V = U^-1 Q D Z: a warp per column, the column in registers (lane l holds rows l + 32 q):
  //      phases, reflectors n-3 .. 0, back substitution ----
  for (int j = warp; j < nwant; j += nwp) {
    double2 y[CC];
#pragma unroll
    for (int q = 0; q < CC; ++q) {
      const int i = lane + 32 * q;
      const double z = i < n ? Z[i * nwant + j] : 0.0;
      y[q] = i < n ? make_double2(sh.ph[i].x * z, sh.ph[i].y * z) : make_double2(0.0, 0.0);
    }
    for (int k = n - 3; k >= 0; --k) {
      const double tk = sh.tau[k];
      const double2* vrow = S0 + (n - 1 - k) * n - (k + 1);   // v_i at vrow[i], i > k
      double2 v[CC];
      double sx = 0.0, sy = 0.0;                                // v^H y
#pragma unroll
      for (int q = 0; q < CC; ++q) {
        const int i = lane + 32 * q;
        v[q] = (i > k && i < n) ? vrow[i] : make_double2(0.0, 0.0);
        sx += v[q].x * y[q].x + v[q].y * y[q].y;
        sy += v[q].x * y[q].y - v[q].y * y[q].x;
      }
      sx = tk * warp_sum(sx);
      sy = tk * warp_sum(sy);
#pragma unroll
      for (int q = 0; q < CC; ++q) {
        y[q].x -= v[q].x * sx - v[q].y * sy;
        y[q].y -= v[q].x * sy + v[q].y * sx;
      }
    }
    if (B) {
      for (int k = n - 1; k >= 0; --k) {
        const int kl = k & 31, kq = k >> 5;
        double2 yk = y[0];
#pragma unroll
        for (int q = 1; q < CC; ++q) if (kq == q) yk = y[q];
        const double r = sh.rinv[k];
        const double2 xk = make_double2(__shfl_sync(0xffffffffu, yk.x, kl) * r,
                                        __shfl_sync(0xffffffffu, yk.y, kl) * r);
#pragma unroll
        for (int q = 0; q < CC; ++q) {
          const int i = lane + 32 * q;
          if (i == k) y[q] = xk;
          const double2 u = i < k ? S0[i * n + k] : make_double2(0.0, 0.0);
          y[q].x -= u.x * xk.x - u.y * xk.y;
          y[q].y -= u.x * xk.y + u.y * xk.x;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < CC; ++q) {
      const int i = lane + 32 * q;
      if (i < n) Vout[i * n + j] = y[q];
    }
  }
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e - i * n;
    if (j >= nwant) Vout[e] = make_double2(0.0, 0.0);
  }
  for (int j = threadIdx.x; j < nwant; j += blockDim.x) w[j] = sh.lam[j];
  __syncthreads();
  return 0;
}

// rr_wanted when it applies (nwant < n, the inverse-iteration arrays fit S1, 512 threads);
// returns -1 when it does not apply
static __device__ int block_eigh_wanted(const double2* __restrict__ A,
                                        const double2* __restrict__ B, int n, int nwant,
                                        double* __restrict__ w, double2* __restrict__ Vout,
                                        double2* S0, double2* S1) {
  __shared__ RrShared sh;
  if (nwant < 1 || nwant >= n || nwant > kMaxBlock || (int)blockDim.x != 32 * kRrWarps ||
      ((n * nwant + 1) & ~1) + 3 * n * nwant > 2 * n * n)
    return -1;
  if (n <= 48) return rr_wanted<3, 2>(A, B, n, nwant, w, Vout, S0, S1, sh);
  return rr_wanted<5, 3>(A, B, n, nwant, w, Vout, S0, S1, sh);
}

// w ascending, V columns permuted accordingly; generalized problem through B = U^H U.
// Returns 0 (ok), 1 (B not positive definite) or 2 (non-finite eigenvalue); block-uniform.
// S0, S1: n x n shared-memory matrices; scratch: 2 n^2 global elements. With 0 < nwant < n only
// the nwant smallest pairs are required (w[0..nwant), V's first nwant columns): block_eigh_wanted
// computes them, the QL path below is taken when it does not apply or its vectors collapse.
static __device__ int block_eigh(const double2* __restrict__ A, const double2* __restrict__ B,
                                 int n, double* __restrict__ w, double2* __restrict__ Vout,
                                 double2* __restrict__ scratch, double2* S0, double2* S1,
                                 int nwant = 0) {
  if (nwant > 0 && nwant < n) {
    const int r = block_eigh_wanted(A, B, n, nwant, w, Vout, S0, S1);
    if (r == 0 || r == 1) return r;                // else: the full problem below
  }
  double2* Ug = scratch;           // Uinv (global)
  double2* Tg = scratch + n * n;   // A Uinv (global)
  __shared__ int rank[kMaxSmall];
  __shared__ double wd[kMaxSmall];
  if (B) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) S0[e] = B[e];
    __syncthreads();
    const int fail = block_cholesky_upper(S0, n);
    if (fail) return 1;
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
  if (block_tql(S0, S1, n, Tg)) return 2;
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
  __syncthreads();
  return bad ? 2 : 0;
}



// Y' = A' C'' for rows [r0, r1) of complex128 blocks on the FP64 MMA (mma.sync.m8n8k4.f64),
// with A' (rows x 2P) the real view of [A_0 | A_1 | A_2] and C'' (2P x 2q) the real
// representation of the stacked complex coefficients: C''_{2i,2j} = Re C_ij,
// C''_{2i,2j+1} = Im C_ij, C''_{2i+1,2j} = -Im C_ij, C''_{2i+1,2j+1} = Re C_ij (negated when
// neg). Nothing is staged: a warp owns 8-row M tiles (tiles warp, warp + warps, ... of the CTA's
// rows) and loads its A fragments from global memory into registers, a ring of k-step pairs
// ahead of the MMAs. The k order is permuted over pairs of k steps: a pair covers complex
// columns c0 .. c0 + 3 of one block, MMA k = t of its first step is Re A[.][c0 + t] and of its
// second step Im A[.][c0 + t] (g = lane / 4, t = lane % 4), so a lane's A values of the pair are
// one 16-byte load, A[row g][c0 + t]. Those loads stream through a ring of kDmRing pairs in
// shared memory private to the warp: each lane cp.async-copies exactly the 16 bytes it later
// reads, so its own cp.async.wait_group orders them and no barrier is needed, and the ring holds
// twice the bytes in flight that registers could. C'' is stored in the pair's k order as one
// 16-byte word per (pair, 8-column N tile, lane): {C''[2 (c0 + t)][n g],
// C''[2 (c0 + t) + 1][n g]}. A row is read (by the four lanes of its quad) before any of its
// outputs is written and no other warp touches it, so Y may alias an input.
constexpr int kUpdRows = 8;
constexpr int kUpdThreads = 256;
constexpr int kUpdWarps = kUpdThreads / 32;
constexpr int kUpdChunk = kUpdRows * kUpdWarps;     // row granularity of a CTA's span
constexpr int kDmRing = 16;                         // k-step pairs in flight per warp (2^k)
constexpr size_t kDmRingBytes = (size_t)kUpdWarps * kDmRing * 32 * sizeof(double2);

// k-step pairs of a list of at most three blocks with P columns in all (ceil(cols / 4) each)
__host__ __device__ __forceinline__ int dmma_pairs_bound(int P) { return (P + 3) / 4 + 2; }
// the warps' load rings, then the packed coefficients
__host__ __device__ __forceinline__ size_t update_smem_bytes(int P, int q, int nout = 1) {
  return kDmRingBytes + (size_t)nout * dmma_pairs_bound(P) * ((q + 3) / 4) * 32 * sizeof(double2);
}

// one k-step pair of an update's A list: columns c0 .. c0 + 3 of a block (p points at c0)
struct DmKStep {
  const double2* p;
  int ld;
  int rem;          // columns of the block from c0 on
};

template <int NT, int NOUT, bool ACC>
static __device__ __forceinline__ void update_dmma_core(const DmKStep* __restrict__ sK,
                                                        const double2* __restrict__ sB,
                                                        double2* __restrict__ ring, int KS,
                                                        int q, long long r0, long long r1,
                                                        double2* Y, double2* Y2, long long ldy) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int nw = blockDim.x >> 5;
  const int ntiles = (int)((r1 - r0 + kUpdRows - 1) / kUpdRows);
  const int mine = ntiles > warp ? (ntiles - warp + nw - 1) / nw : 0;
  const int nitems = mine * KS;
  if (nitems == 0) return;
  // this lane's slots of the warp's ring: ring[slot * 32 + lane]; one commit group per item
  ring += (size_t)warp * kDmRing * 32 + lane;
  int l_tile = warp, l_s = 0;
  auto fetch = [&](int slot) {
    const DmKStep k = sK[l_s];
    const long long ra = r0 + (long long)l_tile * kUpdRows + g;
    double2* dst = ring + slot * 32;
    if (t < k.rem && ra < r1) {
      const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" :: "r"(sa), "l"(k.p + ra * k.ld + t) : "memory");
    } else {
      *dst = make_double2(0.0, 0.0);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    if (++l_s == KS) { l_s = 0; l_tile += nw; }
  };
  for (int d = 0; d < kDmRing; ++d) {
    if (d < nitems) fetch(d);
    else asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  double acc[NOUT][NT][2];
  double2 yo[ACC ? NT : 1];
#pragma unroll
  for (int o = 0; o < NOUT; ++o)
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[o][j][0] = acc[o][j][1] = 0.0;
  int c_s = 0, c_tile = warp;
  {
    for (int it = 0; it < nitems; ++it) {
      const int slot = it & (kDmRing - 1);
      // item it's group is complete once at most kDmRing - 1 younger groups are pending
      asm volatile("cp.async.wait_group %0;\n" :: "n"(kDmRing - 1) : "memory");
      const double2 a = ring[slot * 32];
      const long long ra = r0 + (long long)c_tile * kUpdRows + g;
      if (ACC && c_s == 0) {
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          const int col = j * 4 + t;
          yo[j] = (col < q && ra < r1) ? Y[ra * ldy + col] : make_double2(0.0, 0.0);
        }
      }
      const double2* bp = sB + (size_t)c_s * NT * 32 + lane;
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const double2 b = bp[j * 32];
        dmma(acc[0][j][0], acc[0][j][1], a.x, b.x);
        dmma(acc[0][j][0], acc[0][j][1], a.y, b.y);
        if (NOUT == 2) {
          const double2 b2 = bp[(size_t)KS * NT * 32 + j * 32];
          dmma(acc[NOUT - 1][j][0], acc[NOUT - 1][j][1], a.x, b2.x);
          dmma(acc[NOUT - 1][j][0], acc[NOUT - 1][j][1], a.y, b2.y);
        }
      }
      // refill the slot only now: the MMAs above consumed `a`, so its shared-memory read is done
      if (it + kDmRing < nitems) fetch(slot);
      else asm volatile("cp.async.commit_group;\n" ::: "memory");
      if (++c_s == KS) {
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          const int col = j * 4 + t;
          if (col < q && ra < r1) {
            double2 v = make_double2(acc[0][j][0], acc[0][j][1]);
            if (ACC) { v.x += yo[j].x; v.y += yo[j].y; }
            Y[ra * ldy + col] = v;
            if (NOUT == 2) Y2[ra * ldy + col] = make_double2(acc[NOUT - 1][j][0], acc[NOUT - 1][j][1]);
          }
#pragma unroll
          for (int o = 0; o < NOUT; ++o) acc[o][j][0] = acc[o][j][1] = 0.0;
        }
        c_s = 0;
        c_tile += nw;
      }
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Y (+)= sg A C over rows [r0, r1) and, with C2/Y2, Y2 = sg A C2 (one pass over A; the fused
// X / P Ritz update reads [X | R | P] once for both). C[b] is the cols_b x q row-major
// coefficient block of A's block b (NULL: the block does not enter); q <= kMaxBlock. Called by
// every thread of the CTA; smem holds update_smem_bytes. The two-output form that also
// accumulates into Y takes two passes over A, so there Y must not alias an input.
static __device__ void update_rows(const BlockList<double>& A, const double2* const* C, int q,
                                   long long r0, long long r1, double2* Y, long long ldy,
                                   int accumulate, int neg, unsigned char* smem,
                                   const double2* const* C2 = nullptr, double2* Y2 = nullptr) {
  __shared__ int2 sK[kMaxSmall / 4 + 3];
  __shared__ DmKStep sKp[kMaxSmall / 4 + 3];
  __shared__ int sKS;
  const int nout = Y2 ? 2 : 1;
  const int NT = (q + 3) / 4;
  if (threadIdx.x == 0) {
    int s = 0;
    for (int b = 0; b < A.nblk; ++b)
      for (int c0 = 0; c0 < A.cols[b]; c0 += 4) {
        sKp[s].p = A.p[b] + c0; sKp[s].ld = (int)A.ld[b]; sKp[s].rem = A.cols[b] - c0;
        sK[s++] = make_int2(b, c0);
      }
    sKS = s;
  }
  __syncthreads();
  const int KS = sKS;
  double2* ring = reinterpret_cast<double2*>(smem);
  double2* sB = reinterpret_cast<double2*>(smem + kDmRingBytes);
  const double sg = neg ? -1.0 : 1.0;
  const int per_out = KS * NT * 32;
  for (int e = threadIdx.x; e < nout * per_out; e += blockDim.x) {
    const int o = e / per_out, r = e - o * per_out;
    const int s = r / (NT * 32), r2 = r - s * NT * 32;
    const int j = r2 >> 5, ln = r2 & 31;
    const int gg = ln >> 2, tt = ln & 3;
    const int2 k = sK[s];
    const int cols = k.x == 0 ? A.cols[0] : k.x == 1 ? A.cols[1] : A.cols[2];
    const double2* Cb = (o ? C2 : C)[k.x];
    const int i = k.y + tt, jj = j * 4 + (gg >> 1);
    double2 w = make_double2(0.0, 0.0);
    if (Cb && i < cols && jj < q) {
      const double2 c = Cb[(size_t)i * q + jj];
      const double re = sg * c.x, im = sg * c.y;
      if (gg & 1) w = make_double2(im, re);      // C''[2i][2jj+1], C''[2i+1][2jj+1]
      else w = make_double2(re, -im);            // C''[2i][2jj],   C''[2i+1][2jj]
    }
    sB[e] = w;
  }
  __syncthreads();
#define QDKP_DM_CASE(nt)                                                                          \
  case nt:                                                                                        \
    if (nout == 2 && accumulate) {                                                                \
      update_dmma_core<nt, 1, true>(sKp, sB, ring, KS, q, r0, r1, Y, Y2, ldy);                          \
      update_dmma_core<nt, 1, false>(sKp, sB + per_out, ring, KS, q, r0, r1, Y2, Y2, ldy);              \
    } else if (nout == 2) update_dmma_core<nt, 2, false>(sKp, sB, ring, KS, q, r0, r1, Y, Y2, ldy);     \
    else if (accumulate) update_dmma_core<nt, 1, true>(sKp, sB, ring, KS, q, r0, r1, Y, Y2, ldy);       \
    else update_dmma_core<nt, 1, false>(sKp, sB, ring, KS, q, r0, r1, Y, Y2, ldy);                      \
    break;
  switch (NT) {
    QDKP_DM_CASE(1) QDKP_DM_CASE(2) QDKP_DM_CASE(3) QDKP_DM_CASE(4) QDKP_DM_CASE(5) QDKP_DM_CASE(6)
    default: break;
  }
#undef QDKP_DM_CASE
}

// ---------------------------------------------------------------------------------------------
// Gram core: partial C' = A'^T B' (real views: row r, column 2c + {re, im}) of rows [r0, r1) on
// the FP64 MMA units (mma.sync.m8n8k4.f64; the tcgen05 family has no f64 kind). Rows stream
// through shared memory in chunks (gram_chunk_rows), 2-4 stages in flight with cp.async and one
// CTA barrier per chunk: every block of
// the two lists is copied as a flat run of chunk-rows x cols complex values (the engine's blocks
// are compact, ld = cols; other leading dimensions are handled row by row). Each warp owns a
// rectangle of MR x MC 8x8 tiles of C' and a slice of the chunk's 4-row k steps, reads its
// m8n8k4 fragments from shared memory (lane (g, t4): row k0 + t4, real column 8 tile + g) and
// keeps its tiles in registers. The row slices of a rectangle are summed in shared memory in a
// fixed order at the end (deterministic), giving one RP x RQ partial per CTA. complex64 blocks
// are staged as they are and widened to FP64 in the fragment loads.
// ---------------------------------------------------------------------------------------------
constexpr int kGramCtaThreads = 256;
constexpr int kGramRows = 32;       // fewest rows per shared-memory chunk (a multiple of 8)
constexpr int kGramStageTarget = 24 * 1024;   // bytes a chunk brings in per barrier

// Rows per chunk: about kGramStageTarget bytes of the two lists, a multiple of 8 in
// [kGramRows, 512], so that narrow products still move many rows per CTA barrier.
__host__ __device__ __forceinline__ int gram_chunk_rows(int P, int Q, int elem_bytes) {
  int r = kGramStageTarget / ((P + Q) * elem_bytes);
  r = r / 8 * 8;
  return r < kGramRows ? kGramRows : (r > 512 ? 512 : r);
}

__host__ __device__ __forceinline__ size_t gram_smem_bytes(int P, int Q, int elem_bytes) {
  const size_t RP = (2 * P + 7) / 8 * 8, RQ = (2 * Q + 7) / 8 * 8;
  const size_t stage = (size_t)gram_chunk_rows(P, Q, elem_bytes) * (P + Q) * elem_bytes;
  const size_t red = RP * RQ * sizeof(double);
  const size_t st = stage_count(stage) * stage;
  return st > red ? st : red;
}

template <typename T>
__device__ __forceinline__ void gram_copy_rows(const BlockList<T>& L, long long r, int nrows,
                                               cplx<T>* dst, int crow) {
  int off = 0;
  for (int b = 0; b < L.nblk; ++b) {
    const int cols = L.cols[b];
    const int units = nrows * cols;
    const cplx<T>* src = L.p[b] + r * L.ld[b];
    cplx<T>* d = dst + (long long)off * crow;
    if (L.ld[b] == cols) {
      if (sizeof(cplx<T>) == 8 && (units & 1) == 0 && ((uintptr_t)src & 15) == 0 &&
          ((uintptr_t)d & 15) == 0) {
        // complex64 run that starts and ends on 16 bytes: two values per copy
        for (int u = 2 * threadIdx.x; u < units; u += 2 * blockDim.x) {
          const unsigned sa = (unsigned)__cvta_generic_to_shared(d + u);
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" :: "r"(sa), "l"(src + u) : "memory");
        }
      } else {
        for (int u = threadIdx.x; u < units; u += blockDim.x) {
          const unsigned sa = (unsigned)__cvta_generic_to_shared(d + u);
          if (sizeof(cplx<T>) == 16)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" :: "r"(sa), "l"(src + u) : "memory");
          else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" :: "r"(sa), "l"(src + u) : "memory");
        }
      }
    } else {
      for (int u = threadIdx.x; u < units; u += blockDim.x) {
        const int rr = u / cols, c = u - rr * cols;
        const unsigned sa = (unsigned)__cvta_generic_to_shared(d + u);
        const cplx<T>* g = src + (long long)rr * L.ld[b] + c;
        if (sizeof(cplx<T>) == 16)
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" :: "r"(sa), "l"(g) : "memory");
        else
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" :: "r"(sa), "l"(g) : "memory");
      }
    }
    off += cols;
  }
}

// tile rectangles: tile rows split in groups of MR, tile columns in groups of MC. A CTA covers
// the tile columns [tc_lo, tc_lo + tc_cnt) of C' (a column panel; a wide product is split into
// panels over blockIdx.y so that every rectangle fits one warp's registers) and writes only
// those columns of its partial.
template <int MR, int MC, typename T>
static __device__ void gram_core(const BlockList<T>& A, const BlockList<T>& B,
                                 long long r0, long long r1, double* __restrict__ out,
                                 unsigned char* smem, int tc_lo = 0, int tc_cnt = 1 << 30) {
  const int P = A.total(), Q = B.total();
  const int RP = (2 * P + 7) / 8 * 8, RQ = (2 * Q + 7) / 8 * 8;
  const int TR = RP / 8;
  const int tc_hi = min(RQ / 8, tc_lo + tc_cnt);
  const int TC = tc_hi - tc_lo;                   // this panel's tile columns
  if (TC <= 0) return;                            // an empty panel (uniform over the CTA)
  const int GR = (TR + MR - 1) / MR, GC = (TC + MC - 1) / MC;
  const int G = GR * GC;                          // tile rectangles (<= warps by construction)
  const int nwarps = blockDim.x >> 5;
  const int slices = nwarps / G;                  // warps per rectangle
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int rect = warp % G, slice = warp / G;
  const bool active_warp = slice < slices;
  const int tr0 = (rect / GC) * MR, tc0 = tc_lo + (rect % GC) * MC;
  // stage layout: per list, per block, crow x cols complex values; A's blocks first
  const unsigned avail = dyn_smem_bytes();
  int crow = gram_chunk_rows(P, Q, (int)sizeof(cplx<T>));
  {   // two stages must fit the launch's shared memory
    const int fit = (int)(avail / (2 * (size_t)(P + Q) * sizeof(cplx<T>))) / 8 * 8;
    if (crow > fit) crow = fit;
  }
  const size_t stage_elems = (size_t)crow * (P + Q);
  const int NS = stage_count_fit(stage_elems * sizeof(cplx<T>), avail);
  cplx<T>* stage0 = reinterpret_cast<cplx<T>*>(smem);
  // per tile: the real offset of its column inside a staged row block (-1: outside P / Q)
  // as (block start in complex columns * crow, block width, real column in the row)
  int sa_off[MR], sa_w[MR], sa_c[MR], sb_off[MC], sb_w[MC], sb_c[MC];
#pragma unroll
  for (int i = 0; i < MR; ++i) {
    const int col = (tr0 + i) * 8 + g;           // real column of A'
    int c = col >> 1, blk = 0, start = 0;
    while (blk < A.nblk - 1 && c >= A.cols[blk]) { c -= A.cols[blk]; start += A.cols[blk]; ++blk; }
    const bool ok = active_warp && tr0 + i < TR && col < 2 * P;
    sa_off[i] = ok ? start * crow : -1;
    sa_w[i] = A.cols[blk];
    sa_c[i] = 2 * c + (col & 1);
  }
#pragma unroll
  for (int j = 0; j < MC; ++j) {
    const int col = (tc0 + j) * 8 + g;
    int c = col >> 1, blk = 0, start = 0;
    while (blk < B.nblk - 1 && c >= B.cols[blk]) { c -= B.cols[blk]; start += B.cols[blk]; ++blk; }
    const bool ok = active_warp && tc0 + j < tc_hi && col < 2 * Q;
    sb_off[j] = ok ? (P + start) * crow : -1;
    sb_w[j] = B.cols[blk];
    sb_c[j] = 2 * c + (col & 1);
  }
  double acc[MR][MC][2];
#pragma unroll
  for (int i = 0; i < MR; ++i)
#pragma unroll
    for (int j = 0; j < MC; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const long long nrows = r1 - r0;
  const int nchunks = (int)((nrows + crow - 1) / crow);
  // chunk c lives in stage c % NS; NS - 1 chunks are in flight while one is consumed
  auto issue = [&](int c) {
    if (c < nchunks) {
      const long long rn = r0 + (long long)c * crow;
      const int nn = (int)min((long long)crow, r1 - rn);
      cplx<T>* st = stage0 + (size_t)(c % NS) * stage_elems;
      gram_copy_rows(A, rn, nn, st, crow);
      gram_copy_rows(B, rn, nn, st + (size_t)P * crow, crow);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  for (int c = 0; c < NS - 1; ++c) issue(c);
  for (int ch = 0; ch < nchunks; ++ch) {
    const long long rc = r0 + (long long)ch * crow;
    const int rows = (int)min((long long)crow, r1 - rc);
    // chunk ch has landed once at most NS - 2 groups are pending; the barrier also means every
    // warp is done with chunk ch - 1, whose stage the next copy reuses
    cp_async_wait_pending(NS - 2);
    __syncthreads();
    issue(ch + NS - 1);
    const T* sr = reinterpret_cast<const T*>(stage0 + (size_t)(ch % NS) * stage_elems);
    if (active_warp) {
      for (int k0 = 4 * slice; k0 < rows; k0 += 4 * slices) {
        const int row = k0 + t4;
        const bool ok = row < rows;
        double a[MR], b[MC];
#pragma unroll
        for (int i = 0; i < MR; ++i)
          a[i] = (ok && sa_off[i] >= 0)
                     ? (double)sr[2 * sa_off[i] + row * 2 * sa_w[i] + sa_c[i]] : 0.0;
#pragma unroll
        for (int j = 0; j < MC; ++j)
          b[j] = (ok && sb_off[j] >= 0)
                     ? (double)sr[2 * sb_off[j] + row * 2 * sb_w[j] + sb_c[j]] : 0.0;
#pragma unroll
        for (int i = 0; i < MR; ++i)
#pragma unroll
          for (int j = 0; j < MC; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
      }
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  // fixed-order sum of the row slices of each rectangle
  double* gsm = reinterpret_cast<double*>(smem);
  for (int e = threadIdx.x; e < RP * RQ; e += blockDim.x) gsm[e] = 0.0;
  __syncthreads();
  for (int sl = 0; sl < slices; ++sl) {
    if (active_warp && slice == sl) {
#pragma unroll
      for (int i = 0; i < MR; ++i)
#pragma unroll
        for (int j = 0; j < MC; ++j) {
          const int ti = tr0 + i, tj = tc0 + j;
          if (ti < TR && tj < tc_hi) {
            const int rr = ti * 8 + g, cc = tj * 8 + 2 * t4;
            gsm[rr * RQ + cc] += acc[i][j][0];
            gsm[rr * RQ + cc + 1] += acc[i][j][1];
          }
        }
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < RP * RQ; e += blockDim.x) {
    const int cc = e % RQ;
    if (cc >= 8 * tc_lo && cc < 8 * tc_hi) out[e] = gsm[e];
  }
}

// ---------------------------------------------------------------------------------------------
// complex64 blocks: split-precision TF32 tensor-core products (mma.sync.m16n8k8 .tf32, FP32
// accumulation). Every FP32 value x is split into x = hi + lo with hi, lo TF32 (10-bit
// mantissas; cvt.rna), and a product is formed as lo*hi + hi*lo + hi*hi (the lo*lo term is below
// FP32 rounding), which keeps the FP32 accuracy of the inputs. A CTA accumulates its rows in
// FP32 registers and writes an FP64 partial; partials are summed in FP64.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned tf32_round(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void tf32_split(float x, unsigned& hi, unsigned& lo) {
  hi = tf32_round(x);
  lo = tf32_round(x - __uint_as_float(hi));
}
__device__ __forceinline__ void mma_tf32(float (&d)[4], unsigned a0, unsigned a1, unsigned a2,
                                         unsigned a3, unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
// d += (ahi + alo)(bhi + blo) without the lo * lo term
__device__ __forceinline__ void mma_tf32x3(float (&d)[4], const unsigned (&ah)[4],
                                           const unsigned (&al)[4], const unsigned (&bh)[2],
                                           const unsigned (&bl)[2]) {
  mma_tf32(d, al[0], al[1], al[2], al[3], bh[0], bh[1]);
  mma_tf32(d, ah[0], ah[1], ah[2], ah[3], bl[0], bl[1]);
  mma_tf32(d, ah[0], ah[1], ah[2], ah[3], bh[0], bh[1]);
}

// Gram partial C' = A'^T B' over rows [r0, r1) of complex64 lists (same staging and output as
// gram_core). MMA tiles: 16 columns of A' (M) x 8 columns of B' (N) x 8 rows (K); a warp owns a
// rectangle of kTfMR x kTfMC tiles and a slice of the chunk's 8-row k steps.
// Fragments (m16n8k8 tf32; g = lane / 4, t = lane % 4): A_mma[m][k] = A'[k][m]:
// a0 = (k t, m g), a1 = (k t, m g + 8), a2 = (k t + 4, m g), a3 = (k t + 4, m g + 8);
// B_mma[k][n] = B'[k][n]: b0 = (k t, n g), b1 = (k t + 4, n g); D: (m g, n 2t), (m g, n 2t + 1),
// (m g + 8, n 2t), (m g + 8, n 2t + 1).
constexpr int kTfMR = 3, kTfMC = 3;

__host__ __device__ __forceinline__ int gram_tf32_rects(int P, int Q) {
  const int TR = (2 * P + 15) / 16, TC = (2 * Q + 7) / 8;
  return ((TR + kTfMR - 1) / kTfMR) * ((TC + kTfMC - 1) / kTfMC);
}

static __device__ void gram_core_tf32(const BlockList<float>& A, const BlockList<float>& B,
                                      long long r0, long long r1, double* __restrict__ out,
                                      unsigned char* smem) {
  const int P = A.total(), Q = B.total();
  const int RP = (2 * P + 7) / 8 * 8, RQ = (2 * Q + 7) / 8 * 8;   // partial layout (as FP64 core)
  const int TR = (2 * P + 15) / 16, TC = (2 * Q + 7) / 8;
  const int GC = (TC + kTfMC - 1) / kTfMC;
  const int G = gram_tf32_rects(P, Q);
  const int nwarps = blockDim.x >> 5;
  const int slices = nwarps / G;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int rect = warp % G, slice = warp / G;
  const bool active_warp = slice < slices;
  const int tr0 = (rect / GC) * kTfMR, tc0 = (rect % GC) * kTfMC;
  const unsigned avail = dyn_smem_bytes();
  int crow = gram_chunk_rows(P, Q, (int)sizeof(float2));
  {
    const int fit = (int)(avail / (2 * (size_t)(P + Q) * sizeof(float2))) / 8 * 8;
    if (crow > fit) crow = fit;
  }
  const size_t stage_elems = (size_t)crow * (P + Q);
  const int NS = stage_count_fit(stage_elems * sizeof(float2), avail);
  float2* stage0 = reinterpret_cast<float2*>(smem);
  // staged real offset of a real column of A' (two per M tile: m g, m g + 8) and of B' (n g)
  int ao[kTfMR][2], aw[kTfMR][2], bo[kTfMC], bw[kTfMC];
#pragma unroll
  for (int i = 0; i < kTfMR; ++i)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int col = (tr0 + i) * 16 + g + 8 * h;
      int c = col >> 1, blk = 0, start = 0;
      while (blk < A.nblk - 1 && c >= A.cols[blk]) { c -= A.cols[blk]; start += A.cols[blk]; ++blk; }
      const bool ok = active_warp && tr0 + i < TR && col < 2 * P;
      ao[i][h] = ok ? 2 * start * crow + 2 * c + (col & 1) : -1;
      aw[i][h] = 2 * A.cols[blk];
    }
#pragma unroll
  for (int j = 0; j < kTfMC; ++j) {
    const int col = (tc0 + j) * 8 + g;
    int c = col >> 1, blk = 0, start = 0;
    while (blk < B.nblk - 1 && c >= B.cols[blk]) { c -= B.cols[blk]; start += B.cols[blk]; ++blk; }
    const bool ok = active_warp && tc0 + j < TC && col < 2 * Q;
    bo[j] = ok ? 2 * (P + start) * crow + 2 * c + (col & 1) : -1;
    bw[j] = 2 * B.cols[blk];
  }
  float acc[kTfMR][kTfMC][4];
#pragma unroll
  for (int i = 0; i < kTfMR; ++i)
#pragma unroll
    for (int j = 0; j < kTfMC; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

  const long long nrows = r1 - r0;
  const int nchunks = (int)((nrows + crow - 1) / crow);
  auto issue = [&](int c) {
    if (c < nchunks) {
      const long long rn = r0 + (long long)c * crow;
      const int nn = (int)min((long long)crow, r1 - rn);
      float2* st = stage0 + (size_t)(c % NS) * stage_elems;
      gram_copy_rows(A, rn, nn, st, crow);
      gram_copy_rows(B, rn, nn, st + (size_t)P * crow, crow);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  for (int c = 0; c < NS - 1; ++c) issue(c);
  for (int ch = 0; ch < nchunks; ++ch) {
    const long long rc = r0 + (long long)ch * crow;
    const int rows = (int)min((long long)crow, r1 - rc);
    // chunk ch has landed once at most NS - 2 groups are pending; the barrier also means every
    // warp is done with chunk ch - 1, whose stage the next copy reuses
    cp_async_wait_pending(NS - 2);
    __syncthreads();
    issue(ch + NS - 1);
    const float* sr = reinterpret_cast<const float*>(stage0 + (size_t)(ch % NS) * stage_elems);
    if (active_warp) {
      for (int k0 = 8 * slice; k0 < rows; k0 += 8 * slices) {
        const int ra = k0 + t, rb = k0 + t + 4;      // the two rows of this lane's fragments
        const bool oka = ra < rows, okb = rb < rows;
        unsigned bh[kTfMC][2], bl[kTfMC][2];
#pragma unroll
        for (int j = 0; j < kTfMC; ++j) {
          const float x0 = (oka && bo[j] >= 0) ? sr[bo[j] + ra * bw[j]] : 0.f;
          const float x1 = (okb && bo[j] >= 0) ? sr[bo[j] + rb * bw[j]] : 0.f;
          tf32_split(x0, bh[j][0], bl[j][0]);
          tf32_split(x1, bh[j][1], bl[j][1]);
        }
#pragma unroll
        for (int i = 0; i < kTfMR; ++i) {
          const float v0 = (oka && ao[i][0] >= 0) ? sr[ao[i][0] + ra * aw[i][0]] : 0.f;
          const float v1 = (oka && ao[i][1] >= 0) ? sr[ao[i][1] + ra * aw[i][1]] : 0.f;
          const float v2 = (okb && ao[i][0] >= 0) ? sr[ao[i][0] + rb * aw[i][0]] : 0.f;
          const float v3 = (okb && ao[i][1] >= 0) ? sr[ao[i][1] + rb * aw[i][1]] : 0.f;
          unsigned ah[4], al[4];
          tf32_split(v0, ah[0], al[0]);
          tf32_split(v1, ah[1], al[1]);
          tf32_split(v2, ah[2], al[2]);
          tf32_split(v3, ah[3], al[3]);
#pragma unroll
          for (int j = 0; j < kTfMC; ++j) mma_tf32x3(acc[i][j], ah, al, bh[j], bl[j]);
        }
      }
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  double* gsm = reinterpret_cast<double*>(smem);
  for (int e = threadIdx.x; e < RP * RQ; e += blockDim.x) gsm[e] = 0.0;
  __syncthreads();
  for (int sl = 0; sl < slices; ++sl) {
    if (active_warp && slice == sl) {
#pragma unroll
      for (int i = 0; i < kTfMR; ++i)
#pragma unroll
        for (int j = 0; j < kTfMC; ++j) {
          const int ti = tr0 + i, tj = tc0 + j;
          if (ti < TR && tj < TC) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int rr = ti * 16 + g + 8 * h, cc = tj * 8 + 2 * t;
              if (rr < RP && cc < RQ) {
                gsm[rr * RQ + cc] += (double)acc[i][j][2 * h];
                gsm[rr * RQ + cc + 1] += (double)acc[i][j][2 * h + 1];
              }
            }
          }
        }
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < RP * RQ; e += blockDim.x) out[e] = gsm[e];
}

// Y' = A' C'' for rows [r0, r1) of complex64 blocks on TF32 tensor cores (split as above).
// Nothing is staged: a warp owns 16-row M tiles (tiles warp, warp + warps, ... of the CTA's
// rows) and loads its A fragments from global memory into registers, a ring of k steps ahead of
// the MMAs, so a CTA needs no barrier after its coefficient setup. The MMA's k order is
// permuted so that a lane's two k values of a fragment row are the real and imaginary part of
// one complex element: k step s covers complex columns c0 .. c0 + 3 of one block, and
// MMA k = t <-> Re A[.][c0 + t], k = t + 4 <-> Im A[.][c0 + t] (g = lane / 4, t = lane % 4), so
// a0 a2 = A[row g][c0 + t] and a1 a3 = A[row g + 8][c0 + t] are one 8-byte load each. C'' (the
// real representation of the stacked complex coefficients, as in update_rows) is stored in that
// k order as one 16-byte word per (k step, 8-column N tile, lane): {hi b0, hi b1, lo b0, lo b1}
// with b0 = C''[k t][n g], b1 = C''[k t + 4][n g]. A row is read (by the four lanes of its quad)
// before any of its outputs is written and no other warp touches it, so Y may alias an input.
constexpr int kTfUpdChunk = 128;   // row granularity of a CTA's span (a multiple of the M tile)
constexpr int kTfRing = 8;         // k steps of A fragments in flight per warp (narrow outputs)
constexpr int kTfMaxKs = kMaxSmall / 4 + 3;

// k steps of a list of at most three blocks with P columns in all (ceil(cols / 4) per block)
__host__ __device__ __forceinline__ int tf32_ksteps_bound(int P) { return (P + 3) / 4 + 2; }

__host__ __device__ __forceinline__ size_t update_tf32_smem_bytes(int P, int q, int nout = 1) {
  return (size_t)nout * tf32_ksteps_bound(P) * ((q + 3) / 4) * 32 * sizeof(uint4);
}

// one k step of an update's A list: columns c0 .. c0 + 3 of a block (p points at column c0)
struct TfKStep {
  const float2* p;
  int ld;
  int rem;          // columns of the block from c0 on
};

template <int NT, int NOUT, bool ACC>
static __device__ __forceinline__ void update_tf32_core(const TfKStep* __restrict__ sK,
                                                        const uint4* __restrict__ sB, int KS,
                                                        int q, long long r0, long long r1,
                                                        float2* Y, float2* Y2, long long ldy) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int nw = blockDim.x >> 5;
  const int ntiles = (int)((r1 - r0 + 15) / 16);
  const int mine = ntiles > warp ? (ntiles - warp + nw - 1) / nw : 0;
  const int nitems = mine * KS;
  if (nitems == 0) return;
  // wide outputs hold more accumulators: a shorter ring keeps the warp within 128 registers
  constexpr int RING = NT * NOUT <= 6 ? kTfRing : kTfRing / 2;
  float2 fa[RING], fb[RING];
  int l_tile = warp, l_s = 0;
  auto fetch = [&](float2& xa, float2& xb) {
    const TfKStep k = sK[l_s];
    const long long ra = r0 + (long long)l_tile * 16 + g, rb = ra + 8;
    xa = (t < k.rem && ra < r1) ? __ldcs(k.p + ra * k.ld + t) : make_float2(0.f, 0.f);
    xb = (t < k.rem && rb < r1) ? __ldcs(k.p + rb * k.ld + t) : make_float2(0.f, 0.f);
    if (++l_s == KS) { l_s = 0; l_tile += nw; }
  };
#pragma unroll
  for (int d = 0; d < RING; ++d)
    if (d < nitems) fetch(fa[d], fb[d]);
  float acc[NOUT][NT][4];
  float2 yo[ACC ? NT : 1][2];
#pragma unroll
  for (int o = 0; o < NOUT; ++o)
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[o][j][e] = 0.f;
  int c_s = 0, c_tile = warp;
  for (int base = 0; base < nitems; base += RING) {
#pragma unroll
    for (int d = 0; d < RING; ++d) {
      const int it = base + d;
      if (it >= nitems) break;
      unsigned ah[4], al[4];
      tf32_split(fa[d].x, ah[0], al[0]);
      tf32_split(fb[d].x, ah[1], al[1]);
      tf32_split(fa[d].y, ah[2], al[2]);
      tf32_split(fb[d].y, ah[3], al[3]);
      if (it + RING < nitems) fetch(fa[d], fb[d]);
      const long long ra = r0 + (long long)c_tile * 16 + g, rb = ra + 8;
      if (ACC && c_s == 0) {
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          const int col = j * 4 + t;
          yo[j][0] = (col < q && ra < r1) ? Y[ra * ldy + col] : make_float2(0.f, 0.f);
          yo[j][1] = (col < q && rb < r1) ? Y[rb * ldy + col] : make_float2(0.f, 0.f);
        }
      }
      const uint4* bp = sB + (size_t)c_s * NT * 32 + lane;
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const uint4 b = bp[j * 32];
        const unsigned bh[2] = {b.x, b.y}, bl[2] = {b.z, b.w};
        mma_tf32x3(acc[0][j], ah, al, bh, bl);
        if (NOUT == 2) {
          const uint4 b2 = bp[(size_t)KS * NT * 32 + j * 32];
          const unsigned bh2[2] = {b2.x, b2.y}, bl2[2] = {b2.z, b2.w};
          mma_tf32x3(acc[NOUT - 1][j], ah, al, bh2, bl2);
        }
      }
      if (++c_s == KS) {
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          const int col = j * 4 + t;
          if (col < q) {
            float2 va = make_float2(acc[0][j][0], acc[0][j][1]);
            float2 vb = make_float2(acc[0][j][2], acc[0][j][3]);
            if (ACC) {
              va.x += yo[j][0].x; va.y += yo[j][0].y;
              vb.x += yo[j][1].x; vb.y += yo[j][1].y;
            }
            if (ra < r1) Y[ra * ldy + col] = va;
            if (rb < r1) Y[rb * ldy + col] = vb;
            if (NOUT == 2) {
              if (ra < r1) Y2[ra * ldy + col] = make_float2(acc[NOUT - 1][j][0], acc[NOUT - 1][j][1]);
              if (rb < r1) Y2[rb * ldy + col] = make_float2(acc[NOUT - 1][j][2], acc[NOUT - 1][j][3]);
            }
          }
#pragma unroll
          for (int o = 0; o < NOUT; ++o)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[o][j][e] = 0.f;
        }
        c_s = 0;
        c_tile += nw;
      }
    }
  }
}

// Y (+)= sg A C over rows [r0, r1) and, with C2/Y2, Y2 = sg A C2 (one pass over A). C[b] is the
// cols_b x q row-major coefficient block of A's block b (NULL: the block does not enter);
// q <= kMaxBlock. Called by every thread of the CTA; smem holds update_tf32_smem_bytes. The
// two-output form that also accumulates into Y takes two passes over A, so there Y must not
// alias an input.
static __device__ void update_rows_tf32(const BlockList<float>& A, const double2* const* C, int q,
                                        long long r0, long long r1, float2* Y, long long ldy,
                                        int accumulate, int neg, unsigned char* smem,
                                        const double2* const* C2 = nullptr,
                                        float2* Y2 = nullptr) {
  __shared__ int2 sK[kTfMaxKs];
  __shared__ TfKStep sKp[kTfMaxKs];
  __shared__ int sKS;
  const int nout = Y2 ? 2 : 1;
  const int NT = (q + 3) / 4;
  if (threadIdx.x == 0) {
    int s = 0;
    for (int b = 0; b < A.nblk; ++b)
      for (int c0 = 0; c0 < A.cols[b]; c0 += 4) {
        sKp[s].p = A.p[b] + c0; sKp[s].ld = (int)A.ld[b]; sKp[s].rem = A.cols[b] - c0;
        sK[s++] = make_int2(b, c0);
      }
    sKS = s;
  }
  __syncthreads();
  const int KS = sKS;
  uint4* sB = reinterpret_cast<uint4*>(smem);
  const float sg = neg ? -1.f : 1.f;
  const int per_out = KS * NT * 32;
  for (int e = threadIdx.x; e < nout * per_out; e += blockDim.x) {
    const int o = e / per_out, r = e - o * per_out;
    const int s = r / (NT * 32), r2 = r - s * NT * 32;
    const int j = r2 >> 5, ln = r2 & 31;
    const int gg = ln >> 2, tt = ln & 3;
    const int2 k = sK[s];
    const int cols = k.x == 0 ? A.cols[0] : k.x == 1 ? A.cols[1] : A.cols[2];
    const double2* Cb = (o ? C2 : C)[k.x];
    const int i = k.y + tt, jj = j * 4 + (gg >> 1);
    float v0 = 0.f, v1 = 0.f;
    if (Cb && i < cols && jj < q) {
      const double2 c = Cb[(size_t)i * q + jj];
      const float re = sg * (float)c.x, im = sg * (float)c.y;
      if (gg & 1) { v0 = im; v1 = re; }          // C''[2i][2jj+1], C''[2i+1][2jj+1]
      else { v0 = re; v1 = -im; }                // C''[2i][2jj],   C''[2i+1][2jj]
    }
    uint4 w;
    tf32_split(v0, w.x, w.z);
    tf32_split(v1, w.y, w.w);
    sB[e] = w;
  }
  __syncthreads();
#define QDKP_TF_CASE(nt)                                                                          \
  case nt:                                                                                        \
    if (nout == 2 && accumulate) {                                                                \
      update_tf32_core<nt, 1, true>(sKp, sB, KS, q, r0, r1, Y, Y2, ldy);                          \
      update_tf32_core<nt, 1, false>(sKp, sB + per_out, KS, q, r0, r1, Y2, Y2, ldy);              \
    } else if (nout == 2) update_tf32_core<nt, 2, false>(sKp, sB, KS, q, r0, r1, Y, Y2, ldy);     \
    else if (accumulate) update_tf32_core<nt, 1, true>(sKp, sB, KS, q, r0, r1, Y, Y2, ldy);       \
    else update_tf32_core<nt, 1, false>(sKp, sB, KS, q, r0, r1, Y, Y2, ldy);                      \
    break;
  switch (NT) {
    QDKP_TF_CASE(1) QDKP_TF_CASE(2) QDKP_TF_CASE(3) QDKP_TF_CASE(4) QDKP_TF_CASE(5) QDKP_TF_CASE(6)
    default: break;
  }
#undef QDKP_TF_CASE
}

// Launch plan of an FP64 Gram product of P x Q complex columns: 3 x 3-tile rectangles (the
// register-resident size), 8 or 16 warps, and, for a product wider than 16 rectangles, column
// panels of `ptc` tile columns on blockIdx.y. Depends only on P and Q.
struct GramPlan { int threads, ptc, panels; };
static inline GramPlan gram_plan(int P, int Q) {
  const int TR = ((2 * P + 7) / 8 * 8) / 8, TC = ((2 * Q + 7) / 8 * 8) / 8;
  const int GR = (TR + 2) / 3, GC = (TC + 2) / 3;
  GramPlan g;
  if (GR * GC <= 8) { g.threads = 256; g.ptc = TC; g.panels = 1; return g; }
  if (GR * GC <= 16) { g.threads = 512; g.ptc = TC; g.panels = 1; return g; }
  const int gcp = GR >= 16 ? 1 : 16 / GR;        // rectangle columns per panel
  g.threads = 512;
  g.ptc = 3 * gcp;
  g.panels = (TC + g.ptc - 1) / g.ptc;
  return g;
}

}  // namespace qdkp
