// Batched LOBPCG engine (the served form): many solves resident on the device at once, each in
// a slot, advanced together one LOBPCG iteration per tick. The iteration is scipy's
// (lobpcg.py:688-973, B = M = Y = None, largest = False) exactly as the single-solve driver in
// lobpcg.cu runs it; the difference is that every decision is taken on the device, so a tick is
// a fixed launch sequence over all slots and the host only polls between ticks.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <type_traits>
#include <vector>

#include "engine_dev.cuh"
#include "umma_dev.cuh"

namespace qdkp {

int launch_apply(const qdkp_operator* op, const void* X, int64_t ldx, void* Y, int64_t ldy,
                 int m, double sigma, int shifted, int precision, cudaStream_t st);

constexpr int kERowsPerCta = 512;    // rows per CTA of the row kernels
constexpr int kENormRows = 2048;     // rows per CTA of the norm kernel
// Gram CTAs per slot: ceil(n / 256) up to this many. The split depends only on the slot's own
// size, so the order of every Gram sum -- and so the result -- is the same alone and in a mix.
constexpr int kEGramMaxParts = 296;

enum GramWhich { GR_XR = 0, GR_RR, GR_PP, GR_WW, GR_WAW, GR_BA, GR_BB };
// UP_XPNEW: P = R Cr + P Cp and X = X Cx + R Cr + P Cp from one pass over [X | R | P]
// (lobpcg.py:921-973); UP_AXPNEW: the same for AP and AX.
enum UpdWhich { UP_RPROJ = 0, UP_RNORM, UP_PNORM, UP_APNORM, UP_XPNEW, UP_AXPNEW };
enum RowWhich { RW_COPYBEST = 0, RW_RESID, RW_GATHERP };

// ---------------------------------------------------------------------------------------------
// residual norms of A X - X lambda: partials per CTA, reduced in the decision kernel
// ---------------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void e_norm_body(const ESlot& d, int part) {
  const EState* st = d.st;
  const cplx<T>* AX = blk<T>(d.AX);
  const cplx<T>* X = blk<T>(d.X);
  const int m = d.m;
  const long long r0 = (long long)part * kENormRows;
  const long long r1 = min(d.n, r0 + kENormRows);
  double acc[kMaxBlock];
#pragma unroll
  for (int j = 0; j < kMaxBlock; ++j) acc[j] = 0.0;
  for (long long r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
#pragma unroll
    for (int j = 0; j < kMaxBlock; ++j) {
      if (j < m) {
        const cplx<T> a = AX[r * m + j], x = X[r * m + j];
        const double l = st->lam[j];
        const double re = (double)a.x - l * (double)x.x, im = (double)a.y - l * (double)x.y;
        acc[j] = fma(re, re, fma(im, im, acc[j]));
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
    d.npart[(long long)part * m + threadIdx.x] = s;
  }
}

__global__ void __launch_bounds__(kTallThreads)
e_norm_kernel(const ESlot* __restrict__ S, int ns) {
  const int k = slot_of(S, ns, blockIdx.x, &ESlot::norm0);
  const ESlot& d = S[k];
  if (!d.st->running) return;
  if (d.prec == QDKP_C64) e_norm_body<float>(d, blockIdx.x - d.norm0);
  else e_norm_body<double>(d, blockIdx.x - d.norm0);
}

// ---------------------------------------------------------------------------------------------
// per-slot decisions at the top of an iteration (lobpcg.py:688-760)
// ---------------------------------------------------------------------------------------------
__global__ void e_decide_kernel(const ESlot* __restrict__ S) {
  const ESlot& d = S[blockIdx.x];
  EState* st = d.st;
  __shared__ double nrm[kMaxBlock];
  const int m = d.m;
  if (threadIdx.x < m) {
    double s = 0.0;
    for (int b = 0; b < d.nparts; ++b) s += d.npart[(long long)b * m + threadIdx.x];
    nrm[threadIdx.x] = sqrt(fabs(s));
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  st->idle = 1; st->copy_best = 0; st->skip_recompute = 1; st->skip_p = 1; st->skip_pnorm = 1;
  if (!st->running) return;
  if (st->iter >= d.maxiter) { st->running = 0; st->status = QDKP_LOBPCG_MAXITER; return; }
  if (d.stall_iterations > 0 && st->iter - st->best_iter > d.stall_iterations &&
      st->best_iter <= st->iter) {
    st->running = 0; st->status = QDKP_LOBPCG_MAXITER; return;
  }
  st->iter += 1;
  double mean = 0.0, mx = 0.0;
  bool finite = true;
  for (int j = 0; j < m; ++j) {
    st->norms[j] = nrm[j];
    mean += nrm[j];
    mx = fmax(mx, nrm[j]);
    finite = finite && isfinite(nrm[j]);
  }
  mean /= m;
  if (!finite) { st->running = 0; st->status = QDKP_LOBPCG_NONFINITE; return; }
  if (mean < st->smallest) {
    st->smallest = mean;
    st->best_iter = st->iter;
    st->copy_best = 1;
  } else if (mean > ldexp(1.0, d.restart_control) * st->smallest) {
    st->forced = 1;
    st->skip_recompute = 0;
  }
  int ma = 0;
  for (int j = 0; j < m; ++j) {
    st->active[j] = st->active[j] && (nrm[j] > d.tol);
    if (st->active[j]) st->idx[ma++] = j;
  }
  st->ma = ma;
  if (ma == 0) { st->running = 0; st->status = QDKP_LOBPCG_CONVERGED; return; }
  st->explicit_gram = !(mx > d.sqrt_eps && !st->explicit_gram);
  st->idle = 0;
  st->skip_p = st->iter == 0 ? 1 : 0;
}

// ---------------------------------------------------------------------------------------------
// row kernels: copy of the best iterate, residual gather, P gather
// ---------------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void e_row_body(const ESlot& d, int which, long long r0,
                                           long long r1) {
  const EState* st = d.st;
  const int m = d.m;
  const int ma = st->ma;
  const cplx<T>* X = blk<T>(d.X);
  if (which == RW_COPYBEST) {
    cplx<T>* best = blk<T>(d.best);
    for (long long e = r0 * m + threadIdx.x; e < r1 * m; e += blockDim.x) best[e] = X[e];
  } else if (which == RW_RESID) {
    const cplx<T>* AX = blk<T>(d.AX);
    cplx<T>* Ra = blk<T>(d.Ra);
    for (long long e = r0 * ma + threadIdx.x; e < r1 * ma; e += blockDim.x) {
      const long long r = e / ma;
      const int c = (int)(e - r * ma);
      const int j = st->idx[c];
      const double l = st->lam[j];
      const cplx<T> a = AX[r * m + j], x = X[r * m + j];
      Ra[e] = mk<T>((T)((double)a.x - l * (double)x.x), (T)((double)a.y - l * (double)x.y));
    }
  } else {
    const cplx<T>* P = blk<T>(d.P);
    const cplx<T>* AP = blk<T>(d.AP);
    cplx<T>* Pa = blk<T>(d.Pa);
    cplx<T>* APa = blk<T>(d.APa);
    for (long long e = r0 * ma + threadIdx.x; e < r1 * ma; e += blockDim.x) {
      const long long r = e / ma;
      const int c = (int)(e - r * ma);
      const int j = st->idx[c];
      Pa[e] = P[r * m + j];
      APa[e] = AP[r * m + j];
    }
  }
}

__global__ void __launch_bounds__(kTallThreads)
e_row_kernel(const ESlot* __restrict__ S, int ns, int which) {
  const int k = slot_of(S, ns, blockIdx.x, &ESlot::row0);
  const ESlot& d = S[k];
  const EState* st = d.st;
  if (which == RW_COPYBEST) { if (!st->copy_best) return; }
  else if (st->idle || (which == RW_GATHERP && st->skip_p)) return;
  const long long r0 = (long long)(blockIdx.x - d.row0) * d.rows_per_cta;
  const long long r1 = min(d.n, r0 + d.rows_per_cta);
  if (d.prec == QDKP_C64) e_row_body<float>(d, which, r0, r1);
  else e_row_body<double>(d, which, r0, r1);
}

// ---------------------------------------------------------------------------------------------
// Gram products, multi-slot (same FP64 MMA scheme as gram_partial_kernel)
// ---------------------------------------------------------------------------------------------
template <typename T>
__device__ bool gram_lists(const ESlot& d, int which, BlockList<T>& A, BlockList<T>& B,
                           double2*& out) {
  const EState* st = d.st;
  if (st->idle) return false;
  const int m = d.m, ma = st->ma, mp = st->mp;
  auto set1 = [](BlockList<T>& L, const cplx<T>* p, int c) {
    L.nblk = 1; L.p[0] = p; L.ld[0] = c; L.cols[0] = c;
  };
  const cplx<T>* X = blk<T>(d.X);
  const cplx<T>* AX = blk<T>(d.AX);
  const cplx<T>* Ra = blk<T>(d.Ra);
  const cplx<T>* ARa = blk<T>(d.ARa);
  const cplx<T>* Pa = blk<T>(d.Pa);
  const cplx<T>* APa = blk<T>(d.APa);
  switch (which) {
    case GR_XR: set1(A, X, m); set1(B, Ra, ma); out = d.W; return true;
    case GR_RR: set1(A, Ra, ma); set1(B, Ra, ma); out = d.G; return true;
    case GR_PP:
      if (st->skip_p) return false;
      set1(A, Pa, ma); set1(B, Pa, ma); out = d.G; return true;
    case GR_BA:      // non-explicit: [X | R | P]^H [AR | AP]
      if (st->explicit_gram) return false;
      A.nblk = mp ? 3 : 2;
      A.p[0] = X; A.ld[0] = m; A.cols[0] = m;
      A.p[1] = Ra; A.ld[1] = ma; A.cols[1] = ma;
      A.p[2] = Pa; A.ld[2] = ma; A.cols[2] = mp;
      B.nblk = mp ? 2 : 1;
      B.p[0] = ARa; B.ld[0] = ma; B.cols[0] = ma;
      B.p[1] = APa; B.ld[1] = ma; B.cols[1] = mp;
      out = d.gT;
      return true;
    case GR_BB:      // non-explicit: [X | R]^H P
      if (st->explicit_gram || mp == 0) return false;
      A.nblk = 2;
      A.p[0] = X; A.ld[0] = m; A.cols[0] = m;
      A.p[1] = Ra; A.ld[1] = ma; A.cols[1] = ma;
      set1(B, Pa, mp);
      B.ld[0] = ma;
      out = d.gS;
      return true;
    default: {       // explicit Gram mode: the full W^H W and W^H AW
      if (!st->explicit_gram) return false;
      A.nblk = mp ? 3 : 2;
      A.p[0] = X; A.ld[0] = m; A.cols[0] = m;
      A.p[1] = Ra; A.ld[1] = ma; A.cols[1] = ma;
      A.p[2] = Pa; A.ld[2] = ma; A.cols[2] = mp;
      if (which == GR_WW) { B = A; out = d.gS; return true; }
      B.nblk = A.nblk;
      B.p[0] = AX; B.ld[0] = m; B.cols[0] = m;
      B.p[1] = ARa; B.ld[1] = ma; B.cols[1] = ma;
      B.p[2] = APa; B.ld[2] = ma; B.cols[2] = mp;
      out = d.gT;
      return true;
    }
  }
}

// Launched once per distinct block width m present: the tile shape (and so the order of every
// sum) then depends only on the slot's own sizes, never on which other solves share the batch.
template <int MR, int MC>
__global__ void __launch_bounds__(512)
e_gram_kernel(const ESlot* __restrict__ S, int ns, int which, int m_only, int ptc) {
  extern __shared__ __align__(16) unsigned char gsm_e[];
  const int k = slot_of(S, ns, blockIdx.x, &ESlot::gram0);
  const ESlot& d = S[k];
  if (d.m != m_only) return;
  const int part = blockIdx.x - d.gram0;
  const long long r0 = (long long)part * d.rows_per_gpart;
  double2* out;
  if (d.prec == QDKP_C64) {
    BlockList<float> A, B;
    if (!gram_lists<float>(d, which, A, B, out)) return;
    const int RP = (2 * A.total() + 7) / 8 * 8, RQ = (2 * B.total() + 7) / 8 * 8;
    // complex64 blocks, FP64 products: the Gram matrices of the search stay exact to FP64
    // (the split TF32 form loses convergence in the explicit-Gram regime of scipy's method)
    double* po = d.gpart + (long long)part * RP * RQ;
    gram_core<MR, MC>(A, B, r0, min(d.n, r0 + d.rows_per_gpart), po, gsm_e, blockIdx.y * ptc,
                      ptc);
    gram_finish_last(d.gpart, d.gparts, kEGramSplit, d.st->gram_done, A.total(), B.total(), part, out);
  } else {
    BlockList<double> A, B;
    if (!gram_lists<double>(d, which, A, B, out)) return;
    const int RP = (2 * A.total() + 7) / 8 * 8, RQ = (2 * B.total() + 7) / 8 * 8;
    gram_core<MR, MC>(A, B, r0, min(d.n, r0 + d.rows_per_gpart),
                      d.gpart + (long long)part * RP * RQ, gsm_e, blockIdx.y * ptc, ptc);
    gram_finish_last(d.gpart, d.gparts, kEGramSplit, d.st->gram_done, A.total(), B.total(), part, out);
  }
}

// ---------------------------------------------------------------------------------------------
// block updates, multi-slot (FP64 MMA, rows staged through shared memory: in-place safe)
// ---------------------------------------------------------------------------------------------
template <typename T>
__device__ bool upd_lists(const ESlot& d, int which, BlockList<T>& A, const double2* C[3],
                          int& q, cplx<T>*& Y, int& accumulate, int& neg,
                          const double2* C2[3], cplx<T>*& Y2) {
  const EState* st = d.st;
  if (st->idle) return false;
  const int m = d.m, ma = st->ma, mp = st->mp;
  accumulate = 0; neg = 0;
  Y2 = nullptr;
  auto set = [&](int i, double2* p, int ld, int c, const double2* cf) {
    A.p[i] = blk<T>(p); A.ld[i] = ld; A.cols[i] = c; C[i] = cf;
  };
  switch (which) {
    case UP_RPROJ: A.nblk = 1; set(0, d.X, m, m, d.W); q = ma; Y = blk<T>(d.Ra); accumulate = 1; neg = 1; return true;
    case UP_RNORM: A.nblk = 1; set(0, d.Ra, ma, ma, d.U); q = ma; Y = blk<T>(d.Ra); return true;
    case UP_PNORM:
      if (st->skip_pnorm) return false;
      A.nblk = 1; set(0, d.Pa, ma, ma, d.U); q = ma; Y = blk<T>(d.Pa); return true;
    case UP_APNORM:
      if (st->skip_pnorm) return false;
      A.nblk = 1; set(0, d.APa, ma, ma, d.U); q = ma; Y = blk<T>(d.APa); return true;
    default: {        // UP_XPNEW / UP_AXPNEW
      const bool ax = which == UP_AXPNEW;
      A.nblk = mp ? 3 : 2;
      set(0, ax ? d.AX : d.X, m, m, nullptr);            // X rows do not enter P
      set(1, ax ? d.ARa : d.Ra, ma, ma, d.Cr);
      set(2, ax ? d.APa : d.Pa, ma, mp, d.Cp);
      C2[0] = d.Cx; C2[1] = d.Cr; C2[2] = d.Cp;
      q = m;
      Y = blk<T>(ax ? d.AP : d.P);
      Y2 = blk<T>(ax ? d.AX : d.X);
      return true;
    }
  }
}

// One launch per precision present; CTAs of the other precision's slots return at once.
template <typename T>
__global__ void __launch_bounds__(kUpdThreads, 2)
e_update_kernel(const ESlot* __restrict__ S, int ns, int which) {
  extern __shared__ __align__(16) unsigned char usm_e[];
  const int k = slot_of(S, ns, blockIdx.x, &ESlot::row0);
  const ESlot& d = S[k];
  constexpr int prec = std::is_same<T, float>::value ? QDKP_C64 : QDKP_C128;
  if (d.prec != prec) return;
  const double2* Cf[3];
  const double2* C2[3] = {nullptr, nullptr, nullptr};
  int q, accumulate, neg;
  const long long r0 = (long long)(blockIdx.x - d.row0) * d.rows_per_cta;
  const long long r1 = min(d.n, r0 + d.rows_per_cta);
  BlockList<T> A;
  cplx<T> *Y, *Y2;
  if (!upd_lists<T>(d, which, A, Cf, q, Y, accumulate, neg, C2, Y2)) return;
  if constexpr (std::is_same<T, float>::value)
    update_rows_tf32(A, Cf, q, r0, r1, Y, (long long)q, accumulate, neg, usm_e, C2, Y2);
  else
    update_rows(A, Cf, q, r0, r1, Y, (long long)q, accumulate, neg, usm_e, C2, Y2);
}

// complex64 slots: the same updates on the tcgen05 tensor cores (umma_dev.cuh). The CTAs split
// the 128-row tiles of the group's complex64 slots (slot k's tiles start at utile0) into
// contiguous ranges, one CTA per SM; a CTA's tiles of one slot form one pipelined run. A wait
// that gives up leaves NaN in the outputs, which the slot's next residual check turns into status
// nonfinite. Every row is computed the same way whichever CTA holds it, so results do not depend
// on the mix of slots.
__global__ void __launch_bounds__(kUmmaThreads, 1)
e_update_umma_kernel(const ESlot* __restrict__ S, int ns, int which, int utiles, int m_max) {
  extern __shared__ __align__(128) unsigned char usm_u[];
  const bool fused = which == UP_XPNEW || which == UP_AXPNEW;
  const UmmaPlan pl = umma_plan((fused ? 3 : 1) * m_max, m_max, fused ? 2 : 1, m_max, m_max);
  const long long per = (utiles + gridDim.x - 1) / gridDim.x;
  long long c = (long long)blockIdx.x * per;
  const long long c1 = min((long long)utiles, c + per);
  if (c >= c1) return;
  UmmaCtx cx;
  umma_ctx_init(cx, pl);
  bool ok = true;
  while (c < c1) {
    int k = -1;
    long long nt = 0;
    for (int j = 0; j < ns && k < 0; ++j) {
      if (S[j].prec != QDKP_C64) continue;
      nt = (S[j].n + kUmmaRows - 1) / kUmmaRows;
      if (c >= S[j].utile0 && c < S[j].utile0 + nt) k = j;
    }
    if (k < 0) break;                                  // uniform; not reached
    const ESlot& d = S[k];
    const long long seg_end = min(c1, (long long)d.utile0 + nt);
    const double2* Cf[3];
    const double2* C2[3] = {nullptr, nullptr, nullptr};
    int q, accumulate, neg;
    BlockList<float> A;
    float2 *Y, *Y2;
    if (upd_lists<float>(d, which, A, Cf, q, Y, accumulate, neg, C2, Y2)) {
      const long long r0 = (c - d.utile0) * kUmmaRows;
      const long long r1 = min(d.n, (seg_end - d.utile0) * kUmmaRows);
      if (ok) {
        ok = update_rows_umma(pl, cx, A, Cf, q, r0, r1, Y, (long long)q, accumulate, neg, usm_u, C2, Y2);
      } else {
        float2* const Ys[2] = {Y, Y2};
        umma_fill_nan(Ys, Y2 ? 2 : 1, q, r0, r1, (long long)q);
      }
    }
    c = seg_end;
  }
  umma_ctx_free(cx);
}

// ---------------------------------------------------------------------------------------------
// per-slot Cholesky steps and Rayleigh-Ritz
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kSmallThreads) e_rchol_kernel(const ESlot* __restrict__ S) {
  extern __shared__ double2 ssm_e[];
  const ESlot& d = S[blockIdx.x];
  EState* st = d.st;
  if (st->idle) return;
  const int n = st->ma;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) ssm_e[e] = d.G[e];
  __syncthreads();
  const int fail = block_cholesky_upper(ssm_e, n);
  if (fail) {
    if (threadIdx.x == 0) { st->running = 0; st->status = QDKP_LOBPCG_RCHOL_BREAKDOWN; st->idle = 1; }
    return;
  }
  block_upper_inverse(ssm_e, n, ssm_e + n * n);
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) d.U[e] = ssm_e[n * n + e];
}

__global__ void __launch_bounds__(kSmallThreads) e_pchol_kernel(const ESlot* __restrict__ S) {
  extern __shared__ double2 ssm_e[];
  const ESlot& d = S[blockIdx.x];
  EState* st = d.st;
  if (st->idle) return;
  const int n = st->ma;
  if (st->skip_p) {                        // iteration 0: no P yet, restart stays as it is
    if (threadIdx.x == 0) { st->skip_pnorm = 1; st->mp = st->restart ? 0 : n; }
    return;
  }
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) ssm_e[e] = d.G[e];
  __syncthreads();
  const int fail = block_cholesky_upper(ssm_e, n);
  if (!fail) {
    block_upper_inverse(ssm_e, n, ssm_e + n * n);
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) d.U[e] = ssm_e[n * n + e];
  }
  if (threadIdx.x == 0) {
    st->skip_pnorm = fail ? 1 : 0;
    st->restart = fail ? 1 : st->forced;
    st->mp = st->restart ? 0 : n;
  }
}

// gramA / gramB of lobpcg.py:826-909 from S = W^H W and T = W^H AW, then the generalized eigh,
// with the fall back to the two-block pencil when the three-block one is not definite.
__device__ void e_assemble(const ESlot& d, const EState* st, int restart, int& dim) {
  const int m = d.m, ma = st->ma, mp = restart ? 0 : st->mp;
  const int tot = m + st->ma + st->mp;      // rows of gT; layout of the explicit products
  dim = m + ma + mp;
  const bool ex = st->explicit_gram;
  const int nAB = st->ma + st->mp;          // non-explicit gT = [X|R|P]^H [AR|AP]: tot x nAB
  for (int e = threadIdx.x; e < dim * dim; e += blockDim.x) {
    int i = e / dim, j = e - i * dim;
    bool lower = i > j;
    if (lower) { const int t = i; i = j; j = t; }
    const bool iX = i < m, iR = i >= m && i < m + ma, jX = j < m, jR = j >= m && j < m + ma;
    double2 Tij, Tji, Sij;
    if (ex) {
      Tij = d.gT[i * tot + j]; Tji = d.gT[j * tot + i]; Sij = d.gS[i * tot + j];
    } else {
      // column j >= m of W^H AW is column j - m of [AR | AP]; gS = [X|R]^H P (m+ma x mp)
      Tij = j >= m ? d.gT[i * nAB + (j - m)] : make_double2(0.0, 0.0);
      Tji = (i >= m && j >= m) ? d.gT[j * nAB + (i - m)] : make_double2(0.0, 0.0);
      Sij = (j >= m + ma && i < m + ma) ? d.gS[i * st->mp + (j - m - ma)] : make_double2(0.0, 0.0);
    }
    const double2 herm = make_double2(0.5 * (Tij.x + Tji.x), 0.5 * (Tij.y - Tji.y));
    double2 a, b;
    if (iX && jX) {
      if (ex) { a = herm; b = Sij; }
      else { a = make_double2(i == j ? st->lam[i] : 0.0, 0.0); b = make_double2(i == j ? 1.0 : 0.0, 0.0); }
    } else if (iX && jR) {
      a = Tij; b = ex ? Sij : make_double2(0.0, 0.0);
    } else if ((iR && jR) || (!iX && !iR && !jX && !jR)) {
      a = ex ? herm : Tij;
      b = ex ? Sij : make_double2(i == j ? 1.0 : 0.0, 0.0);
    } else {
      a = Tij; b = Sij;
    }
    if (lower) { a.y = -a.y; b.y = -b.y; }
    d.gA[e] = a;
    d.gB[e] = b;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kSmallThreads) e_rr_kernel(const ESlot* __restrict__ S) {
  extern __shared__ double2 rsm[];
  const ESlot& d = S[blockIdx.x];
  EState* st = d.st;
  if (st->idle) return;
  __shared__ int use_restart, ok, dim_s;
  if (threadIdx.x == 0) { use_restart = st->mp == 0; ok = 0; }
  __syncthreads();
  for (int attempt = 0; attempt < 2; ++attempt) {
    int dim;
    e_assemble(d, st, use_restart, dim);
    // only the first m Ritz pairs are kept
    const int r = block_eigh(d.gA, d.gB, dim, d.w, d.E, d.scr, rsm, rsm + dim * dim, d.m);
    if (threadIdx.x == 0) { ok = r == 0; dim_s = dim; }
    __syncthreads();
    if (ok || use_restart) break;
    if (threadIdx.x == 0) use_restart = 1;    // drop P and retry (lobpcg.py:891-909)
    __syncthreads();
  }
  if (!ok) {
    if (threadIdx.x == 0) { st->running = 0; st->status = QDKP_LOBPCG_EIGH_BREAKDOWN; st->idle = 1; }
    return;
  }
  const int m = d.m, ma = st->ma, dim = dim_s;
  const int mp = dim - m - ma;
  for (int e = threadIdx.x; e < dim * m; e += blockDim.x) {
    const int i = e / m, j = e - i * m;
    const double2 v = d.E[i * dim + j];
    if (i < m) d.Cx[i * m + j] = v;
    else if (i < m + ma) d.Cr[(i - m) * m + j] = v;
    else d.Cp[(i - m - ma) * m + j] = v;
  }
  if (threadIdx.x < m) st->lam[threadIdx.x] = d.w[threadIdx.x];
  if (threadIdx.x == 0) { st->restart = use_restart ? 1 : st->restart; st->mp = mp; }
}

}  // namespace qdkp

// =============================================================================================
// host side
// =============================================================================================
namespace qdkp {
namespace {

struct SlotHost {
  bool used = false;
  const qdkp_operator* op = nullptr;
  qdkp_lobpcg_params prm{};
  ESlot d{};
  size_t gpart_doubles = 0;
  int64_t applies = 0;
};

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

struct SlotLayout {
  size_t blk, small, npart, gpart, total;
  int nparts, gparts;
  long long rows_per_gpart;
};

SlotLayout slot_layout(int64_t n, int m, int prec) {
  SlotLayout L;
  L.blk = align256((size_t)n * m * (prec == QDKP_C64 ? sizeof(float2) : sizeof(double2)));
  L.small = align256((size_t)(3 * m) * (3 * m) * sizeof(double2));
  L.nparts = (int)((n + kENormRows - 1) / kENormRows);
  L.npart = align256((size_t)L.nparts * m * sizeof(double));
  long long parts = (n + 255) / 256;
  if (parts > kEGramMaxParts) parts = kEGramMaxParts;
  if (parts < 1) parts = 1;
  long long rpp = (n + parts - 1) / parts;
  rpp = (rpp + 3) / 4 * 4;
  L.gparts = (int)((n + rpp - 1) / rpp);
  L.rows_per_gpart = rpp;
  const size_t RP = (6 * m + 7) / 8 * 8;
  L.gpart = align256((size_t)(L.gparts + kEGramSplit) * RP * RP * sizeof(double));
  L.total = align256(sizeof(EState)) + 10 * L.blk + 14 * L.small +
            align256(3 * m * sizeof(double)) + L.npart + L.gpart;
  return L;
}

// The used slots are split into up to kEGroups groups whose ticks run on streams of their own:
// the groups share no data, so while one group is in its latency-bound kernels (the
// Rayleigh-Ritz eigensolve and the small Cholesky, reduction and decision kernels, one CTA per
// slot) the other group's tall kernels fill the GPU. A slot's kernels and partitions are the
// same in any group, so grouping changes no result.
constexpr int kEGroups = 2;

struct EGroup {
  ESlot* d_slots = nullptr;            // this group's run of the compact slot array
  HXSlot* d_hx = nullptr;              // [precision][phase][slot]: 2 x 4 x max_slots descriptors
  int ns = 0, norm_ctas = 0, gram_ctas = 0, row_ctas = 0;
  int utiles = 0;                      // 128-row tiles of the complex64 slots (tcgen05 updates)
  int nsm = 148;
  int hx_ns[2] = {0, 0}, hx_tiles[2] = {0, 0};   // per precision (QDKP_C128, QDKP_C64)
  int m_max = 1;
  std::vector<int> widths;             // distinct block widths among the group's slots
};

}  // namespace
}  // namespace qdkp

struct qdkp_engine {
  int device = 0;
  int max_slots = 0;
  std::vector<qdkp::SlotHost> slots;
  qdkp::ESlot* d_slots = nullptr;      // compact array of the used slots (group after group)
  qdkp::HXSlot* d_hx = nullptr;        // H.X descriptors, kEGroups x 8 x max_slots
  int* d_one = nullptr;                // constant 1 (skip flag)
  int ns = 0;                          // used slots
  int ngroups = 0;
  int nsm = 148;                       // SMs of the device (grid of the tcgen05 updates)
  qdkp::EGroup grp[qdkp::kEGroups];
  bool dirty = true;
  // CUDA graph of `graph_ticks` ticks over the current slot layout, replayed by
  // qdkp_engine_step on the engine's own stream (ordered after the caller's stream by events)
  cudaStream_t gstream = nullptr, gstream2 = nullptr;   // group 0 and group 1
  cudaEvent_t ev_in = nullptr, ev_out = nullptr, ev_fork = nullptr, ev_join = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_ticks = 0;
  bool use_graph = true;
  long long launches_per_tick = 0;     // kernels one tick launches (graph replays count them)
};

namespace qdkp {
namespace {

// Host helpers on a slot's tall blocks, in the slot's precision (the block pointers are typed
// double2 in ESlot and hold complex64 values for a QDKP_C64 slot).
int apply_folded(const SlotHost& h, const void* V, int c, void* out, cudaStream_t st) {
  const ESlot& d = h.d;
  if (h.prm.folded) {
    int rc = launch_apply(h.op, V, c, d.T, c, c, h.prm.sigma, 1, d.prec, st);
    if (rc) return rc;
    return launch_apply(h.op, d.T, c, out, c, c, h.prm.sigma, 1, d.prec, st);
  }
  return launch_apply(h.op, V, c, out, c, c, 0.0, 0, d.prec, st);
}

template <typename T>
BlockList<T> one(const void* p, int c) {
  BlockList<T> L;
  L.nblk = 1; L.p[0] = static_cast<const cplx<T>*>(p); L.ld[0] = c; L.cols[0] = c;
  return L;
}

int gram1(const SlotHost& h, const void* A, const void* B, int m, double2* out,
          cudaStream_t st) {
  const size_t elems = h.gpart_doubles / 2;
  double2* part = reinterpret_cast<double2*>(h.d.gpart);
  if (h.d.prec == QDKP_C64)
    return launch_gram(one<float>(A, m), one<float>(B, m), h.d.n, part, elems, out, st);
  return launch_gram(one<double>(A, m), one<double>(B, m), h.d.n, part, elems, out, st);
}

// Y (n x q) = A (n x m) C (m x q)
int update1(const SlotHost& h, const void* A, int m, const double2* C, int q, void* Y,
            cudaStream_t st) {
  const double2* Cs[1] = {C};
  if (h.d.prec == QDKP_C64)
    return launch_update(one<float>(A, m), Cs, q, h.d.n, static_cast<float2*>(Y), q, 0, st);
  return launch_update(one<double>(A, m), Cs, q, h.d.n, static_cast<double2*>(Y), q, 0, st);
}

// out[j] = sum_r |A[r, j] - lambda_j B[r, j]|^2, summed on the device into out (device)
int colnorm1(const SlotHost& h, const void* A, const void* B, const double* lam, int m,
             double* out, cudaStream_t st) {
  const ESlot& d = h.d;
  if (d.prec == QDKP_C64)
    return launch_colnorm2<float>(static_cast<const float2*>(A), m, static_cast<const float2*>(B),
                                  m, lam, m, d.n, d.npart, d.nparts, out, st);
  return launch_colnorm2<double>(static_cast<const double2*>(A), m,
                                 static_cast<const double2*>(B), m, lam, m, d.n, d.npart,
                                 d.nparts, out, st);
}

int copy1(const SlotHost& h, const void* src, int m, void* dst, cudaStream_t st) {
  if (h.d.prec == QDKP_C64)
    return launch_copy<float, float>(static_cast<const float2*>(src), m, m, h.d.n,
                                     static_cast<float2*>(dst), m, st);
  return launch_copy<double, double>(static_cast<const double2*>(src), m, m, h.d.n,
                                     static_cast<double2*>(dst), m, st);
}

int read_sync(void* host, const void* dev, size_t bytes, cudaStream_t st) {
  QDKP_CUDA_TRY(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, st));
  QDKP_CUDA_TRY(cudaStreamSynchronize(st));
  return QDKP_OK;
}

// descriptors of group g (slots `ids`, compact-array positions from `base` on)
int build_group(qdkp_engine* e, int g, const std::vector<int>& ids, int base, cudaStream_t st) {
  EGroup& G = e->grp[g];
  G = EGroup();
  G.d_slots = e->d_slots + base;
  G.d_hx = e->d_hx + (size_t)g * 8 * e->max_slots;
  std::vector<ESlot> compact;
  std::vector<HXSlot> hx(8 * (size_t)e->max_slots);
  int norm0 = 0, gram0 = 0, row0 = 0, m_max = 1, utile0 = 0;
  int tile0[2] = {0, 0}, kp[2] = {0, 0};
  for (int i : ids) {
    SlotHost& h = e->slots[i];
    ESlot d = h.d;
    d.norm0 = norm0; norm0 += d.nparts;
    d.gram0 = gram0; gram0 += d.gparts;
    d.row0 = row0; row0 += (int)((d.n + d.rows_per_cta - 1) / d.rows_per_cta);
    d.utile0 = -1;
    if (d.prec == QDKP_C64) { d.utile0 = utile0; utile0 += (int)((d.n + kUmmaRows - 1) / kUmmaRows); }
    h.d = d;
    compact.push_back(d);
    const int pi = d.prec == QDKP_C64 ? 1 : 0;
    const int k = kp[pi]++;
    const qdkp_operator* op = h.op;
    m_max = std::max(m_max, d.m);
    const int tiles = apply_tiles(op->n_sites, d.m);
    for (int t = 0; t < 4; ++t) {
      HXSlot x{};
      x.rec = pi ? (const void*)op->rec32 : (const void*)op->rec64;
      x.msk = op->nbmask; x.N = (int)op->n_sites;
      x.sx = op->ny * op->nz; x.sy = op->nz;
      x.nzp = op->nzp; x.NP = op->nx * op->ny * op->nzp;
      x.tile0 = tile0[pi]; x.cb = apply_cb_weight(op);
      x.sigma = h.prm.sigma;
      x.shifted = h.prm.folded ? 1 : 0;
      const bool recompute = t < 2;
      if (recompute) { x.m = d.m; x.m_dev = nullptr; x.ld_same = 0; x.ldx = d.m; x.ldy = d.m; }
      else { x.m = 0; x.m_dev = &d.st->ma; x.ld_same = 1; }
      const int* skipflag = recompute ? &d.st->skip_recompute : &d.st->idle;
      if (h.prm.folded) {
        x.X = (t == 0) ? (const void*)d.X : (t == 2) ? (const void*)d.Ra : (const void*)d.T;
        x.Y = (t == 0 || t == 2) ? (void*)d.T : (t == 1) ? (void*)d.AX : (void*)d.ARa;
        x.skip = skipflag;
      } else {
        x.X = recompute ? (const void*)d.X : (const void*)d.Ra;
        x.Y = recompute ? (void*)d.AX : (void*)d.ARa;
        x.skip = (t == 1 || t == 3) ? e->d_one : skipflag;
      }
      hx[((size_t)pi * 4 + t) * e->max_slots + k] = x;
    }
    tile0[pi] += tiles;
  }
  G.ns = (int)compact.size();
  G.norm_ctas = norm0; G.gram_ctas = gram0; G.row_ctas = row0;
  G.utiles = utile0;
  G.nsm = e->nsm;
  for (int pi = 0; pi < 2; ++pi) { G.hx_ns[pi] = kp[pi]; G.hx_tiles[pi] = tile0[pi]; }
  G.m_max = m_max;
  for (const ESlot& d : compact)
    if (std::find(G.widths.begin(), G.widths.end(), d.m) == G.widths.end()) G.widths.push_back(d.m);
  std::sort(G.widths.begin(), G.widths.end());
  if (G.ns) {
    QDKP_CUDA_TRY(cudaMemcpyAsync(G.d_slots, compact.data(), compact.size() * sizeof(ESlot),
                                  cudaMemcpyHostToDevice, st));
    QDKP_CUDA_TRY(cudaMemcpyAsync(G.d_hx, hx.data(), hx.size() * sizeof(HXSlot),
                                  cudaMemcpyHostToDevice, st));
  }
  return QDKP_OK;
}

// Split the used slots into groups, balancing rows x block width greedily in slot order.
int rebuild(qdkp_engine* e, cudaStream_t st) {
  std::vector<int> ids[kEGroups];
  double load[kEGroups] = {};
  int used = 0;
  for (int i = 0; i < e->max_slots; ++i) used += e->slots[i].used ? 1 : 0;
  const int ng = std::max(1, std::min(kEGroups, used));
  for (int i = 0; i < e->max_slots; ++i) {
    const SlotHost& h = e->slots[i];
    if (!h.used) continue;
    int g = 0;
    for (int c = 1; c < ng; ++c) if (load[c] < load[g]) g = c;
    ids[g].push_back(i);
    load[g] += (double)h.d.n * h.d.m;
  }
  e->ns = used;
  e->ngroups = ng;
  int base = 0;
  for (int g = 0; g < kEGroups; ++g) {
    if (g >= ng) { e->grp[g] = EGroup(); continue; }
    const int rc = build_group(e, g, ids[g], base, st);
    if (rc) return rc;
    base += (int)ids[g].size();
  }
  e->dirty = false;
  return QDKP_OK;
}

int launch_gram_multi(const EGroup& G, int which, cudaStream_t st) {
  for (int m : G.widths) {
    int P = m, Q = m;
    if (which == GR_BA) { P = 3 * m; Q = 2 * m; }
    else if (which == GR_BB) { P = 2 * m; Q = m; }
    else if (which == GR_WW || which == GR_WAW) { P = 3 * m; Q = 3 * m; }
    const size_t smem = std::max(gram_smem_bytes(P, Q, (int)sizeof(double2)),
                                 gram_smem_bytes(P, Q, (int)sizeof(float2)));
    // the plan for the widest product this width can form; a narrower one on the device leaves
    // its last panels empty
    const GramPlan gp = gram_plan(P, Q);
    e_gram_kernel<3, 3><<<dim3(G.gram_ctas, gp.panels), gp.threads, smem, st>>>(
        G.d_slots, G.ns, which, m, gp.ptc);
    count_launch();
  }
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

int launch_update_multi(const EGroup& G, int which, cudaStream_t st) {
  const bool fused = which == UP_XPNEW || which == UP_AXPNEW;
  const int P = (fused ? 3 : 1) * G.m_max, nout = fused ? 2 : 1;
  if (G.hx_ns[0]) {
    const size_t smem = update_smem_bytes(P, G.m_max, nout);
    e_update_kernel<double><<<G.row_ctas, kUpdThreads, smem, st>>>(G.d_slots, G.ns, which);
    count_launch();
  }
  if (G.hx_ns[1] && !c64_update_tcgen05()) {
    const size_t smem = update_tf32_smem_bytes(P, G.m_max, nout);
    e_update_kernel<float><<<G.row_ctas, kUpdThreads, smem, st>>>(G.d_slots, G.ns, which);
    count_launch();
  } else if (G.hx_ns[1] && G.utiles) {
    const UmmaPlan pl = umma_plan(P, G.m_max, nout, G.m_max, G.m_max);
    if (!pl.nout_pass) { set_error("tcgen05 update plan does not fit shared memory"); return QDKP_ERR_ARG; }
    e_update_umma_kernel<<<std::min(G.utiles, G.nsm), kUmmaThreads, pl.bytes, st>>>(
        G.d_slots, G.ns, which, G.utiles, G.m_max);
    count_launch();
  }
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

// one H.X phase of a tick: a multi-slot launch per precision present
int launch_hx_phase(const qdkp_engine* e, const EGroup& G, int phase, cudaStream_t st) {
  for (int pi = 0; pi < 2; ++pi) {
    if (!G.hx_ns[pi]) continue;
    int rc = launch_apply_multi(G.d_hx + ((size_t)pi * 4 + phase) * e->max_slots, G.hx_ns[pi],
                                G.hx_tiles[pi], pi ? QDKP_C64 : QDKP_C128, st);
    if (rc) return rc;
  }
  return QDKP_OK;
}

// one LOBPCG iteration of every running slot of group G
int tick(const qdkp_engine* e, const EGroup& G, cudaStream_t st) {
  const int ns = G.ns;
  if (!ns) return QDKP_OK;
  int rc;
#define ETRY(x) do { rc = (x); if (rc != QDKP_OK) return rc; } while (0)
  const size_t small_smem = 2 * (size_t)G.m_max * G.m_max * sizeof(double2);
  const size_t rr_smem = 2 * (size_t)(3 * G.m_max) * (3 * G.m_max) * sizeof(double2);
  e_norm_kernel<<<G.norm_ctas, kTallThreads, 0, st>>>(G.d_slots, ns);
  e_decide_kernel<<<ns, 32, 0, st>>>(G.d_slots);
  e_row_kernel<<<G.row_ctas, kTallThreads, 0, st>>>(G.d_slots, ns, RW_COPYBEST);
  e_row_kernel<<<G.row_ctas, kTallThreads, 0, st>>>(G.d_slots, ns, RW_RESID);
  count_launch(4);
  QDKP_CUDA_TRY(cudaGetLastError());
  ETRY(launch_hx_phase(e, G, 0, st));
  ETRY(launch_hx_phase(e, G, 1, st));
  e_row_kernel<<<G.row_ctas, kTallThreads, 0, st>>>(G.d_slots, ns, RW_GATHERP);
  count_launch();
  ETRY(launch_gram_multi(G, GR_XR, st));
  ETRY(launch_update_multi(G, UP_RPROJ, st));
  ETRY(launch_gram_multi(G, GR_RR, st));
  e_rchol_kernel<<<ns, kSmallThreads, small_smem, st>>>(G.d_slots);
  count_launch();
  ETRY(launch_update_multi(G, UP_RNORM, st));
  ETRY(launch_hx_phase(e, G, 2, st));
  ETRY(launch_hx_phase(e, G, 3, st));
  ETRY(launch_gram_multi(G, GR_PP, st));
  e_pchol_kernel<<<ns, kSmallThreads, small_smem, st>>>(G.d_slots);
  count_launch();
  ETRY(launch_update_multi(G, UP_PNORM, st));
  ETRY(launch_update_multi(G, UP_APNORM, st));
  ETRY(launch_gram_multi(G, GR_BA, st));
  ETRY(launch_gram_multi(G, GR_BB, st));
  ETRY(launch_gram_multi(G, GR_WW, st));
  ETRY(launch_gram_multi(G, GR_WAW, st));
  e_rr_kernel<<<ns, kSmallThreads, rr_smem, st>>>(G.d_slots);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  ETRY(launch_update_multi(G, UP_XPNEW, st));
  ETRY(launch_update_multi(G, UP_AXPNEW, st));
#undef ETRY
  return QDKP_OK;
}

}  // namespace
}  // namespace qdkp

namespace qdkp {

// `ticks` ticks of every group: group 0 on `st`, group 1 on the engine's second stream, forked
// from and joined back to `st` (the groups share no data, so their ticks interleave freely)
static int run_ticks(qdkp_engine* e, int ticks, cudaStream_t st) {
  int rc = QDKP_OK;
  if (e->ngroups > 1) {
    QDKP_CUDA_TRY(cudaEventRecord(e->ev_fork, st));
    QDKP_CUDA_TRY(cudaStreamWaitEvent(e->gstream2, e->ev_fork, 0));
  }
  for (int t = 0; t < ticks && rc == QDKP_OK; ++t) rc = tick(e, e->grp[0], st);
  for (int t = 0; t < ticks && rc == QDKP_OK && e->ngroups > 1; ++t) rc = tick(e, e->grp[1], e->gstream2);
  if (e->ngroups > 1) {
    // join even after an error, so that a capture in progress ends with no stream left forked
    const cudaError_t r1 = cudaEventRecord(e->ev_join, e->gstream2);
    const cudaError_t r2 = cudaStreamWaitEvent(st, e->ev_join, 0);
    if (rc == QDKP_OK && (r1 != cudaSuccess || r2 != cudaSuccess)) {
      set_error(std::string("engine stream join: ") + cudaGetErrorString(r1 != cudaSuccess ? r1 : r2));
      rc = QDKP_ERR_CUDA;
    }
  }
  return rc;
}

static void drop_graph(qdkp_engine* e) {
  if (e->graph) cudaGraphExecDestroy(e->graph);
  e->graph = nullptr;
  e->graph_ticks = 0;
}

// Capture `ticks` ticks of the current layout into e->graph (from the engine's stream; the
// second group's branch is forked off and joined back inside the graph).
static int capture_ticks(qdkp_engine* e, int ticks) {
  drop_graph(e);
  QDKP_CUDA_TRY(cudaStreamBeginCapture(e->gstream, cudaStreamCaptureModeThreadLocal));
  const long long l0 = launches_so_far();
  const int rc = run_ticks(e, ticks, e->gstream);
  // captured launches are not executions: take them back off the counter
  const long long captured = launches_so_far() - l0;
  count_launch((int)-captured);
  e->launches_per_tick = ticks ? captured / ticks : 0;
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(e->gstream, &g);
  if (rc != QDKP_OK) { if (g) cudaGraphDestroy(g); return rc; }
  if (ce != cudaSuccess) {
    set_error(std::string("engine graph capture: ") + cudaGetErrorString(ce));
    return QDKP_ERR_CUDA;
  }
  const cudaError_t ie = cudaGraphInstantiate(&e->graph, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) {
    e->graph = nullptr;
    set_error(std::string("engine graph instantiate: ") + cudaGetErrorString(ie));
    return QDKP_ERR_CUDA;
  }
  e->graph_ticks = ticks;
  return QDKP_OK;
}

}  // namespace qdkp

using namespace qdkp;

extern "C" {

int qdkp_engine_create(int max_slots, int device, qdkp_engine** out) {
  QDKP_CHECK_ARG(out && max_slots >= 1 && max_slots <= 4096, "bad engine arguments");
  QDKP_CUDA_TRY(cudaSetDevice(device));
  auto* e = new qdkp_engine();
  e->device = device;
  e->max_slots = max_slots;
  e->slots.resize(max_slots);
  cudaError_t err = cudaMalloc(&e->d_slots, sizeof(ESlot) * max_slots);
  if (err == cudaSuccess) err = cudaMalloc(&e->d_hx, sizeof(HXSlot) * kEGroups * 8 * max_slots);
  if (err == cudaSuccess) err = cudaMalloc(&e->d_one, sizeof(int));
  if (err == cudaSuccess) { const int one = 1; err = cudaMemcpy(e->d_one, &one, sizeof(int), cudaMemcpyHostToDevice); }
  if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&e->gstream, cudaStreamNonBlocking);
  if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&e->gstream2, cudaStreamNonBlocking);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->ev_in, cudaEventDisableTiming);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->ev_out, cudaEventDisableTiming);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming);
  if (err == cudaSuccess) err = cudaDeviceGetAttribute(&e->nsm, cudaDevAttrMultiProcessorCount, device);
  if (err != cudaSuccess) {
    set_error(std::string("engine tables: ") + cudaGetErrorString(err));
    cudaFree(e->d_slots); cudaFree(e->d_hx); cudaFree(e->d_one);
    if (e->gstream) cudaStreamDestroy(e->gstream);
    if (e->gstream2) cudaStreamDestroy(e->gstream2);
    if (e->ev_in) cudaEventDestroy(e->ev_in);
    if (e->ev_out) cudaEventDestroy(e->ev_out);
    if (e->ev_fork) cudaEventDestroy(e->ev_fork);
    if (e->ev_join) cudaEventDestroy(e->ev_join);
    delete e;
    return QDKP_ERR_CUDA;
  }
  // dynamic shared memory limits of the engine kernels
  const int big = 200 * 1024;
  cudaFuncSetAttribute(e_gram_kernel<3, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(e_update_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(e_update_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(e_update_umma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kUmmaSmemLimit);
  cudaFuncSetAttribute(e_rr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(e_rchol_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  cudaFuncSetAttribute(e_pchol_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  *out = e;
  return QDKP_OK;
}

int qdkp_engine_destroy(qdkp_engine* e) {
  if (!e) return QDKP_OK;
  cudaSetDevice(e->device);
  drop_graph(e);
  if (e->gstream) { cudaStreamSynchronize(e->gstream); cudaStreamDestroy(e->gstream); }
  if (e->gstream2) { cudaStreamSynchronize(e->gstream2); cudaStreamDestroy(e->gstream2); }
  if (e->ev_in) cudaEventDestroy(e->ev_in);
  if (e->ev_out) cudaEventDestroy(e->ev_out);
  if (e->ev_fork) cudaEventDestroy(e->ev_fork);
  if (e->ev_join) cudaEventDestroy(e->ev_join);
  cudaFree(e->d_slots);
  cudaFree(e->d_hx);
  cudaFree(e->d_one);
  delete e;
  return QDKP_OK;
}

size_t qdkp_engine_slot_workspace_size(const qdkp_operator* op, const qdkp_lobpcg_params* prm) {
  if (!op || !prm || prm->block < 1 || prm->block > kMaxBlock) return 0;
  if (prm->precision != QDKP_C128 && prm->precision != QDKP_C64) return 0;
  return slot_layout((int64_t)op->n_bands * op->n_sites, prm->block, prm->precision).total;
}

int qdkp_engine_admit(qdkp_engine* e, const qdkp_operator* op, const qdkp_lobpcg_params* prm,
                      const void* X0, void* ws, size_t ws_bytes, void* stream, int* slot_out) {
  QDKP_CHECK_ARG(e && op && prm && X0 && ws && slot_out, "NULL argument");
  QDKP_CHECK_ARG(op->n_bands == 8, "the batched engine serves eight-band operators");
  QDKP_CHECK_ARG(prm->block >= 1 && prm->block <= kMaxBlock, "block must be in [1, 24]");
  QDKP_CHECK_ARG(prm->precision == QDKP_C128 || prm->precision == QDKP_C64,
                 "precision must be QDKP_C128 or QDKP_C64");
  QDKP_CHECK_ARG(op->device == e->device, "operator lives on another device");
  const int64_t n = (int64_t)op->n_bands * op->n_sites;
  const int m = prm->block;
  QDKP_CHECK_ARG(n >= 5 * m, "problem too small for LOBPCG");
  QDKP_CHECK_ARG(n * m < (int64_t(1) << 31), "n * block must stay below 2^31 elements");
  const SlotLayout L = slot_layout(n, m, prm->precision);
  if (ws_bytes < L.total) { set_error("engine slot workspace too small"); return QDKP_ERR_WORKSPACE; }
  int id = -1;
  for (int i = 0; i < e->max_slots; ++i) if (!e->slots[i].used) { id = i; break; }
  if (id < 0) { set_error("no free engine slot"); return QDKP_ERR_WORKSPACE; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  SlotHost& h = e->slots[id];
  h = SlotHost();
  h.op = op;
  h.prm = *prm;
  char* p = static_cast<char*>(ws);
  auto take = [&](size_t b) { char* r = p; p += align256(b); return r; };
  ESlot& d = h.d;
  d.st = (EState*)take(sizeof(EState));
  d.X = (double2*)take(L.blk); d.AX = (double2*)take(L.blk); d.P = (double2*)take(L.blk);
  d.AP = (double2*)take(L.blk); d.best = (double2*)take(L.blk); d.Ra = (double2*)take(L.blk);
  d.ARa = (double2*)take(L.blk); d.Pa = (double2*)take(L.blk); d.APa = (double2*)take(L.blk);
  d.T = (double2*)take(L.blk);
  d.W = (double2*)take(L.small); d.G = (double2*)take(L.small); d.U = (double2*)take(L.small);
  d.gS = (double2*)take(L.small); d.gT = (double2*)take(L.small); d.gA = (double2*)take(L.small);
  d.gB = (double2*)take(L.small); d.E = (double2*)take(L.small);
  d.scr = (double2*)take(2 * L.small);
  d.Cx = (double2*)take(L.small); d.Cr = (double2*)take(L.small); d.Cp = (double2*)take(L.small);
  d.Im = (double2*)take(L.small);
  d.w = (double*)take(3 * m * sizeof(double));
  d.npart = (double*)take(L.npart);
  d.gpart = (double*)take(L.gpart);
  h.gpart_doubles = L.gpart / sizeof(double);
  d.n = n; d.m = m; d.folded = prm->folded;
  d.prec = prm->precision;
  d.sqrt_eps = d.prec == QDKP_C64 ? std::sqrt((double)std::numeric_limits<float>::epsilon())
                                  : std::sqrt(std::numeric_limits<double>::epsilon());
  d.tol = prm->tol > 0 ? prm->tol : std::sqrt(std::numeric_limits<double>::epsilon()) * (double)n;
  d.maxiter = prm->maxiter;
  d.stall_iterations = prm->stall_iterations;
  d.restart_control = prm->restart_control > 0 ? prm->restart_control : 20;
  d.nparts = L.nparts; d.gparts = L.gparts; d.rows_per_gpart = L.rows_per_gpart;
  d.rows_per_cta = kERowsPerCta;
  int rc;
#define ATRY(x) do { rc = (x); if (rc != QDKP_OK) return rc; } while (0)
  // X = orthonormalise(X0) (lobpcg.py:620-630)
  if (d.prec == QDKP_C64)
    ATRY((launch_copy<double, float>(static_cast<const double2*>(X0), m, m, n,
                                     reinterpret_cast<float2*>(d.X), m, st)));
  else
    ATRY(launch_copy(static_cast<const double2*>(X0), m, m, n, d.X, m, st));
  ATRY(gram1(h, d.X, d.X, m, d.G, st));
  ATRY(launch_chol_inv(d.G, m, d.U, (int*)d.w, st));
  int stat = 0;
  ATRY(read_sync(&stat, d.w, sizeof(int), st));
  if (stat) { set_error("Linearly dependent initial approximations"); return QDKP_ERR_NUMERIC; }
  ATRY(update1(h, d.X, m, d.U, m, d.X, st));
  // initial Ritz vectors (lobpcg.py:633-660)
  ATRY(apply_folded(h, d.X, m, d.AX, st));
  ATRY(gram1(h, d.X, d.AX, m, d.gT, st));
  ATRY(launch_eigh(d.gT, nullptr, m, d.w, d.E, d.scr, (int*)d.G, st));
  ATRY(read_sync(&stat, d.G, sizeof(int), st));
  // the eigensolve fails only on non-finite input (a NaN or inf in the operator's fields or in
  // X0): the slot is admitted already stopped with status nonfinite, and retires like any other
  const bool nonfinite = stat != 0;
  std::vector<double> w(m, std::numeric_limits<double>::quiet_NaN());
  if (!nonfinite) {
    ATRY(update1(h, d.X, m, d.E, m, d.X, st));
    ATRY(update1(h, d.AX, m, d.E, m, d.AX, st));
    ATRY(read_sync(w.data(), d.w, m * sizeof(double), st));
  }
  EState s0{};
  s0.running = nonfinite ? 0 : 1;
  s0.status = nonfinite ? QDKP_LOBPCG_NONFINITE : QDKP_LOBPCG_MAXITER;
  s0.iter = -1; s0.idle = 1;
  s0.ma = m; s0.mp = 0; s0.restart = 1; s0.forced = 0; s0.explicit_gram = 0;
  s0.best_iter = prm->maxiter; s0.skip_recompute = 1; s0.skip_p = 1; s0.skip_pnorm = 1;
  s0.smallest = std::numeric_limits<double>::max();
  for (int j = 0; j < m; ++j) { s0.active[j] = 1; s0.lam[j] = w[j]; }
  std::vector<double2> Im((size_t)m * m, make_double2(0.0, 0.0));
  for (int j = 0; j < m; ++j) Im[(size_t)j * m + j] = make_double2(1.0, 0.0);
  QDKP_CUDA_TRY(cudaMemcpyAsync(d.Im, Im.data(), Im.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
  QDKP_CUDA_TRY(cudaMemcpyAsync(d.st, &s0, sizeof(EState), cudaMemcpyHostToDevice, st));
  QDKP_CUDA_TRY(cudaStreamSynchronize(st));
#undef ATRY
  h.used = true;
  e->dirty = true;
  *slot_out = id;
  return QDKP_OK;
}

int qdkp_engine_step(qdkp_engine* e, int ticks, void* stream) {
  QDKP_CHECK_ARG(e && ticks >= 0, "bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  QDKP_CUDA_TRY(cudaSetDevice(e->device));
  if (e->dirty) {
    drop_graph(e);
    int rc = rebuild(e, st);
    if (rc) return rc;
  }
  if (ticks == 0 || e->ns == 0) return QDKP_OK;
  if (!e->use_graph) return run_ticks(e, ticks, st);
  // the tick sequence is fixed for a slot layout: replay it as one graph launch
  if (!e->graph || e->graph_ticks != ticks) {
    QDKP_CUDA_TRY(cudaStreamSynchronize(st));   // descriptor uploads of rebuild() landed
    int rc = capture_ticks(e, ticks);
    if (rc) return rc;
  }
  QDKP_CUDA_TRY(cudaEventRecord(e->ev_in, st));
  QDKP_CUDA_TRY(cudaStreamWaitEvent(e->gstream, e->ev_in, 0));
  QDKP_CUDA_TRY(cudaGraphLaunch(e->graph, e->gstream));
  count_launch(e->launches_per_tick * ticks);
  QDKP_CUDA_TRY(cudaEventRecord(e->ev_out, e->gstream));
  QDKP_CUDA_TRY(cudaStreamWaitEvent(st, e->ev_out, 0));
  return QDKP_OK;
}

int qdkp_engine_set_graphs(qdkp_engine* e, int enable) {
  QDKP_CHECK_ARG(e != nullptr, "NULL engine");
  e->use_graph = enable != 0;
  if (!e->use_graph) drop_graph(e);
  return QDKP_OK;
}

int qdkp_engine_poll(qdkp_engine* e, int* state, int* status, int* iterations, void* stream) {
  QDKP_CHECK_ARG(e && state, "bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::vector<EState> hs(e->max_slots);
  for (int i = 0; i < e->max_slots; ++i) {
    const SlotHost& h = e->slots[i];
    if (!h.used) continue;
    QDKP_CUDA_TRY(cudaMemcpyAsync(&hs[i], h.d.st, sizeof(EState), cudaMemcpyDeviceToHost, st));
  }
  QDKP_CUDA_TRY(cudaStreamSynchronize(st));
  for (int i = 0; i < e->max_slots; ++i) {
    const SlotHost& h = e->slots[i];
    state[i] = !h.used ? -1 : (hs[i].running ? 1 : 0);
    if (status) status[i] = h.used ? hs[i].status : -1;
    if (iterations) iterations[i] = h.used ? hs[i].iter + 1 : 0;
  }
  return QDKP_OK;
}

int qdkp_engine_retire(qdkp_engine* e, int slot, double* lambda_out, void* V,
                       double* residuals_out, qdkp_lobpcg_info* info, void* stream) {
  QDKP_CHECK_ARG(e && slot >= 0 && slot < e->max_slots && e->slots[slot].used, "bad slot");
  QDKP_CHECK_ARG(lambda_out && V && info, "NULL argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  SlotHost& h = e->slots[slot];
  ESlot& d = h.d;
  const int m = d.m;
  const int64_t n = d.n;
  int rc;
#define RTRY(x) do { rc = (x); if (rc != QDKP_OK) return rc; } while (0)
  EState s;
  RTRY(read_sync(&s, d.st, sizeof(EState), st));
  std::vector<double> lam(s.lam, s.lam + m), rn2(m), norms(m);
  // residuals of the last iterate; it becomes the best one if it improved (lobpcg.py:975-995)
  double* dl = d.w;
  QDKP_CUDA_TRY(cudaMemcpyAsync(dl, lam.data(), m * sizeof(double), cudaMemcpyHostToDevice, st));
  RTRY(colnorm1(h, d.AX, d.X, dl, m, d.gpart, st));
  RTRY(read_sync(rn2.data(), d.gpart, m * sizeof(double), st));
  double mean = 0.0;
  for (int j = 0; j < m; ++j) mean += std::sqrt(std::fabs(rn2[j]));
  mean /= m;
  int best_iter = s.best_iter;
  if (s.status != QDKP_LOBPCG_NONFINITE && mean < s.smallest) {
    RTRY(copy1(h, d.X, m, d.best, st));
    best_iter = s.iter + 1;
  }
  if (s.status == QDKP_LOBPCG_NONFINITE) {
    // a non-finite residual: no Rayleigh-Ritz on it; the last iterate is returned as it is with
    // NaN Ritz values and residuals, and the slot is freed for the next request
    if (d.prec == QDKP_C64)
      RTRY((launch_copy<float, double>(reinterpret_cast<const float2*>(d.X), m, m, n,
                                       static_cast<double2*>(V), m, st)));
    else
      RTRY((launch_copy<double, double>(reinterpret_cast<const double2*>(d.X), m, m, n,
                                        static_cast<double2*>(V), m, st)));
    QDKP_CUDA_TRY(cudaStreamSynchronize(st));
    for (int j = 0; j < m; ++j) lambda_out[j] = std::numeric_limits<double>::quiet_NaN();
    if (residuals_out)
      for (int j = 0; j < m; ++j) residuals_out[j] = std::numeric_limits<double>::quiet_NaN();
    std::memset(info, 0, sizeof(*info));
    info->iterations = std::min(s.iter + 1, h.prm.maxiter + 3);
    info->best_iteration = best_iter;
    info->status = s.status;
    info->explicit_gram = s.explicit_gram;
    info->best_mean_residual = s.smallest;
    h.used = false;
    e->dirty = true;
    return QDKP_OK;
  }
  // final Rayleigh-Ritz on the best iterate (lobpcg.py:1009-1060)
  RTRY(apply_folded(h, d.best, m, d.AX, st));
  RTRY(gram1(h, d.best, d.AX, m, d.gT, st));
  RTRY(gram1(h, d.best, d.best, m, d.gS, st));
  {
    std::vector<double2> t((size_t)m * m), s2((size_t)m * m), a((size_t)m * m), bb((size_t)m * m);
    RTRY(read_sync(t.data(), d.gT, t.size() * sizeof(double2), st));
    RTRY(read_sync(s2.data(), d.gS, s2.size() * sizeof(double2), st));
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        const double2 x = t[(size_t)i * m + j], y = t[(size_t)j * m + i];
        a[(size_t)i * m + j] = make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
        const double2 u = s2[(size_t)i * m + j], v = s2[(size_t)j * m + i];
        bb[(size_t)i * m + j] = make_double2(0.5 * (u.x + v.x), 0.5 * (u.y - v.y));
      }
    QDKP_CUDA_TRY(cudaMemcpyAsync(d.gA, a.data(), a.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
    QDKP_CUDA_TRY(cudaMemcpyAsync(d.gB, bb.data(), bb.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
  }
  RTRY(launch_eigh(d.gA, d.gB, m, d.w, d.E, d.scr, (int*)d.G, st));
  int stat = 0;
  RTRY(read_sync(&stat, d.G, sizeof(int), st));
  if (stat) { set_error("eigh has failed in lobpcg postprocessing"); return QDKP_ERR_NUMERIC; }
  RTRY(read_sync(lam.data(), d.w, m * sizeof(double), st));
  // Ritz vectors of the best iterate; a complex64 slot forms them in its own precision (in the
  // free folded scratch T) and widens them into the caller's complex128 V
  void* Vs = d.prec == QDKP_C64 ? static_cast<void*>(d.T) : V;
  RTRY(update1(h, d.best, m, d.E, m, Vs, st));
  RTRY(update1(h, d.AX, m, d.E, m, d.AX, st));
  RTRY(colnorm1(h, d.AX, Vs, d.w, m, d.gpart, st));
  if (d.prec == QDKP_C64)
    RTRY((launch_copy<float, double>(reinterpret_cast<const float2*>(d.T), m, m, n,
                                     static_cast<double2*>(V), m, st)));
  RTRY(read_sync(rn2.data(), d.gpart, m * sizeof(double), st));
  bool all = true;
  for (int j = 0; j < m; ++j) {
    norms[j] = std::sqrt(std::fabs(rn2[j]));
    all = all && norms[j] <= d.tol;
  }
  std::memcpy(lambda_out, lam.data(), m * sizeof(double));
  if (residuals_out) std::memcpy(residuals_out, norms.data(), m * sizeof(double));
  int status = s.status;
  if (status == QDKP_LOBPCG_MAXITER && all) status = QDKP_LOBPCG_CONVERGED;
  std::memset(info, 0, sizeof(*info));
  info->iterations = std::min(best_iter + 2, h.prm.maxiter + 3);
  info->best_iteration = best_iter;
  info->status = status;
  info->explicit_gram = s.explicit_gram;
  info->best_mean_residual = s.smallest;
#undef RTRY
  h.used = false;
  e->dirty = true;
  return QDKP_OK;
}

}  // extern "C"
