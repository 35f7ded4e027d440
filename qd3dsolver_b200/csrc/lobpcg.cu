// LOBPCG on the device: the iteration of scipy.sparse.linalg.lobpcg (scipy 1.18.1,
// _eigen/lobpcg/lobpcg.py:688-1060) as qd3Dsolver calls it (eigensolvers.py:247-248, 352-353:
// B = None, M = None, Y = None, largest = False), with every block operation on the GPU.
//
// Per iteration (scipy line ranges in brackets):
//   R = A X - X diag(lambda), residual norms                       [688-700]
//   best-iterate bookkeeping, forced restart                       [702-718]
//   active mask                                                    [720-731]
//   R_act -= X (X^H R_act); Cholesky-orthonormalise R_act          [762-787]
//   A R_act                                                        [788]
//   Cholesky-orthonormalise P_act, A P_act (restart on failure)    [790-809]
//   explicit-Gram switch (sticky)                                  [815-824]
//   Gram blocks, generalized eigh of 3m x 3m (2m x 2m on restart)  [826-909]
//   Ritz update of X, A X, P, A P                                  [911-973]
// then the final Rayleigh-Ritz on the best iterate               [975-1060].
// Decisions that scipy takes on host scalars (active mask, restart, breakdown) are taken here
// on the host from small device-to-host reads; all vectors stay in device memory.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <vector>

#include "blockops.cuh"

namespace qdkp {

int launch_apply(const qdkp_operator* op, const void* X, int64_t ldx, void* Y, int64_t ldy,
                 int m, double sigma, int shifted, int precision, cudaStream_t st);

namespace {

constexpr int kNormParts = 296;

struct Layout {
  size_t blk;          // bytes of one n x m complex128 block
  size_t gpart_elems;  // gram partial elements
  size_t total;
};

Layout layout(int64_t n, int m, int folded) {
  Layout L;
  L.blk = ((size_t)n * m * sizeof(double2) + 255) / 256 * 256;
  L.gpart_elems = gram_partial_elems(3 * m, 3 * m);
  const size_t small = (size_t)(3 * m) * (3 * m) * sizeof(double2);
  L.total = (size_t)(9 + (folded ? 1 : 0)) * L.blk          // X AX P AP best Ra ARa Pa APa [T]
            + L.gpart_elems * sizeof(double2)                 // gram partials
            + 12 * small                                      // small matrices
            + (size_t)kNormParts * m * sizeof(double)         // norm partials
            + 4096 * 4;                                       // vectors, flags
  return L;
}

struct Bufs {
  double2 *X, *AX, *P, *AP, *best, *Ra, *ARa, *Pa, *APa, *T;
  double2* gpart;
  double2 *gS, *gT, *gA, *gB, *E, *scr, *U1, *W;
  double *npart, *norms, *lam, *w;
  int *idx, *status;
};

Bufs carve(void* ws, const Layout& L, int m, int folded) {
  char* p = static_cast<char*>(ws);
  auto take = [&](size_t bytes) { char* r = p; p += (bytes + 255) / 256 * 256; return r; };
  Bufs b;
  b.X = (double2*)take(L.blk); b.AX = (double2*)take(L.blk);
  b.P = (double2*)take(L.blk); b.AP = (double2*)take(L.blk);
  b.best = (double2*)take(L.blk);
  b.Ra = (double2*)take(L.blk); b.ARa = (double2*)take(L.blk);
  b.Pa = (double2*)take(L.blk); b.APa = (double2*)take(L.blk);
  b.T = folded ? (double2*)take(L.blk) : nullptr;
  b.gpart = (double2*)take(L.gpart_elems * sizeof(double2));
  const size_t small = (size_t)(3 * m) * (3 * m) * sizeof(double2);
  b.gS = (double2*)take(small); b.gT = (double2*)take(small);
  b.gA = (double2*)take(small); b.gB = (double2*)take(small);
  b.E = (double2*)take(small); b.scr = (double2*)take(2 * small);
  b.U1 = (double2*)take(small); b.W = (double2*)take(small);
  b.npart = (double*)take((size_t)kNormParts * m * sizeof(double));
  b.norms = (double*)take(m * sizeof(double));
  b.lam = (double*)take(m * sizeof(double));
  b.w = (double*)take(3 * m * sizeof(double));
  b.idx = (int*)take(m * sizeof(int));
  b.status = (int*)take(16 * sizeof(int));
  return b;
}

BlockList<double> blist(std::initializer_list<std::pair<const double2*, int>> blocks, long long ld_default = -1) {
  BlockList<double> L;
  L.nblk = 0;
  for (auto& b : blocks) {
    L.p[L.nblk] = b.first;
    L.cols[L.nblk] = b.second;
    L.ld[L.nblk] = ld_default;
    ++L.nblk;
  }
  return L;
}

struct Solver {
  const qdkp_operator* op;
  qdkp_lobpcg_params prm;
  cudaStream_t st;
  int64_t n;
  int m;
  Layout L;
  Bufs b;
  int64_t applies = 0;
  int64_t hx_launches = 0;
  double hx_bytes = 0.0;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;   // per-launch timing (time_hx)
  size_t ev_used = 0;

  int hx(const double2* V, int c, double2* out, double sigma, int shifted) {
    ++hx_launches;
    hx_bytes += (double)op->n_sites * (15.0 * 8.0 + 2.0 * 8.0 * c * 16.0);
    if (!prm.time_hx) return launch_apply(op, V, c, out, c, c, sigma, shifted, QDKP_C128, st);
    if (ev_used == ev.size()) {
      cudaEvent_t a, b2;
      QDKP_CUDA_TRY(cudaEventCreate(&a));
      QDKP_CUDA_TRY(cudaEventCreate(&b2));
      ev.emplace_back(a, b2);
    }
    auto& e = ev[ev_used++];
    QDKP_CUDA_TRY(cudaEventRecord(e.first, st));
    int rc = launch_apply(op, V, c, out, c, c, sigma, shifted, QDKP_C128, st);
    QDKP_CUDA_TRY(cudaEventRecord(e.second, st));
    return rc;
  }

  // Sum the recorded launch durations (events are complete after the caller's sync).
  double hx_seconds() {
    double t = 0.0;
    for (size_t i = 0; i < ev_used; ++i) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ev[i].first, ev[i].second) == cudaSuccess) t += ms * 1e-3;
    }
    return t;
  }

  ~Solver() {
    for (auto& e : ev) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
  }

  // A(V) for V (n x c, ld c) into out (ld c)
  int applyA(const double2* V, int c, double2* out) {
    applies += c;
    if (prm.folded) {
      int rc = hx(V, c, b.T, prm.sigma, 1);
      if (rc) return rc;
      return hx(b.T, c, out, prm.sigma, 1);
    }
    return hx(V, c, out, 0.0, 0);
  }

  int gram(BlockList<double> A, BlockList<double> B, double2* out) {
    return launch_gram(A, B, n, b.gpart, L.gpart_elems, out, st);
  }

  int sync_read(void* host, const void* dev, size_t bytes) {
    QDKP_CUDA_TRY(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, st));
    QDKP_CUDA_TRY(cudaStreamSynchronize(st));
    return QDKP_OK;
  }

  int put(void* dev, const void* host, size_t bytes) {
    QDKP_CUDA_TRY(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, st));
    return QDKP_OK;
  }
};

// Host-side assembly of the Rayleigh-Ritz pencils from the Gram pieces (scipy lobpcg.py:826-909).
// S = W^H W and T = W^H AW with W = [X | R | P] (sizes m, ma, mp); hS, hT row-major (tot x tot).
void assemble(const std::vector<double2>& hS, const std::vector<double2>& hT, int m, int ma,
              int mp, bool restart, bool explicit_gram, const std::vector<double>& lam,
              std::vector<double2>& gA, std::vector<double2>& gB, int& dim) {
  const int tot = m + ma + mp;
  dim = restart ? m + ma : tot;
  gA.assign((size_t)dim * dim, make_double2(0.0, 0.0));
  gB.assign((size_t)dim * dim, make_double2(0.0, 0.0));
  auto S = [&](int i, int j) { return hS[(size_t)i * tot + j]; };
  auto T = [&](int i, int j) { return hT[(size_t)i * tot + j]; };
  auto herm = [](double2 a, double2 b) {   // (a + conj(b)) / 2
    return make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
  };
  auto conjv = [](double2 a) { return make_double2(a.x, -a.y); };
  // block ranges
  const int x0 = 0, r0 = m, p0 = m + ma;
  for (int i = 0; i < dim; ++i)
    for (int j = i; j < dim; ++j) {
      const bool iX = i < r0, iR = i >= r0 && i < p0, jX = j < r0, jR = j >= r0 && j < p0;
      double2 a, bb;
      if (iX && jX) {                                   // XAX, XBX
        if (explicit_gram) { a = herm(T(i, j), T(j, i)); bb = S(i, j); }
        else { a = make_double2(i == j ? lam[i] : 0.0, 0.0); bb = make_double2(i == j ? 1.0 : 0.0, 0.0); }
      } else if (iX && jR) {                            // XAR, XBR
        a = T(i, j);
        bb = explicit_gram ? S(i, j) : make_double2(0.0, 0.0);
      } else if (iR && jR) {                            // RAR, RBR
        a = explicit_gram ? herm(T(i, j), T(j, i)) : T(i, j);
        bb = explicit_gram ? S(i, j) : make_double2(i == j ? 1.0 : 0.0, 0.0);
      } else if (!iR && !iX && !jR && !jX) {            // PAP, PBP
        a = explicit_gram ? herm(T(i, j), T(j, i)) : T(i, j);
        bb = explicit_gram ? S(i, j) : make_double2(i == j ? 1.0 : 0.0, 0.0);
      } else {                                          // XAP, RAP, XBP, RBP
        a = T(i, j);
        bb = S(i, j);
      }
      gA[(size_t)i * dim + j] = a;
      gB[(size_t)i * dim + j] = bb;
      if (j != i) {
        gA[(size_t)j * dim + i] = conjv(a);
        gB[(size_t)j * dim + i] = conjv(bb);
      }
    }
  (void)x0;
}

}  // namespace
}  // namespace qdkp

using namespace qdkp;

extern "C" {

size_t qdkp_lobpcg_workspace_size(const qdkp_operator* op, const qdkp_lobpcg_params* prm) {
  if (!op || !prm || prm->block < 1 || prm->block > kMaxBlock) return 0;
  const int64_t n = (int64_t)op->n_bands * op->n_sites;
  return layout(n, prm->block, prm->folded).total;
}

int qdkp_lobpcg_solve(const qdkp_operator* op, const qdkp_lobpcg_params* prm, const void* X0,
                      double* lambda_out, void* V, double* resid_history,
                      qdkp_lobpcg_info* info, void* ws, size_t ws_bytes, void* stream) {
  QDKP_CHECK_ARG(op && prm && X0 && lambda_out && V && info, "NULL argument");
  QDKP_CHECK_ARG(prm->block >= 1 && prm->block <= kMaxBlock, "block must be in [1, 24]");
  QDKP_CHECK_ARG(prm->maxiter >= 0, "maxiter must be >= 0");
  if (prm->precision != QDKP_C128) {
    set_error("qdkp_lobpcg_solve: only QDKP_C128 is built for the single-solve form");
    return QDKP_ERR_UNSUPPORTED;
  }
  const auto t_start = std::chrono::steady_clock::now();
  Solver s;
  s.op = op;
  s.prm = *prm;
  s.st = static_cast<cudaStream_t>(stream);
  s.n = (int64_t)op->n_bands * op->n_sites;
  s.m = prm->block;
  const int m = s.m;
  const int64_t n = s.n;
  QDKP_CHECK_ARG(n >= 5 * m, "problem too small for LOBPCG (scipy switches to dense eigh)");
  s.L = layout(n, m, prm->folded);
  if (!ws || ws_bytes < s.L.total) {
    set_error("qdkp_lobpcg_solve: workspace too small (see qdkp_lobpcg_workspace_size)");
    return QDKP_ERR_WORKSPACE;
  }
  s.b = carve(ws, s.L, m, prm->folded);
  Bufs& b = s.b;
  cudaStream_t st = s.st;
  const double eps = std::numeric_limits<double>::epsilon();
  const double tol = prm->tol > 0 ? prm->tol : std::sqrt(eps) * (double)n;
  const int maxiter = prm->maxiter;
  const int restart_control = prm->restart_control > 0 ? prm->restart_control : 20;
  const int hist_rows = maxiter + 3;
  std::vector<double> hist((size_t)hist_rows * m, 0.0);
  int rc;
#define TRY(x) do { rc = (x); if (rc != QDKP_OK) return rc; } while (0)

  // ---- X = orthonormalise(X0) ------------------------------------------------------------
  TRY(launch_copy((const double2*)X0, m, m, n, b.X, m, st));
  TRY(s.gram(blist({{b.X, m}}, m), blist({{b.X, m}}, m), b.gS));
  TRY(launch_chol_inv(b.gS, m, b.U1, b.status, st));
  int hstat[4];
  TRY(s.sync_read(hstat, b.status, sizeof(int)));
  if (hstat[0]) { set_error("Linearly dependent initial approximations"); return QDKP_ERR_NUMERIC; }
  {
    const double2* C[1] = {b.U1};
    TRY(launch_update(blist({{b.X, m}}, m), C, m, n, b.Ra, m, 0, st));
    std::swap(b.X, b.Ra);
  }
  // ---- initial Ritz vectors ------------------------------------------------------------------
  TRY(s.applyA(b.X, m, b.AX));
  TRY(s.gram(blist({{b.X, m}}, m), blist({{b.AX, m}}, m), b.gT));
  TRY(launch_eigh(b.gT, nullptr, m, b.w, b.E, b.scr, b.status, st));
  std::vector<double> lam(m);
  TRY(s.sync_read(lam.data(), b.w, m * sizeof(double)));
  {
    const double2* C[1] = {b.E};
    TRY(launch_update(blist({{b.X, m}}, m), C, m, n, b.X, m, 0, st));
    TRY(launch_update(blist({{b.AX, m}}, m), C, m, n, b.AX, m, 0, st));
  }
  TRY(s.put(b.lam, lam.data(), m * sizeof(double)));

  std::vector<char> active(m, 1);
  std::vector<double> norms(m), rn2(m);
  double smallest = std::numeric_limits<double>::max();
  int best_iter = maxiter;
  bool have_best = false;
  int it = -1;
  bool restart = true, forced = false, explicit_gram = false;
  int status = QDKP_LOBPCG_MAXITER;
  const int M3 = 3 * m;
  std::vector<double2> hS((size_t)M3 * M3), hT((size_t)M3 * M3), gA, gB;
  std::vector<int> idx;

  while (it < maxiter) {
    ++it;
    // residual norms of A X - X lambda
    TRY(launch_colnorm2(b.AX, m, b.X, m, b.lam, m, n, b.npart, kNormParts, b.norms, st));
    TRY(s.sync_read(rn2.data(), b.norms, m * sizeof(double)));
    double mean = 0.0;
    bool finite = true;
    for (int j = 0; j < m; ++j) {
      norms[j] = std::sqrt(std::fabs(rn2[j]));
      mean += norms[j];
      finite = finite && std::isfinite(norms[j]);
    }
    mean /= m;
    std::memcpy(&hist[(size_t)it * m], norms.data(), m * sizeof(double));
    if (!finite) { status = QDKP_LOBPCG_NONFINITE; break; }
    bool do_forced = false;
    if (mean < smallest) {
      smallest = mean;
      best_iter = it;
      TRY(launch_copy(b.X, m, m, n, b.best, m, st));
      have_best = true;
    } else if (mean > std::ldexp(1.0, restart_control) * smallest) {
      forced = true;
      do_forced = true;
    }
    idx.clear();
    for (int j = 0; j < m; ++j) {
      active[j] = active[j] && (norms[j] > tol);
      if (active[j]) idx.push_back(j);
    }
    const int ma = (int)idx.size();
    if (do_forced) {
      // scipy recomputes A X here but keeps the residual block computed from the old A X
      if (ma > 0) {
        TRY(s.put(b.idx, idx.data(), ma * sizeof(int)));
        TRY(launch_resid_gather(b.AX, m, b.X, m, b.lam, b.idx, ma, n, b.Ra, ma, st));
      }
      TRY(s.applyA(b.X, m, b.AX));
    }
    if (ma == 0) { status = QDKP_LOBPCG_CONVERGED; break; }
    if (!do_forced) {
      TRY(s.put(b.idx, idx.data(), ma * sizeof(int)));
      // R_act = A X[:, act] - X[:, act] lambda[act]
      TRY(launch_resid_gather(b.AX, m, b.X, m, b.lam, b.idx, ma, n, b.Ra, ma, st));
    }
    if (it > 0) {
      TRY(launch_gather(b.P, m, b.idx, ma, n, b.Pa, ma, st));
      TRY(launch_gather(b.AP, m, b.idx, ma, n, b.APa, ma, st));
    }
    // R_act -= X (X^H R_act)
    TRY(s.gram(blist({{b.X, m}}, m), blist({{b.Ra, ma}}, ma), b.W));
    {
      // coefficient -W
      std::vector<double2> hW((size_t)m * ma);
      TRY(s.sync_read(hW.data(), b.W, hW.size() * sizeof(double2)));
      for (auto& v : hW) { v.x = -v.x; v.y = -v.y; }
      TRY(s.put(b.W, hW.data(), hW.size() * sizeof(double2)));
      const double2* C[1] = {b.W};
      TRY(launch_update(blist({{b.X, m}}, m), C, ma, n, b.Ra, ma, 1, st));
    }
    // Cholesky-orthonormalise R_act
    TRY(s.gram(blist({{b.Ra, ma}}, ma), blist({{b.Ra, ma}}, ma), b.gS));
    TRY(launch_chol_inv(b.gS, ma, b.U1, b.status, st));
    TRY(s.sync_read(hstat, b.status, sizeof(int)));
    if (hstat[0]) { status = QDKP_LOBPCG_RCHOL_BREAKDOWN; break; }
    {
      const double2* C[1] = {b.U1};
      TRY(launch_update(blist({{b.Ra, ma}}, ma), C, ma, n, b.Ra, ma, 0, st));
    }
    TRY(s.applyA(b.Ra, ma, b.ARa));
    int mp = 0;
    if (it > 0) {
      TRY(s.gram(blist({{b.Pa, ma}}, ma), blist({{b.Pa, ma}}, ma), b.gS));
      TRY(launch_chol_inv(b.gS, ma, b.U1, b.status, st));
      TRY(s.sync_read(hstat, b.status, sizeof(int)));
      if (!hstat[0]) {
        const double2* C[1] = {b.U1};
        TRY(launch_update(blist({{b.Pa, ma}}, ma), C, ma, n, b.Pa, ma, 0, st));
        TRY(launch_update(blist({{b.APa, ma}}, ma), C, ma, n, b.APa, ma, 0, st));
        restart = forced;
      } else {
        restart = true;
      }
    }
    double maxnorm = 0.0;
    for (int j = 0; j < m; ++j) maxnorm = std::max(maxnorm, norms[j]);
    const double myeps = std::sqrt(eps);
    explicit_gram = !(maxnorm > myeps && !explicit_gram);
    if (!restart) mp = ma;
    // Gram pieces S = W^H W, T = W^H AW over W = [X | R_act | P_act]
    const int tot = m + ma + mp;
    BlockList<double> Wl = mp ? blist({{b.X, m}, {b.Ra, ma}, {b.Pa, mp}})
                              : blist({{b.X, m}, {b.Ra, ma}});
    Wl.ld[0] = m; Wl.ld[1] = ma; if (mp) Wl.ld[2] = mp;
    BlockList<double> AWl = mp ? blist({{b.AX, m}, {b.ARa, ma}, {b.APa, mp}})
                               : blist({{b.AX, m}, {b.ARa, ma}});
    AWl.ld[0] = m; AWl.ld[1] = ma; if (mp) AWl.ld[2] = mp;
    hS.assign((size_t)tot * tot, make_double2(0.0, 0.0));
    hT.assign((size_t)tot * tot, make_double2(0.0, 0.0));
    if (explicit_gram) {
      TRY(s.gram(Wl, Wl, b.gS));
      TRY(s.gram(Wl, AWl, b.gT));
      TRY(s.sync_read(hS.data(), b.gS, hS.size() * sizeof(double2)));
      TRY(s.sync_read(hT.data(), b.gT, hT.size() * sizeof(double2)));
    } else {
      // only the blocks the non-explicit pencils read (lobpcg.py:856-861): [X|R|P]^H [AR|AP]
      // and [X|R]^H P, scattered into the full W^H AW / W^H W layouts
      const int nAB = ma + mp;
      BlockList<double> ABl = mp ? blist({{b.ARa, ma}, {b.APa, mp}}) : blist({{b.ARa, ma}});
      ABl.ld[0] = ma; if (mp) ABl.ld[1] = ma;
      TRY(s.gram(Wl, ABl, b.gT));
      std::vector<double2> t2((size_t)tot * nAB);
      TRY(s.sync_read(t2.data(), b.gT, t2.size() * sizeof(double2)));
      for (int i = 0; i < tot; ++i)
        for (int c = 0; c < nAB; ++c) hT[(size_t)i * tot + m + c] = t2[(size_t)i * nAB + c];
      if (mp) {
        BlockList<double> XR = blist({{b.X, m}, {b.Ra, ma}});
        XR.ld[0] = m; XR.ld[1] = ma;
        TRY(s.gram(XR, blist({{b.Pa, mp}}, ma), b.gS));
        std::vector<double2> s2((size_t)(m + ma) * mp);
        TRY(s.sync_read(s2.data(), b.gS, s2.size() * sizeof(double2)));
        for (int i = 0; i < m + ma; ++i)
          for (int c = 0; c < mp; ++c) hS[(size_t)i * tot + m + ma + c] = s2[(size_t)i * mp + c];
      }
    }
    int dim = 0;
    bool solved = false;
    std::vector<double> w(tot);
    for (int attempt = 0; attempt < 2 && !solved; ++attempt) {
      if (attempt == 1) { if (restart) break; restart = true; }
      assemble(hS, hT, m, ma, mp, restart, explicit_gram, lam, gA, gB, dim);
      TRY(s.put(b.gA, gA.data(), gA.size() * sizeof(double2)));
      TRY(s.put(b.gB, gB.data(), gB.size() * sizeof(double2)));
      TRY(launch_eigh(b.gA, b.gB, dim, b.w, b.E, b.scr, b.status, st, m));   // m pairs kept
      TRY(s.sync_read(hstat, b.status, sizeof(int)));
      solved = hstat[0] == 0;
    }
    if (!solved) { status = QDKP_LOBPCG_EIGH_BREAKDOWN; break; }
    TRY(s.sync_read(w.data(), b.w, dim * sizeof(double)));
    for (int j = 0; j < m; ++j) lam[j] = w[j];
    TRY(s.put(b.lam, lam.data(), m * sizeof(double)));
    // Ritz vectors: eigenvector rows [0, m) -> X, [m, m+ma) -> R, [m+ma, dim) -> P; first m cols
    std::vector<double2> E((size_t)dim * dim), Ex((size_t)m * m), Er((size_t)ma * m),
        Ep((size_t)mp * m);
    TRY(s.sync_read(E.data(), b.E, E.size() * sizeof(double2)));
    for (int i = 0; i < dim; ++i)
      for (int j = 0; j < m; ++j) {
        const double2 v = E[(size_t)i * dim + j];
        if (i < m) Ex[(size_t)i * m + j] = v;
        else if (i < m + ma) Er[(size_t)(i - m) * m + j] = v;
        else Ep[(size_t)(i - m - ma) * m + j] = v;
      }
    double2* dEx = b.gA;                              // reuse small buffers for the pieces
    double2* dEr = b.gA + (size_t)m * m;
    double2* dEp = b.gB;
    TRY(s.put(dEx, Ex.data(), Ex.size() * sizeof(double2)));
    TRY(s.put(dEr, Er.data(), Er.size() * sizeof(double2)));
    if (!restart) TRY(s.put(dEp, Ep.data(), Ep.size() * sizeof(double2)));
    {
      // P = R Er + P_act Ep ; AP = AR Er + AP_act Ep
      if (!restart) {
        const double2* C[2] = {dEr, dEp};
        BlockList<double> l1 = blist({{b.Ra, ma}, {b.Pa, ma}});
        l1.ld[0] = ma; l1.ld[1] = ma;
        TRY(launch_update(l1, C, m, n, b.P, m, 0, st));
        BlockList<double> l2 = blist({{b.ARa, ma}, {b.APa, ma}});
        l2.ld[0] = ma; l2.ld[1] = ma;
        TRY(launch_update(l2, C, m, n, b.AP, m, 0, st));
      } else {
        const double2* C[1] = {dEr};
        TRY(launch_update(blist({{b.Ra, ma}}, ma), C, m, n, b.P, m, 0, st));
        TRY(launch_update(blist({{b.ARa, ma}}, ma), C, m, n, b.AP, m, 0, st));
      }
      // X = X Ex + P ; AX = AX Ex + AP
      const double2* C2[2] = {dEx, nullptr};
      std::vector<double2> Id((size_t)m * m, make_double2(0.0, 0.0));
      for (int j = 0; j < m; ++j) Id[(size_t)j * m + j] = make_double2(1.0, 0.0);
      TRY(s.put(b.U1, Id.data(), Id.size() * sizeof(double2)));
      C2[1] = b.U1;
      BlockList<double> lx = blist({{b.X, m}, {b.P, m}});
      lx.ld[0] = m; lx.ld[1] = m;
      TRY(launch_update(lx, C2, m, n, b.X, m, 0, st));
      BlockList<double> lax = blist({{b.AX, m}, {b.AP, m}});
      lax.ld[0] = m; lax.ld[1] = m;
      TRY(launch_update(lax, C2, m, n, b.AX, m, 0, st));
    }
    if (prm->verbosity > 1)
      fprintf(stderr, "lobpcg it %d active %d mean %.3e restart %d explicit %d\n", it, ma, mean,
              (int)restart, (int)explicit_gram);
  }
  // ---- final residuals of the last iterate -------------------------------------------------
  if (status != QDKP_LOBPCG_NONFINITE) {
    TRY(launch_colnorm2(b.AX, m, b.X, m, b.lam, m, n, b.npart, kNormParts, b.norms, st));
    TRY(s.sync_read(rn2.data(), b.norms, m * sizeof(double)));
    double mean = 0.0;
    for (int j = 0; j < m; ++j) { norms[j] = std::sqrt(std::fabs(rn2[j])); mean += norms[j]; }
    mean /= m;
    if (it + 1 < hist_rows) std::memcpy(&hist[(size_t)(it + 1) * m], norms.data(), m * sizeof(double));
    if (mean < smallest) {
      smallest = mean;
      best_iter = it + 1;
      TRY(launch_copy(b.X, m, m, n, b.best, m, st));
      have_best = true;
    }
  }
  if (!have_best) TRY(launch_copy(b.X, m, m, n, b.best, m, st));
  if (status == QDKP_LOBPCG_NONFINITE) {
    // a non-finite residual: nothing to refine; the iterate is returned as it is, Ritz values NaN
    TRY(launch_copy(b.best, m, m, n, (double2*)V, m, st));
    for (int j = 0; j < m; ++j) lambda_out[j] = std::numeric_limits<double>::quiet_NaN();
    const int rows = std::min(it + 1, hist_rows);
    if (resid_history) std::memcpy(resid_history, hist.data(), (size_t)rows * m * sizeof(double));
    info->iterations = rows;
    info->best_iteration = have_best ? best_iter : -1;
    info->status = status;
    info->explicit_gram = explicit_gram;
    info->best_mean_residual = smallest;
    info->hx_applications = s.applies * (prm->folded ? 2 : 1);
    info->hx_launches = s.hx_launches;
    info->hx_bytes = s.hx_bytes;
    QDKP_CUDA_TRY(cudaStreamSynchronize(st));
    info->hx_seconds = prm->time_hx ? s.hx_seconds() : 0.0;
    info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    return QDKP_OK;
  }
  // ---- final Rayleigh-Ritz on the best iterate (scipy lobpcg.py:1009-1060) -----------------
  TRY(s.applyA(b.best, m, b.AX));
  TRY(s.gram(blist({{b.best, m}}, m), blist({{b.AX, m}}, m), b.gT));
  TRY(s.gram(blist({{b.best, m}}, m), blist({{b.best, m}}, m), b.gS));
  {
    std::vector<double2> t((size_t)m * m), s2((size_t)m * m), a((size_t)m * m), bb((size_t)m * m);
    TRY(s.sync_read(t.data(), b.gT, t.size() * sizeof(double2)));
    TRY(s.sync_read(s2.data(), b.gS, s2.size() * sizeof(double2)));
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        const double2 x = t[(size_t)i * m + j], y = t[(size_t)j * m + i];
        a[(size_t)i * m + j] = make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
        const double2 u = s2[(size_t)i * m + j], v = s2[(size_t)j * m + i];
        bb[(size_t)i * m + j] = make_double2(0.5 * (u.x + v.x), 0.5 * (u.y - v.y));
      }
    TRY(s.put(b.gA, a.data(), a.size() * sizeof(double2)));
    TRY(s.put(b.gB, bb.data(), bb.size() * sizeof(double2)));
  }
  TRY(launch_eigh(b.gA, b.gB, m, b.w, b.E, b.scr, b.status, st));
  TRY(s.sync_read(hstat, b.status, sizeof(int)));
  if (hstat[0]) { set_error("eigh has failed in lobpcg postprocessing"); return QDKP_ERR_NUMERIC; }
  TRY(s.sync_read(lam.data(), b.w, m * sizeof(double)));
  {
    const double2* C[1] = {b.E};
    TRY(launch_update(blist({{b.best, m}}, m), C, m, n, (double2*)V, m, 0, st));
    TRY(launch_update(blist({{b.AX, m}}, m), C, m, n, b.AX, m, 0, st));
  }
  TRY(s.put(b.lam, lam.data(), m * sizeof(double)));
  TRY(launch_colnorm2(b.AX, m, (const double2*)V, m, b.lam, m, n, b.npart, kNormParts, b.norms, st));
  TRY(s.sync_read(rn2.data(), b.norms, m * sizeof(double)));
  for (int j = 0; j < m; ++j) norms[j] = std::sqrt(std::fabs(rn2[j]));
  if (best_iter + 1 < hist_rows)
    std::memcpy(&hist[(size_t)(best_iter + 1) * m], norms.data(), m * sizeof(double));
  std::memcpy(lambda_out, lam.data(), m * sizeof(double));
  const int rows = std::min(best_iter + 2, hist_rows);
  if (resid_history) std::memcpy(resid_history, hist.data(), (size_t)rows * m * sizeof(double));
  if (status == QDKP_LOBPCG_MAXITER) {
    bool all = true;
    for (int j = 0; j < m; ++j) all = all && norms[j] <= tol;
    if (all) status = QDKP_LOBPCG_CONVERGED;
  }
  info->iterations = rows;
  info->best_iteration = best_iter;
  info->status = status;
  info->explicit_gram = explicit_gram;
  info->best_mean_residual = smallest;
  info->hx_applications = s.applies * (prm->folded ? 2 : 1);
  info->hx_launches = s.hx_launches;
  info->hx_bytes = s.hx_bytes;
  QDKP_CUDA_TRY(cudaStreamSynchronize(st));
  info->hx_seconds = prm->time_hx ? s.hx_seconds() : 0.0;
  info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
#undef TRY
  return QDKP_OK;
}

size_t qdkp_residuals_workspace_size(const qdkp_operator* op, int k) {
  if (!op || k < 1 || k > kMaxBlock) return 0;
  const size_t blk = ((size_t)op->n_bands * op->n_sites * k * sizeof(double2) + 255) / 256 * 256;
  return blk + (size_t)kNormParts * k * sizeof(double) + 4096 + gram_partial_elems(k, k) * sizeof(double2)
         + (size_t)k * k * sizeof(double2) * 2 + 4096;
}

int qdkp_residuals(const qdkp_operator* op, const void* V, int64_t ldv, int k, const double* E_in,
                   double* rq, double* res, void* ws, size_t ws_bytes, void* stream) {
  QDKP_CHECK_ARG(op && V && rq && res, "NULL argument");
  QDKP_CHECK_ARG(k >= 1 && k <= kMaxBlock && ldv >= k, "k must be in [1, 24] and ldv >= k");
  const size_t need = qdkp_residuals_workspace_size(op, k);
  if (!ws || ws_bytes < need) { set_error("qdkp_residuals: workspace too small"); return QDKP_ERR_WORKSPACE; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t n = (int64_t)op->n_bands * op->n_sites;
  char* p = static_cast<char*>(ws);
  const size_t blk = ((size_t)n * k * sizeof(double2) + 255) / 256 * 256;
  double2* HV = (double2*)p; p += blk;
  double* part = (double*)p; p += ((size_t)kNormParts * k * sizeof(double) + 255) / 256 * 256;
  double* out = (double*)p; p += 2048;
  double* lam = (double*)p; p += 2048;
  double2* gpart = (double2*)p; p += gram_partial_elems(k, k) * sizeof(double2);
  double2* g1 = (double2*)p; p += (size_t)k * k * sizeof(double2);
  double2* g2 = (double2*)p;
  int rc = launch_apply(op, V, ldv, HV, k, k, 0.0, 0, QDKP_C128, st);
  if (rc) return rc;
  // Rayleigh quotients: diag(V^H H V) / diag(V^H V)
  BlockList<double> Lv = blist({{(const double2*)V, k}}, ldv);
  BlockList<double> Lh = blist({{HV, k}}, k);
  rc = launch_gram(Lv, Lh, n, gpart, gram_partial_elems(k, k), g1, st); if (rc) return rc;
  rc = launch_gram(Lv, Lv, n, gpart, gram_partial_elems(k, k), g2, st); if (rc) return rc;
  std::vector<double2> a((size_t)k * k), bb((size_t)k * k);
  QDKP_CUDA_TRY(cudaMemcpyAsync(a.data(), g1, a.size() * sizeof(double2), cudaMemcpyDeviceToHost, st));
  QDKP_CUDA_TRY(cudaMemcpyAsync(bb.data(), g2, bb.size() * sizeof(double2), cudaMemcpyDeviceToHost, st));
  QDKP_CUDA_TRY(cudaStreamSynchronize(st));
  std::vector<double> E(k), nrm(k);
  for (int j = 0; j < k; ++j) {
    rq[j] = a[(size_t)j * k + j].x / bb[(size_t)j * k + j].x;
    nrm[j] = std::sqrt(bb[(size_t)j * k + j].x);
    E[j] = E_in ? E_in[j] : rq[j];
  }
  QDKP_CUDA_TRY(cudaMemcpyAsync(lam, E.data(), k * sizeof(double), cudaMemcpyHostToDevice, st));
  rc = launch_colnorm2(HV, k, (const double2*)V, ldv, lam, k, n, part, kNormParts, out, st);
  if (rc) return rc;
  std::vector<double> r2(k);
  QDKP_CUDA_TRY(cudaMemcpyAsync(r2.data(), out, k * sizeof(double), cudaMemcpyDeviceToHost, st));
  QDKP_CUDA_TRY(cudaStreamSynchronize(st));
  for (int j = 0; j < k; ++j) res[j] = std::sqrt(std::fabs(r2[j])) / nrm[j];
  return QDKP_OK;
}

}  // extern "C"
