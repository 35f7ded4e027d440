// Device side of the batched LOBPCG engine: per-slot state, descriptors and the multi-slot
// kernels. One tick advances every running slot by one iteration of scipy's LOBPCG
// (lobpcg.py:688-973); the decisions scipy takes on host scalars are taken here by one-CTA
// kernels per slot, so a tick is a fixed sequence of launches with no host round trip.
#pragma once
#include "dense_dev.cuh"

namespace qdkp {

// Per-slot mutable state (device memory, written by the decision kernels).
constexpr int kEGramSplit = 16;      // groups of Gram partials summed by their last CTA

struct EState {
  int running;          // 1 while the slot iterates
  int status;           // QDKP_LOBPCG_* once it stopped
  int iter;             // scipy's iterationNumber of the current tick (starts at -1)
  int idle;             // 1: the remaining kernels of this tick skip the slot
  int ma;               // active residual columns this tick
  int mp;               // P columns in this tick's Rayleigh-Ritz (0: restart)
  int restart, forced, explicit_gram;
  int best_iter;
  int copy_best;        // X of this tick is the new best iterate
  int skip_recompute;   // 0: forced restart recomputes A X this tick
  int skip_p;           // 1: no P block this tick (iteration 0 or idle)
  int skip_pnorm;       // 1: P orthonormalisation is not applied
  double smallest;
  int active[kMaxBlock];
  int idx[kMaxBlock];
  double lam[kMaxBlock];
  double norms[kMaxBlock];
  // CTAs of the current Gram product done, per partial group; the last slot counts the groups
  // reduced. The CTA that completes a count resets it to 0.
  int gram_done[kEGramSplit + 1];
};

// Per-slot constant descriptor (built on the host at admission, device resident).
// The tall blocks (X ... T) hold complex128 or, for a complex64 slot (prec = QDKP_C64), complex64
// values; they are declared double2 and reinterpreted through blk<T>(). Everything small (Gram
// matrices, Ritz coefficients, residual norms) is FP64 in both cases.
struct ESlot {
  long long n;          // rows (8 N)
  int m;                // block width
  int prec;             // QDKP_C128 or QDKP_C64: arithmetic of the tall blocks and of H.X
  double sqrt_eps;      // sqrt(machine epsilon) of that arithmetic (explicit Gram switch)
  int folded;
  double tol;
  int maxiter;
  int stall_iterations;  // > 0: stop once the best mean residual is this many iterations old
  int restart_control;
  double2 *X, *AX, *P, *AP, *best, *Ra, *ARa, *Pa, *APa, *T;
  double2 *W, *G, *U, *gS, *gT, *gA, *gB, *E, *scr, *Cx, *Cr, *Cp, *Im;
  double* w;
  double* npart;        // [nparts][m] residual-norm partials
  double* gpart;        // Gram partials (real), then the split sums
  int nparts;           // CTAs of the norm kernel
  int gparts;           // CTAs of the Gram kernel
  long long rows_per_gpart;
  int norm0, gram0, row0;   // first CTA of this slot in the norm / Gram / row-kernel launches
  int utile0;           // complex64 slots: first 128-row tile in the group's tcgen05 update space
  int rows_per_cta;     // rows per CTA in the row kernels (gather, update)
  EState* st;
};

template <typename T>
__device__ __forceinline__ cplx<T>* blk(double2* p) { return reinterpret_cast<cplx<T>*>(p); }

__device__ __forceinline__ int slot_of(const ESlot* __restrict__ S, int ns, int b,
                                       int ESlot::*first) {
  int k = 0;
  while (k + 1 < ns && b >= S[k + 1].*first) ++k;
  return k;
}

}  // namespace qdkp
