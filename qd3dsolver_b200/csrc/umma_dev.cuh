// Complex64 block updates on the fifth-generation tensor cores (sm_100a): tcgen05.mma kind::tf32
// with the accumulators in tensor memory (TMEM), fed by bulk asynchronous copies.
//
// Y (+)= sg [A_0 | A_1 | A_2] [C_0; C_1; C_2] in the real form Y' = A' C'' (A' the rows of the
// complex64 blocks read as floats, C'' the 2x2 real blocks [[Re, Im], [-Im, Re]] of the complex
// coefficients), every FP32 value split into two TF32 parts, x = hi + lo (hi = x rounded to TF32,
// lo = the rest rounded to TF32), and the product formed as hi*hi + hi*lo + lo*hi with FP32
// accumulation: FP32 accuracy from TF32 tensor cores.
//
// Work unit: a "chunk" = one block of one 128-row tile. A CTA of 13 warps runs its tiles as a
// warp-specialised pipeline; the roles meet only on mbarriers, so each runs ahead of the next as
// far as its ring allows:
//  * producer / MMA warp (one lane): copies each chunk's rows (128 x ld complex64, contiguous in
//    global memory) into one of S raw stages with cp.async.bulk, S chunks ahead, completion counted
//    on the stage's mbarrier; when a chunk has been converted, issues its MMAs into one of two
//    TMEM accumulators (M = 128, K = 8 per instruction; per K step Ahi [Bhi | Blo] with N = 2 Nr
//    and Alo Bhi with N = Nr into the first Nr columns, Nr = outputs x 2q padded to 16, so that
//    the accumulator holds Ahi Bhi + Alo Bhi beside Ahi Blo) and commits them to the operand
//    buffer's "empty" mbarrier and, after a tile's last block, to the accumulator's "full" one;
//  * eight converter warps: split the raw chunk into TF32 hi / lo parts and store them in one of
//    two operand buffers in the no-swizzle K-major layout the MMA reads (8-row x 16-byte core
//    matrices: element (row, k) at float offset ((k / 4) (R / 8) + row / 8) 32 + (row % 8) 4 + k % 4
//    for R rows; leading-byte offset between the two 16-byte halves of an MMA-K step (R / 8) 128,
//    stride-byte offset between 8-row groups 128);
//  * four epilogue warps: read a finished accumulator (tcgen05.ld 32x32b; warp w reads lane
//    quarter w % 4), add its two halves and write the tile's output rows.
// The coefficients are staged once per run as B = [Bhi; Blo], Bhi / Blo the TF32 parts of C''^T
// (all outputs stacked along N, all blocks along K).
#pragma once
#include <cstdint>

#include "blockops.cuh"

namespace qdkp {

constexpr int kUmmaRows = 128;          // MMA M: rows of a tile
constexpr int kUmmaConvWarps = 8;      // converter warps (0-7)
constexpr int kUmmaEpiWarps = 4;       // epilogue warps (8-11): one per TMEM lane quarter
constexpr int kUmmaMmaWarp = kUmmaConvWarps + kUmmaEpiWarps;   // producer / MMA warp (12)
constexpr int kUmmaRowGroups = kUmmaRows / 8 / kUmmaConvWarps;  // 8-row groups per converter warp
constexpr int kUmmaThreads = 32 * (kUmmaMmaWarp + 1);
constexpr int kUmmaMaxStages = 8;       // raw chunk stages
constexpr int kUmmaSmemLimit = 224 * 1024;
// Complex64 block updates default to the split-TF32 mma.sync kernel, which measured faster on
// the Fig-4 sweep's engine ticks (0.77 against 0.88 ms per complex64 tick of the b = 10 nm
// valence solve); QDKP_C64_UPDATE=tcgen05 selects this pipeline.
constexpr bool kC64UpdateTcgen05Default = false;

__device__ __forceinline__ uint32_t umma_saddr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// x rounded to TF32 (10 explicit mantissa bits), to nearest with ties away from zero: the bits of
// an IEEE float order its magnitudes, so adding half of the dropped unit and clearing the 13
// dropped bits rounds the magnitude (integer ops at full rate; infinities and NaNs stay so)
__device__ __forceinline__ uint32_t umma_tf32(float x) {
  return (__float_as_uint(x) + 0x1000u) & 0xFFFFE000u;
}
// shared-memory matrix descriptor, no swizzle: start, leading and stride byte offsets (16-byte
// units), descriptor version 1 at bit 46
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}
// instruction descriptor: D f32 (bits 4-5 = 1), A and B tf32 (bits 7-9, 10-12 = 2), both
// K-major, N / 8 at bit 17, M / 16 at bit 24 (M = 128)
__host__ __device__ constexpr uint32_t umma_idesc_tf32(int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void umma_mma(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :: "r"(dtmem), "l"(ad), "l"(bd), "r"(idesc), "r"(accumulate),
         "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(mbar) : "memory");
}
// try_wait with a suspend-time hint (10 ms): a thread whose phase has not completed is suspended
// until it completes or the hint runs out, instead of spinning on the issue slots its warp's
// neighbours need
__device__ __forceinline__ bool umma_try(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n\t.reg .pred q;\n\t"
               "mbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2, %3;\n\t"
               "selp.u32 %0, 1, 0, q;\n\t}\n"
               : "=r"(ok) : "r"(mbar), "r"(parity), "r"(10000000u) : "memory");
  return ok != 0;
}
// Bounded wait on the completion of the phase of the given parity: false after ~1 s of clocks.
__device__ __forceinline__ bool umma_wait(uint32_t mbar, uint32_t parity) {
  if (umma_try(mbar, parity)) return true;
  const long long t0 = clock64();
  while (!umma_try(mbar, parity))
    if (clock64() - t0 > 2000000000LL) return false;
  return true;
}
__device__ __forceinline__ void umma_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(mbar), "r"(bytes)
               : "memory");
}
// bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from global memory into
// this CTA's shared memory, completion counted on mbar
__device__ __forceinline__ void umma_bulk_load(uint32_t dst, const void* src, uint32_t bytes,
                                               uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      :: "r"(dst), "l"(src), "r"(bytes), "r"(mbar) : "memory");
}
// bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from this CTA's shared
// memory to global memory, in the issuing thread's current bulk async-group
__device__ __forceinline__ void umma_bulk_store(void* dst, uint32_t src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
               :: "l"(dst), "r"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void umma_bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// the issuing thread's bulk stores have read their shared memory, all but the newest `keep` groups
__device__ __forceinline__ void umma_bulk_wait_read(int keep) {
  if (keep) asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
  else asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void umma_bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
// barrier 1 among the epilogue warps only
__device__ __forceinline__ void umma_epi_sync() {
  asm volatile("bar.sync 1, %0;" :: "r"(32 * kUmmaEpiWarps) : "memory");
}
// barrier 1 among the epilogue warps, returning whether v held for any of them (a decision all
// of them take alike)
__device__ __forceinline__ bool umma_epi_any(bool v) {
  uint32_t r;
  asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\t"
               "bar.red.or.pred p, 1, %2, q;\n\tselp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(r) : "r"((uint32_t)v), "r"(32 * kUmmaEpiWarps) : "memory");
  return r != 0;
}
__device__ __forceinline__ void umma_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__host__ __device__ __forceinline__ int umma_off(int row, int k, int R) {
  return ((k >> 2) * (R >> 3) + (row >> 3)) * 32 + (row & 7) * 4 + (k & 3);
}
__host__ __device__ __forceinline__ int umma_N(int q) { return ((2 * q + 15) / 16) * 16; }
// K (floats) of a block of `cols` complex columns: 2 cols padded to the MMA's K step of 8
__host__ __device__ __forceinline__ int umma_Kb(int cols) { return ((cols + 3) / 4) * 8; }

// Shared-memory plan of a run, a function of the launch's bounds only (P columns in all, q output
// columns, nout outputs, blocks at most cmax columns wide; raw stages hold rows of up to ldmax
// complex values, blocks with a larger leading dimension are read directly), so that the host
// sizes and the device lays out the same bytes.
struct UmmaPlan {
  int nout_pass;      // outputs formed per pass over A (1 or 2)
  int N;              // accumulator columns per output
  int Ntot;           // nout_pass N
  int Kcap;           // K capacity of B (floats): every split of P columns over three blocks fits
  int KbMax;          // K of one operand buffer (floats)
  int nbuf;           // operand buffers (2: the MMA of chunk i overlaps the conversion of i + 1)
  int nob;            // output staging buffers (0: the epilogue writes rows directly)
  int S;              // raw stages
  int ldmax, q;
  unsigned ostage;    // bytes of one output staging buffer (all outputs of a tile)
  unsigned offA, offOut, offRaw, bytes;
};
__host__ __device__ inline UmmaPlan umma_plan(int P, int q, int nout, int cmax, int ldmax) {
  UmmaPlan p{};
  p.N = umma_N(q);
  p.Kcap = 8 * ((P + 3) / 4 + 2);
  p.KbMax = umma_Kb(cmax < P ? cmax : P);
  p.ldmax = ldmax;
  p.q = q;
  const unsigned raw = (unsigned)kUmmaRows * ldmax * 8u;
  const unsigned abuf = 2u * kUmmaRows * p.KbMax * 4u;
  // one pass over A first, then two operand buffers, then double-buffered output staging
  for (int np = nout; np >= 1; --np)
    for (int nb = 2; nb >= 1; --nb)
      for (int nob = 2; nob >= 0; --nob) {
        const unsigned b = 2u * np * p.N * p.Kcap * 4u;
        const unsigned ost = (unsigned)np * kUmmaRows * q * 8u;
        const unsigned fixed = b + nb * abuf + nob * ost;
        if (fixed + 2 * raw > (unsigned)kUmmaSmemLimit) continue;
        int S = (int)(((unsigned)kUmmaSmemLimit - fixed) / raw);
        if (S > kUmmaMaxStages) S = kUmmaMaxStages;
        p.nout_pass = np; p.Ntot = np * p.N; p.nbuf = nb; p.nob = nob; p.ostage = ost; p.S = S;
        p.offA = b; p.offOut = b + nb * abuf; p.offRaw = fixed; p.bytes = fixed + S * raw;
        return p;
      }
  p.nout_pass = 0;                 // does not fit (rejected by the launchers)
  return p;
}
// accumulator columns a CTA allocates: two accumulators of 2 Ntot columns, a power of two >= 32
__host__ __device__ __forceinline__ uint32_t umma_tmem_cols(const UmmaPlan& p) {
  uint32_t c = 32;
  while ((int)c < 4 * p.Ntot) c <<= 1;
  return c;
}

__device__ __forceinline__ void umma_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(mbar) : "memory");
}

// Per-CTA state carried across runs: the TMEM accumulators, the barriers and how many chunks
// and tiles earlier runs took (from which every role derives the phase of each wait).
// Barriers (8 bytes apart from bar0): full[s] (raw stage s landed), cfull[h] (operand buffer h
// converted), cempty[h] (its MMAs done), afull[a] (accumulator a final), aempty[a] (read out).
struct UmmaCtx {
  uint32_t tmem, ncols, bar0;
  long long chunks, tiles;
};
__device__ __forceinline__ uint32_t umma_bar_full(const UmmaCtx& c, int s) { return c.bar0 + 8u * s; }
__device__ __forceinline__ uint32_t umma_bar_cfull(const UmmaCtx& c, int h) { return c.bar0 + 8u * (kUmmaMaxStages + h); }
__device__ __forceinline__ uint32_t umma_bar_cempty(const UmmaCtx& c, int h) { return c.bar0 + 8u * (kUmmaMaxStages + 2 + h); }
__device__ __forceinline__ uint32_t umma_bar_afull(const UmmaCtx& c, int a) { return c.bar0 + 8u * (kUmmaMaxStages + 4 + a); }
__device__ __forceinline__ uint32_t umma_bar_aempty(const UmmaCtx& c, int a) { return c.bar0 + 8u * (kUmmaMaxStages + 6 + a); }

// Allocates the accumulators and initialises the barriers; called by every thread of the CTA.
static __device__ void umma_ctx_init(UmmaCtx& cx, const UmmaPlan& pl) {
  __shared__ __align__(8) uint64_t bars[kUmmaMaxStages + 8];
  __shared__ uint32_t tmem_base;
  cx.ncols = umma_tmem_cols(pl);
  if ((threadIdx.x >> 5) == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(umma_saddr(&tmem_base)), "r"(cx.ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  cx.bar0 = umma_saddr(&bars[0]);
  if (threadIdx.x == 0) {
    auto init = [](uint32_t bar, uint32_t count) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count) : "memory");
    };
    for (int s = 0; s < kUmmaMaxStages; ++s) init(umma_bar_full(cx, s), 1);
    for (int h = 0; h < 2; ++h) {
      init(umma_bar_cfull(cx, h), kUmmaConvWarps);
      init(umma_bar_cempty(cx, h), 1);
      init(umma_bar_afull(cx, h), 1);
      init(umma_bar_aempty(cx, h), kUmmaEpiWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  cx.tmem = tmem_base;
  cx.chunks = 0;
  cx.tiles = 0;
}

// Frees the accumulators; every tcgen05 operation of the CTA has completed (a run ends only
// after its epilogue has read its last accumulator).
static __device__ void umma_ctx_free(const UmmaCtx& cx) {
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if ((threadIdx.x >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(cx.tmem), "r"(cx.ncols));
}

// v in rows [r0, r1) of the outputs
static __device__ void umma_fill(float2* const* Ys, int nout, int q, long long r0, long long r1,
                                 long long ldy, float v) {
  for (int o = 0; o < nout; ++o)
    for (long long e = threadIdx.x; e < (r1 - r0) * q; e += blockDim.x) {
      const long long r = r0 + e / q;
      Ys[o][r * ldy + e % q] = make_float2(v, v);
    }
}
static __device__ void umma_fill_nan(float2* const* Ys, int nout, int q, long long r0,
                                     long long r1, long long ldy) {
  umma_fill(Ys, nout, q, r0, r1, ldy, __int_as_float(0x7fc00000));
}

// One run: outputs o < nout of the coefficient lists Cs[o] into Ys[o] over rows [r0, r1)
// (accumulate: output 0 adds the product to its old value). nout <= pl.nout_pass. Called by
// every thread of a kUmmaThreads CTA; returns false if a wait gave up (the outputs then hold NaN).
static __device__ __noinline__ bool umma_run(const UmmaPlan& pl_in, UmmaCtx& cx_in,
                                             unsigned char* smem, const BlockList<float>& A,
                                             const double2* const* const* Cs,
                                             float2* const* Ys_in, int nout, int q, long long r0,
                                             long long r1, long long ldy, int accumulate, int neg) {
  __shared__ int s_fault;
  if (r0 >= r1) return true;
  // the plan, the context and the output pointers in registers for the run (the caller's
  // copies are in memory, which every fence and wait would make the run read again)
  const UmmaPlan pl = pl_in;
  const UmmaCtx cx = cx_in;
  float2* const Ys[2] = {Ys_in[0], nout == 2 ? Ys_in[1] : nullptr};
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // the blocks that have columns (a block of width 0 takes no chunk)
  const float2* bp[3] = {nullptr, nullptr, nullptr};
  long long bld[3] = {1, 1, 1};
  const double2* bc[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  int cols[3] = {0, 0, 0}, kb0[4] = {0, 0, 0, 0};
  bool blk_bulk[3] = {false, false, false};
  int nb = 0;
  for (int b = 0; b < A.nblk; ++b) {
    if (A.cols[b] <= 0) continue;
    bp[nb] = A.p[b]; bld[nb] = A.ld[b]; cols[nb] = A.cols[b];
    for (int o = 0; o < nout; ++o) bc[o][nb] = Cs[o][b];
    kb0[nb + 1] = kb0[nb] + umma_Kb(cols[nb]);
    blk_bulk[nb] = (reinterpret_cast<uintptr_t>(bp[nb]) & 15) == 0 && bld[nb] <= pl.ldmax;
    ++nb;
  }
  if (nb == 0) {                               // no columns: the product is zero
    if (!accumulate) umma_fill(Ys, nout, q, r0, r1, ldy, 0.f);
    else if (nout == 2) umma_fill(Ys + 1, 1, q, r0, r1, ldy, 0.f);
    __syncthreads();
    return true;
  }
  const int P = cols[0] + cols[1] + cols[2];
  const int N = pl.N, Nr = nout * N;          // accumulator columns of this run
  float* Bs = reinterpret_cast<float*>(smem);   // [Bhi; Blo]: 2 Nr rows x Kcap
  const int Ktot = kb0[nb];
  const float sg = neg ? -1.f : 1.f;
  // B = C''^T (Nr x Ktot): for the coefficient of A's column c (block b, local i) and output
  // column jj of output o, the 2 x 2 block [[Re, Im], [-Im, Re]] at rows o N + 2 jj (+1) and
  // K kb0[b] + 2 i (+1); zero where no coefficient enters (padding, NULL lists)
  for (int e = tid; e < nout * P * q; e += blockDim.x) {
    const int o = e / (P * q), r = e - o * P * q;
    const int c = r / q, jj = r - c * q;
    const int b = c < cols[0] ? 0 : (c < cols[0] + cols[1] ? 1 : 2);
    const int i = c - (b == 0 ? 0 : (b == 1 ? cols[0] : cols[0] + cols[1]));
    const double2* Cb = bc[o][b];
    float re = 0.f, im = 0.f;
    if (Cb) {
      const double2 cc = Cb[(size_t)i * q + jj];
      re = sg * (float)cc.x;
      im = sg * (float)cc.y;
    }
    const float v[4] = {re, -im, im, re};        // (j, k): (2jj, 2i) (2jj, 2i+1) (2jj+1, 2i) (2jj+1, 2i+1)
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int j = o * N + 2 * jj + (t >> 1), k = kb0[b] + 2 * i + (t & 1);
      const uint32_t hi = umma_tf32(v[t]);
      Bs[umma_off(j, k, 2 * Nr)] = __uint_as_float(hi);
      Bs[umma_off(Nr + j, k, 2 * Nr)] = __uint_as_float(umma_tf32(v[t] - __uint_as_float(hi)));
    }
  }
  for (int e = tid; e < Nr * Ktot; e += blockDim.x) {
    const int j = e / Ktot, k = e - j * Ktot;
    const int b = k < kb0[1] ? 0 : (k < kb0[2] ? 1 : 2);
    if (((j % N) >> 1) >= q || ((k - kb0[b]) >> 1) >= cols[b]) {
      Bs[umma_off(j, k, 2 * Nr)] = 0.f;
      Bs[umma_off(Nr + j, k, 2 * Nr)] = 0.f;
    }
  }
  if (tid == 0) s_fault = 0;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  volatile int* vfault = &s_fault;

  const long long T = (r1 - r0 + kUmmaRows - 1) / kUmmaRows;
  const long long nch = T * nb;
  const long long g0 = cx.chunks, tg0 = cx.tiles;
  const int S = pl.S, nbuf = pl.nbuf;
  const unsigned rawb = (unsigned)kUmmaRows * pl.ldmax * 8u;
  const unsigned abytes = 2u * kUmmaRows * pl.KbMax * 4u;
  unsigned char* raw0 = smem + pl.offRaw;
  auto tile_rows = [&](long long ti) { return (int)min((long long)kUmmaRows, r1 - r0 - ti * kUmmaRows); };
  auto bulk = [&](long long ti, int b) {
    return blk_bulk[b] && tile_rows(ti) == kUmmaRows && (((r0 + ti * kUmmaRows) * bld[b]) & 1) == 0;
  };

  if (warp < kUmmaConvWarps) {
    // ---------------- converters: raw chunk -> TF32 hi / lo operand buffer ----------------
    // stage / buffer indices and phase parities advance incrementally (no divisions per chunk)
    int s = (int)(g0 % S), h = (int)(g0 % nbuf);
    uint32_t fpar = (uint32_t)((g0 / S) & 1), hpar = (uint32_t)((g0 / nbuf) & 1);
    bool hused = g0 >= nbuf;                     // buffer h was filled by an earlier chunk
    // a thread's elements: rows (warp + W p) 8 + lane % 8 (W converter warps, p < 16 / W),
    // complex columns 4 kk + lane / 8
    const int lrow = lane & 7, lq = lane >> 3;
    int rowp[kUmmaRowGroups], offp[kUmmaRowGroups];
#pragma unroll
    for (int p = 0; p < kUmmaRowGroups; ++p) {
      rowp[p] = (warp + kUmmaConvWarps * p) * 8 + lrow;
      offp[p] = (((lq >> 1) * 16) + warp + kUmmaConvWarps * p) * 32 + lrow * 4 + (lq & 1) * 2;
    }
    long long ti = 0;
    int b = 0;
    for (long long i = 0; i < nch; ++i) {
      if (*vfault) break;
      bool ok = umma_wait(umma_bar_full(cx, s), fpar);
      if (hused) ok = umma_wait(umma_bar_cempty(cx, h), hpar ^ 1u) && ok;
      const bool bk = bulk(ti, b);
      float* Ah = reinterpret_cast<float*>(smem + pl.offA + (size_t)h * abytes);
      float* Al = Ah + kUmmaRows * pl.KbMax;
      const float2* rw = reinterpret_cast<const float2*>(raw0 + (size_t)s * rawb);
      const long long ldl = bld[b], t0 = r0 + ti * kUmmaRows;
      const int ld = (int)ldl, rows = tile_rows(ti), cb = cols[b], nq = (cb + 3) / 4;
      const float2* gp = bp[b];
      constexpr int kQuads = kMaxBlock / 4;
      float2 x[kUmmaRowGroups][kQuads];
      if (bk && (ld & 1) == 0) {
        // complex pairs: lane (8-row offset lane % 8, pair lane / 8) loads columns c, c + 1
        // (c = 8 kk + 2 (lane / 8)) of its rows as one 16-byte word and stores their four K
        // values as one 16-byte word each of hi and lo
        const int lp = lane >> 3, cmaxe = (cb - 1) & ~1, c4 = (cb + 3) / 4 * 4;
        constexpr int kPairs = (kMaxBlock + 7) / 8;
        float4 y[kUmmaRowGroups][kPairs];
#pragma unroll
        for (int kk = 0; kk < kPairs; ++kk) {
          const int c = 8 * kk + 2 * lp, cl = min(c, cmaxe);
#pragma unroll
          for (int p = 0; p < kUmmaRowGroups; ++p) {
            float4 v = reinterpret_cast<const float4*>(rw)[(rowp[p] * ld + cl) >> 1];
            if (c >= cb) { v.x = 0.f; v.y = 0.f; }
            if (c + 1 >= cb) { v.z = 0.f; v.w = 0.f; }
            y[p][kk] = v;
          }
        }
#pragma unroll
        for (int kk = 0; kk < kPairs; ++kk) {
          const int c = 8 * kk + 2 * lp;
#pragma unroll
          for (int p = 0; p < kUmmaRowGroups; ++p)
            if (c < c4) {
              const float4 v = y[p][kk];
              const int off = ((4 * kk + lp) * 16 + warp + kUmmaConvWarps * p) * 32 + lrow * 4;
              float4 hi, lo;
              hi.x = __uint_as_float(umma_tf32(v.x)); lo.x = __uint_as_float(umma_tf32(v.x - hi.x));
              hi.y = __uint_as_float(umma_tf32(v.y)); lo.y = __uint_as_float(umma_tf32(v.y - hi.y));
              hi.z = __uint_as_float(umma_tf32(v.z)); lo.z = __uint_as_float(umma_tf32(v.z - hi.z));
              hi.w = __uint_as_float(umma_tf32(v.w)); lo.w = __uint_as_float(umma_tf32(v.w - hi.w));
              *reinterpret_cast<float4*>(Ah + off) = hi;
              *reinterpret_cast<float4*>(Al + off) = lo;
            }
        }
      } else {
      if (bk) {
        // straight-line shared loads (an in-range index everywhere, zero selected past the
        // block's columns), so that all of a thread's loads are in flight together
#pragma unroll
        for (int kk = 0; kk < kQuads; ++kk) {
          const int c = 4 * kk + lq, cc = min(c, cb - 1);
#pragma unroll
          for (int p = 0; p < kUmmaRowGroups; ++p) {
            const float2 v = kk < nq ? rw[rowp[p] * ld + cc] : make_float2(0.f, 0.f);
            x[p][kk] = c < cb ? v : make_float2(0.f, 0.f);
          }
        }
      } else {
#pragma unroll
        for (int kk = 0; kk < kQuads; ++kk)
#pragma unroll
          for (int p = 0; p < kUmmaRowGroups; ++p) {
            const int c = 4 * kk + lq;
            x[p][kk] = make_float2(0.f, 0.f);
            if (kk < nq && c < cb && rowp[p] < rows) x[p][kk] = gp[(t0 + rowp[p]) * ldl + c];
          }
      }
#pragma unroll
      for (int kk = 0; kk < kQuads; ++kk) {
        if (kk >= nq) break;
#pragma unroll
        for (int p = 0; p < kUmmaRowGroups; ++p) {
          const float2 v = x[p][kk];
          const uint32_t hx = umma_tf32(v.x), hy = umma_tf32(v.y);
          const int off = offp[p] + kk * 1024;
          *reinterpret_cast<float2*>(Ah + off) = make_float2(__uint_as_float(hx), __uint_as_float(hy));
          *reinterpret_cast<float2*>(Al + off) =
              make_float2(__uint_as_float(umma_tf32(v.x - __uint_as_float(hx))),
                          __uint_as_float(umma_tf32(v.y - __uint_as_float(hy))));
        }
      }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) umma_arrive(umma_bar_cfull(cx, h));
      if (!ok) *vfault = 1;
      if (++b == nb) { b = 0; ++ti; }
      if (++s == S) { s = 0; fpar ^= 1u; }
      if (++h == nbuf) { h = 0; hpar ^= 1u; hused = true; }
    }
  } else if (warp < kUmmaMmaWarp) {
    // ---------------- epilogue: accumulator -> output rows ----------------
    // With staging (pl.nob > 0) a tile's rows go to a shared-memory image of the output rows first
    // and from there to global memory: one bulk store per output for a full tile of contiguous
    // rows (ldy == q), otherwise a coalesced copy by the epilogue warps.
    constexpr int kParts = kUmmaEpiWarps / 4;    // warps per lane quarter, each a column part
    const int e = warp - kUmmaConvWarps, quarter = warp & 3, part = e / 4;
    const int et = tid - 32 * kUmmaConvWarps;   // 0 .. 32 kUmmaEpiWarps - 1
    const int ng = Nr / 8, gh = ng / kParts, gfirst = part * gh;   // this part's 8-column groups
    const bool stage = pl.nob > 0;
    uintptr_t al = 0;
    for (int o = 0; o < nout; ++o) al |= reinterpret_cast<uintptr_t>(Ys[o]);
    const bool vec = (ldy & 1) == 0 && (al & 15) == 0;
    const bool bulk_out = stage && ldy == q && (q & 1) == 0 && (al & 15) == 0;
    const bool svec = (q & 1) == 0;              // 16-byte staging writes
    int ob = 0, pending = 0;                     // staging buffer; bulk groups not yet read
    for (long long ti = 0; ti < T; ++ti) {
      // with staging the epilogue warps meet on barrier 1, so they stop together
      if (stage ? umma_epi_any(*vfault != 0) : (*vfault != 0)) break;
      const long long tg = tg0 + ti;
      const int a = (int)(tg & 1);
      const bool ok = umma_wait(umma_bar_afull(cx, a), (uint32_t)((tg >> 1) & 1));
      __syncwarp();                              // converged for the aligned TMEM loads
      asm volatile("tcgen05.fence::after_thread_sync;");
      const int rows = tile_rows(ti), rl = quarter * 32 + lane;
      const long long r = r0 + ti * kUmmaRows + rl;
      float2* sb = reinterpret_cast<float2*>(smem + pl.offOut + (size_t)ob * pl.ostage);
      if (stage) {                               // the buffer's last bulk store has read it
        if (et == 0 && pending >= pl.nob) { umma_bulk_wait_read(pl.nob - 1); --pending; }
        umma_epi_sync();
      }
      const uint32_t tb = cx.tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(a * 2 * pl.Ntot);
      for (int u0 = 0; u0 < gh; u0 += 2) {       // two groups at a time
        float v[2][8], w[2][8];
#pragma unroll
        for (int du = 0; du < 2; ++du)
          if (u0 + du < gh) {
            umma_ld8(tb + (uint32_t)(8 * (gfirst + u0 + du)), v[du]);
            umma_ld8(tb + (uint32_t)(Nr + 8 * (gfirst + u0 + du)), w[du]);
          }
        float2 old[2][4];
#pragma unroll
        for (int du = 0; du < 2; ++du) {
          const int col0 = 8 * (gfirst + u0 + du), jj0 = (col0 % N) / 2;
#pragma unroll
          for (int x = 0; x < 4; ++x)
            old[du][x] = (accumulate && u0 + du < gh && col0 < N && jj0 + x < q && rl < rows)
                             ? Ys[0][r * ldy + jj0 + x] : make_float2(0.f, 0.f);
        }
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int du = 0; du < 2; ++du) {
          if (u0 + du >= gh || rl >= rows) continue;
          const int col0 = 8 * (gfirst + u0 + du), o = col0 / N, jj0 = (col0 - o * N) / 2;
          float2 y[4];
#pragma unroll
          for (int x = 0; x < 4; ++x) {
            y[x] = make_float2(v[du][2 * x] + w[du][2 * x], v[du][2 * x + 1] + w[du][2 * x + 1]);
            if (o == 0) { y[x].x += old[du][x].x; y[x].y += old[du][x].y; }
          }
          float2* dst = stage ? sb + ((size_t)o * kUmmaRows + rl) * q + jj0 : Ys[o] + r * ldy + jj0;
          if ((stage ? svec : vec) && jj0 + 4 <= q) {
            reinterpret_cast<float4*>(dst)[0] = make_float4(y[0].x, y[0].y, y[1].x, y[1].y);
            reinterpret_cast<float4*>(dst)[1] = make_float4(y[2].x, y[2].y, y[3].x, y[3].y);
          } else {
#pragma unroll
            for (int x = 0; x < 4; ++x)
              if (jj0 + x < q) dst[x] = y[x];
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) umma_arrive(umma_bar_aempty(cx, a));   // the accumulator is free again
      if (stage) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        umma_epi_sync();
        const long long row0 = r0 + ti * kUmmaRows;
        if (bulk_out && rows == kUmmaRows) {
          if (et == 0) {
            for (int o = 0; o < nout; ++o)
              umma_bulk_store(Ys[o] + row0 * q, umma_saddr(sb + (size_t)o * kUmmaRows * q),
                              (uint32_t)(kUmmaRows * q * 8));
            umma_bulk_commit();
            ++pending;
          }
        } else {
          for (int o = 0; o < nout; ++o)
            for (int k = et; k < rows * q; k += 32 * kUmmaEpiWarps)
              Ys[o][(row0 + k / q) * ldy + k % q] = sb[(size_t)o * kUmmaRows * q + k];
          umma_epi_sync();                       // read before the buffer is written again
        }
        if (pl.nob == 2) ob ^= 1;
      }
      if (!ok) *vfault = 1;
    }
    if (et == 0 && pending) umma_bulk_wait_all();   // the output rows are written
  } else if (lane == 0) {
    // ---------------- producer / MMA issue (one thread) ----------------
    const uint32_t idesc2 = umma_idesc_tf32(2 * Nr), idesc1 = umma_idesc_tf32(Nr);
    const uint32_t lboA = (kUmmaRows / 8) * 128, lboB = (uint32_t)(2 * Nr / 8) * 128;
    const uint64_t dB = umma_desc(umma_saddr(Bs), lboB, 128);
    uint64_t dAh[2], dAl[2];
    for (int h = 0; h < 2; ++h) {
      const uint32_t aH = umma_saddr(smem + pl.offA + (size_t)h * abytes);
      dAh[h] = umma_desc(aH, lboA, 128);
      dAl[h] = umma_desc(aH + (uint32_t)(kUmmaRows * pl.KbMax * 4), lboA, 128);
    }
    // chunk `issued`'s rows into its raw stage (a plain arrival for a chunk the converters read
    // directly); the producer's stage, tile and block advance incrementally
    int ps = (int)(g0 % S), pb = 0;
    long long pti = 0, issued = 0;               // chunks < issued have been produced
    auto produce = [&]() {
      const uint32_t bar = umma_bar_full(cx, ps);
      if (bulk(pti, pb)) {
        const uint32_t bytes = (uint32_t)(kUmmaRows * bld[pb] * 8);
        umma_expect_tx(bar, bytes);
        umma_bulk_load(umma_saddr(raw0 + (size_t)ps * rawb),
                       bp[pb] + (r0 + pti * kUmmaRows) * bld[pb], bytes, bar);
      } else {
        umma_arrive(bar);
      }
      ++issued;
      if (++pb == nb) { pb = 0; ++pti; }
      if (++ps == S) ps = 0;
    };
    while (issued < nch && issued < S) produce();
    long long ti = 0, done = 0;
    int b = 0, h = (int)(g0 % nbuf);
    uint32_t hpar = (uint32_t)((g0 / nbuf) & 1);
    bool ok = true;
    for (long long i = 0; i < nch; ++i) {
      if (*vfault) { ok = false; break; }
      const long long tg = tg0 + ti;
      const int a = (int)(tg & 1);
      ok = umma_wait(umma_bar_cfull(cx, h), hpar);
      if (ok && b == 0 && tg >= 2) ok = umma_wait(umma_bar_aempty(cx, a), (uint32_t)(((tg >> 1) & 1) ^ 1));
      if (!ok) break;
      done = i + 1;                              // chunk i has been converted (its stage is free)
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t d = cx.tmem + (uint32_t)(a * 2 * pl.Ntot);
      const int steps = umma_Kb(cols[b]) / 8;
      const uint64_t ah = dAh[h], al = dAl[h];
      uint64_t bd = dB + (uint64_t)((kb0[b] / 4) * lboB >> 4);
      uint64_t oa = 0;
      const uint64_t sa = (2 * lboA) >> 4, sb = (2 * lboB) >> 4;
      for (int st = 0; st < steps; ++st) {
        umma_mma(d, ah + oa, bd, idesc2, (b > 0 || st > 0) ? 1u : 0u);   // Ahi [Bhi | Blo]
        umma_mma(d, al + oa, bd, idesc1, 1u);                             // + Alo Bhi
        oa += sa; bd += sb;
      }
      umma_commit(umma_bar_cempty(cx, h));
      if (b == nb - 1) umma_commit(umma_bar_afull(cx, a));
      if (issued < nch) produce();
      if (++b == nb) { b = 0; ++ti; }
      if (++h == nbuf) { h = 0; hpar ^= 1u; }
    }
    if (!ok) {
      *vfault = 1;
      // copies still in flight land before the shared memory is reused or released; the MMAs
      // issued complete (bounded waits either way)
      for (long long j = done; j < issued; ++j) {
        const long long g = g0 + j;
        umma_wait(umma_bar_full(cx, (int)(g % S)), (uint32_t)((g / S) & 1));
      }
      if (done > 0) {
        const long long g = g0 + done - 1;
        umma_wait(umma_bar_cempty(cx, (int)(g % nbuf)), (uint32_t)((g / nbuf) & 1));
      }
    }
  }
  __syncthreads();
  const bool fault = *vfault != 0;
  if (fault) {
    __syncthreads();
    umma_fill_nan(Ys, nout, q, r0, r1, ldy);
  }
  cx_in.chunks = g0 + nch;
  cx_in.tiles = tg0 + T;
  __syncthreads();
  return !fault;
}

// Y (+)= sg A C over rows [r0, r1) and, with C2 / Y2, Y2 = sg A C2 (C[b] the cols_b x q row-major
// complex coefficients of A's block b, NULL: the block does not enter; accumulate applies to Y).
// Both outputs in one pass over A when the plan allows, then either may alias an input block;
// otherwise Y is formed first and Y2 second, each in its own pass, so Y must not alias an input
// (Y2 may). Called by every thread of a kUmmaThreads CTA whose context was set up for `pl`;
// returns false if a wait gave up (the outputs then hold NaN).
static __device__ bool update_rows_umma(const UmmaPlan& pl, UmmaCtx& cx, const BlockList<float>& A,
                                        const double2* const* C, int q, long long r0, long long r1,
                                        float2* Y, long long ldy, int accumulate, int neg,
                                        unsigned char* smem, const double2* const* C2 = nullptr,
                                        float2* Y2 = nullptr) {
  if (Y2 && pl.nout_pass == 2) {
    const double2* const* Cs[2] = {C, C2};
    float2* const Ys[2] = {Y, Y2};
    return umma_run(pl, cx, smem, A, Cs, Ys, 2, q, r0, r1, ldy, accumulate, neg);
  }
  const double2* const* Cs1[1] = {C};
  float2* const Ys1[1] = {Y};
  bool ok = umma_run(pl, cx, smem, A, Cs1, Ys1, 1, q, r0, r1, ldy, accumulate, neg);
  if (Y2) {
    const double2* const* Cs2[1] = {C2};
    float2* const Ys2[1] = {Y2};
    if (ok) ok = umma_run(pl, cx, smem, A, Cs2, Ys2, 1, q, r0, r1, ldy, 0, neg);
    else umma_fill_nan(Ys2, 1, q, r0, r1, ldy);
  }
  return ok;
}

}  // namespace qdkp
