// Complex64 block updates on the fifth-generation tensor cores (sm_100a): tcgen05.mma kind::tf32
// with the accumulators in tensor memory (TMEM).
//
// Y (+)= sg [A_0 | A_1 | A_2] [C_0; C_1; C_2] over a CTA's rows, in the real form
// Y' = A' C'' (A' the rows of the complex64 blocks read as floats, C'' the 2x2 real blocks
// [[Re, Im], [-Im, Re]] of the complex coefficients), with every FP32 value split into two TF32
// parts, x = hi + lo (hi = x rounded to TF32, lo = the rest rounded to TF32), and the product
// formed as hi*hi + hi*lo + lo*hi with FP32 accumulation: FP32 accuracy from TF32 tensor cores.
//
// A CTA of 128 threads stages a tile of 128 rows of A' in shared memory in the no-swizzle
// K-major layout the MMA reads (8-row x 16-byte core matrices: element (row, k) at float offset
// ((k / 4) (128 / 8) + row / 8) 32 + (row % 8) 4 + k % 4; leading-byte offset between the two
// 16-byte halves of an MMA-K step = 2048, stride-byte offset between 8-row groups = 128), and the
// coefficients once per CTA as B = C''^T (N x K, same layout). One thread issues the MMAs
// (M = 128, N = 2q padded to a multiple of 16, K = 8 per instruction; three per K step for the
// split) into a TMEM accumulator and commits them to an mbarrier; after a bounded wait every
// thread reads its row of the accumulator (tcgen05.ld 32x32b) and writes it. A tile's rows are
// all staged before any of its outputs is written and no other CTA touches them, so Y may alias
// an input block (the in-place X = [X R P] C updates).
#pragma once
#include <cstdint>

#include "blockops.cuh"

namespace qdkp {

constexpr int kUmmaRows = 128;          // MMA M, rows of a tile, threads of a CTA
constexpr int kUmmaSmemLimit = 220 * 1024;

__device__ __forceinline__ uint32_t umma_saddr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint32_t umma_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
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
__device__ __forceinline__ bool umma_wait(uint32_t mbar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred q;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, q;\n\t}\n" : "=r"(ok) : "r"(mbar), "r"(parity) : "memory");
    if (ok) return true;
    if (clock64() - t0 > 2000000000LL) return false;      // ~1 s: report, never hang
  }
}
__device__ __forceinline__ void umma_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
               "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                 "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__host__ __device__ __forceinline__ int umma_off(int row, int k, int R) {
  return ((k >> 2) * (R >> 3) + (row >> 3)) * 32 + (row & 7) * 4 + (k & 3);
}
__host__ __device__ __forceinline__ int umma_K(int P) { return ((2 * P + 7) / 8) * 8; }
__host__ __device__ __forceinline__ int umma_N(int q) { return ((2 * q + 15) / 16) * 16; }
__host__ __device__ __forceinline__ size_t umma_smem_bytes(int P, int q, int nout) {
  return (size_t)(2 * kUmmaRows * umma_K(P) + 2 * nout * umma_N(q) * umma_K(P)) * sizeof(float);
}
// outputs per pass: both at once when they fit the shared memory, else one pass each
__host__ __device__ __forceinline__ int umma_nout_per_pass(int P, int q, int nout) {
  return (nout == 2 && umma_smem_bytes(P, q, 2) <= (size_t)kUmmaSmemLimit) ? 2 : 1;
}
__host__ __device__ __forceinline__ size_t umma_update_smem_bytes(int P, int q, int nout) {
  return umma_smem_bytes(P, q, umma_nout_per_pass(P, q, nout));
}

// One pass: outputs o < nout of the coefficient lists Cs[o] into Ys[o] (accumulate only for one
// output). Returns false if an MMA completion wait timed out (the outputs then hold NaN).
// tmem: the CTA's accumulator columns (>= nout N); mbar: its MMA-completion barrier, whose
// phase the caller carries across passes
static __device__ bool umma_pass(const BlockList<float>& A, const double2* const* const* Cs,
                                 float2* const* Ys, int nout, int q, long long r0, long long r1,
                                 long long ldy, int accumulate, int neg, float* smf,
                                 uint32_t tmem, uint32_t mbar, uint32_t& phase) {
  const int P = A.total();
  const int K = umma_K(P), N = umma_N(q);
  float* Ahi = smf;
  float* Alo = Ahi + kUmmaRows * K;
  float* Bhi = Alo + kUmmaRows * K;
  float* Blo = Bhi + nout * N * K;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cs1 = A.cols[0], cs2 = cs1 + (A.nblk > 1 ? A.cols[1] : 0);
  const float sg = neg ? -1.f : 1.f;
  // B = C''^T per output: B[j][k], k = 2 (column start of block b + i) + {0: Re, 1: Im} row of A'
  for (int e = tid; e < nout * N * K; e += blockDim.x) {
    const int o = e / (N * K), r = e - o * N * K;
    const int j = r / K, k = r - j * K;
    const int c = k >> 1, jj = j >> 1;
    float v = 0.f;
    if (c < P && jj < q) {
      const int b = c < cs1 ? 0 : (c < cs2 ? 1 : 2);
      const int i = c - (b == 0 ? 0 : (b == 1 ? cs1 : cs2));
      const double2* Cb = Cs[o][b];
      if (Cb) {
        const double2 cc = Cb[(size_t)i * q + jj];
        const float re = sg * (float)cc.x, im = sg * (float)cc.y;
        v = (k & 1) ? ((j & 1) ? re : -im) : ((j & 1) ? im : re);
      }
    }
    const uint32_t hi = umma_tf32(v);
    const int off = o * N * K + umma_off(j, k, N);
    Bhi[off] = __uint_as_float(hi);
    Blo[off] = __uint_as_float(umma_tf32(v - __uint_as_float(hi)));
  }
  // the K padding of A' stays zero for every tile
  for (int e = tid; e < kUmmaRows * (K - 2 * P); e += blockDim.x) {
    const int row = e % kUmmaRows, k = 2 * P + e / kUmmaRows;
    Ahi[umma_off(row, k, kUmmaRows)] = 0.f;
    Alo[umma_off(row, k, kUmmaRows)] = 0.f;
  }
  __syncthreads();
  const uint32_t idesc = umma_idesc_tf32(N);
  const uint32_t lboA = (kUmmaRows / 8) * 128, lboB = (N / 8) * 128;
  const int J = (P + 3) / 4;                 // quads of complex columns
  bool fault = false;
  for (long long t0 = r0; t0 < r1; t0 += kUmmaRows) {
    const int rows = (int)min((long long)kUmmaRows, r1 - t0);
    // stage: a warp instruction covers 8 rows x 4 consecutive complex columns
    for (int p = warp; p < 16 * J; p += 4) {
      const int row = (p & 15) * 8 + (lane & 7), c = (p >> 4) * 4 + (lane >> 3);
      if (row < rows && c < P) {
        const int b = c < cs1 ? 0 : (c < cs2 ? 1 : 2);
        const int i = c - (b == 0 ? 0 : (b == 1 ? cs1 : cs2));
        const float2 a = A.p[b][(t0 + row) * A.ld[b] + i];
        const uint32_t hx = umma_tf32(a.x), hy = umma_tf32(a.y);
        const int off = umma_off(row, 2 * c, kUmmaRows);
        *reinterpret_cast<float2*>(Ahi + off) = make_float2(__uint_as_float(hx), __uint_as_float(hy));
        *reinterpret_cast<float2*>(Alo + off) =
            make_float2(__uint_as_float(umma_tf32(a.x - __uint_as_float(hx))),
                        __uint_as_float(umma_tf32(a.y - __uint_as_float(hy))));
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t aH = umma_saddr(Ahi), aL = umma_saddr(Alo);
      for (int o = 0; o < nout; ++o) {
        const uint32_t bH = umma_saddr(Bhi + o * N * K), bL = umma_saddr(Blo + o * N * K);
        const uint32_t d = tmem + (uint32_t)(o * N);
        for (int s = 0; s < K / 8; ++s) {
          const uint32_t ka = 2 * s * lboA, kb = 2 * s * lboB;
          umma_mma(d, umma_desc(aH + ka, lboA, 128), umma_desc(bH + kb, lboB, 128), idesc, s > 0);
          umma_mma(d, umma_desc(aH + ka, lboA, 128), umma_desc(bL + kb, lboB, 128), idesc, 1);
          umma_mma(d, umma_desc(aL + ka, lboA, 128), umma_desc(bH + kb, lboB, 128), idesc, 1);
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   :: "r"(mbar) : "memory");
    }
    const bool ok = umma_wait(mbar, phase);
    fault = __syncthreads_or(!ok) != 0;
    phase ^= 1;
    asm volatile("tcgen05.fence::after_thread_sync;");
    const long long r = t0 + tid;
    for (int o = 0; o < nout; ++o) {
      float2* Yo = Ys[o];
      for (int c0 = 0; c0 < N; c0 += 16) {
        float v[16];
        umma_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(o * N + c0), v);
        if (tid < rows) {
#pragma unroll
          for (int i = 0; i < 16; i += 2) {
            const int jj = (c0 + i) >> 1;
            if (jj < q) {
              float2 y = fault ? make_float2(__int_as_float(0x7fc00000), __int_as_float(0x7fc00000))
                               : make_float2(v[i], v[i + 1]);
              if (accumulate && !fault) {
                const float2 old = Yo[r * ldy + jj];
                y.x += old.x; y.y += old.y;
              }
              Yo[r * ldy + jj] = y;
            }
          }
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (fault) break;                            // uniform
  }
  return !fault;
}

// Y (+)= sg A C over rows [r0, r1) and, with C2 / Y2, Y2 = sg A C2: the contract of
// update_rows_tf32 (C[b] the cols_b x q row-major complex coefficients of A's block b, NULL:
// the block does not enter). 128 threads; `smem` holds umma_update_smem_bytes(P, q, nout).
// When both outputs do not fit one pass, Y is formed first and Y2 second, each in its own pass
// over A, so Y must not alias an input there (Y2 may). Returns false on a timed-out wait.
static __device__ bool update_rows_umma(const BlockList<float>& A, const double2* const* C, int q,
                                        long long r0, long long r1, float2* Y, long long ldy,
                                        int accumulate, int neg, unsigned char* smem,
                                        const double2* const* C2 = nullptr, float2* Y2 = nullptr) {
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  if (r0 >= r1) return true;
  float* smf = reinterpret_cast<float*>(smem);
  const int P = A.total();
  const int nout = Y2 ? 2 : 1;
  const bool one_pass = nout == 2 && !accumulate && umma_nout_per_pass(P, q, 2) == 2;
  uint32_t ncols = 32;
  while ((int)ncols < (one_pass ? 2 : 1) * umma_N(q)) ncols <<= 1;
  if ((threadIdx.x >> 5) == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(umma_saddr(&tmem_base)), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(umma_saddr(&mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base, bar = umma_saddr(&mbar);
  uint32_t phase = 0;
  bool ok;
  if (one_pass) {
    const double2* const* Cs[2] = {C, C2};
    float2* const Ys[2] = {Y, Y2};
    ok = umma_pass(A, Cs, Ys, 2, q, r0, r1, ldy, 0, neg, smf, tmem, bar, phase);
  } else {
    const double2* const* Cs1[1] = {C};
    float2* const Ys1[1] = {Y};
    ok = umma_pass(A, Cs1, Ys1, 1, q, r0, r1, ldy, accumulate, neg, smf, tmem, bar, phase);
    if (nout == 2 && ok) {
      const double2* const* Cs2[1] = {C2};
      float2* const Ys2[1] = {Y2};
      ok = umma_pass(A, Cs2, Ys2, 1, q, r0, r1, ldy, 0, neg, smf, tmem, bar, phase);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if ((threadIdx.x >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(ncols));
  return ok;
}

}  // namespace qdkp
