// Matrix-free H.X for the discretised Pryor eight-band k.p operator (sm_100a).
//
// Replaces the CSR product `H @ X` of qd3Dsolver (H from kp_pryor.confined_hamiltonian,
// kp_pryor.py:363-466) with a fused 8x8-block, 19-point stencil. The operator is the sum of
//   * a local Hermitian 8x8 block per site (band edges, spin-orbit, Bir-Pikus Q/R/S strain
//     terms kp_pryor.py:111-113, and the diagonal of every second-derivative stencil),
//   * six face couplings: the three-point face-averaged k2_a stencils (kp_confined.py:88-143)
//     feeding A, P, Q and the real part of R, and the symmetrised first-derivative terms U, V
//     (kp_pryor.py:430-454, central differences kp_confined.py:58-85),
//   * twelve in-plane edge couplings: the symmetrised cross terms cross(g3, a, b)
//     (kp_confined.py:146-183) feeding the imaginary part of R and all of S.
// The block layout of those pieces is Pryor's table (kp_pryor.py:244-301) with the lower
// triangle the adjoint of the upper (kp_pryor.py:216-241).
//
// Two kernels:
//   kp_record_kernel  once per operator (and per band-edge update): folds the 15 raw per-site
//                     fields into a per-site record of stencil weights (local block, the three
//                     "+" faces, the twelve edge weights) and a neighbour mask. The record is
//                     kept in FP64 and FP32; the sign of the hole convention / negation is
//                     folded in, so the apply kernel never branches on it.
//   kp_apply_kernel   one thread per (site, column): loads the eight band components of the
//                     site, its six faces and twelve edges (valence bands only) for that
//                     column, and accumulates all eight output bands in registers. A "-" face
//                     reads its weights from the neighbour's "+" face (the face weights are
//                     symmetric; the first-order ones change sign). The edge terms of a plane
//                     are summed with their scalar weights first and the constant band-mixing
//                     matrix of that plane is applied once.
#include <cuda.h>   // CUtensorMap and its enums (the encoder is fetched from the runtime)

#include <algorithm>
#include <type_traits>

#include "qdkp_common.cuh"

namespace qdkp {

// Record layout: entry k of site (ix, iy, iz) at rec[k * NP + (ix * ny + iy) * nzp + iz], with z
// padded to nzp = a multiple of 4 (zeros in the padding) so that a z-run of a tile row starts on
// a 16-byte boundary for the staged kernel's copies; NP = nx ny nzp.
enum RecEntry {
  K_A = 0,      // sign (Ec + 6 G / h^2): conduction diagonal
  K_A2,         // sign (-P + Q): LH/HH diagonals of rows 2, 5
  K_A3,         // sign (-P - Q): rows 3, 4
  K_A6,         // sign (-P - Delta): split-off rows 6, 7
  K_Q2,         // sign sqrt2 Q
  K_RRE, K_RIM, K_SRE, K_SIM,
  K_FACE = 9,   // per face f (x+, x-, y+, y-, z+, z-): K_FACE + 5f + {0 kp, 1 k2, 2 su, 3 svr, 4 svi}
  K_EDGE = 39,  // per plane pl (xy, zx, zy) and edge e: K_EDGE + 4 pl + e
  K_COUNT = 51
};

// ---------------------------------------------------------------------------------------------
// Record construction (FP64, once per operator)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void first_order_coefs(const double* __restrict__ F, long long N,
                                                  long long q, bool inter, double cu[3],
                                                  double2 cv[3]) {
  const double r3 = 0.57735026918962576451, r6 = 0.40824829046386301637;
  const double P0 = F[F_P0 * N + q];
  if (inter) {
    const double exx = F[F_EXX * N + q], eyy = F[F_EYY * N + q], ezz = F[F_EZZ * N + q];
    const double exy = F[F_EXY * N + q], eyz = F[F_EYZ * N + q], ezx = F[F_EZX * N + q];
    cu[0] = -P0 * ezx * r3;
    cu[1] = -P0 * eyz * r3;
    cu[2] = P0 * (1.0 - ezz) * r3;
    cv[0] = make_double2(P0 * (1.0 - exx) * r6, P0 * exy * r6);
    cv[1] = make_double2(-P0 * exy * r6, P0 * (eyy - 1.0) * r6);
    cv[2] = make_double2(-P0 * ezx * r6, P0 * eyz * r6);
  } else {
    cu[0] = 0.0; cu[1] = 0.0; cu[2] = P0 * r3;
    cv[0] = make_double2(P0 * r6, 0.0);
    cv[1] = make_double2(0.0, -P0 * r6);
    cv[2] = make_double2(0.0, 0.0);
  }
}

__global__ void kp_record_kernel(const double* __restrict__ F, long long N, int nx, int ny,
                                 int nz, int nzp, double h, int flags, int nb, double sign,
                                 double* __restrict__ rec64, float* __restrict__ rec32,
                                 unsigned* __restrict__ nbmask) {
  const double G = kG;
  const double ih2 = 1.0 / (h * h);
  const double i4h = 1.0 / (4.0 * h);
  const double i8h2 = 1.0 / (8.0 * h * h);
  const double sq2 = 1.41421356237309504880, sq3 = 1.73205080756887729353;
  const bool strain = (flags & QDKP_STRAIN) != 0;
  const bool inter = nb == 8 && strain && (flags & QDKP_INTERBAND_STRAIN);
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N;
       s += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(s % nz);
    const long long t = s / nz;
    const int iy = (int)(t % ny);
    const int ix = (int)(t / ny);
    const int coord[3] = {ix, iy, iz};
    const int ext[3] = {nx, ny, nz};
    const long long str[3] = {(long long)ny * nz, (long long)nz, 1LL};
    double r[K_COUNT];
    // neighbour mask: bit f (0..5) face x+, x-, y+, y-, z+, z-; bit 6 + 4 pl + e the in-plane
    // edge e of plane pl (xy, zx, zy) with signs sa = e & 1 ? -1 : 1, sb = e & 2 ? -1 : 1
    unsigned msk = 0;
    for (int ax = 0; ax < 3; ++ax) {
      if (coord[ax] + 1 < ext[ax]) msk |= 1u << (2 * ax);
      if (coord[ax] > 0) msk |= 1u << (2 * ax + 1);
    }
    const double g1 = F[F_G1 * N + s], g2 = F[F_G2 * N + s];
    double cu_p[3]; double2 cv_p[3];
    if (nb == 8) first_order_coefs(F, N, s, inter, cu_p, cv_p);
    double dk1 = 0.0, dk2[3];
    for (int ax = 0; ax < 3; ++ax) {
      double d1 = 0.0, d2 = 0.0;
      for (int dir = 0; dir < 2; ++dir) {
        const bool in = dir == 0 ? (coord[ax] + 1 < ext[ax]) : (coord[ax] > 0);
        double kp = 0.0, k2 = 0.0, su = 0.0, svr = 0.0, svi = 0.0;
        if (in) {
          const long long q = dir == 0 ? s + str[ax] : s - str[ax];
          const double t1 = (g1 + F[F_G1 * N + q]) * 0.5 * ih2;
          const double t2 = (g2 + F[F_G2 * N + q]) * 0.5 * ih2;
          d1 += t1; d2 += t2;
          kp = -G * t1; k2 = -G * t2;
          if (nb == 8) {
            // symmetrised first derivative: (cu_p + cu_q) / 4h, signed by the face direction
            double cu_q[3]; double2 cv_q[3];
            first_order_coefs(F, N, q, inter, cu_q, cv_q);
            const double sg = dir == 0 ? i4h : -i4h;
            su = (cu_p[ax] + cu_q[ax]) * sg;
            svr = (cv_p[ax].x + cv_q[ax].x) * sg;
            svi = (cv_p[ax].y + cv_q[ax].y) * sg;
          }
        } else {  // hard wall: ghost term alpha_p / h^2 (kp_confined.py:133-137)
          d1 += g1 * ih2; d2 += g2 * ih2;
        }
        const int kf = K_FACE + 5 * (2 * ax + dir);
        r[kf + 0] = sign * kp;
        r[kf + 1] = sign * k2;
        r[kf + 2] = sign * su;
        r[kf + 3] = sign * svr;
        r[kf + 4] = sign * svi;
      }
      dk1 += d1; dk2[ax] = d2;
    }
    double Q = G * (dk2[0] + dk2[1] - 2.0 * dk2[2]);
    double Rre = -sq3 * G * (dk2[0] - dk2[1]), Rim = 0.0, Sre = 0.0, Sim = 0.0;
    if (strain) {
      const double b = F[F_B * N + s], d = F[F_D * N + s];
      const double exx = F[F_EXX * N + s], eyy = F[F_EYY * N + s], ezz = F[F_EZZ * N + s];
      const double exy = F[F_EXY * N + s], eyz = F[F_EYZ * N + s], ezx = F[F_EZX * N + s];
      Q += -(b / 2.0) * (exx + eyy - 2.0 * ezz);
      Rre += (sq3 / 2.0) * b * (exx - eyy);
      Rim += -d * exy;
      Sre = -d * ezx;
      Sim = d * eyz;
    }
    const double A = F[F_EC * N + s] + 6.0 * G * ih2;
    const double P = -F[F_EV * N + s] + G * dk1;
    const double Dl = F[F_DSO * N + s];
    r[K_A] = sign * A;
    r[K_A2] = sign * (-P + Q);
    r[K_A3] = sign * (-P - Q);
    r[K_A6] = sign * (-P - Dl);
    r[K_Q2] = sign * sq2 * Q;
    r[K_RRE] = sign * Rre; r[K_RIM] = sign * Rim;
    r[K_SRE] = sign * Sre; r[K_SIM] = sign * Sim;
    // cross(g3, a, b): coefficient of x(p + sa e_a + sb e_b) in the R / S slots is
    // 2 sqrt3 G * (-(sa sb) / (8 h^2)) (g3(p + sa e_a) + g3(p + sb e_b))
    for (int pl = 0; pl < 3; ++pl) {
      const int ea = pl == 0 ? 0 : 2, eb = pl == 0 ? 1 : (pl == 1 ? 0 : 1);
      for (int e = 0; e < 4; ++e) {
        const int sa = (e & 1) ? -1 : 1, sb = (e & 2) ? -1 : 1;
        const int ca = coord[ea] + sa, cb = coord[eb] + sb;
        double c = 0.0;
        if (ca >= 0 && ca < ext[ea] && cb >= 0 && cb < ext[eb]) {
          msk |= 1u << (6 + 4 * pl + e);
          const double ga = F[F_G3 * N + s + sa * str[ea]];
          const double gb = F[F_G3 * N + s + sb * str[eb]];
          c = 2.0 * sq3 * G * (-(double)(sa * sb) * i8h2) * (ga + gb);
        }
        r[K_EDGE + 4 * pl + e] = sign * c;
      }
    }
    const long long NP = (long long)nx * ny * nzp;
    const long long sp = t * nzp + iz;
    for (int k = 0; k < K_COUNT; ++k) {
      rec64[k * NP + sp] = r[k];
      rec32[k * NP + sp] = (float)r[k];
    }
    nbmask[s] = msk;
  }
}

// ---------------------------------------------------------------------------------------------
// The stencil arithmetic, shared by the kernels below. `L` supplies the neighbour values of one
// column (centre, face f = x+, x-, y+, y-, z+, z-, edge (pl, e)); `Rc` the site's record
// entries (own(k); face(ax, dir, k): entry k of face (ax, dir)).
// ---------------------------------------------------------------------------------------------
template <int NB> __device__ __forceinline__ constexpr bool has_band(int b) {
  return NB == 8 ? true : (NB == 6 ? b >= 2 : (b >= 2 && b <= 5));
}
template <int NB> __device__ __forceinline__ constexpr int band_off() { return NB == 8 ? 0 : 2; }

template <typename T, int NB, class L, class Rc>
__device__ __forceinline__ void hx_math(const L& ld, const Rc& rc, unsigned msk, T shift, T cb,
                                        cplx<T> (&y)[8]) {
  const T sq2 = T(1.41421356237309504880), sq3 = T(1.73205080756887729353);
  const T sq32 = T(1.22474487139158904910), isq2 = T(0.70710678118654752440);
  const T wQ[3] = {T(1), T(1), T(-2)};
  const T wR[3] = {-sq3, sq3, T(0)};
  cplx<T> x[8];

  // ---- local block (with the shift -sigma) -------------------------------------------
  ld.centre(x);
#pragma unroll
  for (int b = 0; b < 8; ++b) y[b] = cscale(shift, x[b]);
  {
    const T a2 = rc.own(K_A2), a3 = rc.own(K_A3), a6 = rc.own(K_A6), q2 = rc.own(K_Q2);
    const cplx<T> Rr = mk<T>(rc.own(K_RRE), rc.own(K_RIM));
    const cplx<T> Sx = mk<T>(rc.own(K_SRE), rc.own(K_SIM));
    if (NB == 8) {
      const T A = rc.own(K_A);
      caxpy(y[0], A, x[0]); caxpy(y[1], A, x[1]);
    }
    const cplx<T> R2 = cscale(sq2, Rr), S32 = cscale(sq32, Sx), Si2 = cscale(isq2, Sx);
    caxpy(y[2], a2, x[2]); cfmac(y[2], Sx, cscale(T(-1), x[3])); cfma(y[2], Rr, x[4]);
    cfma(y[2], S32, x[6]); caxpy(y[2], -q2, x[7]);
    cfma(y[3], Sx, cscale(T(-1), x[2])); caxpy(y[3], a3, x[3]); cfma(y[3], Rr, x[5]);
    cfma(y[3], R2, cscale(T(-1), x[6])); cfma(y[3], Si2, x[7]);
    cfmac(y[4], Rr, x[2]); caxpy(y[4], a3, x[4]); cfmac(y[4], Sx, x[5]);
    cfmac(y[4], Si2, x[6]); cfmac(y[4], R2, x[7]);
    cfmac(y[5], Rr, x[3]); cfma(y[5], Sx, x[4]); caxpy(y[5], a2, x[5]);
    caxpy(y[5], q2, x[6]); cfmac(y[5], S32, x[7]);
    cfmac(y[6], S32, x[2]); cfmac(y[6], R2, cscale(T(-1), x[3]));
    cfma(y[6], Si2, x[4]); caxpy(y[6], q2, x[5]); caxpy(y[6], a6, x[6]);
    caxpy(y[7], -q2, x[2]); cfmac(y[7], Si2, x[3]); cfma(y[7], R2, x[4]);
    cfma(y[7], S32, x[5]); caxpy(y[7], a6, x[7]);
  }

  // ---- six face neighbours ------------------------------------------------------------
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const int ax = f >> 1, dir = f & 1;
    if (!(msk & (1u << f))) continue;
    ld.face(f, x);
    const T kp = rc.face(ax, dir, 0), k2 = rc.face(ax, dir, 1);
    const T kq = wQ[ax] * k2;
    if (NB == 8) { caxpy(y[0], cb, x[0]); caxpy(y[1], cb, x[1]); }
    caxpy(y[2], -kp + kq, x[2]); caxpy(y[2], -sq2 * kq, x[7]);
    caxpy(y[3], -kp - kq, x[3]);
    caxpy(y[4], -kp - kq, x[4]);
    caxpy(y[5], -kp + kq, x[5]); caxpy(y[5], sq2 * kq, x[6]);
    caxpy(y[6], -kp, x[6]); caxpy(y[6], sq2 * kq, x[5]);
    caxpy(y[7], -kp, x[7]); caxpy(y[7], -sq2 * kq, x[2]);
    if (ax < 2) {
      const T kr = wR[ax] * k2;
      caxpy(y[2], kr, x[4]);
      caxpy(y[3], kr, x[5]); caxpy(y[3], -sq2 * kr, x[6]);
      caxpy(y[4], kr, x[2]); caxpy(y[4], sq2 * kr, x[7]);
      caxpy(y[5], kr, x[3]);
      caxpy(y[6], -sq2 * kr, x[3]);
      caxpy(y[7], sq2 * kr, x[4]);
    }
    if (NB == 8) {
      // first-order weights of this face; U w = -i su w, V w = -i sv w, V^H w = -i conj(sv) w
      // for the neighbour value w.
      const T su = rc.face(ax, dir, 2);
      const cplx<T> sv = mk<T>(rc.face(ax, dir, 3), rc.face(ax, dir, 4));
      // conduction rows from valence inputs
      cplx<T> m1 = x[2]; caxpy(m1, sq2, x[7]);                   // V^H (x2 + sqrt2 x7)
      const cplx<T> m2 = cscale(sq3, x[4]);                      // V (sqrt3 x4)
      cplx<T> m3 = cscale(-sq2, x[5]); m3 = csub(m3, x[6]);      // U (-sqrt2 x5 - x6)
      cplx<T> acc = czero<T>();
      cfmac(acc, sv, m1); cfma(acc, sv, m2); caxpy(acc, su, m3);
      caxpy_i(y[0], T(-1), acc);
      cplx<T> n1 = cscale(-sq2, x[2]); n1 = cadd(n1, x[7]);      // U (-sqrt2 x2 + x7)
      const cplx<T> n2 = cscale(-sq3, x[3]);                     // V^H (-sqrt3 x3)
      cplx<T> n3 = cscale(sq2, x[6]); n3 = csub(n3, x[5]);       // V (-x5 + sqrt2 x6)
      acc = czero<T>();
      caxpy(acc, su, n1); cfmac(acc, sv, n2); cfma(acc, sv, n3);
      caxpy_i(y[1], T(-1), acc);
      // valence rows from conduction inputs
      cplx<T> Vw0 = czero<T>(), VHw0 = czero<T>(), Vw1 = czero<T>(), VHw1 = czero<T>();
      cfma(Vw0, sv, x[0]); cfmac(VHw0, sv, x[0]); cfma(Vw1, sv, x[1]); cfmac(VHw1, sv, x[1]);
      const cplx<T> Uw0 = cscale(su, x[0]), Uw1 = cscale(su, x[1]);
      // every term carries the common factor -i
      cplx<T> t2 = Vw0; caxpy(t2, -sq2, Uw1); caxpy_i(y[2], T(-1), t2);
      caxpy_i(y[3], sq3, Vw1);
      caxpy_i(y[4], -sq3, VHw0);
      cplx<T> t5 = cscale(-sq2, Uw0); t5 = csub(t5, VHw1); caxpy_i(y[5], T(-1), t5);
      cplx<T> t6 = cscale(sq2, VHw1); t6 = csub(t6, Uw0); caxpy_i(y[6], T(-1), t6);
      cplx<T> t7 = cscale(sq2, Vw0); t7 = cadd(t7, Uw1); caxpy_i(y[7], T(-1), t7);
    }
  }

  // ---- twelve edge neighbours: cross(g3, a, b) ---------------------------------------
  // z = sum_e c_e x(p + sa e_a + sb e_b) over the plane's edges, then the plane's constant
  // band mixing: xy -> R (+i z) / R^H (-i z); zx -> S, S^H (z); zy -> S (-i z), S^H (+i z).
#pragma unroll
  for (int pl = 0; pl < 3; ++pl) {
    if (!(msk & (0xFu << (6 + 4 * pl)))) continue;
    cplx<T> z[8];
#pragma unroll
    for (int b = 0; b < 8; ++b) z[b] = czero<T>();
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (!(msk & (1u << (6 + 4 * pl + e)))) continue;
      ld.edge(pl, e, x);
      const T c = rc.own(K_EDGE + 4 * pl + e);
#pragma unroll
      for (int b = 2; b < 8; ++b) caxpy(z[b], c, x[b]);
    }
    if (pl == 0) {
      caxpy_i(y[2], T(1), z[4]);
      caxpy_i(y[4], T(-1), z[2]);
      caxpy_i(y[3], T(1), z[5]);
      caxpy_i(y[5], T(-1), z[3]);
      caxpy_i(y[3], -sq2, z[6]);
      caxpy_i(y[6], sq2, z[3]);
      caxpy_i(y[4], -sq2, z[7]);
      caxpy_i(y[7], sq2, z[4]);
    } else if (pl == 1) {
      caxpy(y[3], T(-1), z[2]); caxpy(y[2], sq32, z[6]); caxpy(y[3], isq2, z[7]);
      caxpy(y[5], T(1), z[4]); caxpy(y[6], isq2, z[4]); caxpy(y[7], sq32, z[5]);
      caxpy(y[2], T(-1), z[3]); caxpy(y[6], sq32, z[2]); caxpy(y[7], isq2, z[3]);
      caxpy(y[4], T(1), z[5]); caxpy(y[4], isq2, z[6]); caxpy(y[5], sq32, z[7]);
    } else {
      caxpy_i(y[3], T(1), z[2]); caxpy_i(y[2], -sq32, z[6]); caxpy_i(y[3], -isq2, z[7]);
      caxpy_i(y[5], T(-1), z[4]); caxpy_i(y[6], -isq2, z[4]); caxpy_i(y[7], -sq32, z[5]);
      caxpy_i(y[2], T(-1), z[3]); caxpy_i(y[6], sq32, z[2]); caxpy_i(y[7], isq2, z[3]);
      caxpy_i(y[4], T(1), z[5]); caxpy_i(y[4], isq2, z[6]); caxpy_i(y[5], sq32, z[7]);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// complex64 form of the same arithmetic on packed f32x2 registers (sm_100 `fma.rn.f32x2`):
// a complex value is one 64-bit register pair, and every term is a real scalar (broadcast to
// both halves) times a neighbour value. Products that carry a factor i go to a second
// accumulator yi, so the result is Y = y + i yi and complex coefficients c = cr + i ci split
// into cr -> y and ci -> yi. Half the issue slots of the scalar form for the same arithmetic.
// ---------------------------------------------------------------------------------------------
typedef unsigned long long f2;
__device__ __forceinline__ f2 f2pk(float a, float b) {
  f2 r; asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b)); return r;
}
__device__ __forceinline__ f2 f2bc(float s) { return f2pk(s, s); }
__device__ __forceinline__ float2 f2up(f2 v) {
  float2 r; asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v)); return r;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
  f2 d; asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c)); return d;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
  f2 d; asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b)); return d;
}
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
  f2 d; asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b)); return d;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
  f2 d; asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b)); return d;
}

template <class L, class Rc>
__device__ __forceinline__ void hx_math_packed(const L& ld, const Rc& rc, unsigned msk,
                                               float shift, float cb, float2 (&Y)[8]) {
  const float sq2 = 1.41421356237309504880f, sq3 = 1.73205080756887729353f;
  const float sq32 = 1.22474487139158904910f, isq2 = 0.70710678118654752440f;
  const f2 C2 = f2bc(sq2), CN2 = f2bc(-sq2), C3 = f2bc(sq3), C32 = f2bc(sq32);
  const f2 CN32 = f2bc(-sq32), Ci2 = f2bc(isq2), CNi2 = f2bc(-isq2), CN1 = f2bc(-1.f);
  const f2 CB = f2bc(cb);
  f2 y[8], yi[8], x[8];

  // ---- local block, the shift -sigma folded into the diagonal ---------------------------
  ld.centre2(x);
  {
    const float Rr = rc.own(K_RRE), Ri = rc.own(K_RIM), Sr = rc.own(K_SRE), Si = rc.own(K_SIM);
    const float q2 = rc.own(K_Q2);
    const f2 PA = f2bc(rc.own(K_A) + shift), P2 = f2bc(rc.own(K_A2) + shift);
    const f2 P3 = f2bc(rc.own(K_A3) + shift), P6 = f2bc(rc.own(K_A6) + shift);
    const f2 Q2 = f2bc(q2), NQ2 = f2bc(-q2);
    const f2 SR = f2bc(Sr), NSR = f2bc(-Sr), SI = f2bc(Si), NSI = f2bc(-Si);
    const f2 RR = f2bc(Rr), RI = f2bc(Ri), NRI = f2bc(-Ri);
    const f2 S32R = f2bc(sq32 * Sr), S32I = f2bc(sq32 * Si), NS32I = f2bc(-sq32 * Si);
    const f2 R2R = f2bc(sq2 * Rr), NR2R = f2bc(-sq2 * Rr), R2I = f2bc(sq2 * Ri);
    const f2 NR2I = f2bc(-sq2 * Ri);
    const f2 SI2R = f2bc(isq2 * Sr), SI2I = f2bc(isq2 * Si), NSI2I = f2bc(-isq2 * Si);
    y[0] = mul2(PA, x[0]); y[1] = mul2(PA, x[1]);
    yi[0] = 0ull; yi[1] = 0ull;
    y[2] = fma2(NSR, x[3], mul2(P2, x[2]));   yi[2] = mul2(SI, x[3]);
    y[2] = fma2(RR, x[4], y[2]);              yi[2] = fma2(RI, x[4], yi[2]);
    y[2] = fma2(S32R, x[6], y[2]);            yi[2] = fma2(S32I, x[6], yi[2]);
    y[2] = fma2(NQ2, x[7], y[2]);
    y[3] = fma2(NSR, x[2], mul2(P3, x[3]));   yi[3] = mul2(NSI, x[2]);
    y[3] = fma2(RR, x[5], y[3]);              yi[3] = fma2(RI, x[5], yi[3]);
    y[3] = fma2(NR2R, x[6], y[3]);            yi[3] = fma2(NR2I, x[6], yi[3]);
    y[3] = fma2(SI2R, x[7], y[3]);            yi[3] = fma2(SI2I, x[7], yi[3]);
    y[4] = fma2(RR, x[2], mul2(P3, x[4]));    yi[4] = mul2(NRI, x[2]);
    y[4] = fma2(SR, x[5], y[4]);              yi[4] = fma2(NSI, x[5], yi[4]);
    y[4] = fma2(SI2R, x[6], y[4]);            yi[4] = fma2(NSI2I, x[6], yi[4]);
    y[4] = fma2(R2R, x[7], y[4]);             yi[4] = fma2(NR2I, x[7], yi[4]);
    y[5] = fma2(RR, x[3], mul2(P2, x[5]));    yi[5] = mul2(NRI, x[3]);
    y[5] = fma2(SR, x[4], y[5]);              yi[5] = fma2(SI, x[4], yi[5]);
    y[5] = fma2(Q2, x[6], y[5]);
    y[5] = fma2(S32R, x[7], y[5]);            yi[5] = fma2(NS32I, x[7], yi[5]);
    y[6] = fma2(S32R, x[2], mul2(P6, x[6]));  yi[6] = mul2(NS32I, x[2]);
    y[6] = fma2(NR2R, x[3], y[6]);            yi[6] = fma2(R2I, x[3], yi[6]);
    y[6] = fma2(SI2R, x[4], y[6]);            yi[6] = fma2(SI2I, x[4], yi[6]);
    y[6] = fma2(Q2, x[5], y[6]);
    y[7] = fma2(NQ2, x[2], mul2(P6, x[7]));
    y[7] = fma2(SI2R, x[3], y[7]);            yi[7] = mul2(NSI2I, x[3]);
    y[7] = fma2(R2R, x[4], y[7]);             yi[7] = fma2(R2I, x[4], yi[7]);
    y[7] = fma2(S32R, x[5], y[7]);            yi[7] = fma2(S32I, x[5], yi[7]);
  }

  // ---- six face neighbours ------------------------------------------------------------
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const int ax = f >> 1, dir = f & 1;
    if (!(msk & (1u << f))) continue;
    ld.face2(f, x);
    const float kp = rc.face(ax, dir, 0), k2 = rc.face(ax, dir, 1);
    const float kq = (ax == 2 ? -2.f : 1.f) * k2;
    y[0] = fma2(CB, x[0], y[0]); y[1] = fma2(CB, x[1], y[1]);
    const f2 KPQ = f2bc(kq - kp), NKPQ = f2bc(-kp - kq), NKP = f2bc(-kp);
    const f2 K2Q = f2bc(sq2 * kq), NK2Q = f2bc(-sq2 * kq);
    y[2] = fma2(KPQ, x[2], y[2]); y[2] = fma2(NK2Q, x[7], y[2]);
    y[3] = fma2(NKPQ, x[3], y[3]);
    y[4] = fma2(NKPQ, x[4], y[4]);
    y[5] = fma2(KPQ, x[5], y[5]); y[5] = fma2(K2Q, x[6], y[5]);
    y[6] = fma2(NKP, x[6], y[6]); y[6] = fma2(K2Q, x[5], y[6]);
    y[7] = fma2(NKP, x[7], y[7]); y[7] = fma2(NK2Q, x[2], y[7]);
    if (ax < 2) {
      const float kr = (ax == 0 ? -sq3 : sq3) * k2;
      const f2 KR = f2bc(kr), K2R = f2bc(sq2 * kr), NK2R = f2bc(-sq2 * kr);
      y[2] = fma2(KR, x[4], y[2]);
      y[3] = fma2(KR, x[5], y[3]); y[3] = fma2(NK2R, x[6], y[3]);
      y[4] = fma2(KR, x[2], y[4]); y[4] = fma2(K2R, x[7], y[4]);
      y[5] = fma2(KR, x[3], y[5]);
      y[6] = fma2(NK2R, x[3], y[6]);
      y[7] = fma2(K2R, x[4], y[7]);
    }
    // first-order (U, V) couplings with the face weights su (real), sv = svr + i svi:
    //   y0 += -i [conj(sv)(x2 + sqrt2 x7) + sv sqrt3 x4 + su (-sqrt2 x5 - x6)]
    //   y1 += -i [su (-sqrt2 x2 + x7) - conj(sv) sqrt3 x3 + sv (-x5 + sqrt2 x6)]
    //   y2..y7 from x0, x1 (the adjoint blocks)
    const float su = rc.face(ax, dir, 2), svr = rc.face(ax, dir, 3), svi = rc.face(ax, dir, 4);
    const f2 SVI = f2bc(svi), SVR = f2bc(svr), SU = f2bc(su), NSVR = f2bc(-svr), NSU = f2bc(-su);
    const f2 S2SU = f2bc(sq2 * su), N3SVI = f2bc(-sq3 * svi), S3SVR = f2bc(sq3 * svr);
    const f2 N3SVR = f2bc(-sq3 * svr), N2SVI = f2bc(-sq2 * svi), N2SVR = f2bc(-sq2 * svr);
    const f2 S2SVI = f2bc(sq2 * svi);
    {
      const f2 t = fma2(C2, x[7], x[2]);        // x2 + sqrt2 x7
      const f2 u = mul2(C3, x[4]);              // sqrt3 x4
      y[0] = fma2(SVI, sub2(u, t), y[0]);
      yi[0] = fma2(NSVR, add2(u, t), yi[0]);
      yi[0] = fma2(SU, fma2(C2, x[5], x[6]), yi[0]);
      const f2 v = mul2(C3, x[3]);              // sqrt3 x3
      const f2 w = fma2(CN2, x[6], x[5]);       // x5 - sqrt2 x6
      y[1] = fma2(SVI, sub2(v, w), y[1]);
      yi[1] = fma2(SVR, add2(v, w), yi[1]);
      yi[1] = fma2(SU, fma2(C2, x[2], mul2(CN1, x[7])), yi[1]);
    }
    y[2] = fma2(SVI, x[0], y[2]);   yi[2] = fma2(NSVR, x[0], yi[2]); yi[2] = fma2(S2SU, x[1], yi[2]);
    y[3] = fma2(N3SVI, x[1], y[3]); yi[3] = fma2(S3SVR, x[1], yi[3]);
    y[4] = fma2(N3SVI, x[0], y[4]); yi[4] = fma2(N3SVR, x[0], yi[4]);
    y[5] = fma2(SVI, x[1], y[5]);   yi[5] = fma2(S2SU, x[0], yi[5]); yi[5] = fma2(SVR, x[1], yi[5]);
    y[6] = fma2(N2SVI, x[1], y[6]); yi[6] = fma2(N2SVR, x[1], yi[6]); yi[6] = fma2(SU, x[0], yi[6]);
    y[7] = fma2(S2SVI, x[0], y[7]); yi[7] = fma2(N2SVR, x[0], yi[7]); yi[7] = fma2(NSU, x[1], yi[7]);
  }

  // ---- twelve edge neighbours: z = sum_e c_e x_e, then the plane's band mixing ---------
#pragma unroll
  for (int pl = 0; pl < 3; ++pl) {
    if (!(msk & (0xFu << (6 + 4 * pl)))) continue;
    f2 z[8];
#pragma unroll
    for (int b = 2; b < 8; ++b) z[b] = 0ull;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (!(msk & (1u << (6 + 4 * pl + e)))) continue;
      ld.edge2(pl, e, x);
      const f2 C = f2bc(rc.own(K_EDGE + 4 * pl + e));
#pragma unroll
      for (int b = 2; b < 8; ++b) z[b] = fma2(C, x[b], z[b]);
    }
    if (pl == 0) {            // R: +i z, R^H: -i z
      yi[2] = add2(yi[2], z[4]); yi[4] = sub2(yi[4], z[2]);
      yi[3] = add2(yi[3], z[5]); yi[5] = sub2(yi[5], z[3]);
      yi[3] = fma2(CN2, z[6], yi[3]); yi[6] = fma2(C2, z[3], yi[6]);
      yi[4] = fma2(CN2, z[7], yi[4]); yi[7] = fma2(C2, z[4], yi[7]);
    } else if (pl == 1) {     // S, S^H: z
      y[3] = sub2(y[3], z[2]); y[2] = fma2(C32, z[6], y[2]); y[3] = fma2(Ci2, z[7], y[3]);
      y[5] = add2(y[5], z[4]); y[6] = fma2(Ci2, z[4], y[6]); y[7] = fma2(C32, z[5], y[7]);
      y[2] = sub2(y[2], z[3]); y[6] = fma2(C32, z[2], y[6]); y[7] = fma2(Ci2, z[3], y[7]);
      y[4] = add2(y[4], z[5]); y[4] = fma2(Ci2, z[6], y[4]); y[5] = fma2(C32, z[7], y[5]);
    } else {                  // S: -i z, S^H: +i z
      yi[3] = add2(yi[3], z[2]); yi[2] = fma2(CN32, z[6], yi[2]); yi[3] = fma2(CNi2, z[7], yi[3]);
      yi[5] = sub2(yi[5], z[4]); yi[6] = fma2(CNi2, z[4], yi[6]); yi[7] = fma2(CN32, z[5], yi[7]);
      yi[2] = sub2(yi[2], z[3]); yi[6] = fma2(C32, z[2], yi[6]); yi[7] = fma2(Ci2, z[3], yi[7]);
      yi[4] = add2(yi[4], z[5]); yi[4] = fma2(Ci2, z[6], yi[4]); yi[5] = fma2(C32, z[7], yi[5]);
    }
  }

  // ---- Y = y + i yi -------------------------------------------------------------------
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const float2 a = f2up(y[b]), c = f2up(yi[b]);
    Y[b] = make_float2(a.x - c.y, a.y + c.x);
  }
}

// complex64 eight-band blocks take the packed form, everything else the scalar one
template <typename T, int NB, class L, class Rc>
__device__ __forceinline__ void hx_compute(const L& ld, const Rc& rc, unsigned msk, T shift,
                                           T cb, cplx<T> (&y)[8]) {
  if constexpr (std::is_same<T, float>::value && NB == 8) hx_math_packed(ld, rc, msk, shift, cb, y);
  else hx_math<T, NB>(ld, rc, msk, shift, cb, y);
}

// neighbour mask of site (ix, iy, iz): bit f (0..5) face x+, x-, y+, y-, z+, z-; bit
// 6 + 4 pl + e the in-plane edge e of plane pl (xy, zx, zy), sa = e & 1 ? -1 : 1,
// sb = e & 2 ? -1 : 1 (a = x, z, z; b = y, x, y). An edge exists when both of its faces do.
__device__ __forceinline__ unsigned site_mask(int ix, int iy, int iz, int nx, int ny, int nz) {
  const unsigned xp = ix + 1 < nx, xm = ix > 0, yp = iy + 1 < ny, ym = iy > 0;
  const unsigned zp = iz + 1 < nz, zm = iz > 0;
  unsigned m = xp | (xm << 1) | (yp << 2) | (ym << 3) | (zp << 4) | (zm << 5);
  m |= (xp & yp) << 6 | (xm & yp) << 7 | (xp & ym) << 8 | (xm & ym) << 9;      // xy
  m |= (zp & xp) << 10 | (zm & xp) << 11 | (zp & xm) << 12 | (zm & xm) << 13;  // zx
  m |= (zp & yp) << 14 | (zm & yp) << 15 | (zp & ym) << 16 | (zm & ym) << 17;  // zy
  return m;
}

// ---------------------------------------------------------------------------------------------
// Direct kernel: one thread per (site, column), neighbours read through L1/L2. Serves the six-
// and four-band slices, blocks the staged kernel cannot take, and the batched engine.
// ---------------------------------------------------------------------------------------------
template <typename T>
struct HXArgs {
  const T* __restrict__ rec;
  const unsigned* __restrict__ msk;
  const cplx<T>* __restrict__ X;
  cplx<T>* __restrict__ Y;
  int N, ldx, ldy, m, sx, sy;   // sites, leading dimensions, columns, site strides of x and y
  int nz, nzp, NP;              // z extent, its padded record extent, record entry stride
  T shift;                      // -sigma for a shifted apply, else 0
  T cb;                         // conduction-band face weight sign (-G / h^2)
};

// x[b] = X[band b, site s + offset, column j] with xs = &X[0, s, j], bs = N ldx (elements);
// every offset fits 32 bits for the grids this library accepts (n ldx < 2^31).
template <typename T, int NB>
struct GlobalLoader {
  const cplx<T>* __restrict__ xs;
  int bs, xstr[3];
  __device__ __forceinline__ void at(int off, bool vb_only, cplx<T> (&x)[8]) const {
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      if (!has_band<NB>(b) || (vb_only && b < 2)) { x[b] = czero<T>(); continue; }
      x[b] = __ldg(xs + ((b - band_off<NB>()) * bs + off));
    }
  }
  __device__ __forceinline__ void centre(cplx<T> (&x)[8]) const { at(0, false, x); }
  __device__ __forceinline__ void face(int f, cplx<T> (&x)[8]) const {
    at((f & 1) ? -xstr[f >> 1] : xstr[f >> 1], false, x);
  }
  __device__ __forceinline__ void edge(int pl, int e, cplx<T> (&x)[8]) const {
    const int ea = pl == 0 ? 0 : 2, eb = pl == 0 ? 1 : (pl == 1 ? 0 : 1);
    const int sa = (e & 1) ? -1 : 1, sb = (e & 2) ? -1 : 1;
    at(sa * xstr[ea] + sb * xstr[eb], true, x);
  }
  // packed complex64 loads (eight bands only)
  __device__ __forceinline__ void at2(int off, int b0, f2 (&x)[8]) const {
    const unsigned long long* p = reinterpret_cast<const unsigned long long*>(xs);
#pragma unroll
    for (int b = b0; b < 8; ++b) x[b] = __ldg(p + (b * bs + off));
  }
  __device__ __forceinline__ void centre2(f2 (&x)[8]) const { at2(0, 0, x); }
  __device__ __forceinline__ void face2(int f, f2 (&x)[8]) const {
    at2((f & 1) ? -xstr[f >> 1] : xstr[f >> 1], 0, x);
  }
  __device__ __forceinline__ void edge2(int pl, int e, f2 (&x)[8]) const {
    const int ea = pl == 0 ? 0 : 2, eb = pl == 0 ? 1 : (pl == 1 ? 0 : 1);
    const int sa = (e & 1) ? -1 : 1, sb = (e & 2) ? -1 : 1;
    at2(sa * xstr[ea] + sb * xstr[eb], 2, x);
  }
};

template <typename T>
struct GlobalRecord {
  const T* __restrict__ R;   // record base + padded site index
  int NP;
  __device__ __forceinline__ T own(int k) const { return __ldg(R + k * NP); }
  __device__ __forceinline__ T face(int ax, int dir, int k) const {
    return own(K_FACE + 5 * (2 * ax + dir) + k);
  }
};

template <typename T, int NB>
__device__ __forceinline__ void hx_item(const HXArgs<T>& a, int s, int j) {
  GlobalLoader<T, NB> ld;
  ld.xs = a.X + ((long long)s * a.ldx + j);
  ld.bs = a.N * a.ldx;
  ld.xstr[0] = a.sx * a.ldx; ld.xstr[1] = a.sy * a.ldx; ld.xstr[2] = a.ldx;
  GlobalRecord<T> rc;
  rc.R = a.rec + (s + (s / a.nz) * (a.nzp - a.nz));
  rc.NP = a.NP;
  cplx<T> y[8];
  hx_compute<T, NB>(ld, rc, __ldg(a.msk + s), a.shift, a.cb, y);
  cplx<T>* __restrict__ ys = a.Y + ((long long)s * a.ldy + j);
  const int ybs = a.N * a.ldy;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    if (!has_band<NB>(b)) continue;
    ys[(b - band_off<NB>()) * ybs] = y[b];
  }
}

constexpr int kApplyThreads = 256;
template <typename T> struct ApplyOcc;
template <> struct ApplyOcc<double> { static constexpr int kMinBlocks = 2; };
template <> struct ApplyOcc<float> { static constexpr int kMinBlocks = 3; };

template <typename T, int NB>
__global__ void __launch_bounds__(kApplyThreads, ApplyOcc<T>::kMinBlocks)
kp_apply_kernel(const HXArgs<T> a) {
  const int it = blockIdx.x * kApplyThreads + threadIdx.x;
  if (it >= a.N * a.m) return;
  const int s = it / a.m;
  hx_item<T, NB>(a, s, it - s * a.m);
}

// ---------------------------------------------------------------------------------------------
// Staged kernel (eight bands): a CTA owns a TY x TZ tile of (y, z) sites and MC consecutive
// columns and walks a run of x planes. A ring of four shared-memory plane buffers holds planes
// x-1, x, x+1 of the tile with a one-site halo in y and z while plane x+2 streams in with
// cp.async, so every X value crosses L2 about once (plus the halo) and the 19-point stencil reads
// come from shared memory. Smem layout of a plane: [band][y + 1][z + 1][column].
// ---------------------------------------------------------------------------------------------
template <typename T, int MC_, int TY_, int TZ_>
struct Staged {
  static constexpr int MC = MC_, TY = TY_, TZ = TZ_;
  static constexpr int PY = TY + 2, PZ = TZ + 2;
  static constexpr int BAND = PY * PZ * MC;        // complex elements per band of a plane
  static constexpr int PLANE = 8 * BAND;
  static constexpr int NSLOT = 4;
  static constexpr int RPLANE = K_COUNT * TY * TZ;   // record values of one tile plane
  static constexpr int THREADS = TY * TZ * MC;
  static constexpr size_t VEC_BYTES = (size_t)NSLOT * PLANE * sizeof(cplx<T>);
  static constexpr size_t SMEM = VEC_BYTES + (size_t)2 * RPLANE * sizeof(T);
  static_assert(TZ % 4 == 0, "record rows are copied in 16-byte z runs");
  static_assert(SMEM <= 231424, "over the opt-in shared memory of one CTA");
};

template <typename T>
struct StagedArgs {
  const T* __restrict__ rec;
  const cplx<T>* __restrict__ X;
  cplx<T>* __restrict__ Y;
  int N, nx, ny, nz, ldx, ldy, m;
  int nzp, NP;
  int tiles_z, chunks, xsplit, xlen;
  T shift, cb;
};

template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem_dst, const void* gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  if (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" :: "r"(d), "l"(gmem_src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" :: "r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <typename T, class G>
struct SmemLoader {
  const cplx<T>* p[3];   // planes x-1, x, x+1 at this thread's (y, z, column)
  __device__ __forceinline__ void at(const cplx<T>* q, int off, bool vb_only, cplx<T> (&x)[8]) const {
#pragma unroll
    for (int b = 0; b < 8; ++b) x[b] = (vb_only && b < 2) ? czero<T>() : q[b * G::BAND + off];
  }
  __device__ __forceinline__ void centre(cplx<T> (&x)[8]) const { at(p[1], 0, false, x); }
  __device__ __forceinline__ void face(int f, cplx<T> (&x)[8]) const {
    const int ax = f >> 1, sg = (f & 1) ? -1 : 1;
    if (ax == 0) at(p[1 + sg], 0, false, x);
    else if (ax == 1) at(p[1], sg * G::PZ * G::MC, false, x);
    else at(p[1], sg * G::MC, false, x);
  }
  __device__ __forceinline__ void edge(int pl, int e, cplx<T> (&x)[8]) const {
    const int sa = (e & 1) ? -1 : 1, sb = (e & 2) ? -1 : 1;
    if (pl == 0) at(p[1 + sa], sb * G::PZ * G::MC, true, x);                 // a = x, b = y
    else if (pl == 1) at(p[1 + sb], sa * G::MC, true, x);                    // a = z, b = x
    else at(p[1], sa * G::MC + sb * G::PZ * G::MC, true, x);                 // a = z, b = y
  }
  // packed complex64 loads
  __device__ __forceinline__ void at2(const cplx<T>* q, int off, int b0, f2 (&x)[8]) const {
#pragma unroll
    for (int b = b0; b < 8; ++b) x[b] = *reinterpret_cast<const f2*>(q + b * G::BAND + off);
  }
  __device__ __forceinline__ void centre2(f2 (&x)[8]) const { at2(p[1], 0, 0, x); }
  __device__ __forceinline__ void face2(int f, f2 (&x)[8]) const {
    const int ax = f >> 1, sg = (f & 1) ? -1 : 1;
    if (ax == 0) at2(p[1 + sg], 0, 0, x);
    else if (ax == 1) at2(p[1], sg * G::PZ * G::MC, 0, x);
    else at2(p[1], sg * G::MC, 0, x);
  }
  __device__ __forceinline__ void edge2(int pl, int e, f2 (&x)[8]) const {
    const int sa = (e & 1) ? -1 : 1, sb = (e & 2) ? -1 : 1;
    if (pl == 0) at2(p[1 + sa], sb * G::PZ * G::MC, 2, x);
    else if (pl == 1) at2(p[1 + sb], sa * G::MC, 2, x);
    else at2(p[1], sa * G::MC + sb * G::PZ * G::MC, 2, x);
  }
};

template <typename T, class G, bool V16>
__device__ __forceinline__ void copy_plane(const StagedArgs<T>& a, cplx<T>* slot, int xp,
                                           int y0, int z0, int c0) {
  constexpr int EPU = V16 ? (int)(16 / sizeof(cplx<T>)) : 1;   // complex elements per copy
  constexpr int UPC = G::MC / EPU;                              // copies per (band, y, z) cell
  constexpr int UNITS = 8 * G::PY * G::PZ * UPC;
  for (int u = threadIdx.x; u < UNITS; u += G::THREADS) {
    const int cu = u % UPC;
    int r = u / UPC;
    const int zz = r % G::PZ; r /= G::PZ;
    const int yy = r % G::PY;
    const int bb = r / G::PY;
    const int gy = y0 - 1 + yy, gz = z0 - 1 + zz, gc = c0 + cu * EPU;
    if (gy < 0 || gy >= a.ny || gz < 0 || gz >= a.nz || gc >= a.m) continue;
    const int site = (xp * a.ny + gy) * a.nz + gz;
    const cplx<T>* src = a.X + ((long long)(bb * a.N + site) * a.ldx + gc);
    cplx<T>* dst = slot + ((bb * G::PY + yy) * G::PZ + zz) * G::MC + cu * EPU;
    cp_async<V16 ? 16 : (int)sizeof(cplx<T>)>(dst, src);
  }
}

// The tile's records of plane xp: rows (entry k, y) of TZ values, in 16-byte runs (z0 and TZ are
// multiples of 4, nzp too, so a run never straddles the padded row end).
template <typename T, class G>
__device__ __forceinline__ void copy_record(const StagedArgs<T>& a, T* slot, int xp, int y0,
                                            int z0) {
  constexpr int EPU = (int)(16 / sizeof(T));
  constexpr int RUNS = G::TZ / EPU;
  constexpr int UNITS = K_COUNT * G::TY * RUNS;
  for (int u = threadIdx.x; u < UNITS; u += G::THREADS) {
    const int ru = u % RUNS;
    const int r = u / RUNS;
    const int ty = r % G::TY;
    const int k = r / G::TY;
    const int gy = y0 + ty, gz = z0 + ru * EPU;
    if (gy >= a.ny || gz >= a.nzp) continue;
    const T* src = a.rec + ((long long)k * a.NP + ((long long)xp * a.ny + gy) * a.nzp + gz);
    cp_async<16>(slot + (k * G::TY + ty) * G::TZ + ru * EPU, src);
  }
}

template <typename T, class G>
struct SmemRecord {
  const T* r;     // record slot + ty * TZ + tz
  __device__ __forceinline__ T own(int k) const { return r[k * G::TY * G::TZ]; }
  __device__ __forceinline__ T face(int ax, int dir, int k) const {
    return own(K_FACE + 5 * (2 * ax + dir) + k);
  }
};

template <typename T, class G, bool V16>
__global__ void __launch_bounds__(G::THREADS, 1) kp_apply_staged_kernel(const StagedArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* ring = reinterpret_cast<cplx<T>*>(smem_raw);
  T* rring = reinterpret_cast<T*>(smem_raw + G::VEC_BYTES);
  int bid = blockIdx.x;
  const int xs = bid % a.xsplit; bid /= a.xsplit;
  const int ch = bid % a.chunks; bid /= a.chunks;
  const int tzi = bid % a.tiles_z;
  const int tyi = bid / a.tiles_z;
  const int c0 = ch * G::MC, y0 = tyi * G::TY, z0 = tzi * G::TZ;
  const int xa = xs * a.xlen, xb = min(a.nx, xa + a.xlen);
  if (c0 >= a.m || xa >= xb) return;          // uniform over the CTA
  const int t = threadIdx.x;
  const int c = t % G::MC, tz = (t / G::MC) % G::TZ, ty = t / (G::MC * G::TZ);
  const int iy = y0 + ty, iz = z0 + tz, col = c0 + c;
  const bool active = iy < a.ny && iz < a.nz && col < a.m;
  const int cell = ((ty + 1) * G::PZ + (tz + 1)) * G::MC + c;

  if (xa > 0) copy_plane<T, G, V16>(a, ring + ((xa - 1) & 3) * G::PLANE, xa - 1, y0, z0, c0);
  cp_async_commit();
  copy_plane<T, G, V16>(a, ring + (xa & 3) * G::PLANE, xa, y0, z0, c0);
  copy_record<T, G>(a, rring + (xa & 1) * G::RPLANE, xa, y0, z0);
  cp_async_commit();
  if (xa + 1 < a.nx) copy_plane<T, G, V16>(a, ring + ((xa + 1) & 3) * G::PLANE, xa + 1, y0, z0, c0);
  cp_async_commit();
  for (int x = xa; x < xb; ++x) {
    cp_async_wait_all();
    __syncthreads();                          // planes x-1..x+1 landed; slot (x+2) & 3 is free
    if (x + 2 <= xb && x + 2 < a.nx)
      copy_plane<T, G, V16>(a, ring + ((x + 2) & 3) * G::PLANE, x + 2, y0, z0, c0);
    if (x + 1 < xb) copy_record<T, G>(a, rring + ((x + 1) & 1) * G::RPLANE, x + 1, y0, z0);
    cp_async_commit();
    if (!active) continue;
    SmemLoader<T, G> ld;
    ld.p[0] = ring + ((x + 3) & 3) * G::PLANE + cell;
    ld.p[1] = ring + (x & 3) * G::PLANE + cell;
    ld.p[2] = ring + ((x + 1) & 3) * G::PLANE + cell;
    const int s = (x * a.ny + iy) * a.nz + iz;
    SmemRecord<T, G> rc;
    rc.r = rring + (x & 1) * G::RPLANE + ty * G::TZ + tz;
    cplx<T> y[8];
    hx_compute<T, 8>(ld, rc, site_mask(x, iy, iz, a.nx, a.ny, a.nz), a.shift, a.cb, y);
    cplx<T>* __restrict__ ys = a.Y + ((long long)s * a.ldy + col);
    const int ybs = a.N * a.ldy;
#pragma unroll
    for (int b = 0; b < 8; ++b) ys[b * ybs] = y[b];
  }
  cp_async_wait_all();
}

// ---------------------------------------------------------------------------------------------
// TMA kernel (eight bands, complex64). The same x walk as the staged kernel, with three changes:
//   * the planes and the record rows are brought in by the tensor-memory accelerator
//     (cp.async.bulk.tensor, one elected thread, completion on an mbarrier per ring slot) from
//     tensor maps over this GPU's X and record; coordinates outside the grid (the halo at a wall,
//     planes -1 and nx) read as zeros, so no thread computes an address or a neighbour mask:
//     every weight a missing neighbour would need is zero in the record anyway;
//   * every thread owns one site and two adjacent columns: each coefficient broadcast and record
//     read serves both, and a band of both columns is one 16-byte shared load;
//   * a ring of NSLOT planes keeps NSLOT - 3 planes in flight ahead of the compute.
// Smem of a plane as the TMA box lands it: [band][y + 1][z + 1][column] (MC columns).
// ---------------------------------------------------------------------------------------------
template <int C, class L, class Rc>
__device__ __forceinline__ void hx_packed_cols(const L& ld, const Rc& rc, float shift, float cb,
                                               float2 (&Y)[C][8]) {
  const float sq2 = 1.41421356237309504880f, sq3 = 1.73205080756887729353f;
  const float sq32 = 1.22474487139158904910f, isq2 = 0.70710678118654752440f;
  const f2 C2 = f2bc(sq2), CN2 = f2bc(-sq2), C3 = f2bc(sq3), C32 = f2bc(sq32);
  const f2 CN32 = f2bc(-sq32), Ci2 = f2bc(isq2), CNi2 = f2bc(-isq2), CN1 = f2bc(-1.f);
  const f2 CB = f2bc(cb);
  f2 y[C][8], yi[C][8], x[C][8];

  // ---- local block, the shift -sigma folded into the diagonal ---------------------------
  ld.centre(x);
  {
    const float Rr = rc.own(K_RRE), Ri = rc.own(K_RIM), Sr = rc.own(K_SRE), Si = rc.own(K_SIM);
    const float q2 = rc.own(K_Q2);
    const f2 PA = f2bc(rc.own(K_A) + shift), P2 = f2bc(rc.own(K_A2) + shift);
    const f2 P3 = f2bc(rc.own(K_A3) + shift), P6 = f2bc(rc.own(K_A6) + shift);
    const f2 Q2 = f2bc(q2), NQ2 = f2bc(-q2);
    const f2 SR = f2bc(Sr), NSR = f2bc(-Sr), SI = f2bc(Si), NSI = f2bc(-Si);
    const f2 RR = f2bc(Rr), RI = f2bc(Ri), NRI = f2bc(-Ri);
    const f2 S32R = f2bc(sq32 * Sr), S32I = f2bc(sq32 * Si), NS32I = f2bc(-sq32 * Si);
    const f2 R2R = f2bc(sq2 * Rr), NR2R = f2bc(-sq2 * Rr), R2I = f2bc(sq2 * Ri);
    const f2 NR2I = f2bc(-sq2 * Ri);
    const f2 SI2R = f2bc(isq2 * Sr), SI2I = f2bc(isq2 * Si), NSI2I = f2bc(-isq2 * Si);
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const f2* xc = x[c];
      f2* yc = y[c];
      f2* ic = yi[c];
      yc[0] = mul2(PA, xc[0]); yc[1] = mul2(PA, xc[1]);
      ic[0] = 0ull; ic[1] = 0ull;
      yc[2] = fma2(NSR, xc[3], mul2(P2, xc[2]));   ic[2] = mul2(SI, xc[3]);
      yc[2] = fma2(RR, xc[4], yc[2]);              ic[2] = fma2(RI, xc[4], ic[2]);
      yc[2] = fma2(S32R, xc[6], yc[2]);            ic[2] = fma2(S32I, xc[6], ic[2]);
      yc[2] = fma2(NQ2, xc[7], yc[2]);
      yc[3] = fma2(NSR, xc[2], mul2(P3, xc[3]));   ic[3] = mul2(NSI, xc[2]);
      yc[3] = fma2(RR, xc[5], yc[3]);              ic[3] = fma2(RI, xc[5], ic[3]);
      yc[3] = fma2(NR2R, xc[6], yc[3]);            ic[3] = fma2(NR2I, xc[6], ic[3]);
      yc[3] = fma2(SI2R, xc[7], yc[3]);            ic[3] = fma2(SI2I, xc[7], ic[3]);
      yc[4] = fma2(RR, xc[2], mul2(P3, xc[4]));    ic[4] = mul2(NRI, xc[2]);
      yc[4] = fma2(SR, xc[5], yc[4]);              ic[4] = fma2(NSI, xc[5], ic[4]);
      yc[4] = fma2(SI2R, xc[6], yc[4]);            ic[4] = fma2(NSI2I, xc[6], ic[4]);
      yc[4] = fma2(R2R, xc[7], yc[4]);             ic[4] = fma2(NR2I, xc[7], ic[4]);
      yc[5] = fma2(RR, xc[3], mul2(P2, xc[5]));    ic[5] = mul2(NRI, xc[3]);
      yc[5] = fma2(SR, xc[4], yc[5]);              ic[5] = fma2(SI, xc[4], ic[5]);
      yc[5] = fma2(Q2, xc[6], yc[5]);
      yc[5] = fma2(S32R, xc[7], yc[5]);            ic[5] = fma2(NS32I, xc[7], ic[5]);
      yc[6] = fma2(S32R, xc[2], mul2(P6, xc[6]));  ic[6] = mul2(NS32I, xc[2]);
      yc[6] = fma2(NR2R, xc[3], yc[6]);            ic[6] = fma2(R2I, xc[3], ic[6]);
      yc[6] = fma2(SI2R, xc[4], yc[6]);            ic[6] = fma2(SI2I, xc[4], ic[6]);
      yc[6] = fma2(Q2, xc[5], yc[6]);
      yc[7] = fma2(NQ2, xc[2], mul2(P6, xc[7]));
      yc[7] = fma2(SI2R, xc[3], yc[7]);            ic[7] = mul2(NSI2I, xc[3]);
      yc[7] = fma2(R2R, xc[4], yc[7]);             ic[7] = fma2(R2I, xc[4], ic[7]);
      yc[7] = fma2(S32R, xc[5], yc[7]);            ic[7] = fma2(S32I, xc[5], ic[7]);
    }
  }

  // ---- six face neighbours (a missing neighbour reads as zero, its weights are zero) ----
#pragma unroll
  for (int f = 0; f < 6; ++f) {
    const int ax = f >> 1, dir = f & 1;
    ld.face(f, x);
    const float kp = rc.face(ax, dir, 0), k2 = rc.face(ax, dir, 1);
    const float kq = (ax == 2 ? -2.f : 1.f) * k2;
    const f2 KPQ = f2bc(kq - kp), NKPQ = f2bc(-kp - kq), NKP = f2bc(-kp);
    const f2 K2Q = f2bc(sq2 * kq), NK2Q = f2bc(-sq2 * kq);
    const float kr = (ax == 0 ? -sq3 : sq3) * k2;
    const f2 KR = f2bc(kr), K2R = f2bc(sq2 * kr), NK2R = f2bc(-sq2 * kr);
    const float su = rc.face(ax, dir, 2), svr = rc.face(ax, dir, 3), svi = rc.face(ax, dir, 4);
    const f2 SVI = f2bc(svi), SVR = f2bc(svr), SU = f2bc(su), NSVR = f2bc(-svr), NSU = f2bc(-su);
    const f2 S2SU = f2bc(sq2 * su), N3SVI = f2bc(-sq3 * svi), S3SVR = f2bc(sq3 * svr);
    const f2 N3SVR = f2bc(-sq3 * svr), N2SVI = f2bc(-sq2 * svi), N2SVR = f2bc(-sq2 * svr);
    const f2 S2SVI = f2bc(sq2 * svi);
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const f2* xc = x[c];
      f2* yc = y[c];
      f2* ic = yi[c];
      yc[0] = fma2(CB, xc[0], yc[0]); yc[1] = fma2(CB, xc[1], yc[1]);
      yc[2] = fma2(KPQ, xc[2], yc[2]); yc[2] = fma2(NK2Q, xc[7], yc[2]);
      yc[3] = fma2(NKPQ, xc[3], yc[3]);
      yc[4] = fma2(NKPQ, xc[4], yc[4]);
      yc[5] = fma2(KPQ, xc[5], yc[5]); yc[5] = fma2(K2Q, xc[6], yc[5]);
      yc[6] = fma2(NKP, xc[6], yc[6]); yc[6] = fma2(K2Q, xc[5], yc[6]);
      yc[7] = fma2(NKP, xc[7], yc[7]); yc[7] = fma2(NK2Q, xc[2], yc[7]);
      if (ax < 2) {
        yc[2] = fma2(KR, xc[4], yc[2]);
        yc[3] = fma2(KR, xc[5], yc[3]); yc[3] = fma2(NK2R, xc[6], yc[3]);
        yc[4] = fma2(KR, xc[2], yc[4]); yc[4] = fma2(K2R, xc[7], yc[4]);
        yc[5] = fma2(KR, xc[3], yc[5]);
        yc[6] = fma2(NK2R, xc[3], yc[6]);
        yc[7] = fma2(K2R, xc[4], yc[7]);
      }
      {
        const f2 t = fma2(C2, xc[7], xc[2]);        // x2 + sqrt2 x7
        const f2 u = mul2(C3, xc[4]);               // sqrt3 x4
        yc[0] = fma2(SVI, sub2(u, t), yc[0]);
        ic[0] = fma2(NSVR, add2(u, t), ic[0]);
        ic[0] = fma2(SU, fma2(C2, xc[5], xc[6]), ic[0]);
        const f2 v = mul2(C3, xc[3]);               // sqrt3 x3
        const f2 w = fma2(CN2, xc[6], xc[5]);       // x5 - sqrt2 x6
        yc[1] = fma2(SVI, sub2(v, w), yc[1]);
        ic[1] = fma2(SVR, add2(v, w), ic[1]);
        ic[1] = fma2(SU, fma2(C2, xc[2], mul2(CN1, xc[7])), ic[1]);
      }
      yc[2] = fma2(SVI, xc[0], yc[2]);   ic[2] = fma2(NSVR, xc[0], ic[2]); ic[2] = fma2(S2SU, xc[1], ic[2]);
      yc[3] = fma2(N3SVI, xc[1], yc[3]); ic[3] = fma2(S3SVR, xc[1], ic[3]);
      yc[4] = fma2(N3SVI, xc[0], yc[4]); ic[4] = fma2(N3SVR, xc[0], ic[4]);
      yc[5] = fma2(SVI, xc[1], yc[5]);   ic[5] = fma2(S2SU, xc[0], ic[5]); ic[5] = fma2(SVR, xc[1], ic[5]);
      yc[6] = fma2(N2SVI, xc[1], yc[6]); ic[6] = fma2(N2SVR, xc[1], ic[6]); ic[6] = fma2(SU, xc[0], ic[6]);
      yc[7] = fma2(S2SVI, xc[0], yc[7]); ic[7] = fma2(N2SVR, xc[0], ic[7]); ic[7] = fma2(NSU, xc[1], ic[7]);
    }
  }

  // ---- twelve edge neighbours: z = sum_e c_e x_e, then the plane's band mixing ---------
#pragma unroll
  for (int pl = 0; pl < 3; ++pl) {
    f2 z[C][8];
#pragma unroll
    for (int c = 0; c < C; ++c)
#pragma unroll
      for (int b = 2; b < 8; ++b) z[c][b] = 0ull;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      ld.edge(pl, e, x);
      const f2 W = f2bc(rc.own(K_EDGE + 4 * pl + e));
#pragma unroll
      for (int c = 0; c < C; ++c)
#pragma unroll
        for (int b = 2; b < 8; ++b) z[c][b] = fma2(W, x[c][b], z[c][b]);
    }
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const f2* zc = z[c];
      f2* yc = y[c];
      f2* ic = yi[c];
      if (pl == 0) {            // R: +i z, R^H: -i z
        ic[2] = add2(ic[2], zc[4]); ic[4] = sub2(ic[4], zc[2]);
        ic[3] = add2(ic[3], zc[5]); ic[5] = sub2(ic[5], zc[3]);
        ic[3] = fma2(CN2, zc[6], ic[3]); ic[6] = fma2(C2, zc[3], ic[6]);
        ic[4] = fma2(CN2, zc[7], ic[4]); ic[7] = fma2(C2, zc[4], ic[7]);
      } else if (pl == 1) {     // S, S^H: z
        yc[3] = sub2(yc[3], zc[2]); yc[2] = fma2(C32, zc[6], yc[2]); yc[3] = fma2(Ci2, zc[7], yc[3]);
        yc[5] = add2(yc[5], zc[4]); yc[6] = fma2(Ci2, zc[4], yc[6]); yc[7] = fma2(C32, zc[5], yc[7]);
        yc[2] = sub2(yc[2], zc[3]); yc[6] = fma2(C32, zc[2], yc[6]); yc[7] = fma2(Ci2, zc[3], yc[7]);
        yc[4] = add2(yc[4], zc[5]); yc[4] = fma2(Ci2, zc[6], yc[4]); yc[5] = fma2(C32, zc[7], yc[5]);
      } else {                  // S: -i z, S^H: +i z
        ic[3] = add2(ic[3], zc[2]); ic[2] = fma2(CN32, zc[6], ic[2]); ic[3] = fma2(CNi2, zc[7], ic[3]);
        ic[5] = sub2(ic[5], zc[4]); ic[6] = fma2(CNi2, zc[4], ic[6]); ic[7] = fma2(CN32, zc[5], ic[7]);
        ic[2] = sub2(ic[2], zc[3]); ic[6] = fma2(C32, zc[2], ic[6]); ic[7] = fma2(Ci2, zc[3], ic[7]);
        ic[4] = add2(ic[4], zc[5]); ic[4] = fma2(Ci2, zc[6], ic[4]); ic[5] = fma2(C32, zc[7], ic[5]);
      }
    }
  }

  // ---- Y = y + i yi -------------------------------------------------------------------
#pragma unroll
  for (int c = 0; c < C; ++c)
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const float2 a = f2up(y[c][b]), d = f2up(yi[c][b]);
      Y[c][b] = make_float2(a.x - d.y, a.y + d.x);
    }
}

// Two adjacent complex64 columns of one site from global memory, eight bands, for
// hx_packed_cols: a band of both columns is one 16-byte load. A neighbour outside the grid reads
// the site itself instead: its weight in the record is zero, so it adds nothing.
struct GlobalPairLoader {
  const unsigned long long* __restrict__ xs;   // &X[0, s, j], j even
  long long bs;                                // band stride N ldx (complex values)
  int xstr[3];                                 // site strides of x, y, z (complex values)
  unsigned msk;                                // neighbour mask of the site (site_mask)
  __device__ __forceinline__ void at(int off, int b0, f2 (&x)[2][8]) const {
#pragma unroll
    for (int b = b0; b < 8; ++b) {
      const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(xs + (b * bs + off)));
      x[0][b] = v.x;
      x[1][b] = v.y;
    }
  }
  __device__ __forceinline__ void centre(f2 (&x)[2][8]) const { at(0, 0, x); }
  __device__ __forceinline__ void face(int f, f2 (&x)[2][8]) const {
    const int off = (f & 1) ? -xstr[f >> 1] : xstr[f >> 1];
    at(((msk >> f) & 1u) ? off : 0, 0, x);
  }
  __device__ __forceinline__ void edge(int pl, int e, f2 (&x)[2][8]) const {
    const int ea = pl == 0 ? 0 : 2, eb = pl == 0 ? 1 : (pl == 1 ? 0 : 1);
    const int sa = (e & 1) ? -1 : 1, sb = (e & 2) ? -1 : 1;
    const int off = sa * xstr[ea] + sb * xstr[eb];
    at(((msk >> (6 + 4 * pl + e)) & 1u) ? off : 0, 2, x);
  }
};

// complex64, eight bands: columns j, j + 1 of site s (m, ldx and ldy even, X and Y 16-byte
// aligned)
__device__ __forceinline__ void hx_item_pair(const HXArgs<float>& a, int s, int j) {
  GlobalPairLoader ld;
  ld.xs = reinterpret_cast<const unsigned long long*>(a.X + ((long long)s * a.ldx + j));
  ld.bs = (long long)a.N * a.ldx;
  ld.xstr[0] = a.sx * a.ldx; ld.xstr[1] = a.sy * a.ldx; ld.xstr[2] = a.ldx;
  ld.msk = __ldg(a.msk + s);
  GlobalRecord<float> rc;
  rc.R = a.rec + (s + (s / a.nz) * (a.nzp - a.nz));
  rc.NP = a.NP;
  float2 y[2][8];
  hx_packed_cols<2>(ld, rc, a.shift, a.cb, y);
  float2* __restrict__ ys = a.Y + ((long long)s * a.ldy + j);
  const long long ybs = (long long)a.N * a.ldy;
#pragma unroll
  for (int b = 0; b < 8; ++b)
    *reinterpret_cast<float4*>(ys + b * ybs) = make_float4(y[0][b].x, y[0][b].y, y[1][b].x, y[1][b].y);
}

// Many operators and blocks in one launch (the batched engine): CTA b serves slot k with
// tile0[k] <= b < tile0[k+1]; the column count is read on the device (the slot's active width).
template <typename T>
__global__ void __launch_bounds__(kApplyThreads, 2)
kp_apply_multi_kernel(const HXSlot* __restrict__ slots, int nslots) {
  int k = 0;
  while (k + 1 < nslots && (int)blockIdx.x >= slots[k + 1].tile0) ++k;
  const HXSlot& d = slots[k];
  if (d.skip && *d.skip) return;
  const int m = d.m_dev ? *d.m_dev : d.m;
  const int it = (blockIdx.x - d.tile0) * kApplyThreads + threadIdx.x;
  if (m <= 0 || it >= d.N * m) return;
  HXArgs<T> a;
  a.rec = static_cast<const T*>(d.rec);
  a.msk = d.msk;
  a.X = static_cast<const cplx<T>*>(d.X);
  a.Y = static_cast<cplx<T>*>(d.Y);
  a.N = d.N; a.ldx = d.ld_same ? m : d.ldx; a.ldy = d.ld_same ? m : d.ldy;
  a.m = m; a.sx = d.sx; a.sy = d.sy;
  a.nz = d.sy; a.nzp = d.nzp; a.NP = d.NP;
  a.shift = d.shifted ? (T)(-d.sigma) : T(0);
  a.cb = (T)d.cb;
  if constexpr (std::is_same<T, float>::value) {
    // complex64: two columns per thread where the widths and pointers allow 16-byte words (the
    // slot's CTAs past the pairs' count exit)
    if (((m | a.ldx | a.ldy) & 1) == 0 &&
        ((reinterpret_cast<uintptr_t>(a.X) | reinterpret_cast<uintptr_t>(a.Y)) & 15) == 0) {
      const int mp = m >> 1;
      if (it >= d.N * mp) return;
      const int s = it / mp;
      hx_item_pair(a, s, 2 * (it - s * mp));
      return;
    }
  }
  const int s = it / m;
  hx_item<T, 8>(a, s, it - s * m);
}


// mbarrier and bulk-tensor copy primitives (PTX ISA: mbarrier, cp.async.bulk.tensor)
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
               " selp.b32 %0, 1, 0, p;\n}\n" : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
  return ok != 0;
}
// Bounded wait: gives up after about a second of SM clocks (a copy that never lands).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > 2000000000LL) return false;
  return true;
}
__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int c0, int c1, int c2, int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];"
      :: "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2),
         "r"(c3), "r"(c4) : "memory");
}
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, uint32_t bar,
                                            int c0, int c1, int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6}], [%2];"
      :: "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2),
         "r"(c3) : "memory");
}

struct RegRecord {                 // a site's record row in registers
  float v[K_COUNT];
  __device__ __forceinline__ float own(int k) const { return v[k]; }
  __device__ __forceinline__ float face(int ax, int dir, int k) const {
    return v[K_FACE + 5 * (2 * ax + dir) + k];
  }
};

// Set by a TMA kernel whose wait on a copy gave up (qdkp_device_fault reads and clears it).
__device__ int g_apply_fault;

// RREG: the record row of each site is prefetched by its threads into registers one plane ahead
// (no record slots in shared memory, which leaves room for larger tiles)
template <int TY_, int TZ_, int G_, int NSLOT_, int MINB_ = 1, bool RREG_ = false>
struct Tma {
  static constexpr int TY = TY_, TZ = TZ_, G = G_, NSLOT = NSLOT_, MINB = MINB_;
  static constexpr bool RREG = RREG_;
  static constexpr int CPT = 2;                          // columns per thread
  static constexpr int MC = CPT * G;                     // columns per CTA
  static constexpr int PY = TY + 2, PZ = TZ + 2;
  static constexpr int BAND = PY * PZ * MC;              // complex64 elements per band of a plane
  static constexpr int PLANE_BYTES = 8 * BAND * 8;
  static constexpr int RPLANE_BYTES = K_COUNT * TY * TZ * 4;
  static constexpr int RSTRIDE = (RPLANE_BYTES + 127) / 128 * 128;
  static constexpr int THREADS = TY * TZ * G;
  static constexpr int BARS = NSLOT + (RREG ? 0 : 2);
  static constexpr size_t SMEM = 1024 + (size_t)NSLOT * PLANE_BYTES + (RREG ? 0 : 2 * RSTRIDE) +
                                 8 * BARS;
  static_assert(TZ % 4 == 0, "record rows are copied in 16-byte z runs");
  static_assert(PLANE_BYTES % 128 == 0, "ring slots stay 128-byte aligned");
  static_assert(NSLOT >= 4, "planes x-1, x, x+1 and at least one in flight");
  static_assert(SMEM * MINB <= 232448, "over the shared memory of one SM");
};

struct TmaArgs {
  float2* __restrict__ Y;
  const float* __restrict__ rec;   // the FP32 record (read directly by RREG shapes)
  int nzp, NP;
  int N, nx, ny, nz, ldy, m;
  int tiles_z, chunks, xsplit, xlen;
  int vec_store;          // Y is 16-byte aligned with an even leading dimension
  float shift, cb;
};

template <class G>
struct TmaLoader {
  const unsigned long long* p[3];   // planes x-1, x, x+1 at this thread's (y, z, column pair)
  __device__ __forceinline__ void at(const unsigned long long* q, int off, int b0,
                                     f2 (&x)[2][8]) const {
#pragma unroll
    for (int b = b0; b < 8; ++b) {
      const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(q + b * G::BAND + off);
      x[0][b] = v.x;
      x[1][b] = v.y;
    }
  }
  __device__ __forceinline__ void centre(f2 (&x)[2][8]) const { at(p[1], 0, 0, x); }
  __device__ __forceinline__ void face(int f, f2 (&x)[2][8]) const {
    const int ax = f >> 1, sg = (f & 1) ? -1 : 1;
    if (ax == 0) at(p[1 + sg], 0, 0, x);
    else if (ax == 1) at(p[1], sg * G::PZ * G::MC, 0, x);
    else at(p[1], sg * G::MC, 0, x);
  }
  __device__ __forceinline__ void edge(int pl, int e, f2 (&x)[2][8]) const {
    const int sa = (e & 1) ? -1 : 1, sb = (e & 2) ? -1 : 1;
    if (pl == 0) at(p[1 + sa], sb * G::PZ * G::MC, 2, x);                 // a = x, b = y
    else if (pl == 1) at(p[1 + sb], sa * G::MC, 2, x);                    // a = z, b = x
    else at(p[1], sa * G::MC + sb * G::PZ * G::MC, 2, x);                 // a = z, b = y
  }
};

template <class G>
__global__ void __launch_bounds__(G::THREADS, G::MINB)
kp_apply_tma_kernel(const __grid_constant__ CUtensorMap tmx, const __grid_constant__ CUtensorMap tmr,
                    const TmaArgs a) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t pad = ((raw + 1023u) & ~1023u) - raw;
  unsigned char* sb = smem_raw + pad;
  const uint32_t ring = raw + pad;
  const uint32_t rring = ring + G::NSLOT * G::PLANE_BYTES;
  // NSLOT plane barriers, then 2 record ones (staged records only)
  const uint32_t bars = rring + (G::RREG ? 0 : 2 * G::RSTRIDE);
  int bid = blockIdx.x;
  const int xs = bid % a.xsplit; bid /= a.xsplit;
  const int ch = bid % a.chunks; bid /= a.chunks;
  const int tzi = bid % a.tiles_z;
  const int tyi = bid / a.tiles_z;
  const int c0 = ch * G::MC, y0 = tyi * G::TY, z0 = tzi * G::TZ;
  const int xa = xs * a.xlen, xb = min(a.nx, xa + a.xlen);
  if (c0 >= a.m || xa >= xb) return;          // uniform over the CTA
  const int t = threadIdx.x;
  const int g = t % G::G, tz = (t / G::G) % G::TZ, ty = t / (G::G * G::TZ);
  const int iy = y0 + ty, iz = z0 + tz, col = c0 + g * G::CPT;
  const bool active = iy < a.ny && iz < a.nz && col < a.m;
  const int cell = ((ty + 1) * G::PZ + (tz + 1)) * G::MC + g * G::CPT;

  // plane with sequence number q (plane index xa - 1 + q) lives in slot q % NSLOT, and its
  // barrier completes phase q / NSLOT; the record of plane xa + r in slot r & 1, phase r >> 1
  auto plane_bar = [&](int q) { return bars + 8u * (uint32_t)(q % G::NSLOT); };
  auto rec_bar = [&](int r) { return bars + 8u * (uint32_t)(G::NSLOT + (r & 1)); };
  auto issue_plane = [&](int q) {
    const uint32_t bar = plane_bar(q);
    mbar_expect_tx(bar, G::PLANE_BYTES);
    tma_load_5d(ring + (uint32_t)(q % G::NSLOT) * G::PLANE_BYTES, &tmx, bar, c0, z0 - 1, y0 - 1,
                xa - 1 + q, 0);
  };
  auto issue_record = [&](int r) {
    const uint32_t bar = rec_bar(r);
    mbar_expect_tx(bar, G::RPLANE_BYTES);
    tma_load_4d(rring + (uint32_t)(r & 1) * G::RSTRIDE, &tmr, bar, z0, y0, xa + r, 0);
  };

  if (t == 0) {
    for (int i = 0; i < G::BARS; ++i) mbar_init(bars + 8u * i, 1);
    mbar_fence_init();
  }
  __syncthreads();
  const int nplanes = xb - xa + 2;            // planes xa - 1 .. xb
  int q_issued = 0, r_issued = 0;
  if (t == 0) {
    for (; q_issued < G::NSLOT - 1 && q_issued < nplanes; ++q_issued) issue_plane(q_issued);
    if (!G::RREG) issue_record(r_issued++);
  }
  // RREG: this thread's record row of plane x, and the one of plane x + 1 in flight
  RegRecord rcur, rnxt;
  const long long rsite = (long long)iy * a.nzp + iz;
  if (G::RREG && active) {
    const float* rp = a.rec + (long long)xa * a.ny * a.nzp + rsite;
#pragma unroll
    for (int k = 0; k < K_COUNT; ++k) rcur.v[k] = __ldg(rp + (long long)k * a.NP);
  }
  bool ok = true;
  for (int x = xa; x < xb; ++x) {
    const int qx = x - xa + 1;
    ok = ok && mbar_wait(plane_bar(qx - 1), ((qx - 1) / G::NSLOT) & 1) &&
         mbar_wait(plane_bar(qx), (qx / G::NSLOT) & 1) &&
         mbar_wait(plane_bar(qx + 1), ((qx + 1) / G::NSLOT) & 1);
    // every thread is past plane x - 1: its ring slot and record slot may be refilled
    const bool all_ok = __syncthreads_and(ok) != 0;
    if (t == 0 && all_ok) {
      if (q_issued < nplanes) issue_plane(q_issued++);
      if (!G::RREG && x + 1 < xb) issue_record(r_issued++);
    }
    const int r = x - xa;
    if (G::RREG) ok = all_ok;
    else ok = all_ok && mbar_wait(rec_bar(r), (r >> 1) & 1);
    if (!ok || !active) continue;
    if (G::RREG && x + 1 < xb) {                // prefetch plane x + 1's record row
      const float* rp = a.rec + (long long)(x + 1) * a.ny * a.nzp + rsite;
#pragma unroll
      for (int k = 0; k < K_COUNT; ++k) rnxt.v[k] = __ldg(rp + (long long)k * a.NP);
    }
    TmaLoader<G> ld;
    const unsigned long long* pl = reinterpret_cast<const unsigned long long*>(sb);
    ld.p[0] = pl + (size_t)((qx - 1) % G::NSLOT) * (G::PLANE_BYTES / 8) + cell;
    ld.p[1] = pl + (size_t)(qx % G::NSLOT) * (G::PLANE_BYTES / 8) + cell;
    ld.p[2] = pl + (size_t)((qx + 1) % G::NSLOT) * (G::PLANE_BYTES / 8) + cell;
    float2 yv[2][8];
    if constexpr (G::RREG) {
      hx_packed_cols<2>(ld, rcur, a.shift, a.cb, yv);
#pragma unroll
      for (int k = 0; k < K_COUNT; ++k) rcur.v[k] = rnxt.v[k];
    } else {
      SmemRecord<float, G> rc;                  // record slot layout [k][ty][tz]
      rc.r = reinterpret_cast<const float*>(sb + G::NSLOT * G::PLANE_BYTES + (r & 1) * G::RSTRIDE) +
             ty * G::TZ + tz;
      hx_packed_cols<2>(ld, rc, a.shift, a.cb, yv);
    }
    const int s = (x * a.ny + iy) * a.nz + iz;
    float2* __restrict__ ys = a.Y + ((long long)s * a.ldy + col);
    const long long ybs = (long long)a.N * a.ldy;
    if (a.vec_store && col + 1 < a.m) {
#pragma unroll
      for (int b = 0; b < 8; ++b)
        *reinterpret_cast<float4*>(ys + b * ybs) = make_float4(yv[0][b].x, yv[0][b].y,
                                                               yv[1][b].x, yv[1][b].y);
    } else {
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        ys[b * ybs] = yv[0][b];
        if (col + 1 < a.m) ys[b * ybs + 1] = yv[1][b];
      }
    }
  }
  if (__syncthreads_or(!ok) && t == 0) {
    // a copy never landed: flag it, then give the copies still in flight a bounded chance to
    // finish before the CTA's shared memory is released (thread 0 keeps the CTA resident)
    atomicExch(&g_apply_fault, 1);
    for (int q = max(0, q_issued - G::NSLOT); q < q_issued; ++q)
      mbar_wait(plane_bar(q), (q / G::NSLOT) & 1);
    for (int r = max(0, r_issued - 2); r < r_issued; ++r) mbar_wait(rec_bar(r), (r >> 1) & 1);
  }
}

// ---------------------------------------------------------------------------------------------
// TMA kernel with a producer warp (eight bands, complex64). The ring of NSLOT planes is filled
// by one producer warp; every ring slot has a "full" barrier (the copy landed) and an "empty"
// barrier (every compute warp is done with the plane), so compute warps never meet at a CTA-wide
// barrier: a warp moves on to plane x + 1 as soon as that plane has landed, and releases plane
// x - 1 when it finishes x. Each site's record row is read by its own threads straight from
// global memory (a record entry is used by the two threads of its site only), which leaves the
// shared memory to the plane ring: larger tiles, or two CTAs per SM.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(bar) : "memory");
}

template <int TY_, int TZ_, int G_, int NSLOT_, int MINB_>
struct Tma2 {
  static constexpr int TY = TY_, TZ = TZ_, G = G_, NSLOT = NSLOT_, MINB = MINB_;
  static constexpr int CPT = 2;
  static constexpr int MC = CPT * G;
  static constexpr int PY = TY + 2, PZ = TZ + 2;
  static constexpr int BAND = PY * PZ * MC;
  static constexpr int PLANE_BYTES = 8 * BAND * 8;
  static constexpr int CTHREADS = TY * TZ * G;            // compute threads
  static constexpr int CWARPS = CTHREADS / 32;
  static constexpr int THREADS = CTHREADS + 32;           // + the producer warp
  static constexpr size_t SMEM = 1024 + (size_t)NSLOT * PLANE_BYTES + 16 * NSLOT;
  static_assert(CTHREADS % 32 == 0, "compute threads fill whole warps");
  static_assert(PLANE_BYTES % 128 == 0, "ring slots stay 128-byte aligned");
  static_assert(NSLOT >= 4, "planes x-1, x, x+1 and at least one in flight");
  static_assert(SMEM * MINB <= 232448, "over the shared memory of one SM");
};


struct Tma2Args {
  float2* __restrict__ Y;
  const float* __restrict__ rec;
  int N, nx, ny, nz, nzp, NP, ldy, m;
  int tiles_z, chunks, xsplit, xlen;
  int vec_store;
  float shift, cb;
};

template <class G>
__global__ void __launch_bounds__(G::THREADS, G::MINB)
kp_apply_tma2_kernel(const __grid_constant__ CUtensorMap tmx, const Tma2Args a) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t pad = ((raw + 1023u) & ~1023u) - raw;
  unsigned char* sb = smem_raw + pad;
  const uint32_t ring = raw + pad;
  const uint32_t full = ring + G::NSLOT * G::PLANE_BYTES;        // NSLOT barriers
  const uint32_t empty = full + 8 * G::NSLOT;                     // NSLOT barriers
  int bid = blockIdx.x;
  const int xs = bid % a.xsplit; bid /= a.xsplit;
  const int ch = bid % a.chunks; bid /= a.chunks;
  const int tzi = bid % a.tiles_z;
  const int tyi = bid / a.tiles_z;
  const int c0 = ch * G::MC, y0 = tyi * G::TY, z0 = tzi * G::TZ;
  const int xa = xs * a.xlen, xb = min(a.nx, xa + a.xlen);
  if (c0 >= a.m || xa >= xb) return;          // uniform over the CTA
  const int t = threadIdx.x;
  if (t == 0) {
    for (int i = 0; i < G::NSLOT; ++i) {
      mbar_init(full + 8u * i, 1);
      mbar_init(empty + 8u * i, G::CWARPS);
    }
    mbar_fence_init();
  }
  __syncthreads();
  const int nplanes = xb - xa + 2;            // planes xa - 1 .. xb, sequence q = plane - xa + 1
  // plane sequence q lives in slot q % NSLOT; its full barrier completes phase q / NSLOT, and
  // the empty barrier of that slot completes phase q / NSLOT once every compute warp is done
  if (t >= G::CTHREADS) {
    // ---- producer warp -----------------------------------------------------------------
    if (t == G::CTHREADS) {
      bool ok = true;
      int q = 0;
      for (; q < nplanes && ok; ++q) {
        const int s = q % G::NSLOT;
        if (q >= G::NSLOT) ok = mbar_wait(empty + 8u * s, ((q / G::NSLOT) - 1) & 1);
        if (!ok) break;
        mbar_expect_tx(full + 8u * s, G::PLANE_BYTES);
        tma_load_5d(ring + (uint32_t)s * G::PLANE_BYTES, &tmx, full + 8u * s, c0, z0 - 1, y0 - 1,
                    xa - 1 + q, 0);
      }
      // keep the CTA resident until the last copies issued have landed (or given up)
      for (int r = max(0, q - G::NSLOT); r < q; ++r)
        ok = mbar_wait(full + 8u * (r % G::NSLOT), (r / G::NSLOT) & 1) && ok;
      if (!ok) atomicExch(&g_apply_fault, 1);
    }
    return;
  }
  // ---- compute warps -----------------------------------------------------------------------
  const int lane = t & 31;
  const int g = t % G::G, tz = (t / G::G) % G::TZ, ty = t / (G::G * G::TZ);
  const int iy = y0 + ty, iz = z0 + tz, col = c0 + g * G::CPT;
  const bool active = iy < a.ny && iz < a.nz && col < a.m;
  const int cell = ((ty + 1) * G::PZ + (tz + 1)) * G::MC + g * G::CPT;
  const unsigned long long* pl = reinterpret_cast<const unsigned long long*>(sb);
  bool ok = true;
  for (int x = xa; x < xb; ++x) {
    const int qx = x - xa + 1;
    ok = ok && mbar_wait(full + 8u * ((qx - 1) % G::NSLOT), ((qx - 1) / G::NSLOT) & 1) &&
         mbar_wait(full + 8u * (qx % G::NSLOT), (qx / G::NSLOT) & 1) &&
         mbar_wait(full + 8u * ((qx + 1) % G::NSLOT), ((qx + 1) / G::NSLOT) & 1);
    if (ok && active) {
      RegRecord rc;
      const float* rp = a.rec + ((long long)x * a.ny + iy) * a.nzp + iz;
#pragma unroll
      for (int k = 0; k < K_COUNT; ++k) rc.v[k] = __ldg(rp + (long long)k * a.NP);
      TmaLoader<G> ld;
      ld.p[0] = pl + (size_t)((qx - 1) % G::NSLOT) * (G::PLANE_BYTES / 8) + cell;
      ld.p[1] = pl + (size_t)(qx % G::NSLOT) * (G::PLANE_BYTES / 8) + cell;
      ld.p[2] = pl + (size_t)((qx + 1) % G::NSLOT) * (G::PLANE_BYTES / 8) + cell;
      float2 yv[2][8];
      hx_packed_cols<2>(ld, rc, a.shift, a.cb, yv);
      const int s = (x * a.ny + iy) * a.nz + iz;
      float2* __restrict__ ys = a.Y + ((long long)s * a.ldy + col);
      const long long ybs = (long long)a.N * a.ldy;
      if (a.vec_store && col + 1 < a.m) {
#pragma unroll
        for (int b = 0; b < 8; ++b)
          *reinterpret_cast<float4*>(ys + b * ybs) = make_float4(yv[0][b].x, yv[0][b].y,
                                                                 yv[1][b].x, yv[1][b].y);
      } else {
#pragma unroll
        for (int b = 0; b < 8; ++b) {
          ys[b * ybs] = yv[0][b];
          if (col + 1 < a.m) ys[b * ybs + 1] = yv[1][b];
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(empty + 8u * ((qx - 1) % G::NSLOT));   // plane x - 1 is done
  }
  if (!ok && lane == 0) atomicExch(&g_apply_fault, 1);
}

// Tile shapes the staged kernel is built for: {precision, MC, TY, TZ}.
template <typename T> struct StagedCfgs;
template <> struct StagedCfgs<float> {
  using C0 = Staged<float, 4, 8, 12>;
  using C1 = Staged<float, 4, 6, 16>;
  using C2 = Staged<float, 4, 4, 20>;
  using C3 = Staged<float, 2, 8, 24>;
};
template <> struct StagedCfgs<double> {
  using C0 = Staged<double, 2, 8, 12>;
  using C1 = Staged<double, 2, 6, 16>;
  using C2 = Staged<double, 2, 4, 20>;
  using C3 = Staged<double, 1, 8, 16>;
};
constexpr int kStagedCfgs = 4;
constexpr int kDirect = -2;      // staged_cfg value selecting the direct kernel
constexpr int kDefaultTma = 3;   // TMA shape taken when no tile was tuned or set

struct StagedGeom { int tiles_y, tiles_z, chunks, xsplit, xlen, ctas; };

// CTA decomposition for a grid: x is split so that the CTA count fills whole waves of one CTA
// per SM, trading the two halo planes each extra x run costs.
static StagedGeom staged_geom(int nx, int ny, int nz, int m, int MC, int TY, int TZ, int sms) {
  StagedGeom g;
  g.tiles_y = (ny + TY - 1) / TY;
  g.tiles_z = (nz + TZ - 1) / TZ;
  g.chunks = (m + MC - 1) / MC;
  const long long base = (long long)g.tiles_y * g.tiles_z * g.chunks;
  double best = 1e30;
  g.xsplit = 1;
  for (int xs = 1; xs <= nx; ++xs) {
    const int xlen = (nx + xs - 1) / xs;
    if ((long long)(xs - 1) * xlen >= nx) continue;
    const long long ctas = base * xs;
    const double cost = (double)((ctas + sms - 1) / sms) * (xlen + 2);
    if (cost < best - 1e-9) { best = cost; g.xsplit = xs; }
  }
  g.xlen = (nx + g.xsplit - 1) / g.xsplit;
  g.ctas = (int)(base * g.xsplit);
  return g;
}

template <typename T, class G, bool V16>
static int launch_staged_g(const qdkp_operator* op, const T* rec, const void* X, int ldx,
                           void* Y, int ldy, int m, T shift, T cb, int sms, cudaStream_t st) {
  static bool attr_done = false;     // per instantiation; the attribute is per device function
  if (!attr_done) {
    QDKP_CUDA_TRY(cudaFuncSetAttribute(kp_apply_staged_kernel<T, G, V16>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM));
    attr_done = true;
  }
  const StagedGeom g = staged_geom(op->nx, op->ny, op->nz, m, G::MC, G::TY, G::TZ, sms);
  StagedArgs<T> a;
  a.rec = rec;
  a.X = static_cast<const cplx<T>*>(X);
  a.Y = static_cast<cplx<T>*>(Y);
  a.N = (int)op->n_sites; a.nx = op->nx; a.ny = op->ny; a.nz = op->nz;
  a.ldx = ldx; a.ldy = ldy; a.m = m;
  a.nzp = op->nzp; a.NP = op->nx * op->ny * op->nzp;
  a.tiles_z = g.tiles_z; a.chunks = g.chunks; a.xsplit = g.xsplit; a.xlen = g.xlen;
  a.shift = shift; a.cb = cb;
  kp_apply_staged_kernel<T, G, V16><<<g.ctas, G::THREADS, G::SMEM, st>>>(a);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

template <typename T, class G>
static int launch_staged_v(const qdkp_operator* op, const T* rec, const void* X, int ldx,
                           void* Y, int ldy, int m, T shift, T cb, int sms, cudaStream_t st) {
  // 16-byte copies need 16-byte aligned sources: always true for complex128 (with an aligned
  // base); for complex64 the leading dimension, the column count and the chunk must be even.
  const bool aligned = ((uintptr_t)X & 15) == 0;
  const bool v16 = aligned && (sizeof(T) == 8 || (ldx % 2 == 0 && m % 2 == 0 && G::MC % 2 == 0));
  if (v16) return launch_staged_g<T, G, true>(op, rec, X, ldx, Y, ldy, m, shift, cb, sms, st);
  return launch_staged_g<T, G, false>(op, rec, X, ldx, Y, ldy, m, shift, cb, sms, st);
}

template <typename T>
static int launch_staged(int cfg, const qdkp_operator* op, const T* rec, const void* X, int ldx,
                         void* Y, int ldy, int m, T shift, T cb, int sms, cudaStream_t st) {
  using C = StagedCfgs<T>;
  switch (cfg) {
    case 0: return launch_staged_v<T, typename C::C0>(op, rec, X, ldx, Y, ldy, m, shift, cb, sms, st);
    case 1: return launch_staged_v<T, typename C::C1>(op, rec, X, ldx, Y, ldy, m, shift, cb, sms, st);
    case 2: return launch_staged_v<T, typename C::C2>(op, rec, X, ldx, Y, ldy, m, shift, cb, sms, st);
    default: return launch_staged_v<T, typename C::C3>(op, rec, X, ldx, Y, ldy, m, shift, cb, sms, st);
  }
}

// ---- TMA kernel launch ------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda)
static EncodeTiledFn tensor_map_encoder() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// TMA tile shapes {TY, TZ, column pairs per CTA, ring slots}; staged_cfg kTmaBase + i selects
// shape i (complex64 only).
struct TmaCfgs {
  using C0 = Tma<6, 16, 2, 4>;
  using C1 = Tma<6, 16, 2, 5>;
  using C2 = Tma<8, 12, 2, 5>;
  using C3 = Tma<4, 24, 2, 4>;
  using C4 = Tma<4, 12, 2, 4, 2>;      // two CTAs per SM: one CTA's plane barrier overlaps
  using C5 = Tma<6, 8, 2, 4, 2>;       // the other's compute
  using C6 = Tma<8, 16, 2, 4, 1, true>;   // records in registers: 256 and 288 threads
  using C7 = Tma<6, 24, 2, 4, 1, true>;
};
constexpr int kTmaBase = 4;
constexpr int kTmaCfgs = 8;

template <class G>
static bool tma_fits(const qdkp_operator* op, const void* X, int64_t ldx, int m) {
  // tensor-map rules: 16-byte aligned base and strides; every box no larger than its tensor
  return op->n_bands == 8 && ((uintptr_t)X & 15) == 0 && ldx % 2 == 0 && m >= G::MC &&
         op->ny >= G::PY && op->nz >= G::PZ && op->nzp >= G::TZ && tensor_map_encoder() != nullptr;
}

static bool tma_fits_cfg(int i, const qdkp_operator* op, const void* X, int64_t ldx, int m) {
  switch (i) {
    case 0: return tma_fits<TmaCfgs::C0>(op, X, ldx, m);
    case 1: return tma_fits<TmaCfgs::C1>(op, X, ldx, m);
    case 2: return tma_fits<TmaCfgs::C2>(op, X, ldx, m);
    case 3: return tma_fits<TmaCfgs::C3>(op, X, ldx, m);
    case 4: return tma_fits<TmaCfgs::C4>(op, X, ldx, m);
    case 5: return tma_fits<TmaCfgs::C5>(op, X, ldx, m);
    case 6: return tma_fits<TmaCfgs::C6>(op, X, ldx, m);
    default: return tma_fits<TmaCfgs::C7>(op, X, ldx, m);
  }
}

template <class G>
static int launch_tma_g(const qdkp_operator* op, const void* X, int ldx, void* Y, int ldy, int m,
                        float shift, float cb, int sms, cudaStream_t st) {
  const EncodeTiledFn enc = tensor_map_encoder();
  static bool attr_done = false;     // per instantiation; the attribute is per device function
  if (!attr_done) {
    QDKP_CUDA_TRY(cudaFuncSetAttribute(kp_apply_tma_kernel<G>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM));
    attr_done = true;
  }
  const cuuint64_t N = (cuuint64_t)op->n_sites, ld = (cuuint64_t)ldx;
  CUtensorMap tmx, tmr;
  // X as [band][x][y][z][column] with the column innermost (8-byte elements)
  const cuuint64_t xdim[5] = {(cuuint64_t)m, (cuuint64_t)op->nz, (cuuint64_t)op->ny,
                              (cuuint64_t)op->nx, 8};
  const cuuint64_t xstr[4] = {ld * 8, (cuuint64_t)op->nz * ld * 8,
                              (cuuint64_t)op->ny * op->nz * ld * 8, N * ld * 8};
  const cuuint32_t xbox[5] = {(cuuint32_t)G::MC, (cuuint32_t)G::PZ, (cuuint32_t)G::PY, 1, 8};
  const cuuint32_t ones[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(&tmx, CU_TENSOR_MAP_DATA_TYPE_INT64, 5, const_cast<void*>(X), xdim, xstr,
                   xbox, ones, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed for the X block (code " + std::to_string((int)r) + ")");
    return QDKP_ERR_CUDA;
  }
  // the FP32 record as [entry][x][y][z_padded]
  const cuuint64_t NP = (cuuint64_t)op->nx * op->ny * op->nzp;
  const cuuint64_t rdim[4] = {(cuuint64_t)op->nzp, (cuuint64_t)op->ny, (cuuint64_t)op->nx,
                              (cuuint64_t)K_COUNT};
  const cuuint64_t rstr[3] = {(cuuint64_t)op->nzp * 4, (cuuint64_t)op->ny * op->nzp * 4, NP * 4};
  const cuuint32_t rbox[4] = {(cuuint32_t)G::TZ, (cuuint32_t)G::TY, 1, (cuuint32_t)K_COUNT};
  r = enc(&tmr, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, op->rec32, rdim, rstr, rbox, ones,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed for the record (code " + std::to_string((int)r) + ")");
    return QDKP_ERR_CUDA;
  }
  const StagedGeom g = staged_geom(op->nx, op->ny, op->nz, m, G::MC, G::TY, G::TZ,
                                   sms * G::MINB);
  TmaArgs a;
  a.Y = static_cast<float2*>(Y);
  a.rec = op->rec32;
  a.nzp = op->nzp; a.NP = op->nx * op->ny * op->nzp;
  a.N = (int)op->n_sites; a.nx = op->nx; a.ny = op->ny; a.nz = op->nz;
  a.ldy = ldy; a.m = m;
  a.tiles_z = g.tiles_z; a.chunks = g.chunks; a.xsplit = g.xsplit; a.xlen = g.xlen;
  a.vec_store = ((uintptr_t)Y & 15) == 0 && ldy % 2 == 0;
  a.shift = shift; a.cb = cb;
  kp_apply_tma_kernel<G><<<g.ctas, G::THREADS, G::SMEM, st>>>(tmx, tmr, a);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

static int launch_tma(int i, const qdkp_operator* op, const void* X, int ldx, void* Y, int ldy,
                      int m, float shift, float cb, int sms, cudaStream_t st) {
  switch (i) {
    case 0: return launch_tma_g<TmaCfgs::C0>(op, X, ldx, Y, ldy, m, shift, cb, sms, st);
    case 1: return launch_tma_g<TmaCfgs::C1>(op, X, ldx, Y, ldy, m, shift, cb, sms, st);
    case 2: return launch_tma_g<TmaCfgs::C2>(op, X, ldx, Y, ldy, m, shift, cb, sms, st);
    case 3: return launch_tma_g<TmaCfgs::C3>(op, X, ldx, Y, ldy, m, shift, cb, sms, st);
    case 4: return launch_tma_g<TmaCfgs::C4>(op, X, ldx, Y, ldy, m, shift, cb, sms, st);
    case 5: return launch_tma_g<TmaCfgs::C5>(op, X, ldx, Y, ldy, m, shift, cb, sms, st);
    case 6: return launch_tma_g<TmaCfgs::C6>(op, X, ldx, Y, ldy, m, shift, cb, sms, st);
    default: return launch_tma_g<TmaCfgs::C7>(op, X, ldx, Y, ldy, m, shift, cb, sms, st);
  }
}

// Producer-warp TMA shapes {TY, TZ, column pairs per CTA, ring slots, CTAs per SM};
// staged_cfg kTma2Base + i selects shape i (complex64 only).
struct Tma2Cfgs {
  using D0 = Tma2<6, 16, 2, 4, 1>;
  using D1 = Tma2<8, 16, 2, 4, 1>;
  using D2 = Tma2<8, 16, 1, 4, 2>;
  using D3 = Tma2<6, 16, 2, 5, 1>;
  using D4 = Tma2<4, 24, 2, 4, 1>;
};
constexpr int kTma2Base = kTmaBase + kTmaCfgs;
constexpr int kTma2Cfgs = 5;

template <class G>
static bool tma2_fits(const qdkp_operator* op, const void* X, int64_t ldx, int m) {
  return op->n_bands == 8 && ((uintptr_t)X & 15) == 0 && ldx % 2 == 0 && m >= G::MC &&
         op->ny >= G::PY && op->nz >= G::PZ && tensor_map_encoder() != nullptr;
}

static bool tma2_fits_cfg(int i, const qdkp_operator* op, const void* X, int64_t ldx, int m) {
  switch (i) {
    case 0: return tma2_fits<Tma2Cfgs::D0>(op, X, ldx, m);
    case 1: return tma2_fits<Tma2Cfgs::D1>(op, X, ldx, m);
    case 2: return tma2_fits<Tma2Cfgs::D2>(op, X, ldx, m);
    case 3: return tma2_fits<Tma2Cfgs::D3>(op, X, ldx, m);
    default: return tma2_fits<Tma2Cfgs::D4>(op, X, ldx, m);
  }
}

template <class G>
static int launch_tma2_g(const qdkp_operator* op, const void* X, int ldx, void* Y, int ldy, int m,
                         float shift, float cb, int sms, cudaStream_t st) {
  const EncodeTiledFn enc = tensor_map_encoder();
  static bool attr_done = false;
  if (!attr_done) {
    QDKP_CUDA_TRY(cudaFuncSetAttribute(kp_apply_tma2_kernel<G>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM));
    attr_done = true;
  }
  const cuuint64_t N = (cuuint64_t)op->n_sites, ld = (cuuint64_t)ldx;
  CUtensorMap tmx;
  const cuuint64_t xdim[5] = {(cuuint64_t)m, (cuuint64_t)op->nz, (cuuint64_t)op->ny,
                              (cuuint64_t)op->nx, 8};
  const cuuint64_t xstr[4] = {ld * 8, (cuuint64_t)op->nz * ld * 8,
                              (cuuint64_t)op->ny * op->nz * ld * 8, N * ld * 8};
  const cuuint32_t xbox[5] = {(cuuint32_t)G::MC, (cuuint32_t)G::PZ, (cuuint32_t)G::PY, 1, 8};
  const cuuint32_t ones[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(&tmx, CU_TENSOR_MAP_DATA_TYPE_INT64, 5, const_cast<void*>(X), xdim, xstr,
                   xbox, ones, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed for the X block (code " + std::to_string((int)r) + ")");
    return QDKP_ERR_CUDA;
  }
  // one wave holds MINB CTAs per SM
  const StagedGeom g = staged_geom(op->nx, op->ny, op->nz, m, G::MC, G::TY, G::TZ,
                                   sms * G::MINB);
  Tma2Args a;
  a.Y = static_cast<float2*>(Y);
  a.rec = op->rec32;
  a.N = (int)op->n_sites; a.nx = op->nx; a.ny = op->ny; a.nz = op->nz;
  a.nzp = op->nzp; a.NP = op->nx * op->ny * op->nzp;
  a.ldy = ldy; a.m = m;
  a.tiles_z = g.tiles_z; a.chunks = g.chunks; a.xsplit = g.xsplit; a.xlen = g.xlen;
  a.vec_store = ((uintptr_t)Y & 15) == 0 && ldy % 2 == 0;
  a.shift = shift; a.cb = cb;
  kp_apply_tma2_kernel<G><<<g.ctas, G::THREADS, G::SMEM, st>>>(tmx, a);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

static int launch_tma2(int i, const qdkp_operator* op, const void* X, int ldx, void* Y, int ldy,
                       int m, float shift, float cb, int sms, cudaStream_t st) {
  switch (i) {
    case 0: return launch_tma2_g<Tma2Cfgs::D0>(op, X, ldx, Y, ldy, m, shift, cb, sms, st);
    case 1: return launch_tma2_g<Tma2Cfgs::D1>(op, X, ldx, Y, ldy, m, shift, cb, sms, st);
    case 2: return launch_tma2_g<Tma2Cfgs::D2>(op, X, ldx, Y, ldy, m, shift, cb, sms, st);
    case 3: return launch_tma2_g<Tma2Cfgs::D3>(op, X, ldx, Y, ldy, m, shift, cb, sms, st);
    default: return launch_tma2_g<Tma2Cfgs::D4>(op, X, ldx, Y, ldy, m, shift, cb, sms, st);
  }
}

int launch_apply_multi(const HXSlot* slots_dev, int nslots, int total_tiles, int precision,
                       cudaStream_t st) {
  if (total_tiles <= 0) return QDKP_OK;
  if (precision == QDKP_C128)
    kp_apply_multi_kernel<double><<<total_tiles, kApplyThreads, 0, st>>>(slots_dev, nslots);
  else
    kp_apply_multi_kernel<float><<<total_tiles, kApplyThreads, 0, st>>>(slots_dev, nslots);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

int apply_tiles(int64_t n_sites, int m) {
  return (int)((n_sites * m + kApplyThreads - 1) / kApplyThreads);
}

// sign of the operator as applied: -1 for a hole-convention 6/4-band slice, flipped by NEGATE
static double op_sign(const qdkp_operator* op) {
  double sign = ((op->flags & QDKP_HOLE_CONVENTION) && op->n_bands != 8) ? -1.0 : 1.0;
  if (op->flags & QDKP_NEGATE) sign = -sign;
  return sign;
}

double apply_cb_weight(const qdkp_operator* op) { return op_sign(op) * (-kG / (op->h * op->h)); }

int build_records(qdkp_operator* op) {
  const long long N = op->n_sites;
  const int blocks = (int)std::min<long long>((N + 127) / 128, 148 * 16);
  kp_record_kernel<<<blocks, 128>>>(op->fields64, N, op->nx, op->ny, op->nz, op->nzp, op->h,
                                     op->flags, op->n_bands, op_sign(op), op->rec64, op->rec32,
                                     op->nbmask);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  QDKP_CUDA_TRY(cudaDeviceSynchronize());
  return QDKP_OK;
}

size_t record_doubles(int nx, int ny, int nzp) { return (size_t)K_COUNT * nx * ny * nzp; }

static int num_sms(int device) {
  static int cached[64] = {0};
  if (device < 0 || device >= 64) return 148;
  if (!cached[device]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || v <= 0)
      v = 148;
    cached[device] = v;
  }
  return cached[device];
}

// Default kernel for a launch without a tuned choice, from measurements of both kernels over
// grids of 23x23x20 to 128x128x96 and blocks of 12 and 24 columns on B200: complex128 is FP64-
// issue bound and the direct kernel (more resident warps) is as fast or faster everywhere;
// complex64 takes a shared-memory kernel on grids of 50k sites and more, where its reuse pays:
// the TMA kernel where its tensor maps fit, else the cp.async staged kernel with the tile shape
// that pads the (y, z) plane least. qdkp_operator_tune refines this per operator.
static int pick_staged_cfg(const qdkp_operator* op, int precision, const void* X, int64_t ldx,
                           int m) {
  if (precision == QDKP_C128 || op->n_sites < 50000) return kDirect;
  if (tma_fits_cfg(kDefaultTma, op, X, ldx, m)) return kTmaBase + kDefaultTma;
  // the four-column shapes (0, 1) measured fastest on every grid; pick the one that pads less
  static const int shape[2][2] = {{8, 12}, {6, 16}};   // TY, TZ
  int best = 0;
  double best_w = 1e30;
  for (int c = 0; c < 2; ++c) {
    const int TY = shape[c][0], TZ = shape[c][1];
    const double w = (double)((op->ny + TY - 1) / TY * TY) * ((op->nz + TZ - 1) / TZ * TZ) *
                     (1.0 + 2.0 / TY) * (1.0 + 2.0 / TZ);
    if (w < best_w - 1e-9) { best_w = w; best = c; }
  }
  return best;
}

template <typename T>
static int launch_apply_t(const qdkp_operator* op, const T* rec, const void* X, int64_t ldx,
                          void* Y, int64_t ldy, int m, double sigma, int shifted, int precision,
                          cudaStream_t st) {
  if ((int64_t)op->n_bands * op->n_sites * std::max(ldx, ldy) >= (int64_t(1) << 31)) {
    set_error("H.X: n * leading dimension must stay below 2^31 elements");
    return QDKP_ERR_UNSUPPORTED;
  }
  const T shift = shifted ? (T)(-sigma) : T(0);
  const T cb = (T)apply_cb_weight(op);
  const int forced = op->staged_cfg[precision == QDKP_C64];
  int cfg = forced == QDKP_TILE_AUTO ? pick_staged_cfg(op, precision, X, ldx, m) : forced;
  if (cfg >= kTma2Base) {
    if (std::is_same<T, float>::value && tma2_fits_cfg(cfg - kTma2Base, op, X, ldx, m))
      return launch_tma2(cfg - kTma2Base, op, X, (int)ldx, Y, (int)ldy, m, (float)shift,
                         (float)cb, num_sms(op->device), st);
    cfg = 1;       // a block the tensor maps cannot describe: the cp.async staged kernel
  } else if (cfg >= kTmaBase) {
    if (std::is_same<T, float>::value && tma_fits_cfg(cfg - kTmaBase, op, X, ldx, m))
      return launch_tma(cfg - kTmaBase, op, X, (int)ldx, Y, (int)ldy, m, (float)shift, (float)cb,
                        num_sms(op->device), st);
    cfg = 1;
  }
  if (op->n_bands == 8 && cfg >= 0 && ((uintptr_t)X % sizeof(cplx<T>)) == 0)
    return launch_staged<T>(cfg, op, rec, X, (int)ldx, Y, (int)ldy, m, shift, cb,
                            num_sms(op->device), st);
  HXArgs<T> a;
  a.rec = rec;
  a.msk = op->nbmask;
  a.X = static_cast<const cplx<T>*>(X);
  a.Y = static_cast<cplx<T>*>(Y);
  a.N = (int)op->n_sites; a.ldx = (int)ldx; a.ldy = (int)ldy; a.m = m;
  a.sx = op->ny * op->nz; a.sy = op->nz;
  a.nz = op->nz; a.nzp = op->nzp; a.NP = op->nx * op->ny * op->nzp;
  a.shift = shift;
  a.cb = cb;
  const unsigned grid = (unsigned)apply_tiles(op->n_sites, m);
  switch (op->n_bands) {
    case 8: kp_apply_kernel<T, 8><<<grid, kApplyThreads, 0, st>>>(a); break;
    case 6: kp_apply_kernel<T, 6><<<grid, kApplyThreads, 0, st>>>(a); break;
    case 4: kp_apply_kernel<T, 4><<<grid, kApplyThreads, 0, st>>>(a); break;
    default: set_error("n_bands must be 8, 6 or 4"); return QDKP_ERR_ARG;
  }
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

// Y = sign*H X (- sigma X if shifted) for one block in the given precision.
int launch_apply(const qdkp_operator* op, const void* X, int64_t ldx, void* Y, int64_t ldy,
                 int m, double sigma, int shifted, int precision, cudaStream_t st) {
  if (precision == QDKP_C128)
    return launch_apply_t<double>(op, op->rec64, X, ldx, Y, ldy, m, sigma, shifted, precision, st);
  if (precision == QDKP_C64)
    return launch_apply_t<float>(op, op->rec32, X, ldx, Y, ldy, m, sigma, shifted, precision, st);
  set_error("precision must be QDKP_C128 or QDKP_C64");
  return QDKP_ERR_ARG;
}

}  // namespace qdkp

using namespace qdkp;

extern "C" {

int qdkp_operator_set_tile(qdkp_operator* op, int precision, int tile) {
  QDKP_CHECK_ARG(op != nullptr, "operator must not be NULL");
  QDKP_CHECK_ARG(precision == QDKP_C128 || precision == QDKP_C64, "bad precision");
  QDKP_CHECK_ARG(tile >= QDKP_TILE_DIRECT && tile < kStagedCfgs + kTmaCfgs + kTma2Cfgs,
                 "tile out of range");
  QDKP_CHECK_ARG(precision == QDKP_C64 || tile < kStagedCfgs,
                 "the TMA tile shapes are built for complex64 only");
  op->staged_cfg[precision == QDKP_C64] = tile;
  return QDKP_OK;
}

int qdkp_operator_get_tile(const qdkp_operator* op, int precision, int* tile) {
  QDKP_CHECK_ARG(op != nullptr && tile != nullptr, "NULL argument");
  QDKP_CHECK_ARG(precision == QDKP_C128 || precision == QDKP_C64, "bad precision");
  *tile = op->staged_cfg[precision == QDKP_C64];
  return QDKP_OK;
}

int qdkp_operator_tune(qdkp_operator* op, const void* X, int64_t ldx, void* Y, int64_t ldy,
                       int m, int precision, int reps, double* seconds, void* stream) {
  QDKP_CHECK_ARG(op != nullptr && X != nullptr && Y != nullptr, "NULL argument");
  QDKP_CHECK_ARG(precision == QDKP_C128 || precision == QDKP_C64, "bad precision");
  QDKP_CHECK_ARG(m > 0 && ldx >= m && ldy >= m && reps > 0, "bad block or repetitions");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  QDKP_CUDA_TRY(cudaSetDevice(op->device));
  const int pi = precision == QDKP_C64;
  const int saved = op->staged_cfg[pi];
  cudaEvent_t e0, e1;
  QDKP_CUDA_TRY(cudaEventCreate(&e0));
  QDKP_CUDA_TRY(cudaEventCreate(&e1));
  int best = saved;
  float best_ms = 3.4e38f;
  int rc = QDKP_OK;
  // candidates: the staged shapes, the TMA shapes (complex64), the direct kernel last; the
  // seconds array has one entry per candidate, -1 for one that does not apply
  const int nbuilt = kStagedCfgs + kTmaCfgs + kTma2Cfgs;
  const int ncand = nbuilt + 1;
  for (int c = 0; c < ncand && rc == QDKP_OK; ++c) {
    const int tile = c < nbuilt ? c : kDirect;
    if (seconds) seconds[c] = -1.0;
    if (op->n_bands != 8 && tile != kDirect) continue;                // 6/4-band: direct only
    if (tile >= kTmaBase && precision != QDKP_C64) continue;
    if (tile >= kTma2Base && !tma2_fits_cfg(tile - kTma2Base, op, X, ldx, m)) continue;
    if (tile >= kTmaBase && tile < kTma2Base && !tma_fits_cfg(tile - kTmaBase, op, X, ldx, m))
      continue;
    op->staged_cfg[pi] = tile;
    rc = launch_apply(op, X, ldx, Y, ldy, m, 0.0, 0, precision, st);      // warm-up
    if (rc != QDKP_OK) break;
    if (cudaEventRecord(e0, st) != cudaSuccess) { rc = QDKP_ERR_CUDA; break; }
    for (int r = 0; r < reps && rc == QDKP_OK; ++r)
      rc = launch_apply(op, X, ldx, Y, ldy, m, 0.0, 0, precision, st);
    if (rc != QDKP_OK) break;
    float ms = 0.f;
    if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) { rc = QDKP_ERR_CUDA; break; }
    if (seconds) seconds[c] = ms * 1e-3 / reps;
    if (ms < best_ms) { best_ms = ms; best = tile; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  op->staged_cfg[pi] = rc == QDKP_OK ? best : saved;
  if (rc == QDKP_ERR_CUDA) set_error("qdkp_operator_tune: CUDA event failure");
  return rc;
}

int qdkp_device_fault(int device, int clear, int* fault) {
  QDKP_CHECK_ARG(fault != nullptr, "NULL argument");
  int prev = 0;
  QDKP_CUDA_TRY(cudaGetDevice(&prev));
  QDKP_CUDA_TRY(cudaSetDevice(device));
  cudaError_t e = cudaMemcpyFromSymbol(fault, g_apply_fault, sizeof(int));
  if (e == cudaSuccess && clear) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(g_apply_fault, &zero, sizeof(int));
  }
  cudaSetDevice(prev);
  QDKP_CUDA_TRY(e);
  return QDKP_OK;
}

}  // extern "C"
