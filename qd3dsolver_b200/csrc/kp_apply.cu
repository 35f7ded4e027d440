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
// Work split: a CTA owns S consecutive sites. Phase 1 builds one coefficient record per site
// into shared memory (face-averaged stencil weights, first-order face weights, the local
// block), reading the 15 raw fields of the site and its six face neighbours. Phase 2 gives each
// thread (site, column) items: it loads the eight band components of the site, its six faces
// and twelve edges for that column, and accumulates all eight output bands in registers.
#include <algorithm>

#include "qdkp_common.cuh"

namespace qdkp {

enum RecSlot {
  R_A = 0, R_P, R_Q, R_RRE, R_RIM, R_SRE, R_SIM, R_DL,
  R_T1 = 8,     // -G t1 per face (x+, x-, y+, y-, z+, z-): P kinetic
  R_T2 = 14,    // -G t2 per face: Q and R kinetic
  R_G3 = 20,    // gamma3 at the face neighbour (cross terms)
  R_SU = 26,    // (cu_p + cu_q) / 4h, signed by the face direction: U
  R_SVR = 32,   // (cv_p + cv_q) / 4h, signed, real part: V
  R_SVI = 38,   // imaginary part
  R_COUNT = 44
};

template <typename T>
struct ApplyArgs {
  const T* __restrict__ F;   // F_COUNT * N
  const cplx<T>* __restrict__ X;
  cplx<T>* __restrict__ Y;
  long long N, ldx, ldy;
  int nx, ny, nz, m, flags, S;
  T h, sigma, sign;          // sign = -1 for the hole convention
  int shifted;
};

template <typename T>
__device__ __forceinline__ void first_order_coefs(const T* __restrict__ F, long long N,
                                                  long long q, bool inter, T cu[3],
                                                  cplx<T> cv[3]) {
  const T r3 = T(0.57735026918962576451), r6 = T(0.40824829046386301637);
  const T P0 = F[F_P0 * N + q];
  if (inter) {
    const T exx = F[F_EXX * N + q], eyy = F[F_EYY * N + q], ezz = F[F_EZZ * N + q];
    const T exy = F[F_EXY * N + q], eyz = F[F_EYZ * N + q], ezx = F[F_EZX * N + q];
    cu[0] = -P0 * ezx * r3;
    cu[1] = -P0 * eyz * r3;
    cu[2] = P0 * (T(1) - ezz) * r3;
    cv[0] = mk<T>(P0 * (T(1) - exx) * r6, P0 * exy * r6);
    cv[1] = mk<T>(-P0 * exy * r6, P0 * (eyy - T(1)) * r6);
    cv[2] = mk<T>(-P0 * ezx * r6, P0 * eyz * r6);
  } else {
    cu[0] = T(0); cu[1] = T(0); cu[2] = P0 * r3;
    cv[0] = mk<T>(P0 * r6, T(0));
    cv[1] = mk<T>(T(0), -P0 * r6);
    cv[2] = czero<T>();
  }
}

template <typename T, int NB>
__device__ void build_record(const ApplyArgs<T>& a, long long s, T* rec, int S,
                             unsigned* nbmask) {
  const T* __restrict__ F = a.F;
  const long long N = a.N;
  const int iz = (int)(s % a.nz);
  const long long t = s / a.nz;
  const int iy = (int)(t % a.ny);
  const int ix = (int)(t / a.ny);
  const int coord[3] = {ix, iy, iz};
  const int ext[3] = {a.nx, a.ny, a.nz};
  const long long str[3] = {(long long)a.ny * a.nz, (long long)a.nz, 1LL};
  const T G = T(kG);
  const T ih2 = T(1) / (a.h * a.h);
  const T i4h = T(1) / (T(4) * a.h);
  const bool strain = (a.flags & QDKP_STRAIN) != 0;
  const bool inter = NB == 8 && strain && (a.flags & QDKP_INTERBAND_STRAIN);

  // neighbour mask: bit f (0..5) face x+, x-, y+, y-, z+, z-; bit 6 + 4 pl + e the in-plane
  // edge e of plane pl (xy, zx, zy) with signs sa = e & 1 ? -1 : 1, sb = e & 2 ? -1 : 1
  {
    unsigned msk = 0;
    for (int ax = 0; ax < 3; ++ax) {
      if (coord[ax] + 1 < ext[ax]) msk |= 1u << (2 * ax);
      if (coord[ax] > 0) msk |= 1u << (2 * ax + 1);
    }
    for (int pl = 0; pl < 3; ++pl) {
      const int ea = pl == 0 ? 0 : 2, eb = pl == 0 ? 1 : (pl == 1 ? 0 : 1);
      for (int e = 0; e < 4; ++e) {
        const int ca = coord[ea] + ((e & 1) ? -1 : 1), cb = coord[eb] + ((e & 2) ? -1 : 1);
        if (ca >= 0 && ca < ext[ea] && cb >= 0 && cb < ext[eb]) msk |= 1u << (6 + 4 * pl + e);
      }
    }
    *nbmask = msk;
  }
  const T g1 = F[F_G1 * N + s], g2 = F[F_G2 * N + s];
  T cu_p[3]; cplx<T> cv_p[3];
  if (NB == 8) first_order_coefs<T>(F, N, s, inter, cu_p, cv_p);
  T dk1 = T(0), dk2[3];
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    T d1 = T(0), d2 = T(0);
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
      const int f = 2 * ax + dir;
      const bool in = dir == 0 ? (coord[ax] + 1 < ext[ax]) : (coord[ax] > 0);
      T t1n = T(0), t2n = T(0), g3n = T(0), su = T(0), svr = T(0), svi = T(0);
      if (in) {
        const long long q = dir == 0 ? s + str[ax] : s - str[ax];
        const T t1 = (g1 + F[F_G1 * N + q]) * T(0.5) * ih2;
        const T t2 = (g2 + F[F_G2 * N + q]) * T(0.5) * ih2;
        d1 += t1; d2 += t2;
        t1n = -G * t1; t2n = -G * t2;
        g3n = F[F_G3 * N + q];
        if (NB == 8) {
          T cu_q[3]; cplx<T> cv_q[3];
          first_order_coefs<T>(F, N, q, inter, cu_q, cv_q);
          const T sg = dir == 0 ? T(1) : T(-1);
          su = sg * (cu_p[ax] + cu_q[ax]) * i4h;
          svr = sg * (cv_p[ax].x + cv_q[ax].x) * i4h;
          svi = sg * (cv_p[ax].y + cv_q[ax].y) * i4h;
        }
      } else {  // hard wall: ghost term alpha_p / h^2 (kp_confined.py:133-137)
        d1 += g1 * ih2; d2 += g2 * ih2;
      }
      rec[(R_T1 + f) * S] = t1n;
      rec[(R_T2 + f) * S] = t2n;
      rec[(R_G3 + f) * S] = g3n;
      rec[(R_SU + f) * S] = su;
      rec[(R_SVR + f) * S] = svr;
      rec[(R_SVI + f) * S] = svi;
    }
    dk1 += d1; dk2[ax] = d2;
  }
  const T sq3 = T(1.73205080756887729353);
  T Q = G * (dk2[0] + dk2[1] - T(2) * dk2[2]);
  T Rre = -sq3 * G * (dk2[0] - dk2[1]), Rim = T(0), Sre = T(0), Sim = T(0);
  if (strain) {
    const T b = F[F_B * N + s], d = F[F_D * N + s];
    const T exx = F[F_EXX * N + s], eyy = F[F_EYY * N + s], ezz = F[F_EZZ * N + s];
    const T exy = F[F_EXY * N + s], eyz = F[F_EYZ * N + s], ezx = F[F_EZX * N + s];
    Q += -(b / T(2)) * (exx + eyy - T(2) * ezz);
    Rre += (sq3 / T(2)) * b * (exx - eyy);
    Rim += -d * exy;
    Sre = -d * ezx;
    Sim = d * eyz;
  }
  rec[R_A * S] = F[F_EC * N + s] + T(6) * G * ih2;
  rec[R_P * S] = -F[F_EV * N + s] + G * dk1;
  rec[R_Q * S] = Q;
  rec[R_RRE * S] = Rre;
  rec[R_RIM * S] = Rim;
  rec[R_SRE * S] = Sre;
  rec[R_SIM * S] = Sim;
  rec[R_DL * S] = F[F_DSO * N + s];
}

template <int NB> __device__ __forceinline__ constexpr bool has_band(int b) {
  return NB == 8 ? true : (NB == 6 ? b >= 2 : (b >= 2 && b <= 5));
}
template <int NB> __device__ __forceinline__ constexpr int band_off() { return NB == 8 ? 0 : 2; }

// x[b] = X[band b, site s + offset, column j] with xs = &X[0, s, j], bstr = N ldx (elements);
// every offset fits 32 bits for the grids this library accepts (n ldx < 2^31).
template <typename T, int NB, bool VB_ONLY>
__device__ __forceinline__ void load_site(const cplx<T>* __restrict__ xs, int bstr, int off,
                                          cplx<T> (&x)[8]) {
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    if (!has_band<NB>(b) || (VB_ONLY && b < 2)) { x[b] = czero<T>(); continue; }
    x[b] = __ldg(xs + ((b - band_off<NB>()) * bstr + off));
  }
}

template <typename T> struct ApplyOcc;
template <> struct ApplyOcc<double> { static constexpr int kMinBlocks = 2; };
template <> struct ApplyOcc<float> { static constexpr int kMinBlocks = 2; };

template <typename T, int NB>
__device__ __forceinline__ void apply_tile(const ApplyArgs<T>& a, long long s0, T* rec) {
  const int S = a.S;
  const int ns = (int)min((long long)S, a.N - s0);

  unsigned* nbm = reinterpret_cast<unsigned*>(rec + R_COUNT * S);
  for (int i = threadIdx.x; i < ns; i += blockDim.x)
    build_record<T, NB>(a, s0 + i, rec + i, S, nbm + i);
  __syncthreads();

  const T G = T(kG);
  const T ih2 = T(1) / (a.h * a.h);
  const T sq2 = T(1.41421356237309504880), sq3 = T(1.73205080756887729353);
  const T sq32 = T(1.22474487139158904910), isq2 = T(0.70710678118654752440);
  const T i8h2 = T(1) / (T(8) * a.h * a.h);
  const T wQ[3] = {T(1), T(1), T(-2)};
  const T wR[3] = {-sq3, sq3, T(0)};
  const int m = a.m;
  const int items = ns * m;

  const int bstr = (int)(a.N * a.ldx);
  const int ystr = (int)(a.N * a.ldy);
  const int sx = a.ny * a.nz, sy = a.nz;
  for (int it = threadIdx.x; it < items; it += blockDim.x) {
    const int i = it / m;
    const int j = it - i * m;
    const long long s = s0 + i;
    const T* r = rec + i;
    const unsigned msk = nbm[i];
    const cplx<T>* __restrict__ xs = a.X + (s * a.ldx + j);
    const int str[3] = {sx * (int)a.ldx, sy * (int)a.ldx, (int)a.ldx};
    cplx<T> y[8], x[8];

    // ---- local block ------------------------------------------------------------------
    // y = sign (H x) - sigma x is accumulated as sign (H x - sign sigma x): start from the
    // shift term so the centre values need not stay live until the end.
    load_site<T, NB, false>(xs, bstr, 0, x);
    {
      const T sh = a.shifted ? -a.sigma * a.sign : T(0);
#pragma unroll
      for (int b = 0; b < 8; ++b) y[b] = cscale(sh, x[b]);
    }
    {
      const T A = r[R_A * S], P = r[R_P * S], Q = r[R_Q * S], Dl = r[R_DL * S];
      const cplx<T> R = mk<T>(r[R_RRE * S], r[R_RIM * S]);
      const cplx<T> Sx = mk<T>(r[R_SRE * S], r[R_SIM * S]);
      if (NB == 8) { caxpy(y[0], A, x[0]); caxpy(y[1], A, x[1]); }
      caxpy(y[2], -P + Q, x[2]); cfmac(y[2], Sx, cscale(T(-1), x[3])); cfma(y[2], R, x[4]);
      cfma(y[2], Sx, cscale(sq32, x[6])); caxpy(y[2], -sq2 * Q, x[7]);
      cfma(y[3], Sx, cscale(T(-1), x[2])); caxpy(y[3], -P - Q, x[3]); cfma(y[3], R, x[5]);
      cfma(y[3], R, cscale(-sq2, x[6])); cfma(y[3], Sx, cscale(isq2, x[7]));
      cfmac(y[4], R, x[2]); caxpy(y[4], -P - Q, x[4]); cfmac(y[4], Sx, x[5]);
      cfmac(y[4], Sx, cscale(isq2, x[6])); cfmac(y[4], R, cscale(sq2, x[7]));
      cfmac(y[5], R, x[3]); cfma(y[5], Sx, x[4]); caxpy(y[5], -P + Q, x[5]);
      caxpy(y[5], sq2 * Q, x[6]); cfmac(y[5], Sx, cscale(sq32, x[7]));
      cfmac(y[6], Sx, cscale(sq32, x[2])); cfmac(y[6], R, cscale(-sq2, x[3]));
      cfma(y[6], Sx, cscale(isq2, x[4])); caxpy(y[6], sq2 * Q, x[5]); caxpy(y[6], -P - Dl, x[6]);
      caxpy(y[7], -sq2 * Q, x[2]); cfmac(y[7], Sx, cscale(isq2, x[3])); cfma(y[7], R, cscale(sq2, x[4]));
      cfma(y[7], Sx, cscale(sq32, x[5])); caxpy(y[7], -P - Dl, x[7]);
    }

    // ---- six face neighbours ------------------------------------------------------------
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const int ax = f >> 1, dir = f & 1;
      if (!(msk & (1u << f))) continue;
      load_site<T, NB, false>(xs, bstr, dir == 0 ? str[ax] : -str[ax], x);
      const T kp = r[(R_T1 + f) * S], k2 = r[(R_T2 + f) * S];
      const T kq = wQ[ax] * k2, kr = wR[ax] * k2;
      if (NB == 8) { caxpy(y[0], -G * ih2, x[0]); caxpy(y[1], -G * ih2, x[1]); }
      caxpy(y[2], -kp + kq, x[2]); caxpy(y[2], -sq2 * kq, x[7]);
      caxpy(y[3], -kp - kq, x[3]);
      caxpy(y[4], -kp - kq, x[4]);
      caxpy(y[5], -kp + kq, x[5]); caxpy(y[5], sq2 * kq, x[6]);
      caxpy(y[6], -kp, x[6]); caxpy(y[6], sq2 * kq, x[5]);
      caxpy(y[7], -kp, x[7]); caxpy(y[7], -sq2 * kq, x[2]);
      if (ax < 2) {
        caxpy(y[2], kr, x[4]);
        caxpy(y[3], kr, x[5]); caxpy(y[3], -sq2 * kr, x[6]);
        caxpy(y[4], kr, x[2]); caxpy(y[4], sq2 * kr, x[7]);
        caxpy(y[5], kr, x[3]);
        caxpy(y[6], -sq2 * kr, x[3]);
        caxpy(y[7], sq2 * kr, x[4]);
      }
      if (NB == 8) {
        // w = signed neighbour value is folded into su/sv; U w = -i su w, V w = -i sv w,
        // V^H w = -i conj(sv) w.
        const T su = r[(R_SU + f) * S];
        const cplx<T> sv = mk<T>(r[(R_SVR + f) * S], r[(R_SVI + f) * S]);
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
    // plane xy -> R (+i cR) / R^H (-i cR); plane zx -> S, S^H (cS); plane zy -> S (-i cS),
    // S^H (+i cS). Coefficient of x(p + sa e_a + sb e_b): -(sa sb)/(8h^2) (g_{sa a} + g_{sb b}).
#pragma unroll
    for (int pl = 0; pl < 3; ++pl) {
      const int ea = pl == 0 ? 0 : 2;      // xy: a = x; zx, zy: a = z
      const int eb = pl == 0 ? 1 : (pl == 1 ? 0 : 1);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int sa = (e & 1) ? -1 : 1, sb = (e & 2) ? -1 : 1;
        if (!(msk & (1u << (6 + 4 * pl + e)))) continue;
        const T ga = r[(R_G3 + 2 * ea + (sa < 0)) * S];
        const T gb = r[(R_G3 + 2 * eb + (sb < 0)) * S];
        const T c = T(2) * sq3 * G * (-(T)(sa * sb) * i8h2) * (ga + gb);
        load_site<T, NB, true>(xs, bstr, sa * str[ea] + sb * str[eb], x);
        if (pl == 0) {
          caxpy_i(y[2], c, x[4]);
          caxpy_i(y[4], -c, x[2]);
          caxpy_i(y[3], c, x[5]);
          caxpy_i(y[5], -c, x[3]);
          caxpy_i(y[3], -sq2 * c, x[6]);
          caxpy_i(y[6], sq2 * c, x[3]);
          caxpy_i(y[4], -sq2 * c, x[7]);
          caxpy_i(y[7], sq2 * c, x[4]);
        } else if (pl == 1) {
          caxpy(y[3], -c, x[2]); caxpy(y[2], sq32 * c, x[6]); caxpy(y[3], isq2 * c, x[7]);
          caxpy(y[5], c, x[4]); caxpy(y[6], isq2 * c, x[4]); caxpy(y[7], sq32 * c, x[5]);
          caxpy(y[2], -c, x[3]); caxpy(y[6], sq32 * c, x[2]); caxpy(y[7], isq2 * c, x[3]);
          caxpy(y[4], c, x[5]); caxpy(y[4], isq2 * c, x[6]); caxpy(y[5], sq32 * c, x[7]);
        } else {
          // S entries get -i c, S^H entries +i c
          caxpy_i(y[3], c, x[2]); caxpy_i(y[2], -sq32 * c, x[6]); caxpy_i(y[3], -isq2 * c, x[7]);
          caxpy_i(y[5], -c, x[4]); caxpy_i(y[6], -isq2 * c, x[4]); caxpy_i(y[7], -sq32 * c, x[5]);
          caxpy_i(y[2], -c, x[3]); caxpy_i(y[6], sq32 * c, x[2]); caxpy_i(y[7], isq2 * c, x[3]);
          caxpy_i(y[4], c, x[5]); caxpy_i(y[4], isq2 * c, x[6]); caxpy_i(y[5], sq32 * c, x[7]);
        }
      }
    }

    // ---- sign (hole convention / negation), store ---------------------------------------
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      if (!has_band<NB>(b)) continue;
      a.Y[(s * a.ldy + j) + (long long)((b - band_off<NB>()) * ystr)] = cscale(a.sign, y[b]);
    }
  }
}

template <typename T, int NB>
__global__ void __launch_bounds__(256, ApplyOcc<T>::kMinBlocks) kp_apply_kernel(const ApplyArgs<T> a) {
  extern __shared__ unsigned char smem_raw[];
  apply_tile<T, NB>(a, (long long)blockIdx.x * a.S, reinterpret_cast<T*>(smem_raw));
}

// Many operators and blocks in one launch (the batched engine): CTA b serves slot k with
// tile0[k] <= b < tile0[k+1]; the column count is read on the device (the slot's active width).
template <typename T>
__global__ void __launch_bounds__(256, ApplyOcc<T>::kMinBlocks)
kp_apply_multi_kernel(const HXSlot* __restrict__ slots, int nslots) {
  extern __shared__ unsigned char smem_raw[];
  int k = 0;
  while (k + 1 < nslots && (int)blockIdx.x >= slots[k + 1].tile0) ++k;
  const HXSlot& d = slots[k];
  if (d.skip && *d.skip) return;
  const int m = d.m_dev ? *d.m_dev : d.m;
  if (m <= 0) return;
  ApplyArgs<T> a;
  a.F = static_cast<const T*>(d.F);
  a.X = static_cast<const cplx<T>*>(d.X);
  a.Y = static_cast<cplx<T>*>(d.Y);
  a.N = d.N; a.ldx = d.ld_same ? m : d.ldx; a.ldy = d.ld_same ? m : d.ldy;
  a.nx = d.nx; a.ny = d.ny; a.nz = d.nz; a.m = m; a.flags = d.flags; a.S = d.S;
  a.h = (T)d.h; a.sigma = (T)d.sigma; a.sign = (T)d.sign; a.shifted = d.shifted;
  apply_tile<T, 8>(a, (long long)(blockIdx.x - d.tile0) * d.S, reinterpret_cast<T*>(smem_raw));
}

int launch_apply_multi(const HXSlot* slots_dev, int nslots, int total_tiles, int S_max,
                       int precision, cudaStream_t st) {
  if (total_tiles <= 0) return QDKP_OK;
  if (precision == QDKP_C128) {
    kp_apply_multi_kernel<double><<<total_tiles, 256,
        (size_t)R_COUNT * S_max * sizeof(double) + S_max * sizeof(unsigned), st>>>(slots_dev, nslots);
  } else {
    kp_apply_multi_kernel<float><<<total_tiles, 256,
        (size_t)R_COUNT * S_max * sizeof(float) + S_max * sizeof(unsigned), st>>>(slots_dev, nslots);
  }
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

int apply_tile_sites(int m) {
  int S = (512 + m - 1) / m;
  return S < 32 ? 32 : (S > 128 ? 128 : S);
}

template <typename T>
static int launch_apply_t(const qdkp_operator* op, const T* F, const void* X, int64_t ldx,
                          void* Y, int64_t ldy, int m, double sigma, int shifted,
                          cudaStream_t st) {
  if ((int64_t)op->n_bands * op->n_sites * std::max(ldx, ldy) >= (int64_t(1) << 31)) {
    set_error("H.X: n * leading dimension must stay below 2^31 elements");
    return QDKP_ERR_UNSUPPORTED;
  }
  ApplyArgs<T> a;
  a.F = F;
  a.X = static_cast<const cplx<T>*>(X);
  a.Y = static_cast<cplx<T>*>(Y);
  a.N = op->n_sites; a.ldx = ldx; a.ldy = ldy;
  a.nx = op->nx; a.ny = op->ny; a.nz = op->nz; a.m = m; a.flags = op->flags;
  a.h = (T)op->h; a.sigma = (T)sigma; a.shifted = shifted;
  a.sign = ((op->flags & QDKP_HOLE_CONVENTION) && op->n_bands != 8) ? T(-1) : T(1);
  if (op->flags & QDKP_NEGATE) a.sign = -a.sign;
  const int S = apply_tile_sites(m);
  a.S = S;
  const size_t smem = (size_t)R_COUNT * S * sizeof(T) + (size_t)S * sizeof(unsigned);
  const unsigned grid = (unsigned)((op->n_sites + S - 1) / S);
  switch (op->n_bands) {
    case 8: kp_apply_kernel<T, 8><<<grid, 256, smem, st>>>(a); break;
    case 6: kp_apply_kernel<T, 6><<<grid, 256, smem, st>>>(a); break;
    case 4: kp_apply_kernel<T, 4><<<grid, 256, smem, st>>>(a); break;
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
    return launch_apply_t<double>(op, op->fields64, X, ldx, Y, ldy, m, sigma, shifted, st);
  if (precision == QDKP_C64)
    return launch_apply_t<float>(op, op->fields32, X, ldx, Y, ldy, m, sigma, shifted, st);
  set_error("precision must be QDKP_C128 or QDKP_C64");
  return QDKP_ERR_ARG;
}

}  // namespace qdkp
