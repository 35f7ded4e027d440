// Homogeneous Fourier strain and the first-order piezoelectric potential on the device (sm_100a).
//
//   strain_fourier.solve_strain (strain_fourier.py:142-235): chi = dot mask; u_k = -i eps_T
//     (C11 + 2 C12) chi_k K(k)^-1 k with K the cubic Christoffel matrix K_ik = C_ijkl k_j k_l
//     (its inverse by cofactors, 0 where det K = 0, i.e. the k = 0 mode); total strain = the
//     symmetric spectral gradient of u; elastic = total - eps_T chi on the diagonal
//     (eps_T = -eps_star).
//   piezoelectric.potential (piezoelectric.py:59-99): P = 2 e14 (eyz, ezx, exy) sign;
//     rho = -Re ifft(i k . fft P) CHARGE_UNIT; phi = Re ifft(fft(rho) POISSON_CONST / (eps_r k^2))
//     with the k = 0 mode dropped.
// k = 2 pi fftfreq(n, h) on a C-ordered (nx, ny, nz) grid: the same periodic cell as numpy's fftn.
// The plain 3-D transforms are cuFFT double-complex plans (one per grid shape, kept for reuse,
// work area in the caller's workspace); the Christoffel inverse, the spectral derivatives, the
// Poisson filter and the real parts are this file's kernels. Every step is a fixed-order
// computation: the result does not depend on other work on the GPU.
#include <cufft.h>

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "qdkp_common.cuh"

namespace qdkp {

constexpr double kEcharge = 1.602176634e-19;                 // C (poisson_solver.py:25)
constexpr double kEps0 = 8.8541878128e-12;                   // F/m (poisson_solver.py:26)
constexpr double kPoissonConst = kEcharge * 1e9 / kEps0;     // V nm (poisson_solver.py:30)
constexpr double kChargeUnit = 1.0 / (kEcharge * 1e18);      // piezoelectric.py:50

struct Grid3 { int nx, ny, nz; double h; };

__device__ __forceinline__ double kcomp(int i, int n, double h) {
  const int f = (i <= (n - 1) / 2) ? i : i - n;                // numpy fftfreq order
  return 6.283185307179586476925286766559 * (double)f / ((double)n * h);
}

__device__ __forceinline__ void kvec(long long s, Grid3 g, double& kx, double& ky, double& kz) {
  const int iz = (int)(s % g.nz);
  const long long t = s / g.nz;
  const int iy = (int)(t % g.ny), ix = (int)(t / g.ny);
  kx = kcomp(ix, g.nx, g.h); ky = kcomp(iy, g.ny, g.h); kz = kcomp(iz, g.nz, g.h);
}

__global__ void mask_to_complex(const unsigned char* __restrict__ mask, long long N,
                                double2* __restrict__ chi) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N;
       s += (long long)gridDim.x * blockDim.x)
    chi[s] = make_double2(mask[s] ? 1.0 : 0.0, 0.0);
}

__global__ void mask_to_double(const unsigned char* __restrict__ mask, long long N,
                               double* __restrict__ chi) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N;
       s += (long long)gridDim.x * blockDim.x)
    chi[s] = mask[s] ? 1.0 : 0.0;
}

// six strain spectra from chi_k (cubic Christoffel inverse by cofactors, strain_fourier.py:142-173)
__global__ void strain_spectra(const double2* __restrict__ chik, long long N, Grid3 g,
                               double C11, double C12, double C44, double eps_T,
                               double2* __restrict__ out) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N;
       s += (long long)gridDim.x * blockDim.x) {
    double kx, ky, kz;
    kvec(s, g, kx, ky, kz);
    const double cs = C12 + C44;
    const double k11 = C11 * kx * kx + C44 * (ky * ky + kz * kz);
    const double k22 = C11 * ky * ky + C44 * (kx * kx + kz * kz);
    const double k33 = C11 * kz * kz + C44 * (kx * kx + ky * ky);
    const double k12 = cs * kx * ky, k13 = cs * kx * kz, k23 = cs * ky * kz;
    const double c11 = k22 * k33 - k23 * k23, c12 = k13 * k23 - k12 * k33;
    const double c13 = k12 * k23 - k13 * k22, c22 = k11 * k33 - k13 * k13;
    const double c23 = k12 * k13 - k11 * k23, c33 = k11 * k22 - k12 * k12;
    const double det = k11 * c11 + k12 * c12 + k13 * c13;
    const double inv = det != 0.0 ? 1.0 / det : 0.0;
    const double i11 = c11 * inv, i12 = c12 * inv, i13 = c13 * inv;
    const double i22 = c22 * inv, i23 = c23 * inv, i33 = c33 * inv;
    // pref = -i eps_T (C11 + 2 C12) chi_k
    const double a = eps_T * (C11 + 2.0 * C12);
    const double2 ck = chik[s];
    const double2 pref = make_double2(a * ck.y, -a * ck.x);
    const double gx = i11 * kx + i12 * ky + i13 * kz;
    const double gy = i12 * kx + i22 * ky + i23 * kz;
    const double gz = i13 * kx + i23 * ky + i33 * kz;
    const double2 ux = make_double2(pref.x * gx, pref.y * gx);
    const double2 uy = make_double2(pref.x * gy, pref.y * gy);
    const double2 uz = make_double2(pref.x * gz, pref.y * gz);
    // i c w = (-c w.y, c w.x)
    auto ic = [](double c, double2 w) { return make_double2(-c * w.y, c * w.x); };
    auto add = [](double2 p, double2 q) { return make_double2(p.x + q.x, p.y + q.y); };
    out[0 * N + s] = ic(kx, ux);
    out[1 * N + s] = ic(ky, uy);
    out[2 * N + s] = ic(kz, uz);
    out[3 * N + s] = ic(0.5, add(make_double2(ky * ux.x, ky * ux.y), make_double2(kx * uy.x, kx * uy.y)));
    out[4 * N + s] = ic(0.5, add(make_double2(kz * uy.x, kz * uy.y), make_double2(ky * uz.x, ky * uz.y)));
    out[5 * N + s] = ic(0.5, add(make_double2(kx * uz.x, kx * uz.y), make_double2(kz * ux.x, kz * ux.y)));
  }
}

// strain[c] = Re(spec[c]) / N - (c < 3 ? eps_T chi : 0)
__global__ void strain_real(const double2* __restrict__ spec, const unsigned char* __restrict__ mask,
                            long long N, double eps_T, double* __restrict__ strain) {
  const double invN = 1.0 / (double)N;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < 6 * N;
       e += (long long)gridDim.x * blockDim.x) {
    const long long c = e / N, s = e - c * N;
    double v = spec[e].x * invN;
    if (c < 3 && mask[s]) v -= eps_T;
    strain[e] = v;
  }
}

// P components as complex: (eyz, ezx, exy) * 2 e14 sign
__global__ void polarization_k(const double* __restrict__ strain, const double* __restrict__ e14,
                               long long N, double sign, double2* __restrict__ P) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N;
       s += (long long)gridDim.x * blockDim.x) {
    const double f = 2.0 * e14[s] * sign;
    P[s] = make_double2(f * strain[4 * N + s], 0.0);             // eyz
    P[N + s] = make_double2(f * strain[5 * N + s], 0.0);         // ezx
    P[2 * N + s] = make_double2(f * strain[3 * N + s], 0.0);     // exy
  }
}

// div_k = i kx P0 + i ky P1 + i kz P2
__global__ void divergence_k(const double2* __restrict__ P, long long N, Grid3 g,
                             double2* __restrict__ div) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N;
       s += (long long)gridDim.x * blockDim.x) {
    double kx, ky, kz;
    kvec(s, g, kx, ky, kz);
    const double2 a = P[s], b = P[N + s], c = P[2 * N + s];
    div[s] = make_double2(-(kx * a.y + ky * b.y + kz * c.y), kx * a.x + ky * b.x + kz * c.x);
  }
}

// rho = -Re(ifft div) CHARGE_UNIT, as complex input of the next forward transform
__global__ void charge_density(double2* __restrict__ d, long long N) {
  const double f = -kChargeUnit / (double)N;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N;
       s += (long long)gridDim.x * blockDim.x)
    d[s] = make_double2(d[s].x * f, 0.0);
}

__global__ void poisson_filter(double2* __restrict__ r, long long N, Grid3 g, double eps_r) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N;
       s += (long long)gridDim.x * blockDim.x) {
    double kx, ky, kz;
    kvec(s, g, kx, ky, kz);
    const double k2 = kx * kx + ky * ky + kz * kz;
    const double inv = k2 != 0.0 ? 1.0 / k2 : 0.0;
    const double f = kPoissonConst * inv / eps_r;
    r[s] = make_double2(r[s].x * f, r[s].y * f);
  }
}

__global__ void real_part(const double2* __restrict__ z, long long N, double* __restrict__ out) {
  const double invN = 1.0 / (double)N;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N;
       s += (long long)gridDim.x * blockDim.x)
    out[s] = z[s].x * invN;
}

// ---- cuFFT plans: one per (shape, batch), no automatic allocation ------------------------------
struct Plan { cufftHandle h; size_t work; };
static std::mutex g_plan_mu;
static std::map<std::tuple<int, int, int, int, int>, Plan> g_plans;

static int get_plan(int device, int nx, int ny, int nz, int batch, Plan* out) {
  std::lock_guard<std::mutex> lk(g_plan_mu);
  const auto key = std::make_tuple(device, nx, ny, nz, batch);
  auto it = g_plans.find(key);
  if (it != g_plans.end()) { *out = it->second; return QDKP_OK; }
  Plan p;
  if (cufftCreate(&p.h) != CUFFT_SUCCESS) { set_error("cufftCreate failed"); return QDKP_ERR_CUDA; }
  cufftSetAutoAllocation(p.h, 0);
  int n[3] = {nx, ny, nz};
  const long long N = (long long)nx * ny * nz;
  if (cufftMakePlanMany(p.h, 3, n, nullptr, 1, (int)N, nullptr, 1, (int)N, CUFFT_Z2Z, batch,
                        &p.work) != CUFFT_SUCCESS) {
    cufftDestroy(p.h);
    set_error("cufftMakePlanMany failed");
    return QDKP_ERR_CUDA;
  }
  g_plans[key] = p;
  *out = p;
  return QDKP_OK;
}

static int run_fft(int device, int nx, int ny, int nz, int batch, double2* data, int dir,
                   void* work, size_t work_bytes, cudaStream_t st) {
  Plan p;
  int rc = get_plan(device, nx, ny, nz, batch, &p);
  if (rc != QDKP_OK) return rc;
  if (p.work > work_bytes) { set_error("FFT work area larger than the workspace"); return QDKP_ERR_WORKSPACE; }
  std::lock_guard<std::mutex> lk(g_plan_mu);      // the plan's stream and work area are per call
  if (cufftSetStream(p.h, st) != CUFFT_SUCCESS || cufftSetWorkArea(p.h, work) != CUFFT_SUCCESS ||
      cufftExecZ2Z(p.h, reinterpret_cast<cufftDoubleComplex*>(data),
                   reinterpret_cast<cufftDoubleComplex*>(data), dir) != CUFFT_SUCCESS) {
    set_error("cufftExecZ2Z failed");
    return QDKP_ERR_CUDA;
  }
  return QDKP_OK;
}

static size_t plan_work(int device, int nx, int ny, int nz, int batch) {
  Plan p;
  if (get_plan(device, nx, ny, nz, batch, &p) != QDKP_OK) return 0;
  return p.work;
}

static int grid_blocks(long long N) { return (int)std::min<long long>((N + 255) / 256, 148 * 16); }

static size_t al(size_t b) { return (b + 255) / 256 * 256; }


// ---- inhomogeneous FD elasticity (elasticity_fd.solve_strain_fd, elasticity_fd.py:211-419) ----
// Trilinear (Q1) hexahedral elements with 2x2x2 Gauss quadrature on the periodic cell:
// displacements u (3 x N, component-major) on nodes, materials (chi in {0, 1}) and strain on
// elements; element e spans the nodes e + c for the corners c in {0,1}^3 (corner index
// 4 cx + 2 cy + cz). The stiffness of a node p gathers, over the eight elements e = p - c_a,
// sum_{b,l} K_{mat(e)}[a,b,j,l] u_l[p + c_b - c_a]: a 27-point stencil per node whose blocks
// switch between the matrix's and the dot's element arrays (computed on the host from C11, C12,
// C44 and h, elasticity_fd.py:90-153). Preconditioner: the exact inverse of the symbol of the
// volume-averaged homogeneous stencil, S(k) = sum_d Kavg_d exp(i k.d), per wavevector, zero
// where the reference's scale-free test calls it singular (elasticity_fd.py:179-241).

struct FdArrays {
  double Km[8][8][3][3];        // matrix element stiffness
  double Kd[8][8][3][3];        // dot element stiffness
  double S27[27][3][3];         // volume-averaged stencil blocks by node offset d + 1 (x, y, z)
  double Wd[8][3];              // eigenstrain load shape of a dot element
  double G0[8][3];              // shape-function gradients at the element centre
};

__device__ __forceinline__ int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// F = K u on the nodes (a thread per node, grid-stride)
__global__ void __launch_bounds__(256)
fd_apply(const double* __restrict__ u, const unsigned char* __restrict__ chi, Grid3 g,
         const FdArrays* __restrict__ arr, double* __restrict__ f) {
  __shared__ double sK[2][8][8][3][3];
  for (int t = threadIdx.x; t < 2 * 576; t += blockDim.x)
    (&sK[0][0][0][0][0])[t] = t < 576 ? (&arr->Km[0][0][0][0])[t] : (&arr->Kd[0][0][0][0])[t - 576];
  __syncthreads();
  const long long N = (long long)g.nx * g.ny * g.nz;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(p % g.nz);
    const long long t = p / g.nz;
    const int y = (int)(t % g.ny), x = (int)(t / g.ny);
    int mat[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int ex = wrapi(x - (a >> 2), g.nx), ey = wrapi(y - ((a >> 1) & 1), g.ny), ez = wrapi(z - (a & 1), g.nz);
      mat[a] = chi[((long long)ex * g.ny + ey) * g.nz + ez] ? 1 : 0;
    }
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
#pragma unroll
    for (int dx = -1; dx <= 1; ++dx)
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dz = -1; dz <= 1; ++dz) {
          const long long q = ((long long)wrapi(x + dx, g.nx) * g.ny + wrapi(y + dy, g.ny)) * g.nz + wrapi(z + dz, g.nz);
          const double u0 = u[q], u1 = u[N + q], u2 = u[2 * N + q];
#pragma unroll
          for (int a = 0; a < 8; ++a) {
            const int bx = (a >> 2) + dx, by = ((a >> 1) & 1) + dy, bz = (a & 1) + dz;
            if (bx < 0 || bx > 1 || by < 0 || by > 1 || bz < 0 || bz > 1) continue;   // compile time
            const double* K = &sK[mat[a]][a][bx * 4 + by * 2 + bz][0][0];
            f0 += K[0] * u0 + K[1] * u1 + K[2] * u2;
            f1 += K[3] * u0 + K[4] * u1 + K[5] * u2;
            f2 += K[6] * u0 + K[7] * u1 + K[8] * u2;
          }
        }
    f[p] = f0; f[N + p] = f1; f[2 * N + p] = f2;
  }
}

// the eigenstrain load F_j[p] = sum_a W_d[a, j] bulk[p - c_a], bulk = eps_T (C11 + 2 C12)_dot chi
__global__ void fd_load(const unsigned char* __restrict__ chi, Grid3 g, const FdArrays* __restrict__ arr,
                        double bulk, double* __restrict__ f) {
  const long long N = (long long)g.nx * g.ny * g.nz;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(p % g.nz);
    const long long t = p / g.nz;
    const int y = (int)(t % g.ny), x = (int)(t / g.ny);
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
    for (int a = 0; a < 8; ++a) {
      const int ex = wrapi(x - (a >> 2), g.nx), ey = wrapi(y - ((a >> 1) & 1), g.ny), ez = wrapi(z - (a & 1), g.nz);
      if (!chi[((long long)ex * g.ny + ey) * g.nz + ez]) continue;
      f0 += arr->Wd[a][0] * bulk; f1 += arr->Wd[a][1] * bulk; f2 += arr->Wd[a][2] * bulk;
    }
    f[p] = f0; f[N + p] = f1; f[2 * N + p] = f2;
  }
}

// S(k) of the averaged stencil (Hermitian; the six upper entries) at wavevector index s of the
// full (nx, ny, nz) spectrum, k = 2 pi fftfreq per axis in grid units
__device__ void fd_symbol(long long s, Grid3 g, const FdArrays* __restrict__ arr, double2 S[6]) {
  const int iz = (int)(s % g.nz);
  const long long t = s / g.nz;
  const int iy = (int)(t % g.ny), ix = (int)(t / g.ny);
  double sx, cx, sy, cy, sz, cz;
  sincos(kcomp(ix, g.nx, 1.0), &sx, &cx);
  sincos(kcomp(iy, g.ny, 1.0), &sy, &cy);
  sincos(kcomp(iz, g.nz, 1.0), &sz, &cz);
  const double2 ex[3] = {make_double2(cx, -sx), make_double2(1.0, 0.0), make_double2(cx, sx)};
  const double2 ey[3] = {make_double2(cy, -sy), make_double2(1.0, 0.0), make_double2(cy, sy)};
  const double2 ez[3] = {make_double2(cz, -sz), make_double2(1.0, 0.0), make_double2(cz, sz)};
  const int jj[6] = {0, 0, 0, 1, 1, 2}, ll[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int e = 0; e < 6; ++e) S[e] = make_double2(0.0, 0.0);
  for (int d = 0; d < 27; ++d) {
    const double2 ph = cmul(cmul(ex[d / 9], ey[(d / 3) % 3]), ez[d % 3]);
#pragma unroll
    for (int e = 0; e < 6; ++e) {
      const double kv = arr->S27[d][jj[e]][ll[e]];
      S[e].x += kv * ph.x;
      S[e].y += kv * ph.y;
    }
  }
}

// tr(S)/3 per wavevector, for the global maximum of the singularity test
__global__ void fd_symbol_trace(Grid3 g, const FdArrays* __restrict__ arr, double* __restrict__ tr) {
  const long long N = (long long)g.nx * g.ny * g.nz;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N;
       s += (long long)gridDim.x * blockDim.x) {
    double2 S[6];
    fd_symbol(s, g, arr, S);
    tr[s] = (S[0].x + S[3].x + S[5].x) / 3.0;
  }
}

// Z = Re ifft(Sinv(k) fft(R)): the spectra of the three components (batch-major) in place;
// dropped modes are counted once (count != nullptr) by the first call of a solve
__global__ void fd_precondition_k(double2* __restrict__ Rk, Grid3 g, const FdArrays* __restrict__ arr,
                                  const double* __restrict__ trmax, unsigned long long* count) {
  const long long N = (long long)g.nx * g.ny * g.nz;
  const double tmax = *trmax;
  unsigned long long dropped = 0;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N;
       s += (long long)gridDim.x * blockDim.x) {
    double2 S[6];
    fd_symbol(s, g, arr, S);
    const double2 a = S[0], b = S[1], c = S[2], d = S[3], e = S[4], f = S[5];
    const double2 bc = make_double2(b.x, -b.y), cc = make_double2(c.x, -c.y), ec = make_double2(e.x, -e.y);
    // cofactors of [[a b c] [b* d e] [c* e* f]]
    const double2 i00 = csub(cmul(d, f), cmul(e, ec));
    const double2 i01 = csub(cmul(c, ec), cmul(b, f));
    const double2 i02 = csub(cmul(b, e), cmul(c, d));
    const double2 i11 = csub(cmul(a, f), cmul(c, cc));
    const double2 i12 = csub(cmul(c, bc), cmul(a, e));
    const double2 i22 = csub(cmul(a, d), cmul(b, bc));
    const double2 det = cadd(cadd(cmul(a, i00), cmul(b, make_double2(i01.x, -i01.y))),
                             cmul(c, make_double2(i02.x, -i02.y)));
    const double tr = (a.x + d.x + f.x) / 3.0;
    const double adet = sqrt(det.x * det.x + det.y * det.y);
    const double sc = fmax(tr, 0.0);
    const bool good = tr > 1e-12 * tmax && adet > 1e-9 * sc * sc * sc;
    dropped += !good;
    const double2 r0 = Rk[s], r1 = Rk[N + s], r2 = Rk[2 * N + s];
    double2 u0 = make_double2(0.0, 0.0), u1 = u0, u2 = u0;
    if (good) {
      const double dd = det.x * det.x + det.y * det.y;
      const double2 id = make_double2(det.x / dd, -det.y / dd);
      // inverse = adj / det, adj Hermitian: rows (i00 i01 i02), (i01* i11 i12), (i02* i12* i22)
      u0 = cmul(id, cadd(cadd(cmul(i00, r0), cmul(i01, r1)), cmul(i02, r2)));
      u1 = cmul(id, cadd(cadd(cmul(make_double2(i01.x, -i01.y), r0), cmul(i11, r1)), cmul(i12, r2)));
      u2 = cmul(id, cadd(cadd(cmul(make_double2(i02.x, -i02.y), r0), cmul(make_double2(i12.x, -i12.y), r1)),
                         cmul(i22, r2)));
    }
    Rk[s] = u0; Rk[N + s] = u1; Rk[2 * N + s] = u2;
  }
  if (count && dropped) atomicAdd(count, dropped);
}

__global__ void fd_to_complex(const double* __restrict__ r, long long n3, double2* __restrict__ z) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n3;
       s += (long long)gridDim.x * blockDim.x)
    z[s] = make_double2(r[s], 0.0);
}

__global__ void fd_real_scaled(const double2* __restrict__ z, long long n3, double invN,
                               double* __restrict__ r) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n3;
       s += (long long)gridDim.x * blockDim.x)
    r[s] = z[s].x * invN;
}

// deterministic reductions: fixed-size grid of per-block partials, then one block in order
constexpr int kFdRedBlocks = 592;
constexpr int kFdRedThreads = 256;

template <int OP>       // 0: sum a b, 1: max a, 2: sum a (per component, 3 results)
__global__ void __launch_bounds__(kFdRedThreads)
fd_reduce_partial(const double* __restrict__ a, const double* __restrict__ b, long long n,
                  long long comp_n, double* __restrict__ part) {
  __shared__ double red[3][kFdRedThreads];
  double acc[3] = {0.0, 0.0, 0.0};
  if (OP == 1) acc[0] = -INFINITY;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n;
       s += (long long)gridDim.x * blockDim.x) {
    if (OP == 0) acc[0] = fma(a[s], b[s], acc[0]);
    else if (OP == 1) acc[0] = fmax(acc[0], a[s]);
    else acc[s / comp_n] += a[s];
  }
  for (int c = 0; c < 3; ++c) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int w = kFdRedThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int c = 0; c < 3; ++c)
        red[c][threadIdx.x] = OP == 1 ? fmax(red[c][threadIdx.x], red[c][threadIdx.x + w])
                                      : red[c][threadIdx.x] + red[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 3) part[threadIdx.x * kFdRedBlocks + blockIdx.x] = red[threadIdx.x][0];
}

template <int OP>
__global__ void __launch_bounds__(kFdRedThreads)
fd_reduce_final(const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double red[kFdRedThreads];
  for (int c = 0; c < (OP == 2 ? 3 : 1); ++c) {
    double acc = OP == 1 ? -INFINITY : 0.0;
    for (int i = threadIdx.x; i < kFdRedBlocks; i += blockDim.x)
      acc = OP == 1 ? fmax(acc, part[c * kFdRedBlocks + i]) : acc + part[c * kFdRedBlocks + i];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kFdRedThreads / 2; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w)
        red[threadIdx.x] = OP == 1 ? fmax(red[threadIdx.x], red[threadIdx.x + w]) : red[threadIdx.x] + red[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[c] = red[0];
    __syncthreads();
  }
}

// x += alpha p and r -= alpha q with alpha = *num / *den from device memory
__global__ void fd_cg_step(double* __restrict__ x, const double* __restrict__ p, double* __restrict__ r,
                           const double* __restrict__ q, const double* __restrict__ num,
                           const double* __restrict__ den, long long n3) {
  if (!(*den > 0.0)) return;                   // breakdown: the caller stops, x and r unchanged
  const double alpha = *num / *den;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n3;
       s += (long long)gridDim.x * blockDim.x) {
    x[s] = fma(alpha, p[s], x[s]);
    r[s] = fma(-alpha, q[s], r[s]);
  }
}

// p = z + (rz_new / rz_old) p
__global__ void fd_direction(double* __restrict__ p, const double* __restrict__ z,
                             const double* __restrict__ rz_new, const double* __restrict__ rz_old,
                             long long n3) {
  const double beta = *rz_new / *rz_old;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n3;
       s += (long long)gridDim.x * blockDim.x)
    p[s] = fma(beta, p[s], z[s]);
}

// v -= the mean of each component (means from the component sums)
__global__ void fd_remove_mean(double* __restrict__ v, const double* __restrict__ sums, long long N) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < 3 * N;
       s += (long long)gridDim.x * blockDim.x)
    v[s] -= sums[s / N] / (double)N;
}

// elastic strain at the element centres: grad_ij = sum_n G0[n, i] u_j[e + c_n]; the diagonal
// minus eps_T chi (elasticity_fd.py:343-362); out (6 x N): exx eyy ezz exy eyz ezx, and the
// total strain (optional) without the eigenstrain term
__global__ void fd_strain(const double* __restrict__ u, const unsigned char* __restrict__ chi, Grid3 g,
                          const FdArrays* __restrict__ arr, double eps_T, double* __restrict__ out,
                          double* __restrict__ total) {
  const long long N = (long long)g.nx * g.ny * g.nz;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < N;
       e += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(e % g.nz);
    const long long t = e / g.nz;
    const int y = (int)(t % g.ny), x = (int)(t / g.ny);
    double gr[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int n = 0; n < 8; ++n) {
      const long long q = ((long long)wrapi(x + (n >> 2), g.nx) * g.ny + wrapi(y + ((n >> 1) & 1), g.ny)) * g.nz
                          + wrapi(z + (n & 1), g.nz);
      const double uj[3] = {u[q], u[N + q], u[2 * N + q]};
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) gr[i][j] = fma(arr->G0[n][i], uj[j], gr[i][j]);
    }
    const double tot[6] = {gr[0][0], gr[1][1], gr[2][2], 0.5 * (gr[0][1] + gr[1][0]),
                           0.5 * (gr[1][2] + gr[2][1]), 0.5 * (gr[2][0] + gr[0][2])};
    const double off = chi[e] ? eps_T : 0.0;
    for (int c = 0; c < 6; ++c) {
      out[c * N + e] = tot[c] - (c < 3 ? off : 0.0);
      if (total) total[c * N + e] = tot[c];
    }
  }
}


// ---- host: element arrays (elasticity_fd.py:90-153) and the PCG driver (elasticity_fd.py:366-419)
// dN_n/dx_d at the local point xi of the cube [-1, 1]^3 of side h, N_n = prod (1 + s_nd xi_d) / 2
static void fd_shape_gradients(const double xi[3], double h, double G[8][3]) {
  for (int n = 0; n < 8; ++n) {
    const double sn[3] = {(n >> 2) ? 1.0 : -1.0, ((n >> 1) & 1) ? 1.0 : -1.0, (n & 1) ? 1.0 : -1.0};
    for (int d = 0; d < 3; ++d) {
      double v = 0.5 * sn[d];
      for (int e = 0; e < 3; ++e)
        if (e != d) v *= 0.5 * (1.0 + sn[e] * xi[e]);
      G[n][d] = v * (2.0 / h);
    }
  }
}

// K[a][b][j][l] = (h/2)^3 sum_gauss sum_ik C_ijkl G[a][i] G[b][k] for a cubic C, and W[a][j]
static void fd_element(double C11, double C12, double C44, double h, double K[8][8][3][3],
                       double W[8][3]) {
  double C[3][3][3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l)
          C[i][j][k][l] = C12 * (i == j) * (k == l) + C44 * ((i == k) * (j == l) + (i == l) * (j == k))
                          + (C11 - C12 - 2.0 * C44) * (i == j && j == k && k == l);
  const double w = (h / 2.0) * (h / 2.0) * (h / 2.0);
  std::memset(K, 0, sizeof(double) * 576);
  std::memset(W, 0, sizeof(double) * 24);
  for (int gq = 0; gq < 8; ++gq) {
    const double r = 1.0 / std::sqrt(3.0);
    const double xi[3] = {(gq >> 2) ? r : -r, ((gq >> 1) & 1) ? r : -r, (gq & 1) ? r : -r};
    double G[8][3];
    fd_shape_gradients(xi, h, G);
    for (int a = 0; a < 8; ++a) {
      for (int j = 0; j < 3; ++j) W[a][j] += w * G[a][j];
      for (int b = 0; b < 8; ++b)
        for (int j = 0; j < 3; ++j)
          for (int l = 0; l < 3; ++l) {
            double sacc = 0.0;
            for (int i = 0; i < 3; ++i)
              for (int k = 0; k < 3; ++k) sacc += C[i][j][k][l] * G[a][i] * G[b][k];
            K[a][b][j][l] += w * sacc;
          }
    }
  }
}

static int fd_blocks(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 8); }

}  // namespace qdkp

using namespace qdkp;

extern "C" {

size_t qdkp_fd_strain_workspace_size(int nx, int ny, int nz) {
  if (nx < 1 || ny < 1 || nz < 1) return 0;
  const long long N = (long long)nx * ny * nz;
  int dev = 0;
  cudaGetDevice(&dev);
  return 6 * al(3 * N * sizeof(double)) + al(3 * N * sizeof(double2)) + al(sizeof(FdArrays))
         + al(3 * kFdRedBlocks * sizeof(double)) + al(16 * sizeof(double)) + al(plan_work(dev, nx, ny, nz, 3))
         + 256;
}

int qdkp_fd_strain(int nx, int ny, int nz, double h, const unsigned char* mask, double eps_star,
                   const double* C_dot, const double* C_matrix, double tol, int maxiter,
                   double* strain, double* total, qdkp_fd_info* info, void* ws, size_t ws_bytes,
                   void* stream) {
  QDKP_CHECK_ARG(nx >= 1 && ny >= 1 && nz >= 1 && h > 0.0, "grid extents must be >= 1, h > 0");
  QDKP_CHECK_ARG(mask && strain && C_dot && C_matrix && info, "NULL argument");
  QDKP_CHECK_ARG(tol > 0.0 && maxiter >= 1, "tol must be > 0 and maxiter >= 1");
  const long long N = (long long)nx * ny * nz;
  QDKP_CHECK_ARG(3 * N < (1LL << 31), "grid too large for one transform");
  const size_t need = qdkp_fd_strain_workspace_size(nx, ny, nz);
  if (!ws || ws_bytes < need || need == 0) {
    set_error("qdkp_fd_strain: workspace too small (see qdkp_fd_strain_workspace_size)");
    return QDKP_ERR_WORKSPACE;
  }
  int dev = 0;
  QDKP_CUDA_TRY(cudaGetDevice(&dev));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const Grid3 g{nx, ny, nz, h};
  const long long n3 = 3 * N;
  char* p = static_cast<char*>(ws);
  auto take = [&](size_t b) { char* r = p; p += al(b); return r; };
  double* U = reinterpret_cast<double*>(take(n3 * sizeof(double)));
  double* R = reinterpret_cast<double*>(take(n3 * sizeof(double)));
  double* Z = reinterpret_cast<double*>(take(n3 * sizeof(double)));
  double* P = reinterpret_cast<double*>(take(n3 * sizeof(double)));
  double* AP = reinterpret_cast<double*>(take(n3 * sizeof(double)));
  double* F = reinterpret_cast<double*>(take(n3 * sizeof(double)));
  double2* Ck = reinterpret_cast<double2*>(take(n3 * sizeof(double2)));
  FdArrays* dArr = reinterpret_cast<FdArrays*>(take(sizeof(FdArrays)));
  double* part = reinterpret_cast<double*>(take(3 * kFdRedBlocks * sizeof(double)));
  double* sc = reinterpret_cast<double*>(take(16 * sizeof(double)));
  char* work = p;
  const size_t work_bytes = ws_bytes - (size_t)(p - static_cast<char*>(ws));
  // scalars: 0 ||F||^2, 1 r.z (current), 2 r.z (new), 3 p.Ap, 4 r.r, 5 trmax, 6..8 sums, 9 f
  unsigned long long* dropped = reinterpret_cast<unsigned long long*>(sc + 12);
  const int B = fd_blocks(N), B3 = fd_blocks(n3);
  auto reduce = [&](int op, const double* a, const double* b, long long n, double* out) {
    if (op == 0) fd_reduce_partial<0><<<kFdRedBlocks, kFdRedThreads, 0, st>>>(a, b, n, N, part);
    else if (op == 1) fd_reduce_partial<1><<<kFdRedBlocks, kFdRedThreads, 0, st>>>(a, b, n, N, part);
    else fd_reduce_partial<2><<<kFdRedBlocks, kFdRedThreads, 0, st>>>(a, b, n, N, part);
    if (op == 0) fd_reduce_final<0><<<1, kFdRedThreads, 0, st>>>(part, out);
    else if (op == 1) fd_reduce_final<1><<<1, kFdRedThreads, 0, st>>>(part, out);
    else fd_reduce_final<2><<<1, kFdRedThreads, 0, st>>>(part, out);
    count_launch(2);
  };
  // ---- element arrays; the preconditioner averages the materials by the dot's volume fraction
  FdArrays h_arr;
  double Wm[8][3];
  fd_element(C_matrix[0], C_matrix[1], C_matrix[2], h, h_arr.Km, Wm);
  fd_element(C_dot[0], C_dot[1], C_dot[2], h, h_arr.Kd, h_arr.Wd);
  {
    const double xi0[3] = {0.0, 0.0, 0.0};
    fd_shape_gradients(xi0, h, h_arr.G0);
  }
  // volume fraction: sum of the mask (as doubles, through Z)
  mask_to_double<<<B, 256, 0, st>>>(mask, N, Z);
  count_launch();
  reduce(2, Z, nullptr, N, sc + 6);       // component 0 holds the count
  double hsc[16];
  QDKP_CUDA_TRY(cudaMemcpyAsync(hsc, sc, 16 * sizeof(double), cudaMemcpyDeviceToHost, st));
  QDKP_CUDA_TRY(cudaStreamSynchronize(st));
  const double frac = hsc[6] / (double)N;
  std::memset(h_arr.S27, 0, sizeof(h_arr.S27));
  for (int a = 0; a < 8; ++a)
    for (int b = 0; b < 8; ++b) {
      const int dx = (b >> 2) - (a >> 2), dy = ((b >> 1) & 1) - ((a >> 1) & 1), dz = (b & 1) - (a & 1);
      const int d = (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1);
      for (int j = 0; j < 3; ++j)
        for (int l = 0; l < 3; ++l)
          h_arr.S27[d][j][l] += h_arr.Km[a][b][j][l] + frac * (h_arr.Kd[a][b][j][l] - h_arr.Km[a][b][j][l]);
    }
  QDKP_CUDA_TRY(cudaMemcpyAsync(dArr, &h_arr, sizeof(FdArrays), cudaMemcpyHostToDevice, st));
  // max over k of tr(S)/3, and the dropped-mode counter
  fd_symbol_trace<<<B, 256, 0, st>>>(g, dArr, Z);
  count_launch();
  reduce(1, Z, nullptr, N, sc + 5);
  QDKP_CUDA_TRY(cudaMemsetAsync(dropped, 0, sizeof(unsigned long long), st));
  // ---- load, projected; R = F, U = 0
  const double eps_T = -eps_star;
  fd_load<<<B, 256, 0, st>>>(mask, g, dArr, eps_T * (C_dot[0] + 2.0 * C_dot[1]), F);
  count_launch();
  reduce(2, F, nullptr, n3, sc + 6);
  fd_remove_mean<<<B3, 256, 0, st>>>(F, sc + 6, N);
  count_launch();
  QDKP_CUDA_TRY(cudaMemsetAsync(U, 0, n3 * sizeof(double), st));
  QDKP_CUDA_TRY(cudaMemcpyAsync(R, F, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
  reduce(0, F, F, n3, sc + 0);
  int rc;
  // Z = M R
  auto precondition = [&](bool count_modes) -> int {
    fd_to_complex<<<B3, 256, 0, st>>>(R, n3, Ck);
    count_launch();
    int r2 = run_fft(dev, nx, ny, nz, 3, Ck, CUFFT_FORWARD, work, work_bytes, st);
    if (r2 != QDKP_OK) return r2;
    fd_precondition_k<<<B, 256, 0, st>>>(Ck, g, dArr, sc + 5, count_modes ? dropped : nullptr);
    count_launch();
    if ((r2 = run_fft(dev, nx, ny, nz, 3, Ck, CUFFT_INVERSE, work, work_bytes, st)) != QDKP_OK) return r2;
    fd_real_scaled<<<B3, 256, 0, st>>>(Ck, n3, 1.0 / (double)N, Z);
    count_launch();
    return QDKP_OK;
  };
  if ((rc = precondition(true)) != QDKP_OK) return rc;
  QDKP_CUDA_TRY(cudaMemcpyAsync(P, Z, n3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
  reduce(0, R, Z, n3, sc + 1);
  QDKP_CUDA_TRY(cudaMemcpyAsync(hsc, sc, 16 * sizeof(double), cudaMemcpyDeviceToHost, st));
  QDKP_CUDA_TRY(cudaStreamSynchronize(st));
  unsigned long long hdrop = 0;
  QDKP_CUDA_TRY(cudaMemcpy(&hdrop, dropped, sizeof(hdrop), cudaMemcpyDeviceToHost));
  const double fnorm = std::sqrt(hsc[0]);
  int it = 0, breakdown = 0;
  double rel = 1.0;
  if (fnorm == 0.0) {
    rel = 0.0;
  } else if (!(hsc[1] > 0.0)) {
    breakdown = 1;                                        // preconditioner not positive definite
  } else {
    // r.z of the current direction in sc[irz]; each iteration writes the new one to sc[irzn]
    int irz = 1, irzn = 2;
    for (it = 1; it <= maxiter; ++it) {
      fd_apply<<<B, 256, 0, st>>>(P, mask, g, dArr, AP);
      count_launch();
      reduce(0, P, AP, n3, sc + 3);
      fd_cg_step<<<B3, 256, 0, st>>>(U, P, R, AP, sc + irz, sc + 3, n3);
      count_launch();
      reduce(0, R, R, n3, sc + 4);
      if ((rc = precondition(false)) != QDKP_OK) return rc;
      reduce(0, R, Z, n3, sc + irzn);
      QDKP_CUDA_TRY(cudaMemcpyAsync(hsc, sc, 6 * sizeof(double), cudaMemcpyDeviceToHost, st));
      QDKP_CUDA_TRY(cudaStreamSynchronize(st));
      if (!(hsc[3] > 0.0)) { breakdown = 2; break; }    // non-positive curvature (step skipped)
      rel = std::sqrt(hsc[4]) / fnorm;
      if (rel < tol) break;
      if (!(hsc[irzn] > 0.0)) { breakdown = 3; break; } // preconditioner lost definiteness
      fd_direction<<<B3, 256, 0, st>>>(P, Z, sc + irzn, sc + irz, n3);
      count_launch();
      std::swap(irz, irzn);
    }
    if (it > maxiter) it = maxiter;
  }
  // ---- project U, strain at the element centres
  reduce(2, U, nullptr, n3, sc + 6);
  fd_remove_mean<<<B3, 256, 0, st>>>(U, sc + 6, N);
  count_launch();
  fd_strain<<<B, 256, 0, st>>>(U, mask, g, dArr, eps_T, strain, total);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  QDKP_CUDA_TRY(cudaStreamSynchronize(st));
  info->iterations = it;
  info->residual = rel;
  info->modes_dropped = (int)hdrop;
  info->breakdown = breakdown;
  info->converged = rel < tol && !breakdown && hdrop <= 1;
  return QDKP_OK;
}

}  // extern "C"

extern "C" {

size_t qdkp_fourier_strain_workspace_size(int nx, int ny, int nz) {
  if (nx < 1 || ny < 1 || nz < 1) return 0;
  const long long N = (long long)nx * ny * nz;
  int dev = 0;
  cudaGetDevice(&dev);
  const size_t w = std::max(plan_work(dev, nx, ny, nz, 1), plan_work(dev, nx, ny, nz, 6));
  const size_t w3 = plan_work(dev, nx, ny, nz, 3);
  return al(7 * N * sizeof(double2)) + al(std::max(w, w3)) + 256;
}

int qdkp_fourier_strain(int nx, int ny, int nz, double h, const unsigned char* mask,
                        double eps_star, double C11, double C12, double C44, double* strain,
                        void* ws, size_t ws_bytes, void* stream) {
  QDKP_CHECK_ARG(nx >= 1 && ny >= 1 && nz >= 1 && h > 0.0, "grid extents must be >= 1, h > 0");
  QDKP_CHECK_ARG(mask && strain, "NULL argument");
  const long long N = (long long)nx * ny * nz;
  QDKP_CHECK_ARG(N < (1LL << 31), "grid too large for one transform");
  const size_t need = qdkp_fourier_strain_workspace_size(nx, ny, nz);
  if (!ws || ws_bytes < need || need == 0) {
    set_error("qdkp_fourier_strain: workspace too small (see qdkp_fourier_strain_workspace_size)");
    return QDKP_ERR_WORKSPACE;
  }
  int dev = 0;
  QDKP_CUDA_TRY(cudaGetDevice(&dev));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double2* chi = static_cast<double2*>(ws);
  double2* spec = chi + N;                                     // 6 N
  char* work = reinterpret_cast<char*>(ws) + al(7 * N * sizeof(double2));
  const size_t work_bytes = ws_bytes - al(7 * N * sizeof(double2));
  const Grid3 g{nx, ny, nz, h};
  const double eps_T = -eps_star;
  const int B = grid_blocks(N);
  mask_to_complex<<<B, 256, 0, st>>>(mask, N, chi);
  count_launch();
  int rc = run_fft(dev, nx, ny, nz, 1, chi, CUFFT_FORWARD, work, work_bytes, st);
  if (rc != QDKP_OK) return rc;
  strain_spectra<<<B, 256, 0, st>>>(chi, N, g, C11, C12, C44, eps_T, spec);
  count_launch();
  rc = run_fft(dev, nx, ny, nz, 6, spec, CUFFT_INVERSE, work, work_bytes, st);
  if (rc != QDKP_OK) return rc;
  strain_real<<<grid_blocks(6 * N), 256, 0, st>>>(spec, mask, N, eps_T, strain);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

size_t qdkp_piezo_potential_workspace_size(int nx, int ny, int nz) {
  return qdkp_fourier_strain_workspace_size(nx, ny, nz);
}

int qdkp_piezo_potential(int nx, int ny, int nz, double h, const double* strain,
                         const double* e14, double eps_r, double sign, double* phi, void* ws,
                         size_t ws_bytes, void* stream) {
  QDKP_CHECK_ARG(nx >= 1 && ny >= 1 && nz >= 1 && h > 0.0, "grid extents must be >= 1, h > 0");
  QDKP_CHECK_ARG(strain && e14 && phi, "NULL argument");
  QDKP_CHECK_ARG(eps_r > 0.0, "eps_r must be positive");
  const long long N = (long long)nx * ny * nz;
  QDKP_CHECK_ARG(N < (1LL << 31), "grid too large for one transform");
  const size_t need = qdkp_piezo_potential_workspace_size(nx, ny, nz);
  if (!ws || ws_bytes < need || need == 0) {
    set_error("qdkp_piezo_potential: workspace too small (see qdkp_piezo_potential_workspace_size)");
    return QDKP_ERR_WORKSPACE;
  }
  int dev = 0;
  QDKP_CUDA_TRY(cudaGetDevice(&dev));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double2* P = static_cast<double2*>(ws);                      // 3 N
  double2* D = P + 3 * N;                                      // N
  char* work = reinterpret_cast<char*>(ws) + al(7 * N * sizeof(double2));
  const size_t work_bytes = ws_bytes - al(7 * N * sizeof(double2));
  const Grid3 g{nx, ny, nz, h};
  const int B = grid_blocks(N);
  polarization_k<<<B, 256, 0, st>>>(strain, e14, N, sign, P);
  count_launch();
  int rc = run_fft(dev, nx, ny, nz, 3, P, CUFFT_FORWARD, work, work_bytes, st);
  if (rc != QDKP_OK) return rc;
  divergence_k<<<B, 256, 0, st>>>(P, N, g, D);
  count_launch();
  if ((rc = run_fft(dev, nx, ny, nz, 1, D, CUFFT_INVERSE, work, work_bytes, st)) != QDKP_OK) return rc;
  charge_density<<<B, 256, 0, st>>>(D, N);
  count_launch();
  if ((rc = run_fft(dev, nx, ny, nz, 1, D, CUFFT_FORWARD, work, work_bytes, st)) != QDKP_OK) return rc;
  poisson_filter<<<B, 256, 0, st>>>(D, N, g, eps_r);
  count_launch();
  if ((rc = run_fft(dev, nx, ny, nz, 1, D, CUFFT_INVERSE, work, work_bytes, st)) != QDKP_OK) return rc;
  real_part<<<B, 256, 0, st>>>(D, N, phi);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  return QDKP_OK;
}

}  // extern "C"
