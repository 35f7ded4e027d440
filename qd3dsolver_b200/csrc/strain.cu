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

}  // namespace qdkp

using namespace qdkp;

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
