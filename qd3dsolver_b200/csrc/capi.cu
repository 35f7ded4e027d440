// extern "C" entry points of libqdkp.so: operator lifecycle and H.X application.
// The LOBPCG entry points live in lobpcg.cu.
#include <atomic>
#include <cstring>
#include <string>
#include <vector>

#include "qdkp_common.cuh"

namespace qdkp {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
static std::atomic<long long> g_launches{0};
void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launches_so_far() { return g_launches.load(); }

int launch_apply(const qdkp_operator* op, const void* X, int64_t ldx, void* Y, int64_t ldy,
                 int m, double sigma, int shifted, int precision, cudaStream_t st);

// Nonzero count of the CSR the reference assembles, counted from the stencil structure: each
// (row band, column band) block couples a site to the offsets its operators reach, clipped at
// the walls. First-derivative blocks reach the six faces, except that without strain U only
// reaches z faces and V only x/y faces (kp_pryor.py:436-437); VB-VB blocks reach faces where
// they carry a k2 (P, Q, the K part of R) and in-plane edges where they carry a cross term.
static int64_t count_nnz(int nx_, int ny_, int nz_, int n_bands, int flags) {
  const long long nx = nx_, ny = ny_, nz = nz_;
  const long long N = nx * ny * nz;
  const long long faces[3] = {(nx - 1) * ny * nz, nx * (ny - 1) * nz, nx * ny * (nz - 1)};
  const long long edges_xy = 2 * (nx - 1) * (ny - 1) * nz;   // per diagonal direction pair
  const long long edges_zx = 2 * (nx - 1) * ny * (nz - 1);
  const long long edges_zy = 2 * nx * (ny - 1) * (nz - 1);
  const bool strain = flags & QDKP_STRAIN;
  const bool inter = strain && (flags & QDKP_INTERBAND_STRAIN);
  // offsets used by each operator: bit0 centre, bit1..3 faces x,y,z, bit4..6 edges xy,zx,zy
  enum { C = 1, FX = 2, FY = 4, FZ = 8, EXY = 16, EZX = 32, EZY = 64 };
  const int oA = C | FX | FY | FZ, oP = C | FX | FY | FZ, oQ = C | FX | FY | FZ;
  const int oR = C | FX | FY | EXY;   // k2x - k2y reaches x/y faces only; strain adds centre
  const int oS = EZX | EZY | (strain ? C : 0);
  const int oQmix = FX | FY | FZ | C;
  const int oU = inter ? (FX | FY | FZ) : FZ;
  const int oV = inter ? (FX | FY | FZ) : (FX | FY);
  int blk[8][8];
  for (int i = 0; i < 8; ++i) for (int j = 0; j < 8; ++j) blk[i][j] = 0;
  auto set = [&](int i, int j, int o) { blk[i][j] |= o; blk[j][i] |= o; };
  set(0, 0, oA); set(1, 1, oA);
  set(0, 2, oV); set(0, 4, oV); set(0, 5, oU); set(0, 6, oU); set(0, 7, oV);
  set(1, 2, oU); set(1, 3, oV); set(1, 5, oV); set(1, 6, oV); set(1, 7, oU);
  set(2, 2, oP | oQ); set(2, 3, oS); set(2, 4, oR); set(2, 6, oS); set(2, 7, oQmix);
  set(3, 3, oP | oQ); set(3, 5, oR); set(3, 6, oR); set(3, 7, oS);
  set(4, 4, oP | oQ); set(4, 5, oS); set(4, 6, oS); set(4, 7, oR);
  set(5, 5, oP | oQ); set(5, 6, oQmix); set(5, 7, oS);
  set(6, 6, oP); set(7, 7, oP);
  const int lo = n_bands == 8 ? 0 : 2;
  const int hi = n_bands == 4 ? 6 : 8;
  int64_t total = 0;
  for (int i = lo; i < hi; ++i)
    for (int j = lo; j < hi; ++j) {
      const int o = blk[i][j];
      if (o & C) total += N;
      if (o & FX) total += 2 * faces[0];
      if (o & FY) total += 2 * faces[1];
      if (o & FZ) total += 2 * faces[2];
      if (o & EXY) total += 2 * edges_xy;
      if (o & EZX) total += 2 * edges_zx;
      if (o & EZY) total += 2 * edges_zy;
    }
  return total;
}

}  // namespace qdkp

using namespace qdkp;

extern "C" {

const char* qdkp_last_error(void) { return g_last_error.c_str(); }

int64_t qdkp_kernel_launches(void) { return g_launches.load(); }

const char* qdkp_version(void) { return "qdkp 0.1 sm_100a"; }

int qdkp_operator_create(int nx, int ny, int nz, double h, int n_bands, int flags,
                         const double* const* fields, int device, qdkp_operator** out) {
  QDKP_CHECK_ARG(out != nullptr, "out must not be NULL");
  *out = nullptr;
  QDKP_CHECK_ARG(nx > 0 && ny > 0 && nz > 0, "grid extents must be positive");
  QDKP_CHECK_ARG(h > 0.0, "grid spacing h must be positive");
  QDKP_CHECK_ARG(n_bands == 8 || n_bands == 6 || n_bands == 4, "n_bands must be 8, 6 or 4");
  QDKP_CHECK_ARG(fields != nullptr, "fields must not be NULL");
  const bool strain = flags & QDKP_STRAIN;
  for (int f = 0; f < F_COUNT; ++f) {
    const bool needed = f <= F_G3 || f == F_EC || f == F_EV || f == F_DSO ||
                        (f == F_P0 && n_bands == 8) ||
                        (strain && (f == F_B || f == F_D || f >= F_EXX));
    if (needed && fields[f] == nullptr) {
      set_error("coefficient field " + std::to_string(f) + " is required but NULL");
      return QDKP_ERR_ARG;
    }
  }
  QDKP_CUDA_TRY(cudaSetDevice(device));
  auto* op = new qdkp_operator();
  op->fields64 = nullptr; op->rec64 = nullptr; op->rec32 = nullptr; op->nbmask = nullptr;
  op->staged_cfg[0] = op->staged_cfg[1] = -1;
  op->nx = nx; op->ny = ny; op->nz = nz;
  op->n_sites = (int64_t)nx * ny * nz;
  op->h = h; op->n_bands = n_bands; op->flags = flags; op->device = device;
  const size_t bytes64 = (size_t)F_COUNT * op->n_sites * sizeof(double);
  op->nzp = (nz + 3) / 4 * 4;
  const size_t rec_doubles = record_doubles(nx, ny, op->nzp);
  cudaError_t e = cudaMalloc(&op->fields64, bytes64);
  if (e == cudaSuccess) e = cudaMalloc(&op->rec64, rec_doubles * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&op->rec32, rec_doubles * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&op->nbmask, (size_t)op->n_sites * sizeof(unsigned));
  // the z padding of the record stays zero
  if (e == cudaSuccess) e = cudaMemset(op->rec64, 0, rec_doubles * sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(op->rec32, 0, rec_doubles * sizeof(float));
  if (e != cudaSuccess) {
    set_error(std::string("cudaMalloc of operator fields: ") + cudaGetErrorString(e));
    qdkp_operator_destroy(op);
    return QDKP_ERR_CUDA;
  }
  for (int f = 0; f < F_COUNT; ++f) {
    double* dst = op->fields64 + (size_t)f * op->n_sites;
    const size_t nb = (size_t)op->n_sites * sizeof(double);
    e = fields[f] ? cudaMemcpy(dst, fields[f], nb, cudaMemcpyHostToDevice)
                  : cudaMemset(dst, 0, nb);
    if (e != cudaSuccess) break;
  }
  if (e != cudaSuccess) {
    set_error(std::string("uploading operator fields: ") + cudaGetErrorString(e));
    qdkp_operator_destroy(op);
    return QDKP_ERR_CUDA;
  }
  int rc = build_records(op);
  if (rc != QDKP_OK) { qdkp_operator_destroy(op); return rc; }
  op->nnz_equiv = count_nnz(nx, ny, nz, n_bands, flags);
  *out = op;
  return QDKP_OK;
}

int qdkp_operator_update_diagonal(qdkp_operator* op, const double* Ec, const double* Ev) {
  QDKP_CHECK_ARG(op != nullptr, "operator must not be NULL");
  QDKP_CUDA_TRY(cudaSetDevice(op->device));
  const size_t nb = (size_t)op->n_sites * sizeof(double);
  if (Ec) QDKP_CUDA_TRY(cudaMemcpy(op->fields64 + (size_t)F_EC * op->n_sites, Ec, nb,
                                   cudaMemcpyHostToDevice));
  if (Ev) QDKP_CUDA_TRY(cudaMemcpy(op->fields64 + (size_t)F_EV * op->n_sites, Ev, nb,
                                   cudaMemcpyHostToDevice));
  return build_records(op);
}

int qdkp_operator_info(const qdkp_operator* op, int* nx, int* ny, int* nz, int* n_bands,
                       int64_t* n, int64_t* nnz) {
  QDKP_CHECK_ARG(op != nullptr, "operator must not be NULL");
  if (nx) *nx = op->nx;
  if (ny) *ny = op->ny;
  if (nz) *nz = op->nz;
  if (n_bands) *n_bands = op->n_bands;
  if (n) *n = (int64_t)op->n_bands * op->n_sites;
  if (nnz) *nnz = op->nnz_equiv;
  return QDKP_OK;
}

int64_t qdkp_structural_nnz(int nx, int ny, int nz, int n_bands, int flags) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || (n_bands != 8 && n_bands != 6 && n_bands != 4)) {
    set_error("qdkp_structural_nnz: bad grid or band count");
    return -1;
  }
  return count_nnz(nx, ny, nz, n_bands, flags);
}

int qdkp_operator_destroy(qdkp_operator* op) {
  if (!op) return QDKP_OK;
  cudaSetDevice(op->device);
  cudaFree(op->fields64);
  cudaFree(op->rec64);
  cudaFree(op->rec32);
  cudaFree(op->nbmask);
  delete op;
  return QDKP_OK;
}

int qdkp_apply(const qdkp_operator* op, const void* X, int64_t ldx, void* Y, int64_t ldy,
               int m, double sigma, int mode, int precision, void* ws, size_t ws_bytes,
               void* stream) {
  QDKP_CHECK_ARG(op != nullptr && X != nullptr && Y != nullptr, "NULL operator or block");
  QDKP_CHECK_ARG(m > 0 && ldx >= m && ldy >= m, "need m > 0 and leading dimensions >= m");
  QDKP_CHECK_ARG(mode >= QDKP_APPLY_PLAIN && mode <= QDKP_APPLY_FOLDED, "bad apply mode");
  QDKP_CHECK_ARG(precision == QDKP_C128 || precision == QDKP_C64, "bad precision");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (mode != QDKP_APPLY_FOLDED)
    return launch_apply(op, X, ldx, Y, ldy, m, sigma, mode == QDKP_APPLY_SHIFTED, precision, st);
  const size_t esz = precision == QDKP_C128 ? 16 : 8;
  const int64_t n = (int64_t)op->n_bands * op->n_sites;
  if (ws == nullptr || ws_bytes < (size_t)n * m * esz) {
    set_error("folded apply needs a workspace of n * m complex elements");
    return QDKP_ERR_WORKSPACE;
  }
  int rc = launch_apply(op, X, ldx, ws, m, m, sigma, 1, precision, st);
  if (rc != QDKP_OK) return rc;
  return launch_apply(op, ws, m, Y, ldy, m, sigma, 1, precision, st);
}

size_t qdkp_apply_host_workspace_size(const qdkp_operator* op, int m, int mode) {
  if (!op || m <= 0) return 0;
  const size_t blk = (size_t)op->n_bands * op->n_sites * m * 16;
  return (mode == QDKP_APPLY_FOLDED ? 3 : 2) * blk;
}

int qdkp_apply_host(const qdkp_operator* op, const void* X_host, void* Y_host, int m,
                    double sigma, int mode, void* ws, size_t ws_bytes, void* stream) {
  QDKP_CHECK_ARG(op != nullptr && X_host != nullptr && Y_host != nullptr, "NULL argument");
  QDKP_CHECK_ARG(m > 0, "m must be positive");
  const size_t need = qdkp_apply_host_workspace_size(op, m, mode);
  if (ws == nullptr || ws_bytes < need) {
    set_error("qdkp_apply_host: workspace too small");
    return QDKP_ERR_WORKSPACE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t blk = (size_t)op->n_bands * op->n_sites * m * 16;
  char* base = static_cast<char*>(ws);
  void* dX = base;
  void* dY = base + blk;
  void* dT = mode == QDKP_APPLY_FOLDED ? base + 2 * blk : nullptr;
  QDKP_CUDA_TRY(cudaMemcpyAsync(dX, X_host, blk, cudaMemcpyHostToDevice, st));
  int rc = qdkp_apply(op, dX, m, dY, m, m, sigma, mode, QDKP_C128, dT, dT ? blk : 0, stream);
  if (rc != QDKP_OK) return rc;
  QDKP_CUDA_TRY(cudaMemcpyAsync(Y_host, dY, blk, cudaMemcpyDeviceToHost, st));
  QDKP_CUDA_TRY(cudaStreamSynchronize(st));
  return QDKP_OK;
}

}  // extern "C"
