// Local band edges of the strained eight-band model on the device (sm_100a): the sigma providers
// of the folded solves.
//
//   kp_pryor.local_band_edges (kp_pryor.py:469-531): at k = 0 the eight-band matrix splits into
//     the conduction band (Ec) and a 6x6 Hermitian valence block built from -P = Ev (the
//     hydrostatic shift already in Ev), the Bir-Pikus terms Q, R, S of the local strain
//     (kp_pryor.py:74-114) and the spin-orbit splitting; its eigenvalues come in Kramers pairs,
//     v1 >= v2 >= v3 being the three levels (the top one, v1, is the local valence-band edge).
//   kp_pryor.hole_sigma (kp_pryor.py:156-191): the largest v1 inside the dot, plus a margin.
//
// One thread per site builds the valence block in registers (rows/columns 2..7 of Pryor's table
// at k = 0, kp_pryor.py:244-301, lower triangle the adjoint) and diagonalises it by cyclic
// complex Jacobi rotations (each rotation zeroes one off-diagonal pair exactly; sweeps stop once
// the off-diagonal mass is below eps^2 of the diagonal's). Every CTA then reduces its sites' v1
// over the mask and the Kramers splittings to one maximum each; a last CTA takes the maxima of
// those (a maximum does not depend on the order).
#include <algorithm>

#include "qdkp_common.cuh"

namespace qdkp {

constexpr int kEdgeThreads = 128;
constexpr int kEdgeMaxParts = 2368;

__device__ __forceinline__ void jacobi_rotate(double2 (&a)[6][6], int p, int q) {
  const double2 apq = a[p][q];
  const double mag = sqrt(apq.x * apq.x + apq.y * apq.y);
  if (mag == 0.0) return;
  const double ex = apq.x / mag, ey = apq.y / mag;          // e = a_pq / |a_pq|
  const double alpha = a[p][p].x, beta = a[q][q].x;
  const double tau = (beta - alpha) / (2.0 * mag);
  const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
  const double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
  // G = I except G_pp = c, G_pq = s e, G_qp = -s conj(e), G_qq = c; A <- G^H A G zeroes a_pq
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    if (r == p || r == q) continue;
    const double2 arp = a[r][p], arq = a[r][q];
    // a_rp' = c a_rp - s conj(e) a_rq ; a_rq' = s e a_rp + c a_rq
    const double2 np_ = make_double2(c * arp.x - s * (ex * arq.x + ey * arq.y),
                                     c * arp.y - s * (ex * arq.y - ey * arq.x));
    const double2 nq_ = make_double2(s * (ex * arp.x - ey * arp.y) + c * arq.x,
                                     s * (ex * arp.y + ey * arp.x) + c * arq.y);
    a[r][p] = np_; a[r][q] = nq_;
    a[p][r] = make_double2(np_.x, -np_.y); a[q][r] = make_double2(nq_.x, -nq_.y);
  }
  a[p][p] = make_double2(alpha - t * mag, 0.0);
  a[q][q] = make_double2(beta + t * mag, 0.0);
  a[p][q] = make_double2(0.0, 0.0);
  a[q][p] = make_double2(0.0, 0.0);
}

// Eigenvalues (ascending) of the k = 0 valence block of one site.
__device__ __forceinline__ void valence_levels(const double* __restrict__ F, long long N,
                                               long long s, double (&ev)[6]) {
  const double sq2 = 1.41421356237309504880, sq3 = 1.73205080756887729353;
  const double sq32 = 1.22474487139158904910;
  const double exx = F[F_EXX * N + s], eyy = F[F_EYY * N + s], ezz = F[F_EZZ * N + s];
  const double exy = F[F_EXY * N + s], eyz = F[F_EYZ * N + s], ezx = F[F_EZX * N + s];
  const double b = F[F_B * N + s], d = F[F_D * N + s];
  const double P = -F[F_EV * N + s], Dl = F[F_DSO * N + s];
  const double q = -(b / 2.0) * (exx + eyy - 2.0 * ezz);                       // Q_eps
  const double2 r = make_double2((sq3 / 2.0) * b * (exx - eyy), -d * exy);      // R_eps
  const double2 sv = make_double2(-d * ezx, d * eyz);                          // S_eps
  const double2 z = make_double2(0.0, 0.0);
  auto cj = [](double2 v) { return make_double2(v.x, -v.y); };
  auto sc = [](double k, double2 v) { return make_double2(k * v.x, k * v.y); };
  double2 a[6][6];
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) a[i][j] = z;
  // upper triangle of rows/columns 2..7 of Pryor's table at k = 0 (U = V = 0)
  a[0][0] = make_double2(-P + q, 0.0); a[0][1] = sc(-1.0, cj(sv)); a[0][2] = r;
  a[0][4] = sc(sq32, sv); a[0][5] = make_double2(-sq2 * q, 0.0);
  a[1][1] = make_double2(-P - q, 0.0); a[1][3] = r; a[1][4] = sc(-sq2, r);
  a[1][5] = sc(1.0 / sq2, sv);
  a[2][2] = make_double2(-P - q, 0.0); a[2][3] = cj(sv); a[2][4] = sc(1.0 / sq2, cj(sv));
  a[2][5] = sc(sq2, cj(r));
  a[3][3] = make_double2(-P + q, 0.0); a[3][4] = make_double2(sq2 * q, 0.0);
  a[3][5] = sc(sq32, cj(sv));
  a[4][4] = make_double2(-P - Dl, 0.0); a[5][5] = make_double2(-P - Dl, 0.0);
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = i + 1; j < 6; ++j) a[j][i] = cj(a[i][j]);
  for (int sweep = 0; sweep < 12; ++sweep) {
    double off = 0.0, dia = 0.0;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      dia += a[i][i].x * a[i][i].x;
#pragma unroll
      for (int j = i + 1; j < 6; ++j) off += a[i][j].x * a[i][j].x + a[i][j].y * a[i][j].y;
    }
    if (off <= 1e-32 * dia || off == 0.0) break;
#pragma unroll
    for (int p = 0; p < 5; ++p)
#pragma unroll
      for (int qq = p + 1; qq < 6; ++qq) jacobi_rotate(a, p, qq);
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) ev[i] = a[i][i].x;
  // sort ascending (six values)
#pragma unroll
  for (int i = 0; i < 5; ++i)
#pragma unroll
    for (int j = 0; j < 5 - i; ++j) {
      const double lo = fmin(ev[j], ev[j + 1]), hi = fmax(ev[j], ev[j + 1]);
      ev[j] = lo; ev[j + 1] = hi;
    }
}

// levels: v1, v2, v3 (3 x N, may be NULL); part: per CTA {max v1 over the mask, max split}
__global__ void __launch_bounds__(kEdgeThreads)
band_edge_kernel(const double* __restrict__ F, long long N, const unsigned char* __restrict__ mask,
                 double* __restrict__ levels, double* __restrict__ part) {
  __shared__ double s_top[kEdgeThreads], s_split[kEdgeThreads];
  double top = -INFINITY, split = 0.0;
  for (long long s = blockIdx.x * (long long)kEdgeThreads + threadIdx.x; s < N;
       s += (long long)gridDim.x * kEdgeThreads) {
    double ev[6];
    valence_levels(F, N, s, ev);
    if (levels) {
      levels[s] = ev[5];
      levels[N + s] = ev[3];
      levels[2 * N + s] = ev[1];
    }
    if (!mask || mask[s]) top = fmax(top, ev[5]);
    split = fmax(split, fmax(ev[1] - ev[0], fmax(ev[3] - ev[2], ev[5] - ev[4])));
  }
  s_top[threadIdx.x] = top;
  s_split[threadIdx.x] = split;
  __syncthreads();
  for (int o = kEdgeThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      s_top[threadIdx.x] = fmax(s_top[threadIdx.x], s_top[threadIdx.x + o]);
      s_split[threadIdx.x] = fmax(s_split[threadIdx.x], s_split[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = s_top[0]; part[2 * blockIdx.x + 1] = s_split[0]; }
}

__global__ void band_edge_final(const double* __restrict__ part, int parts, double* out) {
  if (threadIdx.x != 0) return;
  double top = -INFINITY, split = 0.0;
  for (int p = 0; p < parts; ++p) { top = fmax(top, part[2 * p]); split = fmax(split, part[2 * p + 1]); }
  out[0] = top;
  out[1] = split;
}

static int edge_parts(long long N) {
  return (int)std::max(1LL, std::min<long long>((N + kEdgeThreads - 1) / kEdgeThreads,
                                                kEdgeMaxParts));
}

}  // namespace qdkp

using namespace qdkp;

extern "C" {

size_t qdkp_local_band_edges_workspace_size(const qdkp_operator* op) {
  if (!op) return 0;
  return ((size_t)edge_parts(op->n_sites) * 2 + 2) * sizeof(double) + 256;
}

int qdkp_local_band_edges(const qdkp_operator* op, const unsigned char* mask, double* levels,
                          double* top_v1, double* kramers_split, void* ws, size_t ws_bytes,
                          void* stream) {
  QDKP_CHECK_ARG(op && top_v1, "NULL argument");
  QDKP_CHECK_ARG(op->n_bands == 8 || op->n_bands == 6, "the valence block needs 8 or 6 bands");
  const long long N = op->n_sites;
  const int parts = edge_parts(N);
  if (!ws || ws_bytes < qdkp_local_band_edges_workspace_size(op)) {
    set_error("qdkp_local_band_edges: workspace too small");
    return QDKP_ERR_WORKSPACE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* part = static_cast<double*>(ws);
  double* out = part + 2 * (size_t)parts;
  band_edge_kernel<<<parts, kEdgeThreads, 0, st>>>(op->fields64, N, mask, levels, part);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  band_edge_final<<<1, 32, 0, st>>>(part, parts, out);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  double host[2];
  QDKP_CUDA_TRY(cudaMemcpyAsync(host, out, sizeof(host), cudaMemcpyDeviceToHost, st));
  QDKP_CUDA_TRY(cudaStreamSynchronize(st));
  *top_v1 = host[0];
  if (kramers_split) *kramers_split = host[1];
  return QDKP_OK;
}

}  // extern "C"
