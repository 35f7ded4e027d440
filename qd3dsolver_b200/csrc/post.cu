// Post-processing of eigenvector blocks on the device (sm_100a): localisation in the dot and the
// Kramers pairing of the levels.
//
//   pryor_fig4.localization (pryor_fig4.py:179-193): for every column j of V (rows band * N +
//     site), loc_j = sum over dot sites and bands of |V|^2 / sum over all sites and bands of |V|^2.
//   pryor_fig4.kramers_levels (pryor_fig4.py:222-236): consecutive entries of E, in the order the
//     caller gives them, form pairs; level = the pair's mean, its localisation the mean of the
//     pair's, and the worst within-pair splitting is reported.
//
// Two launches: every CTA sums a fixed range of sites for all columns (one thread per
// (site, column) of a row of the range, so a warp reads consecutive columns of a row), then one
// CTA adds the per-CTA partial sums in a fixed order and pairs the levels. The result does not
// depend on the launch or on any other work on the GPU.
#include <algorithm>

#include "qdkp_common.cuh"

namespace qdkp {

constexpr int kLocThreads = 256;
constexpr int kLocMaxParts = 1184;         // eight CTAs per SM on 148 SMs
constexpr int kLocMaxCols = 128;

template <typename T>
__global__ void __launch_bounds__(kLocThreads)
loc_partial_kernel(const cplx<T>* __restrict__ V, long long ldv, int k, long long N, int nb,
                   const unsigned char* __restrict__ mask, long long sites_per_part,
                   double* __restrict__ partial) {
  __shared__ double s_in[kLocThreads], s_tot[kLocThreads];
  const int per = kLocThreads / k;           // sites handled side by side
  const int t = threadIdx.x;
  const int j = t % k, r = t / k;
  const long long s0 = (long long)blockIdx.x * sites_per_part;
  const long long s1 = min(N, s0 + sites_per_part);
  double in = 0.0, tot = 0.0;
  if (r < per) {
    for (long long s = s0 + r; s < s1; s += per) {
      double a = 0.0;
      for (int b = 0; b < nb; ++b) {
        const cplx<T> v = V[((long long)b * N + s) * ldv + j];
        a += (double)v.x * (double)v.x + (double)v.y * (double)v.y;
      }
      tot += a;
      if (mask[s]) in += a;
    }
  }
  s_in[t] = in;
  s_tot[t] = tot;
  __syncthreads();
  if (t < k) {
    double a = 0.0, b = 0.0;
    for (int q = 0; q < per; ++q) { a += s_in[t + q * k]; b += s_tot[t + q * k]; }
    partial[((long long)blockIdx.x * k + t) * 2] = a;
    partial[((long long)blockIdx.x * k + t) * 2 + 1] = b;
  }
}

// out: loc[k], levels[k/2], level_loc[k/2], worst split (one value)
__global__ void __launch_bounds__(kLocMaxCols)
loc_final_kernel(const double* __restrict__ partial, int parts, int k,
                 const double* __restrict__ E, double* __restrict__ out) {
  __shared__ double loc[kLocMaxCols];
  const int j = threadIdx.x;
  if (j < k) {
    double a = 0.0, b = 0.0;
    for (int p = 0; p < parts; ++p) {
      a += partial[((long long)p * k + j) * 2];
      b += partial[((long long)p * k + j) * 2 + 1];
    }
    loc[j] = b > 0.0 ? a / b : 0.0;
    out[j] = loc[j];
  }
  __syncthreads();
  if (E == nullptr) return;
  const int np = k / 2;
  if (j < np) {
    out[k + j] = 0.5 * (E[2 * j] + E[2 * j + 1]);
    out[k + np + j] = 0.5 * (loc[2 * j] + loc[2 * j + 1]);
  }
  if (j == 0) {
    double worst = 0.0;
    for (int p = 0; p < np; ++p) worst = fmax(worst, fabs(E[2 * p + 1] - E[2 * p]));
    out[k + 2 * np] = worst;
  }
}

struct LocLayout {
  int parts;
  long long sites_per_part;
  size_t partial, e, out, total;
};

static LocLayout loc_layout(long long N, int k) {
  LocLayout L;
  long long parts = (N + 63) / 64;
  parts = std::max(1LL, std::min<long long>(parts, kLocMaxParts));
  L.sites_per_part = (N + parts - 1) / parts;
  L.parts = (int)((N + L.sites_per_part - 1) / L.sites_per_part);
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  L.partial = al((size_t)L.parts * k * 2 * sizeof(double));
  L.e = al((size_t)k * sizeof(double));
  L.out = al((size_t)(2 * k + 1) * sizeof(double));
  L.total = L.partial + L.e + L.out;
  return L;
}

}  // namespace qdkp

using namespace qdkp;

extern "C" {

size_t qdkp_state_summary_workspace_size(const qdkp_operator* op, int k) {
  if (!op || k < 1 || k > kLocMaxCols) return 0;
  return loc_layout(op->n_sites, k).total;
}

int qdkp_state_summary(const qdkp_operator* op, const void* V, int64_t ldv, int k, int precision,
                       const unsigned char* mask, const double* E, double* loc, double* levels,
                       double* level_loc, double* worst_split, void* ws, size_t ws_bytes,
                       void* stream) {
  QDKP_CHECK_ARG(op && V && mask && loc, "NULL argument");
  QDKP_CHECK_ARG(k >= 1 && k <= kLocMaxCols && ldv >= k, "need 1 <= k <= 128 and ldv >= k");
  QDKP_CHECK_ARG(precision == QDKP_C128 || precision == QDKP_C64, "bad precision");
  QDKP_CHECK_ARG(E == nullptr || (levels && level_loc && worst_split),
                 "pairing needs levels, level_loc and worst_split");
  const LocLayout L = loc_layout(op->n_sites, k);
  if (!ws || ws_bytes < L.total) {
    set_error("qdkp_state_summary: workspace too small (see qdkp_state_summary_workspace_size)");
    return QDKP_ERR_WORKSPACE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  char* base = static_cast<char*>(ws);
  double* partial = reinterpret_cast<double*>(base);
  double* Ed = reinterpret_cast<double*>(base + L.partial);
  double* out = reinterpret_cast<double*>(base + L.partial + L.e);
  if (E) QDKP_CUDA_TRY(cudaMemcpyAsync(Ed, E, k * sizeof(double), cudaMemcpyHostToDevice, st));
  if (precision == QDKP_C128)
    loc_partial_kernel<double><<<L.parts, kLocThreads, 0, st>>>(
        static_cast<const double2*>(V), ldv, k, op->n_sites, op->n_bands, mask,
        L.sites_per_part, partial);
  else
    loc_partial_kernel<float><<<L.parts, kLocThreads, 0, st>>>(
        static_cast<const float2*>(V), ldv, k, op->n_sites, op->n_bands, mask,
        L.sites_per_part, partial);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  loc_final_kernel<<<1, kLocMaxCols, 0, st>>>(partial, L.parts, k, E ? Ed : nullptr, out);
  count_launch();
  QDKP_CUDA_TRY(cudaGetLastError());
  const int nout = E ? 2 * k + 1 - (k % 2 ? 1 : 0) : k;
  double host[2 * kLocMaxCols + 1];
  QDKP_CUDA_TRY(cudaMemcpyAsync(host, out, (size_t)std::max(nout, k) * sizeof(double),
                                cudaMemcpyDeviceToHost, st));
  QDKP_CUDA_TRY(cudaStreamSynchronize(st));
  for (int j = 0; j < k; ++j) loc[j] = host[j];
  if (E) {
    const int np = k / 2;
    for (int p = 0; p < np; ++p) { levels[p] = host[k + p]; level_loc[p] = host[k + np + p]; }
    *worst_split = host[k + 2 * np];
  }
  return QDKP_OK;
}

}  // extern "C"
