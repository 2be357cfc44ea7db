// Peak diagnostics on the GPU: the reductions of pbhgr/pbhgr/pm3d.py:132-159 (analyse)
// over all particles, and the Lagrangian radius keys used to pick its core sets.
#include "../../include/pmb200.h"
#include "common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kVals = 34;  // 3 sets x (count, sum r (3), sum r r^T (6)) + 4 radius counts

__device__ __forceinline__ double wrapc(double d, double L) {
  // (x - c + L/2) % L - L/2 with Python's float modulo (pm3d.py:142)
  double r = fmod(d + L / 2, L);
  if (r != 0.0 && (r < 0) != (L < 0)) r += L;
  return r - L / 2;
}

__device__ __forceinline__ double r_ell_q(long long id, int Np, double L, const double* A) {
  const int jz = (int)(id % Np), jy = (int)((id / Np) % Np), jx = (int)(id / ((long long)Np * Np));
  const double dq = L / Np;
  const double q[3] = {(jx + 0.5) * dq - L / 2, (jy + 0.5) * dq - L / 2, (jz + 0.5) * dq - L / 2};
  double s = 0.0;
  for (int d = 0; d < 3; ++d) s += (q[d] / A[d]) * (q[d] / A[d]);
  return sqrt(s);  // pm3d.py:71
}

__global__ void k_rell_keys(int Np, double L, double a0, double a1, double a2, u64* keys) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)Np * Np * Np;
  if (i >= n) return;
  const double A[3] = {a0, a1, a2};
  // Non-negative doubles order like their bit patterns.
  keys[i] = (u64)__double_as_longlong(r_ell_q(i, Np, L, A));
}

__global__ void k_analyse(const double* __restrict__ x, int Np, double L, double a0, double a1, double a2, double cx,
                          double cy, double cz, double t0, double t1, double t2, double r0, double r1, double r2,
                          double r3, double* __restrict__ part) {
  __shared__ double sh[kThreads / 32][kVals];
  double v[kVals];
  for (int k = 0; k < kVals; ++k) v[k] = 0.0;
  const long long n = (long long)Np * Np * Np;
  const double A[3] = {a0, a1, a2};
  const double th[3] = {t0, t1, t2};
  const double rr[4] = {r0, r1, r2, r3};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double rel[3] = {wrapc(x[3 * i] - cx, L), wrapc(x[3 * i + 1] - cy, L), wrapc(x[3 * i + 2] - cz, L)};
    const double re = r_ell_q(i, Np, L, A);
    for (int s = 0; s < 3; ++s) {
      if (re < th[s]) {
        double* o = v + 10 * s;
        o[0] += 1.0;
        o[1] += rel[0];
        o[2] += rel[1];
        o[3] += rel[2];
        o[4] += rel[0] * rel[0];
        o[5] += rel[0] * rel[1];
        o[6] += rel[0] * rel[2];
        o[7] += rel[1] * rel[1];
        o[8] += rel[1] * rel[2];
        o[9] += rel[2] * rel[2];
      }
    }
    const double r2 = rel[0] * rel[0] + rel[1] * rel[1] + rel[2] * rel[2];
    for (int k = 0; k < 4; ++k)
      if (sqrt(r2) < rr[k]) v[30 + k] += 1.0;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < kVals; ++k) {
    double s = v[k];
    for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
    if (lane == 0) sh[warp][k] = s;
  }
  __syncthreads();
  if (threadIdx.x < kVals) {
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) s += sh[w][threadIdx.x];
    part[(size_t)blockIdx.x * kVals + threadIdx.x] = s;
  }
}

}  // namespace

extern "C" int pm_rell_keys(int Np, double L, const double* A, unsigned long long* keys) {
  if (Np < 1 || !A || !keys || !(L > 0)) return -2000;
  const long long n = (long long)Np * Np * Np;
  k_rell_keys<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads>>>(Np, L, A[0], A[1], A[2], (u64*)keys);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  return e == cudaSuccess ? 0 : -(int)e;
}

extern "C" int pm_analyse_partials(const double* x, int Np, double L, const double* A, const double* centre,
                                   const double* set_radii, const double* radii, int nblocks, double* partials) {
  if (!x || Np < 1 || !A || !centre || !set_radii || !radii || nblocks < 1 || !partials) return -2000;
  k_analyse<<<nblocks, kThreads>>>(x, Np, L, A[0], A[1], A[2], centre[0], centre[1], centre[2], set_radii[0],
                                   set_radii[1], set_radii[2], radii[0], radii[1], radii[2], radii[3], partials);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  return e == cudaSuccess ? 0 : -(int)e;
}
