// Initial conditions on the GPU in float64: PM3D.make_ic (pbhgr/pbhgr/pm3d.py:40-73) and the
// benchmark's Gaussian-peak recipe, both ending in the reference's Zel'dovich tail
// (pm3d.py:59-72): delta_k -> displacement potential -> psi = -grad phi -> CIC-interpolated
// displacements of the quiet-start lattice.
#include <cufft.h>

#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <utility>
#include <vector>

#include "../../include/pmb200.h"
#include "common.cuh"

namespace {

constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double kPi = 3.14159265358979323846264338328;
constexpr int kThreads = 256;

#define CU(x)                                         \
  do {                                                \
    cudaError_t e_ = (x);                             \
    if (e_ != cudaSuccess) { rc = -(int)e_; goto done; } \
  } while (0)
#define CF(x)                                         \
  do {                                                \
    cufftResult r_ = (x);                             \
    if (r_ != CUFFT_SUCCESS) { rc = -1000 - (int)r_; goto done; } \
  } while (0)

__device__ __forceinline__ double kline(int i, int N, double kf) { return kf * (double)(i < N / 2 ? i : i - N); }

// Piecewise cubic (scipy PPoly layout: c[k*m + i] multiplies (r - x_i)^(3-k)); interval by
// searchsorted(x, r, 'right') - 1 clipped to [0, m-1], as CubicSpline.__call__ does.
__device__ double spline_eval(const double* __restrict__ xs, const double* __restrict__ c, int m, double r) {
  int lo = 0, hi = m;  // find last i in [0, m] with xs[i] <= r
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (xs[mid] <= r) lo = mid; else hi = mid - 1;
  }
  int i = lo;
  if (i > m - 1) i = m - 1;
  if (i < 0) i = 0;
  const double t = r - xs[i];
  return ((c[i] * t + c[m + i]) * t + c[2 * m + i]) * t + c[3 * m + i];
}

// Field on the centred cell grid x = (i + 1/2) dx - L/2 (pm3d.py:42-46).
__global__ void k_field(int N, double L, int kind, double amp, double a0, double a1, double a2,
                        const double* __restrict__ xs, const double* __restrict__ c, int m, double* __restrict__ out) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long N3 = (long long)N * N * N;
  if (g >= N3) return;
  const int iz = (int)(g % N), iy = (int)((g / N) % N), ix = (int)(g / ((long long)N * N));
  const double dx = L / N;
  const double X = (ix + 0.5) * dx - L / 2, Y = (iy + 0.5) * dx - L / 2, Z = (iz + 0.5) * dx - L / 2;
  if (kind == 0) {
    const double r = sqrt((X / a0) * (X / a0) + (Y / a1) * (Y / a1) + (Z / a2) * (Z / a2));
    out[g] = amp * spline_eval(xs, c, m, fmin(r, xs[m]));
  } else {
    out[g] = amp * exp(-(X * X / (2 * a0 * a0) + Y * Y / (2 * a1 * a1) + Z * Z / (2 * a2 * a2)));
  }
}

// Noise spectrum shaping.  kind 0: band-limited P flat in ln k (pm3d.py:49-54);
// kind 1: sqrt(P) = 1/k, P(0) = 0 (benchmark recipe).
__global__ void k_shape(cufftDoubleComplex* __restrict__ s, int N, double L, int kind, double tail_rms, double k1,
                        double k2) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int Nh = N / 2 + 1;
  const long long M = (long long)N * N * Nh;
  if (m >= M) return;
  const int kz = (int)(m % Nh), iy = (int)((m / Nh) % N), ix = (int)(m / ((long long)Nh * N));
  const double kf = kTwoPi / L;
  const double kx = kline(ix, N, kf), ky = kline(iy, N, kf), kzv = kf * kz;
  const double kk = m == 0 ? 0.0 : sqrt(kx * kx + ky * ky + kzv * kzv);
  double f;
  if (kind == 0) {
    const bool band = kk >= k1 && kk <= k2;
    const double P = band ? 2 * kPi * kPi * tail_rms * tail_rms / (fmax(kk, 1e-30) * fmax(kk, 1e-30) * fmax(kk, 1e-30) * log(k2 / k1)) : 0.0;
    f = sqrt(P * (double)N * N * N / (L * L * L));
  } else {
    f = m == 0 ? 0.0 : 1.0 / kk;
  }
  s[m].x *= f;
  s[m].y *= f;
}

// Counter-based normal deviates for seeded noise generated on the device: Philox4x32-10
// (Salmon, Moraes, Dror & Shaw, SC'11: 10 rounds of the two 32x32->64 multiplies with a Weyl-
// sequence key schedule) feeding the Box-Muller transform.  Element i of the field is a
// deterministic function of (seed, i), so a run is reproducible and independent of launch shape.
__device__ __forceinline__ void philox_round(u32 (&c)[4], u32 k0, u32 k1) {
  const u32 M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const u32 hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
  const u32 hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
  const u32 n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
  c[0] = n0;
  c[1] = n1;
  c[2] = n2;
  c[3] = n3;
}

__global__ void k_philox_normal(double* __restrict__ out, long long n, unsigned long long seed) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // one Philox call -> 4 normals
  if (4 * q >= n) return;
  u32 c[4] = {(u32)q, (u32)((unsigned long long)q >> 32), 0x5eedu, 0x1ce5u};
  u32 k0 = (u32)seed, k1 = (u32)(seed >> 32);
  for (int r = 0; r < 10; ++r) {
    philox_round(c, k0, k1);
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  // 53-bit uniforms in (0, 1] from pairs of words, then Box-Muller pairs.
  const double inv53 = 1.0 / 9007199254740992.0;
  const double u0 = ((double)((((unsigned long long)c[0] << 32) | c[1]) >> 11) + 1.0) * inv53;
  const double u1 = (double)((((unsigned long long)c[2] << 32) | c[3]) >> 11) * inv53;
  const double r = sqrt(-2.0 * log(u0));
  double sn, cs;
  sincospi(2.0 * u1, &sn, &cs);
  // The second pair reuses the words with halves swapped.
  const double v0 = ((double)((((unsigned long long)c[3] << 32) | c[2]) >> 11) + 1.0) * inv53;
  const double v1 = (double)((((unsigned long long)c[1] << 32) | c[0]) >> 11) * inv53;
  const double r2 = sqrt(-2.0 * log(v0));
  double sn2, cs2;
  sincospi(2.0 * v1, &sn2, &cs2);
  const double z[4] = {r * cs, r * sn, r2 * cs2, r2 * sn2};
  for (int k = 0; k < 4; ++k)
    if (4 * q + k < n) out[4 * q + k] = z[k];
}

// y += a x with a = 1 (kind 0: make_ic's tail noise is already at its amplitude) or
// a = noise_frac * amp / rms (kind 1: the recipe's noise scaled to noise_frac of the peak), rms
// read from stat[1] on the device.
__global__ void k_axpy_spec(cufftDoubleComplex* __restrict__ y, const cufftDoubleComplex* __restrict__ x,
                            const double* __restrict__ stat, int kind, double noise_frac, double amp, long long M) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  const double a = kind == 0 ? 1.0 : noise_frac * amp / stat[1];
  y[m].x += a * x[m].x;
  y[m].y += a * x[m].y;
}

// delta_k (kind 0: 0.4 k^2 zeta_k / H_i^2, pm3d.py:59), zero mode removed; then the four
// spectra inverted at once: delta_lin = irfftn(dk) (pm3d.py:70) and psi_c = -irfftn(i k_c phi),
// phi = -dk/k^2 (pm3d.py:61-62).  Each spectrum carries numpy's 1/N^3 and, in the kz = 0 and
// kz = N/2 planes, its Hermitian part (numpy's irfftn uses only that part there).
__device__ __forceinline__ void four_spectra(const cufftDoubleComplex z, int kind, double kx, double ky, double kz,
                                            long long m, double* re, double* im) {
  const double k2 = m == 0 ? 1.0 : kx * kx + ky * ky + kz * kz;
  double dr = z.x, di = z.y;
  if (kind == 0) {
    const double f = 0.4 * k2 / (PM_H_I * PM_H_I);
    dr *= f;
    di *= f;
  }
  if (m == 0) dr = di = 0.0;
  const double pr = -dr / k2, pi = -di / k2;
  re[0] = dr;
  im[0] = di;
  const double kc[3] = {kx, ky, kz};
  for (int c = 0; c < 3; ++c) {  // -(i k phi) = (k pi, -k pr)
    re[c + 1] = kc[c] * pi;
    im[c + 1] = -kc[c] * pr;
  }
}

__global__ void k_disp_spectra(const cufftDoubleComplex* __restrict__ s, int N, double L, int kind,
                               cufftDoubleComplex* __restrict__ out) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int Nh = N / 2 + 1;
  const long long M = (long long)N * N * Nh;
  if (m >= M) return;
  const int kz = (int)(m % Nh), iy = (int)((m / Nh) % N), ix = (int)(m / ((long long)Nh * N));
  const double kf = kTwoPi / L;
  const double kx = kline(ix, N, kf), ky = kline(iy, N, kf), kzv = kf * kz;
  double re[4], im[4];
  four_spectra(s[m], kind, kx, ky, kzv, m, re, im);
  if (kz == 0 || kz == N / 2) {
    const int px = (-ix) & (N - 1), py = (-iy) & (N - 1);
    const long long mp = ((long long)px * N + py) * Nh + kz;
    double rp[4], ip[4];
    four_spectra(s[mp], kind, kline(px, N, kf), kline(py, N, kf), kzv, mp, rp, ip);
    for (int c = 0; c < 4; ++c) {
      re[c] = 0.5 * (re[c] + rp[c]);
      im[c] = 0.5 * (im[c] - ip[c]);
    }
  }
  const double inv = 1.0 / ((double)N * N * N);
  for (int c = 0; c < 4; ++c) {
    out[c * M + m].x = re[c] * inv;
    out[c * M + m].y = im[c] * inv;
  }
}

// Lattice (pm3d.py:64-65), CIC displacement at (Q + L/2) % L (pm3d.py:66), x and p
// (pm3d.py:67-68).  Python's float % is x - L*floor(x/L).
__device__ __forceinline__ double pymod(double x, double L) {
  double r = fmod(x, L);
  if (r != 0.0 && ((r < 0) != (L < 0))) r += L;
  return r;
}

__global__ void k_lattice(int N, int Np, double L, const double* __restrict__ psi, double* __restrict__ x,
                          double* __restrict__ p) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)Np * Np * Np;
  if (i >= n) return;
  const int jz = (int)(i % Np), jy = (int)((i / Np) % Np), jx = (int)(i / ((long long)Np * Np));
  const double dq = L / Np, dx = L / N;
  const double Q[3] = {(jx + 0.5) * dq - L / 2, (jy + 0.5) * dq - L / 2, (jz + 0.5) * dq - L / 2};
  long long i0[3], i1[3];
  double f[3];
  for (int d = 0; d < 3; ++d) {
    const double at = pymod(Q[d] + L / 2, L);
    const double g = at / dx - 0.5;
    const double fl = floor(g);
    const long long c = (long long)fl;
    f[d] = g - fl;
    i0[d] = ((c % N) + N) % N;
    i1[d] = (((c + 1) % N) + N) % N;
  }
  const long long N3 = (long long)N * N * N;
  double disp[3] = {0.0, 0.0, 0.0};
  for (int c = 0; c < 8; ++c) {
    const int cx = c >> 2, cy = (c >> 1) & 1, cz = c & 1;
    const long long o = ((cx ? i1[0] : i0[0]) * N + (cy ? i1[1] : i0[1])) * N + (cz ? i1[2] : i0[2]);
    const double w = (cx ? f[0] : 1.0 - f[0]) * (cy ? f[1] : 1.0 - f[1]) * (cz ? f[2] : 1.0 - f[2]);
    for (int d = 0; d < 3; ++d) disp[d] += psi[(1 + d) * N3 + o] * w;
  }
  for (int d = 0; d < 3; ++d) {
    x[3 * i + d] = pymod(Q[d] + disp[d] + L / 2, L);
    p[3 * i + d] = PM_H_I * disp[d];
  }
}

// Block partial sums of x and (x - mean)^2 for numpy's std (mean first, then the spread).
// Block partials of sum v (squares = 0) or of sum (v - stat[0])^2 (squares = 1).
__global__ void k_partial(const double* __restrict__ v, long long n, const double* __restrict__ stat, int squares,
                          double* __restrict__ part) {
  __shared__ double sh[kThreads];
  const double mean = squares ? stat[0] : 0.0;
  double s = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double d = squares ? v[i] - mean : v[i];
    s += squares ? d * d : d;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// The partials summed in block order by one thread: stat[0] = mean (squares = 0), or stat[1] =
// rms / N3 of the unnormalised inverse transform (squares = 1), the noise field's rms.
__global__ void k_reduce_partials(const double* __restrict__ part, int nb, long long n, long long N3, int squares,
                                  double* __restrict__ stat) {
  double t = 0.0;
  for (int b = 0; b < nb; ++b) t += part[b];
  if (!squares) stat[0] = t / (double)n;
  else stat[1] = sqrt(t / (double)n) / (double)N3;
}

constexpr int kStdBlocks = 1024;

// Standard deviation of v (two passes, fixed order) into stat[1], divided by N3; on stream s.
void grid_std(const double* v, long long n, long long N3, double* part, double* stat, cudaStream_t s) {
  k_partial<<<kStdBlocks, kThreads, 0, s>>>(v, n, stat, 0, part);
  k_reduce_partials<<<1, 1, 0, s>>>(part, kStdBlocks, n, N3, 0, stat);
  k_partial<<<kStdBlocks, kThreads, 0, s>>>(v, n, stat, 1, part);
  k_reduce_partials<<<1, 1, 0, s>>>(part, kStdBlocks, n, N3, 1, stat);
}

unsigned nblk(long long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// Device buffers and FP64 cuFFT plans of pm_make_ic, kept per (device, N) after first use so
// that repeated calls (a request loop) neither allocate nor plan again.
struct ICWork {
  double *field = nullptr, *real4 = nullptr, *tmp_real = nullptr, *noise = nullptr;
  cufftDoubleComplex *spec = nullptr, *nspec = nullptr, *spec4 = nullptr, *tmp_spec = nullptr;
  double* part = nullptr;  // kStdBlocks partials, then stat[2] (mean, noise rms)
  cufftHandle d2z = 0, z2d = 0, z2d4 = 0;
  bool ok = false;
};
std::mutex g_ic_mu;
// Keyed by (device, N, path): the synchronous pm_make_ic and the stream-ordered
// pm_make_ic_async keep separate work areas, so the two never share buffers in flight.
std::map<std::tuple<int, int, int>, ICWork> g_ic;

int ic_work(int device, int N, int path, ICWork** out) {
  std::lock_guard<std::mutex> lock(g_ic_mu);
  ICWork& w = g_ic[{device, N, path}];
  if (!w.ok) {
    const long long N3 = (long long)N * N * N, M = (long long)N * N * (N / 2 + 1);
    int rc = 0;
    int n3[3] = {N, N, N};
    CU(cudaMalloc(&w.field, sizeof(double) * N3));
    CU(cudaMalloc(&w.real4, sizeof(double) * 4 * N3));
    CU(cudaMalloc(&w.tmp_real, sizeof(double) * N3));
    CU(cudaMalloc(&w.noise, sizeof(double) * N3));
    CU(cudaMalloc(&w.spec, sizeof(cufftDoubleComplex) * M));
    CU(cudaMalloc(&w.nspec, sizeof(cufftDoubleComplex) * M));
    CU(cudaMalloc(&w.spec4, sizeof(cufftDoubleComplex) * 4 * M));
    CU(cudaMalloc(&w.tmp_spec, sizeof(cufftDoubleComplex) * M));
    CU(cudaMalloc(&w.part, sizeof(double) * (kStdBlocks + 2)));
    CF(cufftPlan3d(&w.d2z, N, N, N, CUFFT_D2Z));
    CF(cufftPlan3d(&w.z2d, N, N, N, CUFFT_Z2D));
    CF(cufftPlanMany(&w.z2d4, 3, n3, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2D, 4));
    w.ok = true;
  done:
    if (rc) {
      g_ic.erase({device, N, path});
      return rc;
    }
  }
  *out = &w;
  return 0;
}

}  // namespace

extern "C" int pm_ic_release_cache(void) {
  std::lock_guard<std::mutex> lock(g_ic_mu);
  for (auto& kv : g_ic) {
    ICWork& w = kv.second;
    cudaSetDevice(std::get<0>(kv.first));
    cudaFree(w.field);
    cudaFree(w.real4);
    cudaFree(w.tmp_real);
    cudaFree(w.noise);
    cudaFree(w.spec);
    cudaFree(w.nspec);
    cudaFree(w.spec4);
    cudaFree(w.tmp_spec);
    cudaFree(w.part);
    if (w.ok) {
      cufftDestroy(w.d2z);
      cufftDestroy(w.z2d);
      cufftDestroy(w.z2d4);
    }
  }
  g_ic.clear();
  return 0;
}

namespace {

int check_params(const pm_ic_params* prm, const double* x_out, const double* p_out) {
  if (!prm || !x_out || !p_out) return -2000;
  const int N = prm->N, Np = prm->Np;
  if (N < 4 || (N & (N - 1)) || Np < 1 || !(prm->L > 0)) return -2001;
  if (prm->kind == 0 && (!prm->spline_x || !prm->spline_c || prm->spline_m < 1)) return -2002;
  if (prm->kind != 0 && prm->kind != 1) return -2003;
  return 0;
}

// The IC pipeline on stream s with work area w (spline arrays xs, cs on the device for kind 0).
// The noise rms is left in w->part[kStdBlocks + 1].
int make_ic_on(const pm_ic_params* prm, double* x_out, double* p_out, double* delta_lin_out, const double* xs,
               const double* cs, ICWork* w, cudaStream_t s) {
  const int N = prm->N, Np = prm->Np;
  const long long N3 = (long long)N * N * N, M = (long long)N * N * (N / 2 + 1);
  const double L = prm->L;
  int rc = 0;
  double* stat = w->part + kStdBlocks;
  const bool want_noise = (prm->kind == 0 && prm->tail_rms > 0) || (prm->kind == 1 && prm->noise_frac > 0);
  const bool noisy = want_noise && (prm->noise || prm->noise_seed);
  CF(cufftSetStream(w->d2z, s));
  CF(cufftSetStream(w->z2d, s));
  CF(cufftSetStream(w->z2d4, s));
  CU(cudaMemsetAsync(stat, 0, sizeof(double) * 2, s));
  k_field<<<nblk(N3), kThreads, 0, s>>>(N, L, prm->kind, prm->amp, prm->axes[0], prm->axes[1], prm->axes[2], xs, cs,
                                        prm->kind == 0 ? prm->spline_m : 0, w->field);
  CU(cudaGetLastError());
  CF(cufftExecD2Z(w->d2z, w->field, w->spec));
  if (noisy) {
    if (!prm->noise) {  // seeded device noise
      k_philox_normal<<<nblk((N3 + 3) / 4), kThreads, 0, s>>>(w->noise, N3, prm->noise_seed);
      CU(cudaGetLastError());
    }
    CF(cufftExecD2Z(w->d2z, prm->noise ? (double*)prm->noise : w->noise, w->nspec));
    k_shape<<<nblk(M), kThreads, 0, s>>>(w->nspec, N, L, prm->kind, prm->tail_rms, prm->k1, prm->k2);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(w->tmp_spec, w->nspec, sizeof(cufftDoubleComplex) * M, cudaMemcpyDeviceToDevice, s));
    CF(cufftExecZ2D(w->z2d, w->tmp_spec, w->tmp_real));  // unnormalised inverse; numpy divides by N^3
    grid_std(w->tmp_real, N3, N3, w->part, stat, s);
    k_axpy_spec<<<nblk(M), kThreads, 0, s>>>(w->spec, w->nspec, stat, prm->kind, prm->noise_frac, prm->amp, M);
    CU(cudaGetLastError());
  }
  k_disp_spectra<<<nblk(M), kThreads, 0, s>>>(w->spec, N, L, prm->kind, w->spec4);
  CU(cudaGetLastError());
  CF(cufftExecZ2D(w->z2d4, w->spec4, w->real4));
  k_lattice<<<nblk((long long)Np * Np * Np), kThreads, 0, s>>>(N, Np, L, w->real4, x_out, p_out);
  CU(cudaGetLastError());
  if (delta_lin_out)
    CU(cudaMemcpyAsync(delta_lin_out, w->real4, sizeof(double) * N3, cudaMemcpyDeviceToDevice, s));
done:
  return rc;
}

}  // namespace

extern "C" int pm_make_ic(const pm_ic_params* prm, double* x_out, double* p_out, double* delta_lin_out,
                          double* noise_rms_out) {
  if (int r = check_params(prm, x_out, p_out)) return r;
  int rc = 0, device = 0;
  double *xs = nullptr, *cs = nullptr;
  double stat[2] = {0.0, 0.0};
  ICWork* w = nullptr;
  CU(cudaGetDevice(&device));
  rc = ic_work(device, prm->N, 0, &w);
  if (rc) return rc;
  if (prm->kind == 0) {
    const int m = prm->spline_m;
    CU(cudaMalloc(&xs, sizeof(double) * (m + 1)));
    CU(cudaMalloc(&cs, sizeof(double) * 4 * m));
    CU(cudaMemcpy(xs, prm->spline_x, sizeof(double) * (m + 1), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(cs, prm->spline_c, sizeof(double) * 4 * m, cudaMemcpyHostToDevice));
  }
  rc = make_ic_on(prm, x_out, p_out, delta_lin_out, xs, cs, w, 0);
  if (rc) goto done;
  CU(cudaMemcpy(stat, w->part + kStdBlocks, sizeof(stat), cudaMemcpyDeviceToHost));
  CU(cudaDeviceSynchronize());
  if (noise_rms_out) *noise_rms_out = stat[1];
done:
  cudaFree(xs);
  cudaFree(cs);
  return rc;
}

extern "C" int pm_make_ic_async(const pm_ic_params* prm, double* x_out, double* p_out, void* stream) {
  if (int r = check_params(prm, x_out, p_out)) return r;
  if (prm->kind != 1) return -2003;  // the curvature-profile ICs copy a host spline: pm_make_ic
  int device = 0;
  const cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return -(int)e;
  ICWork* w = nullptr;
  if (int r = ic_work(device, prm->N, 1, &w)) return r;
  return make_ic_on(prm, x_out, p_out, nullptr, nullptr, nullptr, w, (cudaStream_t)stream);
}
