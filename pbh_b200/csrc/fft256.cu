// Native 3D real FFT for the 256^3 mesh (sm_100a), two passes over HBM per direction, with the
// Green's-function gradient (pm3d.py:105-112) fused into the inverse.
//
// Layouts (one field; fields of a batch are consecutive):
//   real field      r[x][y][z]          256^3 float (the deposit's delta, the force grids)
//   spectrum        s[kz][kx][ky]       129 x 256 x 256 complex ("plane-major")
// numpy's rfftn(r)[kx][ky][kz] is s[kz][kx][ky]: the same transform, stored with kz outermost.
//
// Forward (R2C).  Pass Z: a real FFT along z of 32 (x, y) lines per CTA -- a complex FFT of the
// 128 packed (even, odd) pairs, then the split into 129 outputs -- written transposed into the
// kz planes.  Pass XY: a 2D complex FFT of every kz plane by a cluster of 4 CTAs: CTA c holds
// the rows x = 4 x1 + c (64 rows, 128 KB of shared memory), transforms them along y and then
// along x1, and the final 4-point combination reads the other CTAs' rows through distributed
// shared memory and writes each output row exactly once.
// Inverse (C2R).  Pass XY with the Green multiply on load (-i k_i G(k) delta_k / N^3, the
// Hermitian projection of the kz = 0, N/2 planes, the potential-energy partials), one cluster
// per plane and gradient component; pass Z, the real inverse along z, written as force rows.
// The 1D transforms are in-place radix-4 decimation in frequency (radix 2 first for length
// 128), so their outputs sit in digit-reversed order and are read back through the reversal.
// Twiddles come from a 256-entry table computed in double precision on the host.
// Transforms are unnormalised like cuFFT's; the Green factor carries numpy's 1/N^3.
#include <cooperative_groups.h>

#include <cmath>

#include "pm_kernels.cuh"

namespace cg = cooperative_groups;

namespace {

constexpr int FN = 256;            // mesh side
constexpr int FNH = FN / 2 + 1;    // kz planes
constexpr int FM = FN / 2;         // packed complex length of a z line
constexpr int XR = FN / 4;         // plane rows per CTA of a cluster
constexpr int XS = FN + 1;         // padded row stride (float2) of a plane slice
constexpr int ZT = 32;             // z lines per CTA in the Z passes
constexpr int ZS = FM + 8;         // stride of a packed z line (two 64-halves + pad)
constexpr int TT = ZT + 1;         // padded stride of the transposed kz tile
constexpr int FT = 256;            // threads per CTA of the Z passes
constexpr int XT = 1024;           // threads per CTA of the plane (XY) pass
constexpr long long N2 = (long long)FN * FN;
constexpr long long N3 = N2 * FN;

__device__ float2 g_tw[FN];        // exp(-2 pi i k / 256) of this device

__device__ __forceinline__ float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// times W_4 = -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 mul_w4(float2 a) { return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x); }
// W_256^e (forward) or its conjugate
template <bool INV>
__device__ __forceinline__ float2 w256(const float2* t, int e) {
  const float2 v = t[e & (FN - 1)];
  return INV ? cconj(v) : v;
}

__device__ __forceinline__ int rev4_3(int p) { return ((p & 3) << 4) | (p & 12) | ((p >> 4) & 3); }
__device__ __forceinline__ int rev4_4(int p) {
  return ((p & 3) << 6) | (((p >> 2) & 3) << 4) | (((p >> 4) & 3) << 2) | ((p >> 6) & 3);
}
// Where output k of the 128-point transform (radix 2, then radix 4 x 3) sits.
__device__ __forceinline__ int pos128(int k) { return ((k & 1) << 6) | rev4_3(k >> 1); }

// Radix-4 DIF stages with sub-lengths LS, LS/4, ..., 4 on nseq sequences of length L whose
// element i sits at buf[base(seq) + i * es], by NT threads.  All divisors are compile-time
// powers of two.  SEQ_FAST: consecutive threads take consecutive sequences (for sequences
// that run across rows); otherwise consecutive butterflies of one sequence.  Ends with a barrier.
template <bool INV, int L, int LS, int NT, bool SEQ_FAST, class Base>
__device__ __forceinline__ void dif4(float2* buf, int nseq, Base base, int es, const float2* t) {
  constexpr int q = LS / 4, step = FN / LS, BPS = L / 4;
  const int nb = nseq * BPS;
  for (int b = threadIdx.x; b < nb; b += NT) {
    int seq, r;
    if (SEQ_FAST) {
      seq = b % nseq;
      r = b / nseq;
    } else {
      seq = b / BPS;
      r = b % BPS;
    }
    const int blk = r / q, j = r % q;
    float2* p = buf + base(seq) + (blk * LS + j) * es;
    const int qs = q * es;
    const float2 x0 = p[0], x1 = p[qs], x2 = p[2 * qs], x3 = p[3 * qs];
    const float2 a = cadd(x0, x2), c = csub(x0, x2), s = cadd(x1, x3), d = mul_w4<INV>(csub(x1, x3));
    // y_r = sum_q x_q W_4^{q r}; quarter r takes y_r W_LS^{j r}
    p[0] = cadd(a, s);
    p[qs] = cmul(cadd(c, d), w256<INV>(t, j * step));
    p[2 * qs] = cmul(csub(a, s), w256<INV>(t, 2 * j * step));
    p[3 * qs] = cmul(csub(c, d), w256<INV>(t, 3 * j * step));
  }
  __syncthreads();
  if constexpr (LS > 4) dif4<INV, L, LS / 4, NT, SEQ_FAST>(buf, nseq, base, es, t);
}

// 128-point transforms of nseq sequences at buf[seq * ZS + i]: radix 2, then radix 4 on the two
// 64-point halves.
template <bool INV, int NT>
__device__ __forceinline__ void fft128(float2* buf, int nseq, const float2* t) {
  for (int b = threadIdx.x; b < nseq * 64; b += NT) {
    const int seq = b >> 6, j = b & 63;
    float2* p = buf + seq * ZS + j;
    const float2 a = p[0], c = p[64];
    p[0] = cadd(a, c);
    p[64] = cmul(csub(a, c), w256<INV>(t, 2 * j));  // W_128^j
  }
  __syncthreads();
  dif4<INV, 64, 64, NT, false>(buf, 2 * nseq, [](int h) { return (h >> 1) * ZS + (h & 1) * 64; }, 1, t);
}

__device__ __forceinline__ void cpa8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cpa16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <int NT>
__device__ __forceinline__ void load_tw(float2* t) {
  for (int i = threadIdx.x; i < FN; i += NT) t[i] = g_tw[i];
}

// Pass Z forward: fields in[f][x][y][z] -> planes out[f][kz][x][y].  grid (FN/ZT, FN, nf).
__global__ void __launch_bounds__(FT) k_fft_z_r2c(const float* __restrict__ in, float2* __restrict__ out) {
  extern __shared__ __align__(16) float2 zs[];
  float2* t = zs;                  // [FN]
  float2* buf = t + FN;            // [ZT][ZS]
  float2* T = buf + ZT * ZS;       // [FNH][TT]
  load_tw<FT>(t);
  const int y0 = blockIdx.x * ZT, x = blockIdx.y, f = blockIdx.z;
  const float2* src = reinterpret_cast<const float2*>(in + (long long)f * N3 + ((long long)x * FN + y0) * FN);
  for (int e = threadIdx.x; e < ZT * FM / 2; e += FT) {  // two packed pairs (16 bytes) per copy
    const int yl = e / (FM / 2), n = 2 * (e - yl * (FM / 2));
    cpa16(buf + yl * ZS + n, src + (long long)yl * FM + n);  // (r[2n], r[2n+1]) packed as one complex
  }
  cpa_wait();
  __syncthreads();
  fft128<false, FT>(buf, ZT, t);
  // X_k = E_k + W_256^k O_k with E = (Z_k + conj Z_{M-k})/2, O = -i (Z_k - conj Z_{M-k})/2
  for (int e = threadIdx.x; e < FNH * ZT; e += FT) {
    const int k = e / ZT, yl = e - k * ZT;
    const float2 zk = buf[yl * ZS + pos128(k & (FM - 1))];
    const float2 zm = cconj(buf[yl * ZS + pos128((FM - k) & (FM - 1))]);
    const float2 E = cscale(cadd(zk, zm), 0.5f);
    const float2 O = cscale(mul_w4<false>(csub(zk, zm)), 0.5f);
    T[k * TT + yl] = cadd(E, cmul(w256<false>(t, k), O));
  }
  __syncthreads();
  float2* dst = out + (long long)f * FNH * N2 + (long long)x * FN + y0;
  for (int e = threadIdx.x; e < FNH * ZT; e += FT) {
    const int k = e / ZT, yl = e - k * ZT;
    dst[(long long)k * N2 + yl] = T[k * TT + yl];
  }
}

// Pass Z inverse: planes in[f][kz][x][y] -> fields out[f][x][y][z].  grid (FN/ZT, FN, nf).
__global__ void __launch_bounds__(FT) k_fft_z_c2r(const float2* __restrict__ in, float* __restrict__ out) {
  extern __shared__ __align__(16) float2 zs[];
  float2* t = zs;
  float2* buf = t + FN;
  float2* T = buf + ZT * ZS;
  load_tw<FT>(t);
  const int y0 = blockIdx.x * ZT, x = blockIdx.y, f = blockIdx.z;
  const float2* src = in + (long long)f * FNH * N2 + (long long)x * FN + y0;
  for (int e = threadIdx.x; e < FNH * ZT; e += FT) {
    const int k = e / ZT, yl = e - k * ZT;
    cpa8(T + k * TT + yl, src + (long long)k * N2 + yl);
  }
  cpa_wait();
  __syncthreads();
  if (threadIdx.x < 2 * ZT) T[(threadIdx.x < ZT ? 0 : FM) * TT + (threadIdx.x & (ZT - 1))].y = 0.f;  // C2R reads
  __syncthreads();                                                                                  // only Re of DC, Nyquist
  // Z_k = E_k + i O_k with E = X_k + conj X_{M-k}, O = (X_k - conj X_{M-k}) W_256^{-k}
  for (int e = threadIdx.x; e < ZT * FM; e += FT) {
    const int yl = e / FM, k = e - yl * FM;
    const float2 xk = T[k * TT + yl], xm = cconj(T[(FM - k) * TT + yl]);
    const float2 O = cmul(csub(xk, xm), w256<true>(t, k));
    buf[yl * ZS + k] = cadd(cadd(xk, xm), make_float2(-O.y, O.x));
  }
  __syncthreads();
  fft128<true, FT>(buf, ZT, t);
  float2* dst = reinterpret_cast<float2*>(out + (long long)f * N3 + ((long long)x * FN + y0) * FN);
  for (int e = threadIdx.x; e < ZT * FM; e += FT) {
    const int yl = e / FM, n = e - yl * FM;
    dst[(long long)yl * FM + n] = buf[yl * ZS + pos128(n)];  // (r[2n], r[2n+1])
  }
}

// Green's-function multiply of one spectral value (the per-mode work of k_green).
struct GreenPlane {
  float s_c, kf, dx, sd2;
  int gm;
};
__device__ __forceinline__ float kl(int i, float kf) { return kf * (float)(i < FN / 2 ? i : i - FN); }
__device__ __forceinline__ float gk(float k, float dx, int mode) {
  if (mode == 1) return sinf(k * dx) / dx;
  if (mode == 2) return (8.0f * sinf(k * dx) - sinf(2.0f * k * dx)) / (6.0f * dx);
  return k;
}

// Pass XY: 2D FFT of every kz plane, one cluster of 4 CTAs per plane (and component).
// Forward: in = out = planes[slot][kz][x][y] (in place).  Inverse with GREEN: in = spectrum
// planes[slot][kz][kx][ky], out = planes[slot][comp][kz][x][y], comp = blockIdx.y, the
// multiply applied on load; slot_peak maps a slot to its peak.  Inverse without GREEN:
// in = out layout [f][kz][.][.].  grid (4 * nslots * FNH, ncomp), cluster (4, 1, 1).
template <bool INV, bool GREEN>
__global__ void __launch_bounds__(XT, 1) k_fft_xy(const float2* in, float2* out, StepArgs A, const int* slot_peak) {
  extern __shared__ __align__(16) float2 xs[];
  float2* t = xs;              // [FN]
  float2* buf = t + FN;        // [XR][XS]
  cg::cluster_group cluster = cg::this_cluster();
  const int c = (int)cluster.block_rank();
  const int pl = blockIdx.x >> 2, slot = pl / FNH, kz = pl - slot * FNH;
  const int comp = blockIdx.y, ncomp = gridDim.y;
  GreenPlane gp{};
  int pk = 0;
  if (GREEN) {
    pk = slot_peak[slot];
    if (!A.clocks[pk].has_delta) return;  // uniform over the cluster: nobody reaches a barrier
    const PeakDesc& P = A.peaks[pk];
    gp.s_c = (float)(-1.5 * PM_H_I * PM_H_I / A.clocks[pk].a_grid / (double)N3);
    gp.kf = (float)(2.0 * M_PI / P.L);
    gp.dx = (float)P.dx;
    gp.sd2 = P.smooth > 0 ? (float)(P.smooth * P.dx) * (float)(P.smooth * P.dx) : 0.f;
    gp.gm = P.gradient;
  }
  load_tw<XT>(t);
  const float2* src = in + (long long)pl * N2;
  double w = 0.0;  // potential-energy partial (component 0 of the Green pass)
  constexpr int PER = XR * FN / XT;  // elements per thread
  float2 vin[PER];
  if (GREEN) {
#pragma unroll
    for (int i = 0; i < PER; ++i) {  // all loads in flight before any is used
      const int e = threadIdx.x + i * XT, x1 = e / FN, y = e - x1 * FN;
      vin[i] = src[(long long)(4 * x1 + c) * FN + y];
    }
  } else {
    for (int e = threadIdx.x; e < XR * FN; e += XT) {
      const int x1 = e / FN, y = e - x1 * FN;
      cpa8(buf + x1 * XS + y, src + (long long)(4 * x1 + c) * FN + y);
    }
    cpa_wait();
  }
#pragma unroll
  for (int i = 0; i < (GREEN ? PER : 0); ++i) {
    const int e = threadIdx.x + i * XT;
    const int x1 = e / FN, y = e - x1 * FN, x = 4 * x1 + c;
    float2 v = vin[i];
    {
      const float kx = kl(x, gp.kf), ky = kl(y, gp.kf), kzv = gp.kf * (float)kz;
      const float k2 = kx * kx + ky * ky + kzv * kzv;
      if (x == 0 && y == 0 && kz == 0) {
        v = make_float2(0.f, 0.f);
      } else {
        float G = gp.s_c / k2;
        if (gp.sd2 > 0.f) G *= expf(-0.5f * k2 * gp.sd2);
        const float kc = comp == 0 ? kx : (comp == 1 ? ky : kzv);
        const float g = gk(kc, gp.dx, gp.gm) * G;
        if (comp == 0) w += (double)(((kz == 0 || kz == FM) ? 1.0f : 2.0f) * G * (v.x * v.x + v.y * v.y));
        float2 o = make_float2(g * v.y, -g * v.x);  // -i g v
        if (kz == 0 || kz == FM) {  // (o + conj(o at -k)) / 2: numpy's C2R sees this plane's Hermitian part
          const int px = (-x) & (FN - 1), py = (-y) & (FN - 1);
          const float2 dp = src[(long long)px * FN + py];
          const float kpc = comp == 0 ? kl(px, gp.kf) : (comp == 1 ? kl(py, gp.kf) : kzv);
          const float h = gk(kpc, gp.dx, gp.gm) * G;
          o = make_float2(0.5f * (o.x + h * dp.y), 0.5f * (o.y + h * dp.x));
        }
        v = o;
      }
    }
    buf[x1 * XS + y] = v;
  }
  if (GREEN && comp == 0) {
    for (int d = 16; d > 0; d >>= 1) w += __shfl_down_sync(0xffffffffu, w, d);
    if ((threadIdx.x & 31) == 0)
      A.wpart[A.peaks[pk].mode_base * (PM_THREADS / 32) + ((long long)kz * 4 + c) * (XT / 32) + (threadIdx.x >> 5)] = w;
  }
  __syncthreads();
  dif4<INV, FN, FN, XT, false>(buf, XR, [](int s) { return s * XS; }, 1, t);   // along y, 64 rows
  dif4<INV, XR, XR, XT, true>(buf, FN, [](int s) { return s; }, XS, t);        // along x1, 256 columns
  // Undo the digit reversal along y in place (an involution: swap each pair once), so the
  // cross-CTA reads below run along consecutive addresses.
  for (int e = threadIdx.x; e < XR * FN; e += XT) {
    const int row = e / FN, y = e - row * FN, ry = rev4_4(y);
    if (y < ry) {
      float2* r = buf + row * XS;
      const float2 v = r[y];
      r[y] = r[ry];
      r[ry] = v;
    }
  }
  cluster.sync();
  // out[k1 + 64 c][y] = sum_cc W_256^{cc k1} W_4^{cc c} F_cc[k1][y]
  float2* dst = out + ((long long)(slot * ncomp + comp) * FNH + kz) * N2;
  const float2* rbs[4];
#pragma unroll
  for (int cc = 0; cc < 4; ++cc) rbs[cc] = cluster.map_shared_rank(buf, cc);
  for (int e = threadIdx.x; e < XR * FN; e += XT) {
    const int k1 = e / FN, yn = e - k1 * FN;
    const int at = rev4_3(k1) * XS + yn;
    float2 acc = make_float2(0.f, 0.f);
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) {
      const float2 f = cmul(rbs[cc][at], w256<INV>(t, cc * k1));
      // W_4^{cc c}: 1, -i, -1, +i (forward; conjugate for the inverse)
      const int m = (cc * c) & 3;
      const float2 r = m == 0 ? f : (m == 2 ? make_float2(-f.x, -f.y) : (m == 1 ? mul_w4<INV>(f) : mul_w4<!INV>(f)));
      acc = cadd(acc, r);
    }
    dst[(long long)(k1 + XR * c) * FN + yn] = acc;
  }
  cluster.sync();  // the other CTAs have finished reading this CTA's rows
}

constexpr size_t kZSmem = sizeof(float2) * (FN + ZT * ZS + FNH * TT);
constexpr size_t kXYSmem = sizeof(float2) * (FN + XR * XS);

template <bool INV, bool GREEN>
cudaError_t launch_xy(const float2* in, float2* out, const StepArgs& A, const int* slot_peak, int nslots, int ncomp,
                      cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(4u * (unsigned)nslots * FNH, (unsigned)ncomp, 1);
  cfg.blockDim = dim3(XT, 1, 1);
  cfg.dynamicSmemBytes = kXYSmem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 4;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_fft_xy<INV, GREEN>, in, out, A, slot_peak);
}

}  // namespace

// Per-device set-up: twiddle table and shared-memory limits.  Call with the device current.
int fft256_init() {
  float2 h[FN];
  for (int k = 0; k < FN; ++k) {
    const double a = -2.0 * M_PI * (double)k / (double)FN;
    h[k] = make_float2((float)cos(a), (float)sin(a));
  }
  cudaError_t e = cudaMemcpyToSymbol(g_tw, h, sizeof(h));
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fft_z_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kZSmem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fft_z_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kZSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_fft_xy<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kXYSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_fft_xy<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kXYSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_fft_xy<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kXYSmem);
  return e == cudaSuccess ? 0 : -(int)e;
}

// delta fields [slot][x][y][z] -> spectra [slot][kz][kx][ky]
int fft256_r2c(const float* delta, float2* spec, int nslots, cudaStream_t s) {
  if (nslots <= 0) return 0;
  k_fft_z_r2c<<<dim3(FN / ZT, FN, nslots), FT, kZSmem, s>>>(delta, spec);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = launch_xy<false, false>(spec, spec, StepArgs{}, nullptr, nslots, 1, s);
  return e == cudaSuccess ? 0 : -(int)e;
}

// spectra [slot][kz][kx][ky] -> 3 force grids per slot [slot][comp][x][y][z] through the
// Green multiply; gwork holds [slot][comp][kz][x][y].
int fft256_green_c2r(const float2* spec, float2* gwork, float* force, const StepArgs& A, const int* slot_peak,
                     int nslots, cudaStream_t s) {
  if (nslots <= 0) return 0;
  cudaError_t e = launch_xy<true, true>(spec, gwork, A, slot_peak, nslots, 3, s);
  if (e == cudaSuccess) {
    k_fft_z_c2r<<<dim3(FN / ZT, FN, 3 * nslots), FT, kZSmem, s>>>(gwork, force);
    e = cudaGetLastError();
  }
  return e == cudaSuccess ? 0 : -(int)e;
}

// Plain unnormalised inverse: spectra [f][kz][kx][ky] -> fields [f][x][y][z]; gwork as spec.
int fft256_c2r(const float2* spec, float2* gwork, float* out, int nfields, cudaStream_t s) {
  if (nfields <= 0) return 0;
  cudaError_t e = launch_xy<true, false>(spec, gwork, StepArgs{}, nullptr, nfields, 1, s);
  if (e == cudaSuccess) {
    k_fft_z_c2r<<<dim3(FN / ZT, FN, nfields), FT, kZSmem, s>>>(gwork, out);
    e = cudaGetLastError();
  }
  return e == cudaSuccess ? 0 : -(int)e;
}

namespace {
int ensure_fft256_init() {
  static int done[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return -(int)e;
  if (dev < 0 || dev >= 64) return -2004;
  if (!done[dev]) {
    if (int r = fft256_init()) return r;
    done[dev] = 1;
  }
  return 0;
}
}  // namespace

extern "C" int pm_rfft3_256(const float* x, void* spec, int nfields, void* stream) {
  if (!x || !spec || nfields < 0) return -2000;
  if (int r = ensure_fft256_init()) return r;
  return fft256_r2c(x, (float2*)spec, nfields, (cudaStream_t)stream);
}

extern "C" int pm_irfft3_256(const void* spec, void* work, float* x, int nfields, void* stream) {
  if (!spec || !work || !x || nfields < 0) return -2000;
  if (int r = ensure_fft256_init()) return r;
  return fft256_c2r((const float2*)spec, (float2*)work, x, nfields, (cudaStream_t)stream);
}
