// Native 3D real FFT for the 256^3 mesh (sm_100a), with the Green's-function gradient
// (pm3d.py:105-112) fused into the inverse.
//
// Layouts (one field; fields of a batch are consecutive):
//   real field      r[x][y][z]          256^3 float (the deposit's delta, the force grids)
//   spectrum        s[kz][kx][ky]       129 x 256 x 256 complex ("plane-major")
// numpy's rfftn(r)[kx][ky][kz] is s[kz][kx][ky]: the same transform, stored with kz outermost.
//
// Every 1D transform is a two-factor (Cooley-Tukey "four-step") transform held in registers:
// a line of length L = 16 T is owned by T threads, thread t holding the 16 elements
// n = T n1 + t, n1 = 0..15.  Each thread runs a 16-point DFT over n1 in registers and scales by
// W_L^{t k1}; one shared-memory exchange hands every thread the T values of its k1 for the
// T-point DFTs of the second factor; output k = k1 + 16 k2.  Register DFTs are radix-2
// decimation in frequency, so their outputs sit in bit-reversed register order (compile-time).
// Exchange layouts are laid out (XOR-swizzled where needed) so that both the write and the
// read side of every exchange hit distinct shared-memory banks within each half-warp.
//
// Forward (R2C), three passes over HBM.  Pass Z: a real FFT along z of 32 (x, y) lines per CTA
// -- a complex 128-point FFT of the packed (even, odd) pairs, then the split into 129 outputs --
// written transposed into the kz planes.  Pass Y: 16 rows of a kz plane per CTA, in place.
// Pass X: 16 columns of a kz plane per CTA (128-byte row segments), in place.  Every pass is
// 256 threads and 34-38 KB of shared memory, 4 CTAs per SM, with no inter-CTA communication.
// Inverse (C2R).  Pass Y with the Green multiply on load (-i k_i G(k) delta_k / N^3, the
// Hermitian projection of the kz = 0, N/2 planes, the potential-energy partials), one CTA per
// row block and gradient component (the three components of a row block adjacent in the grid,
// so the spectrum is read from HBM once); pass X in place; pass Z, the real inverse along z,
// written as force rows.
// Twiddles come from a 256-entry table computed in double precision on the host; the register
// DFTs use the exact constants cos(pi/8), cos(pi/4), cos(3 pi/8).
// Transforms are unnormalised like cuFFT's; the Green factor carries numpy's 1/N^3.
#include <cmath>
#include <cstdint>

#include "pm_kernels.cuh"


namespace {

constexpr int FN = 256;            // mesh side
constexpr int FNH = FN / 2 + 1;    // kz planes
constexpr int FM = FN / 2;         // packed complex length of a z line
constexpr int ZL = 32;             // z lines per CTA in the Z passes
constexpr int ZTH = ZL * 8;        // threads of a Z-pass CTA (8 per line)
constexpr int ZX = FM + 8;         // row stride (float2) of a z line in shared memory, = 8 mod 16
constexpr int ZC = ZL + 2;         // stride of the kz-major input tile of the inverse, = 2 mod 16
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

__host__ __device__ constexpr int brev(int p, int bits) {
  int r = 0;
  for (int i = 0; i < bits; ++i) r |= ((p >> i) & 1) << (bits - 1 - i);
  return r;
}

// x W_16^e (conjugate twiddle for the inverse).  e is a compile-time constant wherever this is
// called from the unrolled register DFTs, so the branches and constants fold away.
template <bool INV>
__device__ __forceinline__ float2 mul_w16(float2 x, int e) {
  e &= 15;
  if (e == 0) return x;
  if (e == 8) return make_float2(-x.x, -x.y);
  if (e == 4) return mul_w4<INV>(x);
  if (e == 12) return mul_w4<!INV>(x);
  constexpr float C1 = 0.923879532511286756f, C2 = 0.707106781186547524f, C3 = 0.382683432365089772f;
  const int q = e >> 2, r = e & 3;
  const float cb = r == 1 ? C1 : (r == 2 ? C2 : C3), sb = r == 1 ? C3 : (r == 2 ? C2 : C1);
  // (cos, sin) of 2 pi e / 16: the base angle r pi / 8 turned by q quarter turns
  const float c = q == 0 ? cb : (q == 1 ? -sb : (q == 2 ? -cb : sb));
  const float s = q == 0 ? sb : (q == 1 ? cb : (q == 2 ? -sb : -cb));
  return cmul(x, make_float2(c, INV ? s : -s));
}

// Radix-2 DIF DFT of length L on v[OFF .. OFF + L - 1] in registers: afterwards v[OFF + p] holds
// output brev(p, log2 L).
template <bool INV, int L, int OFF, int NV>
__device__ __forceinline__ void dft_reg(float2 (&v)[NV]) {
  if constexpr (L > 1) {
#pragma unroll
    for (int j = 0; j < L / 2; ++j) {
      const float2 a = v[OFF + j], b = v[OFF + j + L / 2];
      v[OFF + j] = cadd(a, b);
      v[OFF + j + L / 2] = mul_w16<INV>(csub(a, b), j * (16 / L));
    }
    dft_reg<INV, L / 2, OFF, NV>(v);
    dft_reg<INV, L / 2, OFF + L / 2, NV>(v);
  }
}

__device__ __forceinline__ void cpa16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Shared twiddle tables of the Z passes: tw[e] = W_256^e, t8[k1 * 8 + t] = W_128^{t k1}
// (conjugated for the inverse).
template <bool INV>
__device__ __forceinline__ void load_ztw(float2* tw, float2* t8) {
  for (int i = threadIdx.x; i < FN; i += ZTH) {
    const float2 w = g_tw[i];
    tw[i] = INV ? cconj(w) : w;
  }
  for (int i = threadIdx.x; i < FM; i += ZTH) {
    const float2 w = g_tw[(2 * (i >> 3) * (i & 7)) & (FN - 1)];
    t8[i] = INV ? cconj(w) : w;
  }
}

// The 128-point transform of one packed z line shared by 8 threads (thread t holds v[n1] =
// element 8 n1 + t): returns u[8 s + q] = element k1 + 16 brev(q, 3) of the transform, k1 = t + 8 s.
// row: this line's exchange row in shared memory.  Ends after the exchange has been read: the
// caller must barrier before it writes the row again.
template <bool INV>
__device__ __forceinline__ void fft128_line(float2 (&v)[16], float2 (&u)[16], float2* row, const float2* t8, int t) {
  dft_reg<INV, 16, 0, 16>(v);
#pragma unroll
  for (int p = 0; p < 16; ++p) {
    const int k1 = brev(p, 4);
    row[k1 * 8 + (t ^ (k1 & 7))] = k1 ? cmul(v[p], t8[k1 * 8 + t]) : v[p];
  }
  __syncthreads();
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int j = 0; j < 8; ++j) u[8 * s + j] = row[(t + 8 * s) * 8 + (j ^ t)];
  dft_reg<INV, 8, 0, 16>(u);
  dft_reg<INV, 8, 8, 16>(u);
}

// Pass Z forward: fields in[f][x][y][z] -> planes out[f][kz][x][y].  grid (FN/ZL, FN, nf).
__global__ void __launch_bounds__(ZTH, 4) k_fft_z_r2c(const float* __restrict__ in, float2* __restrict__ out) {
  __shared__ float2 tw[FN], t8[FM];
  __shared__ __align__(16) float2 xb[ZL * ZX];
  load_ztw<false>(tw, t8);
  const int t = threadIdx.x & 7, l = threadIdx.x >> 3;
  const int y0 = blockIdx.x * ZL, x = blockIdx.y, f = blockIdx.z;
  const float2* src = reinterpret_cast<const float2*>(in + (long long)f * N3 + ((long long)x * FN + y0 + l) * FN);
  float2 v[16], u[16];
#pragma unroll
  for (int n1 = 0; n1 < 16; ++n1) v[n1] = __ldg(src + 8 * n1 + t);  // (r[2n], r[2n+1]), n = 8 n1 + t
  __syncthreads();  // tables
  float2* row = xb + l * ZX;
  fft128_line<false>(v, u, row, t8, t);
  __syncthreads();
  // Z_k into the line's row in natural order, swizzled so that the column reads below are
  // conflict-free: Z_k at row[k ^ sw(l)].
  const int sw = (l >> 1) & 7;
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int q = 0; q < 8; ++q) row[(t + 8 * s + 16 * brev(q, 3)) ^ sw] = u[8 * s + q];
  __syncthreads();
  // X_k = E_k + W_256^k O_k with E = (Z_k + conj Z_{M-k})/2, O = -i (Z_k - conj Z_{M-k})/2
  float2* dst = out + (long long)f * FNH * N2 + (long long)x * FN + y0;
  for (int e = threadIdx.x; e < FNH * ZL; e += ZTH) {
    const int k = e / ZL, ll = e - k * ZL, sl = (ll >> 1) & 7;
    const float2* zr = xb + ll * ZX;
    const float2 zk = zr[(k & (FM - 1)) ^ sl];
    const float2 zm = cconj(zr[((FM - k) & (FM - 1)) ^ sl]);
    const float2 E = cscale(cadd(zk, zm), 0.5f);
    const float2 O = cscale(mul_w4<false>(csub(zk, zm)), 0.5f);
    dst[(long long)k * N2 + ll] = cadd(E, cmul(tw[k], O));
  }
}

// Pass Z inverse: planes in[f][kz][x][y] -> fields out[f][x][y][z].  grid (FN/ZL, FN, nf).
__global__ void __launch_bounds__(ZTH, 4) k_fft_z_c2r(const float2* __restrict__ in, float* __restrict__ out) {
  __shared__ float2 tw[FN], t8[FM];
  __shared__ __align__(16) float2 xb[FNH * ZC];  // the kz-major tile, later the exchange rows
  static_assert(FNH * ZC >= ZL * ZX, "exchange rows fit in the tile");
  const int y0 = blockIdx.x * ZL, x = blockIdx.y, f = blockIdx.z;
  const float2* src = in + (long long)f * FNH * N2 + (long long)x * FN + y0;
  for (int e = threadIdx.x; e < FNH * ZL / 2; e += ZTH) {  // two complex values (16 bytes) per copy
    const int k = e / (ZL / 2), ll = 2 * (e - k * (ZL / 2));
    cpa16(xb + k * ZC + ll, src + (long long)k * N2 + ll);
  }
  load_ztw<true>(tw, t8);
  cpa_wait();
  __syncthreads();
  const int t = threadIdx.x & 7, l = threadIdx.x >> 3;
  // Z_n = E_n + i O_n with E = X_n + conj X_{M-n}, O = (X_n - conj X_{M-n}) W_256^{-n}; a C2R
  // reads only the real parts of X_0 and X_M.
  float2 v[16], u[16];
#pragma unroll
  for (int n1 = 0; n1 < 16; ++n1) {
    const int n = 8 * n1 + t;
    float2 xk = xb[n * ZC + l], xm = cconj(xb[(FM - n) * ZC + l]);
    if (n == 0) {
      xk.y = 0.f;
      xm.y = 0.f;
    }
    const float2 O = cmul(csub(xk, xm), tw[n]);
    v[n1] = cadd(cadd(xk, xm), make_float2(-O.y, O.x));
  }
  __syncthreads();  // the tile is read; its memory becomes the exchange rows
  fft128_line<true>(v, u, xb + l * ZX, t8, t);
  float2* dst = reinterpret_cast<float2*>(out + (long long)f * N3 + ((long long)x * FN + y0 + l) * FN);
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int q = 0; q < 8; ++q) dst[t + 8 * s + 16 * brev(q, 3)] = u[8 * s + q];  // (r[2n], r[2n+1])
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
// -i g_comp(k) G(k) delta_k at mode (x, y, kz) of a plane whose values start at plane; adds the
// mode's weight in the potential energy to w (component 0).
__device__ __forceinline__ float2 green_mode(float2 v, int x, int y, int kz, int comp, const GreenPlane& gp,
                                             const float2* plane, double& w) {
  const float kx = kl(x, gp.kf), ky = kl(y, gp.kf), kzv = gp.kf * (float)kz;
  const float k2 = kx * kx + ky * ky + kzv * kzv;
  if (x == 0 && y == 0 && kz == 0) return make_float2(0.f, 0.f);
  float G = gp.s_c / k2;
  if (gp.sd2 > 0.f) G *= expf(-0.5f * k2 * gp.sd2);
  const float kc = comp == 0 ? kx : (comp == 1 ? ky : kzv);
  const float g = gk(kc, gp.dx, gp.gm) * G;
  if (comp == 0) w += (double)(((kz == 0 || kz == FM) ? 1.0f : 2.0f) * G * (v.x * v.x + v.y * v.y));
  float2 o = make_float2(g * v.y, -g * v.x);  // -i g v
  if (kz == 0 || kz == FM) {  // (o + conj(o at -k)) / 2: numpy's C2R sees this plane's Hermitian part
    const int px = (-x) & (FN - 1), py = (-y) & (FN - 1);
    const float2 dp = plane[(long long)px * FN + py];
    const float kpc = comp == 0 ? kl(px, gp.kf) : (comp == 1 ? kl(py, gp.kf) : kzv);
    const float h = gk(kpc, gp.dx, gp.gm) * G;
    o = make_float2(0.5f * (o.x + h * dp.y), 0.5f * (o.y + h * dp.x));
  }
  return o;
}

constexpr int RB = 16;        // lines per CTA of the plane passes
constexpr int RT = RB * 16;   // threads (16 per line)

// Pass Y: rows x = RB rb + r of one kz plane, 16 threads per row.  Forward: in = out =
// planes[slot][kz][x][y] (in place: a CTA reads its rows before it writes them).  Inverse with
// GREEN: in = spectrum planes[slot][kz][kx][ky], out = planes[slot][comp][kz][kx][y], the
// multiply applied on load; slot_peak maps a slot to its peak.  Inverse without GREEN: in and
// out [f][kz][.][.].  grid (FN/RB * nslots * FNH * ncomp), block index
// ((slot * FNH + kz) * (FN/RB) + rb) * ncomp + comp (the components of a row block adjacent).
template <bool INV, bool GREEN>
__global__ void __launch_bounds__(RT, 4) k_fft_rows(const float2* in, float2* out, StepArgs A, const int* slot_peak,
                                                     int ncomp) {
  __shared__ float2 ty[FN];
  __shared__ __align__(16) float2 buf[RB * FN];
  for (int i = threadIdx.x; i < FN; i += RT) {
    const float2 b = g_tw[((i >> 4) * (i & 15)) & (FN - 1)];
    ty[i] = INV ? cconj(b) : b;
  }
  const int bi = blockIdx.x, comp = bi % ncomp, q = bi / ncomp, rb = q % (FN / RB), pl = q / (FN / RB);
  const int slot = pl / FNH, kz = pl - slot * FNH;
  GreenPlane gp{};
  int pk = 0;
  if (GREEN) {
    pk = slot_peak[slot];
    if (!A.clocks[pk].has_delta) return;
    const PeakDesc& P = A.peaks[pk];
    gp.s_c = (float)(-1.5 * PM_H_I * PM_H_I / A.clocks[pk].a_grid / (double)N3);
    gp.kf = (float)(2.0 * M_PI / P.L);
    gp.dx = (float)P.dx;
    gp.sd2 = P.smooth > 0 ? (float)(P.smooth * P.dx) * (float)(P.smooth * P.dx) : 0.f;
    gp.gm = P.gradient;
  }
  const int t = threadIdx.x & 15, r = threadIdx.x >> 4, x = RB * rb + r;
  const float2* plane = in + (long long)pl * N2;
  float2 v[16], u[16];
#pragma unroll
  for (int n1 = 0; n1 < 16; ++n1) v[n1] = plane[(long long)x * FN + 16 * n1 + t];
  float2* row = buf + r * FN;
  double w = 0.0;
  if (GREEN) {
    if (kz != 0 && kz != FM && (gp.gm == 0 || comp != 1)) {
      // Interior planes (no Hermitian partner, k != 0), with the gradient factor constant along
      // the row (components x and z) or the spectral ky (component y): unrolled, in registers.
      const float kx = kl(x, gp.kf), kzv = gp.kf * (float)kz, a = kx * kx + kzv * kzv;
      const float gc = gk(comp == 0 ? kx : kzv, gp.dx, gp.gm);
#pragma unroll
      for (int n1 = 0; n1 < 16; ++n1) {
        const float ky = kl(16 * n1 + t, gp.kf), k2 = a + ky * ky;
        float G = gp.s_c / k2;
        if (gp.sd2 > 0.f) G *= expf(-0.5f * k2 * gp.sd2);
        const float g = (comp == 1 ? ky : gc) * G;
        const float2 d = v[n1];
        if (comp == 0) w += (double)(2.0f * G * (d.x * d.x + d.y * d.y));
        v[n1] = make_float2(g * d.y, -g * d.x);  // -i g d
      }
    } else {
      // The general multiply in a rolled loop over this thread's slots of its row in shared
      // memory (one copy of its code keeps the kernel within the instruction cache).
      float2* own = row + t;
#pragma unroll
      for (int n1 = 0; n1 < 16; ++n1) own[16 * n1] = v[n1];
#pragma unroll 1
      for (int n1 = 0; n1 < 16; ++n1) own[16 * n1] = green_mode(own[16 * n1], x, 16 * n1 + t, kz, comp, gp, plane, w);
#pragma unroll
      for (int n1 = 0; n1 < 16; ++n1) v[n1] = own[16 * n1];
    }
    if (comp == 0)
      for (int d = 16; d > 0; d >>= 1) w += __shfl_down_sync(0xffffffffu, w, d);
  }
  __syncthreads();
  dft_reg<INV, 16, 0, 16>(v);
#pragma unroll
  for (int p = 0; p < 16; ++p) {
    const int k1 = brev(p, 4);
    row[k1 * 16 + (t ^ k1)] = k1 ? cmul(v[p], ty[k1 * 16 + t]) : v[p];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < 16; ++j) u[j] = row[t * 16 + (j ^ t)];
  dft_reg<INV, 16, 0, 16>(u);
  float2* dst = out + ((long long)(slot * ncomp + comp) * FNH + kz) * N2 + (long long)x * FN;
#pragma unroll
  for (int p = 0; p < 16; ++p) dst[t + 16 * brev(p, 4)] = u[p];
  if (GREEN && comp == 0 && (threadIdx.x & 31) == 0)
    A.wpart[A.peaks[pk].mode_base * (PM_THREADS / 32) + ((long long)kz * (FN / RB) + rb) * (RT / 32) + (threadIdx.x >> 5)] = w;
}

// Pass X, in place: columns ky = RB cb + j of one kz plane, 16 threads per column (a warp reads
// and writes 128-byte segments of two rows).  grid (FN/RB * nplanes).
template <bool INV>
__global__ void __launch_bounds__(RT, 4) k_fft_cols(float2* io) {
  __shared__ float2 ty[FN];
  __shared__ __align__(16) float2 buf[RB * FN];  // [k1][t][j]
  for (int i = threadIdx.x; i < FN; i += RT) {
    const float2 b = g_tw[((i >> 4) * (i & 15)) & (FN - 1)];
    ty[i] = INV ? cconj(b) : b;
  }
  const int cb = blockIdx.x % (FN / RB), pl = blockIdx.x / (FN / RB);
  const int j = threadIdx.x & 15, t = threadIdx.x >> 4, ky = RB * cb + j;
  float2* plane = io + (long long)pl * N2 + ky;
  float2 v[16], u[16];
#pragma unroll
  for (int n1 = 0; n1 < 16; ++n1) v[n1] = plane[(long long)(16 * n1 + t) * FN];
  __syncthreads();
  dft_reg<INV, 16, 0, 16>(v);
#pragma unroll
  for (int p = 0; p < 16; ++p) {
    const int k1 = brev(p, 4);
    buf[(k1 * 16 + t) * RB + j] = k1 ? cmul(v[p], ty[k1 * 16 + t]) : v[p];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 16; ++i) u[i] = buf[(t * 16 + i) * RB + j];
  dft_reg<INV, 16, 0, 16>(u);
#pragma unroll
  for (int p = 0; p < 16; ++p) plane[(long long)(t + 16 * brev(p, 4)) * FN] = u[p];
}

}  // namespace

// Per-device set-up: the twiddle table.  Call with the device current.
int fft256_init() {
  float2 h[FN];
  for (int k = 0; k < FN; ++k) {
    const double a = -2.0 * M_PI * (double)k / (double)FN;
    h[k] = make_float2((float)cos(a), (float)sin(a));
  }
  cudaError_t e = cudaMemcpyToSymbol(g_tw, h, sizeof(h));
  return e == cudaSuccess ? 0 : -(int)e;
}

// delta fields [slot][x][y][z] -> spectra [slot][kz][kx][ky]
int fft256_r2c(const float* delta, float2* spec, int nslots, cudaStream_t s) {
  if (nslots <= 0) return 0;
  k_fft_z_r2c<<<dim3(FN / ZL, FN, nslots), ZTH, 0, s>>>(delta, spec);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    k_fft_rows<false, false><<<(unsigned)((FN / RB) * nslots * FNH), RT, 0, s>>>(spec, spec, StepArgs{}, nullptr, 1);
    k_fft_cols<false><<<(unsigned)((FN / RB) * nslots * FNH), RT, 0, s>>>(spec);
    e = cudaGetLastError();
  }
  return e == cudaSuccess ? 0 : -(int)e;
}

// spectra [slot][kz][kx][ky] -> 3 force grids per slot [slot][comp][x][y][z] through the
// Green multiply; gwork holds [slot][comp][kz][x][y].
int fft256_green_c2r(const float2* spec, float2* gwork, float* force, const StepArgs& A, const int* slot_peak,
                     int nslots, cudaStream_t s) {
  if (nslots <= 0) return 0;
  k_fft_rows<true, true><<<(unsigned)((FN / RB) * nslots * FNH * 3), RT, 0, s>>>(spec, gwork, A, slot_peak, 3);
  k_fft_cols<true><<<(unsigned)((FN / RB) * nslots * FNH * 3), RT, 0, s>>>(gwork);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    k_fft_z_c2r<<<dim3(FN / ZL, FN, 3 * nslots), ZTH, 0, s>>>(gwork, force);
    e = cudaGetLastError();
  }
  return e == cudaSuccess ? 0 : -(int)e;
}

// Plain unnormalised inverse: spectra [f][kz][kx][ky] -> fields [f][x][y][z]; gwork as spec.
int fft256_c2r(const float2* spec, float2* gwork, float* out, int nfields, cudaStream_t s) {
  if (nfields <= 0) return 0;
  k_fft_rows<true, false><<<(unsigned)((FN / RB) * nfields * FNH), RT, 0, s>>>(spec, gwork, StepArgs{}, nullptr, 1);
  k_fft_cols<true><<<(unsigned)((FN / RB) * nfields * FNH), RT, 0, s>>>(gwork);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    k_fft_z_c2r<<<dim3(FN / ZL, FN, nfields), ZTH, 0, s>>>(gwork, out);
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
  if (((uintptr_t)x | (uintptr_t)spec) & 15) return -2001;  // 16-byte copies
  if (int r = ensure_fft256_init()) return r;
  return fft256_r2c(x, (float2*)spec, nfields, (cudaStream_t)stream);
}

extern "C" int pm_irfft3_256(const void* spec, void* work, float* x, int nfields, void* stream) {
  if (!spec || !work || !x || nfields < 0) return -2000;
  if (((uintptr_t)x | (uintptr_t)spec | (uintptr_t)work) & 15) return -2001;
  if (int r = ensure_fft256_init()) return r;
  return fft256_c2r((const float2*)spec, (float2*)work, x, nfields, (cudaStream_t)stream);
}
