// Native 3D real FFT for meshes of 64^3 to 512^3 (sm_100a), with the Green's-function gradient
// (pm3d.py:105-112) fused into the inverse.
//
// Layouts (one field; fields of a batch are consecutive), N = 64, 128, 256 or 512:
//   real field      r[x][y][z]          N^3 float (the deposit's delta, the force grids)
//   spectrum        s[kz][kx][ky]       (N/2+1) x N x N complex ("plane-major")
// numpy's rfftn(r)[kx][ky][kz] is s[kz][kx][ky]: the same transform, stored with kz outermost.
//
// Every 1D transform is a two-factor (Cooley-Tukey "four-step") transform held in registers:
// a line of length L = 16 T is owned by T threads, thread t holding the 16 elements
// n = T n1 + t, n1 = 0..15.  Each thread runs a 16-point DFT over n1 in registers and scales by
// W_L^{t k1}; one shared-memory exchange hands the threads the T values of each k1 for the
// T-point DFTs of the second factor; output k = k1 + 16 k2.  For T <= 16 a thread does 16/T
// DFTs of T points; for T = 32 a pair of threads shares each 32-point DFT (two 16-point halves
// and a radix-2 step across the pair by warp shuffle).  Register DFTs are radix-2
// decimation in frequency, so their outputs sit in bit-reversed register order (compile-time).
// Exchange layouts are XOR-swizzled and rows padded so that both the write and the read side of
// every exchange hit distinct shared-memory banks within each half-warp (for the 64^3 Z pass,
// at most two-way).
//
// Forward (R2C), three passes over HBM.  Pass Z: a real FFT along z of 256/T consecutive (x, y)
// lines per CTA (T = N/32) -- a complex FFT of the N/2 packed (even, odd) pairs, then the split
// into N/2+1 outputs -- written transposed into the kz planes.  Pass Y: 256/(N/16) rows of a kz
// plane per CTA, in place.  Pass X: the same number of columns of a kz plane per CTA, in place.
// Every
// kernel: 256 threads, at most 43 KB of static shared memory, 64 registers, 4 CTAs per SM, no
// inter-CTA communication.
// Inverse (C2R).  Pass Y with the Green multiply on load (-i k_i G(k) delta_k / N^3, the
// Hermitian projection of the kz = 0, N/2 planes, the potential-energy partials), one CTA per
// row block and gradient component (the three components of a row block adjacent in the grid,
// so the spectrum is read from HBM once); pass X in place; pass Z, the real inverse along z,
// written as force rows.
// Twiddles come from a 512-entry table of W_512^e computed in double precision on the host; the
// register DFTs use the exact constants cos(pi/8), cos(pi/4), cos(3 pi/8).
// Transforms are unnormalised like cuFFT's; the Green factor carries numpy's 1/N^3.
#include <cmath>
#include <cstdint>

#include <mutex>

#include "pm_kernels.cuh"

namespace {

constexpr int TWN = 512;           // entries of the twiddle table
constexpr int CTA = 256;           // threads of every kernel here

__device__ float2 g_tw[TWN];       // exp(-2 pi i e / 512) of this device

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

// W_L^e from the table (conjugated for the inverse); L divides 512.
template <bool INV, int L>
__device__ __forceinline__ float2 tw_global(int e) {
  const float2 w = g_tw[(e * (TWN / L)) & (TWN - 1)];
  return INV ? cconj(w) : w;
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

template <int T>
__host__ __device__ constexpr int log2i() { return T <= 1 ? 0 : 1 + log2i<T / 2>(); }

// T-point DFTs of the 16 / T consecutive groups of u.
template <bool INV, int T, int S = 0>
__device__ __forceinline__ void dft_groups(float2 (&u)[16]) {
  if constexpr (S < 16 / T) {
    dft_reg<INV, T, T * S, 16>(u);
    dft_groups<INV, T, S + 1>(u);
  }
}

// Output element held in u[p] by thread t of a line of T threads after line_fft: for T <= 16
// group s = p / T of the thread's 16 / T groups, element q = p % T of its T-point DFT.
template <int T>
__device__ __forceinline__ int line_k(int t, int p) {
  if constexpr (T <= 16) return t + T * (p / T) + 16 * brev(p % T, log2i<T>());
  else return (t >> 1) + 16 * brev(p, 4) + 256 * (t & 1);
}

// Swizzled position of Y[k1][t] in a line's exchange row.
template <int T>
__device__ __forceinline__ int line_slot(int k1, int t) {
  if constexpr (T <= 16) return k1 * T + (t ^ (k1 & (T - 1)));
  else return k1 * 32 + (t ^ (2 * k1));
}

// The transform of one line of L = 16 T points shared by its T threads: thread t holds v[n1] =
// x[T n1 + t] on entry and u[p] = X[line_k<T>(t, p)] on exit.  row: the line's exchange row in
// shared memory (16 T values); tl: W_L^{t k1} at [k1 * T + t].  The threads of a line are
// consecutive lanes of one warp (T = 32: the whole warp).  Ends after the exchange has been read:
// the caller must barrier before it writes the row again.
template <bool INV, int T>
__device__ __forceinline__ void line_fft(float2 (&v)[16], float2 (&u)[16], float2* row, const float2* tl, int t) {
  dft_reg<INV, 16, 0, 16>(v);
#pragma unroll
  for (int p = 0; p < 16; ++p) {
    const int k1 = brev(p, 4);
    row[line_slot<T>(k1, t)] = k1 ? cmul(v[p], tl[k1 * T + t]) : v[p];
  }
  __syncthreads();
  if constexpr (T <= 16) {
    // this thread's k1 = t + T s, s < 16 / T: one T-point DFT each
#pragma unroll
    for (int s = 0; s < 16 / T; ++s)
#pragma unroll
      for (int j = 0; j < T; ++j) u[T * s + j] = row[line_slot<T>(t + T * s, j)];
    dft_groups<INV, T>(u);
  } else {
    // k1 = t / 2; this thread's half t0 = t & 1 of the 32 values: Y[k1][2 t1 + t0], t1 = 0..15
    const int k1 = t >> 1, t0 = t & 1;
#pragma unroll
    for (int j = 0; j < 16; ++j) u[j] = row[line_slot<32>(k1, 2 * j + t0)];
    dft_reg<INV, 16, 0, 16>(u);  // u[p] = A_t0[m], m = brev(p)
#pragma unroll
    for (int p = 0; p < 16; ++p) {
      if (t0) u[p] = cmul(u[p], tl[brev(p, 4) * 32 + 16]);  // W_32^m = W_512^{16 m}
      const float ox = __shfl_xor_sync(0xffffffffu, u[p].x, 1), oy = __shfl_xor_sync(0xffffffffu, u[p].y, 1);
      // X[k1 + 16 m] = A_0 + W_32^m A_1 (even lane), X[k1 + 16 m + 256] = A_0 - W_32^m A_1 (odd lane)
      u[p] = t0 ? make_float2(ox - u[p].x, oy - u[p].y) : make_float2(u[p].x + ox, u[p].y + oy);
    }
  }
}

// Z pass geometry for mesh N: a z line is M = N/2 packed pairs shared by T = M/16 threads.
template <int N>
struct ZGeo {
  static constexpr int M = N / 2, NH = N / 2 + 1, T = M / 16, L = CTA / T;  // L lines per CTA
  // Row stride (float2) of a line in shared memory and the swizzle of its natural-order row,
  // chosen so that the exchange, the row writes and the column reads of the split are free of
  // bank conflicts (T = 2: at most two-way).
  static constexpr int X = M + (T >= 8 ? 8 : T);
  static constexpr int C = L + 2;       // stride of the kz-major input tile of the inverse
  static constexpr int TILE = (NH * C > L * X) ? NH * C : L * X;
  static constexpr long long N2 = (long long)N * N, N3 = N2 * N;
  static_assert(L <= N * N, "lines per CTA");
  __device__ static int sw(int l) { return T >= 8 ? (l >> 1) & 7 : (l & 15); }
};

// Shared twiddle tables of the Z passes: tw[e] = W_N^e (e <= N/2), tl[k1 * T + t] = W_M^{t k1}.
template <bool INV, int N>
__device__ __forceinline__ void load_ztw(float2* tw, float2* tl) {
  using G = ZGeo<N>;
  for (int i = threadIdx.x; i <= G::M; i += CTA) tw[i] = tw_global<INV, N>(i);
  for (int i = threadIdx.x; i < 16 * G::T; i += CTA) tl[i] = tw_global<INV, G::M>((i / G::T) * (i % G::T));
}

__device__ __forceinline__ void cpa16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Pass Z forward: fields in[f][x][y][z] -> planes out[f][kz][x][y].  A CTA takes L consecutive
// (x, y) lines.  grid (N^2/L, nf).
template <int N>
__global__ void __launch_bounds__(CTA, 4) k_fft_z_r2c(const float* __restrict__ in, float2* __restrict__ out) {
  using G = ZGeo<N>;
  __shared__ float2 tw[G::M + 1], tl[16 * G::T];
  __shared__ __align__(16) float2 xb[G::L * G::X];
  load_ztw<false, N>(tw, tl);
  const int t = threadIdx.x % G::T, l = threadIdx.x / G::T;
  const long long g0 = (long long)blockIdx.x * G::L;  // first line (x N + y) of this CTA
  const int f = blockIdx.y;
  const float2* src = reinterpret_cast<const float2*>(in + (long long)f * G::N3 + (g0 + l) * N);
  float2 v[16], u[16];
#pragma unroll
  for (int n1 = 0; n1 < 16; ++n1) v[n1] = __ldg(src + G::T * n1 + t);  // (r[2n], r[2n+1]), n = T n1 + t
  __syncthreads();  // tables
  float2* row = xb + l * G::X;
  line_fft<false, G::T>(v, u, row, tl, t);
  __syncthreads();
  // Z_k into the line's row in natural order, swizzled so that the column reads below are
  // conflict-free: Z_k at row[k ^ sw(l)].
  const int sw = G::sw(l);
#pragma unroll
  for (int p = 0; p < 16; ++p) row[line_k<G::T>(t, p) ^ sw] = u[p];
  __syncthreads();
  // X_k = E_k + W_N^k O_k with E = (Z_k + conj Z_{M-k})/2, O = -i (Z_k - conj Z_{M-k})/2
  float2* dst = out + (long long)f * G::NH * G::N2 + g0;
  for (int e = threadIdx.x; e < G::NH * G::L; e += CTA) {
    const int k = e / G::L, ll = e - k * G::L, sl = G::sw(ll);
    const float2* zr = xb + ll * G::X;
    const float2 zk = zr[(k & (G::M - 1)) ^ sl];
    const float2 zm = cconj(zr[((G::M - k) & (G::M - 1)) ^ sl]);
    const float2 E = cscale(cadd(zk, zm), 0.5f);
    const float2 O = cscale(mul_w4<false>(csub(zk, zm)), 0.5f);
    dst[(long long)k * G::N2 + ll] = cadd(E, cmul(tw[k], O));
  }
}

// Pass Z inverse: planes in[f][kz][x][y] -> fields out[f][x][y][z].  A CTA takes L consecutive
// (x, y) lines.  grid (N^2/L, nf).
template <int N>
__global__ void __launch_bounds__(CTA, 4) k_fft_z_c2r(const float2* __restrict__ in, float* __restrict__ out) {
  using G = ZGeo<N>;
  __shared__ float2 tw[G::M + 1], tl[16 * G::T];
  __shared__ __align__(16) float2 xb[G::TILE];  // the kz-major tile, later the exchange rows
  const long long g0 = (long long)blockIdx.x * G::L;
  const int f = blockIdx.y;
  const float2* src = in + (long long)f * G::NH * G::N2 + g0;
  for (int e = threadIdx.x; e < G::NH * G::L / 2; e += CTA) {  // two complex values (16 bytes) per copy
    const int k = e / (G::L / 2), ll = 2 * (e - k * (G::L / 2));
    cpa16(xb + k * G::C + ll, src + (long long)k * G::N2 + ll);
  }
  load_ztw<true, N>(tw, tl);
  cpa_wait();
  __syncthreads();
  const int t = threadIdx.x % G::T, l = threadIdx.x / G::T;
  // Z_n = E_n + i O_n with E = X_n + conj X_{M-n}, O = (X_n - conj X_{M-n}) W_N^{-n}; a C2R
  // reads only the real parts of X_0 and X_M.
  float2 v[16], u[16];
#pragma unroll
  for (int n1 = 0; n1 < 16; ++n1) {
    const int n = G::T * n1 + t;
    float2 xk = xb[n * G::C + l], xm = cconj(xb[(G::M - n) * G::C + l]);
    if (n == 0) {
      xk.y = 0.f;
      xm.y = 0.f;
    }
    const float2 O = cmul(csub(xk, xm), tw[n]);
    v[n1] = cadd(cadd(xk, xm), make_float2(-O.y, O.x));
  }
  __syncthreads();  // the tile is read; its memory becomes the exchange rows
  line_fft<true, G::T>(v, u, xb + l * G::X, tl, t);
  float2* dst = reinterpret_cast<float2*>(out + (long long)f * G::N3 + (g0 + l) * N);
#pragma unroll
  for (int p = 0; p < 16; ++p) dst[line_k<G::T>(t, p)] = u[p];  // (r[2n], r[2n+1])
}

// Green's-function multiply of one spectral value (the per-mode work of k_green).
struct GreenPlane {
  float s_c, kf, dx, sd2;
  int gm;
};
template <int N>
__device__ __forceinline__ float kl(int i, float kf) { return kf * (float)(i < N / 2 ? i : i - N); }
__device__ __forceinline__ float gk(float k, float dx, int mode) {
  if (mode == 1) return sinf(k * dx) / dx;
  if (mode == 2) return (8.0f * sinf(k * dx) - sinf(2.0f * k * dx)) / (6.0f * dx);
  return k;
}
// -i g_comp(k) G(k) delta_k at mode (x, y, kz) of a plane whose values start at plane; adds the
// mode's weight in the potential energy to w (component 0).
template <int N>
__device__ __forceinline__ float2 green_mode(float2 v, int x, int y, int kz, int comp, const GreenPlane& gp,
                                             const float2* plane, double& w) {
  const float kx = kl<N>(x, gp.kf), ky = kl<N>(y, gp.kf), kzv = gp.kf * (float)kz;
  const float k2 = kx * kx + ky * ky + kzv * kzv;
  if (x == 0 && y == 0 && kz == 0) return make_float2(0.f, 0.f);
  float G = gp.s_c / k2;
  if (gp.sd2 > 0.f) G *= expf(-0.5f * k2 * gp.sd2);
  const float kc = comp == 0 ? kx : (comp == 1 ? ky : kzv);
  const float g = gk(kc, gp.dx, gp.gm) * G;
  if (comp == 0) w += (double)(((kz == 0 || kz == N / 2) ? 1.0f : 2.0f) * G * (v.x * v.x + v.y * v.y));
  float2 o = make_float2(g * v.y, -g * v.x);  // -i g v
  if (kz == 0 || kz == N / 2) {  // (o + conj(o at -k)) / 2: numpy's C2R sees this plane's Hermitian part
    const int px = (-x) & (N - 1), py = (-y) & (N - 1);
    const float2 dp = plane[(long long)px * N + py];
    const float kpc = comp == 0 ? kl<N>(px, gp.kf) : (comp == 1 ? kl<N>(py, gp.kf) : kzv);
    const float h = gk(kpc, gp.dx, gp.gm) * G;
    o = make_float2(0.5f * (o.x + h * dp.y), 0.5f * (o.y + h * dp.x));
  }
  return o;
}

// Plane-pass geometry for mesh N: a line (row or column) of N points shared by T = N/16 threads,
// B = 256/T lines per CTA.
template <int N>
struct PGeo {
  static constexpr int T = N / 16, B = CTA / T, NH = N / 2 + 1;
  static constexpr int RS = N + (T <= 8 ? T : 0);  // row stride in shared memory (bank-conflict free)
  static constexpr long long N2 = (long long)N * N, N3 = N2 * N;
  static_assert(B <= N, "a CTA's rows (columns) lie in one plane");
};

template <bool INV, int N>
__device__ __forceinline__ void load_ptw(float2* tl) {
  constexpr int T = PGeo<N>::T;
  for (int i = threadIdx.x; i < 16 * T; i += CTA) tl[i] = tw_global<INV, N>((i / T) * (i % T));
}

// Pass Y: rows x = B rb + r of one kz plane, T threads per row.  Forward: in = out =
// planes[slot][kz][x][y] (in place: a CTA reads its rows before it writes them).  Inverse with
// GREEN: in = spectrum planes[slot][kz][kx][ky], out = planes[slot][comp][kz][kx][y], the
// multiply applied on load; slot_peak maps a slot to its peak.  Inverse without GREEN: in and
// out [f][kz][.][.].  grid (N/B * nslots * NH * ncomp), block index
// ((slot * NH + kz) * (N/B) + rb) * ncomp + comp (the components of a row block adjacent).
template <int N, bool INV, bool GREEN>
__global__ void __launch_bounds__(CTA, 4) k_fft_rows(const float2* in, float2* out, StepArgs A, const int* slot_peak,
                                                      int ncomp) {
  using G = PGeo<N>;
  constexpr int T = G::T, B = G::B;
  __shared__ float2 tl[16 * T];
  __shared__ __align__(16) float2 buf[B * G::RS];
  load_ptw<INV, N>(tl);
  const int bi = blockIdx.x, comp = bi % ncomp, q = bi / ncomp, rb = q % (N / B), pl = q / (N / B);
  const int slot = pl / G::NH, kz = pl - slot * G::NH;
  GreenPlane gp{};
  int pk = 0;
  if (GREEN) {
    pk = slot_peak[slot];
    if (!A.clocks[pk].has_delta) return;
    const PeakDesc& P = A.peaks[pk];
    gp.s_c = (float)(-1.5 * PM_H_I * PM_H_I / A.clocks[pk].a_grid / (double)G::N3);
    gp.kf = (float)(2.0 * M_PI / P.L);
    gp.dx = (float)P.dx;
    gp.sd2 = P.smooth > 0 ? (float)(P.smooth * P.dx) * (float)(P.smooth * P.dx) : 0.f;
    gp.gm = P.gradient;
  }
  const int t = threadIdx.x % T, r = threadIdx.x / T, x = B * rb + r;
  const float2* plane = in + (long long)pl * G::N2;
  float2 v[16], u[16];
#pragma unroll
  for (int n1 = 0; n1 < 16; ++n1) v[n1] = plane[(long long)x * N + T * n1 + t];
  float2* row = buf + r * G::RS;
  double w = 0.0;
  if (GREEN) {
    if (kz != 0 && kz != N / 2 && (gp.gm == 0 || comp != 1)) {
      // Interior planes (no Hermitian partner, k != 0), with the gradient factor constant along
      // the row (components x and z) or the spectral ky (component y): unrolled, in registers.
      const float kx = kl<N>(x, gp.kf), kzv = gp.kf * (float)kz, a = kx * kx + kzv * kzv;
      const float gc = gk(comp == 0 ? kx : kzv, gp.dx, gp.gm);
#pragma unroll
      for (int n1 = 0; n1 < 16; ++n1) {
        const float ky = kl<N>(T * n1 + t, gp.kf), k2 = a + ky * ky;
        float Gk = gp.s_c / k2;
        if (gp.sd2 > 0.f) Gk *= expf(-0.5f * k2 * gp.sd2);
        const float g = (comp == 1 ? ky : gc) * Gk;
        const float2 d = v[n1];
        if (comp == 0) w += (double)(2.0f * Gk * (d.x * d.x + d.y * d.y));
        v[n1] = make_float2(g * d.y, -g * d.x);  // -i g d
      }
    } else {
      // The general multiply in a rolled loop over this thread's slots of its row in shared
      // memory (one copy of its code keeps the kernel within the instruction cache).
      float2* own = row + t;
#pragma unroll
      for (int n1 = 0; n1 < 16; ++n1) own[T * n1] = v[n1];
#pragma unroll 1
      for (int n1 = 0; n1 < 16; ++n1) own[T * n1] = green_mode<N>(own[T * n1], x, T * n1 + t, kz, comp, gp, plane, w);
#pragma unroll
      for (int n1 = 0; n1 < 16; ++n1) v[n1] = own[T * n1];
    }
    if (comp == 0)
      for (int d = 16; d > 0; d >>= 1) w += __shfl_down_sync(0xffffffffu, w, d);
  }
  __syncthreads();  // table; the rolled Green loop's slots
  line_fft<INV, T>(v, u, row, tl, t);
  float2* dst = out + ((long long)(slot * ncomp + comp) * G::NH + kz) * G::N2 + (long long)x * N;
#pragma unroll
  for (int p = 0; p < 16; ++p) dst[line_k<T>(t, p)] = u[p];
  if (GREEN && comp == 0 && (threadIdx.x & 31) == 0)
    A.wpart[A.peaks[pk].mode_base * (PM_THREADS / 32) + ((long long)kz * (N / B) + rb) * (CTA / 32) + (threadIdx.x >> 5)] = w;
}

// Pass X, in place: columns ky = B cb + j of one kz plane, T threads per column.  Consecutive
// lanes hold consecutive columns, so each warp access covers 32/B rows, B columns (8 B bytes)
// of each.  grid (N/B * nplanes).
template <int N, bool INV>
__global__ void __launch_bounds__(CTA, 4) k_fft_cols(float2* io) {
  using G = PGeo<N>;
  constexpr int T = G::T, B = G::B;
  __shared__ float2 tl[16 * T];
  __shared__ __align__(16) float2 buf[16 * T * B];  // [k1][t][j]
  load_ptw<INV, N>(tl);
  const int cb = blockIdx.x % (N / B), pl = blockIdx.x / (N / B);
  const int j = threadIdx.x % B, t = threadIdx.x / B, ky = B * cb + j;
  float2* plane = io + (long long)pl * G::N2 + ky;
  float2 v[16], u[16];
#pragma unroll
  for (int n1 = 0; n1 < 16; ++n1) v[n1] = plane[(long long)(T * n1 + t) * N];
  __syncthreads();
  dft_reg<INV, 16, 0, 16>(v);
#pragma unroll
  for (int p = 0; p < 16; ++p) {
    const int k1 = brev(p, 4);
    buf[(k1 * T + t) * B + j] = k1 ? cmul(v[p], tl[k1 * T + t]) : v[p];
  }
  __syncthreads();
  if constexpr (T <= 16) {
    // this thread's k1 = t + T s, s < 16 / T: one T-point DFT each
#pragma unroll
    for (int s = 0; s < 16 / T; ++s)
#pragma unroll
      for (int i = 0; i < T; ++i) u[T * s + i] = buf[((t + T * s) * T + i) * B + j];
    dft_groups<INV, T>(u);
  } else {
    static_assert(T == 32, "column pass for N <= 512");
    const int k1 = t >> 1, t0 = t & 1;
#pragma unroll
    for (int i = 0; i < 16; ++i) u[i] = buf[(k1 * 32 + 2 * i + t0) * B + j];
    dft_reg<INV, 16, 0, 16>(u);
#pragma unroll
    for (int p = 0; p < 16; ++p) {
      if (t0) u[p] = cmul(u[p], tl[brev(p, 4) * 32 + 16]);  // W_32^m
      // partner: thread t ^ 1 of the same column, B lanes away
      const float ox = __shfl_xor_sync(0xffffffffu, u[p].x, B), oy = __shfl_xor_sync(0xffffffffu, u[p].y, B);
      u[p] = t0 ? make_float2(ox - u[p].x, oy - u[p].y) : make_float2(u[p].x + ox, u[p].y + oy);
    }
  }
#pragma unroll
  for (int p = 0; p < 16; ++p) plane[(long long)line_k<T>(t, p) * N] = u[p];
}

template <int N>
int r2c_n(const float* delta, float2* spec, int nslots, cudaStream_t s) {
  using Z = ZGeo<N>;
  using G = PGeo<N>;
  const unsigned planes = (unsigned)(nslots * G::NH), blocks = (unsigned)(N / G::B) * planes;
  k_fft_z_r2c<N><<<dim3((unsigned)(Z::N2 / Z::L), nslots), CTA, 0, s>>>(delta, spec);
  k_fft_rows<N, false, false><<<blocks, CTA, 0, s>>>(spec, spec, StepArgs{}, nullptr, 1);
  k_fft_cols<N, false><<<blocks, CTA, 0, s>>>(spec);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : -(int)e;
}

template <int N>
int green_c2r_n(const float2* spec, float2* gwork, float* force, const StepArgs& A, const int* slot_peak, int nslots,
                cudaStream_t s) {
  using Z = ZGeo<N>;
  using G = PGeo<N>;
  const unsigned blocks = (unsigned)(N / G::B) * (unsigned)(nslots * G::NH) * 3u;
  k_fft_rows<N, true, true><<<blocks, CTA, 0, s>>>(spec, gwork, A, slot_peak, 3);
  k_fft_cols<N, true><<<blocks, CTA, 0, s>>>(gwork);
  k_fft_z_c2r<N><<<dim3((unsigned)(Z::N2 / Z::L), 3 * nslots), CTA, 0, s>>>(gwork, force);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : -(int)e;
}

template <int N>
int c2r_n(const float2* spec, float2* gwork, float* out, int nfields, cudaStream_t s) {
  using Z = ZGeo<N>;
  using G = PGeo<N>;
  const unsigned blocks = (unsigned)(N / G::B) * (unsigned)(nfields * G::NH);
  k_fft_rows<N, true, false><<<blocks, CTA, 0, s>>>(spec, gwork, StepArgs{}, nullptr, 1);
  k_fft_cols<N, true><<<blocks, CTA, 0, s>>>(gwork);
  k_fft_z_c2r<N><<<dim3((unsigned)(Z::N2 / Z::L), nfields), CTA, 0, s>>>(gwork, out);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : -(int)e;
}

}  // namespace

bool fft_native_size(int N) { return N == 64 || N == 128 || N == 256 || N == 512; }

// Per-device set-up: the twiddle table.  Call with the device current.
int fft_native_init() {
  float2 h[TWN];
  for (int k = 0; k < TWN; ++k) {
    const double a = -2.0 * M_PI * (double)k / (double)TWN;
    h[k] = make_float2((float)cos(a), (float)sin(a));
  }
  const cudaError_t e = cudaMemcpyToSymbol(g_tw, h, sizeof(h));
  return e == cudaSuccess ? 0 : -(int)e;
}

// delta fields [slot][x][y][z] -> spectra [slot][kz][kx][ky]
int fft_native_r2c(int N, const float* delta, float2* spec, int nslots, cudaStream_t s) {
  if (nslots <= 0) return 0;
  switch (N) {
    case 64: return r2c_n<64>(delta, spec, nslots, s);
    case 128: return r2c_n<128>(delta, spec, nslots, s);
    case 256: return r2c_n<256>(delta, spec, nslots, s);
    case 512: return r2c_n<512>(delta, spec, nslots, s);
    default: return -2000;
  }
}

// spectra [slot][kz][kx][ky] -> 3 force grids per slot [slot][comp][x][y][z] through the
// Green multiply; gwork holds [slot][comp][kz][x][y].
int fft_native_green_c2r(int N, const float2* spec, float2* gwork, float* force, const StepArgs& A,
                         const int* slot_peak, int nslots, cudaStream_t s) {
  if (nslots <= 0) return 0;
  switch (N) {
    case 64: return green_c2r_n<64>(spec, gwork, force, A, slot_peak, nslots, s);
    case 128: return green_c2r_n<128>(spec, gwork, force, A, slot_peak, nslots, s);
    case 256: return green_c2r_n<256>(spec, gwork, force, A, slot_peak, nslots, s);
    case 512: return green_c2r_n<512>(spec, gwork, force, A, slot_peak, nslots, s);
    default: return -2000;
  }
}

// Plain unnormalised inverse: spectra [f][kz][kx][ky] -> fields [f][x][y][z]; gwork as spec.
int fft_native_c2r(int N, const float2* spec, float2* gwork, float* out, int nfields, cudaStream_t s) {
  if (nfields <= 0) return 0;
  switch (N) {
    case 64: return c2r_n<64>(spec, gwork, out, nfields, s);
    case 128: return c2r_n<128>(spec, gwork, out, nfields, s);
    case 256: return c2r_n<256>(spec, gwork, out, nfields, s);
    case 512: return c2r_n<512>(spec, gwork, out, nfields, s);
    default: return -2000;
  }
}

namespace {
// Per-device set-up of the twiddle table, once per device; the lock keeps two host threads that
// make their first call on one device at the same time from racing on it.
std::mutex g_init_mu;
int ensure_native_init() {
  static int done[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return -(int)e;
  if (dev < 0 || dev >= 64) return -2004;
  std::lock_guard<std::mutex> lock(g_init_mu);
  if (!done[dev]) {
    if (int r = fft_native_init()) return r;
    done[dev] = 1;
  }
  return 0;
}
}  // namespace

extern "C" int pm_rfft3_native(int n, const float* x, void* spec, int nfields, void* stream) {
  if (!fft_native_size(n)) return -2000;
  if (!x || !spec) return -2001;
  if (nfields < 0) return -2003;
  if (((uintptr_t)x | (uintptr_t)spec) & 15) return -2001;  // 16-byte copies
  if (int r = ensure_native_init()) return r;
  return fft_native_r2c(n, x, (float2*)spec, nfields, (cudaStream_t)stream);
}

extern "C" int pm_irfft3_native(int n, const void* spec, void* work, float* x, int nfields, void* stream) {
  if (!fft_native_size(n)) return -2000;
  if (!spec || !work || !x) return -2001;
  if (nfields < 0) return -2004;
  if (((uintptr_t)x | (uintptr_t)spec | (uintptr_t)work) & 15) return -2001;
  if (int r = ensure_native_init()) return r;
  return fft_native_c2r(n, (const float2*)spec, (float2*)work, x, nfields, (cudaStream_t)stream);
}

extern "C" int pm_rfft3_256(const float* x, void* spec, int nfields, void* stream) {
  return pm_rfft3_native(256, x, spec, nfields, stream);
}

extern "C" int pm_irfft3_256(const void* spec, void* work, float* x, int nfields, void* stream) {
  return pm_irfft3_native(256, spec, work, x, nfields, stream);
}
