// Step kernels: push (CIC interp + kicks + drift), clock advance, bucket starts,
// deterministic tiled CIC deposit, Green's function + gradient, and particle I/O.
#include "pm_kernels.cuh"

namespace {

constexpr double kTwoPi = 6.283185307179586476925286766559;

__device__ __forceinline__ u32 lanemask_le() {
  u32 m;
  asm("mov.u32 %0, %%lanemask_le;" : "=r"(m));
  return m;
}

__device__ __forceinline__ u64 shfl_up_u64(u64 v, int d) {
  const u32 lo = __shfl_up_sync(0xffffffffu, (u32)v, d);
  const u32 hi = __shfl_up_sync(0xffffffffu, (u32)(v >> 32), d);
  return ((u64)hi << 32) | lo;
}

// Locate the peak and tile of this CTA (uniform across the block).
struct TileRef {
  int pk;
  long long t;
};

__device__ __forceinline__ TileRef find_tile(const StepArgs& A) {
  __shared__ int s_pk;
  if (threadIdx.x == 0) s_pk = pm_find(A.tile_base, A.npeaks, (long long)blockIdx.x);
  __syncthreads();
  TileRef r;
  r.pk = s_pk;
  r.t = (long long)blockIdx.x - A.tile_base[r.pk];
  return r;
}

// ------------------------------------------------------------------------------------------
// Push: CIC gather of the three force grids (pm3d.py:91-99) fused with the pending closing
// kick of the previous step, the opening kick and the drift of this one (pm3d.py:122-127).
// One CTA per tile: the (T+1)^3 node patch of all three grids is staged in shared memory,
// then every particle whose CIC cell lies in the tile reads its 8 corners from there.
// Output is written in sorted order into the other state buffer, with the new cell key.
__global__ void __launch_bounds__(PM_THREADS) k_push(StepArgs A) {
  extern __shared__ float s_f[];
  __shared__ float s_coef[5];
  const TileRef tr = find_tile(A);
  const PeakClock C = A.clocks[tr.pk];
  if (C.state != PS_RUN && C.state != PS_FINALIZE) return;
  const PeakDesc& P = A.peaks[tr.pk];
  const int N = P.N, T = P.T, T1 = T + 1, T13 = T1 * T1 * T1;
  const u32 tc = (u32)tr.t;
  const u32* bs = A.bstart + P.bucket_off;
  const long long b = bs[tc * 8], e = bs[tc * 8 + 8];
  if (b == e) return;
  const int tx = pm_compact3(tc >> 2), ty = pm_compact3(tc >> 1), tz = pm_compact3(tc);
  const long long N3 = (long long)N * N * N;
  // Stage the force patch, one row of T+1 nodes per warp iteration.
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int row = warp; row < 3 * T1 * T1; row += PM_THREADS / 32) {
    const int comp = row / (T1 * T1);
    const int rem = row - comp * T1 * T1;
    const int lx = rem / T1, ly = rem - (rem / T1) * T1;
    const int gx = (tx * T + lx) & (N - 1), gy = (ty * T + ly) & (N - 1);
    const float* src = P.force + comp * N3 + ((long long)gx * N + gy) * N;
    for (int lz = lane; lz < T1; lz += 32) s_f[comp * T13 + (lx * T1 + ly) * T1 + lz] = src[(tz * T + lz) & (N - 1)];
  }
  if (threadIdx.x == 0) {
    const double a = C.a, da = C.da;
    const bool run = C.state == PS_RUN;
    const double kB = run ? 0.5 * da / (a * pm_hubble(a)) : 0.0;
    const double amid = a + 0.5 * da;
    const double D = run ? da / (amid * amid * amid * pm_hubble(amid)) / P.dx : 0.0;
    s_coef[0] = (float)C.kpend;
    s_coef[1] = (float)kB;
    s_coef[2] = (float)D;
    s_coef[3] = (float)(C.a_grid / a);
  }
  __syncthreads();
  const float kA = s_coef[0], kB = s_coef[1], D = s_coef[2], gscale = s_coef[3];
  const bool run = C.state == PS_RUN;
  const int buf = C.buf;
  const int4* __restrict__ pin = A.pos[buf];
  const float4* __restrict__ min_ = A.mom[buf];
  int4* __restrict__ pout = A.pos[buf ^ 1];
  float4* __restrict__ mout = A.mom[buf ^ 1];
  const int l2 = 2 * P.log2N;
  bool bad = false;
  for (long long j = b + threadIdx.x; j < e; j += PM_THREADS) {
    const u32 q = A.perm[j];
    const int4 ps = pin[q];
    const float4 m = min_[q];
    int ix = ps.x >> l2, iy = (ps.x >> P.log2N) & (N - 1), iz = ps.x & (N - 1);
    float f[3] = {__int_as_float(ps.y), __int_as_float(ps.z), __int_as_float(ps.w)};
    const int lx = ix - tx * T, ly = iy - ty * T, lz = iz - tz * T;
    if ((unsigned)lx >= (unsigned)T || (unsigned)ly >= (unsigned)T || (unsigned)lz >= (unsigned)T) {
      bad = true;  // state and sort disagree: flag it, never index outside the patch
      continue;
    }
    const float wx[2] = {1.0f - f[0], f[0]}, wy[2] = {1.0f - f[1], f[1]}, wz[2] = {1.0f - f[2], f[2]};
    float acc[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int cx = c >> 2, cy = (c >> 1) & 1, cz = c & 1;
      const float w = wx[cx] * wy[cy] * wz[cz];
      const int o = ((lx + cx) * T1 + ly + cy) * T1 + lz + cz;
      acc[0] += w * s_f[o];
      acc[1] += w * s_f[T13 + o];
      acc[2] += w * s_f[2 * T13 + o];
    }
    float p[3] = {m.x, m.y, m.z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float g = acc[d] * gscale;
      p[d] += kA * g;
      if (run) p[d] += kB * g;
    }
    bad |= !(isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]));
    int ii[3] = {ix, iy, iz};
    if (run) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        float fn = f[d] + D * p[d];
        float cfl = floorf(fn);
        fn -= cfl;
        if (fn >= 1.0f) {
          fn -= 1.0f;
          cfl += 1.0f;
        }
        f[d] = fn;
        ii[d] = (ii[d] + (int)cfl) & (N - 1);
      }
    }
    const int cell = (ii[0] << l2) | (ii[1] << P.log2N) | ii[2];
    pout[j] = make_int4(cell, __float_as_int(f[0]), __float_as_int(f[1]), __float_as_int(f[2]));
    mout[j] = make_float4(p[0], p[1], p[2], m.w);
    A.keys_push[j] = ((u64)tr.pk << 32) | pm_cell_key(P, ii[0], ii[1], ii[2]);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&A.stats[tr.pk].status, 1u);
}

// Clock advance (one thread per peak): applies the step that the push kernel just made,
// selects the next step size and sets which peaks re-deposit this step.
__global__ void k_advance(StepArgs A) {
  for (int pk = threadIdx.x; pk < A.npeaks; pk += blockDim.x) {
    PeakClock c = A.clocks[pk];
    int dep = 0;
    // Collapse detection on the deposit of the current positions (made by the previous step).
    if (c.has_delta && c.delta_collapse > 0 && c.a_collapse < 0 && c.state != PS_PRIME) {
      const PeakDesc& P = A.peaks[pk];
      const double dmax = (double)A.stats[pk].max_fix / (double)PM_FIX_ONE / P.n_mean - 1.0;
      if (dmax >= c.delta_collapse) c.a_collapse = c.a;
    }
    switch (c.state) {
      case PS_PRIME:
        dep = 1;
        c.kpend = 0.0;
        c.a_grid = c.a;
        c.has_delta = 1;
        c.state = c.mode == SCHED_EXPLICIT ? PS_HOLD : PS_RUN;
        break;
      case PS_RUN: {
        const double an = c.a + c.da;
        c.kpend = 0.5 * c.da / (an * pm_hubble(an));
        c.a = an;
        c.a_grid = an;
        c.nsteps += 1;
        c.buf ^= 1;
        dep = 1;
        if (c.mode == SCHED_RATIO) {
          if (c.nsteps >= c.max_steps) c.state = PS_FINALIZE;
          else c.da = c.a * c.param;
        } else if (c.mode == SCHED_FRAC) {
          if (c.a >= c.a_end) c.state = PS_FINALIZE;
          else c.da = fmin(c.param * c.a, c.a_end - c.a);
        } else {
          c.state = PS_HOLD;
        }
        break;
      }
      case PS_FINALIZE:
        c.kpend = 0.0;
        c.buf ^= 1;
        dep = 1;
        c.state = PS_IDLE;
        break;
      default:
        break;
    }
    c.dep = dep;
    A.clocks[pk] = c;
    A.sortseg[pk].active = dep;
    if (dep) {
      A.stats[pk].max_fix = 0;
      A.stats[pk].mass_defect = 0;
    }
  }
}

// Bucket starts from the sorted keys: bstart[b] = first sorted index whose bucket >= b.
__global__ void k_bucket_starts(StepArgs A, long long ntot) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ntot) return;
  const int pk = pm_find(A.p_base, A.npeaks, j);
  if (!A.clocks[pk].dep) return;
  const PeakDesc& P = A.peaks[pk];
  u32* bs = A.bstart + P.bucket_off;
  const int b = (int)((u32)A.keys_sorted[j] >> P.local_bits);
  const int bprev = j == P.p_off ? -1 : (int)((u32)A.keys_sorted[j - 1] >> P.local_bits);
  for (int bb = bprev + 1; bb <= b; ++bb) bs[bb] = (u32)j;
  if (j == P.p_off + P.n - 1)
    for (int bb = b + 1; bb <= P.nb; ++bb) bs[bb] = (u32)(P.p_off + P.n);
}

// ------------------------------------------------------------------------------------------
// Deterministic CIC deposit (pm3d.py:81-89, 103-104).  One CTA owns the T^3 nodes of one
// tile and accumulates, in 64-bit fixed point in shared memory, every particle contribution
// that lands on them: the tile's own particles (corners outside the tile are left to their
// owners) and, from the 7 lower neighbour tiles, only the boundary-layer buckets whose
// corners reach into this tile.  Consecutive particles in the same cell are first combined
// by a warp-shuffle segmented scan, so dense cells cost one shared-memory update per run.
// Every node is written exactly once as FP32 delta = S/n_mean - 1, with no global atomics.
__global__ void __launch_bounds__(PM_THREADS) k_deposit(StepArgs A, double* rho64) {
  extern __shared__ u64 s_acc[];
  __shared__ long long s_rb[16], s_re[16];
  __shared__ int s_ro[16];
  __shared__ int s_nr;
  __shared__ long long s_red[PM_THREADS / 32];
  __shared__ long long s_max[PM_THREADS / 32];
  const TileRef tr = find_tile(A);
  if (!A.clocks[tr.pk].dep) return;
  const PeakDesc& P = A.peaks[tr.pk];
  const int N = P.N, T = P.T, T3 = T * T * T, NT = N >> P.log2T;
  const u32 tc = (u32)tr.t;
  const int tx = pm_compact3(tc >> 2), ty = pm_compact3(tc >> 1), tz = pm_compact3(tc);
  for (int i = threadIdx.x; i < T3; i += PM_THREADS) s_acc[i] = 0ull;
  if (threadIdx.x == 0) {
    const u32* bs = A.bstart + P.bucket_off;
    int nr = 0;
    s_rb[0] = bs[tc * 8];
    s_re[0] = bs[tc * 8 + 8];
    s_ro[0] = 0;
    nr = s_re[0] > s_rb[0] ? 1 : 0;
    for (int o = 1; o < 8; ++o) {
      const u32 nx = (tx - (o & 1)) & (NT - 1), ny = (ty - ((o >> 1) & 1)) & (NT - 1),
                nz = (tz - ((o >> 2) & 1)) & (NT - 1);
      const u32 tn = pm_morton3(nx, ny, nz);
      for (int m = 0; m < 8; ++m) {
        if ((m & o) != o) continue;
        const long long rb = bs[tn * 8 + m], re = bs[tn * 8 + m + 1];
        if (re <= rb) continue;
        if (nr > 0 && s_ro[nr - 1] == o && s_re[nr - 1] == rb) {
          s_re[nr - 1] = re;
        } else {
          s_rb[nr] = rb;
          s_re[nr] = re;
          s_ro[nr] = o;
          ++nr;
        }
      }
    }
    s_nr = nr;
  }
  __syncthreads();
  const int4* __restrict__ pos = A.pos[A.clocks[tr.pk].buf];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int l2 = 2 * P.log2N;
  const u32 le = lanemask_le();
  const double fix_one = (double)PM_FIX_ONE;
  for (int r = 0; r < s_nr; ++r) {
    const long long rb = s_rb[r], re = s_re[r];
    const int o = s_ro[r];
    for (long long j0 = rb + warp * 32; j0 < re; j0 += PM_THREADS) {
      const long long j = j0 + lane;
      const bool valid = j < re;
      const int4 ps = valid ? pos[A.perm[j]] : make_int4(-1, 0, 0, 0);
      const int ix = ps.x >> l2, iy = (ps.x >> P.log2N) & (N - 1), iz = ps.x & (N - 1);
      const int lx = (o & 1) ? -1 : ix - tx * T;
      const int ly = (o & 2) ? -1 : iy - ty * T;
      const int lz = (o & 4) ? -1 : iz - tz * T;
      const double fx = __int_as_float(ps.y), fy = __int_as_float(ps.z), fz = __int_as_float(ps.w);
      const double wx[2] = {1.0 - fx, fx}, wy[2] = {1.0 - fy, fy}, wz[2] = {1.0 - fz, fz};
      u64 W[8];
      u64 s7 = 0;
#pragma unroll
      for (int c = 0; c < 7; ++c) {
        W[c] = valid ? (u64)__double2ll_rn(wx[c >> 2] * wy[(c >> 1) & 1] * wz[c & 1] * fix_one) : 0ull;
        s7 += W[c];
      }
      // The eighth corner takes the remainder so each particle deposits exactly 2^40.
      W[7] = valid ? PM_FIX_ONE - s7 : 0ull;
      const int prev = __shfl_up_sync(0xffffffffu, ps.x, 1);
      const bool head = !(valid && lane > 0 && prev == ps.x);
      const u32 heads = __ballot_sync(0xffffffffu, head);
      bool tail = true;
      if (heads != 0xffffffffu) {
        const int sstart = 31 - __clz(heads & le);
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            const u64 v = shfl_up_u64(W[c], d);
            if (lane - d >= sstart) W[c] += v;
          }
        }
        tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
      }
      if (valid && tail) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const int cx = lx + (c >> 2), cy = ly + ((c >> 1) & 1), cz = lz + (c & 1);
          if ((unsigned)cx < (unsigned)T && (unsigned)cy < (unsigned)T && (unsigned)cz < (unsigned)T)
            atomicAdd(&s_acc[(cx * T + cy) * T + cz], W[c]);
        }
      }
    }
  }
  __syncthreads();
  long long dsum = 0, smax = 0;
  const long long base = ((long long)tx * T * N + (long long)ty * T) * N + tz * T;
  for (int i = threadIdx.x; i < T3; i += PM_THREADS) {
    const int lz = i & (T - 1), ly = (i >> P.log2T) & (T - 1), lx = i >> (2 * P.log2T);
    const long long S = (long long)s_acc[i];
    const long long Dv = S - P.n_mean_fix;
    const long long g = base + ((long long)lx * N + ly) * N + lz;
    P.delta[g] = (float)((double)Dv * P.inv_fix_nmean);
    if (rho64) rho64[g] = (double)S * (1.0 / (double)PM_FIX_ONE);
    dsum += Dv;
    smax = S > smax ? S : smax;
  }
  for (int d = 16; d > 0; d >>= 1) {
    dsum += __shfl_xor_sync(0xffffffffu, dsum, d);
    const long long om = __shfl_xor_sync(0xffffffffu, smax, d);
    smax = om > smax ? om : smax;
  }
  if (lane == 0) {
    s_red[warp] = dsum;
    s_max[warp] = smax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long ts = 0, tm = 0;
    for (int w = 0; w < PM_THREADS / 32; ++w) {
      ts += s_red[w];
      tm = s_max[w] > tm ? s_max[w] : tm;
    }
    atomicAdd((unsigned long long*)&A.stats[tr.pk].mass_defect, (unsigned long long)ts);
    atomicMax(&A.stats[tr.pk].max_fix, (u64)tm);
  }
}

// ------------------------------------------------------------------------------------------
// Green's function and gradient in k-space (pm3d.py:105-112): for every mode
//   Phi_k = -(3/2) H_i^2 delta_k / (a k^2) [* exp(-k^2 (smooth dx)^2 / 2)],  Phi_0 = 0,
//   G_i   = -i k_i Phi_k / N^3    (the 1/N^3 of numpy's inverse transform),
// written as three spectra for one batched C2R.  numpy's irfftn keeps the Nyquist
// wavenumbers (-pi/dx) and, in the kz = 0 and kz = N/2 planes, uses only the Hermitian part
// of its input (it takes the real part after the two complex inverse transforms).  Those two
// planes are therefore written as (G(k) + conj G(-k))/2, which any correct C2R turns into
// exactly numpy's field.
__device__ __forceinline__ double kline(int i, int N, double kf) { return kf * (double)(i < N / 2 ? i : i - N); }

__device__ __forceinline__ double grad_k(double k, double dx, int mode) {
  if (mode == 1) return sin(k * dx) / dx;
  if (mode == 2) return (8.0 * sin(k * dx) - sin(2.0 * k * dx)) / (6.0 * dx);
  return k;
}

__global__ void __launch_bounds__(PM_THREADS) k_green(StepArgs A) {
  __shared__ int s_pk;
  if (threadIdx.x == 0) s_pk = pm_find(A.mode_base, A.npeaks, (long long)blockIdx.x);
  __syncthreads();
  const int pk = s_pk;
  const PeakClock& C = A.clocks[pk];
  if (!C.has_delta) return;
  const PeakDesc& P = A.peaks[pk];
  const long long m = ((long long)blockIdx.x - A.mode_base[pk]) * PM_THREADS + threadIdx.x;
  if (m >= P.nmodes) return;
  const int N = P.N, Nh = N / 2 + 1;
  const int kz = (int)(m % Nh);
  const long long rest = m / Nh;
  const int iy = (int)(rest & (N - 1)), ix = (int)(rest >> P.log2N);
  const double kf = kTwoPi / P.L;
  const double kx = kline(ix, N, kf), ky = kline(iy, N, kf), kzv = kf * kz;
  const double k2 = kx * kx + ky * ky + kzv * kzv;
  float2* out = P.gspec;
  if (m == 0) {
    out[m] = out[P.nmodes + m] = out[2 * P.nmodes + m] = make_float2(0.f, 0.f);
    return;
  }
  double G = -1.5 * PM_H_I * PM_H_I / C.a_grid / k2;
  if (P.smooth > 0) G *= exp(-0.5 * k2 * (P.smooth * P.dx) * (P.smooth * P.dx));
  G /= (double)N * (double)N * (double)N;
  const float2 d = P.spec[m];
  const double kc[3] = {grad_k(kx, P.dx, P.gradient), grad_k(ky, P.dx, P.gradient), grad_k(kzv, P.dx, P.gradient)};
  // -i k G d = (k G d.y, -k G d.x)
  double vr[3], vi[3];
  for (int c = 0; c < 3; ++c) {
    vr[c] = kc[c] * G * (double)d.y;
    vi[c] = -kc[c] * G * (double)d.x;
  }
  if (kz == 0 || kz == N / 2) {
    const int px = (-ix) & (N - 1), py = (-iy) & (N - 1);
    const long long mp = ((long long)px * N + py) * Nh + kz;
    const float2 dp = P.spec[mp];
    const double kpx = kline(px, N, kf), kpy = kline(py, N, kf);
    const double kpc[3] = {grad_k(kpx, P.dx, P.gradient), grad_k(kpy, P.dx, P.gradient), kc[2]};
    for (int c = 0; c < 3; ++c) {
      const double pr = kpc[c] * G * (double)dp.y, pi = -kpc[c] * G * (double)dp.x;
      vr[c] = 0.5 * (vr[c] + pr);
      vi[c] = 0.5 * (vi[c] - pi);
    }
  }
  for (int c = 0; c < 3; ++c) out[c * P.nmodes + m] = make_float2((float)vr[c], (float)vi[c]);
}

// ------------------------------------------------------------------------------------------
__global__ void k_reset_peak(StepArgs A, int pk, double a0, int mode, double param, double a_end, int max_steps) {
  PeakClock c = A.clocks[pk];
  c.a = a0;
  c.a_grid = a0;
  c.kpend = 0.0;
  c.mode = mode;
  c.param = param;
  c.a_end = a_end;
  c.max_steps = max_steps;
  c.nsteps = 0;
  c.state = PS_PRIME;
  c.has_delta = 0;
  c.dep = 0;
  c.a_collapse = -1.0;
  if (mode == SCHED_RATIO) c.da = a0 * param;
  else if (mode == SCHED_FRAC) c.da = fmin(param * a0, a_end - a0);
  else c.da = 0.0;
  A.clocks[pk] = c;
  A.stats[pk].status = 0;
}

// Particles (n,3) float64 in lattice order -> split state + cell keys (pm3d.py:76-79 convention).
__global__ void k_set_particles(StepArgs A, int pk, PeakDesc P, const double* __restrict__ x,
                                const double* __restrict__ p) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const int buf = A.clocks[pk].buf;
  int ii[3];
  float ff[3];
  for (int d = 0; d < 3; ++d) {
    const double g = x[3 * i + d] / P.dx - 0.5;
    const double fl = floor(g);
    long long c = (long long)fl;
    float f = (float)(g - fl);
    if (f >= 1.0f) {
      f = 0.0f;
      c += 1;
    }
    ii[d] = (int)(((c % P.N) + P.N) % P.N);
    ff[d] = f;
  }
  const int cell = (ii[0] << (2 * P.log2N)) | (ii[1] << P.log2N) | ii[2];
  const long long g = P.p_off + i;
  A.pos[buf][g] = make_int4(cell, __float_as_int(ff[0]), __float_as_int(ff[1]), __float_as_int(ff[2]));
  A.mom[buf][g] = make_float4((float)p[3 * i], (float)p[3 * i + 1], (float)p[3 * i + 2], __int_as_float((int)i));
  A.keys_push[g] = ((u64)pk << 32) | pm_cell_key(P, ii[0], ii[1], ii[2]);
}

// Current state -> float64 x, p (lattice order).  p includes the pending closing kick; acc
// (optional) receives -grad Phi at the particles evaluated for expansion factor a_acc.
__global__ void k_get_particles(StepArgs A, int pk, PeakDesc P, double* __restrict__ x, double* __restrict__ p,
                                double* __restrict__ acc, double a_acc) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const PeakClock C = A.clocks[pk];
  const int4 ps = A.pos[C.buf][P.p_off + i];
  const float4 m = A.mom[C.buf][P.p_off + i];
  const int N = P.N;
  const int ii[3] = {ps.x >> (2 * P.log2N), (ps.x >> P.log2N) & (N - 1), ps.x & (N - 1)};
  const float f[3] = {__int_as_float(ps.y), __int_as_float(ps.z), __int_as_float(ps.w)};
  const long long id = (long long)__float_as_int(m.w);
  double g[3] = {0.0, 0.0, 0.0};
  const bool need_g = C.has_delta && ((p && C.kpend != 0.0) || acc);
  if (need_g) {
    const long long N3 = (long long)N * N * N;
    for (int c = 0; c < 8; ++c) {
      const int cx = c >> 2, cy = (c >> 1) & 1, cz = c & 1;
      const float w = (cx ? f[0] : 1.0f - f[0]) * (cy ? f[1] : 1.0f - f[1]) * (cz ? f[2] : 1.0f - f[2]);
      const long long o = ((long long)((ii[0] + cx) & (N - 1)) * N + ((ii[1] + cy) & (N - 1))) * N + ((ii[2] + cz) & (N - 1));
      g[0] += w * P.force[o];
      g[1] += w * P.force[N3 + o];
      g[2] += w * P.force[2 * N3 + o];
    }
  }
  const double mv[3] = {m.x, m.y, m.z};
  for (int d = 0; d < 3; ++d) {
    if (x) {
      double X = ((double)ii[d] + (double)f[d] + 0.5) * P.dx;
      if (X >= P.L) X -= P.L;
      x[3 * id + d] = X;
    }
    if (p) p[3 * id + d] = mv[d] + C.kpend * (C.a_grid / C.a) * g[d];
    if (acc) acc[3 * id + d] = g[d] * (C.a_grid / a_acc);
  }
}

// Reference-exact float64 CIC gather of an arbitrary field (pm3d.py:91-99).
__global__ void k_interp64(const double* __restrict__ F, const double* __restrict__ X, long long n, int N, double dx,
                           double* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  long long i0[3], i1[3];
  double f[3];
  for (int d = 0; d < 3; ++d) {
    const double g = X[3 * i + d] / dx - 0.5;
    const double fl = floor(g);
    const long long c = (long long)fl;
    f[d] = g - fl;
    i0[d] = ((c % N) + N) % N;
    i1[d] = (((c + 1) % N) + N) % N;
  }
  double s = 0.0;
  for (int c = 0; c < 8; ++c) {
    const int cx = c >> 2, cy = (c >> 1) & 1, cz = c & 1;
    const long long o = ((cx ? i1[0] : i0[0]) * N + (cy ? i1[1] : i0[1])) * N + (cz ? i1[2] : i0[2]);
    s += F[o] * ((cx ? f[0] : 1.0 - f[0]) * (cy ? f[1] : 1.0 - f[1]) * (cz ? f[2] : 1.0 - f[2]));
  }
  out[i] = s;
}

}  // namespace

size_t pm_deposit_smem(int Tmax) { return sizeof(u64) * (size_t)Tmax * Tmax * Tmax; }
size_t pm_push_smem(int Tmax) { return sizeof(float) * 3 * (size_t)(Tmax + 1) * (Tmax + 1) * (Tmax + 1); }

int pm_kernels_init() {
  cudaError_t e = cudaFuncSetAttribute(k_push, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_deposit, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  return e == cudaSuccess ? 0 : -(int)e;
}

void launch_push(const StepArgs& A, long long ntiles, size_t smem, cudaStream_t s) {
  k_push<<<(unsigned)ntiles, PM_THREADS, smem, s>>>(A);
}
void launch_advance(const StepArgs& A, cudaStream_t s) { k_advance<<<1, 256, 0, s>>>(A); }
void launch_bucket_starts(const StepArgs& A, long long ntot, cudaStream_t s) {
  k_bucket_starts<<<(unsigned)((ntot + PM_THREADS - 1) / PM_THREADS), PM_THREADS, 0, s>>>(A, ntot);
}
void launch_deposit(const StepArgs& A, long long ntiles, size_t smem, double* rho64, cudaStream_t s) {
  k_deposit<<<(unsigned)ntiles, PM_THREADS, smem, s>>>(A, rho64);
}
void launch_green(const StepArgs& A, long long nblocks, cudaStream_t s) {
  k_green<<<(unsigned)nblocks, PM_THREADS, 0, s>>>(A);
}
void launch_reset_peak(const StepArgs& A, int pk, double a0, int mode, double param, double a_end, int max_steps,
                       cudaStream_t s) {
  k_reset_peak<<<1, 1, 0, s>>>(A, pk, a0, mode, param, a_end, max_steps);
}
void launch_set_particles(const StepArgs& A, int pk, const PeakDesc& P, const double* x, const double* p,
                          cudaStream_t s) {
  k_set_particles<<<(unsigned)((P.n + PM_THREADS - 1) / PM_THREADS), PM_THREADS, 0, s>>>(A, pk, P, x, p);
}
void launch_get_particles(const StepArgs& A, int pk, const PeakDesc& P, double* x, double* p, double* acc,
                          double a_acc, cudaStream_t s) {
  k_get_particles<<<(unsigned)((P.n + PM_THREADS - 1) / PM_THREADS), PM_THREADS, 0, s>>>(A, pk, P, x, p, acc, a_acc);
}
void launch_interp64(const double* F, const double* X, long long n, int N, double dx, double* out, cudaStream_t s) {
  k_interp64<<<(unsigned)((n + PM_THREADS - 1) / PM_THREADS), PM_THREADS, 0, s>>>(F, X, n, N, dx, out);
}
