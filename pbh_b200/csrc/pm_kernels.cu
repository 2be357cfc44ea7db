// Step kernels of the pm3d engine: push (CIC gather + kicks + drift, re-binning class),
// clock advance, regrouping (re-binning scatter, or radix-sort permutation), halo-exchange CIC
// deposit with its face fix-up, Green's function + gradient, and particle I/O.
#include <algorithm>
#include <type_traits>

#include "pm_kernels.cuh"

// Sweeps of particle positions a deposit thread keeps in flight (loads issued ahead of use).
#ifndef PM_DEP_DEPTH
#define PM_DEP_DEPTH 1
#endif

namespace {

constexpr double kTwoPi = 6.283185307179586476925286766559;

// Shared-memory layout of a (TS+1)^3 node patch: node (lx, ly, lz) at lx*PS + ly*RS + lz.  The
// strides are padded so that the 8 corners read (push) or added to (deposit) by a warp of 32
// Morton-consecutive cells fall in 32 distinct banks, and so that rows start on 16 bytes
// (asynchronous 16-byte copies).
__host__ __device__ constexpr int patch_rs(int TS) { return TS == 4 ? 8 : TS == 8 ? 12 : 20; }
__host__ __device__ constexpr int patch_ps(int TS) { return TS == 4 ? 44 : TS == 8 ? 112 : 368; }
__host__ __device__ constexpr int patch_size(int TS) { return (TS + 1) * patch_ps(TS); }

__device__ __forceinline__ void cp_async16(unsigned dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(unsigned dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ u32 lanemask_lt() {
  u32 m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}


// Super-tile start arrays without indexing the kernel-parameter array dynamically (which would
// copy the parameter struct to local memory).
__device__ __forceinline__ u32* sst(const StepArgs& A, int b) { return b ? A.sstart[1] : A.sstart[0]; }

// Locate the peak and the peak-local index of this CTA (uniform across the block).
struct TileRef {
  int pk;
  long long t;
};

__device__ __forceinline__ TileRef find_tile(const long long* base, int npeaks) {
  __shared__ int s_pk;
  if (threadIdx.x == 0) s_pk = pm_find(base, npeaks, (long long)blockIdx.x);
  __syncthreads();
  TileRef r;
  r.pk = s_pk;
  r.t = (long long)blockIdx.x - base[r.pk];
  return r;
}

// Re-binning classes: per axis, the offset u = (destination - source) mod NS of the super-tile a
// particle moved to is one of 0, +1, +2, -1, -2 (NS - 1, NS - 2), or any offset when NS <= 5.
__device__ __forceinline__ int bin_digit(int u, int NS) {
  if (NS <= 5 || u <= 2) return u;
  if (u >= NS - 2) return 2 + (NS - u);
  return -1;
}
__device__ __forceinline__ int bin_offset(int d, int NS) { return (NS <= 5 || d <= 2) ? d : NS - (d - 2); }

// Re-binning class of a particle of super-tile (sx, sy, sz) whose cell is now `cell`: class 0 is
// "stayed", BIN_FAR "moved more than two super-tiles" (its destination super-tile in *far_st).
__device__ __forceinline__ int bin_class(int cell, int sx, int sy, int sz, const PeakDesc& P, u32* far_st) {
  const int l2 = P.log2N, N = P.N, NS = P.NS;
  const int tx = (cell >> (2 * l2)) >> P.log2TS, ty = ((cell >> l2) & (N - 1)) >> P.log2TS,
            tz = (cell & (N - 1)) >> P.log2TS;
  const int dxc = bin_digit((tx - sx) & (NS - 1), NS), dyc = bin_digit((ty - sy) & (NS - 1), NS),
            dzc = bin_digit((tz - sz) & (NS - 1), NS);
  if (dxc >= 0 && dyc >= 0 && dzc >= 0) return (dxc * P.W + dyc) * P.W + dzc;
  *far_st = pm_morton3(tx, ty, tz);
  return BIN_FAR;
}

// ------------------------------------------------------------------------------------------
// Push: CIC gather of the three force grids (pm3d.py:91-99) fused with the pending closing
// kick of the previous step, the opening kick and the drift of this one (pm3d.py:122-127).
// One CTA per super-tile: the (TS+1)^3 node patch of all three grids is staged in shared
// memory, and the super-tile's particles -- one contiguous range -- read their 8 corners from
// there.  Each result is written to the same position of the temporary state with the class of
// its new super-tile; per-class counts feed the re-binning.
struct PushCoef {
  float kA, kB, D, gscale;
  int run;
};

template <int T>
__device__ __forceinline__ void push_one(const StepArgs& A, const PeakDesc& P, const float* __restrict__ s_f,
                                         const PushCoef& K, int sx, int sy, int sz, int4 ps, float4 m, long long j,
                                         u32* s_cnt, bool& bad, double4& acc_e) {
  constexpr int RS = patch_rs(T), PS = patch_ps(T), CS = patch_size(T);
  const int N = P.N, l2 = P.log2N;
  const int ix = ps.x >> (2 * l2), iy = (ps.x >> l2) & (N - 1), iz = ps.x & (N - 1);
  const int lx = ix - sx * T, ly = iy - sy * T, lz = iz - sz * T;
  if ((unsigned)lx >= (unsigned)T || (unsigned)ly >= (unsigned)T || (unsigned)lz >= (unsigned)T) {
    bad = true;  // grouping and state disagree: flag it, never index outside the patch
    return;
  }
  float fx = __int_as_float(ps.y), fy = __int_as_float(ps.z), fz = __int_as_float(ps.w);
  const float gx = 1.0f - fx, gy = 1.0f - fy, gz = 1.0f - fz;
  const int o = lx * PS + ly * RS + lz;
  float ax = 0.f, ay = 0.f, az = 0.f;
#define PM_CORNER(w, d)                       \
  {                                           \
    const float w_ = (w);                     \
    ax = fmaf(w_, s_f[o + (d)], ax);          \
    ay = fmaf(w_, s_f[CS + o + (d)], ay);     \
    az = fmaf(w_, s_f[2 * CS + o + (d)], az); \
  }
  const float w00 = gx * gy, w01 = gx * fy, w10 = fx * gy, w11 = fx * fy;
  PM_CORNER(w00 * gz, 0)
  PM_CORNER(w00 * fz, 1)
  PM_CORNER(w01 * gz, RS)
  PM_CORNER(w01 * fz, RS + 1)
  PM_CORNER(w10 * gz, PS)
  PM_CORNER(w10 * fz, PS + 1)
  PM_CORNER(w11 * gz, PS + RS)
  PM_CORNER(w11 * fz, PS + RS + 1)
#undef PM_CORNER
  ax *= K.gscale;
  ay *= K.gscale;
  az *= K.gscale;
  float px = m.x + K.kA * ax, py = m.y + K.kA * ay, pz = m.z + K.kA * az;
  // Momentum synchronised with the positions (after the closing kick): energy and momentum sums.
  {
    double4 t = acc_e;
    const double dx = px, dy = py, dz = pz;
    t.x += dx;
    t.y += dy;
    t.z += dz;
    t.w += dx * dx + dy * dy + dz * dz;
    acc_e = t;
  }
  int nx = ix, ny = iy, nz = iz;
  int mx = 0, my = 0, mz = 0;  // cells moved along each axis
  const bool finite = isfinite(px) && isfinite(py) && isfinite(pz);
  if (K.run && finite) {  // a non-finite particle stays where it is (the peak is flagged below)
    px += K.kB * ax;
    py += K.kB * ay;
    pz += K.kB * az;
#define PM_DRIFT(f, p, i, m)    \
  {                             \
    float fn = f + K.D * p;     \
    float c = floorf(fn);       \
    fn -= c;                    \
    if (fn >= 1.0f) {           \
      fn -= 1.0f;               \
      c += 1.0f;                \
    }                           \
    f = fn;                     \
    m = (int)c;                 \
    i = (i + m) & (N - 1);      \
  }
    PM_DRIFT(fx, px, nx, mx)
    PM_DRIFT(fy, py, ny, my)
    PM_DRIFT(fz, pz, nz, mz)
#undef PM_DRIFT
  }
  bad |= !(finite && isfinite(px) && isfinite(py) && isfinite(pz));
  const int cell = (nx << (2 * l2)) | (ny << l2) | nz;
  A.tpos[j] = make_int4(cell, __float_as_int(fx), __float_as_int(fy), __float_as_int(fz));
  A.tmom[j] = make_float4(px, py, pz, m.w);
  // Class of the destination super-tile (re-derived from the cell by the scatter), counted:
  // most particles stay (one warp-aggregated add), the few movers add one each.  With more than
  // five super-tiles per axis the class follows from the local cell and the cells moved
  // (super-tile offsets -2..2 per axis, the same class bin_class gives); anything else, and
  // smaller meshes, go through bin_class.  The sums are formed modulo 2^32: a saturated move of
  // a runaway particle stays far outside -2..2.
  u32 far_st = 0;
  int c;
  const int ox = (int)((u32)lx + (u32)mx) >> P.log2TS, oy = (int)((u32)ly + (u32)my) >> P.log2TS,
            oz = (int)((u32)lz + (u32)mz) >> P.log2TS;
  if (P.NS > 5 && (unsigned)(ox + 2) <= 4u && (unsigned)(oy + 2) <= 4u && (unsigned)(oz + 2) <= 4u)
    c = ((ox >= 0 ? ox : 2 - ox) * 5 + (oy >= 0 ? oy : 2 - oy)) * 5 + (oz >= 0 ? oz : 2 - oz);
  else
    c = bin_class(cell, sx, sy, sz, P, &far_st);
  const u32 stay = __ballot_sync(__activemask(), c == 0);
  if (c == 0) {
    if ((stay & lanemask_lt()) == 0) atomicAdd(&s_cnt[0], (u32)__popc(stay));
  } else if (c == BIN_FAR) {
    atomicAdd(&A.far_count[P.st_base + far_st], 1u);  // counted at its own destination
  } else {
    atomicAdd(&s_cnt[c], 1u);
  }
}

template <int T>
__device__ __forceinline__ void push_super(const StepArgs& A, const PeakDesc& P, const PeakClock& C, int pk, u32 st,
                                           float* s_f, u32* s_cnt, const PushCoef& K) {
  constexpr int T1 = T + 1, RS = patch_rs(T), PS = patch_ps(T), CS = patch_size(T);
  constexpr int CH = T / 4 + 1;  // per patch row: T/4 copies of 16 bytes, then the (wrapped) last node
  const int N = P.N;
  const int sx = pm_compact3(st >> 2), sy = pm_compact3(st >> 1), sz = pm_compact3(st);
  const long long N3 = (long long)N * N * N;
  const u32* ss = sst(A, C.sbuf) + P.sst_off;
  const long long b = ss[st], e = ss[st + 1];
  if (b < e) {
    // Asynchronous copies of the patch rows (every row start is 16-byte aligned on both sides:
    // z0 = sz*T is a multiple of 4 and the grids are 256-byte aligned).
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(s_f);
    const int z0 = sz * T, zl = (sz * T + T) & (N - 1);
    for (int i = threadIdx.x; i < 3 * T1 * T1 * CH; i += PUSH_THREADS) {
      const int row = i / CH, part = i - row * CH;
      const int comp = row / (T1 * T1), r = row - comp * (T1 * T1);
      const int lx = r / T1, ly = r - lx * T1;
      const int gx = (sx * T + lx) & (N - 1), gy = (sy * T + ly) & (N - 1);
      const float* src = P.force + comp * N3 + ((long long)gx * N + gy) * N;
      const unsigned dst = sbase + 4u * (unsigned)(comp * CS + lx * PS + ly * RS + part * 4);
      if (part < T / 4) cp_async16(dst, src + z0 + part * 4);
      else cp_async4(dst, src + zl);
    }
    cp_async_wait_all();
  }
  __syncthreads();
  bool bad = false;
  double4 acc_e = make_double4(0.0, 0.0, 0.0, 0.0);  // this thread's momentum and p^2 sums
  // One particle per thread per sweep, the next two sweeps' particles in flight meanwhile;
  // 32-bit indices inside the super-tile's range.
  const int4* __restrict__ pp = A.pos + b;
  const float4* __restrict__ mp = A.mom + b;
  const int n = (int)(e - b);
  int k = threadIdx.x;
  int4 pa = make_int4(0, 0, 0, 0), pb = pa;
  float4 ma = make_float4(0.f, 0.f, 0.f, 0.f), mb = ma;
  if (k < n) {
    pa = pp[k];
    ma = mp[k];
  }
  if (k + PUSH_THREADS < n) {
    pb = pp[k + PUSH_THREADS];
    mb = mp[k + PUSH_THREADS];
  }
  for (; k < n; k += PUSH_THREADS) {
    const int4 p0 = pa;
    const float4 m0 = ma;
    pa = pb;
    ma = mb;
    if (k + 2 * PUSH_THREADS < n) {
      pb = pp[k + 2 * PUSH_THREADS];
      mb = mp[k + 2 * PUSH_THREADS];
    }
    push_one<T>(A, P, s_f, K, sx, sy, sz, p0, m0, b + k, s_cnt, bad, acc_e);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&A.stats[pk].status, 1u);
  for (int c = threadIdx.x; c < P.NC; c += PUSH_THREADS) A.counts[(P.st_base + st) * BIN_CLASSES + c] = s_cnt[c];
  // Super-tile partials of the momentum and p^2 sums (compensated, fixed order).
  __shared__ CSum s_e[PUSH_THREADS / 32][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double4 ev = acc_e;
  const double ea[4] = {ev.x, ev.y, ev.z, ev.w};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const CSum v = csum_warp(CSum{ea[q], 0.0});
    if (lane == 0) s_e[warp][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    CSum t = s_e[0][threadIdx.x];
    for (int w = 1; w < PUSH_THREADS / 32; ++w) csum_merge(t, s_e[w][threadIdx.x]);
    A.epart[(P.st_base + st) * 4 + threadIdx.x] = make_double2(t.s, t.c);
  }
}

__global__ void __launch_bounds__(PUSH_THREADS, 2) k_push(StepArgs A) {
  extern __shared__ __align__(16) float s_f[];
  __shared__ PushCoef s_k;
  __shared__ u32 s_cnt[BIN_CLASSES];
  const TileRef tr = find_tile(A.st_base, A.npeaks);
  const PeakClock C = A.clocks[tr.pk];
  if (C.state != PS_RUN && C.state != PS_FINALIZE) return;
  const PeakDesc P = A.peaks[tr.pk];
  if (threadIdx.x < BIN_CLASSES) s_cnt[threadIdx.x] = 0u;
  if (threadIdx.x == 0) {
    const double a = C.a, da = C.da;
    const bool run = C.state == PS_RUN;
    const double amid = a + 0.5 * da;
    s_k.kA = (float)C.kpend;
    s_k.kB = run ? (float)(0.5 * da / (a * pm_hubble(a))) : 0.f;
    s_k.D = run ? (float)(da / (amid * amid * amid * pm_hubble(amid)) / P.dx) : 0.f;
    s_k.gscale = (float)(C.a_grid / a);
    s_k.run = run ? 1 : 0;
  }
  __syncthreads();
  const PushCoef K = s_k;
  const u32 st = (u32)tr.t;
  switch (P.TS) {
    case 4: push_super<4>(A, P, C, tr.pk, st, s_f, s_cnt, K); break;
    case 8: push_super<8>(A, P, C, tr.pk, st, s_f, s_cnt, K); break;
    default: push_super<16>(A, P, C, tr.pk, st, s_f, s_cnt, K); break;
  }
}

// Clock advance (one thread per peak): applies the step that the push kernel just made,
// selects the next step size, whether this step regroups by sort, and which peaks re-deposit.
__global__ void k_advance(StepArgs A) {
  int any_sort = 0, any_refresh = 0;
  for (int pk = threadIdx.x; pk < A.npeaks; pk += blockDim.x) {
    PeakClock c = A.clocks[pk];
    const PeakDesc P = A.peaks[pk];
    int dep = 0;
    // Collapse detection on the deposit made by the previous step, i.e. of the positions at c.a.
    // This step's push has already moved a running peak on to c.a + c.da, so a stop takes
    // effect after the step is booked below: the next step applies its closing kick and ends.
    bool stop_now = false;
    if (c.has_delta && c.delta_collapse > 0 && c.a_collapse < 0 && c.state != PS_PRIME) {
      const double dmax = (double)A.stats[pk].max_fix / (double)PM_FIX_ONE / P.n_mean - 1.0;
      if (dmax >= c.delta_collapse) {
        c.a_collapse = c.a;
        stop_now = c.stop_on_collapse && c.state == PS_RUN;
      }
    }
    switch (c.state) {
      case PS_PRIME:
        dep = 1;
        c.sortstep = 1;
        c.refresh = 0;
        c.sbuf ^= 1;
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
        c.sortstep = 0;
        c.refresh = (c.nsteps % P.full_every) == 0 ? 1 : 0;
        c.sbuf ^= 1;
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
        if (stop_now && c.state == PS_RUN) c.state = PS_FINALIZE;
        break;
      }
      case PS_FINALIZE:
        c.kpend = 0.0;
        c.sortstep = 0;
        c.refresh = 0;
        c.sbuf ^= 1;
        dep = 1;
        c.state = PS_IDLE;
        break;
      default:
        break;
    }
    c.dep = dep;
    A.clocks[pk] = c;
    A.sortseg[pk].active = dep && c.sortstep;
    any_sort |= dep && c.sortstep;
    any_refresh |= dep && c.refresh;
    if (dep) {
      A.stats[pk].max_fix = 0;
      A.stats[pk].mass_defect = 0;
    }
  }
  any_sort = __syncthreads_or(any_sort);
  any_refresh = __syncthreads_or(any_refresh);
  if (threadIdx.x == 0) {
    *A.sort_gate = any_sort ? 1u : 0u;
    *A.refresh_gate = any_refresh ? 1u : 0u;
  }
}

// ------------------------------------------------------------------------------------------
// Energy and momentum of every peak that was just pushed (before the clock advances): the push
// partials give K and sum p at the positions' a, the previous step's Green partials give W at
// the same a (the grids were computed there).  ENERGY_SLICES CTAs per peak each reduce a slice
// of the partials; the last one to finish (atomic ticket) merges the slices in slice order and
// updates the statistics.  All sums are compensated, every order fixed.  The Layzer-Irvine
// integral int K da advances by the trapezoid rule between samples.
__global__ void __launch_bounds__(PM_THREADS) k_energy(StepArgs A) {
  const int pk = blockIdx.y, sl = blockIdx.x;
  const PeakClock C = A.clocks[pk];
  if (C.state != PS_RUN && C.state != PS_FINALIZE) return;
  const PeakDesc P = A.peaks[pk];
  __shared__ CSum s_w[PM_THREADS / 32][5];
  __shared__ u32 s_last;
  CSum v[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) v[q] = CSum{0.0, 0.0};
  const long long t0 = P.nst * sl / ENERGY_SLICES, t1 = P.nst * (sl + 1) / ENERGY_SLICES;
  for (long long t = t0 + threadIdx.x; t < t1; t += PM_THREADS) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double2 e = A.epart[(P.st_base + t) * 4 + q];
      csum_merge(v[q], CSum{e.x, e.y});
    }
  }
  // Green partials: one per warp of each Green block of this peak.
  const long long nw = (P.nmodes + PM_THREADS * GREEN_MODES - 1) / (PM_THREADS * GREEN_MODES) * (PM_THREADS / 32);
  const long long g0 = nw * sl / ENERGY_SLICES, g1 = nw * (sl + 1) / ENERGY_SLICES;
  const double* wp = A.wpart + P.mode_base * (PM_THREADS / 32);
  for (long long t = g0 + threadIdx.x; t < g1; t += PM_THREADS) csum_add(v[4], wp[t]);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    const CSum r = csum_warp(v[q]);
    if (lane == 0) s_w[warp][q] = r;
  }
  __syncthreads();
  double2* slice = A.eslice + ((long long)pk * ENERGY_SLICES) * 5;
  if (threadIdx.x < 5) {
    CSum t = s_w[0][threadIdx.x];
    for (int w = 1; w < PM_THREADS / 32; ++w) csum_merge(t, s_w[w][threadIdx.x]);
    slice[sl * 5 + threadIdx.x] = make_double2(t.s, t.c);
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&A.ecount[pk], 1u) == ENERGY_SLICES - 1 ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  __shared__ double s_tot[5];
  if (threadIdx.x < 5) {
    CSum t = CSum{0.0, 0.0};
    for (int q = 0; q < ENERGY_SLICES; ++q) {
      const double2 e = __ldcg(slice + q * 5 + threadIdx.x);
      csum_merge(t, CSum{e.x, e.y});
    }
    s_tot[threadIdx.x] = t.s + t.c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    A.ecount[pk] = 0u;
    PeakStats& S = A.stats[pk];
    const double a = C.a;
    const double kin = P.m_part / (2.0 * a * a) * s_tot[3];
    const double pot = 0.5 * (3.0 * PM_H_I * PM_H_I / (8.0 * M_PI)) * P.dx * P.dx * P.dx * s_tot[4];
    if (S.nsamples == 0) {
      S.li_int = 0.0;
      S.li_e0 = a * (kin + pot);
    } else {
      S.li_int += 0.5 * (S.kin + kin) * (a - S.a_e);
    }
    S.a_e = a;
    S.mom[0] = P.m_part * s_tot[0];
    S.mom[1] = P.m_part * s_tot[1];
    S.mom[2] = P.m_part * s_tot[2];
    S.kin = kin;
    S.pot = pot;
    S.nsamples += 1;
  }
}

// ------------------------------------------------------------------------------------------
// Regrouping by sort (priming and every full_every steps): gather the temporary state in
// sorted order and find the super-tile starts in the sorted keys.
// Both are grid-stride loops over a grid of a few CTAs per SM and return at once on the steps
// where no peak sorts.
__global__ void k_permute(StepArgs A, long long ntot) {
  if (*A.sort_gate == 0u) return;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < ntot; j += (long long)gridDim.x * blockDim.x) {
    const int pk = pm_find(A.p_base, A.npeaks, j);
    const PeakClock C = A.clocks[pk];
    if (!(C.dep && C.sortstep)) continue;
    const u32 q = A.perm[j];
    const PeakDesc& P = A.peaks[pk];
    if ((long long)q < P.p_off || (long long)q >= P.p_off + P.n) {  // a failed sort: never read outside
      atomicOr(&A.stats[pk].status, 2u);
      continue;
    }
    A.pos[j] = A.tpos[q];
    A.mom[j] = A.tmom[q];
  }
}

__global__ void k_st_starts(StepArgs A, long long ntot) {
  if (*A.sort_gate == 0u) return;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < ntot; j += (long long)gridDim.x * blockDim.x) {
    const int pk = pm_find(A.p_base, A.npeaks, j);
    const PeakClock C = A.clocks[pk];
    if (!(C.dep && C.sortstep)) continue;
    const PeakDesc P = A.peaks[pk];
    u32* ss = sst(A, C.sbuf) + P.sst_off;
    // Super-tile of each sorted key; a key outside the peak's key range (a failed sort) is
    // clamped, so no start is ever written outside the peak's table.
    const u32 kb = A.keys_sorted[j] >> P.st_shift;
    if (kb >= (u32)P.nst) atomicOr(&A.stats[pk].status, 2u);
    const int b = (int)min(kb, (u32)(P.nst - 1));
    const int bprev = j == P.p_off ? -1 : (int)min(A.keys_sorted[j - 1] >> P.st_shift, (u32)(P.nst - 1));
    for (int bb = bprev + 1; bb <= b; ++bb) ss[bb] = (u32)j;
    if (j == P.p_off + P.n - 1)
      for (int bb = b + 1; bb <= P.nst; ++bb) ss[bb] = (u32)(P.p_off + P.n);
  }
}

// ------------------------------------------------------------------------------------------
// Regrouping by re-binning (the other steps).  Destination super-tile D takes, in class order,
// the run of each source D - u(c) whose particles moved by u(c), then its far movers.
// scan1: per destination, offsets of its incoming runs and its total.
__global__ void __launch_bounds__(BIN_CLASSES) k_bin_scan1(StepArgs A) {
  __shared__ u32 s_w[BIN_CLASSES / 32];
  const TileRef tr = find_tile(A.st_base, A.npeaks);
  const PeakClock C = A.clocks[tr.pk];
  if (!(C.dep && !C.sortstep)) return;
  const PeakDesc P = A.peaks[tr.pk];
  const u32 D = (u32)tr.t;
  const int dx = pm_compact3(D >> 2), dy = pm_compact3(D >> 1), dz = pm_compact3(D);
  const int c = threadIdx.x, lane = c & 31, warp = c >> 5;
  u32 v = 0, src = 0;
  if (c < P.NC) {
    const int W = P.W, NS = P.NS;
    const int ux = bin_offset(c / (W * W), NS), uy = bin_offset((c / W) % W, NS), uz = bin_offset(c % W, NS);
    src = pm_morton3((dx - ux) & (NS - 1), (dy - uy) & (NS - 1), (dz - uz) & (NS - 1));
    v = A.counts[(P.st_base + src) * BIN_CLASSES + c];
  }
  u32 incl = v;
  for (int d = 1; d < 32; d <<= 1) {
    const u32 t = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += t;
  }
  if (lane == 31) s_w[warp] = incl;
  __syncthreads();
  u32 off = 0;
  for (int w = 0; w < warp; ++w) off += s_w[w];
  if (c < P.NC) A.lpre[(P.st_base + src) * BIN_CLASSES + c] = off + incl - v;
  if (c == BIN_CLASSES - 1) A.totals[P.st_base + D] = off + incl + A.far_count[P.st_base + D];
}

// scan2: per peak, super-tile starts from the totals.
__global__ void __launch_bounds__(1024) k_bin_scan2(StepArgs A) {
  __shared__ u32 s_w[32];
  __shared__ long long s_carry;
  const int pk = blockIdx.x;
  const PeakClock C = A.clocks[pk];
  if (!(C.dep && !C.sortstep)) return;
  const PeakDesc P = A.peaks[pk];
  u32* ss = sst(A, C.sbuf) + P.sst_off;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_carry = P.p_off;
  __syncthreads();
  for (int base = 0; base < P.nst; base += 1024) {
    const int i = base + threadIdx.x;
    const u32 v = i < P.nst ? A.totals[P.st_base + i] : 0u;
    u32 incl = v;
    for (int d = 1; d < 32; d <<= 1) {
      const u32 t = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += t;
    }
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    u32 off = 0;
    for (int w = 0; w < warp; ++w) off += s_w[w];
    const long long carry = s_carry;
    if (i < P.nst) ss[i] = (u32)(carry + off + incl - v);
    __syncthreads();
    if (threadIdx.x == 1023) s_carry = carry + off + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    ss[P.nst] = (u32)(P.p_off + P.n);
    if (s_carry != P.p_off + P.n) atomicOr(&A.stats[pk].status, 4u);  // counts lost a particle
  }
}

// scatter: per source super-tile, every particle to its place in the new grouping.
__global__ void __launch_bounds__(PUSH_THREADS) k_bin_scatter(StepArgs A) {
  __shared__ u32 s_rank[BIN_CLASSES];
  const TileRef tr = find_tile(A.st_base, A.npeaks);
  const PeakClock C = A.clocks[tr.pk];
  if (!(C.dep && !C.sortstep)) return;
  const PeakDesc P = A.peaks[tr.pk];
  const u32 S = (u32)tr.t;
  const u32* old = sst(A, C.sbuf ^ 1) + P.sst_off;
  const u32* ss = sst(A, C.sbuf) + P.sst_off;
  if (threadIdx.x < BIN_CLASSES) s_rank[threadIdx.x] = 0u;
  __syncthreads();
  const int sx = pm_compact3(S >> 2), sy = pm_compact3(S >> 1), sz = pm_compact3(S);
  const int NS = P.NS, W = P.W;
  const long long b = old[S], e = old[S + 1];
  // Run of the stayers (class 0) in this super-tile's own new range.
  const long long stay0 = (long long)ss[S] + A.lpre[(P.st_base + S) * BIN_CLASSES];
  for (long long j = b + threadIdx.x; j < e; j += PUSH_THREADS) {
    const int4 ps = A.tpos[j];
    const float4 m = A.tmom[j];
    u32 D = 0;
    const int c = bin_class(ps.x, sx, sy, sz, P, &D);
    long long dest;
    // Ranks inside a class run: one warp-aggregated add for the stayers, one add per mover.
    // The order inside a run is arbitrary; nothing downstream depends on it.
    const u32 stay = __ballot_sync(__activemask(), c == 0);
    if (c == 0) {
      const int leader = __ffs(stay) - 1;
      u32 base = 0;
      if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(&s_rank[0], (u32)__popc(stay));
      base = __shfl_sync(stay, base, leader);
      dest = stay0 + base + __popc(stay & lanemask_lt());
    } else if (c != BIN_FAR) {
      const int ux = bin_offset(c / (W * W), NS), uy = bin_offset((c / W) % W, NS), uz = bin_offset(c % W, NS);
      D = pm_morton3((sx + ux) & (NS - 1), (sy + uy) & (NS - 1), (sz + uz) & (NS - 1));
      dest = (long long)ss[D] + A.lpre[(P.st_base + S) * BIN_CLASSES + c] + atomicAdd(&s_rank[c], 1u);
    } else {
      dest = (long long)ss[D + 1] - A.far_count[P.st_base + D] + atomicAdd(&A.far_fill[P.st_base + D], 1u);
    }
    if (dest < P.p_off || dest >= P.p_off + P.n) {  // counts and classes disagree: never write outside
      atomicOr(&A.stats[tr.pk].status, 4u);
      continue;
    }
    A.pos[dest] = ps;
    A.mom[dest] = m;
  }
}

// ------------------------------------------------------------------------------------------
// Refresh: every full_every steps, after re-binning, each super-tile's particles are re-sorted
// by cell (local Morton code of the cell inside the super-tile), so the deposit's and the
// push's warps see neighbouring cells and same-cell runs again.  A counting sort per
// super-tile: the order inside one cell is not kept (nothing downstream depends on it; the
// deposit sums integers).  Up to TSORT_CAP particles the super-tile is staged in shared memory
// and written back in place, coalesced (64 bytes of traffic per particle); denser super-tiles
// go through the temporary state (push output, free after re-binning) and back.  Persistent
// grid (one CTA per SM) over the super-tiles; every launch returns at once when no peak
// refreshes this step.
template <int TS>
__device__ __forceinline__ void tile_sort(const StepArgs& A, const PeakDesc& P, const PeakClock& C, u32 st,
                                          unsigned char* smem) {
  constexpr int NCELL = TS * TS * TS;
  u32* hist = (u32*)smem;                                           // [NCELL], then its prefix
  int4* spos = (int4*)(smem + sizeof(u32) * 16 * 16 * 16);          // [TSORT_CAP]
  float4* smom = (float4*)(spos + TSORT_CAP);                       // [TSORT_CAP]
  u32* cr = (u32*)(smom + TSORT_CAP);                               // [TSORT_CAP] cell << 16 | rank
  unsigned short* inv = (unsigned short*)(cr + TSORT_CAP);          // [TSORT_CAP] slot -> particle
  __shared__ u32 s_wsum[TSORT_THREADS / 32];
  const u32* ss = sst(A, C.sbuf) + P.sst_off;
  const long long b = ss[st], e = ss[st + 1];
  const int n = (int)(e - b);
  if (n < 2) return;  // uniform
  const int N = P.N, l2 = P.log2N;
  const int sx = pm_compact3(st >> 2), sy = pm_compact3(st >> 1), sz = pm_compact3(st);
  // Local cell code; masked into the super-tile so a corrupted grouping cannot index outside.
  auto cell_of = [&](int c) -> u32 {
    const int ix = c >> (2 * l2), iy = (c >> l2) & (N - 1), iz = c & (N - 1);
    return pm_morton3((ix - sx * TS) & (TS - 1), (iy - sy * TS) & (TS - 1), (iz - sz * TS) & (TS - 1));
  };
  for (int i = threadIdx.x; i < NCELL; i += TSORT_THREADS) hist[i] = 0u;
  __syncthreads();
  const bool staged = n <= TSORT_CAP;
  if (staged) {
    for (int i = threadIdx.x; i < n; i += TSORT_THREADS) {
      const int4 p = A.pos[b + i];
      spos[i] = p;
      smom[i] = A.mom[b + i];
      const u32 c = cell_of(p.x);
      cr[i] = (c << 16) | atomicAdd(&hist[c], 1u);
    }
  } else {
    for (int i = threadIdx.x; i < n; i += TSORT_THREADS) {
      const u32 c = cell_of(A.pos[b + i].x);
      A.keys_push[b + i] = atomicAdd(&hist[c], 1u);
    }
  }
  __syncthreads();
  // Exclusive prefix of the cell counts (NCELL <= 4096 = 4 per thread).
  {
    constexpr int PER = (NCELL + TSORT_THREADS - 1) / TSORT_THREADS;
    u32 v[PER];
    u32 tot = 0;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int i = threadIdx.x * PER + k;
      v[k] = i < NCELL ? hist[i] : 0u;
      tot += v[k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u32 incl = tot;
    for (int d = 1; d < 32; d <<= 1) {
      const u32 t = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += t;
    }
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    u32 off = 0;
    for (int w = 0; w < warp; ++w) off += s_wsum[w];
    u32 run = off + incl - tot;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int i = threadIdx.x * PER + k;
      if (i < NCELL) hist[i] = run;
      run += v[k];
    }
  }
  __syncthreads();
  if (staged) {
    for (int i = threadIdx.x; i < n; i += TSORT_THREADS) {
      const u32 x = cr[i];
      inv[hist[x >> 16] + (x & 0xFFFFu)] = (unsigned short)i;
    }
    __syncthreads();
    for (int o = threadIdx.x; o < n; o += TSORT_THREADS) {
      const int i = inv[o];
      A.pos[b + o] = spos[i];
      A.mom[b + o] = smom[i];
    }
  } else {
    for (int i = threadIdx.x; i < n; i += TSORT_THREADS) {
      const int4 p = A.pos[b + i];
      const long long d = b + hist[cell_of(p.x)] + A.keys_push[b + i];
      A.tpos[d] = p;
      A.tmom[d] = A.mom[b + i];
    }
    __syncthreads();  // the block's global writes are visible to the block after the barrier
    for (int o = threadIdx.x; o < n; o += TSORT_THREADS) {
      A.pos[b + o] = A.tpos[b + o];
      A.mom[b + o] = A.tmom[b + o];
    }
  }
  __syncthreads();  // shared arrays are reused by the next super-tile
}

__global__ void __launch_bounds__(TSORT_THREADS) k_tile_sort(StepArgs A, long long nst) {
  extern __shared__ __align__(16) unsigned char s_ts[];
  __shared__ int s_pk;
  if (*A.refresh_gate == 0u) return;
  for (long long t = blockIdx.x; t < nst; t += gridDim.x) {
    if (threadIdx.x == 0) s_pk = pm_find(A.st_base, A.npeaks, t);
    __syncthreads();
    const int pk = s_pk;
    __syncthreads();
    const PeakClock C = A.clocks[pk];
    if (!(C.dep && C.refresh)) continue;
    const PeakDesc P = A.peaks[pk];
    const u32 st = (u32)(t - A.st_base[pk]);
    switch (P.TS) {
      case 4: tile_sort<4>(A, P, C, st, s_ts); break;
      case 8: tile_sort<8>(A, P, C, st, s_ts); break;
      default: tile_sort<16>(A, P, C, st, s_ts); break;
    }
  }
}

// ------------------------------------------------------------------------------------------
// Deterministic CIC deposit (pm3d.py:81-89, 103-104).  One CTA per super-tile deposits its own
// particles (one contiguous range) onto the (TS+1)^3 nodes they touch.  Per particle the 8 CIC
// weights are formed in 64-bit fixed point with 38 fractional bits, the 8th corner taking the
// remainder so each particle deposits exactly 2^38.  Each node accumulates in shared memory as two
// native 32-bit words (the signed weight's bits >= 19 and its low 19 bits), exact within a chunk
// of up to 8191 particles, and is folded into a 64-bit register accumulator after every chunk.
// Interior nodes are then final and written as FP32 delta = S/n_mean - 1; nodes on the three
// lower faces (which neighbours also reach) and on the upper halo (which belongs to the
// neighbours) are written as 64-bit partials.
//
// The face fix-up (k_fixup, the next launch) completes the face nodes: own partial plus the
// lower neighbours' halo partials.
// Integer sums make the result independent of particle order, bit for bit; no float atomics.
__device__ __forceinline__ int face_index(int lx, int ly, int lz, int T) {
  if (lx == 0) return ly * T + lz;
  if (ly == 0) return T * T + (lx - 1) * T + lz;
  return T * T + (T - 1) * T + (lx - 1) * (T - 1) + (ly - 1);
}
__device__ __forceinline__ int halo_index(int lx, int ly, int lz, int T) {
  if (lx == T) return ly * (T + 1) + lz;
  if (ly == T) return (T + 1) * (T + 1) + lx * (T + 1) + lz;
  return (T + 1) * (T + 1) + T * (T + 1) + lx * T + ly;
}
// Inverse of face_index.
template <int T>
__device__ __forceinline__ void face_coords(int f, int& lx, int& ly, int& lz) {
  if (f < T * T) {
    lx = 0;
    ly = f / T;
    lz = f % T;
  } else if (f < T * T + (T - 1) * T) {
    const int r = f - T * T;
    lx = 1 + r / T;
    ly = 0;
    lz = r % T;
  } else {
    const int r = f - T * T - (T - 1) * T;
    lx = 1 + r / (T - 1);
    ly = 1 + r % (T - 1);
    lz = 0;
  }
}

// Finish the face nodes of super-tile Y (whole CTA of FIX_THREADS): each face node's own
// partial plus the halo partials of the lower neighbours Y - o, o = (ox, oy, oz) in {0,1}^3 \ 0,
// that reach it (node (lx + TS ox, ...) of the neighbour, which lies on its upper halo, for a
// face node with (lx, ly, lz) zero where o is one).  nb[o]: the neighbours' halo partials.
// Adds to the caller's statistics.
template <int TS>
__device__ __forceinline__ void fixup_faces(const StepArgs& A, const PeakDesc& P, u32 Y, const long long* const* nb,
                                            double* rho64, long long& dsum, long long& smax) {
  constexpr int FC = TS * TS * TS - (TS - 1) * (TS - 1) * (TS - 1);
  const int N = P.N;
  const int sx = pm_compact3(Y >> 2), sy = pm_compact3(Y >> 1), sz = pm_compact3(Y);
  const long long* face = A.face + P.face_off + (long long)Y * FC;
  for (int f = threadIdx.x; f < FC; f += FIX_THREADS) {
    int lx, ly, lz;
    face_coords<TS>(f, lx, ly, lz);
    long long S = __ldcg(face + f);
    const int zmask = (lx == 0 ? 1 : 0) | (ly == 0 ? 2 : 0) | (lz == 0 ? 4 : 0);
    for (int o = zmask; o; o = (o - 1) & zmask) {  // non-empty subsets of zmask
      S += __ldcg(nb[o] + halo_index(lx + TS * (o & 1), ly + TS * ((o >> 1) & 1), lz + TS * (o >> 2), TS));
    }
    const long long Dv = S - P.n_mean_fix;
    const long long node = ((long long)(sx * TS + lx) * N + (sy * TS + ly)) * N + (sz * TS + lz);
    P.delta[node] = (float)((double)Dv * P.inv_fix_nmean);
    if (rho64) rho64[node] = (double)S * (1.0 / (double)PM_FIX_ONE);
    dsum += Dv;
    smax = S > smax ? S : smax;
  }
}

// Nearest integer to the exact product a*b for 0 <= a*b < 2^51: one FMA with 2^52 rounds the
// product to an integer in the mantissa (round half to even), whose low 52 bits are read off.
// The same rounding as __double2ll_rn of the exact product, on the FP64 pipe instead of the
// conversion unit.
__device__ __forceinline__ u64 fix_round(double a, double b) {
  return (u64)__double_as_longlong(fma(a, b, 4503599627370496.0)) & 0xFFFFFFFFFFFFFull;
}

// Shared-memory address of node number `node` (z fastest) of a (TS+1)^3 patch.
template <int TS>
__device__ __forceinline__ int dep_addr(int node) {
  constexpr int T1 = TS + 1;
  const int lx = node / (T1 * T1), r = node - lx * (T1 * T1), ly = r / T1, lz = r - ly * T1;
  return lx * patch_ps(TS) + ly * patch_rs(TS) + lz;
}
// A node's chunk sum from its split accumulators (high word modulo 2^32, see deposit_super).
__device__ __forceinline__ long long chunk_sum(u32 hi, u32 lo) {
  const long long hs = hi >= 0xFFFFE000u ? (long long)hi - (1LL << 32) : (long long)hi;
  return hs * (1LL << 19) + (long long)lo;
}

// Adds a full chunk's node sums into the fold scratch (first chunk: stores) and clears the
// chunk accumulators.  Kept out of line: it runs only for super-tiles of more than one chunk.
template <int TS>
__device__ __noinline__ void fold_chunk(u64* acc64, u32* acc_hi, u32* acc_lo, bool add) {
  constexpr int NN = (TS + 1) * (TS + 1) * (TS + 1);
  for (int node = threadIdx.x; node < NN; node += DEP_THREADS) {
    const int ad = dep_addr<TS>(node);
    acc64[node] = (add ? acc64[node] : 0ull) + (u64)chunk_sum(acc_hi[ad], acc_lo[ad]);
    acc_hi[ad] = 0u;
    acc_lo[ad] = 0u;
  }
}

// One corner weight W (a nearest integer of a product in units of 2^-38, 0 <= W < 2^39, see
// fix_round) split for the two accumulator words: hi = W >> 19, lo = W & (2^19 - 1).  The FMA's
// result has the bits 0x4330000000000000 + W, so hi is one funnel shift of its two words (the
// exponent bits shift out of the 32-bit result) and lo one mask of the low word.
struct Split {
  u32 hi, lo;
};
__device__ __forceinline__ Split fix_split(double a, double b) {
  const double r = fma(a, b, 4503599627370496.0);
  const u32 wl = (u32)__double2loint(r), wh = (u32)__double2hiint(r);
  return Split{__funnelshift_r(wl, wh, 19), wl & 0x7FFFFu};
}

template <int TS>
__device__ __forceinline__ void deposit_super(const StepArgs& A, const PeakDesc& P, const PeakClock& C, int pk,
                                              u32 st, u32* smem, double* rho64) {
  constexpr int T1 = TS + 1, NN = T1 * T1 * T1;
  constexpr int RS = patch_rs(TS), PS = patch_ps(TS), SZ = patch_size(TS);
  constexpr int NG = TS / 4 + 1;        // 4-node groups per patch row (the last holds the upper halo node)
  constexpr int FC = TS * TS * TS - (TS - 1) * (TS - 1) * (TS - 1);
  static_assert(RS % 4 == 0 && PS % 4 == 0 && RS >= 4 * NG, "patch rows are read 16 bytes at a time");
  u32* acc_hi = smem;
  u32* acc_lo = smem + SZ;
  __shared__ long long s_red[DEP_THREADS / 32];
  __shared__ long long s_max[DEP_THREADS / 32];
  const int N = P.N, l2 = P.log2N;
  const int sx = pm_compact3(st >> 2), sy = pm_compact3(st >> 1), sz = pm_compact3(st);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  static_assert((2 * SZ) % 4 == 0, "accumulators are cleared 16 bytes at a time");
  for (int i = threadIdx.x; i < 2 * SZ / 4; i += DEP_THREADS) reinterpret_cast<uint4*>(smem)[i] = make_uint4(0u, 0u, 0u, 0u);
  const u32* ss = sst(A, C.sbuf) + P.sst_off;
  const long long b = ss[st], e = ss[st + 1];
  const long long total = e - b;
  // A cell index belongs to this super-tile iff its bits outside the local ones equal the
  // super-tile's: one mask and one compare (negative or out-of-mesh values never match).
  const int local = ((TS - 1) << (2 * l2)) | ((TS - 1) << l2) | (TS - 1);
  const int tile_bits = ((sx * TS) << (2 * l2)) | ((sy * TS) << l2) | (sz * TS);
  __syncthreads();
  // Nodes' sums of the chunks folded so far, only for a super-tile of more than one chunk: kept
  // in the temporary particle state of its own range (free during the deposit; a range of more
  // than one chunk of 16-byte entries holds the NN 8-byte sums several times over).
  static_assert((8191 / DEP_THREADS) * DEP_THREADS * sizeof(int4) >= NN * sizeof(u64), "fold scratch too small");
  bool folded = false;
  // Split accumulators.  A weight W (at most 2^38, at least -3 for the remainder corner) goes in
  // as hi = W >> 19 in [-1, 2^19] and lo = W & (2^19 - 1).  A node takes at most one contribution
  // per particle of a chunk, so with CHUNK <= 8191 the low sums stay below 2^32 and the high
  // sums lie in [-CHUNK, CHUNK * 2^19], an interval shorter than 2^32 - 8192: kept modulo 2^32
  // in a u32, a value at or above 2^32 - 8192 is the negative one.  Both are exact.  A typical
  // super-tile (about TS^3 particles) is a single chunk.
  constexpr int CH_IT = 8191 / DEP_THREADS;  // sweeps of DEP_THREADS particles per chunk
  static_assert(CH_IT >= 1 && CH_IT * DEP_THREADS <= 8191, "chunk too large for the split accumulators");
  static_assert(PM_FIX_BITS == 38, "the split accumulators assume 38 fractional bits");
  // 32-bit indices inside the super-tile's range (fewer integer instructions than 64-bit ones).
  const int4* __restrict__ pp = A.pos + b;
  const int n = (int)total;
  const int nit = (n + DEP_THREADS - 1) / DEP_THREADS;
  int k = threadIdx.x;
  constexpr int DEPTH = PM_DEP_DEPTH;
  int4 q[DEPTH];  // the particles of the next DEPTH sweeps, loads in flight
#pragma unroll
  for (int d = 0; d < DEPTH; ++d) q[d] = k + d * DEP_THREADS < n ? pp[k + d * DEP_THREADS] : make_int4(-1, 0, 0, 0);
  bool bad = false;
  int left = CH_IT;
  for (int it = 0; it < nit; ++it) {
    const int4 ps = q[0];
    const bool valid = k < n;
#pragma unroll
    for (int d = 0; d + 1 < DEPTH; ++d) q[d] = q[d + 1];
    if (k + DEPTH * DEP_THREADS < n) q[DEPTH - 1] = pp[k + DEPTH * DEP_THREADS];
    k += DEP_THREADS;
    {
      const int c = ps.x;
      const bool in = valid && (c & ~local) == tile_bits;
      bad |= valid && !in;
      const double one = (double)PM_FIX_ONE;
      const double fx = __int_as_float(ps.y), fy = __int_as_float(ps.z), fz = __int_as_float(ps.w);
      const double Fx = fx * one, Gx = one - Fx;   // exact: fx has 24 significant bits
      const double gy = 1.0 - fy, gz = 1.0 - fz;
      const double w00 = Gx * gy, w01 = Gx * fy, w10 = Fx * gy, w11 = Fx * fy;
      // Seven corners rounded to integers in units of 2^-38; the eighth takes the remainder so
      // the particle deposits exactly 2^38 (hi/lo of 2^38 - sum, with lo in [0, 2^19)).
      const Split c0 = fix_split(w00, gz), c1 = fix_split(w00, fz), c2 = fix_split(w01, gz), c3 = fix_split(w01, fz),
                  c4 = fix_split(w10, gz), c5 = fix_split(w10, fz), c6 = fix_split(w11, gz);
      const u32 shi = c0.hi + c1.hi + c2.hi + c3.hi + c4.hi + c5.hi + c6.hi;
      const u32 slo = c0.lo + c1.lo + c2.lo + c3.lo + c4.lo + c5.lo + c6.lo;
      const Split c7{(1u << 19) - shi - ((slo + 0x7FFFFu) >> 19), (0u - slo) & 0x7FFFFu};
      const Split w[8] = {c0, c1, c2, c3, c4, c5, c6, c7};
      if (in) {
        const int nb = ((c >> (2 * l2)) & (TS - 1)) * PS + ((c >> l2) & (TS - 1)) * RS + (c & (TS - 1));
        const int off[8] = {0, 1, RS, RS + 1, PS, PS + 1, PS + RS, PS + RS + 1};
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          atomicAdd(&acc_hi[nb + off[q]], w[q].hi);
          atomicAdd(&acc_lo[nb + off[q]], w[q].lo);
        }
      }
    }
    if (--left == 0 && it + 1 < nit) {  // chunk full and more to come: fold it into acc64
      left = CH_IT;
      __syncthreads();
      fold_chunk<TS>(reinterpret_cast<u64*>(A.tpos + b), acc_hi, acc_lo, folded);
      folded = true;
      __syncthreads();
    }
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&A.stats[pk].status, 1u);
  // Write-out of the last chunk (plus the folded ones), four nodes of a patch row at a time:
  // interior nodes final as FP32 delta (16-byte stores; the first node of an interior row is a
  // face node, stored here from this super-tile's own sum and completed by k_fixup), nodes on
  // the lower faces and on the upper halo as 64-bit partials.
  long long dsum = 0, smax = 0;
  const long long gbase = ((long long)sx * TS * N + (long long)sy * TS) * N + sz * TS;
  long long* face = A.face + P.face_off + (long long)st * FC;
  long long* halo = A.halo + P.halo_off + (long long)st * P.hc;
  const u64* fold = reinterpret_cast<const u64*>(A.tpos + b);
  const long long nmf = P.n_mean_fix;
  const double inv = P.inv_fix_nmean;
  for (int item = threadIdx.x; item < T1 * T1 * NG; item += DEP_THREADS) {
    const int row = item / NG, g = item - row * NG;
    const int lx = row / T1, ly = row - lx * T1;
    const int ad = lx * PS + ly * RS + 4 * g;
    const uint4 h = *reinterpret_cast<const uint4*>(acc_hi + ad);
    const uint4 l = *reinterpret_cast<const uint4*>(acc_lo + ad);
    long long S[4] = {chunk_sum(h.x, l.x), chunk_sum(h.y, l.y), chunk_sum(h.z, l.z), chunk_sum(h.w, l.w)};
    const int nbase = row * T1 + 4 * g;  // dense node number of the group's first node
    if (folded) {
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (4 * g + k <= TS) S[k] += (long long)fold[nbase + k];
    }
    if (lx == TS || ly == TS) {  // a row of the upper halo
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int lz = 4 * g + k;
        if (lz <= TS) halo[halo_index(lx, ly, lz, TS)] = S[k];
      }
    } else if (g == NG - 1) {    // the row's upper-halo node
      halo[halo_index(lx, ly, TS, TS)] = S[0];
    } else if (lx == 0 || ly == 0) {  // a row of a lower face
#pragma unroll
      for (int k = 0; k < 4; ++k) face[face_index(lx, ly, 4 * g + k, TS)] = S[k];
    } else {                     // interior nodes (and the row's lz = 0 face node)
      if (g == 0) face[face_index(lx, ly, 0, TS)] = S[0];
      float4 d;
      float* dv = &d.x;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const long long D = S[k] - nmf;
        dv[k] = (float)((double)D * inv);
        if (g > 0 || k > 0) {
          dsum += D;
          smax = S[k] > smax ? S[k] : smax;
        }
      }
      const long long gi = gbase + ((long long)lx * N + ly) * N + 4 * g;
      *reinterpret_cast<float4*>(P.delta + gi) = d;
      if (rho64) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (g > 0 || k > 0) rho64[gi + k] = (double)S[k] * (1.0 / (double)PM_FIX_ONE);
      }
    }
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
    for (int w = 0; w < DEP_THREADS / 32; ++w) {
      ts += s_red[w];
      tm = s_max[w] > tm ? s_max[w] : tm;
    }
    atomicAdd((unsigned long long*)&A.stats[pk].mass_defect, (unsigned long long)ts);
    atomicMax(&A.stats[pk].max_fix, (u64)tm);
    A.far_count[P.st_base + st] = 0u;  // consumed by this step's regrouping
    A.far_fill[P.st_base + st] = 0u;
  }
}


__global__ void __launch_bounds__(DEP_THREADS, 4) k_deposit(StepArgs A, double* rho64) {
  extern __shared__ __align__(16) u32 s_dep[];
  const TileRef tr = find_tile(A.st_base, A.npeaks);
  const PeakClock C = A.clocks[tr.pk];
  if (!C.dep) return;
  const PeakDesc P = A.peaks[tr.pk];
  switch (P.TS) {
    case 4: deposit_super<4>(A, P, C, tr.pk, (u32)tr.t, s_dep, rho64); break;
    case 8: deposit_super<8>(A, P, C, tr.pk, (u32)tr.t, s_dep, rho64); break;
    default: deposit_super<16>(A, P, C, tr.pk, (u32)tr.t, s_dep, rho64); break;
  }
}

// Face fix-up: one CTA per super-tile whose peak deposited this step.  Small and
// latency-bound, so many CTAs per SM.
__global__ void __launch_bounds__(FIX_THREADS) k_fixup(StepArgs A, double* rho64) {
  __shared__ long long s_red[FIX_THREADS / 32];
  __shared__ long long s_max[FIX_THREADS / 32];
  __shared__ const long long* s_nb[8];
  const TileRef tr = find_tile(A.st_base, A.npeaks);
  if (!A.clocks[tr.pk].dep) return;
  const PeakDesc P = A.peaks[tr.pk];
  const u32 Y = (u32)tr.t;
  if (threadIdx.x < 8) {
    const int o = threadIdx.x, NS = P.NS;
    const u32 sn = pm_morton3((pm_compact3(Y >> 2) - (o & 1)) & (NS - 1), (pm_compact3(Y >> 1) - ((o >> 1) & 1)) & (NS - 1),
                              (pm_compact3(Y) - (o >> 2)) & (NS - 1));
    s_nb[o] = A.halo + P.halo_off + (long long)sn * P.hc;
  }
  __syncthreads();
  long long dsum = 0, smax = 0;
  switch (P.TS) {
    case 4: fixup_faces<4>(A, P, Y, s_nb, rho64, dsum, smax); break;
    case 8: fixup_faces<8>(A, P, Y, s_nb, rho64, dsum, smax); break;
    default: fixup_faces<16>(A, P, Y, s_nb, rho64, dsum, smax); break;
  }
  for (int d = 16; d > 0; d >>= 1) {
    dsum += __shfl_xor_sync(0xffffffffu, dsum, d);
    const long long om = __shfl_xor_sync(0xffffffffu, smax, d);
    smax = om > smax ? om : smax;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    s_red[warp] = dsum;
    s_max[warp] = smax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long ts = 0, tm = 0;
    for (int w = 0; w < FIX_THREADS / 32; ++w) {
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
__device__ __forceinline__ float kline(int i, int N, float kf) { return kf * (float)(i < N / 2 ? i : i - N); }

// Gradient operator in k-space: spectral -i k (the reference), or the transfer function of the
// 2-point / 4-point central differences.
__device__ __forceinline__ float grad_k(float k, float dx, int mode) {
  if (mode == 1) return sinf(k * dx) / dx;
  if (mode == 2) return (8.0f * sinf(k * dx) - sinf(2.0f * k * dx)) / (6.0f * dx);
  return k;
}

// Per-peak constants of the Green kernel, read once into registers.
struct GreenCtx {
  int N, log2N, Nh, gm;
  long long M;
  u32 nh_magic;
  int nh_shift;
  float kf, dx, sd2, s_c;
  const float2* spec;
  float2* out;
};

__device__ __forceinline__ double green_mode(const GreenCtx& g, long long m, float2 d) {
  const int N = g.N, Nh = g.Nh;
  // m = row * Nh + kz (m < N^2 Nh < 2^32 for N <= 1024): division by the invariant Nh.
  const u32 rest = pm_div_by((u32)m, g.nh_magic, g.nh_shift);
  const int kz = (int)((u32)m - rest * (u32)Nh);
  const int iy = (int)(rest & (N - 1)), ix = (int)(rest >> g.log2N);
  const float kx = kline(ix, N, g.kf), ky = kline(iy, N, g.kf), kzv = g.kf * (float)kz;
  const float k2 = kx * kx + ky * ky + kzv * kzv;
  const long long M = g.M;
  if (m == 0) {
    g.out[0] = g.out[M] = g.out[2 * M] = make_float2(0.f, 0.f);
    return 0.0;
  }
  float G = g.s_c / k2;
  if (g.sd2 > 0.f) G *= expf(-0.5f * k2 * g.sd2);
  const float gx = grad_k(kx, g.dx, g.gm) * G, gy = grad_k(ky, g.dx, g.gm) * G, gz = grad_k(kzv, g.dx, g.gm) * G;
  // -i k G d = (k G d.y, -k G d.x)
  float2 ox = make_float2(gx * d.y, -gx * d.x), oy = make_float2(gy * d.y, -gy * d.x),
         oz = make_float2(gz * d.y, -gz * d.x);
  if (kz == 0 || kz == N / 2) {
    const int px = (-ix) & (N - 1), py = (-iy) & (N - 1);
    const float2 dp = g.spec[((long long)px * N + py) * Nh + kz];
    const float hx = grad_k(kline(px, N, g.kf), g.dx, g.gm) * G, hy = grad_k(kline(py, N, g.kf), g.dx, g.gm) * G;
    // (v + conj(v_partner)) / 2 with v_partner = (h dp.y, -h dp.x)
    ox = make_float2(0.5f * (ox.x + hx * dp.y), 0.5f * (ox.y + hx * dp.x));
    oy = make_float2(0.5f * (oy.x + hy * dp.y), 0.5f * (oy.y + hy * dp.x));
    oz = make_float2(0.5f * (oz.x + gz * dp.y), 0.5f * (oz.y + gz * dp.x));
  }
  g.out[m] = ox;
  g.out[M + m] = oy;
  g.out[2 * M + m] = oz;
  // Potential-energy term: sum_x delta Phi = sum_k |delta_k|^2 G_k over the full spectrum; the
  // half spectrum counts each kz in (0, N/2) twice.
  // The term in FP32 (relative rounding ~1e-7, independent from mode to mode), summed in FP64.
  const float wk = (kz == 0 || kz == N / 2) ? 1.0f : 2.0f;
  return (double)(wk * G * (d.x * d.x + d.y * d.y));
}

// Grid: the Green blocks of the peaks in A.green_peak (those without the native transform).
__global__ void __launch_bounds__(PM_THREADS) k_green(StepArgs A) {
  __shared__ int s_pk;
  __shared__ long long s_lb;
  if (threadIdx.x == 0) {
    const int gi = pm_find(A.green_base, A.ngreen, (long long)blockIdx.x);
    s_pk = A.green_peak[gi];
    s_lb = (long long)blockIdx.x - A.green_base[gi];
  }
  __syncthreads();
  const int pk = s_pk;
  const long long lb = s_lb;  // block within the peak
  const PeakClock& C = A.clocks[pk];
  if (!C.has_delta) return;
  const PeakDesc& P = A.peaks[pk];
  GreenCtx g;
  g.N = P.N;
  g.log2N = P.log2N;
  g.Nh = P.N / 2 + 1;
  g.gm = P.gradient;
  g.M = P.nmodes;
  g.nh_magic = P.nh_magic;
  g.nh_shift = P.nh_shift;
  g.kf = (float)(kTwoPi / P.L);
  g.dx = (float)P.dx;
  g.sd2 = P.smooth > 0 ? (float)(P.smooth * P.dx) * (float)(P.smooth * P.dx) : 0.f;
  g.s_c = (float)(-1.5 * PM_H_I * PM_H_I / C.a_grid / ((double)P.N * P.N * P.N));
  g.spec = P.spec;
  g.out = P.gspec;
  const long long m0 = lb * (PM_THREADS * GREEN_MODES) + threadIdx.x;
  // All loads of the block's modes first (the stores below could alias them as far as the
  // compiler knows), then the arithmetic and the stores.
  float2 d[GREEN_MODES];
#pragma unroll
  for (int k = 0; k < GREEN_MODES; ++k) {
    const long long m = m0 + k * PM_THREADS;
    d[k] = m < g.M ? __ldg(g.spec + m) : make_float2(0.f, 0.f);
  }
  double w = 0.0;
#pragma unroll
  for (int k = 0; k < GREEN_MODES; ++k) {
    const long long m = m0 + k * PM_THREADS;
    if (m < g.M) w += green_mode(g, m, d[k]);
  }
  // Within a warp a plain FP64 tree (128 terms); one partial per warp, no block barrier; the
  // energy kernel merges the partials with the compensated sum.
  for (int dd = 16; dd > 0; dd >>= 1) w += __shfl_down_sync(0xffffffffu, w, dd);
  if ((threadIdx.x & 31) == 0) A.wpart[(P.mode_base + lb) * (PM_THREADS / 32) + (threadIdx.x >> 5)] = w;
}

__global__ void k_reset_peak(StepArgs A, int pk, double a0, int mode, double param, double a_end, int max_steps,
                             int set_thr, double delta_collapse, int stop) {
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
  c.sortstep = 0;
  c.refresh = 0;
  c.a_collapse = -1.0;
  c.stop_on_collapse = set_thr ? (stop ? 1 : 0) : 0;
  if (set_thr) c.delta_collapse = delta_collapse;
  if (mode == SCHED_RATIO) c.da = a0 * param;
  else if (mode == SCHED_FRAC) c.da = fmin(param * a0, a_end - a0);
  else c.da = 0.0;
  A.clocks[pk] = c;
  A.stats[pk].status = 0;
  A.stats[pk].nsamples = 0;
  A.sort_err[pk] = 0;
}

__global__ void k_release_peak(StepArgs A, int pk) {
  PeakClock c = A.clocks[pk];
  c.state = PS_IDLE;
  c.has_delta = 0;
  c.dep = 0;
  c.kpend = 0.0;
  A.clocks[pk] = c;
}

// Particles (n,3) float64 in lattice order -> split state + cell keys (pm3d.py:76-79 convention).
__global__ void k_set_particles(StepArgs A, int pk, PeakDesc P, const double* __restrict__ x,
                                const double* __restrict__ p) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
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
  // Loaded into the temporary state in lattice order; the priming step sorts it into place.
  A.tpos[g] = make_int4(cell, __float_as_int(ff[0]), __float_as_int(ff[1]), __float_as_int(ff[2]));
  A.tmom[g] = make_float4((float)p[3 * i], (float)p[3 * i + 1], (float)p[3 * i + 2], __int_as_float((int)i));
  A.keys_push[g] = pm_cell_key(ii[0], ii[1], ii[2]);
}

// Re-priming an existing state: copy it back to the loading area with its sort keys.
__global__ void k_reload(StepArgs A, PeakDesc P) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const long long g = P.p_off + i;
  const int4 ps = A.pos[g];
  A.tpos[g] = ps;
  A.tmom[g] = A.mom[g];
  const int N = P.N, l2 = P.log2N;
  A.keys_push[g] = pm_cell_key(ps.x >> (2 * l2), (ps.x >> l2) & (N - 1), ps.x & (N - 1));
}

// Current state -> float64 x, p (lattice order).  p includes the pending closing kick; acc
// (optional) receives -grad Phi at the particles evaluated for expansion factor a_acc.
__global__ void k_get_particles(StepArgs A, int pk, PeakDesc P, double* __restrict__ x, double* __restrict__ p,
                                double* __restrict__ acc, double a_acc) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const PeakClock C = A.clocks[pk];
  // A peak loaded but not yet primed still has its particles in the loading area.
  const bool loaded_only = C.state == PS_PRIME;
  const int4 ps = loaded_only ? A.tpos[P.p_off + i] : A.pos[P.p_off + i];
  const float4 m = loaded_only ? A.tmom[P.p_off + i] : A.mom[P.p_off + i];
  const int N = P.N;
  const int ii[3] = {ps.x >> (2 * P.log2N), (ps.x >> P.log2N) & (N - 1), ps.x & (N - 1)};
  const float f[3] = {__int_as_float(ps.y), __int_as_float(ps.z), __int_as_float(ps.w)};
  const long long id = (long long)__float_as_int(m.w);
  if (id < 0 || id >= P.n) {  // never write through an id that is not a lattice index
    atomicOr(&A.stats[pk].status, 8u);
    return;
  }
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

// CIC counts of arbitrary float64 positions (pm3d.py:81-89) without an engine: per particle the
// eight corner weights in 64-bit fixed point (38 fractional bits, the eighth corner taking the
// remainder, as in the engine's deposit) added with integer atomics, so the sums do not depend
// on the order; then k_fix_counts turns them into float64 counts.
__global__ void k_deposit64(const double* __restrict__ X, long long n, int N, double dx, u64* __restrict__ work) {
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
  const double one = (double)PM_FIX_ONE;
  const double Fx = f[0] * one, Gx = one - Fx, gy = 1.0 - f[1], gz = 1.0 - f[2];
  const double pl[4] = {Gx * gy, Gx * f[1], Fx * gy, Fx * f[1]};
  u64 w[8], sum = 0;
  for (int c = 0; c < 7; ++c) {
    w[c] = fix_round(pl[c >> 1], (c & 1) ? f[2] : gz);
    sum += w[c];
  }
  w[7] = PM_FIX_ONE - sum;
  for (int c = 0; c < 8; ++c) {
    const int cx = c >> 2, cy = (c >> 1) & 1, cz = c & 1;
    const long long o = ((cx ? i1[0] : i0[0]) * N + (cy ? i1[1] : i0[1])) * N + (cz ? i1[2] : i0[2]);
    atomicAdd((unsigned long long*)&work[o], (unsigned long long)w[c]);
  }
}

__global__ void k_fix_counts(const u64* __restrict__ work, long long n3, double* __restrict__ counts) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) counts[i] = (double)(long long)work[i] * (1.0 / (double)PM_FIX_ONE);
}

}  // namespace

// Dynamic shared memory of the largest super-tile in use (the smaller ones fit inside).
size_t pm_deposit_smem(int TSmax) { return sizeof(u32) * 2 * (size_t)patch_size(TSmax); }
size_t pm_push_smem(int TSmax) { return sizeof(float) * 3 * (size_t)patch_size(TSmax); }

size_t pm_tile_sort_smem() {
  return sizeof(u32) * 16 * 16 * 16 + (size_t)TSORT_CAP * (sizeof(int4) + sizeof(float4) + sizeof(u32) + sizeof(unsigned short));
}

int pm_kernels_init() {
  cudaError_t e = cudaFuncSetAttribute(k_push, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_deposit, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_tile_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pm_tile_sort_smem());
  return e == cudaSuccess ? 0 : -(int)e;
}

static unsigned nb(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// Grid of a grid-stride kernel: enough CTAs to fill every SM `per_sm` times, fewer for small n.
static unsigned stride_grid(long long n, int t, int per_sm) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      sms = 148;
  }
  const long long g = std::min<long long>((long long)nb(n, t), (long long)sms * per_sm);
  return (unsigned)std::max<long long>(g, 1);
}

void launch_push(const StepArgs& A, long long nst, size_t smem, cudaStream_t s) {
  k_push<<<(unsigned)nst, PUSH_THREADS, smem, s>>>(A);
}
void launch_advance(const StepArgs& A, cudaStream_t s) { k_advance<<<1, 256, 0, s>>>(A); }
void launch_energy(const StepArgs& A, cudaStream_t s) {
  k_energy<<<dim3(ENERGY_SLICES, A.npeaks), PM_THREADS, 0, s>>>(A);
}
void launch_permute(const StepArgs& A, long long ntot, cudaStream_t s) {
  k_permute<<<stride_grid(ntot, PM_THREADS, 8), PM_THREADS, 0, s>>>(A, ntot);
}
void launch_st_starts(const StepArgs& A, long long ntot, cudaStream_t s) {
  k_st_starts<<<stride_grid(ntot, PM_THREADS, 8), PM_THREADS, 0, s>>>(A, ntot);
}
void launch_tile_sort(const StepArgs& A, long long nst, cudaStream_t s) {
  k_tile_sort<<<stride_grid(nst, 1, 1), TSORT_THREADS, pm_tile_sort_smem(), s>>>(A, nst);
}
void launch_bin(const StepArgs& A, long long nst, cudaStream_t s) {
  k_bin_scan1<<<(unsigned)nst, BIN_CLASSES, 0, s>>>(A);
  k_bin_scan2<<<(unsigned)A.npeaks, 1024, 0, s>>>(A);
  k_bin_scatter<<<(unsigned)nst, PUSH_THREADS, 0, s>>>(A);
}
void launch_deposit(const StepArgs& A, long long nst, size_t smem, double* rho64, cudaStream_t s) {
  k_deposit<<<(unsigned)nst, DEP_THREADS, smem, s>>>(A, rho64);
}
void launch_fixup(const StepArgs& A, long long nst, double* rho64, cudaStream_t s) {
  k_fixup<<<(unsigned)nst, FIX_THREADS, 0, s>>>(A, rho64);
}
void launch_green(const StepArgs& A, long long nblocks, cudaStream_t s) {
  k_green<<<(unsigned)nblocks, PM_THREADS, 0, s>>>(A);
}
void launch_reset_peak(const StepArgs& A, int pk, double a0, int mode, double param, double a_end,
                       int max_steps, int set_thr, double delta_collapse, int stop, cudaStream_t s) {
  k_reset_peak<<<1, 1, 0, s>>>(A, pk, a0, mode, param, a_end, max_steps, set_thr, delta_collapse, stop);
}
void launch_release_peak(const StepArgs& A, int pk, cudaStream_t s) { k_release_peak<<<1, 1, 0, s>>>(A, pk); }
void launch_set_particles(const StepArgs& A, int pk, const PeakDesc& P, const double* x, const double* p,
                          cudaStream_t s) {
  k_set_particles<<<nb(P.n, PM_THREADS), PM_THREADS, 0, s>>>(A, pk, P, x, p);
}
void launch_reload(const StepArgs& A, const PeakDesc& P, cudaStream_t s) {
  k_reload<<<nb(P.n, PM_THREADS), PM_THREADS, 0, s>>>(A, P);
}
void launch_get_particles(const StepArgs& A, int pk, const PeakDesc& P, double* x, double* p, double* acc,
                          double a_acc, cudaStream_t s) {
  k_get_particles<<<nb(P.n, PM_THREADS), PM_THREADS, 0, s>>>(A, pk, P, x, p, acc, a_acc);
}
void launch_interp64(const double* F, const double* X, long long n, int N, double dx, double* out, cudaStream_t s) {
  k_interp64<<<nb(n, PM_THREADS), PM_THREADS, 0, s>>>(F, X, n, N, dx, out);
}
void launch_deposit64(const double* X, long long n, int N, double dx, u64* work, double* counts, cudaStream_t s) {
  const long long n3 = (long long)N * N * N;
  cudaMemsetAsync(work, 0, sizeof(u64) * (size_t)n3, s);
  if (n > 0) k_deposit64<<<nb(n, PM_THREADS), PM_THREADS, 0, s>>>(X, n, N, dx, work);
  k_fix_counts<<<nb(n3, PM_THREADS), PM_THREADS, 0, s>>>(work, n3, counts);
}
