// Step kernels of the pm3d engine: push (CIC gather + kicks + drift, each particle written into
// the bin of its new super-tile), clock advance, regrouping (bin layouts and relayouts, the
// priming radix-sort permutation, the optional per-super-tile re-sort), halo-exchange CIC
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


// Bin buffers, layouts and fills selected by a per-peak bit without indexing the
// kernel-parameter arrays dynamically (which would copy the parameter struct to local memory).
__device__ __forceinline__ int4* bpos(const StepArgs& A, int b) { return b ? A.pos1 : A.pos0; }
__device__ __forceinline__ float4* bmom(const StepArgs& A, int b) { return b ? A.mom1 : A.mom0; }
__device__ __forceinline__ BinLayout* blay(const StepArgs& A, int g) { return g ? A.lay[1] : A.lay[0]; }
__device__ __forceinline__ BinFill* bfill(const StepArgs& A, int b) { return b ? A.fill[1] : A.fill[0]; }

// The two runs of a filled bin: slots [b0, b0 + n0) (stayers) and [b1 + n0, b1 + n0 + n1)
// (arrivals), i.e. particle k < n0 + n1 of the bin sits at slot (k < n0 ? b0 : b1) + k.  The
// fill's counts are clamped into the bin, so a corrupted fill can never address outside it.
struct BinRuns {
  long long b0, b1;
  int n0, n1;
  __device__ __forceinline__ int total() const { return n0 + n1; }
  __device__ __forceinline__ long long slot(int k) const { return (k < n0 ? b0 : b1) + k; }
};
__device__ __forceinline__ BinRuns bin_runs(const BinLayout& L, const BinFill& F) {
  const u32 gap = min(F.gap, L.cap);
  const u32 stay = min(F.stay, gap);
  const u32 moved = min(F.moved, L.cap - gap);
  BinRuns r;
  r.b0 = L.base;
  r.n0 = (int)stay;
  r.b1 = (long long)L.base + gap - stay;
  r.n1 = (int)moved;
  return r;
}
// Particles in a bin: stayers plus the arrivals that found room.
__device__ __forceinline__ u32 bin_count(const BinLayout& L, const BinFill& F) {
  const u32 gap = min(F.gap, L.cap);
  return min(F.stay, gap) + min(F.moved, L.cap - gap);
}

// Locate the peak and the peak-local index of this CTA (uniform across the block).
struct TileRef {
  int pk;
  long long t;
};

__device__ __forceinline__ TileRef find_tile(const long long* base, const unsigned short* st_peak) {
  TileRef r;
  r.pk = st_peak[blockIdx.x];  // the same for every thread of the CTA
  r.t = (long long)blockIdx.x - base[r.pk];
  return r;
}

// ------------------------------------------------------------------------------------------
// Push: CIC gather of the three force grids (pm3d.py:91-99) fused with the pending closing
// kick of the previous step, the opening kick and the drift of this one (pm3d.py:122-127).
// One CTA per super-tile: the (TS+1)^3 node patch of all three grids is staged in shared
// memory, and the particles of the super-tile's bin read their 8 corners from there.  Each
// result goes straight into the bin of the super-tile it is now in, in the other buffer:
// stayers take ranks from a shared-memory counter (one add per warp), arrivals from an atomic on
// the destination's `moved` count, placed after the destination's count before the step (which
// no stayer rank reaches).  An arrival that finds no room, which the spare capacity makes rare,
// goes to the peak's overflow area and the peak relayouts this step.
struct PushCoef {
  float kA, kB, D, gscale;
  int run;
};

// Where one push CTA reads and writes.
struct PushCtx {
  int sx, sy, sz;        // this super-tile
  long long gS;          // its global index
  u32 base, cap;         // its bin
  const BinLayout* lay;  // bin layouts (global super-tile index)
  const BinFill* fcur;   // fills of the buffer read
  BinFill* fnxt;         // fills of the buffer written
  int4* opos;            // the buffer written
  float4* omom;
};

template <int T>
__device__ __forceinline__ void push_one(const StepArgs& A, const PeakDesc& P, int pk, const float* __restrict__ s_f,
                                         const PushCoef& K, const PushCtx& X, int4 ps, float4 m, u32* s_stay,
                                         bool& bad, bool& lost, double4& acc_e) {
  constexpr int RS = patch_rs(T), PS = patch_ps(T), CS = patch_size(T);
  const int N = P.N, l2 = P.log2N;
  const int ix = (ps.x >> (2 * l2)) & (N - 1), iy = (ps.x >> l2) & (N - 1), iz = ps.x & (N - 1);
  const int lx = ix - X.sx * T, ly = iy - X.sy * T, lz = iz - X.sz * T;
  // A particle outside this super-tile (bins and state disagree) is flagged and moved on
  // unchanged to the bin its cell names; nothing indexes outside the patch.
  const bool inside = ps.x >= 0 && ps.x < N * N * N && (unsigned)lx < (unsigned)T && (unsigned)ly < (unsigned)T &&
                      (unsigned)lz < (unsigned)T;
  bad |= !inside;
  float fx = __int_as_float(ps.y), fy = __int_as_float(ps.z), fz = __int_as_float(ps.w);
  float ax = 0.f, ay = 0.f, az = 0.f;
  if (inside) {
    const float gx = 1.0f - fx, gy = 1.0f - fy, gz = 1.0f - fz;
    const int o = lx * PS + ly * RS + lz;
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
  }
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
  const bool finite = isfinite(px) && isfinite(py) && isfinite(pz);
  if (K.run && finite && inside) {  // a non-finite particle stays where it is (the peak is flagged below)
    px += K.kB * ax;
    py += K.kB * ay;
    pz += K.kB * az;
#define PM_DRIFT(f, p, i)       \
  {                             \
    float fn = f + K.D * p;     \
    float c = floorf(fn);       \
    fn -= c;                    \
    if (fn >= 1.0f) {           \
      fn -= 1.0f;               \
      c += 1.0f;                \
    }                           \
    f = fn;                     \
    i = (i + (int)c) & (N - 1); \
  }
    PM_DRIFT(fx, px, nx)
    PM_DRIFT(fy, py, ny)
    PM_DRIFT(fz, pz, nz)
#undef PM_DRIFT
  }
  bad |= !(finite && isfinite(px) && isfinite(py) && isfinite(pz));
  const int cell = (nx << (2 * l2)) | (ny << l2) | nz;
  const int4 np = make_int4(cell, __float_as_int(fx), __float_as_int(fy), __float_as_int(fz));
  const float4 nm = make_float4(px, py, pz, m.w);
  const int tx = nx >> P.log2TS, ty = ny >> P.log2TS, tz = nz >> P.log2TS;
  const bool stay = tx == X.sx && ty == X.sy && tz == X.sz;
  const u32 sm = __ballot_sync(__activemask(), stay);
  long long dst = -1, gD = X.gS;
  if (stay) {
    const int leader = __ffs(sm) - 1;
    u32 r0 = 0;
    if ((int)(threadIdx.x & 31) == leader) r0 = atomicAdd(s_stay, (u32)__popc(sm));
    r0 = __shfl_sync(sm, r0, leader);
    const u32 r = r0 + (u32)__popc(sm & lanemask_lt());
    if (r < X.cap) dst = (long long)X.base + r;  // always: the stayers are at most the bin's count
  } else {
    gD = P.st_base + pm_morton3(tx, ty, tz);
    const BinLayout L = X.lay[gD];
    const u32 cnt = bin_count(L, X.fcur[gD]);
    const u32 r = atomicAdd(&X.fnxt[gD].moved, 1u);
    if (r < L.cap - cnt) dst = (long long)L.base + cnt + r;
  }
  if (dst >= 0) {
    X.opos[dst] = np;
    X.omom[dst] = nm;
  } else {
    const u32 o = atomicAdd(&A.ovf_n[pk], 1u);
    if (o < (u32)P.n) {
      A.lpos[P.p_off + o] = np;
      A.lmom[P.p_off + o] = nm;
      atomicAdd(&A.ovf_in[gD], 1u);
    } else {
      lost = true;  // more overflows than particles: the bins were corrupted
    }
  }
}

template <int T>
__device__ __forceinline__ void push_super(const StepArgs& A, const PeakDesc& P, const PeakClock& C, int pk, u32 st,
                                           float* s_f, u32* s_stay, const PushCoef& K) {
  constexpr int T1 = T + 1, RS = patch_rs(T), PS = patch_ps(T), CS = patch_size(T);
  constexpr int CH = T / 4 + 1;  // per patch row: T/4 copies of 16 bytes, then the (wrapped) last node
  const int N = P.N;
  PushCtx X;
  X.sx = pm_compact3(st >> 2);
  X.sy = pm_compact3(st >> 1);
  X.sz = pm_compact3(st);
  X.gS = P.st_base + st;
  X.lay = blay(A, C.lgen);
  X.fcur = bfill(A, C.sbuf);
  X.fnxt = bfill(A, C.sbuf ^ 1);
  X.opos = bpos(A, C.sbuf ^ 1);
  X.omom = bmom(A, C.sbuf ^ 1);
  const BinLayout L = X.lay[X.gS];
  X.base = L.base;
  X.cap = L.cap;
  const BinRuns R = bin_runs(L, X.fcur[X.gS]);
  const int n = R.total();
  const long long N3 = (long long)N * N * N;
  if (n > 0) {
    // Asynchronous copies of the patch rows (every row start is 16-byte aligned on both sides:
    // z0 = sz*T is a multiple of 4 and the grids are 256-byte aligned).
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(s_f);
    const int z0 = X.sz * T, zl = (X.sz * T + T) & (N - 1);
    // Thread t copies piece t % CH of patch rows t / CH, t / CH + RSTEP, ... (the row number
    // advanced incrementally: RSTEP rows are DX planes and DY rows further on).
    constexpr int NTH = PUSH_THREADS - PUSH_THREADS % CH, RSTEP = NTH / CH, DX = RSTEP / T1, DY = RSTEP % T1;
    if (threadIdx.x < NTH) {
      const int part = threadIdx.x % CH, r0 = threadIdx.x / CH;
      int comp = r0 / (T1 * T1), lx = (r0 / T1) % T1, ly = r0 % T1;
      for (int row = r0; row < 3 * T1 * T1; row += RSTEP) {
        const int gx = (X.sx * T + lx) & (N - 1), gy = (X.sy * T + ly) & (N - 1);
        const float* src = P.force + comp * N3 + ((long long)gx * N + gy) * N;
        const unsigned dst = sbase + 4u * (unsigned)(comp * CS + lx * PS + ly * RS + part * 4);
        if (part < T / 4) cp_async16(dst, src + z0 + part * 4);
        else cp_async4(dst, src + zl);
        ly += DY;
        if (ly >= T1) {
          ly -= T1;
          ++lx;
        }
        lx += DX;
        while (lx >= T1) {
          lx -= T1;
          ++comp;
        }
      }
    }
    cp_async_wait_all();
  }
  __syncthreads();
  bool bad = false, lost = false;
  double4 acc_e = make_double4(0.0, 0.0, 0.0, 0.0);  // this thread's momentum and p^2 sums
  // One particle per thread per sweep, the next two sweeps' particles in flight meanwhile;
  // 32-bit indices inside the bin's two runs: particle k sits at [k] in the first run, at
  // [k + d1] in the second.
  const int4* __restrict__ pp = bpos(A, C.sbuf) + R.b0;
  const float4* __restrict__ mp = bmom(A, C.sbuf) + R.b0;
  const int n0 = R.n0, d1 = (int)(R.b1 - R.b0);
  int k = threadIdx.x;
  int4 pa = make_int4(0, 0, 0, 0), pb = pa;
  float4 ma = make_float4(0.f, 0.f, 0.f, 0.f), mb = ma;
  if (k < n) {
    const int j = k < n0 ? k : k + d1;
    pa = pp[j];
    ma = mp[j];
  }
  if (k + PUSH_THREADS < n) {
    const int j = k + PUSH_THREADS < n0 ? k + PUSH_THREADS : k + PUSH_THREADS + d1;
    pb = pp[j];
    mb = mp[j];
  }
  for (; k < n; k += PUSH_THREADS) {
    const int4 p0 = pa;
    const float4 m0 = ma;
    pa = pb;
    ma = mb;
    const int k2 = k + 2 * PUSH_THREADS;
    if (k2 < n) {
      const int j = k2 < n0 ? k2 : k2 + d1;
      pb = pp[j];
      mb = mp[j];
    }
    push_one<T>(A, P, pk, s_f, K, X, p0, m0, s_stay, bad, lost, acc_e);
  }
  const bool any_bad = __syncthreads_or(bad), any_lost = __syncthreads_or(lost);
  if (threadIdx.x == 0) {
    if (any_bad) atomicOr(&A.stats[pk].status, 1u);
    if (any_lost) atomicOr(&A.stats[pk].status, 4u);
    // This bin's fill in the buffer written: its stayers, and where its arrivals start.
    X.fnxt[X.gS].stay = *s_stay;
    X.fnxt[X.gS].gap = (u32)n;
  }
  // Super-tile partials of the momentum and p^2 sums, in a fixed order: a plain FP64 tree over
  // the 32 lanes of a warp (about 5e-16 of the sum of magnitudes; compensating it cost 4 % of the
  // push), then compensated merges across the warps here and across super-tiles in k_energy.
  __shared__ CSum s_e[PUSH_THREADS / 32][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double4 ev = acc_e;
  const double ea[4] = {ev.x, ev.y, ev.z, ev.w};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double v = ea[q];
    for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
    if (lane == 0) s_e[warp][q] = CSum{v, 0.0};
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
  __shared__ u32 s_stay;
  const TileRef tr = find_tile(A.st_base, A.st_peak);
  const PeakClock C = A.clocks[tr.pk];
  if (C.state != PS_RUN && C.state != PS_FINALIZE) return;
  const PeakDesc P = A.peaks[tr.pk];
  if (threadIdx.x == 0) {
    const double a = C.a, da = C.da;
    const bool run = C.state == PS_RUN;
    const double amid = a + 0.5 * da;
    s_k.kA = (float)C.kpend;
    s_k.kB = run ? (float)(0.5 * da / (a * pm_hubble(a))) : 0.f;
    s_k.D = run ? (float)(da / (amid * amid * amid * pm_hubble(amid)) / P.dx) : 0.f;
    s_k.gscale = (float)(C.a_grid / a);
    s_k.run = run ? 1 : 0;
    s_stay = 0u;
  }
  __syncthreads();
  const PushCoef K = s_k;
  const u32 st = (u32)tr.t;
  switch (P.TS) {
    case 4: push_super<4>(A, P, C, tr.pk, st, s_f, &s_stay, K); break;
    case 8: push_super<8>(A, P, C, tr.pk, st, s_f, &s_stay, K); break;
    default: push_super<16>(A, P, C, tr.pk, st, s_f, &s_stay, K); break;
  }
}

// Clock advance (one thread per peak): applies the step that the push kernel just made,
// selects the next step size, whether this step primes by sort, relayouts (the push overflowed
// a bin) or re-sorts the super-tiles by cell, and which peaks re-deposit.  A running peak's
// particles are now in the other bin buffer; one that relayouts switches to a new layout
// generation, which the layout kernel fills in.
__global__ void k_advance(StepArgs A) {
  int any_sort = 0, any_layout = 0, any_refresh = 0;
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
    const bool pushed = c.state == PS_RUN || c.state == PS_FINALIZE;
    const int ovf = pushed && A.ovf_n[pk] != 0u ? 1 : 0;
    switch (c.state) {
      case PS_PRIME:
        dep = 1;
        c.sortstep = 1;
        c.relayout = 0;
        c.refresh = 0;
        c.lgen ^= 1;
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
        c.refresh = P.full_every > 0 && (c.nsteps % P.full_every) == 0 ? 1 : 0;
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
        dep = 1;
        c.state = PS_IDLE;
        break;
      default:
        break;
    }
    if (pushed) {  // the particles are now in the buffer the push wrote
      if (ovf) A.stats[pk].relayouts += 1u;
      c.relayout = ovf;
      c.sbuf ^= 1;
      if (ovf) c.lgen ^= 1;
    }
    c.dep = dep;
    A.clocks[pk] = c;
    A.sortseg[pk].active = dep && c.sortstep;
    any_sort |= dep && c.sortstep;
    any_layout |= dep && (c.sortstep || c.relayout);
    any_refresh |= dep && c.refresh;
    if (dep) {
      A.stats[pk].max_fix = 0;
      A.stats[pk].mass_defect = 0;
    }
  }
  any_sort = __syncthreads_or(any_sort);
  any_layout = __syncthreads_or(any_layout);
  any_refresh = __syncthreads_or(any_refresh);
  if (threadIdx.x == 0) {
    *A.sort_gate = any_sort ? 1u : 0u;
    *A.layout_gate = any_layout ? 1u : 0u;
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
// Priming (particles loaded into the loading area): the Morton-key radix sort, the super-tile
// starts in the sorted keys, the bin layout from the counts (k_layout), then the gather of the
// loading area into the bins of the current buffer in sorted order.  Grid-stride loops over a
// grid of a few CTAs per SM that return at once on the steps where no peak primes.
__global__ void k_st_starts(StepArgs A, long long ntot) {
  if (*A.sort_gate == 0u) return;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < ntot; j += (long long)gridDim.x * blockDim.x) {
    const int pk = pm_find(A.p_base, A.npeaks, j);
    const PeakClock C = A.clocks[pk];
    if (!(C.dep && C.sortstep)) continue;
    const PeakDesc P = A.peaks[pk];
    u32* ss = A.sstart + P.sst_off;
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

__global__ void k_permute(StepArgs A, long long ntot) {
  if (*A.sort_gate == 0u) return;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < ntot; j += (long long)gridDim.x * blockDim.x) {
    const int pk = pm_find(A.p_base, A.npeaks, j);
    const PeakClock C = A.clocks[pk];
    if (!(C.dep && C.sortstep)) continue;
    const PeakDesc& P = A.peaks[pk];
    const u32 q = A.perm[j];
    const u32 S = min(A.keys_sorted[j] >> P.st_shift, (u32)(P.nst - 1));
    const BinLayout L = blay(A, C.lgen)[P.st_base + S];
    const long long r = j - (long long)A.sstart[P.sst_off + S];
    // A failed sort (a value outside the peak, a rank outside the bin): never read or write outside.
    if ((long long)q < P.p_off || (long long)q >= P.p_off + P.n || r < 0 || r >= (long long)L.cap) {
      atomicOr(&A.stats[pk].status, 2u);
      continue;
    }
    bpos(A, C.sbuf)[L.base + r] = A.lpos[q];
    bmom(A, C.sbuf)[L.base + r] = A.lmom[q];
  }
}

// Bin layout of every peak that primes or relayouts this step (one CTA per peak).  The new count
// of each super-tile comes from the sorted keys when priming; else it is the bin the push filled
// plus its arrivals in the overflow area.  A bin's base capacity is count + count/8 +
// BIN_SLACK_MIN (the peak's bin_shift and bin_min), rounded up to BIN_ALIGN.  On a relayout a
// bin also asks for room for BIN_ARRIVALS times the arrivals of this step plus bin_grow steps
// of its net growth in this step (a bin that particles stream through needs room for its
// arrivals even when its count stays put), so that collapsing and infalling regions do not
// relayout every step.
//   Partial relayout (clock.relayout = 1): when the free space after the last bin of the peak's
// region holds, with their base capacity and wanted room, every overflowed bin and every bin
// whose remaining room is below another step of its arrivals, only those bins move there (in
// the buffer the push filled, which stays current); the others keep their place and their two
// runs.  The old places stay unused until the next full relayout.
//   Full relayout (clock.relayout = 2): every bin is laid out again from the start of the
// region, the wanted room shared out of the region's spare beyond the base capacities in
// proportion to the wants, and every particle is copied into the other buffer, which becomes
// current.  The region, n + n/8 + n/8 + (BIN_SLACK_MIN + BIN_ALIGN) nst slots, covers every base
// layout.
// The layout goes into generation clock.lgen (the advance kernel switched to it).  The relayout
// copies set the new fills; when priming, this kernel sets them to the counts, which the
// permutation then provides.
__global__ void __launch_bounds__(LAYOUT_THREADS) k_layout(StepArgs A) {
  __shared__ u32 s_w[LAYOUT_THREADS / 32];
  __shared__ unsigned long long s_r[4][LAYOUT_THREADS / 32];
  __shared__ long long s_carry;
  if (*A.layout_gate == 0u) return;
  const int pk = blockIdx.x;
  const PeakClock C = A.clocks[pk];
  if (!(C.dep && (C.sortstep || C.relayout))) return;
  const PeakDesc P = A.peaks[pk];
  const BinLayout* old = blay(A, C.lgen ^ 1) + P.st_base;
  BinLayout* lay = blay(A, C.lgen) + P.st_base;
  const BinFill* pushed = bfill(A, C.sbuf) + P.st_base;  // relayout: the buffer the push filled
  BinFill* cur = bfill(A, C.sbuf) + P.st_base;
  BinFill* nxt = bfill(A, C.sbuf ^ 1) + P.st_base;
  const u32* ss = A.sstart + P.sst_off;
  const u32* ovf_in = A.ovf_in + P.st_base;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // Count, base capacity and wanted extra capacity of bin i.
  auto bin = [&](int i, u32& cnt, u32& cap, u32& want) {
    want = 0u;
    u32 need = 0u;
    if (C.sortstep) {
      cnt = ss[i + 1] >= ss[i] ? ss[i + 1] - ss[i] : 0u;
    } else {
      const u32 prev = min(pushed[i].gap, old[i].cap);  // the bin's count before the push
      cnt = bin_count(old[i], pushed[i]) + ovf_in[i];
      const u32 grow = cnt > prev ? cnt - prev : 0u;
      const unsigned long long nd =
          (unsigned long long)pushed[i].moved * BIN_ARRIVALS + (unsigned long long)grow * (unsigned)P.bin_grow;
      need = (u32)min(nd, (unsigned long long)P.n);
    }
    cnt = min(cnt, (u32)P.n);
    cap = (cnt + (P.bin_shift < 32 ? cnt >> P.bin_shift : 0u) + (u32)P.bin_min + BIN_ALIGN - 1) & ~(u32)(BIN_ALIGN - 1);
    if (P.bin_grow > 0 && need > cap - cnt) want = need - (cap - cnt);
  };
  // Whether a partial relayout moves bin i (new count cnt): it overflowed, or (with spare capacity
  // in use) its remaining room is below another step of its arrivals, so that its neighbours'
  // overflows do not relayout the peak again in the next steps.
  auto moves = [&](int i, u32 cnt) -> bool {
    if (ovf_in[i]) return true;
    if (P.bin_grow == 0) return false;
    const u32 room = old[i].cap > cnt ? old[i].cap - cnt : 0u;
    return (unsigned long long)room < (unsigned long long)pushed[i].moved * BIN_ARRIVALS;
  };
  // Capacity of a bin moved by a partial relayout: base capacity plus its want.
  auto moved_cap = [&](u32 cap, u32 want) -> u32 {
    return (u32)min((unsigned long long)cap + want + BIN_ALIGN - 1, (unsigned long long)P.r_size) &
           ~(u32)(BIN_ALIGN - 1);
  };
  // Relayout: the base capacities' total, the total want, the space the overflowed bins need when
  // moved, and the end of the last bin of the current layout; then partial or full.
  bool partial = false;
  unsigned long long spare = 0, want_tot = 0, tail = 0;
  if (C.relayout) {
    unsigned long long sc = 0, sg = 0, sp = 0, mt = 0;
    for (int i = threadIdx.x; i < P.nst; i += LAYOUT_THREADS) {
      u32 cnt, cap, want;
      bin(i, cnt, cap, want);
      sc += cap;
      sg += want;
      if (moves(i, cnt)) sp += moved_cap(cap, want);
      const unsigned long long e = (unsigned long long)old[i].base + old[i].cap - (unsigned long long)P.r_off;
      mt = e > mt ? e : mt;
    }
    for (int d = 16; d > 0; d >>= 1) {
      sc += __shfl_xor_sync(0xffffffffu, sc, d);
      sg += __shfl_xor_sync(0xffffffffu, sg, d);
      sp += __shfl_xor_sync(0xffffffffu, sp, d);
      const unsigned long long o = __shfl_xor_sync(0xffffffffu, mt, d);
      mt = o > mt ? o : mt;
    }
    if (lane == 0) {
      s_r[0][warp] = sc;
      s_r[1][warp] = sg;
      s_r[2][warp] = sp;
      s_r[3][warp] = mt;
    }
    __syncthreads();
    sc = sg = sp = mt = 0;
    for (int w = 0; w < LAYOUT_THREADS / 32; ++w) {
      sc += s_r[0][w];
      sg += s_r[1][w];
      sp += s_r[2][w];
      mt = s_r[3][w] > mt ? s_r[3][w] : mt;
    }
    tail = mt;
    partial = tail + sp <= (unsigned long long)P.r_size;
    if (!partial && P.bin_grow > 0) {
      spare = (long long)sc < P.r_size ? (unsigned long long)(P.r_size - (long long)sc) : 0ull;
      want_tot = sg;
    }
  }
  if (threadIdx.x == 0) s_carry = partial ? (long long)tail : 0;
  __syncthreads();
  bool bad = false;
  for (int base = 0; base < P.nst; base += LAYOUT_THREADS) {
    const int i = base + threadIdx.x;
    u32 cnt = 0, cap = 0;
    if (i < P.nst) {
      u32 want;
      bin(i, cnt, cap, want);
      if (partial) {
        cap = moves(i, cnt) ? moved_cap(cap, want) : 0u;  // only the moved bins take new space
      } else if (want && want_tot) {  // the wanted extra, or its share of the spare
        const unsigned long long share = (unsigned long long)want * spare / want_tot;
        cap += (u32)(min(share, (unsigned long long)want) & ~(unsigned long long)(BIN_ALIGN - 1));
      }
    }
    u32 incl = cap;
    for (int d = 1; d < 32; d <<= 1) {
      const u32 t = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += t;
    }
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    u32 off = 0;
    for (int w = 0; w < warp; ++w) off += s_w[w];
    const long long carry = s_carry;
    if (i < P.nst) {
      if (partial && cap == 0u) {
        lay[i] = old[i];  // not overflowed: stays where it is
      } else {
        long long b = carry + off + incl - cap;  // bin start inside the peak's region
        if (b + cap > P.r_size) {                // counts above the particle total: never past the region
          bad = true;
          b = min(b, P.r_size);
          cap = (u32)(P.r_size - b);
          cnt = min(cnt, cap);
        }
        lay[i] = BinLayout{(u32)(P.r_off + b), cap};
      }
      if (C.sortstep) {
        cur[i] = BinFill{cnt, cnt, 0u, 0u};
        nxt[i] = BinFill{0u, 0u, 0u, 0u};
        A.ovf_in[P.st_base + i] = 0u;
      }
    }
    __syncthreads();
    if (threadIdx.x == LAYOUT_THREADS - 1) s_carry = carry + off + incl;
    __syncthreads();
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&A.stats[pk].status, 4u);
  if (threadIdx.x == 0) {
    if (C.sortstep) A.ovf_n[pk] = 0u;
    if (C.relayout) {
      A.clocks[pk].relayout = partial ? 1 : 2;
      if (!partial) {  // the full relayout fills the other buffer, which becomes current
        A.clocks[pk].sbuf = C.sbuf ^ 1;
        A.stats[pk].relayouts_full += 1u;
      }
    }
  }
}

// Relayout, per super-tile.  Full (clock.relayout = 2): every bin the push filled (old layout,
// other buffer) is copied in order to the start of its new bin in the current buffer.  Partial
// (1): only the bins that got a new place after the last bin move there, inside the current
// buffer.  Either way the bin's fill is then set to its new count,
// which includes the arrivals k_relayout_ovf places next.
__global__ void __launch_bounds__(PM_THREADS) k_relayout_copy(StepArgs A) {
  if (*A.layout_gate == 0u) return;
  const int pk = blockIdx.y;  // RELAYOUT_COPY_BLOCKS CTAs per peak, each looping over its bins
  const PeakClock C = A.clocks[pk];
  if (!(C.dep && C.relayout)) return;
  const bool full = C.relayout == 2;
  const int src = full ? (C.sbuf ^ 1) : C.sbuf;
  const long long st0 = A.st_base[pk], nst = A.st_base[pk + 1] - st0;
  for (long long t = blockIdx.x; t < nst; t += gridDim.x) {
    const long long g = st0 + t;
    const u32 arrivals = A.ovf_in[g];
    const BinLayout L0 = blay(A, C.lgen ^ 1)[g], L = blay(A, C.lgen)[g];
    if (!full && L.base == L0.base) continue;  // partial relayout: this bin stays as it is (uniform)
    const BinRuns R = bin_runs(L0, bfill(A, src)[g]);
    const int4* ip = bpos(A, src);
    const float4* im = bmom(A, src);
    int4* op = bpos(A, C.sbuf) + L.base;
    float4* om = bmom(A, C.sbuf) + L.base;
    const int n = min(R.total(), (int)L.cap);
    for (int k = threadIdx.x; k < n; k += PM_THREADS) {  // old and new places never overlap
      const long long j = R.slot(k);
      op[k] = ip[j];
      om[k] = im[j];
    }
    __syncthreads();  // every thread has read the old fill (a partial relayout rewrites that entry)
    if (threadIdx.x == 0) {
      const u32 cnt = min((u32)R.total() + arrivals, L.cap);
      bfill(A, C.sbuf)[g] = BinFill{cnt, cnt, 0u, 0u};
    }
  }
}

// Relayout: each particle of a relayouting peak's overflow area to the end of its new bin
// (ovf_in counts down to zero, one rank per particle).  RELAYOUT_OVF_BLOCKS CTAs per peak walk
// only that peak's overflow entries.
__global__ void __launch_bounds__(PM_THREADS) k_relayout_ovf(StepArgs A) {
  if (*A.layout_gate == 0u) return;
  const int pk = blockIdx.y;
  const PeakClock C = A.clocks[pk];
  if (!(C.dep && C.relayout)) return;
  const PeakDesc& P = A.peaks[pk];
  const long long novf = (long long)min(A.ovf_n[pk], (u32)P.n);
  for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < novf; o += (long long)gridDim.x * blockDim.x) {
    const long long j = P.p_off + o;
    const int4 ps = A.lpos[j];
    const int N = P.N, l2 = P.log2N, s = P.log2TS;
    const u32 S = pm_morton3(((ps.x >> (2 * l2)) & (N - 1)) >> s, ((ps.x >> l2) & (N - 1)) >> s, (ps.x & (N - 1)) >> s);
    const long long g = P.st_base + S;
    const BinLayout L = blay(A, C.lgen)[g];
    const u32 cnt = bfill(A, C.sbuf)[g].stay;  // the new count, arrivals from the overflow area included
    const u32 v = atomicSub(&A.ovf_in[g], 1u);
    if (v == 0u || v > cnt || cnt > L.cap) {  // counts that disagree: never write outside the bin
      atomicOr(&A.stats[pk].status, 4u);
      continue;
    }
    bpos(A, C.sbuf)[L.base + cnt - v] = ps;
    bmom(A, C.sbuf)[L.base + cnt - v] = A.lmom[j];
  }
}

// ------------------------------------------------------------------------------------------
// Refresh (optional, off by default): every full_every steps each super-tile's particles are
// re-sorted by cell (local
// Morton code of the cell inside the super-tile), so the deposit's and the push's warps see
// neighbouring cells and same-cell runs again, and the bin's two runs become one.  A counting
// sort per super-tile: the order inside one cell is not kept (nothing downstream depends on it;
// the deposit sums integers).  Up to TSORT_CAP particles the super-tile is staged in shared
// memory and written back to the start of its bin, coalesced (64 bytes of traffic per particle);
// denser super-tiles are copied to the same bin of the other buffer (free until the next push)
// and placed back from there.  Persistent grid (one CTA per SM) over the super-tiles; every
// launch returns at once when no peak refreshes this step.
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
  const long long g = P.st_base + st;
  const BinLayout L = blay(A, C.lgen)[g];
  BinFill* F = bfill(A, C.sbuf) + g;
  const BinRuns R = bin_runs(L, *F);
  const int n = R.total();
  int4* pos = bpos(A, C.sbuf);
  float4* mom = bmom(A, C.sbuf);
  int4* tpos = bpos(A, C.sbuf ^ 1);
  float4* tmom = bmom(A, C.sbuf ^ 1);
  const long long b = L.base;
  __syncthreads();  // every thread has read the fill before it is rewritten
  if (threadIdx.x == 0) *F = BinFill{(u32)n, (u32)n, 0u, 0u};  // one run from here on
  if (n < 2 && R.n0 == n) return;  // uniform: nothing to move
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
      const long long j = R.slot(i);
      const int4 p = pos[j];
      spos[i] = p;
      smom[i] = mom[j];
      const u32 c = cell_of(p.x);
      cr[i] = (c << 16) | atomicAdd(&hist[c], 1u);
    }
  } else {
    for (int i = threadIdx.x; i < n; i += TSORT_THREADS) {
      const long long j = R.slot(i);
      const int4 p = pos[j];
      tpos[b + i] = p;
      tmom[b + i] = mom[j];
      atomicAdd(&hist[cell_of(p.x)], 1u);
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
      pos[b + o] = spos[i];
      mom[b + o] = smom[i];
    }
  } else {
    // The copies in the other buffer are visible to the block after the barrier above; each
    // particle takes the next rank of its cell (order inside a cell arbitrary).
    for (int i = threadIdx.x; i < n; i += TSORT_THREADS) {
      const int4 p = tpos[b + i];
      const u32 o = atomicAdd(&hist[cell_of(p.x)], 1u);
      if (o < (u32)n) {
        pos[b + o] = p;
        mom[b + o] = tmom[b + i];
      }
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
  // Up to KF face nodes per thread, handled together so that their loads are in flight at once:
  // own partials, then each node's first neighbour (every face node has one), then the other
  // neighbours of edge and corner nodes.  Integer sums: the order does not change a bit.
  constexpr int KF = (FC + FIX_THREADS - 1) / FIX_THREADS;
  long long S[KF];
  int zm[KF], cx[KF], cy[KF], cz[KF];
#pragma unroll
  for (int k = 0; k < KF; ++k) {
    const int f = threadIdx.x + k * FIX_THREADS;
    zm[k] = 0;
    S[k] = 0;
    cx[k] = cy[k] = cz[k] = 0;
    if (f < FC) {
      face_coords<TS>(f, cx[k], cy[k], cz[k]);
      S[k] = __ldcg(face + f);
      zm[k] = (cx[k] == 0 ? 1 : 0) | (cy[k] == 0 ? 2 : 0) | (cz[k] == 0 ? 4 : 0);
    }
  }
#pragma unroll
  for (int k = 0; k < KF; ++k) {
    if (zm[k]) {
      const int o = zm[k] & -zm[k];
      S[k] += __ldcg(nb[o] + halo_index(cx[k] + TS * (o & 1), cy[k] + TS * ((o >> 1) & 1), cz[k] + TS * (o >> 2), TS));
    }
  }
#pragma unroll
  for (int k = 0; k < KF; ++k) {
    const int first = zm[k] & -zm[k];
    for (int o = zm[k]; o; o = (o - 1) & zm[k]) {  // the other non-empty subsets of zm[k]
      if (o == first) continue;
      S[k] += __ldcg(nb[o] + halo_index(cx[k] + TS * (o & 1), cy[k] + TS * ((o >> 1) & 1), cz[k] + TS * (o >> 2), TS));
    }
  }
#pragma unroll
  for (int k = 0; k < KF; ++k) {
    if (threadIdx.x + k * FIX_THREADS >= FC) continue;
    const long long Dv = S[k] - P.n_mean_fix;
    const long long node = ((long long)(sx * TS + cx[k]) * N + (sy * TS + cy[k])) * N + (sz * TS + cz[k]);
    P.delta[node] = (float)((double)Dv * P.inv_fix_nmean);
    if (rho64) rho64[node] = (double)S[k] * (1.0 / (double)PM_FIX_ONE);
    dsum += Dv;
    smax = S[k] > smax ? S[k] : smax;
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

template <int TS, int SB>
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
  const long long gst = P.st_base + st;
  const BinLayout L = blay(A, C.lgen)[gst];
  const BinRuns R = bin_runs(L, bfill(A, SB)[gst]);
  // A cell index belongs to this super-tile iff its bits outside the local ones equal the
  // super-tile's: one mask and one compare (negative or out-of-mesh values never match).
  const int local = ((TS - 1) << (2 * l2)) | ((TS - 1) << l2) | (TS - 1);
  const int tile_bits = ((sx * TS) << (2 * l2)) | ((sy * TS) << l2) | (sz * TS);
  __syncthreads();
  // Nodes' sums of the chunks folded so far, only for a super-tile of more than one chunk: kept
  // in the same bin of the other buffer (free until the next push; a bin of more than one chunk
  // of 16-byte entries holds the NN 8-byte sums several times over).
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
  // 32-bit indices inside the bin's two runs (fewer integer instructions and live registers than
  // 64-bit pointers): particle k sits at pp[k] in the first run, at pp[k + d1] in the second.
  const int4* __restrict__ pp = (SB ? A.pos1 : A.pos0) + R.b0;
  const int n = R.total(), n0 = R.n0, d1 = (int)(R.b1 - R.b0);
  u64* const fold = reinterpret_cast<u64*>((SB ? A.pos0 : A.pos1) + L.base);
  const int nit = (n + DEP_THREADS - 1) / DEP_THREADS;
  int k = threadIdx.x;
  constexpr int DEPTH = PM_DEP_DEPTH;
  int4 q[DEPTH];  // the particles of the next DEPTH sweeps, loads in flight
#pragma unroll
  for (int d = 0; d < DEPTH; ++d) {
    const int kk = k + d * DEP_THREADS;
    q[d] = kk < n ? pp[kk < n0 ? kk : kk + d1] : make_int4(-1, 0, 0, 0);
  }
  bool bad = false;
  int left = CH_IT;
  for (int it = 0; it < nit; ++it) {
    const int4 ps = q[0];
    const bool valid = k < n;
#pragma unroll
    for (int d = 0; d + 1 < DEPTH; ++d) q[d] = q[d + 1];
    const int kn = k + DEPTH * DEP_THREADS;
    if (kn < n) q[DEPTH - 1] = pp[kn < n0 ? kn : kn + d1];
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
      fold_chunk<TS>(fold, acc_hi, acc_lo, folded);
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
  }
}


__global__ void __launch_bounds__(DEP_THREADS, 4) k_deposit(StepArgs A, double* rho64) {
  extern __shared__ __align__(16) u32 s_dep[];
  const TileRef tr = find_tile(A.st_base, A.st_peak);
  const PeakClock C = A.clocks[tr.pk];
  if (!C.dep) return;
  const PeakDesc P = A.peaks[tr.pk];
  switch (P.TS) {
    // The bin buffer as a template argument: its pointers are then kernel parameters, not a
    // per-thread select (the particle loop is register-bound).
    case 4:
      if (C.sbuf) deposit_super<4, 1>(A, P, C, tr.pk, (u32)tr.t, s_dep, rho64);
      else deposit_super<4, 0>(A, P, C, tr.pk, (u32)tr.t, s_dep, rho64);
      break;
    case 8:
      if (C.sbuf) deposit_super<8, 1>(A, P, C, tr.pk, (u32)tr.t, s_dep, rho64);
      else deposit_super<8, 0>(A, P, C, tr.pk, (u32)tr.t, s_dep, rho64);
      break;
    default:
      if (C.sbuf) deposit_super<16, 1>(A, P, C, tr.pk, (u32)tr.t, s_dep, rho64);
      else deposit_super<16, 0>(A, P, C, tr.pk, (u32)tr.t, s_dep, rho64);
      break;
  }
}

// Face fix-up: one CTA per super-tile whose peak deposited this step.  Small and
// latency-bound, so many CTAs per SM.
__global__ void __launch_bounds__(FIX_THREADS) k_fixup(StepArgs A, double* rho64) {
  __shared__ long long s_red[FIX_THREADS / 32];
  __shared__ long long s_max[FIX_THREADS / 32];
  __shared__ const long long* s_nb[8];
  const TileRef tr = find_tile(A.st_base, A.st_peak);
  const PeakClock C = A.clocks[tr.pk];
  if (!C.dep) return;
  const PeakDesc P = A.peaks[tr.pk];
  const u32 Y = (u32)tr.t;
  if (threadIdx.x == 0) {
    // Ready for the next push, which fills the other buffer: no arrivals yet, overflow area
    // empty.  (Here rather than in the deposit, whose particle loop is register-bound.)
    bfill(A, C.sbuf ^ 1)[P.st_base + Y].moved = 0u;
    if (Y == 0) A.ovf_n[tr.pk] = 0u;
  }
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
  A.stats[pk].relayouts = 0;
  A.stats[pk].relayouts_full = 0;
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
  // Loaded into the loading area in lattice order; the priming step sorts it into bins.
  A.lpos[g] = make_int4(cell, __float_as_int(ff[0]), __float_as_int(ff[1]), __float_as_int(ff[2]));
  A.lmom[g] = make_float4((float)p[3 * i], (float)p[3 * i + 1], (float)p[3 * i + 2], __int_as_float((int)i));
  A.keys_push[g] = pm_cell_key(ii[0], ii[1], ii[2]);
}

// Re-priming an existing state: copy it back to the loading area with its sort keys.  One CTA
// per super-tile of the peak; places in the loading area from a per-peak counter (ovf_n, zeroed
// by the host before the launch; the priming step zeroes it again), one add per warp.
__global__ void __launch_bounds__(PM_THREADS) k_reload(StepArgs A, int pk, PeakDesc P) {
  const PeakClock C = A.clocks[pk];
  const long long g = P.st_base + blockIdx.x;
  const BinRuns R = bin_runs(blay(A, C.lgen)[g], bfill(A, C.sbuf)[g]);
  const int4* ip = bpos(A, C.sbuf);
  const float4* im = bmom(A, C.sbuf);
  const int N = P.N, l2 = P.log2N;
  const int n = R.total();
  for (int base = 0; base < n; base += PM_THREADS) {  // uniform trip count: the ballot sees whole warps
    const int k = base + threadIdx.x;
    const bool v = k < n;
    const u32 vm = __ballot_sync(0xffffffffu, v);
    u32 o0 = 0;
    if ((threadIdx.x & 31) == 0 && vm) o0 = atomicAdd(&A.ovf_n[pk], (u32)__popc(vm));
    o0 = __shfl_sync(0xffffffffu, o0, 0);
    if (!v) continue;
    const u32 o = o0 + (u32)__popc(vm & lanemask_lt());
    if (o >= (u32)P.n) {
      atomicOr(&A.stats[pk].status, 4u);
      continue;
    }
    const long long j = R.slot(k);
    const int4 ps = ip[j];
    A.lpos[P.p_off + o] = ps;
    A.lmom[P.p_off + o] = im[j];
    A.keys_push[P.p_off + o] = pm_cell_key((ps.x >> (2 * l2)) & (N - 1), (ps.x >> l2) & (N - 1), ps.x & (N - 1));
  }
}

// Current state -> float64 x, p (lattice order).  p includes the pending closing kick; acc
// (optional) receives -grad Phi at the particles evaluated for expansion factor a_acc.  One CTA
// per super-tile of the peak walks its bin; a peak loaded but not yet primed has its particles in
// the loading area instead, where CTA t takes the t-th slice.
__device__ __forceinline__ void get_one(const StepArgs& A, int pk, const PeakDesc& P, const PeakClock& C, int4 ps,
                                        float4 m, double* __restrict__ x, double* __restrict__ p,
                                        double* __restrict__ acc, double a_acc) {
  const int N = P.N;
  const int ii[3] = {(ps.x >> (2 * P.log2N)) & (N - 1), (ps.x >> P.log2N) & (N - 1), ps.x & (N - 1)};
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

__global__ void __launch_bounds__(PM_THREADS) k_get_particles(StepArgs A, int pk, PeakDesc P, double* __restrict__ x,
                                                              double* __restrict__ p, double* __restrict__ acc,
                                                              double a_acc) {
  const PeakClock C = A.clocks[pk];
  if (C.state == PS_PRIME) {
    const long long per = (P.n + P.nst - 1) / P.nst;
    const long long i0 = per * blockIdx.x, i1 = min(P.n, i0 + per);
    for (long long i = i0 + threadIdx.x; i < i1; i += PM_THREADS)
      get_one(A, pk, P, C, A.lpos[P.p_off + i], A.lmom[P.p_off + i], x, p, acc, a_acc);
    return;
  }
  const long long g = P.st_base + blockIdx.x;
  const BinRuns R = bin_runs(blay(A, C.lgen)[g], bfill(A, C.sbuf)[g]);
  const int4* ip = bpos(A, C.sbuf);
  const float4* im = bmom(A, C.sbuf);
  for (int k = threadIdx.x; k < R.total(); k += PM_THREADS) {
    const long long j = R.slot(k);
    get_one(A, pk, P, C, ip[j], im[j], x, p, acc, a_acc);
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
void launch_layout(const StepArgs& A, long long nst, long long ntot, cudaStream_t s) {
  k_layout<<<(unsigned)A.npeaks, LAYOUT_THREADS, 0, s>>>(A);
  k_relayout_copy<<<dim3(RELAYOUT_COPY_BLOCKS, (unsigned)A.npeaks), PM_THREADS, 0, s>>>(A);
  k_relayout_ovf<<<dim3(RELAYOUT_OVF_BLOCKS, (unsigned)A.npeaks), PM_THREADS, 0, s>>>(A);
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
void launch_reload(const StepArgs& A, int pk, const PeakDesc& P, cudaStream_t s) {
  cudaMemsetAsync(A.ovf_n + pk, 0, sizeof(u32), s);
  k_reload<<<(unsigned)P.nst, PM_THREADS, 0, s>>>(A, pk, P);
}
void launch_get_particles(const StepArgs& A, int pk, const PeakDesc& P, double* x, double* p, double* acc,
                          double a_acc, cudaStream_t s) {
  k_get_particles<<<(unsigned)P.nst, PM_THREADS, 0, s>>>(A, pk, P, x, p, acc, a_acc);
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
