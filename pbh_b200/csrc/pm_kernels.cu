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

// Buffer selection without indexing the kernel-parameter arrays dynamically (which would
// copy the whole parameter struct to local memory).
__device__ __forceinline__ int4* posb(const StepArgs& A, int b) { return b ? A.pos[1] : A.pos[0]; }
__device__ __forceinline__ float4* momb(const StepArgs& A, int b) { return b ? A.mom[1] : A.mom[0]; }

// Locate the peak and tile of this CTA (uniform across the block).
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

// ------------------------------------------------------------------------------------------
// Push: CIC gather of the three force grids (pm3d.py:91-99) fused with the pending closing
// kick of the previous step, the opening kick and the drift of this one (pm3d.py:122-127).
// One CTA per tile: the (T+1)^3 node patch of all three grids is staged in shared memory,
// then every particle whose CIC cell lies in the tile reads its 8 corners from there.
// Output is written in sorted order into the other state buffer, with the new cell key.
struct PushCoef {
  float kA, kB, D, gscale;
};

template <int T>
__device__ __forceinline__ void push_one(const PeakDesc& P, const float* __restrict__ s_f, const PushCoef& K,
                                         bool run, int tx, int ty, int tz, int4 ps, float4 m, long long j,
                                         int4* __restrict__ pout, float4* __restrict__ mout, u32* __restrict__ kout,
                                         bool& bad) {
  constexpr int T1 = T + 1, T13 = T1 * T1 * T1;
  const int N = P.N, l2 = P.log2N;
  const int ix = ps.x >> (2 * l2), iy = (ps.x >> l2) & (N - 1), iz = ps.x & (N - 1);
  const int lx = ix - tx * T, ly = iy - ty * T, lz = iz - tz * T;
  if ((unsigned)lx >= (unsigned)T || (unsigned)ly >= (unsigned)T || (unsigned)lz >= (unsigned)T) {
    bad = true;  // state and sort disagree: flag it, never index outside the patch
    return;
  }
  float fx = __int_as_float(ps.y), fy = __int_as_float(ps.z), fz = __int_as_float(ps.w);
  const float gx = 1.0f - fx, gy = 1.0f - fy, gz = 1.0f - fz;
  const int o = (lx * T1 + ly) * T1 + lz;
  float ax = 0.f, ay = 0.f, az = 0.f;
#define PM_CORNER(w, d)                       \
  {                                           \
    const float w_ = (w);                     \
    ax = fmaf(w_, s_f[o + (d)], ax);          \
    ay = fmaf(w_, s_f[T13 + o + (d)], ay);    \
    az = fmaf(w_, s_f[2 * T13 + o + (d)], az); \
  }
  const float w00 = gx * gy, w01 = gx * fy, w10 = fx * gy, w11 = fx * fy;
  PM_CORNER(w00 * gz, 0)
  PM_CORNER(w00 * fz, 1)
  PM_CORNER(w01 * gz, T1)
  PM_CORNER(w01 * fz, T1 + 1)
  PM_CORNER(w10 * gz, T1 * T1)
  PM_CORNER(w10 * fz, T1 * T1 + 1)
  PM_CORNER(w11 * gz, T1 * T1 + T1)
  PM_CORNER(w11 * fz, T1 * T1 + T1 + 1)
#undef PM_CORNER
  ax *= K.gscale;
  ay *= K.gscale;
  az *= K.gscale;
  float px = m.x + K.kA * ax, py = m.y + K.kA * ay, pz = m.z + K.kA * az;
  int nx = ix, ny = iy, nz = iz;
  if (run) {
    px += K.kB * ax;
    py += K.kB * ay;
    pz += K.kB * az;
#define PM_DRIFT(f, p, i)                 \
  {                                       \
    float fn = f + K.D * p;               \
    float c = floorf(fn);                 \
    fn -= c;                              \
    if (fn >= 1.0f) {                     \
      fn -= 1.0f;                         \
      c += 1.0f;                          \
    }                                     \
    f = fn;                               \
    i = (i + (int)c) & (N - 1);           \
  }
    PM_DRIFT(fx, px, nx)
    PM_DRIFT(fy, py, ny)
    PM_DRIFT(fz, pz, nz)
#undef PM_DRIFT
  }
  bad |= !(isfinite(px) && isfinite(py) && isfinite(pz));
  pout[j] = make_int4((nx << (2 * l2)) | (ny << l2) | nz, __float_as_int(fx), __float_as_int(fy), __float_as_int(fz));
  mout[j] = make_float4(px, py, pz, m.w);
  kout[j] = pm_cell_key(P, nx, ny, nz);
}

template <int T>
__device__ __forceinline__ void push_tile(const StepArgs& A, const PeakDesc& P, const PeakClock& C, int pk, u32 tc,
                                          long long b, long long e, float* s_f, const PushCoef& K) {
  constexpr int T1 = T + 1, T12 = T1 * T1, T13 = T1 * T1 * T1;
  const int N = P.N;
  const int tx = pm_compact3(tc >> 2), ty = pm_compact3(tc >> 1), tz = pm_compact3(tc);
  const long long N3 = (long long)N * N * N;
  for (int i = threadIdx.x; i < 3 * T13; i += PUSH_THREADS) {
    const int comp = i / T13, r = i - comp * T13;
    const int lx = r / T12, r2 = r - lx * T12;
    const int ly = r2 / T1, lz = r2 - ly * T1;
    const int gx = (tx * T + lx) & (N - 1), gy = (ty * T + ly) & (N - 1), gz = (tz * T + lz) & (N - 1);
    s_f[i] = __ldg(P.force + comp * N3 + ((long long)gx * N + gy) * N + gz);
  }
  __syncthreads();
  const bool run = C.state == PS_RUN;
  const int buf = C.buf;
  const int4* __restrict__ pin = posb(A, buf);
  const float4* __restrict__ min_ = momb(A, buf);
  int4* __restrict__ pout = posb(A, buf ^ 1);
  float4* __restrict__ mout = momb(A, buf ^ 1);
  u32* __restrict__ kout = A.keys_push;
  bool bad = false;
  // Two particles per thread per sweep, and the next sweep's pair is fetched before this one is
  // computed, so four gathers are in flight while the arithmetic runs.
  long long j = b + threadIdx.x;
  int4 p1n = make_int4(0, 0, 0, 0), p2n = p1n;
  float4 m1n = make_float4(0.f, 0.f, 0.f, 0.f), m2n = m1n;
  if (j < e) {
    const u32 q1 = A.perm[j];
    const u32 q2 = j + PUSH_THREADS < e ? A.perm[j + PUSH_THREADS] : q1;
    p1n = pin[q1];
    m1n = min_[q1];
    p2n = pin[q2];
    m2n = min_[q2];
  }
  for (; j < e; j += 2 * PUSH_THREADS) {
    const long long j2 = j + PUSH_THREADS;
    const bool has2 = j2 < e;
    const int4 p1 = p1n, p2 = p2n;
    const float4 m1 = m1n, m2 = m2n;
    const long long jn = j + 2 * PUSH_THREADS;
    if (jn < e) {
      const u32 q1 = A.perm[jn];
      const u32 q2 = jn + PUSH_THREADS < e ? A.perm[jn + PUSH_THREADS] : q1;
      p1n = pin[q1];
      m1n = min_[q1];
      p2n = pin[q2];
      m2n = min_[q2];
    }
    push_one<T>(P, s_f, K, run, tx, ty, tz, p1, m1, j, pout, mout, kout, bad);
    if (has2) push_one<T>(P, s_f, K, run, tx, ty, tz, p2, m2, j2, pout, mout, kout, bad);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&A.stats[pk].status, 1u);
}

// One CTA per push super-tile of TP^3 cells: its (TP/T)^3 bucket tiles are consecutive Morton
// codes, so its particles are one contiguous range of the sorted order.
__global__ void __launch_bounds__(PUSH_THREADS, 2) k_push(StepArgs A) {
  extern __shared__ float s_f[];
  __shared__ PushCoef s_k;
  const TileRef tr = find_tile(A.ptile_base, A.npeaks);
  const PeakClock C = A.clocks[tr.pk];
  if (C.state != PS_RUN && C.state != PS_FINALIZE) return;
  const PeakDesc& P = A.peaks[tr.pk];
  const u32 st = (u32)tr.t;
  const u32 R = 1u << (3 * (P.log2TP - P.log2T));
  const u32* bs = A.bstart + P.bucket_off;
  const long long b = bs[st * R * 8], e = bs[(st + 1) * R * 8];
  if (b == e) return;
  if (threadIdx.x == 0) {
    const double a = C.a, da = C.da;
    const bool run = C.state == PS_RUN;
    const double amid = a + 0.5 * da;
    s_k.kA = (float)C.kpend;
    s_k.kB = run ? (float)(0.5 * da / (a * pm_hubble(a))) : 0.f;
    s_k.D = run ? (float)(da / (amid * amid * amid * pm_hubble(amid)) / P.dx) : 0.f;
    s_k.gscale = (float)(C.a_grid / a);
  }
  __syncthreads();
  const PushCoef K = s_k;
  switch (P.TP) {
    case 4: push_tile<4>(A, P, C, tr.pk, st, b, e, s_f, K); break;
    case 8: push_tile<8>(A, P, C, tr.pk, st, b, e, s_f, K); break;
    default: push_tile<16>(A, P, C, tr.pk, st, b, e, s_f, K); break;
  }
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
      if (dmax >= c.delta_collapse) {
        c.a_collapse = c.a;
        if (c.stop_on_collapse && c.state == PS_RUN) c.state = PS_FINALIZE;
      }
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
    A.sortseg_full[pk].active = dep;
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
  const int b = (int)(A.keys_sorted[j] >> P.local_bits);
  const int bprev = j == P.p_off ? -1 : (int)(A.keys_sorted[j - 1] >> P.local_bits);
  for (int bb = bprev + 1; bb <= b; ++bb) bs[bb] = (u32)j;
  if (j == P.p_off + P.n - 1)
    for (int bb = b + 1; bb <= P.nb; ++bb) bs[bb] = (u32)(P.p_off + P.n);
}

// ------------------------------------------------------------------------------------------
// Deterministic CIC deposit (pm3d.py:81-89, 103-104).  One CTA owns the TS^3 nodes of one push
// super-tile (TS = 16: 8 bucket tiles of 8^3).  It reads the super-tile's own particles (one
// contiguous sorted range) and, from the 7 lower neighbour super-tiles, only the buckets of
// their boundary-layer cells whose corners reach into it.  Per particle the 8 CIC weights are
// formed in 64-bit fixed point with 40 fractional bits, the 8th corner taking the remainder so
// each particle deposits exactly 2^40; consecutive particles of one cell are first combined by
// a warp-shuffle segmented scan.  Each node accumulates in shared memory as two native 32-bit
// words (the signed weight's bits >= 20 and its low 20 bits), which cannot overflow within a
// chunk of fewer than 2048 particles, and is folded into a 64-bit register accumulator after
// every chunk.
// Integer sums make the result independent of particle order, bit for bit; no global atomics.
// Every node is written once as FP32 delta = S/n_mean - 1.
template <int TS>
__device__ __forceinline__ void deposit_super(const StepArgs& A, const PeakDesc& P, int pk, u32 st, u32* smem,
                                              double* rho64) {
  constexpr int TS3 = TS * TS * TS;
  constexpr int NPT = (TS3 + DEP_THREADS - 1) / DEP_THREADS;  // nodes per thread
  constexpr int NCAND = 7 * 64;                                // (neighbour o, sub-tile, mask) candidates
  u32* acc_hi = smem;
  u32* acc_lo = smem + TS3;
  __shared__ long long s_rb[72], s_rp[73];
  __shared__ int s_ro[72];
  __shared__ int s_nr;
  __shared__ u32 s_wc[DEP_THREADS / 32];
  __shared__ long long s_red[DEP_THREADS / 32];
  __shared__ long long s_max[DEP_THREADS / 32];
  const int N = P.N, l2 = P.log2N;
  const int rb = P.log2TP - P.log2T;      // log2 of sub-tiles per axis: 0 or 1
  const int RS = 1 << (3 * rb);           // sub-tiles per super-tile: 1 or 8
  const int NS = N / TS;                  // super-tiles per axis
  const int sx = pm_compact3(st >> 2), sy = pm_compact3(st >> 1), sz = pm_compact3(st);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const u32* bs = A.bstart + P.bucket_off;
  for (int i = threadIdx.x; i < 2 * TS3; i += DEP_THREADS) smem[i] = 0u;
  // Range table: candidate k = (o - 1) * 64 + s * 8 + m over sub-tiles s of the neighbour
  // super-tile at offset -o that touch this one, and masks m covering o.
  long long cb = 0, ce = 0;
  bool use = false;
  int co = 0;
  if (threadIdx.x < NCAND) {
    const int o = threadIdx.x / 64 + 1, s = (threadIdx.x >> 3) & 7, m = threadIdx.x & 7;
    if (s < RS && (m & o) == o) {
      const int sxl = pm_compact3((u32)s >> 2), syl = pm_compact3((u32)s >> 1), szl = pm_compact3((u32)s);
      const int last = (1 << rb) - 1;
      if ((!(o & 1) || sxl == last) && (!(o & 2) || syl == last) && (!(o & 4) || szl == last)) {
        const u32 nx = (sx - (o & 1)) & (NS - 1), ny = (sy - ((o >> 1) & 1)) & (NS - 1), nz = (sz - ((o >> 2) & 1)) & (NS - 1);
        const u32 b = (pm_morton3(nx, ny, nz) * (u32)RS + (u32)s) * 8 + m;
        cb = bs[b];
        ce = bs[b + 1];
        use = ce > cb;
        co = o;
      }
    }
  }
  // Compact the non-empty candidates (block-wide ballot prefix) behind the own range.
  const u32 bal = __ballot_sync(0xffffffffu, use);
  if (lane == 0) s_wc[warp] = __popc(bal);
  __syncthreads();
  if (threadIdx.x == 0) {
    u32 run = 1;
    for (int w = 0; w < DEP_THREADS / 32; ++w) {
      const u32 c = s_wc[w];
      s_wc[w] = run;
      run += c;
    }
    s_nr = (int)run;
    s_rb[0] = bs[st * RS * 8];
    s_rp[0] = bs[(st + 1) * RS * 8] - s_rb[0];  // length for now
    s_ro[0] = 0;
  }
  __syncthreads();
  if (use) {
    const int slot = s_wc[warp] + __popc(bal & ((1u << lane) - 1u));
    s_rb[slot] = cb;
    s_rp[slot] = ce - cb;
    s_ro[slot] = co;
  }
  __syncthreads();
  const int nr = s_nr;
  if (warp == 0) {  // lengths -> exclusive prefix (nr <= 72)
    long long carry = 0;
    for (int base = 0; base < nr; base += 32) {
      const int i = base + lane;
      const long long len = i < nr ? s_rp[i] : 0;
      long long incl = len;
      for (int d = 1; d < 32; d <<= 1) {
        const long long v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += v;
      }
      if (i < nr) s_rp[i] = carry + incl - len;
      carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) s_rp[nr] = carry;
  }
  __syncthreads();
  const long long total = s_rp[nr];
  const int4* __restrict__ pos = posb(A, A.clocks[pk].buf);
  const u32 le = lanemask_le();
  u64 acc[NPT];
#pragma unroll
  for (int k = 0; k < NPT; ++k) acc[k] = 0ull;
  // A node takes at most one contribution per particle of a chunk.  With CHUNK < 2^11 the high
  // words (each at most 2^20, or -1 for a remainder corner a few units below zero) sum inside
  // int32 and the low words (each < 2^20) inside uint32, so both are exact.
  constexpr int CH_IT = 3;  // sweeps of DEP_THREADS particles per chunk: CHUNK = 1536
  static_assert(CH_IT * DEP_THREADS < 2048, "chunk too large for the split accumulators");
  const long long nit = (total + DEP_THREADS - 1) / DEP_THREADS;
  // Flat particle index k over the concatenated ranges; the range index only moves forward.
  long long k = warp * 32 + lane;
  int r = 0;
  bool v_n = k < total;
  int4 ps_n = make_int4(-1, 0, 0, 0);
  int o_n = 0;
  if (v_n) {
    while (r + 1 < nr && s_rp[r + 1] <= k) ++r;
    ps_n = pos[A.perm[s_rb[r] + (k - s_rp[r])]];
    o_n = s_ro[r];
  }
  for (long long it = 0; it < nit; ++it) {
    const int4 ps = ps_n;
    const bool valid = v_n;
    const int o = o_n;
    // Prefetch the next sweep's particle before working on this one.
    k += DEP_THREADS;
    v_n = k < total;
    if (v_n) {
      while (r + 1 < nr && s_rp[r + 1] <= k) ++r;
      ps_n = pos[A.perm[s_rb[r] + (k - s_rp[r])]];
      o_n = s_ro[r];
    }
    {
      const int ix = ps.x >> (2 * l2), iy = (ps.x >> l2) & (N - 1), iz = ps.x & (N - 1);
      const int lx = (o & 1) ? -1 : ix - sx * TS;
      const int ly = (o & 2) ? -1 : iy - sy * TS;
      const int lz = (o & 4) ? -1 : iz - sz * TS;
      const double fx = __int_as_float(ps.y), fy = __int_as_float(ps.z), fz = __int_as_float(ps.w);
      const double gx = 1.0 - fx, gy = 1.0 - fy, gz = 1.0 - fz;
      const double one = (double)PM_FIX_ONE;
      const double w00 = gx * gy * one, w01 = gx * fy * one, w10 = fx * gy * one, w11 = fx * fy * one;
      u64 W0 = 0, W1 = 0, W2 = 0, W3 = 0, W4 = 0, W5 = 0, W6 = 0, W7 = 0;
      if (valid) {
        W0 = (u64)__double2ll_rn(w00 * gz);
        W1 = (u64)__double2ll_rn(w00 * fz);
        W2 = (u64)__double2ll_rn(w01 * gz);
        W3 = (u64)__double2ll_rn(w01 * fz);
        W4 = (u64)__double2ll_rn(w10 * gz);
        W5 = (u64)__double2ll_rn(w10 * fz);
        W6 = (u64)__double2ll_rn(w11 * gz);
        W7 = PM_FIX_ONE - (W0 + W1 + W2 + W3 + W4 + W5 + W6);
      }
      // Warp-shuffle segmented scan over runs of the same cell (a cell lies in one bucket, so
      // equal cells also share the range and its neighbour offset o).
      const int key = valid ? ps.x : -1 - lane;
      const int prev = __shfl_up_sync(0xffffffffu, key, 1);
      const bool head = lane == 0 || prev != key;
      const u32 heads = __ballot_sync(0xffffffffu, head);
      bool tail = true;
      if (heads != 0xffffffffu) {
        const int sstart = 31 - __clz(heads & le);
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const bool take = lane - d >= sstart;
#define PM_SEG(W)                              \
  {                                            \
    const u64 v_ = shfl_up_u64(W, d);          \
    if (take) W += v_;                         \
  }
          PM_SEG(W0) PM_SEG(W1) PM_SEG(W2) PM_SEG(W3) PM_SEG(W4) PM_SEG(W5) PM_SEG(W6) PM_SEG(W7)
#undef PM_SEG
        }
        tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
      }
      if (valid && tail) {
        const bool x0 = (unsigned)lx < (unsigned)TS, x1 = (unsigned)(lx + 1) < (unsigned)TS;
        const bool y0 = (unsigned)ly < (unsigned)TS, y1 = (unsigned)(ly + 1) < (unsigned)TS;
        const bool z0 = (unsigned)lz < (unsigned)TS, z1 = (unsigned)(lz + 1) < (unsigned)TS;
        const int nb = (lx * TS + ly) * TS + lz;
#define PM_ADD(cond, off, W)                                                  \
  if (cond) {                                                                 \
    atomicAdd(&acc_hi[nb + (off)], (u32)(int)((long long)(W) >> 20));        \
    atomicAdd(&acc_lo[nb + (off)], (u32)((W) & 0xFFFFFu));                   \
  }
        PM_ADD(x0 && y0 && z0, 0, W0)
        PM_ADD(x0 && y0 && z1, 1, W1)
        PM_ADD(x0 && y1 && z0, TS, W2)
        PM_ADD(x0 && y1 && z1, TS + 1, W3)
        PM_ADD(x1 && y0 && z0, TS * TS, W4)
        PM_ADD(x1 && y0 && z1, TS * TS + 1, W5)
        PM_ADD(x1 && y1 && z0, TS * TS + TS, W6)
        PM_ADD(x1 && y1 && z1, TS * TS + TS + 1, W7)
#undef PM_ADD
      }
    }
    if ((it + 1) % CH_IT == 0 || it + 1 == nit) {
      __syncthreads();
#pragma unroll
      for (int q = 0; q < NPT; ++q) {
        const int node = threadIdx.x + q * DEP_THREADS;
        if (node < TS3) {
          acc[q] += (u64)((long long)(int)acc_hi[node] * (1LL << 20)) + (u64)acc_lo[node];
          acc_hi[node] = 0u;
          acc_lo[node] = 0u;
        }
      }
      __syncthreads();
    }
  }
  long long dsum = 0, smax = 0;
  const long long base = ((long long)sx * TS * N + (long long)sy * TS) * N + sz * TS;
#pragma unroll
  for (int k = 0; k < NPT; ++k) {
    const int node = threadIdx.x + k * DEP_THREADS;
    if (node < TS3) {
      const int nz = node & (TS - 1), ny = (node / TS) & (TS - 1), nx = node / (TS * TS);
      const long long S = (long long)acc[k];
      const long long Dv = S - P.n_mean_fix;
      const long long g = base + ((long long)nx * N + ny) * N + nz;
      P.delta[g] = (float)((double)Dv * P.inv_fix_nmean);
      if (rho64) rho64[g] = (double)S * (1.0 / (double)PM_FIX_ONE);
      dsum += Dv;
      smax = S > smax ? S : smax;
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

__global__ void __launch_bounds__(DEP_THREADS) k_deposit(StepArgs A, double* rho64) {
  extern __shared__ __align__(16) u32 s_dep[];
  const TileRef tr = find_tile(A.ptile_base, A.npeaks);
  if (!A.clocks[tr.pk].dep) return;
  const PeakDesc& P = A.peaks[tr.pk];
  switch (P.TP) {
    case 4: deposit_super<4>(A, P, tr.pk, (u32)tr.t, s_dep, rho64); break;
    case 8: deposit_super<8>(A, P, tr.pk, (u32)tr.t, s_dep, rho64); break;
    default: deposit_super<16>(A, P, tr.pk, (u32)tr.t, s_dep, rho64); break;
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

__global__ void __launch_bounds__(PM_THREADS) k_green(StepArgs A) {
  __shared__ int s_pk;
  __shared__ float s_c;
  if (threadIdx.x == 0) {
    s_pk = pm_find(A.mode_base, A.npeaks, (long long)blockIdx.x);
    const PeakDesc& P = A.peaks[s_pk];
    const double n3 = (double)P.N * P.N * P.N;
    s_c = (float)(-1.5 * PM_H_I * PM_H_I / A.clocks[s_pk].a_grid / n3);
  }
  __syncthreads();
  const int pk = s_pk;
  if (!A.clocks[pk].has_delta) return;
  const PeakDesc& P = A.peaks[pk];
  const long long m = ((long long)blockIdx.x - A.mode_base[pk]) * PM_THREADS + threadIdx.x;
  if (m >= P.nmodes) return;
  const int N = P.N, Nh = N / 2 + 1;
  // m = row * Nh + kz without an integer division: the double quotient is off by at most one.
  long long rest = (long long)((double)m * P.inv_nh);
  if (rest * Nh > m) --rest;
  else if ((rest + 1) * Nh <= m) ++rest;
  const int kz = (int)(m - rest * Nh);
  const int iy = (int)(rest & (N - 1)), ix = (int)(rest >> P.log2N);
  const float kf = (float)(kTwoPi / P.L), dx = (float)P.dx;
  const float kx = kline(ix, N, kf), ky = kline(iy, N, kf), kzv = kf * (float)kz;
  const float k2 = kx * kx + ky * ky + kzv * kzv;
  const long long M = P.nmodes;
  float2* out = P.gspec;
  if (m == 0) {
    out[0] = out[M] = out[2 * M] = make_float2(0.f, 0.f);
    return;
  }
  float G = s_c / k2;
  if (P.smooth > 0) {
    const float sd = (float)(P.smooth * P.dx);
    G *= expf(-0.5f * k2 * sd * sd);
  }
  const int gm = P.gradient;
  const float gx = grad_k(kx, dx, gm) * G, gy = grad_k(ky, dx, gm) * G, gz = grad_k(kzv, dx, gm) * G;
  const float2 d = P.spec[m];
  // -i k G d = (k G d.y, -k G d.x)
  float2 ox = make_float2(gx * d.y, -gx * d.x), oy = make_float2(gy * d.y, -gy * d.x),
         oz = make_float2(gz * d.y, -gz * d.x);
  if (kz == 0 || kz == N / 2) {
    const int px = (-ix) & (N - 1), py = (-iy) & (N - 1);
    const float2 dp = P.spec[((long long)px * N + py) * Nh + kz];
    const float hx = grad_k(kline(px, N, kf), dx, gm) * G, hy = grad_k(kline(py, N, kf), dx, gm) * G;
    // (v + conj(v_partner)) / 2 with v_partner = (h dp.y, -h dp.x)
    ox = make_float2(0.5f * (ox.x + hx * dp.y), 0.5f * (ox.y + hx * dp.x));
    oy = make_float2(0.5f * (oy.x + hy * dp.y), 0.5f * (oy.y + hy * dp.x));
    oz = make_float2(0.5f * (oz.x + gz * dp.y), 0.5f * (oz.y + gz * dp.x));
  }
  out[m] = ox;
  out[M + m] = oy;
  out[2 * M + m] = oz;
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
  c.stop_on_collapse = 0;
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
  posb(A, buf)[g] = make_int4(cell, __float_as_int(ff[0]), __float_as_int(ff[1]), __float_as_int(ff[2]));
  momb(A, buf)[g] = make_float4((float)p[3 * i], (float)p[3 * i + 1], (float)p[3 * i + 2], __int_as_float((int)i));
  A.keys_push[g] = pm_cell_key(P, ii[0], ii[1], ii[2]);
}

// Current state -> float64 x, p (lattice order).  p includes the pending closing kick; acc
// (optional) receives -grad Phi at the particles evaluated for expansion factor a_acc.
__global__ void k_get_particles(StepArgs A, int pk, PeakDesc P, double* __restrict__ x, double* __restrict__ p,
                                double* __restrict__ acc, double a_acc) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const PeakClock C = A.clocks[pk];
  const int4 ps = posb(A, C.buf)[P.p_off + i];
  const float4 m = momb(A, C.buf)[P.p_off + i];
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

size_t pm_deposit_smem(int TPmax) { return sizeof(u32) * 2 * (size_t)TPmax * TPmax * TPmax; }
size_t pm_push_smem(int TPmax) { return sizeof(float) * 3 * (size_t)(TPmax + 1) * (TPmax + 1) * (TPmax + 1); }

int pm_kernels_init() {
  cudaError_t e = cudaFuncSetAttribute(k_push, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_deposit, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  return e == cudaSuccess ? 0 : -(int)e;
}

void launch_push(const StepArgs& A, long long nptiles, size_t smem, cudaStream_t s) {
  k_push<<<(unsigned)nptiles, PUSH_THREADS, smem, s>>>(A);
}
void launch_advance(const StepArgs& A, cudaStream_t s) { k_advance<<<1, 256, 0, s>>>(A); }
void launch_bucket_starts(const StepArgs& A, long long ntot, cudaStream_t s) {
  k_bucket_starts<<<(unsigned)((ntot + PM_THREADS - 1) / PM_THREADS), PM_THREADS, 0, s>>>(A, ntot);
}
void launch_deposit(const StepArgs& A, long long nptiles, size_t smem, double* rho64, cudaStream_t s) {
  k_deposit<<<(unsigned)nptiles, DEP_THREADS, smem, s>>>(A, rho64);
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
