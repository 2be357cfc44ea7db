// Shared definitions for the pm3d B200 engine (sm_100a).
//
// Particle state (one 16-byte vector each, so every access is a 128-bit load/store):
//   pos  = int4 {cell, f_x, f_y, f_z}: `cell` is the linear index (ix*N + iy)*N + iz of the
//          lower of the two mesh nodes bracketing the particle on each axis (mesh node i sits
//          at (i + 1/2) dx, pbhgr/pbhgr/pm3d.py:76-79), and f_* in [0, 1) is the FP32 offset
//          from that node in node units.  X = ((i + f + 1/2) dx) mod L.  CIC weights are then
//          (1 - f, f) with no branch (pm3d.py:83-88).
//   mom  = float4 {p_x, p_y, p_z, id}: canonical momentum p = a^2 dx/dt (pm3d.py:4) and the
//          particle's lattice index (the row of PM3D.x) stored as int bits.
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

typedef unsigned long long u64;
typedef unsigned int u32;

// Density is accumulated as unsigned 64-bit fixed point with 38 fractional bits: integer
// sums are associative, so the deposit is bitwise deterministic in any order, and
// delta = S/n_mean - 1 keeps full FP32 relative precision even where |delta| << 1.
#define PM_FIX_BITS 38
#define PM_FIX_ONE (1ULL << PM_FIX_BITS)

#define PM_H_I 5.0

// Per-peak lifecycle, read by the step kernels from device memory so that one captured
// graph serves any mix of peaks.
enum PeakState : int {
  PS_IDLE = 0,      // nothing to do; state and grids are frozen
  PS_PRIME = 1,     // new particles loaded: deposit + forces this step, no push
  PS_RUN = 2,       // regular KDK step
  PS_FINALIZE = 3,  // apply the pending closing kick, then go idle
  PS_HOLD = 4       // stepped once on request; keeps its pending kick until told again
};

enum ScheduleMode : int {
  SCHED_RATIO = 0,     // da = a*param for max_steps steps (uniform in ln a)
  SCHED_FRAC = 1,      // da = min(param*a, a_end - a) until a >= a_end (pbhgr/scripts/pm3d_peak.py:26-27)
  SCHED_EXPLICIT = 2   // one step of the da the host wrote, then hold
};

struct PeakDesc {
  int N, log2N;
  int TS, log2TS;          // super-tile side: the unit of push, deposit and particle grouping
  int NS;                  // super-tiles per axis (N / TS)
  int nst;                 // super-tiles (NS^3)
  int key_bits;            // 3*log2N: Morton key of the CIC cell
  int st_shift;            // 3*log2TS: key >> st_shift is the super-tile
  int fc, hc;              // face nodes (any local coordinate 0) and upper-halo nodes per super-tile
  int gradient;            // 0 spectral (reference), 1 two-point finite difference, 2 four-point
  int full_every;          // every super-tile's particles re-sorted by cell every this many steps (0: never)
  int native_fft;          // 1: the native 256^3 transform carries the Green multiply (no k_green)
  int bin_shift, bin_min;  // bin capacity: count + (count >> bin_shift) + bin_min, rounded up to BIN_ALIGN
  int bin_grow;            // relayout: room for this many more steps of a bin's growth (region allowing)
  int pad_bg;
  double L, dx, smooth, n_mean, m_part;
  long long n_mean_fix;    // round(n_mean * 2^38)
  double inv_fix_nmean;    // 2^-38 / n_mean
  long long p_off, n;      // particle range in the loading/overflow area (and in the sort arrays)
  long long r_off, r_size; // bin region of this peak in each of the two bin buffers
  long long st_base;       // first global super-tile index of this peak
  long long sst_off;       // offset of this peak's super-tile start array (nst + 1 entries)
  long long face_off;      // offset of this peak's face partials (nst * fc)
  long long halo_off;      // offset of this peak's halo partials (nst * hc)
  long long mode_base;     // first global mode-block of this peak (Green kernel)
  long long nmodes;        // N*N*(N/2+1)
  u32 nh_magic;            // m / (N/2+1) = (umulhi(m, nh_magic) + m) >> nh_shift for 32-bit m
  int nh_shift;
  float* delta;            // N^3 FP32 density contrast (R2C input)
  float2* spec;            // N*N*(N/2+1) complex spectrum (R2C output)
  float2* gspec;           // 3 gradient spectra
  float* force;            // 3 force grids of N^3 (C2R output)
};

struct PeakClock {
  double a;        // expansion factor of the current positions
  double da;       // size of the next step
  double a_end;    // SCHED_FRAC end point
  double kpend;    // pending closing-kick coefficient 0.5*da_prev/(a H(a)), 0 if none
  double param;    // ratio (SCHED_RATIO) or da_frac (SCHED_FRAC)
  double a_grid;   // expansion factor the force grids were computed at
  int mode;        // ScheduleMode
  int state;       // PeakState
  int nsteps;      // steps taken
  int max_steps;   // SCHED_RATIO length
  int sbuf;        // bin buffer holding the current particles (the push writes the other one)
  int lgen;        // bin layout generation in use ({base, capacity} per super-tile)
  int dep;         // 1 when this step re-deposits (set by the advance kernel)
  int sortstep;    // 1 when this step groups the loaded particles by a full Morton-key sort (priming)
  int relayout;    // this step's push overflowed a bin: 1 until the layout kernel decides, then 1 for a
                   // partial relayout (the overflowed bins move to free space at the end of the peak's
                   // region) or 2 for a full one (every bin re-laid out, into the other buffer)
  int refresh;     // 1 when this step re-sorts every super-tile's particles by cell
  int has_delta;   // delta/grids hold data
  int stop_on_collapse;  // end the run (finalize) on the step that detects collapse
  double delta_collapse;  // collapse threshold on max delta (<= 0: not tracked)
  double a_collapse;      // first a whose deposit reached delta_collapse (-1: not yet)
};

// Per-peak device statistics.  Integer fields are reduced with integer atomics
// (order-independent); FP64 sums are written per block and reduced in a fixed order.
struct PeakStats {
  u64 max_fix;            // max node count in fixed point
  long long mass_defect;  // sum over nodes of (S - n_mean_fix): 0 when mass is exact
  u32 status;             // bit 0: non-finite force/momentum, bit 1: fixed-point overflow
  u32 nsamples;           // energy samples taken since the peak was loaded
  u32 relayouts;          // steps since the peak was loaded whose push overflowed a bin
  u32 relayouts_full;     // of those, the steps that re-laid out every bin of the peak
  // Energy and momentum at a_e, from compensated FP64 sums in a fixed reduction order.  With
  // p = a^2 dx/dt, dp/dt = -grad Phi (pbhgr/pbhgr/pm3d.py:3-6) the Layzer-Irvine equation reads
  // d[a (K + W)]/da = -K, so a (K + W) + int_{a0}^{a} K da stays equal to a0 (K0 + W0).
  double a_e;             // expansion factor of the last sample
  double mom[3];          // total canonical momentum m_p sum p
  double kin;             // K = m_p/(2 a^2) sum p^2 (peculiar velocity p/a)
  double pot;             // W = (1/2) rho_b a^3 dx^3 sum_nodes delta Phi (mesh potential energy)
  double li_int;          // int K da over the samples so far (trapezoid rule)
  double li_e0;           // a0 (K0 + W0) at the first sample
};

// Neumaier-compensated FP64 sum (s + c is the running total).
struct CSum {
  double s, c;
};
__device__ __forceinline__ void csum_add(CSum& a, double x) {
  const double t = a.s + x;
  a.c += fabs(a.s) >= fabs(x) ? (a.s - t) + x : (x - t) + a.s;
  a.s = t;
}
__device__ __forceinline__ void csum_merge(CSum& a, const CSum& b) {
  csum_add(a, b.s);
  a.c += b.c;
}
// Warp-level merge (lane 0 holds the warp's total); a fixed butterfly, so the order is fixed.
__device__ __forceinline__ CSum csum_warp(CSum v) {
  for (int d = 16; d > 0; d >>= 1) {
    CSum o;
    o.s = __shfl_down_sync(0xffffffffu, v.s, d);
    o.c = __shfl_down_sync(0xffffffffu, v.c, d);
    csum_merge(v, o);
  }
  return v;
}

#define PM_CHECK(x)                                  \
  do {                                               \
    cudaError_t e_ = (x);                            \
    if (e_ != cudaSuccess) return -(int)e_;          \
  } while (0)

// ---------------------------------------------------------------------------- Morton
__host__ __device__ __forceinline__ u32 pm_spread3(u32 v) {
  v &= 0x3FF;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
__host__ __device__ __forceinline__ u32 pm_compact3(u32 v) {
  v &= 0x09249249u;
  v = (v | (v >> 2)) & 0x030C30C3u;
  v = (v | (v >> 4)) & 0x0300F00Fu;
  v = (v | (v >> 8)) & 0x030000FFu;
  v = (v | (v >> 16)) & 0x3FFu;
  return v;
}
// z occupies the lowest bit of each triple, so consecutive codes walk along z (the
// contiguous axis of the mesh).
__host__ __device__ __forceinline__ u32 pm_morton3(u32 x, u32 y, u32 z) {
  return (pm_spread3(x) << 2) | (pm_spread3(y) << 1) | pm_spread3(z);
}

// Cell key of a node-lattice cell: the Morton code of (ix, iy, iz), z in the lowest bit of each
// triple.  Codes nest: key >> (3 log2 TS) is the Morton code of the super-tile.
__host__ __device__ __forceinline__ u32 pm_cell_key(int ix, int iy, int iz) { return pm_morton3(ix, iy, iz); }

__host__ __device__ __forceinline__ double pm_hubble(double a) { return PM_H_I / (a * sqrt(a)); }

// Unsigned division by an invariant divisor d >= 1 (Granlund & Montgomery 1994, the round-up
// method for 32-bit operands): with l = ceil(log2 d) and magic = floor(2^32 (2^l - d) / d) + 1,
// n / d = (umulhi(n, magic) + n) >> l for every 32-bit n (the sum is formed in 64 bits).
inline void pm_div_magic(u32 d, u32* magic, int* shift) {
  int l = 0;
  while ((1ull << l) < d) ++l;
  *magic = (u32)(((1ull << 32) * ((1ull << l) - d)) / d + 1);
  *shift = l;
}
__device__ __forceinline__ u32 pm_div_by(u32 n, u32 magic, int shift) {
  return (u32)(((unsigned long long)__umulhi(n, magic) + n) >> shift);
}
