// Kernels of one PM step (pbhgr/pbhgr/pm3d.py:101-129) over a batch of peaks.
//
// Particles live in bins, one per super-tile (TS^3 cells), in two bin buffers that alternate
// every step.  Both buffers share a bin layout: super-tile S of a peak owns slots
// [base[S], base[S] + cap[S]) of each buffer, with spare capacity (an eighth of its count plus
// 32, and room for further growth after a relayout, set whenever the layout is made).  A filled bin holds two runs: the particles that stayed
// in S, from base[S] up, and the particles that arrived from other super-tiles, from
// base[S] + (the bin's count before the step) up (BinFill).  One step:
//   push       per super-tile: CIC gather of the forces, kicks, drift; each particle appended
//              to the bin of the super-tile it is now in, in the other buffer (stayers ranked in
//              shared memory, arrivals by an atomic on the destination's count); a particle
//              for which the destination bin has no room goes to the peak's overflow area
//   energy     per peak: momentum, kinetic and potential energy, Layzer-Irvine integral
//   advance    per peak clock; a peak whose push overflowed relayouts this step
//   regroup    relayout (new capacities from the counts, bins and overflow area copied into the
//              buffer the push read); every full_every steps each super-tile's particles are
//              re-sorted by cell (local counting sort); when particles are first loaded, a full
//              Morton-key radix sort of the loading area and a permutation into fresh bins
//   deposit    per super-tile: CIC density of its particles into (TS+1)^3 nodes; interior nodes
//              final, face and upper-halo nodes as 64-bit partials
//   fixup      per super-tile: face nodes = own partial + the lower neighbours' halo partials
//   R2C, Green, C2R (x3)
#pragma once
#include "common.cuh"
#include "sort.cuh"

#define PM_THREADS 256
#define PUSH_THREADS 512
#define DEP_THREADS 256    // deposit CTA (4 per SM)
#define GREEN_MODES 4      // modes per thread of the Green kernel (a block covers PM_THREADS * GREEN_MODES)
#define ENERGY_SLICES 16   // CTAs per peak of the energy reduction
#define FIX_THREADS 256    // face fix-up CTA
#define TSORT_THREADS 1024 // super-tile sort (refresh) CTA
#define TSORT_CAP 5120     // particles of a super-tile sorted in shared memory; denser ones via global
// Bin capacities: count + (count >> BIN_SLACK_SHIFT) + BIN_SLACK_MIN, rounded up to BIN_ALIGN;
// a relayout adds room for BIN_ARRIVALS times the arrivals of the step plus BIN_GROW_STEPS times
// its net growth, out of a further (n >> BIN_SPARE_SHIFT) slots of the peak's bin region.
#ifndef BIN_SLACK_SHIFT
#define BIN_SLACK_SHIFT 3
#endif
#ifndef BIN_SPARE_SHIFT
#define BIN_SPARE_SHIFT 3
#endif
#ifndef BIN_ARRIVALS
#define BIN_ARRIVALS 1
#endif
#ifndef BIN_GROW_STEPS
#define BIN_GROW_STEPS 4
#endif
#define BIN_SLACK_MIN 32
#define BIN_ALIGN 8        // bin bases and capacities are multiples of 8 slots (128 bytes)
#define LAYOUT_THREADS 1024
#define RELAYOUT_OVF_BLOCKS 32  // CTAs per peak placing a relayout's overflow area
#define RELAYOUT_COPY_BLOCKS 256  // CTAs per peak moving a relayout's bins

// Fill of one bin in one buffer: the stayers occupy [base, base + stay), the arrivals
// [base + gap, base + gap + min(moved, cap - gap)); gap is the bin's count before the push
// that filled it (no stayer rank reaches it).  `moved` is incremented atomically by the pushes
// of all source super-tiles and may exceed the room; the excess went to the overflow area.
struct BinFill {
  u32 stay, gap, moved, pad;
};
struct BinLayout {
  u32 base, cap;  // slot offset in a bin buffer, capacity
};

// Views of the engine's device arrays handed to every kernel.
struct StepArgs {
  const PeakDesc* peaks;
  PeakClock* clocks;
  PeakStats* stats;
  SortSeg* sortseg;            // sort activity flags, written by the advance kernel
  u32* sort_gate;              // 1 when any peak primes by sort this step (advance kernel)
  u32* layout_gate;            // 1 when any peak primes or relayouts this step (advance kernel)
  u32* refresh_gate;           // 1 when any peak re-sorts its super-tiles this step (advance kernel)
  const long long* st_base;    // [npeaks + 1] prefix of super-tiles
  const unsigned short* st_peak;  // [super-tile] its peak (one load instead of a search)
  const long long* p_base;     // [npeaks + 1] prefix of particles
  const long long* mode_base;  // [npeaks + 1] prefix of Green blocks
  const long long* green_base; // [ngreen + 1] prefix of Green blocks over the peaks k_green serves
  const int* green_peak;       // [ngreen] those peaks (the others use the native transform)
  int npeaks;
  int ngreen;
  int4* pos0;                  // bin buffers 0 and 1 (clock.sbuf: the current one)
  float4* mom0;
  int4* pos1;
  float4* mom1;
  int4* lpos;                  // loading area (set_particles, reload) and overflow area of the push,
  float4* lmom;                // [p_off, p_off + n) per peak
  BinLayout* lay[2];           // [super-tile] bin layouts, two generations (clock.lgen selects)
  BinFill* fill[2];            // [super-tile] bin fills of buffers 0 and 1
  u32* ovf_n;                  // [peak] particles in the overflow area (push), reset by the deposit
  u32* ovf_in;                 // [super-tile] overflowed particles whose destination it is
  u32* keys_push;              // Morton keys written by set_particles / reload (priming sort input)
  const u32* keys_sorted;      // sort output keys
  const u32* perm;             // sort output permutation
  u32* sstart;                 // [peak][nst + 1] starts of the super-tiles in the sorted keys
  long long* face;             // face partials
  long long* halo;             // upper-halo partials
  double2* epart;              // [super-tile][4] push partials (sum, compensation): p_x, p_y, p_z, p^2
  double* wpart;               // [Green block][warp] partials of sum_k w_k |delta_k|^2 G_k
  double2* eslice;             // [peak][ENERGY_SLICES][5] slice partials of the energy kernel
  u32* ecount;                 // [peak] energy slices finished this step (0 between steps)
  int* sort_err;               // [peak] the priming sort's bounded look-back gave up (sort plan)
};

// Binary search: largest i in [0, n) with base[i] <= v.
__device__ __forceinline__ int pm_find(const long long* base, int n, long long v) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (base[mid] <= v) lo = mid; else hi = mid - 1;
  }
  return lo;
}

int pm_kernels_init();  // kernel attributes; call once per device before launching
size_t pm_deposit_smem(int TSmax);
size_t pm_push_smem(int TSmax);

void launch_push(const StepArgs& A, long long nst, size_t smem, cudaStream_t s);
void launch_advance(const StepArgs& A, cudaStream_t s);
void launch_energy(const StepArgs& A, cudaStream_t s);
void launch_permute(const StepArgs& A, long long ntot, cudaStream_t s);
void launch_st_starts(const StepArgs& A, long long ntot, cudaStream_t s);
// Bin layouts of the priming and relayout peaks, then the relayout's copies (gated launches).
void launch_layout(const StepArgs& A, long long nst, long long ntot, cudaStream_t s);
void launch_tile_sort(const StepArgs& A, long long nst, cudaStream_t s);
void launch_deposit(const StepArgs& A, long long nst, size_t smem, double* rho64, cudaStream_t s);
void launch_fixup(const StepArgs& A, long long nst, double* rho64, cudaStream_t s);
void launch_green(const StepArgs& A, long long nblocks, cudaStream_t s);

// Native real FFT of 256^3 and 512^3 meshes (native_fft.cu).  fft_native_init: once per device
// before use.
bool fft_native_size(int N);
int fft_native_init();
int fft_native_r2c(int N, const float* delta, float2* spec, int nslots, cudaStream_t s);
int fft_native_green_c2r(int N, const float2* spec, float2* gwork, float* force, const StepArgs& A,
                         const int* slot_peak, int nslots, cudaStream_t s);
int fft_native_c2r(int N, const float2* spec, float2* gwork, float* out, int nfields, cudaStream_t s);

// Host-requested per-peak operations.  reset: new schedule from a0, status and sort error
// cleared; set_thr = 1 also sets the collapse threshold and its stop flag (else they are kept).
void launch_reset_peak(const StepArgs& A, int pk, double a0, int mode, double param, double a_end,
                       int max_steps, int set_thr, double delta_collapse, int stop, cudaStream_t s);
// release: the peak goes idle (no pending kick, no grids), on the stream, without a host round trip.
void launch_release_peak(const StepArgs& A, int pk, cudaStream_t s);
void launch_set_particles(const StepArgs& A, int pk, const PeakDesc& P, const double* x, const double* p,
                          cudaStream_t s);
void launch_reload(const StepArgs& A, int pk, const PeakDesc& P, cudaStream_t s);  // bins -> loading area + keys
void launch_get_particles(const StepArgs& A, int pk, const PeakDesc& P, double* x, double* p, double* acc,
                          double a_acc, cudaStream_t s);
void launch_interp64(const double* F, const double* X, long long n, int N, double dx, double* out, cudaStream_t s);
void launch_deposit64(const double* X, long long n, int N, double dx, u64* work, double* counts, cudaStream_t s);
