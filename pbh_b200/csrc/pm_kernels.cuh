// Kernels of one PM step (pbhgr/pbhgr/pm3d.py:101-129) over a batch of peaks.
#pragma once
#include "common.cuh"
#include "sort.cuh"

#define PM_THREADS 256
#define PUSH_THREADS 512
#define DEP_THREADS 512

// Views of the engine's device arrays handed to every kernel.
struct StepArgs {
  const PeakDesc* peaks;
  PeakClock* clocks;
  PeakStats* stats;
  SortSeg* sortseg;            // sort activity flags, written by the advance kernel
  SortSeg* sortseg_full;       // the same for the full-key plan
  const long long* tile_base;  // [npeaks + 1] prefix of tiles
  const long long* ptile_base; // [npeaks + 1] prefix of push super-tiles
  const long long* p_base;     // [npeaks + 1] prefix of particles
  const long long* mode_base;  // [npeaks + 1] prefix of Green blocks
  int npeaks;
  int pad;
  int4* pos[2];
  float4* mom[2];
  u32* keys_push;              // cell keys written by the push kernel (sort input); the
                               // peak id, the high word of the 64-bit key, is the segment
  const u32* keys_sorted;      // sort output keys
  const u32* perm;             // sort output permutation (index into the current buffer)
  u32* bstart;                 // bucket starts arena
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
size_t pm_deposit_smem(int TPmax);
size_t pm_push_smem(int TPmax);

void launch_push(const StepArgs& A, long long nptiles, size_t smem, cudaStream_t s);
void launch_advance(const StepArgs& A, cudaStream_t s);
void launch_bucket_starts(const StepArgs& A, long long ntot, cudaStream_t s);
void launch_deposit(const StepArgs& A, long long nptiles, size_t smem, double* rho64, cudaStream_t s);
void launch_green(const StepArgs& A, long long nblocks, cudaStream_t s);

// Host-requested per-peak operations.
void launch_reset_peak(const StepArgs& A, int pk, double a0, int mode, double param, double a_end,
                       int max_steps, cudaStream_t s);
void launch_set_particles(const StepArgs& A, int pk, const PeakDesc& P, const double* x, const double* p,
                          cudaStream_t s);
void launch_get_particles(const StepArgs& A, int pk, const PeakDesc& P, double* x, double* p, double* acc,
                          double a_acc, cudaStream_t s);
void launch_interp64(const double* F, const double* X, long long n, int N, double dx, double* out, cudaStream_t s);
