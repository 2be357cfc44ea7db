/* pmb200 -- C ABI of the B200 particle-mesh engine for the pm3d hot path.
 *
 * The reference path (uniquehuman/pbh, pbhgr/pbhgr/pm3d.py) is a pure-numpy Python class with
 * no FFI of its own; its plugin surface is the PM3D class (pm3d.py:26-129).  This header is
 * the native boundary underneath the drop-in Python class pbh_b200.pm3d.PM3D, and follows the
 * reference repository's own ctypes convention for native code (pbhgr/csrc/kernels.c:36,73
 * loaded by pbhgr/pbhgr/spherical_ev.py:59-78): plain extern "C" functions, caller-owned
 * contiguous buffers, an int return code.
 *
 * Conventions
 *  - All array pointers are DEVICE pointers on the engine's device unless stated otherwise.
 *  - Positions/momenta are (n, 3) float64 in lattice order: row i is the particle that
 *    starts at lattice site i of PM3D's quiet start (pm3d.py:64-65), as PM3D.x / PM3D.p.
 *  - Meshes are (N, N, N) C-order arrays, node (i, j, k) at ((i, j, k) + 1/2) dx (pm3d.py:42).
 *  - Return value: 0 = OK; > 0 = number of flagged items (status words); < 0 = error:
 *    -1..-999 = -(cudaError_t), -1000 - r = cuFFT result r, -2000 - k = invalid argument k.
 *  - Calls are asynchronous on the engine's stream except those that return host data, which
 *    synchronize it.  Use pm_engine_sync before reading device outputs from another stream.
 *  - One host thread drives an engine at a time.
 */
#ifndef PMB200_H
#define PMB200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pm_engine pm_engine;

/* One peak (one PM3D instance): PM3D(N, L, Np, seed, smooth) of pm3d.py:27. */
typedef struct {
  int N;          /* mesh side, power of two, 8..1024 */
  int Np;         /* particles per side (n = Np^3) */
  int tile;       /* super-tile side for push/deposit/grouping: 4, 8 or 16 (0: min(16, N)) */
  int gradient;   /* 0: spectral -i k (the reference, pm3d.py:111-112); 1: 2-point; 2: 4-point FD */
  double L;       /* box side */
  double smooth;  /* Gaussian force smoothing in cells (pm3d.py:107-108) */
  long long n;    /* particle count; 0 means Np^3 (any count is allowed, e.g. PM3D.deposit(X)) */
} pm_peak_cfg;

/* Step schedules (pm_set_particles). */
#define PM_SCHED_RATIO 0    /* da = a*param for max_steps steps (uniform in ln a) */
#define PM_SCHED_FRAC 1     /* da = min(param*a, a_end - a) until a >= a_end (pbhgr/scripts/pm3d_peak.py:26-27) */
#define PM_SCHED_EXPLICIT 2 /* one step per pm_step_explicit call (PM3D.step, pm3d.py:117) */

/* Peak states reported by pm_get_clock. */
#define PM_STATE_IDLE 0
#define PM_STATE_PRIME 1
#define PM_STATE_RUN 2
#define PM_STATE_FINALIZE 3
#define PM_STATE_HOLD 4

typedef struct {
  double a;       /* expansion factor of the current positions */
  double da;      /* next step */
  double a_end;
  double kpend;   /* pending closing-kick coefficient (0 when p is complete) */
  double a_grid;  /* expansion factor the force grids were computed for */
  int mode, state, nsteps, max_steps;
  double a_collapse; /* first a at which max delta reached the collapse threshold, -1 if not yet */
} pm_clock_info;

typedef struct {
  double rho_max_over_mean;  /* max node count / n_mean of the last deposit (pm3d.py:158) */
  double delta_max;          /* max delta of the last deposit (pbhgr/scripts/pm3d_peak.py:30) */
  double mass_defect;        /* sum over nodes of (count - n_mean), exactly 0 unless corrupted */
  unsigned status;           /* bit 0: non-finite momentum or a particle outside its super-tile;
                              * bit 1: sort look-back gave up; bit 2: regrouping lost count;
                              * bit 3: a particle id outside the lattice */
  /* Energy check (no counterpart in pm3d.py; its equations of motion, pm3d.py:3-6): sampled at
   * every step's synchronised positions and momenta, from compensated FP64 sums in a fixed order.
   * Layzer-Irvine: a (K + W) + int_{a0}^{a} K da is constant; li_residual is its change since
   * the first sample, li_scale = a (K + |W|) the size to compare it with. */
  int energy_samples;        /* samples since the peak was loaded (0: fields below are 0) */
  double a_energy;           /* expansion factor of the last sample */
  double momentum[3];        /* m_p sum p (canonical momentum) */
  double kinetic;            /* K = m_p / (2 a^2) sum p^2 */
  double potential;          /* W = (1/2) rho_b a^3 dx^3 sum_nodes delta Phi (the PM mesh potential) */
  double li_residual;
  double li_scale;
  int relayouts;             /* steps since the load whose push overflowed a super-tile's bin (the
                              * overflowed bins were then moved to free space with more capacity) */
  int relayouts_full;        /* of those, the steps with no such space left: every bin of the peak
                              * was re-laid out and all of its particles moved */
} pm_stats_info;

/* Create an engine holding npeaks independent peaks (1 <= npeaks <= 65535; a batched ensemble;
 * npeaks = 1 is the plain single run).  Allocates all device memory and cuFFT plans up front; no later call
 * allocates.  flags: bits 8..15 = re-sort every super-tile's particles by cell every that many
 * steps (never if 0, the default: the push keeps them binned by super-tile, and the order inside
 * a bin was measured not to matter); bit 1 = replay the step as a CUDA
 * graph; bit 2 = dynamic mode for served runs: no graph, and each step's FFTs cover only the
 * slots up to the highest one in use in each mesh size (slots are the peaks of one size, in
 * order); bit 3 = the native transform with the Green multiply fused (pm_rfft3_native) for
 * meshes 64^3-512^3 instead of cuFFT; bit 16 = bins without spare capacity (a test mode: almost
 * every step overflows a bin and relayouts; results are the same bit for bit).
 * Replaces: PM3D(N, L, Np, seed, smooth) (pm3d.py:27-37), once per peak. */
int pm_engine_create(const pm_peak_cfg* cfg, int npeaks, int device, int flags, pm_engine** out);
/* Free the engine's device memory, plans and graphs (no counterpart: the reference's arrays are
 * garbage-collected). */
int pm_engine_destroy(pm_engine* e);
/* Wait for the engine's stream (no counterpart: the reference is synchronous). */
int pm_engine_sync(pm_engine* e);
/* Bytes of device memory the engine holds (no counterpart; the served loop's HBM accounting). */
long long pm_engine_device_bytes(const pm_engine* e);

/* Load particles (lattice order) for one peak at expansion factor a0 and choose its schedule.
 * The peak primes (sort + deposit + forces at a0) on the next pm_run step.
 * Replaces: assignment of PM3D.x / PM3D.p after make_ic (pm3d.py:67-68). */
int pm_set_particles(pm_engine* e, int peak, const double* x, const double* p, double a0, int mode,
                     double param, double a_end, int max_steps);

/* Advance every peak that has work by nsteps engine steps (one batched step each).
 * Replaces: the driver loop of pbhgr/scripts/pm3d_peak.py:26-28. */
int pm_run(pm_engine* e, int nsteps);

/* pm_run without the graph, with a CUDA event between kernel phases on the engine's stream;
 * adds each phase's device time (ms) into phase_ms[8]: push, energy + clock advance, regroup
 * (priming radix sort with its permutation, bin layouts, relayouts of peaks whose push
 * overflowed a bin), super-tile re-sort (refresh steps), deposit (with the face fix-up), R2C,
 * Green, C2R.  For per-kernel rooflines (no counterpart; the reference times nothing finer than
 * the driver's wall clock, pbhgr/scripts/pm3d_peak.py:24,32,35). */
int pm_run_timed(pm_engine* e, int nsteps, double* phase_ms);
/* The engine's CUDA stream (cudaStream_t), for events and stream ordering by callers (no
 * counterpart). */
void* pm_engine_stream(pm_engine* e);
/* info[6]: npeaks, particles, super-tiles, sort passes, mesh classes, device bytes (no
 * counterpart). */
int pm_engine_info(const pm_engine* e, long long* info);

/* PM3D.step(a, da) for one peak (pm3d.py:117-129): a KDK step from a to a + da.  Forces at
 * a are reused when the peak's current state is at a (pm3d.py:119), else recomputed. */
int pm_step_explicit(pm_engine* e, int peak, double a, double da);

/* Current particles, float64, lattice order; p includes the closing kick.  Replaces: reading
 * PM3D.x, PM3D.p (pm3d.py:67-68, 122-128). */
int pm_get_particles(pm_engine* e, int peak, double* x, double* p);
/* -grad Phi at the particles for expansion factor a, lattice order: the acc of
 * PM3D.forces(a) (pm3d.py:101-114) at the current positions. */
int pm_get_acc(pm_engine* e, int peak, double a, double* acc);
/* delta of the last deposit (N^3 float32): the delta returned by PM3D.step/forces
 * (pm3d.py:103-104, 129). */
int pm_get_delta(pm_engine* e, int peak, float* delta);
/* Float64 CIC counts of the current positions (N^3): PM3D.deposit(PM3D.x) (pm3d.py:81-89). */
int pm_get_counts(pm_engine* e, int peak, double* counts);
/* Collapse time tracking: the first a at which max delta of the peak's deposit reaches
 * delta_collapse is recorded on the device (pm_clock_info.a_collapse); <= 0 disables.  With
 * stop != 0 the run ends there: the step on which the crossing is detected (the one after the
 * deposit that crossed) completes, the next applies its closing kick, and the peak goes idle at
 * the a that step reached.  No counterpart in pm3d.py, which defines no collapse time; the
 * criterion reads the max delta that PM3D.step returns (pm3d.py:129), as the driver's rows do
 * (pbhgr/scripts/pm3d_peak.py:30). */
int pm_set_collapse_threshold(pm_engine* e, int peak, double delta_collapse, int stop);
/* Free a peak's slot: it goes idle, its mesh is no longer transformed (dynamic mode).  Ordered
 * on the engine's stream after the work queued so far; returns without waiting.  No counterpart
 * (the reference's driver ends with its process, pbhgr/scripts/pm3d_peak.py:34-35). */
int pm_release(pm_engine* e, int peak);

/* Entry points of a request loop that never waits on the device between steps (the served form
 * with continuous batching; no counterpart in pm3d.py, whose driver runs one peak at a time,
 * pbhgr/scripts/pm3d_peak.py:24-33).  Each is ordered on the engine's stream and returns without
 * waiting.
 *
 * pm_load_peak: pm_set_particles plus pm_set_collapse_threshold in one call, after the engine's
 * stream has waited for wait_event (a cudaEvent_t recorded where x and p were produced, or NULL).
 * x and p must stay valid until the engine's stream has passed this point (record an event on
 * pm_engine_stream after the call). */
int pm_load_peak(pm_engine* e, int peak, const double* x, const double* p, double a0, int mode, double param,
                 double a_end, int max_steps, double delta_collapse, int stop, void* wait_event);
/* pm_snapshot: queue a copy of every peak's clock and statistics, as they stand after the work
 * queued so far, into the engine's host buffer `slot` (0 or 1).  pm_snapshot_read decodes that
 * buffer into host arrays of npeaks entries (either may be NULL) as pm_get_clocks_all and
 * pm_get_stats_all would: with wait = 0 it returns 1 at once if the copy has not finished,
 * with wait != 0 it waits for the copy (only); 0 once decoded. */
int pm_snapshot(pm_engine* e, int slot);
int pm_snapshot_read(pm_engine* e, int slot, int wait, pm_clock_info* clocks, pm_stats_info* stats);
/* pm_get_delta without waiting: the N^3 float32 delta of the peak's last deposit into dst
 * (device memory, or page-locked host memory for a direct copy to the host). */
int pm_get_delta_async(pm_engine* e, int peak, void* dst);

/* Test hook of the failure path: from the next sort on, the look-back words of the first tile
 * of `peak`'s segment are never published in the first digit pass, so the bounded wait of the
 * tile after it runs out after spin_limit polls; the sort then proceeds with that tile counted
 * as empty (every write stays inside the peak's range, the peak's result is wrong) and the
 * peak's status gets bit 1.  peak < 0 or spin_limit <= 0 restores the normal sort.  The peak
 * needs more than one sort tile (2048 particles); synchronizes the engine's stream.  No
 * counterpart (the reference has no device waits). */
int pm_debug_sort_stall(pm_engine* e, int peak, int spin_limit);
/* One peak's clock and statistics (host structs): the a and da of the driver loop
 * (pbhgr/scripts/pm3d_peak.py:24-27), rho_max_over_mean of analyse (pm3d.py:158), max delta of
 * the driver's rows (pm3d_peak.py:30), and the status word in the reference's convention for
 * native code (a count of flagged items, pbhgr/csrc/kernels.c:36,73). */
int pm_get_clock(pm_engine* e, int peak, pm_clock_info* out);
int pm_get_stats(pm_engine* e, int peak, pm_stats_info* out);
/* All peaks at once (host arrays of npeaks); the return value counts flagged peaks. */
int pm_get_stats_all(pm_engine* e, pm_stats_info* out);
int pm_get_clocks_all(pm_engine* e, pm_clock_info* out);

/* Initial particles on the GPU in float64 (setup call: allocates and frees its temporaries).
 * kind 0 = PM3D.make_ic(mu, profile_spline, e, p, tail_rms, tail_k) (pm3d.py:40-73): amp = mu,
 *   axes = zeldovich_axes(e, p), the spline as scipy PPoly breakpoints x[m+1] and
 *   coefficients c[4][m] (HOST arrays), noise = rng.standard_normal((N,N,N)) when tail_rms > 0.
 * kind 1 = Gaussian density peak delta0 exp(-sum x_i^2/2R_i^2) plus noise with P(k) ~ k^-2
 *   scaled to rms noise_frac*delta0 (the benchmark recipe): amp = delta0, axes = R.
 * Both continue with the reference's Zel'dovich tail (pm3d.py:59-72).  Outputs: x, p (n,3) in
 * lattice order, optional delta_lin (N^3), and on the host the rms of the noise field on the
 * grid (PM3D.tail_rms_grid for kind 0). */
typedef struct {
  int N, Np;
  double L;
  int kind;
  double amp;
  double axes[3];
  const double* spline_x;  /* host, m + 1 breakpoints */
  const double* spline_c;  /* host, 4*m coefficients, c[k*m + i] multiplies (r - x_i)^(3-k) */
  int spline_m;
  const double* noise;     /* device, N^3 standard normals, or NULL */
  double tail_rms, k1, k2;
  double noise_frac;
  unsigned long long noise_seed;  /* noise == NULL and seed != 0: N^3 normals generated on the
                                   * device (Philox4x32-10 + Box-Muller) instead of numpy's stream */
} pm_ic_params;
int pm_make_ic(const pm_ic_params* prm, double* x_out, double* p_out, double* delta_lin_out, double* noise_rms_out);
/* pm_make_ic for the recipe peak (kind 1, noise from a device array or noise_seed) ordered on
 * `stream` (a cudaStream_t): returns without waiting, allocates nothing after its first call
 * for a mesh size (its work area is separate from pm_make_ic's), and reports no noise rms.  The
 * same inputs give the same bits as pm_make_ic.  Calls for one mesh size share the work area:
 * issue them on one stream.  kind 0 returns -2003. */
int pm_make_ic_async(const pm_ic_params* prm, double* x_out, double* p_out, void* stream);
/* pm_make_ic and pm_make_ic_async keep their float64 work buffers and cuFFT plans per (device,
 * N) after the first call; this frees them (no counterpart: the reference's make_ic keeps no
 * state between calls, pm3d.py:40-73). */
int pm_ic_release_cache(void);

/* Stateless helpers. */
/* PM3D.interp(F, X) (pm3d.py:91-99) in float64: F (N^3), X (n,3) -> out (n). */
int pm_interp64(const double* F, const double* X, long long n, int N, double L, double* out);
/* PM3D.deposit(X) (pm3d.py:81-89) of arbitrary float64 positions X (n,3) without an engine:
 * counts (N^3 float64), each particle's eight corner weights rounded to 2^-39 in 64-bit fixed
 * point with integer sums (the result does not depend on the order of X).  work: caller scratch
 * of N^3 unsigned 64-bit words.  Synchronizes the device. */
int pm_deposit64(const double* X, long long n, int N, double L, unsigned long long* work, double* counts);
/* Stable sort of n 64-bit keys over bits [lo, hi): keys_out, perm_out (original indices).
 * tmp_keys/tmp_vals are caller scratch of n entries each.  Replaces the argsorts of analyse
 * (pm3d.py:137, 145) and the sort of cell keys that deposit and interp need for unsorted X. */
int pm_sort_u64(const unsigned long long* keys, unsigned long long* keys_out, unsigned int* perm_out,
                unsigned long long* tmp_keys, unsigned int* tmp_vals, long long n, int lo, int hi);
/* Diagnostics of analyse (pm3d.py:132-159).  pm_rell_keys: the Lagrangian ellipsoidal radius
 * r_ell_q of every lattice site (pm3d.py:71) as order-preserving uint64 keys, for picking the
 * innermost sets with pm_sort_u64 (ties then fall to the lower lattice index).
 * pm_analyse_partials: per-block float64 partial sums, 34 per block, over x (n,3, lattice
 * order): for each of the 3 sets r_ell_q < set_radii[s] the count, sum of rel and the 6
 * entries of sum rel rel^T, rel = periodic offset from centre (pm3d.py:142-147); then the 4
 * counts of |rel| < radii[k] (pm3d.py:153-156).  A, centre, set_radii, radii are HOST arrays. */
int pm_rell_keys(int Np, double L, const double* A, unsigned long long* keys);
int pm_analyse_partials(const double* x, int Np, double L, const double* A, const double* centre,
                        const double* set_radii, const double* radii, int nblocks, double* partials);
/* Native 3D real FFT of n^3 fields, n = 64, 128, 256 or 512 (the transform the engine uses for those mesh
 * sizes; replaces np.fft.rfftn of pbhgr/pbhgr/pm3d.py:105 and np.fft.irfftn of pm3d.py:112).
 * x: nfields fields [f][x][y][z] float.  spec: [f][kz][kx][ky] complex (kz = 0..n/2; numpy's
 * rfftn(x)[kx][ky][kz] is spec[kz][kx][ky]).  Both directions are unnormalised (the inverse is
 * n^3 times numpy's irfftn).  work: caller scratch of the spectrum's size.  Device pointers,
 * 16-byte aligned (-2001 otherwise); asynchronous on `stream`; the first call on a device sets
 * up its twiddle table.  pm_rfft3_256 / pm_irfft3_256 are the n = 256 forms. */
int pm_rfft3_native(int n, const float* x, void* spec, int nfields, void* stream);
int pm_irfft3_native(int n, const void* spec, void* work, float* x, int nfields, void* stream);
int pm_rfft3_256(const float* x, void* spec, int nfields, void* stream);
int pm_irfft3_256(const void* spec, void* work, float* x, int nfields, void* stream);

/* pm_sort_u64 for callers that cannot allocate device memory.  No counterpart in the reference
 * (which has no GPU code).  Some callers must not call cudaMalloc or cudaFree: cudaFree waits
 * for the whole device and both can stall on driver locks, so a latency-bound loop (such as a
 * request loop between two steps) cannot afford them, and a process whose device memory is
 * already held by another framework's allocator may have none to give.  This variant takes the
 * same input and outputs but keeps all of its scratch in one static device array of
 * PM_NOALLOC_SCRATCH_BYTES inside this library, which every GPU that loads the library holds
 * until the process exits; it calls no allocating routine.  n must not exceed
 * PM_NOALLOC_MAX_KEYS (larger n returns -2003 and touches nothing).  Each call looks up the
 * array's device address on the current device (cudaGetSymbolAddress, which allocates nothing);
 * the first call on a device also loads this library's kernels there, so make that first call
 * before any stream capture.  Every call shares the
 * array: calls that overlap on the GPU (from several streams or threads) race, and must be
 * serialized by the caller.  Runs on `stream` (a cudaStream_t, NULL for the default stream);
 * each call copies the sort's error word back to the host and waits for `stream` before it
 * returns: 0, 1 if a bounded look-back wait gave up, < 0 on error. */
#define PM_NOALLOC_MAX_KEYS (1LL << 18)
#define PM_NOALLOC_SCRATCH_BYTES (3670016)
int pm_sort_u64_noalloc(const unsigned long long* keys, unsigned long long* keys_out, unsigned int* perm_out,
                        long long n, int lo, int hi, void* stream);
/* Sort keys (Morton code of the CIC cell) of split positions, host pointers; for tests (no
 * counterpart: the reference indexes cells directly, pm3d.py:76-79). */
int pm_cell_keys(const int* cells, long long n, int N, int tile, unsigned int* keys_out);

#ifdef __cplusplus
}
#endif
#endif
