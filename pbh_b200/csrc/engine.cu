// Host side of the engine: memory layout, cuFFT plans, the step launch sequence and the
// extern "C" API declared in include/pmb200.h.
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "../../include/pmb200.h"
#include "pm_kernels.cuh"
#include "sort.cuh"

namespace {

int ilog2(int v) {
  int r = 0;
  while ((1 << r) < v) ++r;
  return (1 << r) == v ? r : -1;
}

#define CU(x)                                         \
  do {                                                \
    cudaError_t e_ = (x);                             \
    if (e_ != cudaSuccess) return -(int)e_;           \
  } while (0)
#define CF(x)                                         \
  do {                                                \
    cufftResult r_ = (x);                             \
    if (r_ != CUFFT_SUCCESS) return -1000 - (int)r_;  \
  } while (0)

struct MeshClass {
  int N = 0;
  std::vector<int> peaks;   // peak indices in slot order
  float* delta = nullptr;
  float2* spec = nullptr;
  float2* gspec = nullptr;
  float* force = nullptr;
  cufftHandle r2c = 0, c2r = 0;
  bool plans = false;
  // Dynamic mode: plans for every batch size 1..B over the leading slots, one shared work area.
  std::vector<cufftHandle> r2c_b, c2r_b;
  void* work = nullptr;
  // The native transform (native_fft.cu) instead of cuFFT, Green multiply fused into it.
  bool native = false;
  int* slot_peak = nullptr;  // device: peak index of each slot
};

}  // namespace

struct pm_engine {
  int device = 0;
  int flags = 0;
  cudaStream_t stream = nullptr;
  int npeaks = 0;
  std::vector<PeakDesc> peaks;
  std::vector<MeshClass> classes;
  long long ntot = 0, nst = 0, nmodeblk = 0, nsst = 0, nfc = 0, nhc = 0;
  int TSmax = 0;
  size_t smem_dep = 0, smem_push = 0;
  // device arrays
  PeakDesc* d_peaks = nullptr;
  PeakClock* d_clocks = nullptr;
  PeakStats* d_stats = nullptr;
  long long* d_st_base = nullptr;
  unsigned short* d_st_peak = nullptr;  // [super-tile] its peak
  long long* d_p_base = nullptr;
  long long* d_mode_base = nullptr;
  long long* d_green_base = nullptr;  // Green blocks of the peaks that k_green serves
  int* d_green_peak = nullptr;
  int ngreen = 0;
  long long ngreenblk = 0;
  long long rtot = 0;                          // slots of each bin buffer
  int4* bpos[2] = {nullptr, nullptr};          // bin buffers (state, binned by super-tile)
  float4* bmom[2] = {nullptr, nullptr};
  int4* lpos = nullptr;                        // loading area / overflow area
  float4* lmom = nullptr;
  BinLayout* lay[2] = {nullptr, nullptr};      // bin layouts, two generations
  BinFill* fill[2] = {nullptr, nullptr};       // bin fills of the two buffers
  u32* ovf_n = nullptr;                        // [peak] overflow-area particles
  u32* ovf_in = nullptr;                       // [super-tile] overflowed arrivals
  u32* keys[2] = {nullptr, nullptr};
  u32* vals[2] = {nullptr, nullptr};
  u32* sstart = nullptr;
  double2* epart = nullptr;  // push partials of the energy sums
  double* wpart = nullptr;   // Green partials of the potential energy (per warp)
  double2* eslice = nullptr; // energy slice partials
  u32* ecount = nullptr;     // energy slices done per peak
  u32* sort_gate = nullptr;  // one word: any peak primes by sort this step
  u32* layout_gate = nullptr;   // one word: any peak primes or relayouts this step
  u32* refresh_gate = nullptr;  // one word: any peak re-sorts its super-tiles this step
  long long* face = nullptr;
  long long* halo = nullptr;
  SortPlan sort{};       // Morton-key sort used by priming
  int sort_result = 0;   // which (keys, vals) pair holds the sorted output
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // replayed step without / with the priming sort
  bool prime_pending = false;  // a peak was (re)loaded: the next step must include the priming sort
  std::vector<char> occupied;  // host view: slots holding a run (dynamic mode FFT extents)
  long long bytes = 0;
  int* sort_dbg = nullptr;     // device {spin limit, silent tile} of the sort plan (test hook)
  // Host snapshots of the clocks and statistics (pm_snapshot): two pinned buffers, each with the
  // event recorded after its copy.
  struct Snapshot {
    PeakClock* clocks = nullptr;
    PeakStats* stats = nullptr;
    int* err = nullptr;
    cudaEvent_t done = nullptr;
    bool queued = false;
  } snap[2];

  StepArgs args() const {
    StepArgs A{};
    A.peaks = d_peaks;
    A.clocks = d_clocks;
    A.stats = d_stats;
    A.sortseg = sort.seg;
    A.st_base = d_st_base;
    A.st_peak = d_st_peak;
    A.p_base = d_p_base;
    A.mode_base = d_mode_base;
    A.green_base = d_green_base;
    A.green_peak = d_green_peak;
    A.ngreen = ngreen;
    A.epart = epart;
    A.wpart = wpart;
    A.eslice = eslice;
    A.ecount = ecount;
    A.npeaks = npeaks;
    A.pos0 = bpos[0];
    A.mom0 = bmom[0];
    A.pos1 = bpos[1];
    A.mom1 = bmom[1];
    A.lpos = lpos;
    A.lmom = lmom;
    A.lay[0] = lay[0];
    A.lay[1] = lay[1];
    A.fill[0] = fill[0];
    A.fill[1] = fill[1];
    A.ovf_n = ovf_n;
    A.ovf_in = ovf_in;
    A.keys_push = keys[0];
    A.keys_sorted = keys[sort_result];
    A.perm = vals[sort_result];
    A.sstart = sstart;
    A.sort_gate = sort_gate;
    A.layout_gate = layout_gate;
    A.refresh_gate = refresh_gate;
    A.face = face;
    A.halo = halo;
    A.sort_err = sort.err;
    return A;
  }

  template <class T>
  int alloc(T** p, size_t count) {
    const size_t b = sizeof(T) * (count ? count : 1);
    cudaError_t e = cudaMalloc((void**)p, b);
    if (e != cudaSuccess) return -(int)e;
    bytes += (long long)b;
    return 0;
  }

  // Slots in use per class (dynamic mode): transforms run over slots [0, extent).
  int extent(const MeshClass& c) const {
    int x = 0;
    for (int k = 0; k < (int)c.peaks.size(); ++k)
      if (occupied[c.peaks[k]]) x = k + 1;
    return x;
  }
  int fft_r2c() {
    for (auto& c : classes) {
      if (c.native) {
        const int x = (flags & 4) ? extent(c) : (int)c.peaks.size();
        if (int r = fft_native_r2c(c.N, c.delta, c.spec, x, stream)) return r;
      } else if (flags & 4) {
        const int x = extent(c);
        if (x) CF(cufftExecR2C(c.r2c_b[x - 1], c.delta, (cufftComplex*)c.spec));
      } else {
        CF(cufftExecR2C(c.r2c, c.delta, (cufftComplex*)c.spec));
      }
    }
    return 0;
  }
  int fft_c2r() {
    const StepArgs A = args();
    for (auto& c : classes) {
      if (c.native) {
        const int x = (flags & 4) ? extent(c) : (int)c.peaks.size();
        if (int r = fft_native_green_c2r(c.N, c.spec, c.gspec, c.force, A, c.slot_peak, x, stream)) return r;
      } else if (flags & 4) {
        const int x = extent(c);
        if (x) CF(cufftExecC2R(c.c2r_b[x - 1], (cufftComplex*)c.gspec, c.force));
      } else {
        CF(cufftExecC2R(c.c2r, (cufftComplex*)c.gspec, c.force));
      }
    }
    return 0;
  }

  // One step for every peak.  With ev != nullptr an event is recorded after each phase and the
  // phase times (push, energy + advance, relayout, priming sort and refresh, deposit with its face
  // fix-up, R2C, Green, C2R) are accumulated.
  int launch_step(bool with_sort, cudaEvent_t* ev = nullptr, double* phase_ms = nullptr) {
    const StepArgs A = args();
    int k = 0;
    auto mark = [&]() -> cudaError_t { return ev ? cudaEventRecord(ev[k++], stream) : cudaSuccess; };
    CU(mark());
    launch_push(A, nst, smem_push, stream);
    CU(mark());
    launch_energy(A, stream);
    launch_advance(A, stream);
    CU(mark());
    int r = 0;
    if (with_sort) {  // only steps that prime a peak: no sort launches at all in the steady state
      if ((r = sort_run<u32>(&sort, keys[0], vals[0], keys[1], vals[1], true, true, stream))) return r;
      launch_st_starts(A, ntot, stream);
    }
    launch_layout(A, nst, ntot, stream);  // layouts of priming peaks; relayouts (gated, rare)
    if (with_sort) launch_permute(A, ntot, stream);
    CU(mark());
    launch_tile_sort(A, nst, stream);
    CU(mark());
    launch_deposit(A, nst, smem_dep, nullptr, stream);
    launch_fixup(A, nst, nullptr, stream);
    CU(mark());
    if ((r = fft_r2c())) return r;
    CU(mark());
    if (ngreenblk) launch_green(A, ngreenblk, stream);  // the native transform does its own
    CU(mark());
    if ((r = fft_c2r())) return r;
    CU(mark());
    CU(cudaGetLastError());
    if (ev) {
      CU(cudaEventSynchronize(ev[k - 1]));
      for (int q = 0; q + 1 < k; ++q) {
        float ms = 0.f;
        CU(cudaEventElapsedTime(&ms, ev[q], ev[q + 1]));
        phase_ms[q] += ms;
      }
    }
    return 0;
  }

  int step() {
    const bool with_sort = prime_pending;
    prime_pending = false;
    if ((flags & 2) && !(flags & 4)) {
      cudaGraphExec_t& g = graph[with_sort ? 1 : 0];
      if (!g) {
        cudaGraph_t cg = nullptr;
        CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        int r = launch_step(with_sort);
        cudaError_t ce = cudaStreamEndCapture(stream, &cg);
        if (r) return r;
        CU(ce);
        CU(cudaGraphInstantiate(&g, cg, 0));
        cudaGraphDestroy(cg);
      }
      CU(cudaGraphLaunch(g, stream));
      return 0;
    }
    return launch_step(with_sort);
  }
  int step_timed(cudaEvent_t* ev, double* phase_ms) {
    const bool with_sort = prime_pending;
    prime_pending = false;
    return launch_step(with_sort, ev, phase_ms);
  }

  int read_clock(int pk, PeakClock* c) {
    CU(cudaMemcpyAsync(c, d_clocks + pk, sizeof(PeakClock), cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    return 0;
  }
  int write_clock(int pk, const PeakClock& c) {
    if (c.state == PS_PRIME) prime_pending = true;
    CU(cudaMemcpyAsync(d_clocks + pk, &c, sizeof(PeakClock), cudaMemcpyHostToDevice, stream));
    CU(cudaStreamSynchronize(stream));
    return 0;
  }

  ~pm_engine() {
    for (auto g : graph)
      if (g) cudaGraphExecDestroy(g);
    for (auto& c : classes) {
      if (c.plans) {
        cufftDestroy(c.r2c);
        cufftDestroy(c.c2r);
      }
      for (auto h : c.r2c_b) cufftDestroy(h);
      for (auto h : c.c2r_b) cufftDestroy(h);
      cudaFree(c.work);
      cudaFree(c.delta);
      cudaFree(c.spec);
      cudaFree(c.gspec);
      cudaFree(c.force);
      cudaFree(c.slot_peak);
    }
    sort_plan_destroy(&sort);
    for (auto& sn : snap) {
      if (sn.clocks) cudaFreeHost(sn.clocks);
      if (sn.stats) cudaFreeHost(sn.stats);
      if (sn.err) cudaFreeHost(sn.err);
      if (sn.done) cudaEventDestroy(sn.done);
    }
    cudaFree(sort_dbg);
    void* bufs[] = {d_peaks, d_clocks, d_stats, d_st_base, d_st_peak, d_p_base, d_mode_base, d_green_base, d_green_peak, epart,
                    wpart, eslice, ecount, bpos[0], bpos[1], bmom[0], bmom[1], lpos, lmom, lay[0], lay[1],
                    fill[0], fill[1], ovf_n, ovf_in, keys[0], keys[1], vals[0], vals[1], sstart,
                    sort_gate, layout_gate, refresh_gate, face, halo};
    for (void* b : bufs) cudaFree(b);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

void fill_stats(const PeakDesc& P, const PeakStats& s, int sort_err, pm_stats_info* o);

void fill_energy(const PeakStats& s, pm_stats_info* o) {
  o->energy_samples = (int)s.nsamples;
  o->a_energy = s.nsamples ? s.a_e : 0.0;
  for (int k = 0; k < 3; ++k) o->momentum[k] = s.nsamples ? s.mom[k] : 0.0;
  o->kinetic = s.nsamples ? s.kin : 0.0;
  o->potential = s.nsamples ? s.pot : 0.0;
  o->li_residual = s.nsamples ? s.a_e * (s.kin + s.pot) + s.li_int - s.li_e0 : 0.0;
  o->li_scale = s.nsamples ? s.a_e * (s.kin + fabs(s.pot)) : 0.0;
}

void fill_stats(const PeakDesc& P, const PeakStats& s, int sort_err, pm_stats_info* o) {
  o->rho_max_over_mean = (double)s.max_fix / (double)PM_FIX_ONE / P.n_mean;
  o->delta_max = o->rho_max_over_mean - 1.0;
  o->mass_defect = (double)s.mass_defect / (double)PM_FIX_ONE;
  o->status = s.status | (sort_err ? 2u : 0u);
  o->relayouts = (int)s.relayouts;
  o->relayouts_full = (int)s.relayouts_full;
  fill_energy(s, o);
}

void fill_clock(const PeakClock& c, pm_clock_info* o) {
  o->a = c.a;
  o->da = c.da;
  o->a_end = c.a_end;
  o->kpend = c.kpend;
  o->a_grid = c.a_grid;
  o->mode = c.mode;
  o->state = c.state;
  o->nsteps = c.nsteps;
  o->max_steps = c.max_steps;
  o->a_collapse = c.a_collapse;
}

int engine_init(pm_engine* E, const pm_peak_cfg* cfg, int npeaks) {
  E->npeaks = npeaks;
  E->peaks.resize(npeaks);
  E->occupied.assign(npeaks, 0);
  std::map<int, int> class_of;
  long long poff = 0, roff = 0, stb = 0, mb = 0, sso = 0, fo = 0, ho = 0;
  int TSmax = 1, max_bits = 0;
  const int full_every = (E->flags >> 8) & 0xFF;  // 0: never (the default; measured not to pay)
  std::vector<long long> st_base(npeaks + 1), p_base(npeaks + 1), mode_base(npeaks + 1);
  for (int i = 0; i < npeaks; ++i) {
    const pm_peak_cfg& c = cfg[i];
    const int l2 = ilog2(c.N);
    if (l2 < 3 || l2 > 10) return -2001;
    const long long npart = c.n > 0 ? c.n : (long long)c.Np * c.Np * c.Np;
    if (c.Np < 1 || npart >= (1LL << 31)) return -2002;
    if (!(c.L > 0)) return -2003;
    // Super-tile side: 16^3 cells (the whole mesh below that); 4 and 8 are also built.
    const int TS = c.tile > 0 ? c.tile : std::min(16, c.N);
    if (ilog2(TS) < 2 || TS > 16 || TS > c.N) return -2004;
    PeakDesc& P = E->peaks[i];
    P = PeakDesc{};
    P.N = c.N;
    P.log2N = l2;
    P.TS = TS;
    P.log2TS = ilog2(TS);
    P.NS = c.N / TS;
    P.nst = P.NS * P.NS * P.NS;
    P.key_bits = 3 * l2;
    P.st_shift = 3 * P.log2TS;
    P.fc = TS * TS * TS - (TS - 1) * (TS - 1) * (TS - 1);
    P.hc = (TS + 1) * (TS + 1) * (TS + 1) - TS * TS * TS;
    P.gradient = c.gradient;
    P.full_every = full_every;
    // Spare bin capacity: count / 8 + BIN_SLACK_MIN, plus room for BIN_GROW_STEPS steps of growth
    // after a relayout; none with flag bit 16 (a test mode in which almost every step overflows
    // a bin and relayouts).
    const bool tight = (E->flags & (1 << 16)) != 0;
    P.bin_shift = tight ? 32 : BIN_SLACK_SHIFT;
    P.bin_min = tight ? 0 : BIN_SLACK_MIN;
    P.bin_grow = tight ? 0 : BIN_GROW_STEPS;
    P.L = c.L;
    P.dx = c.L / c.N;
    P.smooth = c.smooth;
    const double np3 = (double)c.Np * c.Np * c.Np;
    P.n_mean = (double)npart / ((double)c.N * c.N * c.N);
    P.m_part = 3.0 * PM_H_I * PM_H_I / (8.0 * M_PI) * c.L * c.L * c.L / np3;
    P.n_mean_fix = (long long)llround(P.n_mean * (double)PM_FIX_ONE);
    P.inv_fix_nmean = 1.0 / ((double)PM_FIX_ONE * P.n_mean);
    P.p_off = poff;
    P.n = npart;
    // Bin region: every base layout k_layout makes (count + count/8 + BIN_SLACK_MIN per bin,
    // rounded up to BIN_ALIGN) fits in n + n/8 + (BIN_SLACK_MIN + BIN_ALIGN) per super-tile; a
    // further n >> BIN_SPARE_SHIFT slots hold the allowance for arrivals and growth of relayouts.
    P.r_off = roff;
    P.r_size = (npart + (npart >> BIN_SLACK_SHIFT) + (npart >> BIN_SPARE_SHIFT) +
                (long long)(BIN_SLACK_MIN + BIN_ALIGN) * P.nst + BIN_ALIGN - 1) / BIN_ALIGN * BIN_ALIGN;
    roff += P.r_size;
    P.st_base = stb;
    P.sst_off = sso;
    P.face_off = fo;
    P.halo_off = ho;
    P.nmodes = (long long)c.N * c.N * (c.N / 2 + 1);
    pm_div_magic((u32)(c.N / 2 + 1), &P.nh_magic, &P.nh_shift);
    P.mode_base = mb;
    st_base[i] = stb;
    p_base[i] = poff;
    mode_base[i] = mb;
    poff += P.n;
    stb += P.nst;
    sso += P.nst + 1;
    fo += (long long)P.nst * P.fc;
    ho += (long long)P.nst * P.hc;
    mb += (P.nmodes + PM_THREADS * GREEN_MODES - 1) / (PM_THREADS * GREEN_MODES);
    TSmax = std::max(TSmax, TS);
    max_bits = std::max(max_bits, P.key_bits);
    if (!class_of.count(c.N)) {
      class_of[c.N] = (int)E->classes.size();
      E->classes.push_back(MeshClass{});
      E->classes.back().N = c.N;
    }
    E->classes[class_of[c.N]].peaks.push_back(i);
  }
  st_base[npeaks] = stb;
  p_base[npeaks] = poff;
  mode_base[npeaks] = mb;
  if (poff >= (1LL << 32) || roff >= (1LL << 32)) return -2005;
  E->ntot = poff;
  E->rtot = roff;
  E->nst = stb;
  E->nmodeblk = mb;
  E->nsst = sso;
  E->nfc = fo;
  E->nhc = ho;
  E->TSmax = TSmax;
  if (int rk = pm_kernels_init()) return rk;
  E->smem_dep = pm_deposit_smem(TSmax);
  E->smem_push = pm_push_smem(TSmax);

  // Mesh arenas, one per mesh size, peaks of a class contiguous for batched cuFFT plans.
  for (auto& mc : E->classes) {
    const long long N = mc.N, N3 = N * N * N, M = N * N * (N / 2 + 1);
    const int B = (int)mc.peaks.size();
    int r;
    if ((r = E->alloc(&mc.delta, (size_t)(B * N3)))) return r;
    if ((r = E->alloc(&mc.spec, (size_t)(B * M)))) return r;
    if ((r = E->alloc(&mc.gspec, (size_t)(3 * B * M)))) return r;
    if ((r = E->alloc(&mc.force, (size_t)(3 * B * N3)))) return r;
    CU(cudaMemsetAsync(mc.delta, 0, sizeof(float) * B * N3, E->stream));
    CU(cudaMemsetAsync(mc.force, 0, sizeof(float) * 3 * B * N3, E->stream));
    for (int k = 0; k < B; ++k) {
      PeakDesc& P = E->peaks[mc.peaks[k]];
      P.delta = mc.delta + k * N3;
      P.spec = mc.spec + k * M;
      P.gspec = mc.gspec + 3 * k * M;
      P.force = mc.force + 3 * k * N3;
    }
    int n[3] = {(int)N, (int)N, (int)N};
    if ((E->flags & 8) && fft_native_size((int)N)) {
      mc.native = true;
      if ((r = E->alloc(&mc.slot_peak, (size_t)B))) return r;
      CU(cudaMemcpy(mc.slot_peak, mc.peaks.data(), sizeof(int) * B, cudaMemcpyHostToDevice));
      for (int k = 0; k < B; ++k) E->peaks[mc.peaks[k]].native_fft = 1;
      if ((r = fft_native_init())) return r;
    } else if (E->flags & 4) {
      // Dynamic mode: a plan per batch size, all sharing the largest work area, so a step
      // transforms only the slots up to the highest one in use.
      size_t wmax = 0;
      for (int b = 1; b <= B; ++b) {
        cufftHandle h1, h2;
        size_t w1 = 0, w2 = 0;
        CF(cufftCreate(&h1));
        CF(cufftCreate(&h2));
        CF(cufftSetAutoAllocation(h1, 0));
        CF(cufftSetAutoAllocation(h2, 0));
        CF(cufftMakePlanMany(h1, 3, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C, b, &w1));
        CF(cufftMakePlanMany(h2, 3, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2R, 3 * b, &w2));
        CF(cufftSetStream(h1, E->stream));
        CF(cufftSetStream(h2, E->stream));
        mc.r2c_b.push_back(h1);
        mc.c2r_b.push_back(h2);
        wmax = std::max(wmax, std::max(w1, w2));
      }
      int rr;
      if ((rr = E->alloc((char**)&mc.work, wmax))) return rr;
      for (int b = 0; b < B; ++b) {
        CF(cufftSetWorkArea(mc.r2c_b[b], mc.work));
        CF(cufftSetWorkArea(mc.c2r_b[b], mc.work));
      }
    } else {
      CF(cufftPlanMany(&mc.r2c, 3, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C, B));
      CF(cufftPlanMany(&mc.c2r, 3, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2R, 3 * B));
      mc.plans = true;
      CF(cufftSetStream(mc.r2c, E->stream));
      CF(cufftSetStream(mc.c2r, E->stream));
      size_t ws = 0;
      if (cufftGetSize(mc.r2c, &ws) == CUFFT_SUCCESS) E->bytes += (long long)ws;
      if (cufftGetSize(mc.c2r, &ws) == CUFFT_SUCCESS) E->bytes += (long long)ws;
    }
  }

  int r;
  if ((r = E->alloc(&E->d_peaks, npeaks))) return r;
  if ((r = E->alloc(&E->d_clocks, npeaks))) return r;
  if ((r = E->alloc(&E->d_stats, npeaks))) return r;
  if ((r = E->alloc(&E->d_st_base, npeaks + 1))) return r;
  if ((r = E->alloc(&E->d_p_base, npeaks + 1))) return r;
  if ((r = E->alloc(&E->d_mode_base, npeaks + 1))) return r;
  // The Green kernel's grid covers only the peaks without the native transform.
  std::vector<long long> green_base(1, 0);
  std::vector<int> green_peak;
  for (int i = 0; i < npeaks; ++i)
    if (!E->peaks[i].native_fft) {
      green_peak.push_back(i);
      green_base.push_back(green_base.back() + (mode_base[i + 1] - mode_base[i]));
    }
  E->ngreen = (int)green_peak.size();
  E->ngreenblk = green_base.back();
  if ((r = E->alloc(&E->d_green_base, green_base.size()))) return r;
  if ((r = E->alloc(&E->d_green_peak, green_peak.size()))) return r;
  CU(cudaMemcpy(E->d_green_base, green_base.data(), sizeof(long long) * green_base.size(), cudaMemcpyHostToDevice));
  if (E->ngreen)
    CU(cudaMemcpy(E->d_green_peak, green_peak.data(), sizeof(int) * green_peak.size(), cudaMemcpyHostToDevice));
  for (int b = 0; b < 2; ++b) {
    if ((r = E->alloc(&E->bpos[b], E->rtot))) return r;
    if ((r = E->alloc(&E->bmom[b], E->rtot))) return r;
    if ((r = E->alloc(&E->lay[b], E->nst))) return r;
    if ((r = E->alloc(&E->fill[b], E->nst))) return r;
    if ((r = E->alloc(&E->keys[b], E->ntot))) return r;
    if ((r = E->alloc(&E->vals[b], E->ntot))) return r;
  }
  if ((r = E->alloc(&E->lpos, E->ntot))) return r;
  if ((r = E->alloc(&E->lmom, E->ntot))) return r;
  if ((r = E->alloc(&E->sstart, E->nsst))) return r;
  if ((r = E->alloc(&E->ovf_n, npeaks))) return r;
  if ((r = E->alloc(&E->ovf_in, E->nst))) return r;
  if ((r = E->alloc(&E->epart, 4 * E->nst))) return r;
  if ((r = E->alloc(&E->wpart, E->nmodeblk * (PM_THREADS / 32)))) return r;
  if ((r = E->alloc(&E->eslice, (size_t)npeaks * ENERGY_SLICES * 5))) return r;
  if ((r = E->alloc(&E->ecount, npeaks))) return r;
  if ((r = E->alloc(&E->sort_gate, 1))) return r;
  if ((r = E->alloc(&E->layout_gate, 1))) return r;
  if ((r = E->alloc(&E->refresh_gate, 1))) return r;
  if ((r = E->alloc(&E->face, E->nfc))) return r;
  if ((r = E->alloc(&E->halo, E->nhc))) return r;
  CU(cudaMemcpy(E->d_peaks, E->peaks.data(), sizeof(PeakDesc) * npeaks, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(E->d_st_base, st_base.data(), sizeof(long long) * (npeaks + 1), cudaMemcpyHostToDevice));
  {
    std::vector<unsigned short> stp((size_t)E->nst);
    for (int i = 0; i < npeaks; ++i)
      for (long long t = st_base[i]; t < st_base[i + 1]; ++t) stp[(size_t)t] = (unsigned short)i;
    if ((r = E->alloc(&E->d_st_peak, E->nst))) return r;
    CU(cudaMemcpy(E->d_st_peak, stp.data(), sizeof(unsigned short) * E->nst, cudaMemcpyHostToDevice));
  }
  CU(cudaMemcpy(E->d_p_base, p_base.data(), sizeof(long long) * (npeaks + 1), cudaMemcpyHostToDevice));
  CU(cudaMemcpy(E->d_mode_base, mode_base.data(), sizeof(long long) * (npeaks + 1), cudaMemcpyHostToDevice));
  std::vector<PeakClock> clocks(npeaks);
  for (auto& c : clocks) {
    c = PeakClock{};
    c.state = PS_IDLE;
    c.a_collapse = -1.0;
  }
  CU(cudaMemcpy(E->d_clocks, clocks.data(), sizeof(PeakClock) * npeaks, cudaMemcpyHostToDevice));
  CU(cudaMemset(E->d_stats, 0, sizeof(PeakStats) * npeaks));
  for (int b = 0; b < 2; ++b) {
    CU(cudaMemset(E->bpos[b], 0, sizeof(int4) * E->rtot));
    CU(cudaMemset(E->bmom[b], 0, sizeof(float4) * E->rtot));
    CU(cudaMemset(E->lay[b], 0, sizeof(BinLayout) * E->nst));
    CU(cudaMemset(E->fill[b], 0, sizeof(BinFill) * E->nst));
  }
  CU(cudaMemset(E->lpos, 0, sizeof(int4) * E->ntot));
  CU(cudaMemset(E->lmom, 0, sizeof(float4) * E->ntot));
  CU(cudaMemset(E->ovf_n, 0, sizeof(u32) * npeaks));
  CU(cudaMemset(E->ovf_in, 0, sizeof(u32) * E->nst));
  CU(cudaMemset(E->layout_gate, 0, sizeof(u32)));
  CU(cudaMemset(E->epart, 0, sizeof(double2) * 4 * E->nst));
  CU(cudaMemset(E->wpart, 0, sizeof(double) * E->nmodeblk * (PM_THREADS / 32)));
  CU(cudaMemset(E->ecount, 0, sizeof(u32) * npeaks));
  CU(cudaMemset(E->sort_gate, 0, sizeof(u32)));
  CU(cudaMemset(E->refresh_gate, 0, sizeof(u32)));
  CU(cudaMemset(E->sstart, 0, sizeof(u32) * E->nsst));

  // Sort plan: one segment per peak over the whole Morton key (sorted at priming and every
  // full_every steps; the segment of a peak is active only on those steps).
  std::vector<SortSeg> segs(npeaks);
  for (int i = 0; i < npeaks; ++i) {
    const PeakDesc& P = E->peaks[i];
    segs[i] = SortSeg{P.p_off, P.p_off + P.n, 0, P.key_bits, 0, 0};
  }
  const int np = (max_bits + SORT_MAX_BITS - 1) / SORT_MAX_BITS;
  if ((r = sort_plan_create(&E->sort, segs.data(), npeaks, np, max_bits))) return r;
  E->sort.gate = E->sort_gate;
  E->bytes += (long long)E->sort.ntiles * 8 * (1LL << E->sort.bits);
  if ((r = E->alloc(&E->sort_dbg, 2))) return r;
  const int dbg0[2] = {SORT_SPIN_LIMIT, -1};
  CU(cudaMemcpy(E->sort_dbg, dbg0, sizeof(dbg0), cudaMemcpyHostToDevice));
  E->sort.dbg = E->sort_dbg;
  // The sorted key and value buffers start defined, so a sort that fails can only leave
  // values that were once valid for this engine behind.
  for (int b = 0; b < 2; ++b) {
    CU(cudaMemset(E->keys[b], 0, sizeof(u32) * E->ntot));
    CU(cudaMemset(E->vals[b], 0, sizeof(u32) * E->ntot));
  }
  for (auto& sn : E->snap) {
    CU(cudaMallocHost((void**)&sn.clocks, sizeof(PeakClock) * npeaks));
    CU(cudaMallocHost((void**)&sn.stats, sizeof(PeakStats) * npeaks));
    CU(cudaMallocHost((void**)&sn.err, sizeof(int) * npeaks));
    CU(cudaEventCreateWithFlags(&sn.done, cudaEventDisableTiming));
  }
  E->sort_result = np & 1;
  CU(cudaDeviceSynchronize());
  return 0;
}

}  // namespace

extern "C" {

int pm_engine_create(const pm_peak_cfg* cfg, int npeaks, int device, int flags, pm_engine** out) {
  if (!cfg || npeaks < 1 || npeaks > 65535 || !out) return -2000;  // peaks indexed by 16 bits
  *out = nullptr;
  CU(cudaSetDevice(device));
  pm_engine* E = new (std::nothrow) pm_engine();
  if (!E) return -2;
  E->device = device;
  E->flags = flags;
  cudaError_t ce = cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking);
  if (ce != cudaSuccess) {
    delete E;
    return -(int)ce;
  }
  int r = engine_init(E, cfg, npeaks);
  if (r) {
    delete E;
    return r;
  }
  *out = E;
  return 0;
}

int pm_engine_destroy(pm_engine* e) {
  if (!e) return -2000;
  cudaSetDevice(e->device);
  cudaStreamSynchronize(e->stream);
  delete e;
  return 0;
}

int pm_engine_sync(pm_engine* e) {
  if (!e) return -2000;
  CU(cudaStreamSynchronize(e->stream));
  return 0;
}

long long pm_engine_device_bytes(const pm_engine* e) { return e ? e->bytes : 0; }

int pm_set_particles(pm_engine* e, int peak, const double* x, const double* p, double a0, int mode, double param,
                     double a_end, int max_steps) {
  if (!e || peak < 0 || peak >= e->npeaks || !x || !p) return -2000;
  if (!(a0 > 0) || mode < 0 || mode > 2) return -2001;
  CU(cudaSetDevice(e->device));
  const StepArgs A = e->args();
  launch_reset_peak(A, peak, a0, mode, param, a_end, max_steps, 0, 0.0, 0, e->stream);
  e->prime_pending = true;
  launch_set_particles(A, peak, e->peaks[peak], x, p, e->stream);
  e->occupied[peak] = 1;
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(e->stream));
  return 0;
}

int pm_run(pm_engine* e, int nsteps) {
  if (!e || nsteps < 0) return -2000;
  CU(cudaSetDevice(e->device));
  for (int s = 0; s < nsteps; ++s) {
    int r = e->step();
    if (r) return r;
  }
  return 0;
}

int pm_run_timed(pm_engine* e, int nsteps, double* phase_ms) {
  if (!e || nsteps < 0 || !phase_ms) return -2000;
  CU(cudaSetDevice(e->device));
  cudaEvent_t ev[10];
  for (int k = 0; k < 10; ++k) CU(cudaEventCreate(&ev[k]));
  int r = 0;
  for (int s = 0; s < nsteps && !r; ++s) r = e->step_timed(ev, phase_ms);
  for (int k = 0; k < 10; ++k) cudaEventDestroy(ev[k]);
  return r;
}

void* pm_engine_stream(pm_engine* e) { return e ? (void*)e->stream : nullptr; }

int pm_engine_info(const pm_engine* e, long long* info) {
  if (!e || !info) return -2000;
  info[0] = e->npeaks;
  info[1] = e->ntot;
  info[2] = e->nst;
  info[3] = e->sort.npass;
  info[4] = (long long)e->classes.size();
  info[5] = e->bytes;
  return 0;
}

int pm_get_stats_all(pm_engine* e, pm_stats_info* out) {
  if (!e || !out) return -2000;
  CU(cudaSetDevice(e->device));
  std::vector<PeakStats> s(e->npeaks);
  std::vector<int> err(e->npeaks);
  CU(cudaMemcpyAsync(s.data(), e->d_stats, sizeof(PeakStats) * e->npeaks, cudaMemcpyDeviceToHost, e->stream));
  CU(cudaMemcpyAsync(err.data(), e->sort.err, sizeof(int) * e->npeaks, cudaMemcpyDeviceToHost, e->stream));
  CU(cudaStreamSynchronize(e->stream));
  int flagged = 0;
  for (int i = 0; i < e->npeaks; ++i) {
    fill_stats(e->peaks[i], s[i], err[i], &out[i]);
    flagged += out[i].status != 0;
  }
  return flagged;
}

int pm_get_clocks_all(pm_engine* e, pm_clock_info* out) {
  if (!e || !out) return -2000;
  CU(cudaSetDevice(e->device));
  std::vector<PeakClock> c(e->npeaks);
  CU(cudaMemcpyAsync(c.data(), e->d_clocks, sizeof(PeakClock) * e->npeaks, cudaMemcpyDeviceToHost, e->stream));
  CU(cudaStreamSynchronize(e->stream));
  for (int i = 0; i < e->npeaks; ++i) fill_clock(c[i], &out[i]);
  return 0;
}

int pm_step_explicit(pm_engine* e, int peak, double a, double da) {
  if (!e || peak < 0 || peak >= e->npeaks) return -2000;
  if (!(a > 0) || !(da > 0)) return -2001;
  CU(cudaSetDevice(e->device));
  PeakClock c;
  int r;
  if ((r = e->read_clock(peak, &c))) return r;
  // Bring the peak to "forces known at a" (pm3d.py:119-120).
  if (c.state == PS_HOLD && c.a != a) {
    c.state = PS_FINALIZE;  // apply the pending kick with the grids it belongs to
    if ((r = e->write_clock(peak, c)) || (r = e->step()) || (r = e->read_clock(peak, &c))) return r;
  }
  if (c.state == PS_IDLE || c.state == PS_PRIME || (c.state == PS_HOLD && !c.has_delta)) {
    // A loaded peak (PRIME) has its particles in the loading area already; any other state
    // holds them in the grouped state, from where they are reloaded for the priming sort.
    if (c.state != PS_PRIME) launch_reload(e->args(), peak, e->peaks[peak], e->stream);
    c.a = a;
    c.a_grid = a;
    c.mode = SCHED_EXPLICIT;
    c.state = PS_PRIME;
    if ((r = e->write_clock(peak, c)) || (r = e->step()) || (r = e->read_clock(peak, &c))) return r;
  }
  if (c.state != PS_HOLD) return -2002;
  c.mode = SCHED_EXPLICIT;
  c.da = da;
  c.state = PS_RUN;
  if ((r = e->write_clock(peak, c)) || (r = e->step())) return r;
  CU(cudaStreamSynchronize(e->stream));
  return 0;
}

int pm_get_particles(pm_engine* e, int peak, double* x, double* p) {
  if (!e || peak < 0 || peak >= e->npeaks) return -2000;
  CU(cudaSetDevice(e->device));
  launch_get_particles(e->args(), peak, e->peaks[peak], x, p, nullptr, 1.0, e->stream);
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(e->stream));
  return 0;
}

int pm_get_acc(pm_engine* e, int peak, double a, double* acc) {
  if (!e || peak < 0 || peak >= e->npeaks || !acc) return -2000;
  if (!(a > 0)) return -2001;
  CU(cudaSetDevice(e->device));
  launch_get_particles(e->args(), peak, e->peaks[peak], nullptr, nullptr, acc, a, e->stream);
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(e->stream));
  return 0;
}

int pm_get_delta(pm_engine* e, int peak, float* delta) {
  if (!e || peak < 0 || peak >= e->npeaks || !delta) return -2000;
  CU(cudaSetDevice(e->device));
  const PeakDesc& P = e->peaks[peak];
  CU(cudaMemcpyAsync(delta, P.delta, sizeof(float) * (size_t)P.N * P.N * P.N, cudaMemcpyDeviceToDevice, e->stream));
  CU(cudaStreamSynchronize(e->stream));
  return 0;
}

int pm_get_counts(pm_engine* e, int peak, double* counts) {
  if (!e || peak < 0 || peak >= e->npeaks || !counts) return -2000;
  CU(cudaSetDevice(e->device));
  // Re-deposit the current positions of this peak only, writing float64 counts.
  PeakClock c;
  int r;
  if ((r = e->read_clock(peak, &c))) return r;
  if (!c.has_delta) return -2002;
  std::vector<PeakClock> all(e->npeaks);
  CU(cudaMemcpy(all.data(), e->d_clocks, sizeof(PeakClock) * e->npeaks, cudaMemcpyDeviceToHost));
  std::vector<PeakClock> tmp = all;
  for (int i = 0; i < e->npeaks; ++i) tmp[i].dep = i == peak ? 1 : 0;
  CU(cudaMemcpy(e->d_clocks, tmp.data(), sizeof(PeakClock) * e->npeaks, cudaMemcpyHostToDevice));
  PeakStats st;
  CU(cudaMemcpy(&st, e->d_stats + peak, sizeof(PeakStats), cudaMemcpyDeviceToHost));
  st.max_fix = 0;
  st.mass_defect = 0;
  CU(cudaMemcpy(e->d_stats + peak, &st, sizeof(PeakStats), cudaMemcpyHostToDevice));
  // Same kernels with the extra float64 output; delta is rewritten with identical values.
  launch_deposit(e->args(), e->nst, e->smem_dep, counts, e->stream);
  launch_fixup(e->args(), e->nst, counts, e->stream);
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(e->stream));
  CU(cudaMemcpy(e->d_clocks, all.data(), sizeof(PeakClock) * e->npeaks, cudaMemcpyHostToDevice));
  return 0;
}

int pm_set_collapse_threshold(pm_engine* e, int peak, double delta_collapse, int stop) {
  if (!e || peak < 0 || peak >= e->npeaks) return -2000;
  CU(cudaSetDevice(e->device));
  PeakClock c;
  int r;
  if ((r = e->read_clock(peak, &c))) return r;
  c.delta_collapse = delta_collapse;
  c.stop_on_collapse = stop ? 1 : 0;
  return e->write_clock(peak, c);
}

int pm_release(pm_engine* e, int peak) {
  if (!e || peak < 0 || peak >= e->npeaks) return -2000;
  CU(cudaSetDevice(e->device));
  launch_release_peak(e->args(), peak, e->stream);
  CU(cudaGetLastError());
  e->occupied[peak] = 0;
  return 0;
}

int pm_load_peak(pm_engine* e, int peak, const double* x, const double* p, double a0, int mode, double param,
                 double a_end, int max_steps, double delta_collapse, int stop, void* wait_event) {
  if (!e || peak < 0 || peak >= e->npeaks || !x || !p) return -2000;
  if (!(a0 > 0) || mode < 0 || mode > 2) return -2001;
  CU(cudaSetDevice(e->device));
  if (wait_event) CU(cudaStreamWaitEvent(e->stream, (cudaEvent_t)wait_event, 0));
  const StepArgs A = e->args();
  launch_reset_peak(A, peak, a0, mode, param, a_end, max_steps, 1, delta_collapse, stop, e->stream);
  launch_set_particles(A, peak, e->peaks[peak], x, p, e->stream);
  CU(cudaGetLastError());
  e->prime_pending = true;
  e->occupied[peak] = 1;
  return 0;
}

int pm_snapshot(pm_engine* e, int slot) {
  if (!e || slot < 0 || slot > 1) return -2000;
  CU(cudaSetDevice(e->device));
  auto& sn = e->snap[slot];
  const int n = e->npeaks;
  CU(cudaMemcpyAsync(sn.clocks, e->d_clocks, sizeof(PeakClock) * n, cudaMemcpyDeviceToHost, e->stream));
  CU(cudaMemcpyAsync(sn.stats, e->d_stats, sizeof(PeakStats) * n, cudaMemcpyDeviceToHost, e->stream));
  CU(cudaMemcpyAsync(sn.err, e->sort.err, sizeof(int) * n, cudaMemcpyDeviceToHost, e->stream));
  CU(cudaEventRecord(sn.done, e->stream));
  sn.queued = true;
  return 0;
}

int pm_snapshot_read(pm_engine* e, int slot, int wait, pm_clock_info* clocks, pm_stats_info* stats) {
  if (!e || slot < 0 || slot > 1) return -2000;
  auto& sn = e->snap[slot];
  if (!sn.queued) return -2001;
  CU(cudaSetDevice(e->device));
  if (!wait) {
    const cudaError_t q = cudaEventQuery(sn.done);
    if (q == cudaErrorNotReady) return 1;
    if (q != cudaSuccess) return -(int)q;
  } else {
    CU(cudaEventSynchronize(sn.done));
  }
  for (int i = 0; i < e->npeaks; ++i) {
    if (clocks) fill_clock(sn.clocks[i], &clocks[i]);
    if (stats) fill_stats(e->peaks[i], sn.stats[i], sn.err[i], &stats[i]);
  }
  return 0;
}

int pm_get_delta_async(pm_engine* e, int peak, void* dst) {
  if (!e || peak < 0 || peak >= e->npeaks || !dst) return -2000;
  CU(cudaSetDevice(e->device));
  const PeakDesc& P = e->peaks[peak];
  CU(cudaMemcpyAsync(dst, P.delta, sizeof(float) * (size_t)P.N * P.N * P.N, cudaMemcpyDefault, e->stream));
  return 0;
}

int pm_debug_sort_stall(pm_engine* e, int peak, int spin_limit) {
  if (!e || peak >= e->npeaks) return -2000;
  CU(cudaSetDevice(e->device));
  int v[2] = {SORT_SPIN_LIMIT, -1};
  if (peak >= 0 && spin_limit > 0) {
    long long tile = 0;  // the first tile of the peak's segment (segments in peak order)
    for (int i = 0; i < peak; ++i) tile += (e->peaks[i].n + SORT_TILE - 1) / SORT_TILE;
    if (e->peaks[peak].n <= SORT_TILE) return -2001;  // no successor tile waits on the first one
    v[0] = spin_limit;
    v[1] = (int)tile;
  }
  CU(cudaMemcpyAsync(e->sort_dbg, v, sizeof(v), cudaMemcpyHostToDevice, e->stream));
  CU(cudaStreamSynchronize(e->stream));
  return 0;
}

int pm_get_clock(pm_engine* e, int peak, pm_clock_info* out) {
  if (!e || peak < 0 || peak >= e->npeaks || !out) return -2000;
  CU(cudaSetDevice(e->device));
  PeakClock c;
  int r = e->read_clock(peak, &c);
  if (r) return r;
  fill_clock(c, out);
  return 0;
}

int pm_get_stats(pm_engine* e, int peak, pm_stats_info* out) {
  if (!e || peak < 0 || peak >= e->npeaks || !out) return -2000;
  CU(cudaSetDevice(e->device));
  PeakStats s;
  int err = 0;
  CU(cudaMemcpyAsync(&s, e->d_stats + peak, sizeof(PeakStats), cudaMemcpyDeviceToHost, e->stream));
  CU(cudaMemcpyAsync(&err, e->sort.err + peak, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  CU(cudaStreamSynchronize(e->stream));
  fill_stats(e->peaks[peak], s, err, out);
  return (int)(out->status != 0);
}

int pm_interp64(const double* F, const double* X, long long n, int N, double L, double* out) {
  if (!F || !X || !out || n < 0 || N < 1 || !(L > 0)) return -2000;
  if (n == 0) return 0;
  launch_interp64(F, X, n, N, L / N, out, 0);
  CU(cudaGetLastError());
  CU(cudaDeviceSynchronize());
  return 0;
}

int pm_deposit64(const double* X, long long n, int N, double L, unsigned long long* work, double* counts) {
  if (!X || !work || !counts || n < 0 || N < 1 || !(L > 0)) return -2000;
  launch_deposit64(X, n, N, L / N, (u64*)work, counts, 0);
  CU(cudaGetLastError());
  CU(cudaDeviceSynchronize());
  return 0;
}

int pm_sort_u64(const unsigned long long* keys, unsigned long long* keys_out, unsigned int* perm_out,
                unsigned long long* tmp_keys, unsigned int* tmp_vals, long long n, int lo, int hi) {
  if (!keys || !keys_out || !perm_out || !tmp_keys || !tmp_vals || n < 0) return -2000;
  if (lo < 0 || hi > 64 || hi <= lo) return -2001;
  if (n >= (1LL << 32)) return -2002;
  if (n == 0) return 0;
  SortSeg seg{0, n, lo, hi, 1, 0};
  SortPlan plan;
  const int npass = (hi - lo + 7) / 8;
  int r = sort_plan_create(&plan, &seg, 1, npass, hi - lo);
  if (r) {
    sort_plan_destroy(&plan);
    return r;
  }
  // Even pass counts land in the first pair, odd in the second: route so that the final
  // pass writes (keys_out, perm_out).
  u64* k0 = (u64*)tmp_keys;
  u32* v0 = tmp_vals;
  u64* k1 = (u64*)keys_out;
  u32* v1 = perm_out;
  if ((npass & 1) == 0) {
    k0 = (u64*)keys_out;
    v0 = perm_out;
    k1 = (u64*)tmp_keys;
    v1 = tmp_vals;
  }
  cudaError_t ce = cudaMemcpy(k0, keys, sizeof(u64) * n, cudaMemcpyDeviceToDevice);
  if (ce == cudaSuccess) {
    r = sort_run<u64>(&plan, k0, v0, k1, v1, true, true, 0);
    ce = cudaDeviceSynchronize();
  }
  int err = 0;
  if (ce == cudaSuccess) ce = cudaMemcpy(&err, plan.err, sizeof(int), cudaMemcpyDeviceToHost);
  sort_plan_destroy(&plan);
  if (ce != cudaSuccess) return -(int)ce;
  if (r) return r;
  return err ? 1 : 0;
}

int pm_cell_keys(const int* cells, long long n, int N, int tile, unsigned int* keys_out) {
  // Host-side helper (plain host pointers): the key the sort orders particles by.  `tile` is
  // accepted for the layout's super-tile but does not change the key (Morton codes nest).
  if (!cells || !keys_out || n < 0) return -2000;
  const int l2 = ilog2(N);
  if (l2 < 1 || tile < 0 || tile > N) return -2001;
  for (long long i = 0; i < n; ++i) {
    const int c = cells[i];
    keys_out[i] = pm_cell_key(c >> (2 * l2), (c >> l2) & (N - 1), c & (N - 1));
  }
  return 0;
}

}  // extern "C"
