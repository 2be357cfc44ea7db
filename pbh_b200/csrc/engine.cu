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
};

}  // namespace

struct pm_engine {
  int device = 0;
  int flags = 0;
  cudaStream_t stream = nullptr;
  int npeaks = 0;
  std::vector<PeakDesc> peaks;
  std::vector<MeshClass> classes;
  long long ntot = 0, ntiles = 0, nptiles = 0, nmodeblk = 0, nbuckets = 0;
  int Tmax = 0;
  size_t smem_dep = 0, smem_push = 0;
  // device arrays
  PeakDesc* d_peaks = nullptr;
  PeakClock* d_clocks = nullptr;
  PeakStats* d_stats = nullptr;
  long long* d_tile_base = nullptr;
  long long* d_ptile_base = nullptr;
  long long* d_p_base = nullptr;
  long long* d_mode_base = nullptr;
  int4* pos[2] = {nullptr, nullptr};
  float4* mom[2] = {nullptr, nullptr};
  u32* keys[2] = {nullptr, nullptr};
  u32* vals[2] = {nullptr, nullptr};
  u32* bstart = nullptr;
  SortPlan sort{};       // per-step sort: bucket bits only when full_every > 1
  SortPlan sort_full{};  // whole cell key
  int full_every = 1;    // full-key sort every this many steps
  long long replays = 0;
  int sort_result = 0;  // which (keys, vals) pair holds the sorted output (same for both plans)
  cudaGraphExec_t graph = nullptr, graph_full = nullptr;
  std::vector<char> occupied;  // host view: slots holding a run (dynamic mode FFT extents)
  long long bytes = 0;

  StepArgs args() const {
    StepArgs A{};
    A.peaks = d_peaks;
    A.clocks = d_clocks;
    A.stats = d_stats;
    A.sortseg = sort.seg;
    A.sortseg_full = sort_full.seg;
    A.tile_base = d_tile_base;
    A.ptile_base = d_ptile_base;
    A.p_base = d_p_base;
    A.mode_base = d_mode_base;
    A.npeaks = npeaks;
    A.pos[0] = pos[0];
    A.pos[1] = pos[1];
    A.mom[0] = mom[0];
    A.mom[1] = mom[1];
    A.keys_push = keys[0];
    A.keys_sorted = keys[sort_result];
    A.perm = vals[sort_result];
    A.bstart = bstart;
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

  int launch_step(bool full) {
    const StepArgs A = args();
    SortPlan& plan = full ? sort_full : sort;
    launch_push(A, nptiles, smem_push, stream);
    launch_advance(A, stream);
    int r = sort_run<u32>(&plan, keys[0], vals[0], keys[1], vals[1], true, true, stream);
    if (r) return r;
    launch_bucket_starts(A, ntot, stream);
    launch_deposit(A, nptiles, smem_dep, nullptr, stream);
    int r2 = fft_r2c();
    if (r2) return r2;
    launch_green(A, nmodeblk, stream);
    if ((r2 = fft_c2r())) return r2;
    CU(cudaGetLastError());
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
      if (flags & 4) {
        const int x = extent(c);
        if (x) CF(cufftExecR2C(c.r2c_b[x - 1], c.delta, (cufftComplex*)c.spec));
      } else {
        CF(cufftExecR2C(c.r2c, c.delta, (cufftComplex*)c.spec));
      }
    }
    return 0;
  }
  int fft_c2r() {
    for (auto& c : classes) {
      if (flags & 4) {
        const int x = extent(c);
        if (x) CF(cufftExecC2R(c.c2r_b[x - 1], (cufftComplex*)c.gspec, c.force));
      } else {
        CF(cufftExecC2R(c.c2r, (cufftComplex*)c.gspec, c.force));
      }
    }
    return 0;
  }

  // Whether this engine step sorts the full cell key (the in-tile Morton order is refreshed)
  // or only the bucket bits the deposit and push depend on.
  bool next_full() const { return full_every <= 1 || (replays % full_every) == 0; }

  // The step with an event between phases, for per-kernel device times (phase_ms accumulates).
  int launch_step_timed(cudaEvent_t* ev, double* phase_ms) {
    const StepArgs A = args();
    CU(cudaEventRecord(ev[0], stream));
    launch_push(A, nptiles, smem_push, stream);
    CU(cudaEventRecord(ev[1], stream));
    launch_advance(A, stream);
    CU(cudaEventRecord(ev[2], stream));
    const bool full = next_full();
    ++replays;
    int r = sort_run<u32>(full ? &sort_full : &sort, keys[0], vals[0], keys[1], vals[1], true, true, stream);
    if (r) return r;
    CU(cudaEventRecord(ev[3], stream));
    launch_bucket_starts(A, ntot, stream);
    CU(cudaEventRecord(ev[4], stream));
    launch_deposit(A, nptiles, smem_dep, nullptr, stream);
    CU(cudaEventRecord(ev[5], stream));
    if ((r = fft_r2c())) return r;
    CU(cudaEventRecord(ev[6], stream));
    launch_green(A, nmodeblk, stream);
    CU(cudaEventRecord(ev[7], stream));
    if ((r = fft_c2r())) return r;
    CU(cudaEventRecord(ev[8], stream));
    CU(cudaEventSynchronize(ev[8]));
    for (int k = 0; k < 8; ++k) {
      float ms = 0.f;
      CU(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      phase_ms[k] += ms;
    }
    return 0;
  }

  int step() {
    const bool full = next_full();
    ++replays;
    if ((flags & 2) && !(flags & 4)) {
      cudaGraphExec_t& g = full ? graph_full : graph;
      if (!g) {
        cudaGraph_t cg = nullptr;
        CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        int r = launch_step(full);
        cudaError_t ce = cudaStreamEndCapture(stream, &cg);
        if (r) return r;
        CU(ce);
        CU(cudaGraphInstantiate(&g, cg, 0));
        cudaGraphDestroy(cg);
      }
      CU(cudaGraphLaunch(g, stream));
      return 0;
    }
    return launch_step(full);
  }

  int read_clock(int pk, PeakClock* c) {
    CU(cudaMemcpyAsync(c, d_clocks + pk, sizeof(PeakClock), cudaMemcpyDeviceToHost, stream));
    CU(cudaStreamSynchronize(stream));
    return 0;
  }
  int write_clock(int pk, const PeakClock& c) {
    CU(cudaMemcpyAsync(d_clocks + pk, &c, sizeof(PeakClock), cudaMemcpyHostToDevice, stream));
    CU(cudaStreamSynchronize(stream));
    return 0;
  }

  ~pm_engine() {
    if (graph) cudaGraphExecDestroy(graph);
    if (graph_full) cudaGraphExecDestroy(graph_full);
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
    }
    sort_plan_destroy(&sort);
    sort_plan_destroy(&sort_full);
    cudaFree(d_peaks);
    cudaFree(d_clocks);
    cudaFree(d_stats);
    cudaFree(d_tile_base);
    cudaFree(d_ptile_base);
    cudaFree(d_p_base);
    cudaFree(d_mode_base);
    for (int b = 0; b < 2; ++b) {
      cudaFree(pos[b]);
      cudaFree(mom[b]);
      cudaFree(keys[b]);
      cudaFree(vals[b]);
    }
    cudaFree(bstart);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

int engine_init(pm_engine* E, const pm_peak_cfg* cfg, int npeaks) {
  E->npeaks = npeaks;
  E->peaks.resize(npeaks);
  E->occupied.assign(npeaks, 0);
  std::map<int, int> class_of;
  long long poff = 0, tb = 0, mb = 0, bo = 0, ptb = 0;
  int Tmax = 1, TPmax = 1;
  int max_bits = 0, min_lo = 64;
  std::vector<long long> tile_base(npeaks + 1), p_base(npeaks + 1), mode_base(npeaks + 1), ptile_base(npeaks + 1);
  for (int i = 0; i < npeaks; ++i) {
    const pm_peak_cfg& c = cfg[i];
    const int l2 = ilog2(c.N);
    if (l2 < 3 || l2 > 10) return -2001;
    const long long npart = c.n > 0 ? c.n : (long long)c.Np * c.Np * c.Np;
    if (c.Np < 1 || npart >= (1LL << 31)) return -2002;
    if (!(c.L > 0)) return -2003;
    // Bucket tiles of 8^3 (4^3 below 32^3); push super-tiles of 16^3 (the mesh when smaller).
    int T = c.tile > 0 ? c.tile : (c.N >= 32 ? 8 : std::max(2, c.N / 4));
    if (ilog2(T) < 1 || T > 8 || T > c.N) return -2004;
    // The push/deposit super-tile is 2T per side (8 bucket tiles), or T when the mesh is one tile.
    const int TP = std::min(2 * T, c.N);
    PeakDesc& P = E->peaks[i];
    P = PeakDesc{};
    P.N = c.N;
    P.log2N = l2;
    P.T = T;
    P.log2T = ilog2(T);
    P.log2NT = l2 - P.log2T;
    P.ntiles = 1 << (3 * P.log2NT);
    P.TP = TP;
    P.log2TP = ilog2(TP);
    P.nptiles = 1 << (3 * (l2 - P.log2TP));
    P.ptile_base = ptb;
    P.nb = P.ntiles * 8;
    P.local_bits = 3 * P.log2T;
    P.key_bits = 3 * l2 + 3;
    P.gradient = c.gradient;
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
    P.tile_base = tb;
    P.bucket_off = bo;
    P.nmodes = (long long)c.N * c.N * (c.N / 2 + 1);
    P.inv_nh = 1.0 / (double)(c.N / 2 + 1);
    P.mode_base = mb;
    tile_base[i] = tb;
    ptile_base[i] = ptb;
    ptb += P.nptiles;
    p_base[i] = poff;
    mode_base[i] = mb;
    poff += P.n;
    tb += P.ntiles;
    bo += P.nb + 1;
    mb += (P.nmodes + PM_THREADS - 1) / PM_THREADS;
    Tmax = std::max(Tmax, T);
    TPmax = std::max(TPmax, TP);
    max_bits = std::max(max_bits, P.key_bits);
    min_lo = std::min(min_lo, P.local_bits);
    if (!class_of.count(c.N)) {
      class_of[c.N] = (int)E->classes.size();
      E->classes.push_back(MeshClass{});
      E->classes.back().N = c.N;
    }
    E->classes[class_of[c.N]].peaks.push_back(i);
  }
  tile_base[npeaks] = tb;
  ptile_base[npeaks] = ptb;
  E->nptiles = ptb;
  p_base[npeaks] = poff;
  mode_base[npeaks] = mb;
  if (poff >= (1LL << 32)) return -2005;
  E->ntot = poff;
  E->ntiles = tb;
  E->nmodeblk = mb;
  E->nbuckets = bo;
  E->Tmax = Tmax;
  if (int rk = pm_kernels_init()) return rk;
  E->smem_dep = pm_deposit_smem(TPmax);
  E->smem_push = pm_push_smem(TPmax);

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
    if (E->flags & 4) {
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
  if ((r = E->alloc(&E->d_tile_base, npeaks + 1))) return r;
  if ((r = E->alloc(&E->d_ptile_base, npeaks + 1))) return r;
  if ((r = E->alloc(&E->d_p_base, npeaks + 1))) return r;
  if ((r = E->alloc(&E->d_mode_base, npeaks + 1))) return r;
  for (int b = 0; b < 2; ++b) {
    if ((r = E->alloc(&E->pos[b], E->ntot))) return r;
    if ((r = E->alloc(&E->mom[b], E->ntot))) return r;
    if ((r = E->alloc(&E->keys[b], E->ntot))) return r;
    if ((r = E->alloc(&E->vals[b], E->ntot))) return r;
  }
  if ((r = E->alloc(&E->bstart, E->nbuckets))) return r;
  CU(cudaMemcpy(E->d_peaks, E->peaks.data(), sizeof(PeakDesc) * npeaks, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(E->d_tile_base, tile_base.data(), sizeof(long long) * (npeaks + 1), cudaMemcpyHostToDevice));
  CU(cudaMemcpy(E->d_ptile_base, ptile_base.data(), sizeof(long long) * (npeaks + 1), cudaMemcpyHostToDevice));
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
  CU(cudaMemset(E->bstart, 0, sizeof(u32) * E->nbuckets));

  // Sort plans: one segment per peak.  The full plan sorts the whole cell key [0, key_bits);
  // the per-step plan, when flag bit 0 asks for it, only the bucket bits [local_bits, key_bits)
  // that the deposit and push group by, keeping the previous in-bucket order (stable).  Both
  // plans use pass counts of the same parity so the result always lands in the same buffers.
  E->full_every = (E->flags & 1) ? std::max(1, (E->flags >> 8) & 0xFF) : 1;
  if ((E->flags & 1) && ((E->flags >> 8) & 0xFF) == 0) E->full_every = 16;
  std::vector<SortSeg> segs(npeaks), fsegs(npeaks);
  int span_b = 0, span_f = 0;
  for (int i = 0; i < npeaks; ++i) {
    const PeakDesc& P = E->peaks[i];
    fsegs[i] = SortSeg{P.p_off, P.p_off + P.n, 0, P.key_bits, 0, 0};
    segs[i] = SortSeg{P.p_off, P.p_off + P.n, (E->flags & 1) ? P.local_bits : 0, P.key_bits, 0, 0};
    span_b = std::max(span_b, P.key_bits - segs[i].lo);
    span_f = std::max(span_f, P.key_bits);
  }
  const int np_b = (span_b + SORT_MAX_BITS - 1) / SORT_MAX_BITS;
  int np_f = (span_f + SORT_MAX_BITS - 1) / SORT_MAX_BITS;
  if ((np_f & 1) != (np_b & 1)) ++np_f;
  if ((r = sort_plan_create(&E->sort, segs.data(), npeaks, np_b, span_b))) return r;
  if ((r = sort_plan_create(&E->sort_full, fsegs.data(), npeaks, np_f, span_f))) return r;
  E->bytes += (long long)E->sort.ntiles * 8 * ((1LL << E->sort.bits) + (1LL << E->sort_full.bits));
  E->sort_result = np_b & 1;
  CU(cudaDeviceSynchronize());
  return 0;
}

}  // namespace

extern "C" {

int pm_engine_create(const pm_peak_cfg* cfg, int npeaks, int device, int flags, pm_engine** out) {
  if (!cfg || npeaks < 1 || !out) return -2000;
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
  launch_reset_peak(A, peak, a0, mode, param, a_end, max_steps, e->stream);
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
  cudaEvent_t ev[9];
  for (int k = 0; k < 9; ++k) CU(cudaEventCreate(&ev[k]));
  int r = 0;
  for (int s = 0; s < nsteps && !r; ++s) r = e->launch_step_timed(ev, phase_ms);
  for (int k = 0; k < 9; ++k) cudaEventDestroy(ev[k]);
  return r;
}

void* pm_engine_stream(pm_engine* e) { return e ? (void*)e->stream : nullptr; }

int pm_engine_info(const pm_engine* e, long long* info) {
  if (!e || !info) return -2000;
  info[0] = e->npeaks;
  info[1] = e->ntot;
  info[2] = e->ntiles;
  info[3] = e->sort.npass;
  info[4] = (long long)e->classes.size();
  info[5] = e->bytes;
  return 0;
}

int pm_get_stats_all(pm_engine* e, pm_stats_info* out) {
  if (!e || !out) return -2000;
  CU(cudaSetDevice(e->device));
  std::vector<PeakStats> s(e->npeaks);
  int err = 0, err2 = 0;
  CU(cudaMemcpyAsync(s.data(), e->d_stats, sizeof(PeakStats) * e->npeaks, cudaMemcpyDeviceToHost, e->stream));
  CU(cudaMemcpyAsync(&err, e->sort.err, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  CU(cudaMemcpyAsync(&err2, e->sort_full.err, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  err |= err2;
  CU(cudaStreamSynchronize(e->stream));
  int flagged = 0;
  for (int i = 0; i < e->npeaks; ++i) {
    const PeakDesc& P = e->peaks[i];
    out[i].rho_max_over_mean = (double)s[i].max_fix / (double)PM_FIX_ONE / P.n_mean;
    out[i].delta_max = out[i].rho_max_over_mean - 1.0;
    out[i].mass_defect = (double)s[i].mass_defect / (double)PM_FIX_ONE;
    out[i].status = s[i].status | (err ? 2u : 0u);
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
  for (int i = 0; i < e->npeaks; ++i) {
    out[i].a = c[i].a;
    out[i].da = c[i].da;
    out[i].a_end = c[i].a_end;
    out[i].kpend = c[i].kpend;
    out[i].a_grid = c[i].a_grid;
    out[i].mode = c[i].mode;
    out[i].state = c[i].state;
    out[i].nsteps = c[i].nsteps;
    out[i].max_steps = c[i].max_steps;
    out[i].a_collapse = c[i].a_collapse;
  }
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
  // Same kernel with the extra float64 output; delta is rewritten with identical values.
  launch_deposit(e->args(), e->nptiles, e->smem_dep, counts, e->stream);
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
  PeakClock c;
  int r;
  if ((r = e->read_clock(peak, &c))) return r;
  c.state = PS_IDLE;
  c.has_delta = 0;
  c.dep = 0;
  c.kpend = 0.0;
  if ((r = e->write_clock(peak, c))) return r;
  e->occupied[peak] = 0;
  return 0;
}

int pm_get_clock(pm_engine* e, int peak, pm_clock_info* out) {
  if (!e || peak < 0 || peak >= e->npeaks || !out) return -2000;
  CU(cudaSetDevice(e->device));
  PeakClock c;
  int r = e->read_clock(peak, &c);
  if (r) return r;
  out->a = c.a;
  out->da = c.da;
  out->a_end = c.a_end;
  out->kpend = c.kpend;
  out->a_grid = c.a_grid;
  out->mode = c.mode;
  out->state = c.state;
  out->nsteps = c.nsteps;
  out->max_steps = c.max_steps;
  out->a_collapse = c.a_collapse;
  return 0;
}

int pm_get_stats(pm_engine* e, int peak, pm_stats_info* out) {
  if (!e || peak < 0 || peak >= e->npeaks || !out) return -2000;
  CU(cudaSetDevice(e->device));
  PeakStats s;
  int err = 0, err2 = 0;
  CU(cudaMemcpyAsync(&s, e->d_stats + peak, sizeof(PeakStats), cudaMemcpyDeviceToHost, e->stream));
  CU(cudaMemcpyAsync(&err, e->sort.err, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  CU(cudaMemcpyAsync(&err2, e->sort_full.err, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  err |= err2;
  CU(cudaStreamSynchronize(e->stream));
  const PeakDesc& P = e->peaks[peak];
  out->rho_max_over_mean = (double)s.max_fix / (double)PM_FIX_ONE / P.n_mean;
  out->delta_max = out->rho_max_over_mean - 1.0;
  out->mass_defect = (double)s.mass_defect / (double)PM_FIX_ONE;
  out->status = s.status | (err ? 2u : 0u);
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
  // Host-side helper (plain host pointers): the key layout used by the sort.
  if (!cells || !keys_out || n < 0) return -2000;
  const int l2 = ilog2(N);
  const int T = tile > 0 ? tile : std::min(16, N);
  if (l2 < 1 || ilog2(T) < 1 || T > N) return -2001;
  PeakDesc P{};
  P.N = N;
  P.log2N = l2;
  P.T = T;
  P.log2T = ilog2(T);
  P.local_bits = 3 * P.log2T;
  for (long long i = 0; i < n; ++i) {
    const int c = cells[i];
    keys_out[i] = pm_cell_key(P, c >> (2 * l2), (c >> l2) & (N - 1), c & (N - 1));
  }
  return 0;
}

}  // extern "C"
