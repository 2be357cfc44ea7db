// Segmented stable LSD radix sort (see sort.cuh for the design).
#include "sort.cuh"

#include <algorithm>
#include <vector>

namespace {

__device__ __forceinline__ u32 lanemask_lt() {
  u32 m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <int BITS, class K>
__device__ __forceinline__ u32 digit_of(K k, int shift, int hi, bool valid) {
  if (!valid) return 1u << BITS;  // sentinel: counted nowhere
  const int width = min(BITS, hi - shift);
  if (width <= 0 || shift >= (int)(8 * sizeof(K))) return 0u;
  return (u32)(k >> shift) & ((1u << width) - 1u);
}

__device__ __forceinline__ bool gate_closed(const SortPlan& P) { return P.gate && *P.gate == 0u; }

// Digit histograms of every pass in one read of the keys (grid-stride over the tiles).
template <class K, int BITS>
__global__ void __launch_bounds__(SORT_THREADS) k_sort_hist(SortPlan P, const K* __restrict__ keys) {
  constexpr int RADIX = 1 << BITS;
  extern __shared__ u32 sh[];  // [npass][RADIX]
  if (gate_closed(P)) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int t = blockIdx.x; t < P.ntiles; t += gridDim.x) {
    const int seg = P.tile_seg[t];
    const SortSeg S = P.seg[seg];
    if (!S.active) continue;
    for (int i = threadIdx.x; i < P.npass * RADIX; i += SORT_THREADS) sh[i] = 0;
    __syncthreads();
    const long long begin = P.tile_begin[t];
    const long long end = min(begin + (long long)SORT_TILE, S.end);
    const long long wb = begin + (long long)warp * 32 * SORT_IPT;
    for (int j = 0; j < SORT_IPT; ++j) {
      const long long idx = wb + j * 32 + lane;
      const bool valid = idx < end;
      const K k = valid ? keys[idx] : (K)0;
      for (int pass = 0; pass < P.npass; ++pass) {
        const u32 d = digit_of<BITS>(k, S.lo + BITS * pass, S.hi, valid);
        const u32 peers = __match_any_sync(0xffffffffu, d);
        if (d < RADIX && (peers & lanemask_lt()) == 0) atomicAdd(&sh[pass * RADIX + d], __popc(peers));
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < P.npass * RADIX; i += SORT_THREADS) {
      const u32 c = sh[i];
      if (c) atomicAdd(&P.hist[(size_t)seg * SORT_MAX_PASSES * RADIX + i], c);
    }
    __syncthreads();
  }
}

// Exclusive digit offsets per (segment, pass); clears the histograms, resets the tile
// claims and advances the look-back epoch for the passes that follow.  RADIX threads.
template <int BITS>
__global__ void k_sort_scan(SortPlan P) {
  constexpr int RADIX = 1 << BITS;
  __shared__ u32 wsum[RADIX / 32];
  if (gate_closed(P)) return;
  const int seg = blockIdx.x;
  const SortSeg S = P.seg[seg];
  if (seg == 0 && threadIdx.x < SORT_MAX_PASSES) P.counters[threadIdx.x] = 0;
  if (seg == 0 && threadIdx.x == 0) P.counters[SORT_MAX_PASSES] += 1;
  if (!S.active) return;
  const int d = threadIdx.x, lane = d & 31, warp = d >> 5;
  for (int pass = 0; pass < P.npass; ++pass) {
    const size_t o = ((size_t)seg * SORT_MAX_PASSES + pass) * RADIX + d;
    const u32 c = P.hist[o];
    P.hist[o] = 0;
    u32 incl = c;
    for (int s = 1; s < 32; s <<= 1) {
      const u32 v = __shfl_up_sync(0xffffffffu, incl, s);
      if (lane >= s) incl += v;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    u32 off = 0;
    for (int w = 0; w < warp; ++w) off += wsum[w];
    P.base[o] = S.begin + (long long)(off + incl - c);
    __syncthreads();
  }
}

template <class K, int BITS>
__global__ void __launch_bounds__(SORT_THREADS, 3) k_sort_pass(SortPlan P, int pass, const K* __restrict__ kin,
                                                                const u32* __restrict__ vin, K* __restrict__ kout,
                                                                u32* __restrict__ vout) {
  constexpr int RADIX = 1 << BITS;
  constexpr int DPT = RADIX / SORT_THREADS;  // digits per thread in the per-digit phase
  __shared__ u32 s_tile;
  __shared__ u32 whist[SORT_WARPS][RADIX];
  __shared__ long long s_gbase[RADIX];
  if (gate_closed(P)) return;
  const int spin_limit = P.dbg ? P.dbg[0] : SORT_SPIN_LIMIT;
  const int silent_tile = (P.dbg && pass == 0) ? P.dbg[1] : -1;
  for (;;) {
    __syncthreads();  // the previous tile's readers of s_tile, whist and s_gbase are done
    if (threadIdx.x == 0) s_tile = atomicAdd(&P.counters[pass], 1u);
    for (int i = threadIdx.x; i < SORT_WARPS * RADIX; i += SORT_THREADS) (&whist[0][0])[i] = 0;
    __syncthreads();
    const int t = (int)s_tile;
    if (t >= P.ntiles) return;
    const int seg = P.tile_seg[t];
    const SortSeg S = P.seg[seg];
    if (!S.active) continue;
    const int shift = S.lo + BITS * pass;
    const long long begin = P.tile_begin[t];
    const long long end = min(begin + (long long)SORT_TILE, S.end);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long wb = begin + (long long)warp * 32 * SORT_IPT;
    const u32 lt = lanemask_lt();

    K k[SORT_IPT];
    u32 v[SORT_IPT];
    u32 rd[SORT_IPT];  // warp-local rank (low 16 bits) | digit (high 16 bits)
#pragma unroll
    for (int j = 0; j < SORT_IPT; ++j) {
      const long long idx = wb + j * 32 + lane;
      const bool valid = idx < end;
      k[j] = valid ? kin[idx] : (K)0;
      v[j] = valid ? (vin ? vin[idx] : (u32)idx) : 0u;
    }
#pragma unroll
    for (int j = 0; j < SORT_IPT; ++j) {
      const long long idx = wb + j * 32 + lane;
      const u32 d = digit_of<BITS>(k[j], shift, S.hi, idx < end);
      const u32 peers = __match_any_sync(0xffffffffu, d);
      const u32 below = __popc(peers & lt);
      const u32 prev = d < RADIX ? whist[warp][d] : 0u;
      __syncwarp();
      if (d < RADIX && below == 0) whist[warp][d] = prev + __popc(peers);
      __syncwarp();
      rd[j] = (prev + below) | (d << 16);
    }
    __syncthreads();

    // Per digit: warp offsets inside the tile, then the tile's offset inside the segment.
    const u32 ep = (P.counters[SORT_MAX_PASSES] * SORT_MAX_PASSES + (u32)pass) & 0x3FFFFFFFu;
    const u64 tag = (u64)ep << 34;
    volatile u64* st = (volatile u64*)P.status;
    u32 run[DPT];
#pragma unroll
    for (int q = 0; q < DPT; ++q) {
      const int d = threadIdx.x + q * SORT_THREADS;
      u32 r = 0;
#pragma unroll
      for (int w = 0; w < SORT_WARPS; ++w) {
        const u32 c = whist[w][d];
        whist[w][d] = r;
        r += c;
      }
      run[q] = r;
      // Publish this tile's own count first, so successors can look past it at once.
      if (t != silent_tile) st[(size_t)t * RADIX + d] = tag | ((P.tile_first[t] ? 2ull : 1ull) << 32) | r;
    }
    // Look back over the predecessors of this segment, LB words per round trip: the loads of a
    // window are independent, so the walk costs one memory latency per LB tiles.
    constexpr int LB = 8;
#pragma unroll
    for (int q = 0; q < DPT; ++q) {
      const int d = threadIdx.x + q * SORT_THREADS;
      u32 excl = 0;
      if (!P.tile_first[t]) {
        int p = t - 1;
        int spins = 0;
        bool done = false;
        while (!done) {
          u64 w[LB];
#pragma unroll
          for (int i = 0; i < LB; ++i) w[i] = p - i >= S.first_tile ? st[(size_t)(p - i) * RADIX + d] : 0ull;
#pragma unroll
          for (int i = 0; i < LB; ++i) {
            if (done || p - i < S.first_tile) continue;
            u64 v = w[i];
            while ((v >> 34) != (u64)ep || ((u32)(v >> 32) & 3u) == 0) {
              if (++spins > spin_limit) {
                atomicExch(&P.err[seg], 1);
                v = tag | (2ull << 32);  // give up: treat as a zero inclusive prefix
                break;
              }
              __nanosleep(20);
              v = st[(size_t)(p - i) * RADIX + d];
            }
            excl += (u32)v;
            if (((u32)(v >> 32) & 3u) == 2u) done = true;
          }
          p -= LB;
          if (p < S.first_tile) done = true;
        }
        if (t != silent_tile) st[(size_t)t * RADIX + d] = tag | (2ull << 32) | (excl + run[q]);
      }
      s_gbase[d] = P.base[((size_t)seg * SORT_MAX_PASSES + pass) * RADIX + d] + excl;
    }
    __syncthreads();

#pragma unroll
    for (int j = 0; j < SORT_IPT; ++j) {
      const u32 d = rd[j] >> 16;
      if (d < RADIX) {
        const long long pos = s_gbase[d] + whist[warp][d] + (rd[j] & 0xFFFFu);
        if (kout) kout[pos] = k[j];
        vout[pos] = v[j];
      }
    }
  }  // next tile
}

}  // namespace

int sort_plan_create(SortPlan* P, const SortSeg* segs, int nseg, int npass, int span) {
  *P = SortPlan{};
  if (span <= 0) span = 8 * npass;
  if (npass <= 0) npass = (span + SORT_MAX_BITS - 1) / SORT_MAX_BITS;
  if (npass < 1 || npass > SORT_MAX_PASSES || nseg < 1) return 1;
  int bits = (span + npass - 1) / npass;
  bits = bits < 8 ? 8 : bits;
  if (bits > SORT_MAX_BITS) return 2;
  P->bits = bits;
  std::vector<int> tseg, tfirst;
  std::vector<long long> tbeg;
  std::vector<SortSeg> sg(segs, segs + nseg);
  for (int s = 0; s < nseg; ++s) {
    sg[s].first_tile = (int)tseg.size();
    bool first = true;
    for (long long b = segs[s].begin; b < segs[s].end; b += SORT_TILE) {
      tseg.push_back(s);
      tbeg.push_back(b);
      tfirst.push_back(first ? 1 : 0);
      first = false;
    }
  }
  P->nseg = nseg;
  P->gate = nullptr;
  P->ntiles = (int)tseg.size();
  P->npass = npass;
  const size_t nt = tseg.empty() ? 1 : tseg.size();
  PM_CHECK(cudaMalloc(&P->seg, sizeof(SortSeg) * nseg));
  PM_CHECK(cudaMalloc(&P->tile_seg, sizeof(int) * nt));
  PM_CHECK(cudaMalloc(&P->tile_begin, sizeof(long long) * nt));
  PM_CHECK(cudaMalloc(&P->tile_first, sizeof(int) * nt));
  const size_t radix = (size_t)1 << bits;
  PM_CHECK(cudaMalloc(&P->hist, sizeof(u32) * nseg * SORT_MAX_PASSES * radix));
  PM_CHECK(cudaMalloc(&P->base, sizeof(long long) * nseg * SORT_MAX_PASSES * radix));
  PM_CHECK(cudaMalloc(&P->status, sizeof(u64) * nt * radix));
  PM_CHECK(cudaMalloc(&P->counters, sizeof(u32) * (SORT_MAX_PASSES + 1)));
  PM_CHECK(cudaMalloc(&P->err, sizeof(int) * nseg));
  PM_CHECK(cudaMemcpy(P->seg, sg.data(), sizeof(SortSeg) * nseg, cudaMemcpyHostToDevice));
  if (!tseg.empty()) {
    PM_CHECK(cudaMemcpy(P->tile_seg, tseg.data(), sizeof(int) * nt, cudaMemcpyHostToDevice));
    PM_CHECK(cudaMemcpy(P->tile_begin, tbeg.data(), sizeof(long long) * nt, cudaMemcpyHostToDevice));
    PM_CHECK(cudaMemcpy(P->tile_first, tfirst.data(), sizeof(int) * nt, cudaMemcpyHostToDevice));
  }
  PM_CHECK(cudaMemset(P->hist, 0, sizeof(u32) * nseg * SORT_MAX_PASSES * radix));
  PM_CHECK(cudaMemset(P->status, 0, sizeof(u64) * nt * radix));
  PM_CHECK(cudaMemset(P->counters, 0, sizeof(u32) * (SORT_MAX_PASSES + 1)));
  PM_CHECK(cudaMemset(P->err, 0, sizeof(int) * nseg));
  return 0;
}

void sort_plan_destroy(SortPlan* P) {
  cudaFree(P->seg);
  cudaFree(P->tile_seg);
  cudaFree(P->tile_begin);
  cudaFree(P->tile_first);
  cudaFree(P->hist);
  cudaFree(P->base);
  cudaFree(P->status);
  cudaFree(P->counters);
  cudaFree(P->err);
  *P = SortPlan{};
}

template <class K, int BITS>
static int sort_run_bits(const SortPlan* P, K* k0, u32* v0, K* k1, u32* v1, bool identity_vals, bool write_last_keys,
                         cudaStream_t s) {
  constexpr int RADIX = 1 << BITS;
  // Persistent grids: as many CTAs as are resident at once (the passes rely on every claimed
  // tile being held by a running CTA, which a grid of at most this size guarantees).
  int dev = 0, sms = 0, per_sm = 0;
  PM_CHECK(cudaGetDevice(&dev));
  PM_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  PM_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sort_pass<K, BITS>, SORT_THREADS, 0));
  const int grid_pass = std::max(1, std::min(P->ntiles, sms * std::max(per_sm, 1)));
  const int grid_hist = std::max(1, std::min(P->ntiles, sms * 4));
  k_sort_hist<K, BITS><<<grid_hist, SORT_THREADS, sizeof(u32) * P->npass * RADIX, s>>>(*P, k0);
  k_sort_scan<BITS><<<P->nseg, RADIX, 0, s>>>(*P);
  K* kin = k0;
  u32* vin = v0;
  K* kout = k1;
  u32* vout = v1;
  for (int pass = 0; pass < P->npass; ++pass) {
    const bool last = pass == P->npass - 1;
    k_sort_pass<K, BITS><<<grid_pass, SORT_THREADS, 0, s>>>(*P, pass, kin, (pass == 0 && identity_vals) ? nullptr : vin,
                                                            (last && !write_last_keys) ? nullptr : kout, vout);
    K* tk = kin;
    kin = kout;
    kout = tk;
    u32* tv = vin;
    vin = vout;
    vout = tv;
  }
  PM_CHECK(cudaGetLastError());
  return 0;
}

template <class K>
int sort_run(const SortPlan* P, K* k0, u32* v0, K* k1, u32* v1, bool identity_vals, bool write_last_keys,
             cudaStream_t s) {
  if (P->ntiles == 0) return 0;
  switch (P->bits) {
    case 8: return sort_run_bits<K, 8>(P, k0, v0, k1, v1, identity_vals, write_last_keys, s);
    case 9: return sort_run_bits<K, 9>(P, k0, v0, k1, v1, identity_vals, write_last_keys, s);
    case 10: return sort_run_bits<K, 10>(P, k0, v0, k1, v1, identity_vals, write_last_keys, s);
    default: return 3;
  }
}

template int sort_run<u64>(const SortPlan*, u64*, u32*, u64*, u32*, bool, bool, cudaStream_t);
template int sort_run<u32>(const SortPlan*, u32*, u32*, u32*, u32*, bool, bool, cudaStream_t);
