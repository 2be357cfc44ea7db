// Segmented stable LSD radix sort (see sort.cuh for the design).
#include "sort.cuh"

#include <vector>

namespace {

constexpr int kSpinLimit = 1 << 22;

__device__ __forceinline__ u32 lanemask_lt() {
  u32 m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ u32 digit_of(u64 k, int shift, int hi, bool valid) {
  if (!valid) return SORT_RADIX;  // sentinel: counted nowhere
  const int width = min(8, hi - shift);
  if (width <= 0) return 0u;
  return (u32)(k >> shift) & ((1u << width) - 1u);
}

// Digit histograms of every pass in one read of the keys.
__global__ void __launch_bounds__(SORT_THREADS) k_sort_hist(SortPlan P, const u64* __restrict__ keys) {
  __shared__ u32 sh[SORT_MAX_PASSES * SORT_RADIX];
  const int t = blockIdx.x;
  const int seg = P.tile_seg[t];
  const SortSeg S = P.seg[seg];
  if (!S.active) return;
  for (int i = threadIdx.x; i < P.npass * SORT_RADIX; i += SORT_THREADS) sh[i] = 0;
  __syncthreads();
  const long long begin = P.tile_begin[t];
  const long long end = min(begin + (long long)SORT_TILE, S.end);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long wb = begin + (long long)warp * 32 * SORT_IPT;
  for (int j = 0; j < SORT_IPT; ++j) {
    const long long idx = wb + j * 32 + lane;
    const bool valid = idx < end;
    const u64 k = valid ? keys[idx] : 0ull;
    for (int pass = 0; pass < P.npass; ++pass) {
      const u32 d = digit_of(k, S.lo + 8 * pass, S.hi, valid);
      const u32 peers = __match_any_sync(0xffffffffu, d);
      if (d < SORT_RADIX && (peers & lanemask_lt()) == 0) atomicAdd(&sh[pass * SORT_RADIX + d], __popc(peers));
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < P.npass * SORT_RADIX; i += SORT_THREADS) {
    const u32 c = sh[i];
    if (c) atomicAdd(&P.hist[(size_t)seg * SORT_MAX_PASSES * SORT_RADIX + i], c);
  }
}

// Exclusive digit offsets per (segment, pass); clears the histograms, resets the tile
// claims and advances the look-back epoch for the passes that follow.
__global__ void __launch_bounds__(SORT_RADIX) k_sort_scan(SortPlan P) {
  __shared__ u32 wsum[SORT_RADIX / 32];
  const int seg = blockIdx.x;
  const SortSeg S = P.seg[seg];
  if (seg == 0 && threadIdx.x < SORT_MAX_PASSES) P.counters[threadIdx.x] = 0;
  if (seg == 0 && threadIdx.x == 0) P.counters[SORT_MAX_PASSES] += 1;
  if (!S.active) return;
  const int d = threadIdx.x, lane = d & 31, warp = d >> 5;
  for (int pass = 0; pass < P.npass; ++pass) {
    const size_t o = ((size_t)seg * SORT_MAX_PASSES + pass) * SORT_RADIX + d;
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

__global__ void __launch_bounds__(SORT_THREADS) k_sort_pass(SortPlan P, int pass, const u64* __restrict__ kin,
                                                             const u32* __restrict__ vin, u64* __restrict__ kout,
                                                             u32* __restrict__ vout) {
  __shared__ u32 s_tile;
  __shared__ u32 whist[SORT_WARPS][SORT_RADIX];
  __shared__ long long s_gbase[SORT_RADIX];
  if (threadIdx.x == 0) s_tile = atomicAdd(&P.counters[pass], 1u);
  for (int i = threadIdx.x; i < SORT_WARPS * SORT_RADIX; i += SORT_THREADS) (&whist[0][0])[i] = 0;
  __syncthreads();
  const int t = (int)s_tile;
  if (t >= P.ntiles) return;
  const int seg = P.tile_seg[t];
  const SortSeg S = P.seg[seg];
  if (!S.active) return;
  const int shift = S.lo + 8 * pass;
  const long long begin = P.tile_begin[t];
  const long long end = min(begin + (long long)SORT_TILE, S.end);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long wb = begin + (long long)warp * 32 * SORT_IPT;
  const u32 lt = lanemask_lt();

  u64 k[SORT_IPT];
  u32 v[SORT_IPT];
  u32 rd[SORT_IPT];  // warp-local rank (low 16 bits) | digit (high 16 bits)
#pragma unroll
  for (int j = 0; j < SORT_IPT; ++j) {
    const long long idx = wb + j * 32 + lane;
    const bool valid = idx < end;
    k[j] = valid ? kin[idx] : 0ull;
    v[j] = valid ? (vin ? vin[idx] : (u32)idx) : 0u;
    const u32 d = digit_of(k[j], shift, S.hi, valid);
    const u32 peers = __match_any_sync(0xffffffffu, d);
    const u32 below = __popc(peers & lt);
    const u32 prev = d < SORT_RADIX ? whist[warp][d] : 0u;
    __syncwarp();
    if (d < SORT_RADIX && below == 0) whist[warp][d] = prev + __popc(peers);
    __syncwarp();
    rd[j] = (prev + below) | (d << 16);
  }
  __syncthreads();

  // Per digit: warp offsets inside the tile, then the tile's offset inside the segment.
  {
    const int d = threadIdx.x;
    u32 run = 0;
#pragma unroll
    for (int w = 0; w < SORT_WARPS; ++w) {
      const u32 c = whist[w][d];
      whist[w][d] = run;
      run += c;
    }
    const u32 ep = (P.counters[SORT_MAX_PASSES] * SORT_MAX_PASSES + (u32)pass) & 0x3FFFFFFFu;
    const u64 tag = (u64)ep << 34;
    volatile u64* st = (volatile u64*)P.status;
    u32 excl = 0;
    if (P.tile_first[t]) {
      st[(size_t)t * SORT_RADIX + d] = tag | (2ull << 32) | run;
    } else {
      st[(size_t)t * SORT_RADIX + d] = tag | (1ull << 32) | run;
      int p = t - 1;
      int spins = 0;
      while (true) {
        const u64 w = st[(size_t)p * SORT_RADIX + d];
        const u32 flag = (u32)(w >> 32) & 3u;
        if ((w >> 34) != (u64)ep || flag == 0) {
          if (++spins > kSpinLimit) {
            atomicExch(P.err, 1);
            break;
          }
          __nanosleep(32);
          continue;
        }
        excl += (u32)w;
        if (flag == 2) break;
        --p;
      }
      st[(size_t)t * SORT_RADIX + d] = tag | (2ull << 32) | (excl + run);
    }
    s_gbase[d] = P.base[((size_t)seg * SORT_MAX_PASSES + pass) * SORT_RADIX + d] + excl;
  }
  __syncthreads();

#pragma unroll
  for (int j = 0; j < SORT_IPT; ++j) {
    const u32 d = rd[j] >> 16;
    if (d < SORT_RADIX) {
      const long long pos = s_gbase[d] + whist[warp][d] + (rd[j] & 0xFFFFu);
      if (kout) kout[pos] = k[j];
      vout[pos] = v[j];
    }
  }
}

}  // namespace

int sort_plan_create(SortPlan* P, const SortSeg* segs, int nseg, int npass) {
  *P = SortPlan{};
  if (npass < 1 || npass > SORT_MAX_PASSES || nseg < 1) return 1;
  std::vector<int> tseg, tfirst;
  std::vector<long long> tbeg;
  for (int s = 0; s < nseg; ++s) {
    bool first = true;
    for (long long b = segs[s].begin; b < segs[s].end; b += SORT_TILE) {
      tseg.push_back(s);
      tbeg.push_back(b);
      tfirst.push_back(first ? 1 : 0);
      first = false;
    }
  }
  P->nseg = nseg;
  P->ntiles = (int)tseg.size();
  P->npass = npass;
  const size_t nt = tseg.empty() ? 1 : tseg.size();
  PM_CHECK(cudaMalloc(&P->seg, sizeof(SortSeg) * nseg));
  PM_CHECK(cudaMalloc(&P->tile_seg, sizeof(int) * nt));
  PM_CHECK(cudaMalloc(&P->tile_begin, sizeof(long long) * nt));
  PM_CHECK(cudaMalloc(&P->tile_first, sizeof(int) * nt));
  PM_CHECK(cudaMalloc(&P->hist, sizeof(u32) * nseg * SORT_MAX_PASSES * SORT_RADIX));
  PM_CHECK(cudaMalloc(&P->base, sizeof(long long) * nseg * SORT_MAX_PASSES * SORT_RADIX));
  PM_CHECK(cudaMalloc(&P->status, sizeof(u64) * nt * SORT_RADIX));
  PM_CHECK(cudaMalloc(&P->counters, sizeof(u32) * (SORT_MAX_PASSES + 1)));
  PM_CHECK(cudaMalloc(&P->err, sizeof(int)));
  PM_CHECK(cudaMemcpy(P->seg, segs, sizeof(SortSeg) * nseg, cudaMemcpyHostToDevice));
  if (!tseg.empty()) {
    PM_CHECK(cudaMemcpy(P->tile_seg, tseg.data(), sizeof(int) * nt, cudaMemcpyHostToDevice));
    PM_CHECK(cudaMemcpy(P->tile_begin, tbeg.data(), sizeof(long long) * nt, cudaMemcpyHostToDevice));
    PM_CHECK(cudaMemcpy(P->tile_first, tfirst.data(), sizeof(int) * nt, cudaMemcpyHostToDevice));
  }
  PM_CHECK(cudaMemset(P->hist, 0, sizeof(u32) * nseg * SORT_MAX_PASSES * SORT_RADIX));
  PM_CHECK(cudaMemset(P->status, 0, sizeof(u64) * nt * SORT_RADIX));
  PM_CHECK(cudaMemset(P->counters, 0, sizeof(u32) * (SORT_MAX_PASSES + 1)));
  PM_CHECK(cudaMemset(P->err, 0, sizeof(int)));
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

int sort_run(const SortPlan* P, u64* k0, u32* v0, u64* k1, u32* v1, bool identity_vals, bool write_last_keys,
             cudaStream_t s) {
  if (P->ntiles == 0) return 0;
  k_sort_hist<<<P->ntiles, SORT_THREADS, 0, s>>>(*P, k0);
  k_sort_scan<<<P->nseg, SORT_RADIX, 0, s>>>(*P);
  u64* kin = k0;
  u32* vin = v0;
  u64* kout = k1;
  u32* vout = v1;
  for (int pass = 0; pass < P->npass; ++pass) {
    const bool last = pass == P->npass - 1;
    k_sort_pass<<<P->ntiles, SORT_THREADS, 0, s>>>(*P, pass, kin, (pass == 0 && identity_vals) ? nullptr : vin,
                                                   (last && !write_last_keys) ? nullptr : kout, vout);
    u64* tk = kin;
    kin = kout;
    kout = tk;
    u32* tv = vin;
    vin = vout;
    vout = tv;
  }
  PM_CHECK(cudaGetLastError());
  return 0;
}
