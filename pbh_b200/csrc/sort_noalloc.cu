// pm_sort_u64_noalloc: the stable 64-bit radix sort of pm_sort_u64 for callers that cannot
// allocate device memory.  Everything the sort needs beyond the caller's input and outputs --
// the ping-pong key/value buffers, digit histograms, look-back words, tile tables and the
// error word -- lives in one file-scope static device array of PM_NOALLOC_SCRATCH_BYTES
// (about 3.3 MB), which every GPU that loads this library holds until the process exits.
#include "../../include/pmb200.h"
#include "sort.cuh"

namespace {

constexpr long long kMaxKeys = PM_NOALLOC_MAX_KEYS;
constexpr int kTiles = (int)((kMaxKeys + SORT_TILE - 1) / SORT_TILE);

// Byte offsets of the pieces inside the scratch array (each 256-byte aligned).
constexpr size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }
constexpr size_t kOffKeys = 0;
constexpr size_t kOffVals = align256(kOffKeys + sizeof(u64) * kMaxKeys);
constexpr size_t kOffStatus = align256(kOffVals + sizeof(u32) * kMaxKeys);
constexpr size_t kOffHist = align256(kOffStatus + sizeof(u64) * kTiles * SORT_RADIX);
constexpr size_t kOffBase = align256(kOffHist + sizeof(u32) * SORT_MAX_PASSES * SORT_RADIX);
constexpr size_t kOffTileSeg = align256(kOffBase + sizeof(long long) * SORT_MAX_PASSES * SORT_RADIX);
constexpr size_t kOffTileBegin = align256(kOffTileSeg + sizeof(int) * kTiles);
constexpr size_t kOffTileFirst = align256(kOffTileBegin + sizeof(long long) * kTiles);
constexpr size_t kOffSeg = align256(kOffTileFirst + sizeof(int) * kTiles);
constexpr size_t kOffCounters = align256(kOffSeg + sizeof(SortSeg));
constexpr size_t kOffErr = align256(kOffCounters + sizeof(u32) * (SORT_MAX_PASSES + 1));
constexpr size_t kBytes = align256(kOffErr + sizeof(int));
static_assert(kBytes <= PM_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the declared size");

static __device__ __align__(256) unsigned char g_sort_scratch[PM_NOALLOC_SCRATCH_BYTES];

// Device address of g_sort_scratch on the current device.  In host code the array's name
// stands for a host-side shadow, not device memory, so the kernels get this address instead.
// Looked up on every call (it allocates nothing): a cached address would go stale if the
// device were reset and the module loaded again.
int scratch_address(unsigned char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
  if (e != cudaSuccess) return -(int)e;
  *out = (unsigned char*)p;
  return 0;
}

// Per-call set-up of the plan tables for one segment [0, n); also clears the histograms and the
// error word, which the previous call may have left behind.  The look-back words need no
// clearing: each carries the epoch of the pass that wrote it, and the epoch only grows.
__global__ void k_noalloc_setup(unsigned char* base, long long n, int lo, int hi, int ntiles) {
  SortSeg* seg = (SortSeg*)(base + kOffSeg);
  int* tseg = (int*)(base + kOffTileSeg);
  long long* tbeg = (long long*)(base + kOffTileBegin);
  int* tfirst = (int*)(base + kOffTileFirst);
  u32* hist = (u32*)(base + kOffHist);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    *seg = SortSeg{0, n, lo, hi, 1, 0};  // first tile 0
    *(int*)(base + kOffErr) = 0;
  }
  if (i < ntiles) {
    tseg[i] = 0;
    tbeg[i] = (long long)i * SORT_TILE;
    tfirst[i] = i == 0 ? 1 : 0;
  }
  if (i < SORT_MAX_PASSES * SORT_RADIX) hist[i] = 0;
}

}  // namespace

extern "C" int pm_sort_u64_noalloc(const unsigned long long* keys, unsigned long long* keys_out,
                                   unsigned int* perm_out, long long n, int lo, int hi, void* stream) {
  if (!keys || !keys_out || !perm_out || n < 0) return -2000;
  if (lo < 0 || hi > 64 || hi <= lo) return -2001;
  if (n > kMaxKeys) return -2003;  // beyond the static scratch: PM_NOALLOC_MAX_KEYS
  if (n == 0) return 0;
  unsigned char* base = nullptr;
  int r = scratch_address(&base);
  if (r) return r;
  cudaError_t ce = cudaSuccess;
  cudaStream_t s = (cudaStream_t)stream;
  const int ntiles = (int)((n + SORT_TILE - 1) / SORT_TILE);
  const int npass = (hi - lo + 7) / 8;
  k_noalloc_setup<<<(SORT_MAX_PASSES * SORT_RADIX + 255) / 256, 256, 0, s>>>(base, n, lo, hi, ntiles);
  SortPlan P{};
  P.nseg = 1;
  P.ntiles = ntiles;
  P.npass = npass;
  P.bits = 8;
  P.seg = (SortSeg*)(base + kOffSeg);
  P.tile_seg = (int*)(base + kOffTileSeg);
  P.tile_begin = (long long*)(base + kOffTileBegin);
  P.tile_first = (int*)(base + kOffTileFirst);
  P.hist = (u32*)(base + kOffHist);
  P.base = (long long*)(base + kOffBase);
  P.status = (u64*)(base + kOffStatus);
  P.counters = (u32*)(base + kOffCounters);
  P.err = (int*)(base + kOffErr);
  // Passes alternate (k0,v0) -> (k1,v1) -> (k0,v0) ...: start in the buffer pair that the last
  // pass writes into the caller's outputs.  The caller's input keys are only read.
  u64* sk = (u64*)(base + kOffKeys);
  u32* sv = (u32*)(base + kOffVals);
  const bool even = (npass & 1) == 0;
  u64* k0 = even ? (u64*)keys_out : sk;
  u32* v0 = even ? perm_out : sv;
  u64* k1 = even ? sk : (u64*)keys_out;
  u32* v1 = even ? sv : perm_out;
  ce = cudaMemcpyAsync(k0, keys, sizeof(u64) * (size_t)n, cudaMemcpyDeviceToDevice, s);
  if (ce != cudaSuccess) return -(int)ce;
  r = sort_run<u64>(&P, k0, v0, k1, v1, true, true, s);
  if (r) return r;
  int err = 0;
  ce = cudaMemcpyAsync(&err, P.err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
  if (ce != cudaSuccess) return -(int)ce;
  return err ? 1 : 0;
}
