// Segmented, stable LSD radix sort of 64-bit keys with 32-bit values (sm_100a).
//
// One launch per digit.  A persistent grid (as many CTAs as fit on the GPU at once) claims
// tiles of SORT_TILE keys in order through an atomic counter; for each tile a CTA ranks the
// keys with warp-level multi-split (match.any + popc), publishes its digit counts and resolves
// its global offsets by decoupled look-back over the preceding tiles of the same segment, so
// every pass reads and writes each key once.  Claiming in order guarantees that every tile a
// CTA waits on is held by a running CTA that waits only on earlier tiles.  Waits are bounded:
// a CTA that gives up sets its segment's error word, counts the tile it waited on as empty
// (every position it then writes stays inside the segment) and proceeds.  A plan may carry a device gate word:
// when it reads 0 (no segment active this step) every launch returns at once, so a sort
// captured in a graph costs a few microseconds on the steps that do not need it.
//
// A segment is a contiguous key range sorted independently (one peak of the ensemble).
// Because every key of a segment carries the same high word (the peak id), sorting the
// segments separately over the low-word bit range [lo, lo + 8*npass) produces exactly the
// order of a stable sort of the full 64-bit keys.  A plan whose single segment has lo = 0
// and npass = 8 is a plain sort of arbitrary 64-bit keys.
#pragma once
#include "common.cuh"

#define SORT_THREADS 256
#define SORT_WARPS (SORT_THREADS / 32)
#define SORT_IPT 8
#define SORT_TILE (SORT_THREADS * SORT_IPT)
#define SORT_RADIX 256          // digit bins of the default 8-bit digit
#define SORT_MAX_BITS 10        // digits of 8, 9 or 10 bits
#define SORT_MAX_RADIX (1 << SORT_MAX_BITS)
#define SORT_MAX_PASSES 8

struct SortSeg {
  long long begin, end;  // key range
  int lo;                // first key bit sorted in this segment
  int hi;                // one past the last key bit sorted (bits >= hi are ignored)
  int active;            // 0: skip (the segment's buffers are left untouched)
  int first_tile;        // global index of the segment's first tile (filled by the plan)
};

struct SortPlan {
  int nseg;
  int ntiles;
  int npass;             // digit passes (the same for every segment)
  int bits;              // digit width: 8, 9 or 10
  SortSeg* seg;          // [nseg] (device)
  int* tile_seg;         // [ntiles]
  long long* tile_begin; // [ntiles]
  int* tile_first;       // [ntiles] 1 when the tile opens its segment
  u32* hist;             // [nseg][SORT_MAX_PASSES][radix]
  long long* base;       // [nseg][SORT_MAX_PASSES][radix]
  u64* status;           // [ntiles][radix] look-back words: epoch<<34 | flag<<32 | count
  u32* counters;         // [SORT_MAX_PASSES] tile claims, then the epoch word
  int* err;              // [nseg] nonzero after a bounded wait of that segment gave up
  const u32* gate;       // optional (device): when *gate == 0 every launch of the sort returns at once
  const int* dbg;        // optional (device): {spin limit of the look-back waits, tile whose look-back
                         // words the first pass never publishes (-1: none)}, read when the sort runs;
                         // nullptr: SORT_SPIN_LIMIT and no such tile.  A test hook: the waits on an
                         // unpublished tile run out, so the bounded-wait path can be exercised.
};

#define SORT_SPIN_LIMIT (1 << 22)

// Host side (sort.cu).  `segs` is a host array.  The digit width is the smallest of 8..10 bits
// that covers `span` key bits in `npass` passes (npass = 0: as few passes as 10-bit digits allow).
int sort_plan_create(SortPlan* plan, const SortSeg* segs, int nseg, int npass, int span = 0);
void sort_plan_destroy(SortPlan* plan);
// Runs plan->npass passes, ping-ponging (k0,v0) -> (k1,v1) -> (k0,v0) ...  The sorted
// result is in (k0,v0) when npass is even, (k1,v1) when odd.  identity_vals ignores the
// contents of v0 and uses value = global index.  write_last_keys = false skips writing the
// keys on the last pass (only the permutation is then produced).
// Key is u64 or u32 (the engine's cell keys fit 32 bits; the segment supplies the peak id).
template <class K>
int sort_run(const SortPlan* plan, K* k0, u32* v0, K* k1, u32* v1, bool identity_vals, bool write_last_keys,
             cudaStream_t s);
