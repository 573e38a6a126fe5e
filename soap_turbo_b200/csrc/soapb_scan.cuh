// soapb_scan.cuh -- the CSR offset scan shared by the prep kernels and the
// neighbour-list builder, and the error word they report into.
#pragma once

#include "soapb_internal.h"

namespace soapb {

// CSR offsets, per-pair mask bits and input checks.  DevBatch::err holds
// prep_err_words(n_sites) 64-bit words, all cleared by one memset before the
// prep launch:
//   err[0]     the first input error: 2^34 - code under atomicMax, so the
//              smallest code wins (0 = none); code = a bad pair's index, or
//              kErrCsr / kErrScan;
//   err[1]     the scan's tile counter (low 32 bits);
//   err[2 + t] scan tile t's status: flag << 32 | sum, flag 1 = the tile's own
//              sum, 2 = the inclusive prefix up to the tile (0 = not yet);
//   the last word: the two work counters of the persistent site kernels.
// n_neigh is scanned in tiles of 2048 sites with a decoupled look-back: each
// tile publishes its sum, then walks back over its predecessors until it meets
// an inclusive prefix.  A tile takes its index from the counter, so every
// predecessor it waits for has already started; the wait is bounded.  The
// last tile writes off[n_sites] and checks it against n_pairs (skipped when
// n_pairs < 0: the neighbour-list builder scans counts whose total it learns
// from the scan).
constexpr int kScanTile = kScanTileSites;
// Spins of the look-back wait before it gives up (each sleeps ~64 ns).
constexpr int kScanSpins = 1 << 20;

__host__ __device__ inline int prep_scan_tiles(int n_sites) { return (n_sites + kScanTile - 1) / kScanTile; }

__device__ __forceinline__ void prep_error(const DevBatch &B, unsigned long long code) {
  atomicMax(B.err, kErrTop - code);
}

// One scan tile per calling block (NTH threads); sv: kScanTile ints of shared
// memory; max_spins bounds the wait for a predecessor.
template <int NTH>
__device__ __forceinline__ void prep_scan_tile(const DevBatch &B, int scan_tiles, int *sv,
                                               int max_spins = kScanSpins) {
  constexpr int ITEMS = kScanTile / NTH;
  __shared__ int wtot[NTH / 32];
  __shared__ int s_tile, s_excl;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned *counter = (unsigned *)(B.err + 1);
  unsigned long long *status = B.err + 2;
  if (tid == 0) s_tile = (int)atomicAdd(counter, 1u);
  __syncthreads();
  const int tile = s_tile;
  if (tile >= scan_tiles) {
    if (tid == 0) prep_error(B, kErrScan);
    return;
  }
  const int base = tile * kScanTile;
  bool bad = false;
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const int i = base + j * NTH + tid;
    int v = i < B.n_sites ? B.n_neigh[i] : 0;
    if (v < 0) {
      bad = true;
      v = 0;
    }
    sv[j * NTH + tid] = v;
  }
  if (bad) prep_error(B, kErrCsr);
  __syncthreads();
  int sum = 0;
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) sum += sv[tid * ITEMS + j];
  int x = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wtot[warp] = x;
  __syncthreads();
  int wpre = 0, total = 0;
#pragma unroll
  for (int w = 0; w < NTH / 32; ++w) {
    if (w < warp) wpre += wtot[w];
    total += wtot[w];
  }
  const int tpre = wpre + x - sum;  // exclusive prefix of this thread's items in the tile
  if (tid == 0) {
    volatile unsigned long long *vs = status;
    long long excl = 0;
    if (tile == 0) {
      vs[0] = (2ull << 32) | (unsigned)total;
    } else {
      vs[tile] = (1ull << 32) | (unsigned)total;
      int j = tile - 1, spins = 0;
      while (j >= 0) {
        const unsigned long long w = vs[j];
        const unsigned f = (unsigned)(w >> 32);
        if (f == 1u || f == 2u) {
          excl += (unsigned)w;
          if (f == 2u) break;
          --j;
        } else if (++spins > max_spins) {
          prep_error(B, kErrScan);
          break;
        } else {
          __nanosleep(64);
        }
      }
      vs[tile] = (2ull << 32) | (unsigned)(excl + total);
    }
    s_excl = (int)excl;
  }
  __syncthreads();
  // the thread's items again from shared memory, each written as the running
  // offset before it is added
  int run = s_excl + tpre;
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const int i = base + tid * ITEMS + j;
    if (i < B.n_sites) B.off[i] = run;
    run += sv[tid * ITEMS + j];
  }
  if (tile == scan_tiles - 1 && tid == 0) {
    const long long all = (long long)s_excl + total;
    B.off[B.n_sites] = (int)all;
    if (B.n_pairs >= 0 && all != (long long)B.n_pairs) prep_error(B, kErrCsr);
  }
}

// The sites of a batch one scan tile covers, heaviest row first, into
// B.order for the persistent site kernels (a counting sort on min(n_neigh, 255);
// the order within a count is whatever the atomics give, which changes only
// which CTA computes a site, not its result), so that their last sites are the
// lightest.  One CTA of NTH threads, beside the scan CTA; sv: kScanTile ints
// and hist: kScanOrderBuckets ints of shared memory.
constexpr int kScanOrderBuckets = 256;
template <int NTH>
__device__ __forceinline__ void order_sites(const DevBatch &B, int *sv, int *hist) {
  constexpr int ITEMS = kScanTile / NTH, NB = kScanOrderBuckets, BPT = NB / NTH > 0 ? NB / NTH : 1;
  __shared__ int wtot[NTH / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < NB; i += NTH) hist[i] = 0;
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const int i = j * NTH + tid;
    sv[i] = i < B.n_sites ? max(B.n_neigh[i], 0) : 0;
  }
  __syncthreads();
  // the lanes of a warp with equal keys add once (rows of similar length are
  // common, and same-address atomics in one warp would run one by one)
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const int i = j * NTH + tid;
    const int key = i < B.n_sites ? NB - 1 - min(sv[i], NB - 1) : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (key >= 0 && lane == __ffs(peers) - 1) atomicAdd(&hist[key], __popc(peers));
  }
  __syncthreads();
  // exclusive scan of the counts: BPT consecutive buckets per thread
  int loc = 0;
  if (tid * BPT < NB)
#pragma unroll
    for (int b = 0; b < BPT; ++b) loc += hist[tid * BPT + b];
  int xs = loc;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, xs, o);
    if (lane >= o) xs += y;
  }
  if (lane == 31) wtot[warp] = xs;
  __syncthreads();
  int pre = xs - loc;
#pragma unroll
  for (int w = 0; w < NTH / 32; ++w)
    if (w < warp) pre += wtot[w];
  __syncthreads();
  if (tid * BPT < NB)
#pragma unroll
    for (int b = 0; b < BPT; ++b) {
      const int c = hist[tid * BPT + b];
      hist[tid * BPT + b] = pre;
      pre += c;
    }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const int i = j * NTH + tid;
    const int key = i < B.n_sites ? NB - 1 - min(sv[i], NB - 1) : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (key >= 0 && lane == leader) base = atomicAdd(&hist[key], __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (key >= 0) B.order[base + __popc(peers & ((1u << lane) - 1u))] = i;
  }
}

}  // namespace soapb
