// The constraint-graph colouring and the row order on the device: src/graph.js colour() (105-170)
// and the order arrange() lays the rows out in (178-214), exactly.
//
// colour() is a greedy pass in found order: each manifold takes the lowest colour none of the
// earlier manifolds on its moving bodies holds.  So a manifold's colour depends only on the
// manifolds found before it on the same bodies: a dataflow with one chain a body, which the
// device runs as the solve's passes run theirs (stage.cuh, flow_pass): every moving body carries
// a count of its manifolds coloured so far and the mask of the colours they took, and manifold f
// waits until each of its moving bodies' counts reaches f's place among that body's manifolds
// (its rank), reads the masks, takes its colour and moves both counts on.  Warps take runs of 32
// manifolds in found order, each warp its runs in ascending order, so the earliest uncoloured
// manifold always has its predecessors coloured and is running or next: no deadlock.  (Unlike a
// colour's rows, the 32 manifolds of a run can share a body; their lanes wait on one another,
// which independent thread scheduling lets them do.)  Every wait is bounded, as the stage's are.
//
// The row order is then a sort by (colour, b's slot, found order): arrange()'s stable counting
// sorts by b's low and high digits and then by colour give exactly that order.  The device sorts
// the manifolds, taken in found order, by the key colour * slots + b with a stable radix sort of
// 8-bit digits (col_radix_*): each pass counts its digit per tile of 1,024, scans the (digit,
// tile) counts and places each manifold after those of its digit in earlier tiles, warps and
// lanes, so ties keep found order whatever the bins' sizes (a static b under thousands of
// manifolds of one colour costs no more than any other).
#pragma once

#include <stdint.h>

namespace bgcol {

constexpr int kOverflow = 32, kResting = 33, kRuns = kResting + 1, kStarts = 35;
constexpr uint8_t kDynamic = 0, kStatic = 1;

struct ColourParams {
  int32_t n;              // manifolds, in found order
  int32_t nb;             // slots
  const int32_t* a;       // found order
  const int32_t* b;
  const uint8_t* type;    // per slot
  const uint8_t* frozen;  // per slot
  int32_t any_frozen;     // World._frozenCount > 0
  int32_t* deg;           // nb: moving manifolds a body has
  int32_t* off;           // nb + 1: their exclusive scan
  int32_t* cursor;        // nb
  int32_t* list;          // 2n: each body's manifolds, by body, in found order once sorted
  int32_t* rank;          // 2n: rank on a, then rank on b (-1: that side does not move)
  uint32_t* used;         // nb: the colours a body's coloured manifolds took
  unsigned int* done;     // nb: the body's manifolds coloured so far
  int32_t* colour;        // n: each manifold's colour (found order)
  int32_t* keys[2];       // n each: the sort's keys, two buffers it passes between
  int32_t* vals[2];       // n each: the found indices that go with them
  int32_t* rcounts;       // kBuckets * tiles + 1: a pass's (digit, tile) counts, then their scan
  int32_t* colour_counts; // kRuns: manifolds of each colour
  int32_t tiles;          // ceil(n / kRadixThreads)
  int32_t* order;         // n: the manifold found order[o]-th goes to row o
  int32_t* starts;        // kStarts
  int32_t* status;        // 1: a wait ran past its budget
  long long budget;
};

// A body the solve moves, for colouring: dynamic and not frozen (src/graph.js:111-130).
__device__ __forceinline__ bool col_moving(const ColourParams& p, int x) {
  return p.type[x] == kDynamic && !(p.any_frozen && p.frozen[x] != 0);
}

__device__ __forceinline__ bool col_resting(const ColourParams& p, int x, int y) {
  return p.any_frozen && (p.frozen[x] != 0 || p.type[x] == kStatic) && (p.frozen[y] != 0 || p.type[y] == kStatic);
}

// Each manifold's moving sides: the bodies' counts of them, and -1 ranks for the rest.
__global__ void col_degrees(ColourParams p) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < p.n; f += gridDim.x * blockDim.x) {
    const int x = p.a[f], y = p.b[f];
    p.rank[f] = -1;
    p.rank[p.n + f] = -1;
    if (col_resting(p, x, y)) {
      p.colour[f] = kResting;
      continue;
    }
    p.colour[f] = -1;
    if (col_moving(p, x)) atomicAdd(&p.deg[x], 1);
    if (col_moving(p, y)) atomicAdd(&p.deg[y], 1);
  }
}

// Exclusive scan of in[0..n) into out[0..n] (out[n] the total), one block: each thread sums a
// contiguous share, the shares' sums are scanned in shared memory, each thread writes its share.
// in and out may be the same array.
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads) col_scan(const int32_t* in, int32_t* out, int n) {
  __shared__ int32_t sums[kScanThreads];
  const int t = threadIdx.x;
  const int per = (n + kScanThreads - 1) / kScanThreads;
  const int lo = min(n, t * per), hi = min(n, lo + per);
  int32_t s = 0;
  for (int i = lo; i < hi; i++) s += in[i];
  sums[t] = s;
  __syncthreads();
  for (int d = 1; d < kScanThreads; d <<= 1) {
    const int32_t v = t >= d ? sums[t - d] : 0;
    __syncthreads();
    sums[t] += v;
    __syncthreads();
  }
  int32_t at = sums[t] - s;   // exclusive prefix of this thread's share
  for (int i = lo; i < hi; i++) {
    const int32_t v = in[i];
    out[i] = at;
    at += v;
  }
  if (t == kScanThreads - 1) out[n] = sums[t];
}

// The same scan across many blocks, for long arrays (the (colour, b) bins): each block sums a tile
// of kTile entries (col_tile_sums), one block scans the tiles' sums in place (col_scan, n = the
// tile count), and each block then scans its tile from its offset (col_tile_scan).  in and out may
// be the same array.
constexpr int kTile = kScanThreads * 8;
__global__ void __launch_bounds__(kScanThreads) col_tile_sums(const int32_t* in, int n, int32_t* tile_sums) {
  __shared__ int32_t part[kScanThreads / 32];
  const int base = blockIdx.x * kTile;
  int32_t s = 0;
  for (int i = base + threadIdx.x; i < min(n, base + kTile); i += kScanThreads) s += in[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    int32_t t = part[threadIdx.x];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(kScanThreads) col_tile_scan(const int32_t* in, int32_t* out, int n,
                                                             const int32_t* tile_offsets) {
  __shared__ int32_t sums[kScanThreads];
  const int t = threadIdx.x;
  const int lo = min(n, blockIdx.x * kTile + t * 8), hi = min(n, lo + 8);
  int32_t v[8];
  int32_t s = 0;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    v[j] = lo + j < hi ? in[lo + j] : 0;
    s += v[j];
  }
  sums[t] = s;
  __syncthreads();
  for (int d = 1; d < kScanThreads; d <<= 1) {
    const int32_t x = t >= d ? sums[t - d] : 0;
    __syncthreads();
    sums[t] += x;
    __syncthreads();
  }
  int32_t at = tile_offsets[blockIdx.x] + sums[t] - s;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    if (lo + j < hi) out[lo + j] = at;
    at += v[j];
  }
  if (blockIdx.x == gridDim.x - 1 && t == kScanThreads - 1) out[n] = tile_offsets[gridDim.x];
}

// Each body's manifolds into its stretch of `list` (in any order; col_ranks sorts them).
__global__ void col_fill(ColourParams p) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < p.n; f += gridDim.x * blockDim.x) {
    if (p.colour[f] == kResting) continue;
    const int x = p.a[f], y = p.b[f];
    if (col_moving(p, x)) p.list[p.off[x] + atomicAdd(&p.cursor[x], 1)] = f;
    if (col_moving(p, y)) p.list[p.off[y] + atomicAdd(&p.cursor[y], 1)] = f;
  }
}

// Each body's manifolds in found order, and each manifold's rank on each of its moving bodies.
__global__ void col_ranks(ColourParams p) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < p.nb; x += gridDim.x * blockDim.x) {
    int32_t* l = p.list + p.off[x];
    const int d = p.off[x + 1] - p.off[x];
    for (int i = 1; i < d; i++) {
      const int32_t v = l[i];
      int j = i - 1;
      while (j >= 0 && l[j] > v) {
        l[j + 1] = l[j];
        j--;
      }
      l[j + 1] = v;
    }
    for (int i = 0; i < d; i++) {
      const int f = l[i];
      if (p.a[f] == x) p.rank[f] = i;
      else p.rank[p.n + f] = i;
    }
  }
}

__device__ __forceinline__ unsigned int col_load_relaxed(const unsigned int* q) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(q) : "memory");
  return v;
}
__device__ __forceinline__ void col_store_relaxed(unsigned int* q, unsigned int v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(q), "r"(v) : "memory");
}
__device__ __forceinline__ void col_fence() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// The greedy pass (src/graph.js:111-140) as a dataflow over the persistent grid (a cooperative
// launch: every block resident).
__global__ void col_colour(ColourParams p) {
  const int lane = static_cast<int>(threadIdx.x) & 31;
  const int warp = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int warps = static_cast<int>((gridDim.x * blockDim.x) >> 5);
  const int runs = (p.n + 31) / 32;
  for (int c = warp; c < runs; c += warps) {
    const int f = c * 32 + lane;
    if (f >= p.n || p.colour[f] == kResting) continue;
    const int x = p.a[f], y = p.b[f];
    const int ra = p.rank[f], rb = p.rank[p.n + f];
    long long it = 0;
    bool ok = true;
    for (;;) {
      const unsigned int va = ra < 0 ? 0u : col_load_relaxed(p.done + x);
      const unsigned int vb = rb < 0 ? 0u : col_load_relaxed(p.done + y);
      if ((ra < 0 || va >= static_cast<unsigned int>(ra)) && (rb < 0 || vb >= static_cast<unsigned int>(rb))) break;
      if (++it > p.budget || ((it & 255) == 0 && *(volatile int32_t*)p.status != 0)) {
        atomicExch(p.status, 1);
        ok = false;
        break;
      }
      __nanosleep(100);
    }
    if (!ok) return;
    col_fence();
    const uint32_t ux = ra < 0 ? 0u : __ldcg(p.used + x), uy = rb < 0 ? 0u : __ldcg(p.used + y);
    const uint32_t held = ux | uy;
    if (held == 0xffffffffu) {
      p.colour[f] = kOverflow;
    } else {
      // the lowest bit held clear: ~held & (held + 1) keeps just that bit
      const uint32_t bit = ~held & (held + 1u);
      p.colour[f] = 31 - __clz(bit);
      if (ra >= 0) __stcg(p.used + x, ux | bit);
      if (rb >= 0) __stcg(p.used + y, uy | bit);
    }
    col_fence();
    if (ra >= 0) col_store_relaxed(p.done + x, static_cast<unsigned int>(ra) + 1u);
    if (rb >= 0) col_store_relaxed(p.done + y, static_cast<unsigned int>(rb) + 1u);
  }
}

// ---- the row order: a stable radix sort by (colour, b), ties in found order ----

constexpr int kRadixThreads = 1024;   // one block a tile, one manifold a thread
constexpr int kBuckets = 256;         // 8-bit digits

// The first pass's input: each manifold's key in found order (a manifold left uncoloured by a wait
// that ran out sorts last; the call then fails), and each colour's count.
__global__ void col_keys(ColourParams p) {
  __shared__ int32_t local[kRuns];
  for (int k = threadIdx.x; k < kRuns; k += blockDim.x) local[k] = 0;
  __syncthreads();
  const int last = kRuns * p.nb;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < p.n; f += gridDim.x * blockDim.x) {
    const int k = p.colour[f];
    const bool ok = k >= 0 && k <= kResting;
    p.keys[0][f] = ok ? k * p.nb + p.b[f] : last;
    p.vals[0][f] = f;
    if (ok) atomicAdd(&local[k], 1);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < kRuns; k += blockDim.x)
    if (local[k] > 0) atomicAdd(&p.colour_counts[k], local[k]);
}

__global__ void __launch_bounds__(kRadixThreads) col_radix_count(ColourParams p, int from, int shift) {
  __shared__ int32_t hist[kBuckets];
  for (int d = threadIdx.x; d < kBuckets; d += blockDim.x) hist[d] = 0;
  __syncthreads();
  const int i = blockIdx.x * kRadixThreads + threadIdx.x;
  if (i < p.n) atomicAdd(&hist[(p.keys[from][i] >> shift) & (kBuckets - 1)], 1);
  __syncthreads();
  for (int d = threadIdx.x; d < kBuckets; d += blockDim.x) p.rcounts[d * p.tiles + blockIdx.x] = hist[d];
}

// Each manifold after its digit's manifolds in earlier tiles (the scanned counts), earlier warps
// of its tile and earlier lanes of its warp: stable.  The last pass writes the found indices
// straight into `order`.
__global__ void __launch_bounds__(kRadixThreads) col_radix_place(ColourParams p, int from, int shift, int last) {
  constexpr int kWarps = kRadixThreads / 32;
  __shared__ int32_t warp_counts[kWarps][kBuckets];
  for (int i = threadIdx.x; i < kWarps * kBuckets; i += blockDim.x) (&warp_counts[0][0])[i] = 0;
  __syncthreads();
  const int i = blockIdx.x * kRadixThreads + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int key = i < p.n ? p.keys[from][i] : 0;
  const int digit = i < p.n ? (key >> shift) & (kBuckets - 1) : -1;
  const unsigned peers = __match_any_sync(0xffffffffu, digit);
  const int before = __popc(peers & ((1u << lane) - 1u));
  if (digit >= 0 && before == 0) warp_counts[warp][digit] = __popc(peers);
  __syncthreads();
  if (digit < 0) return;
  int at = p.rcounts[digit * p.tiles + blockIdx.x] + before;
  for (int w = 0; w < warp; w++) at += warp_counts[w][digit];
  const int to = 1 - from;
  if (last) {
    p.order[at] = p.vals[from][i];
  } else {
    p.keys[to][at] = key;
    p.vals[to][at] = p.vals[from][i];
  }
}

// starts[k]: where colour k's rows begin (k <= RESTING), starts[RESTING + 1] = n
// (src/graph.js:152-166).
__global__ void col_starts(ColourParams p) {
  if (threadIdx.x != 0) return;
  int at = 0;
  for (int k = 0; k < kRuns; k++) {
    p.starts[k] = at;
    at += p.colour_counts[k];
  }
  p.starts[kRuns] = p.n;
}

}  // namespace bgcol
