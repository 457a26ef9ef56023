// libbearing_gpu.so: the C ABI of include/bearing_gpu.h over the device solve stage in
// stage.cuh.  Per context: one CUDA stream, device buffers grown by doubling (the rule
// src/contact.js:250-255 uses for its columns), a staging block holding every input column in the
// caller's layout (so bg_restore can run the same input again), the packed device layout, pinned
// host staging and a small pool of host threads.
//
// A step is: copy the caller's columns in (straight from page-locked caller memory, or gathered
// into the pinned staging a group at a time, the copies overlapping the gathering) while another
// host thread works out the solve order; unpack them into the device layout; run the solve stage
// (a persistent cooperative grid for a single world, one CTA per world for a batch); pack the written
// columns and copy them out the same way.
//
// Around the solve stage the same context also runs the narrowphase (bg_collide, sources in
// host/collide_impl.hpp), the colouring and row order (bg_colour, colour.cuh), the adjoint
// (bg_backward, adjoint.cuh) and a step's whole contact side from the pair list (bg_contact_step,
// contact.cuh), each with device memory of its own next to the solve stage's.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <unistd.h>

#include "../../include/bearing_gpu.h"
#include "layout.cuh"
#include "stage.cuh"
#include "adjoint.cuh"
#include "../host/collide_impl.hpp"
#include "colour.cuh"
#include "contact.cuh"

namespace {

constexpr int kGridThreads = 256;
constexpr int kBlockThreads = 256;
// bg_batch_solve_step's rows per group of worlds (twice as many for pageable columns; see groups_for).
constexpr int kRowsPerGroup = 131072;
constexpr int kUnpackThreads = 256;
// A single world runs on the whole grid whatever its size: measured against one CTA on B200 it was
// faster at every size tried, from a 10-row stack (0.37 against 0.47 ms a step) and the 590-row
// pyramid (1.60 against 2.00) to a 4,333-row pile (2.23 against 8.67).  One CTA a world is for
// batches, where many worlds share the machine.
constexpr long long kDefaultBudget = 1LL << 24;

// ---- kernels: stage the caller's layout in and out of the device layout ----

struct BodyStage {
  const double* position; const double* rotation; const double* velocity; const double* angular;
  const double* tumbled; const double* ceiling; const double* start; const double* start_q; const double* inv_mass;
  const double* inertia; const double* inv_inertia; const double* dims; const double* damping;
  const double* angular_damping; const double* gravity_scale;
  const uint8_t* type; const uint8_t* shape; const uint8_t* frozen; const uint8_t* framed;
  const uint8_t* lock; const int32_t* joint_head; const uint8_t* awake; const double* inv_i;
};

struct BodyOut {
  double* position; double* rotation; double* velocity; double* angular; double* tumbled;
  double* ceiling; double* start; double* start_q; double* inv_i;
};

struct RowStage {
  const int32_t* row; const int32_t* a; const int32_t* b; const uint8_t* points;
  const double* normal; const double* t1; const double* t2; const double* friction;
  const double* restitution; const double* tolerance; const double* patch; const double* separation;
  const double* point; const double* shift; const double* normal_impulse; const double* ti1;
  const double* ti2; const double* ri1; const double* ri2; const double* si; const double* drift1;
  const double* drift2;
};

struct RowOut {
  double* normal_impulse; double* ti1; double* ti2; double* ri1; double* ri2; double* si;
  double* drift1; double* drift2; double* gap; double* maxni; double* relvel; uint8_t* sliding;
  double* anchor_a; double* anchor_b;
};

// Which world index i (a row or an awake entry) belongs to, from a (count+1) prefix table.
__device__ __forceinline__ int world_of(const int32_t* offset, int count, int i) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (offset[mid] <= i) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void unpack_bodies(BodyStage in, bg::BodiesDev B, int n, const int32_t* awake_in, int nawake,
                              const int32_t* body_offset, const int32_t* awake_offset, int nworlds) {
  const int stride = gridDim.x * blockDim.x;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
    for (int k = 0; k < 3; k++) {
      B.vw[8 * s + k] = in.velocity[3 * s + k];
      B.vw[8 * s + 3 + k] = in.angular[3 * s + k];
      B.pq[8 * s + k] = in.position[3 * s + k];
      B.st[4 * s + k] = in.start[3 * s + k];
      B.tc[4 * s + k] = in.tumbled[3 * s + k];
      B.pr[12 * s + k] = in.inertia[3 * s + k];
      B.pr[12 * s + 3 + k] = in.inv_inertia[3 * s + k];
      B.pr[12 * s + 6 + k] = in.dims[3 * s + k];
    }
    B.vw[8 * s + 6] = 0; B.vw[8 * s + 7] = 0;
    B.pq[8 * s + 3] = 0;
    B.st[4 * s + 3] = 0;
    for (int k = 0; k < 4; k++) { B.pq[8 * s + 4 + k] = in.rotation[4 * s + k]; B.sq[4 * s + k] = in.start_q[4 * s + k]; }
    B.tc[4 * s + 3] = in.ceiling[s];
    B.pr[12 * s + 9] = in.damping[s];
    B.pr[12 * s + 10] = in.angular_damping[s];
    B.pr[12 * s + 11] = in.gravity_scale[s];
    B.mi[8 * s] = in.inv_mass[s];
    for (int k = 0; k < 6; k++) B.mi[8 * s + 1 + k] = in.inv_i[6 * s + k];
    B.mi[8 * s + 7] = 0;
    uint32_t f = static_cast<uint32_t>(in.type[s]) & bg::F_TYPE;
    f |= (static_cast<uint32_t>(in.shape[s]) & 3u) << bg::F_SHAPE_SHIFT;
    if (in.frozen[s]) f |= bg::F_FROZEN;
    if (in.framed[s]) f |= bg::F_FRAMED;
    f |= (static_cast<uint32_t>(in.lock[s]) & 7u) << bg::F_LOCK_SHIFT;
    if (in.joint_head[s] != 0) f |= bg::F_JOINTED;
    if (in.awake[s]) f |= bg::F_AWAKE;
    B.fl[s] = f;
    B.head[s] = 0x7fffffff;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nawake; i += stride) {
    const int w = nworlds > 1 ? world_of(awake_offset, nworlds, i) : 0;
    B.awake_list[i] = awake_in[i] + (nworlds > 1 ? body_offset[w] : 0);
  }
}

// Device row m holds the caller's row perm[m] (rows of one colour sorted by point count, see
// order_rows()); the found-order list maps to device rows through iperm.
__global__ void unpack_rows(RowStage in, bg::RowsDev R, int n, const int32_t* row_offset, const int32_t* body_offset,
                            int nworlds, const double* maxni_in, const double* relvel_in, const double* gap_in,
                            const int32_t* perm, const int32_t* iperm) {
  const int64_t cap = R.cap;
  const int stride = gridDim.x * blockDim.x;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n; f += stride) {
    int r0 = 0;
    if (nworlds > 1) r0 = row_offset[world_of(row_offset, nworlds, f)];
    R.row[f] = iperm[in.row[f] + r0];
  }
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += stride) {
    const int m = perm[d];
    int b0 = 0;
    if (nworlds > 1) b0 = body_offset[world_of(row_offset, nworlds, m)];
    R.a[d] = in.a[m] + b0;
    R.b[d] = in.b[m] + b0;
    R.points[d] = in.points[m];
    for (int c = 0; c < 3; c++) {
      R.n[c * cap + d] = in.normal[3 * m + c];
      R.t1[c * cap + d] = in.t1[3 * m + c];
      R.t2[c * cap + d] = in.t2[3 * m + c];
    }
    R.friction[d] = in.friction[m];
    R.restitution[d] = in.restitution[m];
    R.tolerance[d] = in.tolerance[m];
    R.patch[d] = in.patch[m];
    R.gap[d] = gap_in[m];
    R.sliding[d] = 0;
    for (int c = 0; c < 3; c++) { R.anchorA[c * cap + d] = 0; R.anchorB[c * cap + d] = 0; }
    for (int k = 0; k < bg::P; k++) {
      R.maxni[k * cap + d] = maxni_in[bg::P * m + k];
      R.relvel[k * cap + d] = relvel_in[bg::P * m + k];
      R.separation[k * cap + d] = in.separation[bg::P * m + k];
      R.ni[k * cap + d] = in.normal_impulse[bg::P * m + k];
      for (int c = 0; c < 3; c++) {
        R.point[(k * 3 + c) * cap + d] = in.point[12 * m + 3 * k + c];
        R.shift[(k * 3 + c) * cap + d] = in.shift[12 * m + 3 * k + c];
      }
    }
    R.ti1[d] = in.ti1[m]; R.ti2[d] = in.ti2[m]; R.ri1[d] = in.ri1[m]; R.ri2[d] = in.ri2[m];
    R.si[d] = in.si[m]; R.drift1[d] = in.drift1[m]; R.drift2[d] = in.drift2[m];
  }
}

__global__ void pack_bodies(bg::BodiesDev B, BodyOut out, int n) {
  const int stride = gridDim.x * blockDim.x;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
    for (int k = 0; k < 3; k++) {
      out.velocity[3 * s + k] = B.vw[8 * s + k];
      out.angular[3 * s + k] = B.vw[8 * s + 3 + k];
      out.position[3 * s + k] = B.pq[8 * s + k];
      out.start[3 * s + k] = B.st[4 * s + k];
      out.tumbled[3 * s + k] = B.tc[4 * s + k];
    }
    for (int k = 0; k < 4; k++) { out.rotation[4 * s + k] = B.pq[8 * s + 4 + k]; out.start_q[4 * s + k] = B.sq[4 * s + k]; }
    out.ceiling[s] = B.tc[4 * s + 3];
    for (int k = 0; k < 6; k++) out.inv_i[6 * s + k] = B.mi[8 * s + 1 + k];
  }
}

__global__ void pack_rows(bg::RowsDev R, RowOut out, int n, const int32_t* perm) {
  const int64_t cap = R.cap;
  const int stride = gridDim.x * blockDim.x;
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += stride) {
    const int m = perm[d];
    for (int k = 0; k < bg::P; k++) {
      out.normal_impulse[bg::P * m + k] = R.ni[k * cap + d];
      out.maxni[bg::P * m + k] = R.maxni[k * cap + d];
      out.relvel[bg::P * m + k] = R.relvel[k * cap + d];
    }
    out.ti1[m] = R.ti1[d]; out.ti2[m] = R.ti2[d]; out.ri1[m] = R.ri1[d]; out.ri2[m] = R.ri2[d];
    out.si[m] = R.si[d]; out.drift1[m] = R.drift1[d]; out.drift2[m] = R.drift2[d];
    out.gap[m] = R.gap[d];
    out.sliding[m] = R.sliding[d];
    for (int c = 0; c < 3; c++) {
      out.anchor_a[3 * m + c] = R.anchorA[c * cap + d];
      out.anchor_b[3 * m + c] = R.anchorB[c * cap + d];
    }
  }
}

__global__ void __launch_bounds__(kGridThreads) stage_grid(bg::StageParams p) {
  bg::GridTeam t;
  const bg::WorldDesc w = p.worlds[0];
  bg::solve_stage(p, w, t);
}

__global__ void __launch_bounds__(kGridThreads) stage_grid_batch(bg::StageParams p) { bg::batch_stage(p); }

__global__ void __launch_bounds__(kBlockThreads) stage_block(bg::StageParams p) {
  bg::BlockTeam t;
  for (int k = blockIdx.x; k < p.nworlds; k += gridDim.x) {
    const int wi = p.world_order != nullptr ? p.world_order[k] : k;
    const bg::WorldDesc w = p.worlds[wi];
    if (!bg::solve_stage(p, w, t)) return;
    __syncthreads();
  }
}


// ---- device buffers ----

template <class T>
struct DevBuf {
  T* ptr = nullptr;
  size_t n = 0;
};

// ---- host threads for the copies between the caller's columns and pinned staging ----
//
// A fixed set of worker threads, started on a context's first transfer.  run(n, fn) calls fn(0..n-1)
// on the workers and the calling thread and returns when all are done.  Tasks are claimed from a
// cursor tagged with the call's generation, so a worker that wakes late for a finished call finds
// the tag changed and claims nothing.
class HostPool {
 public:
  explicit HostPool(int workers) {
    for (int i = 0; i < workers; i++) threads_.emplace_back([this] { loop(); });
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> lock(mutex_);
      stop_ = true;
    }
    wake_.notify_all();
    for (std::thread& t : threads_) t.join();
  }
  int size() const { return static_cast<int>(threads_.size()) + 1; }
  void run(int n, const std::function<void(int)>& fn) {
    if (n <= 0) return;
    if (threads_.empty() || n == 1) {
      for (int i = 0; i < n; i++) fn(i);
      return;
    }
    uint32_t gen;
    {
      std::lock_guard<std::mutex> lock(mutex_);
      gen = ++gen_;
      fn_ = &fn;
      n_ = n;
      pending_.store(n);
      cursor_.store(static_cast<uint64_t>(gen) << 32);
    }
    wake_.notify_all();
    work(gen, &fn, n);
    std::unique_lock<std::mutex> lock(mutex_);
    done_.wait(lock, [this] { return pending_.load() == 0; });
  }

 private:
  void work(uint32_t gen, const std::function<void(int)>* fn, int n) {
    for (;;) {
      uint64_t cur = cursor_.load();
      if (static_cast<uint32_t>(cur >> 32) != gen) return;
      const int i = static_cast<int>(cur & 0xffffffffu);
      if (i >= n) return;
      if (!cursor_.compare_exchange_weak(cur, cur + 1)) continue;
      (*fn)(i);
      if (pending_.fetch_sub(1) == 1) {
        std::lock_guard<std::mutex> lock(mutex_);
        done_.notify_all();
      }
    }
  }
  void loop() {
    uint32_t seen = 0;
    for (;;) {
      uint32_t gen;
      const std::function<void(int)>* fn;
      int n;
      {
        std::unique_lock<std::mutex> lock(mutex_);
        wake_.wait(lock, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen = gen_;
        fn = fn_;
        n = n_;
      }
      work(gen, fn, n);
    }
  }
  std::vector<std::thread> threads_;
  std::mutex mutex_;
  std::condition_variable wake_, done_;
  bool stop_ = false;
  uint32_t gen_ = 0;
  const std::function<void(int)>* fn_ = nullptr;
  int n_ = 0;
  std::atomic<uint64_t> cursor_{0};
  std::atomic<int> pending_{0};
};

// ---- staging: every column of one direction in one block, laid out per call ----
//
// The caller's columns are gathered into one pinned host block and moved with a few large
// copies (and the results the other way), instead of one pageable copy per column, which the
// driver would stage through a small bounce buffer of its own.  Each column starts on a 256-byte
// boundary; the device block has the same layout, so the unpack and pack kernels read and write
// it in place.
struct Piece {
  const void* from;   // upload: the caller's column
  void* to;           // download: the caller's column (NULL: not wanted)
  size_t off, bytes;
  const char* name;
};

struct Plan {
  unsigned char* base = nullptr;   // the device block the kernels see
  size_t end = 0;
  std::vector<Piece> pieces;
  template <class T>
  T* in(const T* from, size_t n, const char* name) {
    pieces.push_back(Piece{from, nullptr, end, n * sizeof(T), name});
    return place<T>(n);
  }
  template <class T>
  T* out(T* to, size_t n, const char* name) {
    pieces.push_back(Piece{nullptr, to, end, n * sizeof(T), name});
    return place<T>(n);
  }

 private:
  template <class T>
  T* place(size_t n) {
    T* at = reinterpret_cast<T*>(base + end);
    end = (end + n * sizeof(T) + 255) & ~static_cast<size_t>(255);
    return at;
  }
};

// Splits a plan's pieces into at most `groups` runs of neighbouring pieces of similar size (the
// last run takes whatever is left, empty pieces included).
std::vector<std::pair<size_t, size_t>> piece_groups(const Plan& plan, int groups) {
  std::vector<std::pair<size_t, size_t>> out;   // [first piece, last piece + 1)
  const size_t total = plan.end, n = plan.pieces.size();
  size_t first = 0;
  for (size_t i = 0; i < n; i++) {
    const size_t upto = plan.pieces[i].off + plan.pieces[i].bytes;
    const size_t want = total * (out.size() + 1) / static_cast<size_t>(groups);
    if ((upto >= want && out.size() + 1 < static_cast<size_t>(groups)) || i + 1 == n) {
      out.emplace_back(first, i + 1);
      first = i + 1;
    }
  }
  return out;
}

// The ranges bg_register_host page-locked, every context's together (a registration belongs to
// the process, not to one context): base -> bytes.
std::mutex g_registry_mu;
std::map<uintptr_t, size_t> g_registered;

// Whether the host memory [p, p + bytes) is page-locked, so that the device can copy it directly
// with no gather through the library's own pinned block: inside one range bg_register_host locked,
// or (memory locked some other way, cudaHostAlloc'd say) page-locked as CUDA reports it.  A column
// that starts inside a registered range but runs past its end is staged.
bool host_pinned(const void* p, size_t bytes) {
  const uintptr_t at = reinterpret_cast<uintptr_t>(p);
  {
    std::lock_guard<std::mutex> lock(g_registry_mu);
    auto it = g_registered.upper_bound(at);
    if (it != g_registered.begin()) {
      --it;
      if (at < it->first + it->second) return at + bytes <= it->first + it->second;
    }
  }
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Host copies of up to 4 MiB each for pieces [first, last), run on the pool.
struct Slice {
  const unsigned char* from;
  unsigned char* to;
  size_t bytes;
};

void copy_slices(HostPool* pool, const std::vector<Slice>& slices) {
  pool->run(static_cast<int>(slices.size()), [&](int i) {
    const Slice& sl = slices[static_cast<size_t>(i)];
    std::memcpy(sl.to, sl.from, sl.bytes);
  });
}

void add_slices(std::vector<Slice>& slices, const unsigned char* from, unsigned char* to, size_t bytes) {
  constexpr size_t kSlice = 4u << 20;
  for (size_t at = 0; at < bytes; at += kSlice)
    slices.push_back(Slice{from + at, to + at, std::min(kSlice, bytes - at)});
}

}  // namespace

struct bg_ctx {
  int device = 0;
  uint32_t flags = 0;
  cudaStream_t stream = nullptr;
  std::string error;
  int sms = 0;
  int grid_blocks = 0;
  long long budget = kDefaultBudget;
  int last_launches = 0;
  cudaEvent_t stage_begin = nullptr, stage_end = nullptr;
  bool stage_timed = false;
  // capacities (stage_row_cap: rows the staging blocks hold; in_bytes: the upload block's size)
  int body_cap = 0, row_cap = 0, awake_cap = 0, world_cap = 0, stage_row_cap = 0;
  size_t in_bytes = 0;
  // device allocations, all freed in bg_destroy
  std::vector<void*> allocs;
  // body records
  bg::BodiesDev B = {};
  bg::RowsDev R = {};
  // staging in (caller layout)
  BodyStage bin = {};
  int32_t* awake_in = nullptr;
  RowStage rin = {};
  double* maxni_in = nullptr;
  double* relvel_in = nullptr;
  double* gap_in = nullptr;
  // device row d holds the caller's row perm[d]; iperm the other way (see order_rows)
  int32_t* perm_dev = nullptr;
  int32_t* iperm_dev = nullptr;
  std::vector<int32_t> perm, iperm;
  // the grid's dataflow schedule (see stage.cuh, flow_pass)
  int32_t* rank_dev = nullptr;     // rank_a then rank_b, by device row
  int32_t* deg_dev = nullptr;
  unsigned int* done_dev = nullptr;
  int2* chunks_dev = nullptr;
  int32_t* body_world_dev = nullptr;   // each body's world (a batch on the grid)
  int32_t* brun_rows_dev = nullptr;    // a batch's runs across worlds (see StageParams::bruns)
  int2* bruns_dev = nullptr;
  std::vector<int32_t> rank, deg, body_world, brun_rows;
  std::vector<int2> bruns;
  // batches: the order CTAs take the worlds in, and the threads a world's CTA has (0: tune on the
  // next batched solve, see tune_block_threads)
  int32_t* order_dev = nullptr;
  std::vector<int32_t> world_order;
  int block_threads = 0;
  std::vector<int2> chunks;
  int32_t nchunks = 0;   // the grid's runs (chunks.size(), or as the device worked them out)
  // bg_batch_solve_step's groups of worlds (see batch_in_groups): how many (0 by the batch's rows),
  // and a context of its own for each
  int batch_groups = 0;
  std::vector<bg_ctx*> kids;
  // staging out
  BodyOut bout = {};
  RowOut rout = {};
  // worlds
  bg::WorldDesc* worlds_dev = nullptr;
  int32_t* body_offset_dev = nullptr;
  int32_t* awake_offset_dev = nullptr;
  int32_t* row_offset_dev = nullptr;
  std::vector<bg::WorldDesc> worlds;
  // barrier and status
  unsigned int* bar = nullptr;   // the grid barrier's arrival count
  int32_t* status = nullptr;
  int32_t* block_counts = nullptr;
  // staging blocks, one per direction (see Plan), and the threads that fill and empty them
  unsigned char* d_in = nullptr;
  unsigned char* d_out = nullptr;
  unsigned char* h_in = nullptr;    // pinned
  unsigned char* h_out = nullptr;   // pinned
  unsigned char* h_meta = nullptr;  // pinned: order_rows()'s tables on their way to the device
  std::vector<void*> host_allocs;
  cudaEvent_t in_free = nullptr;    // the last upload's copies have read h_in
  bool in_pending = false;
  static constexpr int kGroups = 4; // copies a direction is split into, to overlap host and DMA
  cudaEvent_t out_ready[kGroups] = {};
  std::unique_ptr<HostPool> pool;
  // what was uploaded
  int nbodies = 0, nrows = 0, nawake = 0, nworlds = 0;
  bool uploaded = false;
  bool batch = false;
  // the host ranges bg_register_host page-locked for this context: (base, bytes)
  std::vector<std::pair<uintptr_t, size_t>> registered;
  // bg_collide's device block (grown by doubling, freed with the context) and its kernel's events
  struct Narrow {
    unsigned char* block = nullptr;
    size_t bodies = 0, pairs = 0;
    cudaEvent_t begin = nullptr, end = nullptr;
    bool timed = false;
  } nw;
  // bg_colour's device block and its events
  struct Colouring {
    unsigned char* block = nullptr;
    size_t bodies = 0, rows = 0;
    cudaEvent_t begin = nullptr, end = nullptr;
    bool timed = false;
  } col;
  // bg_contact_step's device memory: a scratch block for the call (grown by doubling) and two
  // banks of contact memory, the last call's `count` records in bank `current`
  struct Contact {
    unsigned char* block = nullptr;
    size_t bodies = 0, pairs = 0;
    unsigned char* banks = nullptr;
    size_t bank_cap = 0;
    int current = 0;
    int32_t count = 0;
    int32_t* summary = nullptr;   // pinned: the call's few counts on their way to the host
    cudaEvent_t ev[4] = {};
    bool timed = false;
  } ct;
  // bg_backward's own device memory (grown by doubling, freed with the context)
  struct Adjoint {
    std::vector<void*> allocs;
    size_t bodies = 0, rows = 0, awake = 0, worlds = 0, threads = 0;
    int substeps = 0;
    unsigned char* in = nullptr;     // the step's input columns
    unsigned char* work = nullptr;   // the recomputed state, records and adjoints
    bgad::Tape* tapes = nullptr;
    int32_t* status = nullptr;
    cudaEvent_t begin = nullptr, end = nullptr;
    int peak = 0;
    bool timed = false;
    int64_t bytes = 0;   // what the last kernel moves by design (see bg_backward_bytes)
  } adj;
};

namespace {

void set_error(bg_ctx* c, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  c->error = buf;
}

bool cuda_ok(bg_ctx* c, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  set_error(c, "%s: %s", what, cudaGetErrorString(e));
  return false;
}

template <class T>
bool dev_alloc(bg_ctx* c, T** p, size_t n) {
  void* q = nullptr;
  if (n == 0) n = 1;
  if (!cuda_ok(c, cudaMalloc(&q, n * sizeof(T)), "cudaMalloc")) return false;
  c->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return true;
}

bool host_alloc(bg_ctx* c, unsigned char** p, size_t n) {
  void* q = nullptr;
  if (n == 0) n = 1;
  if (!cuda_ok(c, cudaHostAlloc(&q, n, cudaHostAllocDefault), "cudaHostAlloc")) return false;
  c->host_allocs.push_back(q);
  *p = static_cast<unsigned char*>(q);
  return true;
}

void free_all(bg_ctx* c) {
  for (void* p : c->allocs) cudaFree(p);
  c->allocs.clear();
  for (void* p : c->host_allocs) cudaFreeHost(p);
  c->host_allocs.clear();
  c->in_pending = false;
}

// The upload's layout for b slots, r rows and na awake entries: sets the staging pointers the
// unpack kernels read (into `base`) and lists the caller's columns (NULL when only sizing).
Plan plan_in(bg_ctx* c, const bg_bodies* B, const bg_rows* R, size_t b, size_t r, size_t na, unsigned char* base) {
  Plan P;
  P.base = base;
  BodyStage& s = c->bin;
  s.position = P.in<double>(B ? B->position : nullptr, 3 * b, "position");
  s.rotation = P.in<double>(B ? B->rotation : nullptr, 4 * b, "rotation");
  s.velocity = P.in<double>(B ? B->velocity : nullptr, 3 * b, "velocity");
  s.angular = P.in<double>(B ? B->angular : nullptr, 3 * b, "angular");
  s.tumbled = P.in<double>(B ? B->tumbled : nullptr, 3 * b, "tumbled");
  s.ceiling = P.in<double>(B ? B->ceiling : nullptr, b, "ceiling");
  s.start = P.in<double>(B ? B->start : nullptr, 3 * b, "start");
  s.start_q = P.in<double>(B ? B->start_q : nullptr, 4 * b, "start_q");
  s.inv_mass = P.in<double>(B ? B->inv_mass : nullptr, b, "inv_mass");
  s.inertia = P.in<double>(B ? B->inertia : nullptr, 3 * b, "inertia");
  s.inv_inertia = P.in<double>(B ? B->inv_inertia : nullptr, 3 * b, "inv_inertia");
  s.dims = P.in<double>(B ? B->dims : nullptr, 3 * b, "dims");
  s.damping = P.in<double>(B ? B->damping : nullptr, b, "damping");
  s.angular_damping = P.in<double>(B ? B->angular_damping : nullptr, b, "angular_damping");
  s.gravity_scale = P.in<double>(B ? B->gravity_scale : nullptr, b, "gravity_scale");
  s.type = P.in<uint8_t>(B ? B->type : nullptr, b, "type");
  s.shape = P.in<uint8_t>(B ? B->shape : nullptr, b, "shape");
  s.frozen = P.in<uint8_t>(B ? B->frozen : nullptr, b, "frozen");
  s.framed = P.in<uint8_t>(B ? B->framed : nullptr, b, "framed");
  s.lock = P.in<uint8_t>(B ? B->lock : nullptr, b, "lock");
  s.joint_head = P.in<int32_t>(B ? B->joint_head : nullptr, b, "joint_head");
  s.awake = P.in<uint8_t>(B ? B->awake : nullptr, b, "awake");
  c->awake_in = P.in<int32_t>(B ? B->awake_list : nullptr, na, "awake_list");
  s.inv_i = P.in<double>(B ? B->inv_i : nullptr, 6 * b, "inv_i");
  RowStage& q = c->rin;
  q.row = P.in<int32_t>(R ? R->row : nullptr, r, "row");
  q.a = P.in<int32_t>(R ? R->a : nullptr, r, "a");
  q.b = P.in<int32_t>(R ? R->b : nullptr, r, "b");
  q.points = P.in<uint8_t>(R ? R->points : nullptr, r, "points");
  q.normal = P.in<double>(R ? R->normal : nullptr, 3 * r, "normal");
  q.t1 = P.in<double>(R ? R->t1 : nullptr, 3 * r, "t1");
  q.t2 = P.in<double>(R ? R->t2 : nullptr, 3 * r, "t2");
  q.friction = P.in<double>(R ? R->friction : nullptr, r, "friction");
  q.restitution = P.in<double>(R ? R->restitution : nullptr, r, "restitution");
  q.tolerance = P.in<double>(R ? R->tolerance : nullptr, r, "tolerance");
  q.patch = P.in<double>(R ? R->patch : nullptr, r, "patch");
  q.separation = P.in<double>(R ? R->separation : nullptr, 4 * r, "separation");
  q.point = P.in<double>(R ? R->point : nullptr, 12 * r, "point");
  q.shift = P.in<double>(R ? R->shift : nullptr, 12 * r, "shift");
  q.normal_impulse = P.in<double>(R ? R->normal_impulse : nullptr, 4 * r, "normal_impulse");
  q.ti1 = P.in<double>(R ? R->tangent_impulse1 : nullptr, r, "tangent_impulse1");
  q.ti2 = P.in<double>(R ? R->tangent_impulse2 : nullptr, r, "tangent_impulse2");
  q.ri1 = P.in<double>(R ? R->roll_impulse1 : nullptr, r, "roll_impulse1");
  q.ri2 = P.in<double>(R ? R->roll_impulse2 : nullptr, r, "roll_impulse2");
  q.si = P.in<double>(R ? R->spin_impulse : nullptr, r, "spin_impulse");
  q.drift1 = P.in<double>(R ? R->drift1 : nullptr, r, "drift1");
  q.drift2 = P.in<double>(R ? R->drift2 : nullptr, r, "drift2");
  c->maxni_in = P.in<double>(R ? R->max_normal_impulse : nullptr, 4 * r, "max_normal_impulse");
  c->relvel_in = P.in<double>(R ? R->relative_velocity : nullptr, 4 * r, "relative_velocity");
  c->gap_in = P.in<double>(R ? R->gap : nullptr, r, "gap");
  return P;
}

// The download's layout: sets the staging pointers the pack kernels write (into `base`) and lists
// the caller's columns (NULL when only sizing, or when the caller does not want a column).
Plan plan_out(bg_ctx* c, const bg_bodies* B, const bg_rows* R, size_t b, size_t r, unsigned char* base) {
  Plan P;
  P.base = base;
  BodyOut& o = c->bout;
  o.position = P.out<double>(B ? B->position : nullptr, 3 * b, "position");
  o.rotation = P.out<double>(B ? B->rotation : nullptr, 4 * b, "rotation");
  o.velocity = P.out<double>(B ? B->velocity : nullptr, 3 * b, "velocity");
  o.angular = P.out<double>(B ? B->angular : nullptr, 3 * b, "angular");
  o.tumbled = P.out<double>(B ? B->tumbled : nullptr, 3 * b, "tumbled");
  o.ceiling = P.out<double>(B ? B->ceiling : nullptr, b, "ceiling");
  o.start = P.out<double>(B ? B->start : nullptr, 3 * b, "start");
  o.start_q = P.out<double>(B ? B->start_q : nullptr, 4 * b, "start_q");
  o.inv_i = P.out<double>(B ? B->inv_i : nullptr, 6 * b, "inv_i");
  RowOut& q = c->rout;
  q.normal_impulse = P.out<double>(R ? R->normal_impulse : nullptr, 4 * r, "normal_impulse");
  q.ti1 = P.out<double>(R ? R->tangent_impulse1 : nullptr, r, "tangent_impulse1");
  q.ti2 = P.out<double>(R ? R->tangent_impulse2 : nullptr, r, "tangent_impulse2");
  q.ri1 = P.out<double>(R ? R->roll_impulse1 : nullptr, r, "roll_impulse1");
  q.ri2 = P.out<double>(R ? R->roll_impulse2 : nullptr, r, "roll_impulse2");
  q.si = P.out<double>(R ? R->spin_impulse : nullptr, r, "spin_impulse");
  q.drift1 = P.out<double>(R ? R->drift1 : nullptr, r, "drift1");
  q.drift2 = P.out<double>(R ? R->drift2 : nullptr, r, "drift2");
  q.gap = P.out<double>(R ? R->gap : nullptr, r, "gap");
  q.maxni = P.out<double>(R ? R->max_normal_impulse : nullptr, 4 * r, "max_normal_impulse");
  q.relvel = P.out<double>(R ? R->relative_velocity : nullptr, 4 * r, "relative_velocity");
  q.sliding = P.out<uint8_t>(R ? R->sliding : nullptr, r, "sliding");
  q.anchor_a = P.out<double>(R ? R->anchor_a : nullptr, 3 * r, "anchor_a");
  q.anchor_b = P.out<double>(R ? R->anchor_b : nullptr, 3 * r, "anchor_b");
  return P;
}

HostPool* pool_of(bg_ctx* c) {
  if (!c->pool) {
    const unsigned hw = std::thread::hardware_concurrency();
    const int workers = static_cast<int>(std::min(15u, hw > 1 ? hw - 1 : 0u));
    c->pool = std::make_unique<HostPool>(workers);
  }
  return c->pool.get();
}

size_t grown(size_t have, size_t want) {
  size_t c = have > 0 ? have : 64;
  while (c < want) c *= 2;
  return c;
}

// Bytes of the pinned block order_rows()'s tables pass through (see send_order).
size_t meta_bytes(size_t nb, size_t nr) {
  return 5 * nr * sizeof(int32_t) + 2 * nb * sizeof(int32_t) + 2 * (nr + 64) * sizeof(int2) + 8 * 256;
}

// (Re)allocates every buffer for at least the given sizes.  Everything is reallocated together,
// so a resize never leaves a stale pointer behind.  The staging blocks hold the columns of
// `stage_rows` rows (-1: nrows) and at least `in_need` bytes on the way in (bg_contact_step stages
// bodies and pairs, not rows).
bool ensure(bg_ctx* c, int nbodies, int nrows, int nawake, int nworlds, int stage_rows = -1, size_t in_need = 0) {
  if (stage_rows < 0) stage_rows = nrows;
  if (nbodies <= c->body_cap && nrows <= c->row_cap && nawake <= c->awake_cap && nworlds <= c->world_cap &&
      stage_rows <= c->stage_row_cap && in_need <= c->in_bytes && c->bar)
    return true;
  cudaStreamSynchronize(c->stream);
  free_all(c);
  const size_t nb = grown(c->body_cap, static_cast<size_t>(nbodies));
  const size_t nr = grown(c->row_cap, static_cast<size_t>(nrows));
  const size_t na = grown(c->awake_cap, static_cast<size_t>(nawake));
  const size_t nw = grown(c->world_cap, static_cast<size_t>(nworlds));
  const size_t sr = static_cast<size_t>(stage_rows) <= static_cast<size_t>(c->stage_row_cap)
                        ? static_cast<size_t>(c->stage_row_cap) : grown(c->stage_row_cap, static_cast<size_t>(stage_rows));
  bool ok = true;
  bg::BodiesDev& B = c->B;
  B.deg = nullptr;
  B.done = nullptr;
  ok = ok && dev_alloc(c, &B.vw, 8 * nb) && dev_alloc(c, &B.mi, 8 * nb) && dev_alloc(c, &B.pq, 8 * nb) &&
       dev_alloc(c, &B.st, 4 * nb) && dev_alloc(c, &B.sq, 4 * nb) && dev_alloc(c, &B.tc, 4 * nb) &&
       dev_alloc(c, &B.pr, 12 * nb) && dev_alloc(c, &B.fl, nb) && dev_alloc(c, &B.awake_list, na) &&
       dev_alloc(c, &B.head, nb);
  // rows
  bg::RowsDev& R = c->R;
  R.cap = static_cast<int64_t>(nr);
  ok = ok && dev_alloc(c, &R.a, nr) && dev_alloc(c, &R.b, nr) && dev_alloc(c, &R.points, nr) && dev_alloc(c, &R.row, nr) &&
       dev_alloc(c, &R.n, 3 * nr) && dev_alloc(c, &R.t1, 3 * nr) && dev_alloc(c, &R.t2, 3 * nr) &&
       dev_alloc(c, &R.friction, nr) && dev_alloc(c, &R.restitution, nr) && dev_alloc(c, &R.tolerance, nr) &&
       dev_alloc(c, &R.patch, nr) && dev_alloc(c, &R.separation, 4 * nr) && dev_alloc(c, &R.point, 12 * nr) &&
       dev_alloc(c, &R.shift, 12 * nr) && dev_alloc(c, &R.ni, 4 * nr) && dev_alloc(c, &R.ti1, nr) &&
       dev_alloc(c, &R.ti2, nr) && dev_alloc(c, &R.ri1, nr) && dev_alloc(c, &R.ri2, nr) && dev_alloc(c, &R.si, nr) &&
       dev_alloc(c, &R.drift1, nr) && dev_alloc(c, &R.drift2, nr) && dev_alloc(c, &R.gap, nr) &&
       dev_alloc(c, &R.maxni, 4 * nr) && dev_alloc(c, &R.relvel, 4 * nr) && dev_alloc(c, &R.sliding, nr) &&
       dev_alloc(c, &R.anchorA, 3 * nr) && dev_alloc(c, &R.anchorB, 3 * nr) && dev_alloc(c, &R.la, 12 * nr) &&
       dev_alloc(c, &R.lb, 12 * nr) && dev_alloc(c, &R.adjusted, 4 * nr) && dev_alloc(c, &R.now, 4 * nr) &&
       dev_alloc(c, &R.normalMass, 4 * nr) && dev_alloc(c, &R.lever, 4 * nr) && dev_alloc(c, &R.jac, 48 * nr) &&
       dev_alloc(c, &R.K, 16 * nr) && dev_alloc(c, &R.fjac, 24 * nr) && dev_alloc(c, &R.tm, 3 * nr) &&
       dev_alloc(c, &R.rm1, nr) && dev_alloc(c, &R.rm2, nr) && dev_alloc(c, &R.sm, nr) &&
       dev_alloc(c, &R.active, nr) && dev_alloc(c, &R.pending, nr);
  ok = ok && dev_alloc(c, &c->perm_dev, nr) && dev_alloc(c, &c->iperm_dev, nr) && dev_alloc(c, &c->rank_dev, 2 * nr) &&
       dev_alloc(c, &c->deg_dev, nb) && dev_alloc(c, &c->done_dev, nb) && dev_alloc(c, &c->chunks_dev, nr + 64) &&
       dev_alloc(c, &c->body_world_dev, nb) && dev_alloc(c, &c->brun_rows_dev, nr) && dev_alloc(c, &c->bruns_dev, nr + 64);
  // staging blocks, sized for the capacities (a call's own layout is never larger)
  size_t in_bytes = 0;
  {
    in_bytes = std::max(plan_in(c, nullptr, nullptr, nb, sr, na, nullptr).end, in_need);
    const size_t out_bytes = plan_out(c, nullptr, nullptr, nb, sr, nullptr).end;
    ok = ok && dev_alloc(c, &c->d_in, in_bytes) && dev_alloc(c, &c->d_out, out_bytes) &&
         host_alloc(c, &c->h_in, in_bytes) && host_alloc(c, &c->h_out, out_bytes) &&
         host_alloc(c, &c->h_meta, meta_bytes(nb, sr));
  }
  // worlds
  ok = ok && dev_alloc(c, &c->worlds_dev, nw) && dev_alloc(c, &c->order_dev, nw) && dev_alloc(c, &c->body_offset_dev, nw + 1) &&
       dev_alloc(c, &c->awake_offset_dev, nw + 1) && dev_alloc(c, &c->row_offset_dev, nw + 1);
  ok = ok && dev_alloc(c, &c->bar, 2) && dev_alloc(c, &c->status, 1) &&
       dev_alloc(c, &c->block_counts, static_cast<size_t>(c->grid_blocks > 0 ? c->grid_blocks : 1024));
  if (!ok) return false;
  if (!cuda_ok(c, cudaMemsetAsync(c->bar, 0, 2 * sizeof(unsigned int), c->stream), "cudaMemset")) return false;
  c->body_cap = static_cast<int>(nb);
  c->row_cap = static_cast<int>(nr);
  c->awake_cap = static_cast<int>(na);
  c->world_cap = static_cast<int>(nw);
  c->stage_row_cap = static_cast<int>(sr);
  c->in_bytes = in_bytes;
  return true;
}

template <class T>
bool put(bg_ctx* c, T* dst, const T* src, size_t n, const char* what) {
  if (n == 0) return true;
  if (src == nullptr) {
    set_error(c, "upload: column %s is NULL", what);
    return false;
  }
  return cuda_ok(c, cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, c->stream), what);
}

int validate(bg_ctx* c, const bg_bodies* B, const bg_rows* R) {
  if (B == nullptr || R == nullptr) {
    set_error(c, "bodies and rows must not be NULL");
    return BG_EINVAL;
  }
  if (B->capacity < 0 || B->awake_count < 0 || B->awake_count > B->capacity || R->count < 0) {
    set_error(c, "negative or inconsistent counts");
    return BG_EINVAL;
  }
  return BG_OK;
}

// What is wrong with a world's colour starts (src/contact.js:161, src/graph.js:178-214), or NULL:
// they begin at 0, never decrease, the resting run begins at `solved`, and none passes `nrows`.
const char* starts_problem(int nrows, const int32_t* starts, int solved) {
  if (starts[0] != 0) return "rows.starts[0] must be 0";
  for (int k = 0; k < bg::NSTARTS - 1; k++)
    if (starts[k + 1] < starts[k]) return "rows.starts must not decrease";
  if (starts[bg::RESTING_RUN] != solved || solved > nrows || starts[bg::NSTARTS - 1] > nrows)
    return "rows.solved must equal starts[33] and be at most count";
  return nullptr;
}

int validate_world(bg_ctx* c, int nbodies, int nrows, const int32_t* starts, int solved) {
  const char* why = starts_problem(nrows, starts, solved);
  if (why != nullptr) {
    set_error(c, "%s", why);
    return BG_EINVAL;
  }
  (void)nbodies;
  return BG_OK;
}

// Every index the caller hands over for worlds [w0, w1), checked before any of them addresses
// memory (host tables or device records): each row's a and b among its world's slots, its point
// count 1..P, row[] a permutation of the world's rows (the found order, src/graph.js:205-214), and
// each awake entry among the world's slots.  `seen` has one byte per row of the whole upload,
// zero over these worlds' rows.  Returns NULL, or what is wrong (with the row or entry in `why`).
const char* index_problem(const bg_bodies* B, const bg_rows* R, const std::vector<bg::WorldDesc>& worlds, size_t w0,
                          size_t w1, uint8_t* seen, char* why, size_t why_len) {
  if (R->count > 0 && (R->a == nullptr || R->b == nullptr || R->points == nullptr || R->row == nullptr))
    return "rows.a, rows.b, rows.points and rows.row must be given";
  if (B->awake_count > 0 && B->awake_list == nullptr) return "bodies.awake_list must be given";
  for (size_t wi = w0; wi < w1; wi++) {
    const bg::WorldDesc& w = worlds[wi];
    const int32_t* a = R->a + w.row0;
    const int32_t* b = R->b + w.row0;
    const uint8_t* pts = R->points + w.row0;
    for (int m = 0; m < w.nrows; m++) {
      if (static_cast<uint32_t>(a[m]) >= static_cast<uint32_t>(w.nbodies) ||
          static_cast<uint32_t>(b[m]) >= static_cast<uint32_t>(w.nbodies)) {
        snprintf(why, why_len, "rows.a / rows.b of row %d (world %zu) is not one of its %d slots", m, wi, w.nbodies);
        return why;
      }
      if (pts[m] < 1 || pts[m] > bg::P) {
        snprintf(why, why_len, "rows.points of row %d (world %zu) is %d, not 1..%d", m, wi, pts[m], bg::P);
        return why;
      }
    }
    const int32_t* row = R->row + w.row0;
    uint8_t* mark = seen + w.row0;
    for (int f = 0; f < w.nrows; f++) {
      const int32_t x = row[f];
      if (static_cast<uint32_t>(x) >= static_cast<uint32_t>(w.nrows) || mark[x] != 0) {
        snprintf(why, why_len, "rows.row is not a permutation of the rows (entry %d of world %zu)", f, wi);
        return why;
      }
      mark[x] = 1;
    }
    const int32_t* awake = B->awake_list + w.awake0;
    for (int i = 0; i < w.nawake; i++)
      if (static_cast<uint32_t>(awake[i]) >= static_cast<uint32_t>(w.nbodies)) {
        snprintf(why, why_len, "bodies.awake_list entry %d (world %zu) is not one of its %d slots", i, wi, w.nbodies);
        return why;
      }
  }
  return nullptr;
}

// Copies the caller's columns for `nb` slots / `nr` rows / `na` awake entries to the device.  A
// page-locked column is copied straight from the caller's memory; the others are gathered by the
// pool into the library's pinned block a group at a time, each group's copy to the device starting
// as soon as it is gathered, while the next group is.  Returns with the copies in flight.
int upload_plan(bg_ctx* c, const Plan& plan);

int upload_columns(bg_ctx* c, const bg_bodies* B, const bg_rows* R, int nb, int nr, int na) {
  return upload_plan(c, plan_in(c, B, R, static_cast<size_t>(nb), static_cast<size_t>(nr), static_cast<size_t>(na), c->d_in));
}

// The columns a plan lists, copied into the device block at their places (see upload_columns).
int upload_plan(bg_ctx* c, const Plan& plan) {
  for (const Piece& pc : plan.pieces)
    if (pc.bytes > 0 && pc.from == nullptr) {
      set_error(c, "upload: column %s is NULL", pc.name);
      return BG_EINVAL;
    }
  Plan staged;   // the pageable columns, at their places in the device block
  staged.end = plan.end;
  for (const Piece& pc : plan.pieces) {
    if (pc.bytes == 0) continue;
    if (host_pinned(pc.from, pc.bytes)) {
      if (!cuda_ok(c, cudaMemcpyAsync(c->d_in + pc.off, pc.from, pc.bytes, cudaMemcpyHostToDevice, c->stream), "upload"))
        return BG_ECUDA;
    } else {
      staged.pieces.push_back(pc);
    }
  }
  if (staged.pieces.empty()) return BG_OK;
  // The last upload's copies must be done reading the pinned block before it is refilled.
  if (c->in_pending && !cuda_ok(c, cudaEventSynchronize(c->in_free), "upload")) return BG_ECUDA;
  c->in_pending = false;
  HostPool* pool = pool_of(c);
  for (const auto& g : piece_groups(staged, bg_ctx::kGroups)) {
    std::vector<Slice> slices;
    for (size_t k = g.first; k < g.second; k++) {
      const Piece& pc = staged.pieces[k];
      add_slices(slices, static_cast<const unsigned char*>(pc.from), c->h_in + pc.off, pc.bytes);
    }
    copy_slices(pool, slices);
    // One copy per run of staged pieces that lie next to each other in the block: a column copied
    // straight from the caller's memory between two of them must not be overwritten with whatever
    // the staging block holds at its place.
    for (size_t k = g.first; k < g.second;) {
      const size_t lo = staged.pieces[k].off;
      size_t hi = lo + staged.pieces[k].bytes;
      size_t e = k + 1;
      while (e < g.second && staged.pieces[e].off <= ((hi + 255) & ~static_cast<size_t>(255))) {
        hi = staged.pieces[e].off + staged.pieces[e].bytes;
        e++;
      }
      if (hi > lo &&
          !cuda_ok(c, cudaMemcpyAsync(c->d_in + lo, c->h_in + lo, hi - lo, cudaMemcpyHostToDevice, c->stream), "upload"))
        return BG_ECUDA;
      k = e;
    }
  }
  if (!cuda_ok(c, cudaEventRecord(c->in_free, c->stream), "upload")) return BG_ECUDA;
  c->in_pending = true;
  return BG_OK;
}

// The order rows are solved in on the device: within each colour, rows by point count (a
// colour's rows share no body the solve moves, so their order changes no result, src/graph.js:1-33),
// which keeps a warp's 32 rows on one code path.  The overflow and resting runs keep their order
// (the overflow is solved in row order, src/contact.js:1794-1795).
// Every caller index is checked first (index_problem), so nothing here or on the device reads
// through a bad one; a refusal comes back in `err`, since this runs beside the caller's thread.
int order_rows(bg_ctx* c, const bg_bodies* B, const bg_rows* R, std::string& err) {
  {
    std::vector<uint8_t> seen(static_cast<size_t>(c->nrows), 0);
    char why[256];
    const char* bad = index_problem(B, R, c->worlds, 0, c->worlds.size(), seen.data(), why, sizeof why);
    if (bad != nullptr) {
      err = bad;
      return BG_EINVAL;
    }
  }
  const uint8_t* points = R->points;
  const int32_t* a = R->a;
  const int32_t* b = R->b;
  const double* inv_mass = B->inv_mass;
  const int n = c->nrows;
  c->perm.resize(static_cast<size_t>(n));
  c->iperm.resize(static_cast<size_t>(n));
  for (const bg::WorldDesc& w : c->worlds) {
    for (int k = 0; k < bg::NSTARTS - 1; k++) {
      const int from = w.starts[k], to = k < bg::RESTING_RUN ? w.starts[k + 1] : w.nrows;
      if (to <= from) continue;
      if (k >= bg::OVERFLOW_RUN) {
        for (int m = from; m < to; m++) c->perm[static_cast<size_t>(w.row0 + m)] = w.row0 + m;
        continue;
      }
      // a stable counting sort on the point count (1..P): one pass to count, one to place
      auto count_of = [&](int m) {
        const int pc = points[w.row0 + m];
        return pc < 1 ? 1 : pc > bg::P ? bg::P : pc;
      };
      int at[bg::P + 1] = {0};
      for (int m = from; m < to; m++) at[count_of(m)]++;
      for (int k2 = 1, next = from; k2 <= bg::P; k2++) {
        const int here = at[k2];
        at[k2] = next;
        next += here;
      }
      for (int m = from; m < to; m++) c->perm[static_cast<size_t>(w.row0 + at[count_of(m)]++)] = w.row0 + m;
    }
  }
  for (int d = 0; d < n; d++) c->iperm[static_cast<size_t>(c->perm[static_cast<size_t>(d)])] = d;
  // Each solved row's place among the rows on each body it moves, in device (solve) order, and
  // each body's count of them: what the grid's dataflow waits on.
  c->rank.assign(2 * static_cast<size_t>(n), -1);
  c->deg.assign(static_cast<size_t>(c->nbodies), 0);
  for (const bg::WorldDesc& w : c->worlds) {
    for (int d = w.row0; d < w.row0 + w.solved; d++) {
      const int m = c->perm[static_cast<size_t>(d)];
      const int x = a[m] + w.body0, y = b[m] + w.body0;
      if (inv_mass[x] != 0) c->rank[static_cast<size_t>(d)] = c->deg[static_cast<size_t>(x)]++;
      if (inv_mass[y] != 0) c->rank[static_cast<size_t>(n) + d] = c->deg[static_cast<size_t>(y)]++;
    }
  }
  // The grid's runs: each colour's rows in runs of up to 32 that also end where the point count
  // changes, so every warp runs one row solver (a warp whose lanes take two point counts runs the
  // two one after the other), then the overflow's one row a run.
  c->chunks.clear();
  for (const bg::WorldDesc& w : c->worlds) {
    for (int k = 0; k < bg::NCOLOURS; k++) {
      int m = w.row0 + w.starts[k];
      while (m < w.row0 + w.starts[k + 1]) {
        const int pc = points[c->perm[static_cast<size_t>(m)]];
        int e = m + 1;
        while (e < w.row0 + w.starts[k + 1] && e - m < 32 && points[c->perm[static_cast<size_t>(e)]] == pc) e++;
        c->chunks.push_back(make_int2(m, e - m));
        m = e;
      }
    }
    for (int m = w.starts[bg::OVERFLOW_RUN]; m < w.starts[bg::OVERFLOW_RUN + 1]; m++) c->chunks.push_back(make_int2(w.row0 + m, 1));
  }
  c->nchunks = static_cast<int32_t>(c->chunks.size());
  // A batch's runs for the grid: every world's rows of one colour and one point count together
  // (rows of different worlds share no body), 32 a run, colour after colour; then each world's
  // overflow rows, one a run, in their order.  Each run's rows wait only on rows of earlier runs.
  // (A batch of one world needs them too: it may run on the grid as a batch.)
  c->brun_rows.clear();
  c->bruns.clear();
  if (c->batch) {
    for (int k = 0; k < bg::NCOLOURS; k++)
      for (int pc = 1; pc <= bg::P; pc++) {
        const size_t first = c->brun_rows.size();
        for (const bg::WorldDesc& w : c->worlds)
          for (int d = w.row0 + w.starts[k]; d < w.row0 + w.starts[k + 1]; d++) {
            const int q = points[c->perm[static_cast<size_t>(d)]];
            if ((q < 1 ? 1 : q > bg::P ? bg::P : q) == pc) c->brun_rows.push_back(d);
          }
        for (size_t r = first; r < c->brun_rows.size(); r += 32)
          c->bruns.push_back(make_int2(static_cast<int>(r), static_cast<int>(std::min<size_t>(32, c->brun_rows.size() - r))));
      }
    for (const bg::WorldDesc& w : c->worlds)
      for (int m = w.starts[bg::OVERFLOW_RUN]; m < w.starts[bg::OVERFLOW_RUN + 1]; m++) {
        c->bruns.push_back(make_int2(static_cast<int>(c->brun_rows.size()), 1));
        c->brun_rows.push_back(w.row0 + m);
      }
  }
  // each body's world, for the body passes of a batch on the grid
  c->body_world.assign(static_cast<size_t>(c->nbodies), 0);
  for (size_t wi = 0; wi < c->worlds.size(); wi++) {
    const bg::WorldDesc& w = c->worlds[wi];
    for (int x = w.body0; x < w.body0 + w.nbodies; x++) c->body_world[static_cast<size_t>(x)] = static_cast<int32_t>(wi);
  }
  return BG_OK;
}

// order_rows()'s tables to the device, through the pinned block (a copy from pageable memory would
// first wait for everything queued on the stream, the columns' copies included).
int send_order(bg_ctx* c) {
  const size_t n = static_cast<size_t>(c->nrows);
  unsigned char* h = c->h_meta;
  size_t off = 0;
  auto send = [&](void* dev, const void* host, size_t bytes) {
    if (bytes == 0) return true;
    std::memcpy(h + off, host, bytes);
    const bool ok = cuda_ok(c, cudaMemcpyAsync(dev, h + off, bytes, cudaMemcpyHostToDevice, c->stream), "order");
    off = (off + bytes + 255) & ~static_cast<size_t>(255);
    return ok;
  };
  const bool ok = send(c->perm_dev, c->perm.data(), n * sizeof(int32_t)) &&
                  send(c->iperm_dev, c->iperm.data(), n * sizeof(int32_t)) &&
                  send(c->rank_dev, c->rank.data(), 2 * n * sizeof(int32_t)) &&
                  send(c->deg_dev, c->deg.data(), static_cast<size_t>(c->nbodies) * sizeof(int32_t)) &&
                  send(c->chunks_dev, c->chunks.data(), c->chunks.size() * sizeof(int2)) &&
                  send(c->body_world_dev, c->body_world.data(), c->body_world.size() * sizeof(int32_t)) &&
                  send(c->brun_rows_dev, c->brun_rows.data(), c->brun_rows.size() * sizeof(int32_t)) &&
                  send(c->bruns_dev, c->bruns.data(), c->bruns.size() * sizeof(int2));
  return ok ? BG_OK : BG_ECUDA;
}

// The caller's columns and the solve order, together: order_rows() works on its own thread while
// the pool gathers the columns and their copies start.
int upload_and_order(bg_ctx* c, const bg_bodies* B, const bg_rows* R) {
  if ((c->nrows > 0 && (R->points == nullptr || R->a == nullptr || R->b == nullptr)) ||
      (c->nbodies > 0 && B->inv_mass == nullptr)) {
    set_error(c, "upload: rows.points, rows.a, rows.b and bodies.inv_mass must be given");
    return BG_EINVAL;
  }
  int order_rc = BG_OK;
  std::string order_err;
  std::thread orderer([&] {
    try {
      order_rc = order_rows(c, B, R, order_err);
    } catch (const std::exception&) {
      order_rc = BG_ENOMEM;
      order_err = "upload: out of host memory";
    }
  });
  const int rc = upload_columns(c, B, R, c->nbodies, c->nrows, c->nawake);
  orderer.join();
  if (order_rc != BG_OK) {
    // A refused index: no kernel has run on this input.  The copies already issued only read the
    // caller's columns; they finish before the call returns, and the context is left with nothing
    // uploaded (the caller's arrays are untouched).
    cudaStreamSynchronize(c->stream);
    c->in_pending = false;
    set_error(c, "%s", order_err.c_str());
    return order_rc;
  }
  if (rc != BG_OK) return rc;
  return send_order(c);
}

int unpack(bg_ctx* c) {
  const int nb = c->nbodies, nr = c->nrows, na = c->nawake;
  const int blocks = std::max(1, std::min(4 * c->sms, (std::max(nb, std::max(nr, na)) + kUnpackThreads - 1) / kUnpackThreads));
  unpack_bodies<<<blocks, kUnpackThreads, 0, c->stream>>>(c->bin, c->B, nb, c->awake_in, na, c->body_offset_dev,
                                                         c->awake_offset_dev, c->nworlds);
  unpack_rows<<<blocks, kUnpackThreads, 0, c->stream>>>(c->rin, c->R, nr, c->row_offset_dev, c->body_offset_dev, c->nworlds,
                                                       c->maxni_in, c->relvel_in, c->gap_in, c->perm_dev, c->iperm_dev);
  c->last_launches += 2;
  return cuda_ok(c, cudaGetLastError(), "unpack") ? BG_OK : BG_ECUDA;
}

int upload_worlds(bg_ctx* c, const std::vector<int32_t>& body_off, const std::vector<int32_t>& awake_off,
                  const std::vector<int32_t>& row_off) {
  const size_t nw = c->worlds.size();
  // CTAs take a batch's worlds largest first (solved rows, then slots), so the longest worlds
  // start in the first wave rather than the last; worlds are independent, so no result changes.
  c->world_order.resize(nw);
  for (size_t i = 0; i < nw; i++) c->world_order[i] = static_cast<int32_t>(i);
  std::stable_sort(c->world_order.begin(), c->world_order.end(), [&](int32_t x, int32_t y) {
    const bg::WorldDesc &a = c->worlds[static_cast<size_t>(x)], &b = c->worlds[static_cast<size_t>(y)];
    return a.solved != b.solved ? a.solved > b.solved : a.nbodies > b.nbodies;
  });
  bool ok = put(c, c->worlds_dev, c->worlds.data(), nw, "worlds") &&
            put(c, c->order_dev, c->world_order.data(), nw, "world order") &&
            put(c, c->body_offset_dev, body_off.data(), nw + 1, "body_offset") &&
            put(c, c->awake_offset_dev, awake_off.data(), nw + 1, "awake_offset") &&
            put(c, c->row_offset_dev, row_off.data(), nw + 1, "row_offset");
  // The host vectors must outlive the asynchronous copies.
  ok = ok && cuda_ok(c, cudaStreamSynchronize(c->stream), "upload worlds");
  return ok ? BG_OK : BG_ECUDA;
}

// makeSoft: src/contact.js:1591-1597, for STIFFNESS / h and DAMPING_RATIO (src/world.js:115-118).
bg::Soft make_soft(double h) {
  const double hertz = (1.0 / 8.0) / h, zeta = 10;
  const double omega = 2 * 3.141592653589793 * hertz;
  const double a1 = 2 * zeta + h * omega, a2 = h * omega * a1, a3 = 1 / (1 + a2);
  return bg::Soft{omega / a1, a2 * a3, a3};
}

int launch_stage(bg_ctx* c, const bg_step* step) {
  if (step == nullptr || !(step->dt > 0) || step->substeps < 1) {
    set_error(c, "step: dt must be positive and substeps at least 1");
    return BG_EINVAL;
  }
  bg::StageParams p;
  p.B = c->B;
  p.R = c->R;
  p.worlds = c->worlds_dev;
  p.nworlds = c->nworlds;
  p.dt = step->dt;
  p.substeps = step->substeps;
  p.soft = make_soft(step->dt / step->substeps);
  p.bar_count = c->bar;
  p.status = c->status;
  p.block_counts = c->block_counts;
  p.budget = c->budget;
  p.B.deg = c->deg_dev;
  p.B.done = c->done_dev;
  p.R.rank_a = c->rank_dev;
  p.R.rank_b = c->rank_dev + c->nrows;
  p.chunks = c->chunks_dev;
  p.nchunks = c->nchunks;
  p.world_order = c->batch ? c->order_dev : nullptr;
  p.body_world = c->body_world_dev;
  p.nawake_total = c->nawake;
  p.brun_rows = c->brun_rows_dev;
  p.bruns = c->bruns_dev;
  p.nbruns = static_cast<int32_t>(c->bruns.size());
  if (!cuda_ok(c, cudaMemsetAsync(c->done_dev, 0, sizeof(unsigned int) * static_cast<size_t>(c->nbodies > 0 ? c->nbodies : 1),
                                  c->stream), "done")) return BG_ECUDA;
  if (!cuda_ok(c, cudaMemsetAsync(c->status, 0, sizeof(int32_t), c->stream), "status")) return BG_ECUDA;
  // The grid barrier's arrival count starts at zero for every launch (it only grows within one,
  // and a launch that lost its step can leave it anywhere).
  if (!cuda_ok(c, cudaMemsetAsync(c->bar, 0, sizeof(unsigned int), c->stream), "barrier")) return BG_ECUDA;
  c->last_launches += 1;
  cudaEventRecord(c->stage_begin, c->stream);
  if (c->batch && c->block_threads == BG_BATCH_ON_GRID) {
    void* args[] = {&p};
    const cudaError_t e = cudaLaunchCooperativeKernel(reinterpret_cast<void*>(stage_grid_batch), dim3(c->grid_blocks),
                                                      dim3(kGridThreads), args, 0, c->stream);
    if (!cuda_ok(c, e, "stage_grid_batch launch")) return BG_ECUDA;
    cudaEventRecord(c->stage_end, c->stream);
    c->stage_timed = true;
    return BG_OK;
  }
  bool big = !c->batch && c->nworlds == 1;
  if (!c->batch && (c->flags & BG_FLAG_GRID)) big = true;
  if (!c->batch && (c->flags & BG_FLAG_BLOCK)) big = false;
  if (big) {
    void* args[] = {&p};
    const cudaError_t e = cudaLaunchCooperativeKernel(reinterpret_cast<void*>(stage_grid), dim3(c->grid_blocks),
                                                      dim3(kGridThreads), args, 0, c->stream);
    if (!cuda_ok(c, e, "stage_grid launch")) return BG_ECUDA;
  } else {
    const int threads = c->batch && c->block_threads > 0 ? c->block_threads : kBlockThreads;
    const int blocks = std::min(c->nworlds, 64 * c->sms);
    stage_block<<<blocks, threads, 0, c->stream>>>(p);
    if (!cuda_ok(c, cudaGetLastError(), "stage_block launch")) return BG_ECUDA;
  }
  cudaEventRecord(c->stage_end, c->stream);
  c->stage_timed = true;
  return BG_OK;
}

int finish(bg_ctx* c) {
  const int nb = c->nbodies, nr = c->nrows;
  plan_out(c, nullptr, nullptr, static_cast<size_t>(nb), static_cast<size_t>(nr), c->d_out);
  const int blocks = std::max(1, std::min(4 * c->sms, (std::max(nb, nr) + kUnpackThreads - 1) / kUnpackThreads));
  pack_bodies<<<blocks, kUnpackThreads, 0, c->stream>>>(c->B, c->bout, nb);
  pack_rows<<<blocks, kUnpackThreads, 0, c->stream>>>(c->R, c->rout, nr, c->perm_dev);
  c->last_launches += 2;
  return cuda_ok(c, cudaGetLastError(), "pack") ? BG_OK : BG_ECUDA;
}

// The results back to the caller's columns.  A page-locked column is copied straight into the
// caller's memory; for the others, each group of the pinned block is copied from the device and,
// once it has landed, scattered to the caller's columns by the pool while the next group is still
// on its way.
int download_columns(bg_ctx* c, const bg_bodies* B, const bg_rows* R) {
  const Plan all = plan_out(c, B, R, static_cast<size_t>(c->nbodies), static_cast<size_t>(c->nrows), c->d_out);
  Plan plan;   // the columns going through the pinned block
  plan.end = all.end;
  bool ok = true;
  for (const Piece& pc : all.pieces) {
    if (pc.bytes == 0 || pc.to == nullptr) continue;
    if (host_pinned(pc.to, pc.bytes))
      ok = ok && cuda_ok(c, cudaMemcpyAsync(pc.to, c->d_out + pc.off, pc.bytes, cudaMemcpyDeviceToHost, c->stream),
                         "download");
    else
      plan.pieces.push_back(pc);
  }
  const auto groups = plan.pieces.empty() ? std::vector<std::pair<size_t, size_t>>() : piece_groups(plan, bg_ctx::kGroups);
  for (size_t gi = 0; gi < groups.size() && ok; gi++) {
    const auto& g = groups[gi];
    const size_t lo = plan.pieces[g.first].off;
    const size_t hi = plan.pieces[g.second - 1].off + plan.pieces[g.second - 1].bytes;
    if (hi > lo)
      ok = cuda_ok(c, cudaMemcpyAsync(c->h_out + lo, c->d_out + lo, hi - lo, cudaMemcpyDeviceToHost, c->stream), "download");
    ok = ok && cuda_ok(c, cudaEventRecord(c->out_ready[gi], c->stream), "download");
  }
  HostPool* pool = pool_of(c);
  for (size_t gi = 0; gi < groups.size() && ok; gi++) {
    ok = cuda_ok(c, cudaEventSynchronize(c->out_ready[gi]), "download");
    if (!ok) break;
    std::vector<Slice> slices;
    for (size_t k = groups[gi].first; k < groups[gi].second; k++) {
      const Piece& pc = plan.pieces[k];
      if (pc.to != nullptr) add_slices(slices, c->h_out + pc.off, static_cast<unsigned char*>(pc.to), pc.bytes);
    }
    copy_slices(pool, slices);
  }
  int32_t status = 0;
  ok = ok && cuda_ok(c, cudaMemcpyAsync(&status, c->status, sizeof status, cudaMemcpyDeviceToHost, c->stream), "status") &&
       cuda_ok(c, cudaStreamSynchronize(c->stream), "synchronize");
  if (!ok) return BG_ECUDA;
  if (status != 0) {
    set_error(c, "a grid barrier waited past its budget; the step is lost");
    return BG_ETIMEOUT;
  }
  return BG_OK;
}

// Waits for every copy this context (and its groups' contexts) may have in flight, then releases
// the ranges it registered.
void release_registered(bg_ctx* c) {
  if (c->registered.empty()) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (bg_ctx* k : c->kids)
    if (k->stream) cudaStreamSynchronize(k->stream);
  std::lock_guard<std::mutex> lock(g_registry_mu);
  for (const auto& r : c->registered) {
    cudaHostUnregister(reinterpret_cast<void*>(r.first));
    g_registered.erase(r.first);
  }
  cudaGetLastError();
  c->registered.clear();
}

// Every non-NULL column of B and R, in and out, for nb slots and nr rows, as page-aligned
// ranges, sorted, with ranges that overlap or touch merged (two columns on one page are one range).
std::vector<std::pair<uintptr_t, uintptr_t>> column_pages(bg_ctx* c, const bg_bodies* B, const bg_rows* R, size_t nb,
                                                          size_t nr) {
  // plan_in and plan_out set the context's staging pointers as they go: keep the uploaded ones
  const BodyStage bin = c->bin;
  const RowStage rin = c->rin;
  const BodyOut bout = c->bout;
  const RowOut rout = c->rout;
  int32_t* const awake_in = c->awake_in;
  double* const maxni_in = c->maxni_in;
  double* const relvel_in = c->relvel_in;
  double* const gap_in = c->gap_in;
  const Plan in = plan_in(c, B, R, nb, nr, nb, nullptr);
  const Plan out = plan_out(c, B, R, nb, nr, nullptr);
  c->bin = bin; c->rin = rin; c->bout = bout; c->rout = rout; c->awake_in = awake_in;
  c->maxni_in = maxni_in; c->relvel_in = relvel_in; c->gap_in = gap_in;
  const uintptr_t page = static_cast<uintptr_t>(sysconf(_SC_PAGESIZE) > 0 ? sysconf(_SC_PAGESIZE) : 4096);
  std::vector<std::pair<uintptr_t, uintptr_t>> spans;
  auto add = [&](const void* p, size_t bytes) {
    if (p == nullptr || bytes == 0) return;
    const uintptr_t lo = reinterpret_cast<uintptr_t>(p) / page * page;
    const uintptr_t hi = (reinterpret_cast<uintptr_t>(p) + bytes + page - 1) / page * page;
    spans.emplace_back(lo, hi);
  };
  for (const Piece& pc : in.pieces) add(pc.from, pc.bytes);
  for (const Piece& pc : out.pieces) add(pc.to, pc.bytes);
  std::sort(spans.begin(), spans.end());
  std::vector<std::pair<uintptr_t, uintptr_t>> merged;
  for (const auto& s : spans) {
    if (!merged.empty() && s.first <= merged.back().second)
      merged.back().second = std::max(merged.back().second, s.second);
    else
      merged.push_back(s);
  }
  return merged;
}

}  // namespace

extern "C" {

uint32_t bg_version(void) { return (1u << 16) | 0u; }

bg_ctx* bg_create(int32_t device, uint32_t flags) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return nullptr;
  bg_ctx* c = new bg_ctx();
  c->device = device;
  c->flags = flags;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return nullptr;
  }
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
  cudaEventCreate(&c->stage_begin);
  cudaEventCreate(&c->stage_end);
  cudaEventCreateWithFlags(&c->in_free, cudaEventDisableTiming);
  for (cudaEvent_t& e : c->out_ready) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, stage_grid, kGridThreads, 0);
  if (per_sm < 1) per_sm = 1;
  // One block an SM: every colour's rows are spread over all of them (GridTeam::each), and fewer
  // blocks make each grid barrier cheaper.
  (void)per_sm;
  c->grid_blocks = c->sms;
  if (c->grid_blocks > 1024) c->grid_blocks = 1024;
  return c;
}

void bg_destroy(bg_ctx* c) {
  if (c == nullptr) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  release_registered(c);
  for (bg_ctx* k : c->kids) bg_destroy(k);
  c->kids.clear();
  free_all(c);
  for (void* p : c->adj.allocs) cudaFree(p);
  c->adj.allocs.clear();
  if (c->nw.block) cudaFree(c->nw.block);
  if (c->ct.block) cudaFree(c->ct.block);
  if (c->ct.banks) cudaFree(c->ct.banks);
  if (c->ct.summary) cudaFreeHost(c->ct.summary);
  for (cudaEvent_t e : c->ct.ev)
    if (e) cudaEventDestroy(e);
  if (c->col.block) cudaFree(c->col.block);
  if (c->col.begin) cudaEventDestroy(c->col.begin);
  if (c->col.end) cudaEventDestroy(c->col.end);
  if (c->nw.begin) cudaEventDestroy(c->nw.begin);
  if (c->nw.end) cudaEventDestroy(c->nw.end);
  if (c->adj.begin) cudaEventDestroy(c->adj.begin);
  if (c->adj.end) cudaEventDestroy(c->adj.end);
  c->pool.reset();
  if (c->in_free) cudaEventDestroy(c->in_free);
  for (cudaEvent_t e : c->out_ready)
    if (e) cudaEventDestroy(e);
  if (c->stage_begin) cudaEventDestroy(c->stage_begin);
  if (c->stage_end) cudaEventDestroy(c->stage_end);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char* bg_last_error(const bg_ctx* c) { return c == nullptr ? "no context" : c->error.c_str(); }

void* bg_stream(bg_ctx* c) { return c == nullptr ? nullptr : static_cast<void*>(c->stream); }

int32_t bg_register_host(bg_ctx* c, const bg_bodies* B, const bg_rows* R, int32_t row_capacity) {
  if (c == nullptr) return BG_EINVAL;
  if (B == nullptr || R == nullptr) {
    set_error(c, "bg_register_host: bodies or rows is NULL");
    return BG_EINVAL;
  }
  if (B->capacity < 0 || R->count < 0 || row_capacity < R->count) {
    set_error(c, "bg_register_host: capacity %d, row count %d, row capacity %d", B->capacity, R->count, row_capacity);
    return BG_EINVAL;
  }
  cudaSetDevice(c->device);
  const auto spans = column_pages(c, B, R, static_cast<size_t>(B->capacity), static_cast<size_t>(row_capacity));
  release_registered(c);
  std::lock_guard<std::mutex> lock(g_registry_mu);
  for (const auto& s : spans) {
    const size_t bytes = s.second - s.first;
    const cudaError_t e = cudaHostRegister(reinterpret_cast<void*>(s.first), bytes, cudaHostRegisterPortable);
    if (e == cudaErrorHostMemoryAlreadyRegistered) {   // someone else's: theirs to keep or release
      cudaGetLastError();
      continue;
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error(c, "bg_register_host: cudaHostRegister of %zu bytes: %s", bytes, cudaGetErrorString(e));
      return BG_ECUDA;   // the ranges registered so far stay listed, released as usual
    }
    c->registered.emplace_back(s.first, bytes);
    g_registered[s.first] = bytes;
  }
  return BG_OK;
}

int32_t bg_unregister_host(bg_ctx* c) {
  if (c == nullptr) return BG_EINVAL;
  cudaSetDevice(c->device);
  release_registered(c);
  return BG_OK;
}

int64_t bg_registered_bytes(const bg_ctx* c) {
  if (c == nullptr) return 0;
  int64_t n = 0;
  for (const auto& r : c->registered) n += static_cast<int64_t>(r.second);
  return n;
}

int32_t bg_last_launches(const bg_ctx* c) { return c == nullptr ? 0 : c->last_launches; }

int32_t bg_set_block_threads(bg_ctx* c, int32_t threads) {
  if (c == nullptr) return BG_EINVAL;
  if (threads != 0 && threads != BG_BATCH_ON_GRID && threads != 32 && threads != 64 && threads != 128 && threads != 256) {
    set_error(c, "block threads must be 0 (tune), BG_BATCH_ON_GRID, 32, 64, 128 or 256");
    return BG_EINVAL;
  }
  c->block_threads = threads;
  return BG_OK;
}

int32_t bg_block_threads(const bg_ctx* c) { return c == nullptr ? BG_EINVAL : c->block_threads; }

double bg_last_stage_ms(bg_ctx* c) {
  if (c == nullptr || !c->stage_timed) return -1.0;
  cudaSetDevice(c->device);
  if (cudaEventSynchronize(c->stage_end) != cudaSuccess) return -1.0;
  float ms = 0;
  if (cudaEventElapsedTime(&ms, c->stage_begin, c->stage_end) != cudaSuccess) return -1.0;
  return static_cast<double>(ms);
}

int32_t bg_set_wait_budget(bg_ctx* c, int64_t iterations) {
  if (c == nullptr || iterations < 0) return BG_EINVAL;
  c->budget = iterations == 0 ? kDefaultBudget : iterations;
  return BG_OK;
}

int32_t bg_upload(bg_ctx* c, const bg_bodies* B, const bg_rows* R) {
  if (c == nullptr) return BG_EINVAL;
  cudaSetDevice(c->device);
  int rc = validate(c, B, R);
  if (rc != BG_OK) return rc;
  rc = validate_world(c, B->capacity, R->count, R->starts, R->solved);
  if (rc != BG_OK) return rc;
  c->last_launches = 0;
  c->uploaded = false;   // until this upload has passed every check
  if (!ensure(c, B->capacity, R->count, B->awake_count, 1)) return BG_ENOMEM;
  c->nbodies = B->capacity;
  c->nrows = R->count;
  c->nawake = B->awake_count;
  c->nworlds = 1;
  c->batch = false;
  bg::WorldDesc w = {};
  w.body0 = 0; w.nbodies = B->capacity; w.awake0 = 0; w.nawake = B->awake_count;
  w.row0 = 0; w.nrows = R->count; w.solved = R->solved;
  for (int k = 0; k < bg::NSTARTS; k++) w.starts[k] = R->starts[k];
  w.gravity[0] = 0; w.gravity[1] = 0; w.gravity[2] = 0;
  c->worlds.assign(1, w);
  rc = upload_and_order(c, B, R);
  if (rc != BG_OK) return rc;
  std::vector<int32_t> bo = {0, c->nbodies}, ao = {0, c->nawake}, ro = {0, c->nrows};
  rc = upload_worlds(c, bo, ao, ro);
  if (rc != BG_OK) return rc;
  c->uploaded = true;
  return unpack(c);
}

int32_t bg_restore(bg_ctx* c) {
  if (c == nullptr || !c->uploaded) return BG_EINVAL;
  cudaSetDevice(c->device);
  c->last_launches = 0;
  return unpack(c);
}

int32_t bg_solve(bg_ctx* c, const bg_step* step) {
  if (c == nullptr || !c->uploaded) {
    if (c) set_error(c, "solve: nothing uploaded");
    return BG_EINVAL;
  }
  if (step == nullptr) return BG_EINVAL;
  cudaSetDevice(c->device);
  // The world's gravity is the step's (unless a batch gave each world its own).
  if (!c->batch) {
    for (int k = 0; k < 3; k++) c->worlds[0].gravity[k] = step->gravity[k];
    if (!put(c, c->worlds_dev, c->worlds.data(), 1, "worlds")) return BG_ECUDA;
  }
  int rc = launch_stage(c, step);
  if (rc != BG_OK) return rc;
  return finish(c);
}

int32_t bg_download(bg_ctx* c, const bg_bodies* B, const bg_rows* R) {
  if (c == nullptr || B == nullptr || R == nullptr) return BG_EINVAL;
  cudaSetDevice(c->device);
  return download_columns(c, B, R);
}

int32_t bg_solve_step(bg_ctx* c, const bg_bodies* B, const bg_rows* R, const bg_step* step) {
  int rc = bg_upload(c, B, R);
  if (rc != BG_OK) return rc;
  rc = bg_solve(c, step);
  if (rc != BG_OK) return rc;
  return bg_download(c, B, R);
}

}  // extern "C"

namespace {

// A batch's table of worlds from the caller's offsets, every world checked.
int batch_worlds(bg_ctx* c, const bg_bodies* B, const bg_rows* R, const bg_worlds* W, std::vector<bg::WorldDesc>& worlds) {
  int rc = validate(c, B, R);
  if (rc != BG_OK) return rc;
  if (W == nullptr || W->count < 1 || W->body_offset == nullptr || W->awake_offset == nullptr ||
      W->row_offset == nullptr || W->starts == nullptr) {
    set_error(c, "batch: worlds and their offsets must be given");
    return BG_EINVAL;
  }
  const int nw = W->count;
  if (W->body_offset[0] != 0 || W->awake_offset[0] != 0 || W->row_offset[0] != 0 || W->body_offset[nw] != B->capacity ||
      W->awake_offset[nw] != B->awake_count || W->row_offset[nw] != R->count) {
    set_error(c, "batch: offsets must start at 0 and end at the arrays' lengths");
    return BG_EINVAL;
  }
  worlds.assign(static_cast<size_t>(nw), bg::WorldDesc{});
  for (int i = 0; i < nw; i++) {
    bg::WorldDesc& w = worlds[static_cast<size_t>(i)];
    w.body0 = W->body_offset[i];
    w.nbodies = W->body_offset[i + 1] - W->body_offset[i];
    w.awake0 = W->awake_offset[i];
    w.nawake = W->awake_offset[i + 1] - W->awake_offset[i];
    w.row0 = W->row_offset[i];
    w.nrows = W->row_offset[i + 1] - W->row_offset[i];
    if (w.nbodies < 0 || w.nawake < 0 || w.nrows < 0) {
      set_error(c, "batch: offsets must not decrease");
      return BG_EINVAL;
    }
    for (int k = 0; k < bg::NSTARTS; k++) w.starts[k] = W->starts[bg::NSTARTS * i + k];
    w.solved = w.starts[bg::RESTING_RUN];
    rc = validate_world(c, w.nbodies, w.nrows, w.starts, w.solved);
    if (rc != BG_OK) return rc;
    for (int k = 0; k < 3; k++) w.gravity[k] = W->gravity != nullptr ? W->gravity[3 * i + k] : NAN;
  }
  return BG_OK;
}

}  // namespace

extern "C" {

int32_t bg_batch_upload(bg_ctx* c, const bg_bodies* B, const bg_rows* R, const bg_worlds* W) {
  if (c == nullptr) return BG_EINVAL;
  cudaSetDevice(c->device);
  std::vector<bg::WorldDesc> worlds;
  int rc = batch_worlds(c, B, R, W, worlds);
  if (rc != BG_OK) return rc;
  const int nw = W->count;
  c->last_launches = 0;
  c->uploaded = false;   // until this upload has passed every check
  if (!ensure(c, B->capacity, R->count, B->awake_count, nw)) return BG_ENOMEM;
  c->nbodies = B->capacity;
  c->nrows = R->count;
  c->nawake = B->awake_count;
  c->nworlds = nw;
  c->batch = true;
  c->worlds = worlds;
  rc = upload_and_order(c, B, R);
  if (rc != BG_OK) return rc;
  std::vector<int32_t> bo(W->body_offset, W->body_offset + nw + 1), ao(W->awake_offset, W->awake_offset + nw + 1),
      ro(W->row_offset, W->row_offset + nw + 1);
  rc = upload_worlds(c, bo, ao, ro);
  if (rc != BG_OK) return rc;
  c->uploaded = true;
  return unpack(c);
}

// The batch's CTA size, by measurement: a world's CTA holds 255 registers a thread, so an SM runs
// 8, 4, 2 or 1 worlds at once with 32, 64, 128 or 256 threads each; small worlds leave most of a
// large CTA idle, large ones want the threads.  Each candidate solves the uploaded batch once
// (timed with events), the input is restored from staging after each, and the fastest is kept.
// Results do not depend on the choice.
static int tune_block_threads(bg_ctx* c, const bg_step* step) {
  static const int kCandidates[] = {32, 64, 128, 256, BG_BATCH_ON_GRID};
  float best = 0;
  int chosen = kBlockThreads;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (!cuda_ok(c, cudaEventCreate(&e0), "tune") || !cuda_ok(c, cudaEventCreate(&e1), "tune")) return BG_ECUDA;
  int rc = BG_OK;
  for (int threads : kCandidates) {
    c->block_threads = threads;
    cudaEventRecord(e0, c->stream);
    rc = launch_stage(c, step);
    if (rc != BG_OK) break;
    cudaEventRecord(e1, c->stream);
    float ms = 0;
    if (!cuda_ok(c, cudaEventSynchronize(e1), "tune") || !cuda_ok(c, cudaEventElapsedTime(&ms, e0, e1), "tune")) {
      rc = BG_ECUDA;
      break;
    }
    if (best == 0 || ms < best) {
      best = ms;
      chosen = threads;
    }
    rc = unpack(c);   // back to the uploaded input
    if (rc != BG_OK) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->block_threads = chosen;
  return rc;
}

int32_t bg_batch_solve(bg_ctx* c, const bg_step* step) {
  if (c == nullptr || !c->uploaded || !c->batch) {
    if (c) set_error(c, "batch solve: no batch uploaded");
    return BG_EINVAL;
  }
  if (step == nullptr) return BG_EINVAL;
  cudaSetDevice(c->device);
  bool changed = false;
  for (auto& w : c->worlds)
    if (w.gravity[0] != w.gravity[0]) {
      for (int k = 0; k < 3; k++) w.gravity[k] = step->gravity[k];
      changed = true;
    }
  if (changed) {
    if (!put(c, c->worlds_dev, c->worlds.data(), c->worlds.size(), "worlds")) return BG_ECUDA;
    if (!cuda_ok(c, cudaStreamSynchronize(c->stream), "worlds")) return BG_ECUDA;
  }
  if (c->block_threads == 0) {
    const int trc = tune_block_threads(c, step);
    if (trc != BG_OK) return trc;
  }
  int rc = launch_stage(c, step);
  if (rc != BG_OK) return rc;
  return finish(c);
}

int32_t bg_batch_download(bg_ctx* c, const bg_bodies* B, const bg_rows* R) { return bg_download(c, B, R); }

int32_t bg_set_batch_groups(bg_ctx* c, int32_t groups) {
  if (c == nullptr) return BG_EINVAL;
  if (groups < 0 || groups > BG_MAX_BATCH_GROUPS) {
    set_error(c, "batch groups must be 0 (by the batch's rows) to %d", BG_MAX_BATCH_GROUPS);
    return BG_EINVAL;
  }
  c->batch_groups = groups;
  return BG_OK;
}

}  // extern "C"

namespace {

template <class T>
T* advanced(T* p, size_t k) { return p == nullptr ? nullptr : p + k; }

// Worlds [w0, w1) of a batch: the caller's columns advanced to the group's first slot, awake entry
// and row (slots, awake entries and rows are local to their world, so no value changes), and the
// group's own table of offsets.
struct Group {
  bg_bodies B;
  bg_rows R;
  bg_worlds W;
  std::vector<int32_t> body_offset, awake_offset, row_offset;
};

void make_group(Group& g, const bg_bodies* B, const bg_rows* R, const bg_worlds* W, int w0, int w1) {
  const size_t s = static_cast<size_t>(W->body_offset[w0]), a = static_cast<size_t>(W->awake_offset[w0]),
               r = static_cast<size_t>(W->row_offset[w0]);
  for (int i = w0; i <= w1; i++) {
    g.body_offset.push_back(W->body_offset[i] - static_cast<int32_t>(s));
    g.awake_offset.push_back(W->awake_offset[i] - static_cast<int32_t>(a));
    g.row_offset.push_back(W->row_offset[i] - static_cast<int32_t>(r));
  }
  g.B = *B;
  g.B.capacity = g.body_offset.back();
  g.B.awake_count = g.awake_offset.back();
  g.B.awake_list = advanced(B->awake_list, a);
  g.B.awake = advanced(B->awake, s);
  g.B.position = advanced(B->position, 3 * s);
  g.B.rotation = advanced(B->rotation, 4 * s);
  g.B.velocity = advanced(B->velocity, 3 * s);
  g.B.angular = advanced(B->angular, 3 * s);
  g.B.tumbled = advanced(B->tumbled, 3 * s);
  g.B.ceiling = advanced(B->ceiling, s);
  g.B.start = advanced(B->start, 3 * s);
  g.B.start_q = advanced(B->start_q, 4 * s);
  g.B.inv_i = advanced(B->inv_i, 6 * s);
  g.B.inv_mass = advanced(B->inv_mass, s);
  g.B.inertia = advanced(B->inertia, 3 * s);
  g.B.inv_inertia = advanced(B->inv_inertia, 3 * s);
  g.B.dims = advanced(B->dims, 3 * s);
  g.B.damping = advanced(B->damping, s);
  g.B.angular_damping = advanced(B->angular_damping, s);
  g.B.gravity_scale = advanced(B->gravity_scale, s);
  g.B.type = advanced(B->type, s);
  g.B.shape = advanced(B->shape, s);
  g.B.frozen = advanced(B->frozen, s);
  g.B.framed = advanced(B->framed, s);
  g.B.lock = advanced(B->lock, s);
  g.B.joint_head = advanced(B->joint_head, s);
  g.R = *R;
  g.R.count = g.row_offset.back();
  g.R.row = advanced(R->row, r);
  g.R.a = advanced(R->a, r);
  g.R.b = advanced(R->b, r);
  g.R.points = advanced(R->points, r);
  g.R.normal = advanced(R->normal, 3 * r);
  g.R.t1 = advanced(R->t1, 3 * r);
  g.R.t2 = advanced(R->t2, 3 * r);
  g.R.friction = advanced(R->friction, r);
  g.R.restitution = advanced(R->restitution, r);
  g.R.tolerance = advanced(R->tolerance, r);
  g.R.patch = advanced(R->patch, r);
  g.R.separation = advanced(R->separation, 4 * r);
  g.R.point = advanced(R->point, 12 * r);
  g.R.shift = advanced(R->shift, 12 * r);
  g.R.normal_impulse = advanced(R->normal_impulse, 4 * r);
  g.R.tangent_impulse1 = advanced(R->tangent_impulse1, r);
  g.R.tangent_impulse2 = advanced(R->tangent_impulse2, r);
  g.R.roll_impulse1 = advanced(R->roll_impulse1, r);
  g.R.roll_impulse2 = advanced(R->roll_impulse2, r);
  g.R.spin_impulse = advanced(R->spin_impulse, r);
  g.R.drift1 = advanced(R->drift1, r);
  g.R.drift2 = advanced(R->drift2, r);
  g.R.gap = advanced(R->gap, r);
  g.R.max_normal_impulse = advanced(R->max_normal_impulse, 4 * r);
  g.R.relative_velocity = advanced(R->relative_velocity, 4 * r);
  g.R.sliding = advanced(R->sliding, r);
  g.R.anchor_a = advanced(R->anchor_a, 3 * r);
  g.R.anchor_b = advanced(R->anchor_b, 3 * r);
  g.W.count = w1 - w0;
  g.W.body_offset = g.body_offset.data();
  g.W.awake_offset = g.awake_offset.data();
  g.W.row_offset = g.row_offset.data();
  g.W.starts = W->starts + static_cast<size_t>(bg::NSTARTS) * static_cast<size_t>(w0);
  g.W.gravity = advanced(W->gravity, 3 * static_cast<size_t>(w0));
}

// How many groups bg_batch_solve_step splits a batch into: by its rows unless the caller chose.
int groups_for(const bg_ctx* c, const bg_rows* R, const bg_worlds* W) {
  if (R == nullptr || W == nullptr || W->count < 2) return 1;
  int g = c->batch_groups;
  // Page-locked columns go straight to the device, so more groups overlap more; pageable ones are
  // gathered by host threads, and the groups' gathers and scatters then compete for the host's
  // memory bandwidth (4,096 worlds, 845,037 rows: page-locked 36 ms in one piece, 24 ms in 4-6
  // groups; pageable 42 ms, 35 ms in 2-3 groups, 43 ms in 8).
  if (g == 0) {
    const int64_t per = host_pinned(R->normal, 3 * sizeof(double) * static_cast<size_t>(R->count)) ? kRowsPerGroup : 2 * static_cast<int64_t>(kRowsPerGroup);
    g = static_cast<int>(std::min<int64_t>(BG_MAX_BATCH_GROUPS, R->count / per));
  }
  return std::max(1, std::min(g, W->count));
}

// bg_batch_solve_step in groups of whole worlds, each on a context of its own: group g+1's columns
// are gathered and copied in while group g solves, and group g's results go back (on a thread of
// their own) while later groups solve.  Worlds are independent, so each world's results are the
// ones a single launch gives.  The whole batch is checked first, so a refused batch writes nothing.
int batch_in_groups(bg_ctx* c, const bg_bodies* B, const bg_rows* R, const bg_worlds* W, const bg_step* step, int groups) {
  std::vector<bg::WorldDesc> worlds;
  int rc = batch_worlds(c, B, R, W, worlds);
  if (rc != BG_OK) return rc;
  if (step == nullptr || !(step->dt > 0) || step->substeps < 1) {
    set_error(c, "step: dt must be positive and substeps at least 1");
    return BG_EINVAL;
  }
  {
    // Every world's indices before any group runs, so that a refused batch writes nothing: the
    // pool checks runs of whole worlds (their rows, hence their marks, never overlap).
    std::vector<uint8_t> seen(static_cast<size_t>(R->count), 0);
    HostPool* pool = pool_of(c);
    const int tasks = std::max(1, std::min(static_cast<int>(worlds.size()), 4 * pool->size()));
    std::vector<std::array<char, 256>> why(static_cast<size_t>(tasks));
    std::vector<int> bad(static_cast<size_t>(tasks), 0);
    pool->run(tasks, [&](int t) {
      const size_t n = worlds.size(), lo = n * static_cast<size_t>(t) / static_cast<size_t>(tasks),
                   hi = n * static_cast<size_t>(t + 1) / static_cast<size_t>(tasks);
      char* out = why[static_cast<size_t>(t)].data();
      const char* p = index_problem(B, R, worlds, lo, hi, seen.data(), out, 256);
      if (p != nullptr) {
        if (p != out) snprintf(out, 256, "%s", p);
        bad[static_cast<size_t>(t)] = 1;
      }
    });
    for (int t = 0; t < tasks; t++)
      if (bad[static_cast<size_t>(t)]) {
        set_error(c, "%s", why[static_cast<size_t>(t)].data());
        return BG_EINVAL;
      }
  }
  while (static_cast<int>(c->kids.size()) < groups) {
    bg_ctx* k = bg_create(c->device, c->flags);
    if (k == nullptr) {
      set_error(c, "batch: no context for a group of worlds");
      return BG_ENOMEM;
    }
    c->kids.push_back(k);
  }
  // Whole worlds, split where the running count of rows and slots passes each group's share.
  const int nw = W->count;
  const double total = static_cast<double>(R->count) + static_cast<double>(B->capacity);
  std::vector<int> first(1, 0);
  for (int i = 1; i < nw && static_cast<int>(first.size()) < groups; i++) {
    const double upto = static_cast<double>(W->row_offset[i]) + static_cast<double>(W->body_offset[i]);
    if (upto >= total * static_cast<double>(first.size()) / groups) first.push_back(i);
  }
  first.push_back(nw);
  const int n = static_cast<int>(first.size()) - 1;
  std::vector<Group> part(static_cast<size_t>(n));
  for (int g = 0; g < n; g++) make_group(part[static_cast<size_t>(g)], B, R, W, first[static_cast<size_t>(g)], first[static_cast<size_t>(g) + 1]);
  c->uploaded = false;   // what the context held is not this batch
  c->last_launches = 0;
  std::vector<int> rcs(static_cast<size_t>(n), BG_OK);
  std::vector<std::thread> downloads;
  int failed = -1;
  for (int g = 0; g < n && failed < 0; g++) {
    bg_ctx* k = c->kids[static_cast<size_t>(g)];
    Group& p = part[static_cast<size_t>(g)];
    k->budget = c->budget;
    if (c->block_threads != 0) k->block_threads = c->block_threads;
    int r = BG_ENOMEM;
    try {   // nothing may leave this loop by an exception while download threads run
      r = bg_batch_upload(k, &p.B, &p.R, &p.W);
      if (r == BG_OK) r = bg_batch_solve(k, step);
    } catch (const std::exception&) {
      set_error(k, "out of host memory");
    }
    if (r != BG_OK) {
      rcs[static_cast<size_t>(g)] = r;
      failed = g;
      break;
    }
    try {
      downloads.emplace_back([k, &p, &rcs, g] {
        try {
          rcs[static_cast<size_t>(g)] = bg_batch_download(k, &p.B, &p.R);
        } catch (const std::exception&) {
          rcs[static_cast<size_t>(g)] = BG_ENOMEM;
        }
      });
    } catch (const std::exception&) {   // no thread to be had: this group's results come back now
      rcs[static_cast<size_t>(g)] = bg_batch_download(k, &p.B, &p.R);
    }
  }
  for (std::thread& t : downloads) t.join();
  cudaSetDevice(c->device);
  for (int g = 0; g < n; g++) {
    bg_ctx* k = c->kids[static_cast<size_t>(g)];
    c->last_launches += k->last_launches;
    if (rcs[static_cast<size_t>(g)] != BG_OK && rc == BG_OK) {
      rc = rcs[static_cast<size_t>(g)];
      set_error(c, "batch group %d of %d: %s", g, n, k->error.c_str());
    }
  }
  return rc;
}

}  // namespace

extern "C" {

int32_t bg_batch_solve_step(bg_ctx* c, const bg_bodies* B, const bg_rows* R, const bg_worlds* W, const bg_step* step) {
  if (c == nullptr) return BG_EINVAL;
  cudaSetDevice(c->device);
  const int groups = groups_for(c, R, W);
  if (groups > 1) {
    try {
      return batch_in_groups(c, B, R, W, step, groups);
    } catch (const std::bad_alloc&) {
      set_error(c, "batch: out of host memory");
      return BG_ENOMEM;
    }
  }
  int rc = bg_batch_upload(c, B, R, W);
  if (rc != BG_OK) return rc;
  rc = bg_batch_solve(c, step);
  if (rc != BG_OK) return rc;
  return bg_batch_download(c, B, R);
}

}  // extern "C"

// ---- the adjoint of the solve stage (bg_backward) ------------------------------------------
//
// One warp a world: adjoint_step recomputes the world's step with records (bgadj::forward), then
// sweeps it in reverse (bgadj::reverse), each lane replaying rows and bodies on a tape of its own.

namespace bgad {
// This block's tapes, one a thread, set as each block of the adjoint kernel starts.
__shared__ Tape* s_block_tapes;
#ifdef __CUDA_ARCH__
__device__ Tape* thread_tape() { return s_block_tapes + threadIdx.x; }
#else
// Host code of this library never records (only the kernels do).
Tape* thread_tape() { return nullptr; }
#endif
}  // namespace bgad

namespace {

constexpr int kAdjointThreads = 32;   // one warp a world

struct WarpLane {
  int id, n;
  __device__ void sync() const { __syncwarp(); }
};

__global__ void adjoint_tapes(bgad::Tape* tapes, int threads, int32_t* pa, int32_t* pb, double* da, double* db,
                              double* adj, int cap) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= threads) return;
  const size_t o = static_cast<size_t>(t) * static_cast<size_t>(cap);
  tapes[t] = bgad::Tape{0, cap, pa + o, pb + o, da + o, db + o, adj + o, 0, 0};
}

__global__ void __launch_bounds__(kAdjointThreads) adjoint_step(bgadj::AdjParams A, bgad::Tape* tapes) {
  if (threadIdx.x == 0) bgad::s_block_tapes = tapes + static_cast<size_t>(blockIdx.x) * blockDim.x;
  __syncthreads();
  const WarpLane lane{static_cast<int>(threadIdx.x), static_cast<int>(blockDim.x)};
  for (int wi = blockIdx.x; wi < A.nworlds; wi += gridDim.x) {
    const bgadj::AdjWorld W = A.worlds[wi];
    bgadj::forward(A, W, lane);
    bgadj::reverse(A, W, lane);
  }
}

// The recomputed step's row results and the rows' adjoints, from the kernel's per-row state into
// the caller's layout.
struct AdjRowOut {
  double *ni, *ti1, *ti2, *ri1, *ri2, *si, *gap, *maxni, *relvel, *anchor_a, *anchor_b;
  uint8_t* sliding;
  double *g_ni, *g_ti1, *g_ti2, *g_ri1, *g_ri2, *g_si;
};

__global__ void adjoint_pack(const double* st, const double* bst, const double* pr, AdjRowOut o, int n) {
  using namespace bgadj;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
    const double* x = st + RSTATE * static_cast<int64_t>(m);
    const double* g = bst + RSTATE * static_cast<int64_t>(m);
    const double* q = pr + PREP * static_cast<int64_t>(m);
    for (int k = 0; k < bg::P; k++) {
      o.ni[4 * m + k] = x[RS_NI + k]; o.maxni[4 * m + k] = x[RS_MAXNI + k]; o.relvel[4 * m + k] = x[RS_RELVEL + k];
      o.g_ni[4 * m + k] = g[RS_NI + k];
    }
    o.ti1[m] = x[RS_TI1]; o.ti2[m] = x[RS_TI2]; o.ri1[m] = x[RS_RI1]; o.ri2[m] = x[RS_RI2]; o.si[m] = x[RS_SI];
    o.gap[m] = x[RS_GAP]; o.sliding[m] = static_cast<uint8_t>(x[RS_SLID] != 0);
    o.g_ti1[m] = g[RS_TI1]; o.g_ti2[m] = g[RS_TI2]; o.g_ri1[m] = g[RS_RI1]; o.g_ri2[m] = g[RS_RI2]; o.g_si[m] = g[RS_SI];
    for (int k = 0; k < 3; k++) { o.anchor_a[3 * m + k] = q[PR_ANA + k]; o.anchor_b[3 * m + k] = q[PR_ANB + k]; }
  }
}

// A bump allocator over one device block: each piece starts on a 256-byte boundary.
struct Carve {
  unsigned char* base;
  size_t end = 0;
  template <class T>
  T* take(size_t n) {
    T* at = base == nullptr ? nullptr : reinterpret_cast<T*>(base + end);
    end = (end + (n > 0 ? n : 1) * sizeof(T) + 255) & ~static_cast<size_t>(255);
    return at;
  }
};

// The adjoint kernel's arrays for nb slots, nr rows, na awake entries and nw worlds, carved from
// `in` (the step's input, as the caller's columns) and `work` (state, records and adjoints).
// Returns the two blocks' sizes; with NULL bases it only measures.
struct AdjLayout {
  bgadj::AdjParams A;
  bgadj::AdjWorld* worlds;
  // the step's input and seeds, where the caller's columns are copied to
  double *p, *q, *v, *w, *tum, *ceil, *inv_mass, *inertia, *inv_inertia, *dims, *damping, *ang_damping, *grav_scale;
  uint8_t *type, *shape, *framed, *awake, *points;
  int32_t *awake_list, *row, *a, *b;
  double *normal, *t1, *t2, *friction, *restitution, *tolerance, *patch, *separation, *point, *shift;
  double *ni, *ti1, *ti2, *ri1, *ri2, *si, *drift1, *drift2, *maxni, *relvel, *gap;
  double *seed_ni, *seed_ti1, *seed_ti2, *seed_ri1, *seed_ri2, *seed_si;
  AdjRowOut out;
  size_t in_bytes, work_bytes;
};

AdjLayout adj_layout(unsigned char* in, unsigned char* work, size_t nb, size_t nr, size_t na, size_t nw, int substeps) {
  using namespace bgadj;
  AdjLayout L = {};
  Carve ci{in};
  L.p = ci.take<double>(3 * nb); L.q = ci.take<double>(4 * nb); L.v = ci.take<double>(3 * nb);
  L.w = ci.take<double>(3 * nb); L.tum = ci.take<double>(3 * nb); L.ceil = ci.take<double>(nb);
  L.inv_mass = ci.take<double>(nb); L.inertia = ci.take<double>(3 * nb); L.inv_inertia = ci.take<double>(3 * nb);
  L.dims = ci.take<double>(3 * nb); L.damping = ci.take<double>(nb); L.ang_damping = ci.take<double>(nb);
  L.grav_scale = ci.take<double>(nb); L.type = ci.take<uint8_t>(nb); L.shape = ci.take<uint8_t>(nb);
  L.framed = ci.take<uint8_t>(nb); L.awake = ci.take<uint8_t>(nb); L.awake_list = ci.take<int32_t>(na);
  L.row = ci.take<int32_t>(nr); L.a = ci.take<int32_t>(nr); L.b = ci.take<int32_t>(nr); L.points = ci.take<uint8_t>(nr);
  L.normal = ci.take<double>(3 * nr); L.t1 = ci.take<double>(3 * nr); L.t2 = ci.take<double>(3 * nr);
  L.friction = ci.take<double>(nr); L.restitution = ci.take<double>(nr); L.tolerance = ci.take<double>(nr);
  L.patch = ci.take<double>(nr); L.separation = ci.take<double>(4 * nr); L.point = ci.take<double>(12 * nr);
  L.shift = ci.take<double>(12 * nr); L.ni = ci.take<double>(4 * nr); L.ti1 = ci.take<double>(nr);
  L.ti2 = ci.take<double>(nr); L.ri1 = ci.take<double>(nr); L.ri2 = ci.take<double>(nr); L.si = ci.take<double>(nr);
  L.drift1 = ci.take<double>(nr); L.drift2 = ci.take<double>(nr); L.maxni = ci.take<double>(4 * nr);
  L.relvel = ci.take<double>(4 * nr); L.gap = ci.take<double>(nr);
  L.seed_ni = ci.take<double>(4 * nr); L.seed_ti1 = ci.take<double>(nr); L.seed_ti2 = ci.take<double>(nr);
  L.seed_ri1 = ci.take<double>(nr); L.seed_ri2 = ci.take<double>(nr); L.seed_si = ci.take<double>(nr);
  L.worlds = ci.take<AdjWorld>(nw);
  L.in_bytes = ci.end;
  AdjParams& A = L.A;
  A.in_p = L.p; A.in_q = L.q; A.in_v = L.v; A.in_w = L.w; A.in_tum = L.tum; A.in_ceil = L.ceil;
  A.inv_mass = L.inv_mass; A.inertia = L.inertia; A.inv_inertia = L.inv_inertia; A.dims = L.dims; A.damping = L.damping;
  A.ang_damping = L.ang_damping; A.grav_scale = L.grav_scale; A.type = L.type; A.shape = L.shape; A.framed = L.framed;
  A.awake = L.awake; A.awake_list = L.awake_list; A.row = L.row; A.a = L.a; A.b = L.b; A.points = L.points;
  A.normal = L.normal; A.t1 = L.t1; A.t2 = L.t2; A.friction = L.friction; A.restitution = L.restitution;
  A.tolerance = L.tolerance; A.patch = L.patch; A.separation = L.separation; A.point = L.point; A.shift = L.shift;
  A.in_ni = L.ni; A.in_ti1 = L.ti1; A.in_ti2 = L.ti2; A.in_ri1 = L.ri1; A.in_ri2 = L.ri2; A.in_si = L.si;
  A.in_drift1 = L.drift1; A.in_drift2 = L.drift2; A.in_maxni = L.maxni; A.in_relvel = L.relvel; A.in_gap = L.gap;
  A.seed_ni = L.seed_ni; A.seed_ti1 = L.seed_ti1; A.seed_ti2 = L.seed_ti2; A.seed_ri1 = L.seed_ri1;
  A.seed_ri2 = L.seed_ri2; A.seed_si = L.seed_si;
  A.worlds = L.worlds;
  Carve cw{work};
  A.p = cw.take<double>(3 * nb); A.q = cw.take<double>(4 * nb); A.v = cw.take<double>(3 * nb); A.w = cw.take<double>(3 * nb);
  A.tum = cw.take<double>(3 * nb); A.ceil = cw.take<double>(nb); A.start = cw.take<double>(3 * nb);
  A.startq = cw.take<double>(4 * nb); A.invI = cw.take<double>(6 * nb);
  A.st = cw.take<double>(RSTATE * nr); A.pr = cw.take<double>(PREP * nr);
  A.drift1 = cw.take<double>(nr); A.drift2 = cw.take<double>(nr);
  A.rec_row = cw.take<double>(3 * static_cast<size_t>(substeps) * REC_ROW * nr);
  A.rec_body = cw.take<double>(static_cast<size_t>(substeps) * REC_BODY * nb);
  A.rec_rest = cw.take<double>(REC_REST * nr);
  A.bp = cw.take<double>(3 * nb); A.bq = cw.take<double>(4 * nb); A.bv = cw.take<double>(3 * nb);
  A.bw = cw.take<double>(3 * nb); A.btum = cw.take<double>(3 * nb); A.bceil = cw.take<double>(nb);
  A.bstart = cw.take<double>(3 * nb); A.bstartq = cw.take<double>(4 * nb); A.binvI = cw.take<double>(6 * nb);
  A.bst = cw.take<double>(RSTATE * nr); A.bpr = cw.take<double>(PREP * nr);
  A.bdrift1 = cw.take<double>(nr); A.bdrift2 = cw.take<double>(nr); A.bnormal = cw.take<double>(3 * nr);
  A.bt1 = cw.take<double>(3 * nr); A.bt2 = cw.take<double>(3 * nr); A.bfriction = cw.take<double>(nr);
  A.brestitution = cw.take<double>(nr); A.bseparation = cw.take<double>(4 * nr); A.bpoint = cw.take<double>(12 * nr);
  AdjRowOut& o = L.out;
  o.ni = cw.take<double>(4 * nr); o.ti1 = cw.take<double>(nr); o.ti2 = cw.take<double>(nr); o.ri1 = cw.take<double>(nr);
  o.ri2 = cw.take<double>(nr); o.si = cw.take<double>(nr); o.gap = cw.take<double>(nr); o.maxni = cw.take<double>(4 * nr);
  o.relvel = cw.take<double>(4 * nr); o.anchor_a = cw.take<double>(3 * nr); o.anchor_b = cw.take<double>(3 * nr);
  o.sliding = cw.take<uint8_t>(nr); o.g_ni = cw.take<double>(4 * nr); o.g_ti1 = cw.take<double>(nr);
  o.g_ti2 = cw.take<double>(nr); o.g_ri1 = cw.take<double>(nr); o.g_ri2 = cw.take<double>(nr); o.g_si = cw.take<double>(nr);
  L.work_bytes = cw.end;
  return L;
}

// Grows bg_backward's device memory to hold the given sizes (by doubling, all blocks together).
bool adj_ensure(bg_ctx* c, size_t nb, size_t nr, size_t na, size_t nw, int substeps, size_t threads) {
  bg_ctx::Adjoint& d = c->adj;
  if (d.in != nullptr && nb <= d.bodies && nr <= d.rows && na <= d.awake && nw <= d.worlds && substeps <= d.substeps &&
      threads <= d.threads)
    return true;
  cudaStreamSynchronize(c->stream);
  for (void* p : d.allocs) cudaFree(p);
  d.allocs.clear();
  d.in = nullptr;
  d.bodies = grown(d.bodies, nb); d.rows = grown(d.rows, nr); d.awake = grown(d.awake, na);
  d.worlds = grown(d.worlds, nw); d.threads = std::max(d.threads, threads);
  d.substeps = std::max(d.substeps, substeps);
  const AdjLayout size = adj_layout(nullptr, nullptr, d.bodies, d.rows, d.awake, d.worlds, d.substeps);
  const size_t cap = BG_TAPE_NODES;
  const size_t tape_bytes = d.threads * (sizeof(bgad::Tape) + cap * (2 * sizeof(int32_t) + 3 * sizeof(double)));
  void* in = nullptr;
  void* work = nullptr;
  void* tapes = nullptr;
  void* status = nullptr;
  auto fail = [&](const char* what) {
    set_error(c, "bg_backward: cudaMalloc of %s failed", what);
    for (void* p : {in, work, tapes, status})
      if (p) cudaFree(p);
    d.bodies = d.rows = d.awake = d.worlds = d.threads = 0;
    d.substeps = 0;
    cudaGetLastError();
    return false;
  };
  if (cudaMalloc(&in, size.in_bytes) != cudaSuccess) return fail("the step's input");
  if (cudaMalloc(&work, size.work_bytes) != cudaSuccess) return fail("the records");
  if (cudaMalloc(&tapes, tape_bytes) != cudaSuccess) return fail("the tapes");
  if (cudaMalloc(&status, sizeof(int32_t)) != cudaSuccess) return fail("the status word");
  d.allocs = {in, work, tapes, status};
  d.in = static_cast<unsigned char*>(in);
  d.work = static_cast<unsigned char*>(work);
  d.tapes = static_cast<bgad::Tape*>(tapes);
  d.status = static_cast<int32_t*>(status);
  unsigned char* nodes = static_cast<unsigned char*>(tapes) + ((d.threads * sizeof(bgad::Tape) + 255) & ~size_t{255});
  int32_t* pa = reinterpret_cast<int32_t*>(nodes);
  int32_t* pb = pa + d.threads * cap;
  double* da = reinterpret_cast<double*>(pb + d.threads * cap);
  double* db = da + d.threads * cap;
  double* adj = db + d.threads * cap;
  const int blocks = static_cast<int>((d.threads + 255) / 256);
  adjoint_tapes<<<blocks, 256, 0, c->stream>>>(d.tapes, static_cast<int>(d.threads), pa, pb, da, db, adj, static_cast<int>(cap));
  return cuda_ok(c, cudaGetLastError(), "bg_backward tapes");
}

}  // namespace

extern "C" {

int32_t bg_backward(bg_ctx* c, const bg_bodies* B, const bg_rows* R, const bg_worlds* W, const bg_step* S,
                    const bg_body_grads* bs, const bg_row_grads* rs, bg_body_grads* bg, bg_row_grads* rg) {
  if (c == nullptr) return BG_EINVAL;
  cudaSetDevice(c->device);
  std::vector<bg::WorldDesc> worlds;
  int rc = BG_OK;
  if (W != nullptr) {
    rc = batch_worlds(c, B, R, W, worlds);
  } else {
    rc = validate(c, B, R);
    if (rc == BG_OK) rc = validate_world(c, B->capacity, R->count, R->starts, R->solved);
    if (rc == BG_OK) {
      bg::WorldDesc w = {};
      w.nbodies = B->capacity; w.nawake = B->awake_count; w.nrows = R->count; w.solved = R->solved;
      for (int k = 0; k < bg::NSTARTS; k++) w.starts[k] = R->starts[k];
      worlds.assign(1, w);
    }
  }
  if (rc != BG_OK) return rc;
  if (S == nullptr || !(S->dt > 0) || S->substeps < 1 || bs == nullptr || rs == nullptr || bg == nullptr || rg == nullptr) {
    set_error(c, "bg_backward: step, seeds and results must be given, dt positive, substeps at least 1");
    return BG_EINVAL;
  }
  {
    std::vector<uint8_t> seen(static_cast<size_t>(R->count), 0);
    char why[256];
    const char* bad = index_problem(B, R, worlds, 0, worlds.size(), seen.data(), why, sizeof why);
    if (bad != nullptr) {
      set_error(c, "%s", bad);
      return BG_EINVAL;
    }
  }
  const int nb = B->capacity, nr = R->count, na = B->awake_count, nw = static_cast<int>(worlds.size());
  for (int s = 0; s < nb; s++)
    if ((B->type[s] != BG_DYNAMIC && B->type[s] != BG_STATIC) || B->lock[s] != 0 || B->frozen[s] != 0 ||
        B->joint_head[s] != 0 || B->shape[s] > BG_CAPSULE) {
      set_error(c, "bg_backward: slot %d is kinematic, locked, frozen, jointed or not a box, sphere or capsule", s);
      return BG_EUNSUPPORTED;
    }
  // One warp a world, every world at once up to 16 a streaming multiprocessor (more loop).
  const size_t threads = static_cast<size_t>(std::min(nw, 16 * c->sms)) * kAdjointThreads;
  if (!adj_ensure(c, static_cast<size_t>(nb), static_cast<size_t>(nr), static_cast<size_t>(na), static_cast<size_t>(nw),
                  S->substeps, threads))
    return BG_ENOMEM;
  bg_ctx::Adjoint& d = c->adj;
  AdjLayout L = adj_layout(d.in, d.work, d.bodies, d.rows, d.awake, d.worlds, d.substeps);
  bgadj::AdjParams& A = L.A;
  A.rows_total = nr;
  A.bodies_total = nb;
  A.dt = S->dt;
  A.substeps = S->substeps;
  const bg::Soft soft = make_soft(S->dt / S->substeps);
  A.soft = bgadj::SoftK{soft.biasRate, soft.massScale, soft.impulseScale};
  A.nworlds = nw;
  A.status = d.status;
  std::vector<bgadj::AdjWorld> aw(static_cast<size_t>(nw));
  for (int i = 0; i < nw; i++) {
    const bg::WorldDesc& w = worlds[static_cast<size_t>(i)];
    bgadj::AdjWorld& x = aw[static_cast<size_t>(i)];
    x.body0 = w.body0; x.nbodies = w.nbodies; x.awake0 = w.awake0; x.nawake = w.nawake; x.row0 = w.row0;
    x.nrows = w.nrows; x.solved = w.solved;
    for (int k = 0; k < bg::NSTARTS; k++) x.starts[k] = w.starts[k];
    for (int k = 0; k < 3; k++) x.gravity[k] = W != nullptr && W->gravity != nullptr ? W->gravity[3 * i + k] : S->gravity[k];
  }
  cudaStream_t st = c->stream;
  bool ok = true;
  auto h2d = [&](void* dst, const void* src, size_t bytes, const char* what) {
    if (!ok || bytes == 0) return;
    if (src == nullptr) {
      set_error(c, "bg_backward: %s is NULL", what);
      ok = false;
      return;
    }
    ok = cuda_ok(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st), what);
  };
  const size_t b8 = sizeof(double) * static_cast<size_t>(nb), r8 = sizeof(double) * static_cast<size_t>(nr);
  h2d(L.p, B->position, 3 * b8, "position"); h2d(L.q, B->rotation, 4 * b8, "rotation");
  h2d(L.v, B->velocity, 3 * b8, "velocity"); h2d(L.w, B->angular, 3 * b8, "angular");
  h2d(L.tum, B->tumbled, 3 * b8, "tumbled"); h2d(L.ceil, B->ceiling, b8, "ceiling");
  h2d(L.inv_mass, B->inv_mass, b8, "inv_mass"); h2d(L.inertia, B->inertia, 3 * b8, "inertia");
  h2d(L.inv_inertia, B->inv_inertia, 3 * b8, "inv_inertia"); h2d(L.dims, B->dims, 3 * b8, "dims");
  h2d(L.damping, B->damping, b8, "damping"); h2d(L.ang_damping, B->angular_damping, b8, "angular_damping");
  h2d(L.grav_scale, B->gravity_scale, b8, "gravity_scale"); h2d(L.type, B->type, static_cast<size_t>(nb), "type");
  h2d(L.shape, B->shape, static_cast<size_t>(nb), "shape"); h2d(L.framed, B->framed, static_cast<size_t>(nb), "framed");
  h2d(L.awake, B->awake, static_cast<size_t>(nb), "awake");
  h2d(L.awake_list, B->awake_list, sizeof(int32_t) * static_cast<size_t>(na), "awake_list");
  h2d(L.row, R->row, sizeof(int32_t) * static_cast<size_t>(nr), "row"); h2d(L.a, R->a, sizeof(int32_t) * static_cast<size_t>(nr), "a");
  h2d(L.b, R->b, sizeof(int32_t) * static_cast<size_t>(nr), "b"); h2d(L.points, R->points, static_cast<size_t>(nr), "points");
  h2d(L.normal, R->normal, 3 * r8, "normal"); h2d(L.t1, R->t1, 3 * r8, "t1"); h2d(L.t2, R->t2, 3 * r8, "t2");
  h2d(L.friction, R->friction, r8, "friction"); h2d(L.restitution, R->restitution, r8, "restitution");
  h2d(L.tolerance, R->tolerance, r8, "tolerance"); h2d(L.patch, R->patch, r8, "patch");
  h2d(L.separation, R->separation, 4 * r8, "separation"); h2d(L.point, R->point, 12 * r8, "point");
  h2d(L.shift, R->shift, 12 * r8, "shift"); h2d(L.ni, R->normal_impulse, 4 * r8, "normal_impulse");
  h2d(L.ti1, R->tangent_impulse1, r8, "tangent_impulse1"); h2d(L.ti2, R->tangent_impulse2, r8, "tangent_impulse2");
  h2d(L.ri1, R->roll_impulse1, r8, "roll_impulse1"); h2d(L.ri2, R->roll_impulse2, r8, "roll_impulse2");
  h2d(L.si, R->spin_impulse, r8, "spin_impulse"); h2d(L.drift1, R->drift1, r8, "drift1"); h2d(L.drift2, R->drift2, r8, "drift2");
  h2d(L.maxni, R->max_normal_impulse, 4 * r8, "max_normal_impulse");
  h2d(L.relvel, R->relative_velocity, 4 * r8, "relative_velocity"); h2d(L.gap, R->gap, r8, "gap");
  h2d(A.bp, bs->position, 3 * b8, "seed position"); h2d(A.bq, bs->rotation, 4 * b8, "seed rotation");
  h2d(A.bv, bs->velocity, 3 * b8, "seed velocity"); h2d(A.bw, bs->angular, 3 * b8, "seed angular");
  h2d(A.btum, bs->tumbled, 3 * b8, "seed tumbled"); h2d(A.bceil, bs->ceiling, b8, "seed ceiling");
  h2d(L.seed_ni, rs->normal_impulse, 4 * r8, "seed normal_impulse");
  h2d(L.seed_ti1, rs->tangent_impulse1, r8, "seed tangent_impulse1");
  h2d(L.seed_ti2, rs->tangent_impulse2, r8, "seed tangent_impulse2");
  h2d(L.seed_ri1, rs->roll_impulse1, r8, "seed roll_impulse1"); h2d(L.seed_ri2, rs->roll_impulse2, r8, "seed roll_impulse2");
  h2d(L.seed_si, rs->spin_impulse, r8, "seed spin_impulse");
  h2d(A.bdrift1, rs->drift1, r8, "seed drift1"); h2d(A.bdrift2, rs->drift2, r8, "seed drift2");
  h2d(L.worlds, aw.data(), sizeof(bgadj::AdjWorld) * static_cast<size_t>(nw), "worlds");
  ok = ok && cuda_ok(c, cudaMemsetAsync(d.status, 0, sizeof(int32_t), st), "status");
  if (!ok) {
    cudaStreamSynchronize(st);
    return BG_EINVAL;
  }
  if (d.begin == nullptr) {
    cudaEventCreate(&d.begin);
    cudaEventCreate(&d.end);
  }
  // The bytes the kernel moves by design, its roofline's numerator: each solved row, each pass, its
  // record written by the recompute and read back by its replay, its prepared terms read and their
  // adjoints read and written by the replay, and its state's adjoints read and written; each awake
  // body, each substep, its record both ways and its 16 adjoints read and written.
  {
    int64_t solved = 0, awake = 0;
    for (const bg::WorldDesc& w : worlds) {
      solved += w.solved;
      awake += w.nawake;
    }
    const int64_t passes = 3 * static_cast<int64_t>(S->substeps);
    d.bytes = static_cast<int64_t>(sizeof(double)) *
              (solved * passes * (2 * bgadj::REC_ROW + 3 * bgadj::PREP + 2 * bgadj::RSTATE) +
               awake * S->substeps * (2 * bgadj::REC_BODY + 2 * 16));
  }
  cudaEventRecord(d.begin, st);
  const int blocks = static_cast<int>(threads / kAdjointThreads);
  adjoint_step<<<blocks, kAdjointThreads, 0, st>>>(A, d.tapes);
  if (!cuda_ok(c, cudaGetLastError(), "adjoint_step launch")) return BG_ECUDA;
  cudaEventRecord(d.end, st);
  d.timed = true;
  const int pblocks = std::max(1, std::min(4 * c->sms, (nr + 255) / 256));
  adjoint_pack<<<pblocks, 256, 0, st>>>(A.st, A.bst, A.pr, L.out, nr);
  if (!cuda_ok(c, cudaGetLastError(), "adjoint_pack launch")) return BG_ECUDA;
  auto d2h = [&](void* dst, const void* src, size_t bytes, const char* what) {
    if (!ok || bytes == 0 || dst == nullptr) return;
    ok = cuda_ok(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st), what);
  };
  // the recomputed step's results, as bg_solve_step leaves them
  d2h(B->position, A.p, 3 * b8, "position"); d2h(B->rotation, A.q, 4 * b8, "rotation");
  d2h(B->velocity, A.v, 3 * b8, "velocity"); d2h(B->angular, A.w, 3 * b8, "angular");
  d2h(B->tumbled, A.tum, 3 * b8, "tumbled"); d2h(B->ceiling, A.ceil, b8, "ceiling");
  d2h(R->normal_impulse, L.out.ni, 4 * r8, "normal_impulse"); d2h(R->tangent_impulse1, L.out.ti1, r8, "tangent_impulse1");
  d2h(R->tangent_impulse2, L.out.ti2, r8, "tangent_impulse2"); d2h(R->roll_impulse1, L.out.ri1, r8, "roll_impulse1");
  d2h(R->roll_impulse2, L.out.ri2, r8, "roll_impulse2"); d2h(R->spin_impulse, L.out.si, r8, "spin_impulse");
  d2h(R->drift1, A.drift1, r8, "drift1"); d2h(R->drift2, A.drift2, r8, "drift2"); d2h(R->gap, L.out.gap, r8, "gap");
  d2h(R->max_normal_impulse, L.out.maxni, 4 * r8, "max_normal_impulse");
  d2h(R->relative_velocity, L.out.relvel, 4 * r8, "relative_velocity");
  d2h(R->sliding, L.out.sliding, static_cast<size_t>(nr), "sliding");
  d2h(R->anchor_a, L.out.anchor_a, 3 * r8, "anchor_a"); d2h(R->anchor_b, L.out.anchor_b, 3 * r8, "anchor_b");
  // the adjoints of the step's input
  d2h(bg->position, A.bp, 3 * b8, "grad position"); d2h(bg->rotation, A.bq, 4 * b8, "grad rotation");
  d2h(bg->velocity, A.bv, 3 * b8, "grad velocity"); d2h(bg->angular, A.bw, 3 * b8, "grad angular");
  d2h(bg->tumbled, A.btum, 3 * b8, "grad tumbled"); d2h(bg->ceiling, A.bceil, b8, "grad ceiling");
  d2h(rg->normal_impulse, L.out.g_ni, 4 * r8, "grad normal_impulse");
  d2h(rg->tangent_impulse1, L.out.g_ti1, r8, "grad tangent_impulse1");
  d2h(rg->tangent_impulse2, L.out.g_ti2, r8, "grad tangent_impulse2");
  d2h(rg->roll_impulse1, L.out.g_ri1, r8, "grad roll_impulse1"); d2h(rg->roll_impulse2, L.out.g_ri2, r8, "grad roll_impulse2");
  d2h(rg->spin_impulse, L.out.g_si, r8, "grad spin_impulse");
  d2h(rg->drift1, A.bdrift1, r8, "grad drift1"); d2h(rg->drift2, A.bdrift2, r8, "grad drift2");
  d2h(rg->normal, A.bnormal, 3 * r8, "grad normal"); d2h(rg->t1, A.bt1, 3 * r8, "grad t1"); d2h(rg->t2, A.bt2, 3 * r8, "grad t2");
  d2h(rg->friction, A.bfriction, r8, "grad friction"); d2h(rg->restitution, A.brestitution, r8, "grad restitution");
  d2h(rg->separation, A.bseparation, 4 * r8, "grad separation"); d2h(rg->point, A.bpoint, 12 * r8, "grad point");
  int32_t status = 0;
  std::vector<bgad::Tape> tapes(threads);
  d2h(&status, d.status, sizeof status, "status");
  d2h(tapes.data(), d.tapes, sizeof(bgad::Tape) * threads, "tapes");
  ok = ok && cuda_ok(c, cudaStreamSynchronize(st), "bg_backward");
  if (!ok) return BG_ECUDA;
  d.peak = 0;
  for (const bgad::Tape& t : tapes) d.peak = std::max(d.peak, std::max(t.peak, t.n));
  if (status != 0) {
    set_error(c, "bg_backward: a replay needed more than %d tape nodes", BG_TAPE_NODES);
    return BG_ENOMEM;
  }
  return BG_OK;
}

int32_t bg_backward_tape_peak(const bg_ctx* c) { return c == nullptr ? BG_EINVAL : c->adj.peak; }

int64_t bg_backward_bytes(const bg_ctx* c) { return c == nullptr ? 0 : c->adj.bytes; }

double bg_backward_ms(bg_ctx* c) {
  if (c == nullptr || !c->adj.timed) return -1.0;
  cudaSetDevice(c->device);
  if (cudaEventSynchronize(c->adj.end) != cudaSuccess) return -1.0;
  float ms = 0;
  if (cudaEventElapsedTime(&ms, c->adj.begin, c->adj.end) != cudaSuccess) return -1.0;
  return static_cast<double>(ms);
}

}  // extern "C"

// ---- the solve stage without allocation --------------------------------------------------
//
// bg_solve_step_static: for callers that may not allocate device memory themselves, such as a
// host runtime (a game engine's or a JavaScript embedding's) that owns every device buffer in a
// pool of its own and hands this library only pointers into it, or a per-frame loop that cannot
// take the device-wide synchronisation a cudaMalloc may cause.  Its working memory is one
// file-scope device array, sized for a world of at most BG_STATIC_MAX_BODIES slots and
// BG_STATIC_MAX_ROWS rows, which every GPU that loads this library holds until the process ends.

namespace {

constexpr int kStaticBodies = BG_STATIC_MAX_BODIES;
constexpr int kStaticRows = BG_STATIC_MAX_ROWS;
// Per slot: vw 8, mi 8, pq 8, st 4, sq 4, tc 4, pr 12 doubles, then fl, awake, head, deg, done.
constexpr size_t kStaticBodyDoubles = 48;
// Per row, doubles: n 3, t1 3, t2 3, friction, restitution, tolerance, patch, separation 4,
// point 12, shift 12, ni 4, ti1, ti2, ri1, ri2, si, drift1, drift2, gap, maxni 4, relvel 4,
// anchorA 3, anchorB 3, la 12, lb 12, adjusted 4, now 4, normalMass 4, lever 4, jac 48, K 16,
// fjac 24, tm 3, rm1, rm2, sm; then ints a, b, row, active, pending, rank_a, rank_b; bytes
// points, sliding.
constexpr size_t kStaticRowDoubles = 3 + 3 + 3 + 4 + 4 + 12 + 12 + 4 + 7 + 1 + 4 + 4 + 3 + 3 + 12 + 12 + 4 + 4 + 4 + 4 + 48 +
                                     16 + 24 + 3 + 3;
constexpr size_t kStaticBytes =
    256 + kStaticBodies * (kStaticBodyDoubles * 8 + 5 * 4) + kStaticRows * (kStaticRowDoubles * 8 + 7 * 4 + 2) + 4096;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

// The status word's value when the kernel refused the caller's indices (1 is a wait past its budget).
constexpr int32_t kStaticRefused = 2;

// The scratch array's device address, per device: set up by the first call on that device.
void* g_static_addr[64] = {};
std::mutex g_static_mutex;

struct StaticIn {
  bg_bodies B;
  bg_rows R;
};

__global__ void __launch_bounds__(kBlockThreads) stage_static(StaticIn in, unsigned char* base, double dt, int substeps,
                                                               bg::Soft soft, double gx, double gy, double gz) {
  const bg_bodies& Bi = in.B;
  const bg_rows& Ri = in.R;
  const int nb = Bi.capacity, nr = Ri.count, na = Bi.awake_count;
  const int64_t cap = kStaticRows;
  // Carve the scratch array: status word first, then the bodies' records, then the rows' columns.
  int32_t* status = reinterpret_cast<int32_t*>(base);
  double* d = reinterpret_cast<double*>(base + 256);
  bg::BodiesDev B;
  B.vw = d; d += 8 * kStaticBodies;
  B.mi = d; d += 8 * kStaticBodies;
  B.pq = d; d += 8 * kStaticBodies;
  B.st = d; d += 4 * kStaticBodies;
  B.sq = d; d += 4 * kStaticBodies;
  B.tc = d; d += 4 * kStaticBodies;
  B.pr = d; d += 12 * kStaticBodies;
  bg::RowsDev R;
  R.cap = cap;
  R.n = d; d += 3 * cap; R.t1 = d; d += 3 * cap; R.t2 = d; d += 3 * cap;
  R.friction = d; d += cap; R.restitution = d; d += cap; R.tolerance = d; d += cap; R.patch = d; d += cap;
  R.separation = d; d += 4 * cap; R.point = d; d += 12 * cap; R.shift = d; d += 12 * cap; R.ni = d; d += 4 * cap;
  R.ti1 = d; d += cap; R.ti2 = d; d += cap; R.ri1 = d; d += cap; R.ri2 = d; d += cap; R.si = d; d += cap;
  R.drift1 = d; d += cap; R.drift2 = d; d += cap; R.gap = d; d += cap; R.maxni = d; d += 4 * cap; R.relvel = d; d += 4 * cap;
  R.anchorA = d; d += 3 * cap; R.anchorB = d; d += 3 * cap; R.la = d; d += 12 * cap; R.lb = d; d += 12 * cap;
  R.adjusted = d; d += 4 * cap; R.now = d; d += 4 * cap; R.normalMass = d; d += 4 * cap; R.lever = d; d += 4 * cap;
  R.jac = d; d += 48 * cap; R.K = d; d += 16 * cap; R.fjac = d; d += 24 * cap; R.tm = d; d += 3 * cap;
  R.rm1 = d; d += cap; R.rm2 = d; d += cap; R.sm = d; d += cap;
  int32_t* q = reinterpret_cast<int32_t*>(d);
  B.fl = reinterpret_cast<uint32_t*>(q); q += kStaticBodies;
  B.awake_list = q; q += kStaticBodies;
  B.head = q; q += kStaticBodies;
  B.deg = q; q += kStaticBodies;
  B.done = reinterpret_cast<unsigned int*>(q); q += kStaticBodies;
  R.a = q; q += cap; R.b = q; q += cap; R.row = q; q += cap; R.active = q; q += cap; R.pending = q; q += cap;
  R.rank_a = q; q += cap; R.rank_b = q; q += cap;
  uint8_t* u = reinterpret_cast<uint8_t*>(q);
  R.points = u; u += cap;
  R.sliding = u; u += cap;
  // The caller's indices first, before anything is written (they are in device memory, which the
  // host side cannot read): each row's a and b among the slots, its point count 1..P, row[] a
  // permutation of the rows (no entry out of range, none twice), each awake entry among the slots.
  __shared__ uint32_t seen[kStaticRows / 32];
  __shared__ int refused;
  if (threadIdx.x == 0) refused = 0;
  for (int i = threadIdx.x; i < kStaticRows / 32; i += blockDim.x) seen[i] = 0;
  __syncthreads();
  for (int m = threadIdx.x; m < nr; m += blockDim.x) {
    const int32_t a = Ri.a[m], b = Ri.b[m], x = Ri.row[m];
    const int pc = Ri.points[m];
    bool bad = static_cast<uint32_t>(a) >= static_cast<uint32_t>(nb) || static_cast<uint32_t>(b) >= static_cast<uint32_t>(nb) ||
               pc < 1 || pc > bg::P || static_cast<uint32_t>(x) >= static_cast<uint32_t>(nr);
    if (!bad) {
      const uint32_t bit = 1u << (x & 31);
      if (atomicOr(&seen[x >> 5], bit) & bit) bad = true;
    }
    if (bad) atomicExch(&refused, 1);
  }
  for (int i = threadIdx.x; i < na; i += blockDim.x)
    if (static_cast<uint32_t>(Bi.awake_list[i]) >= static_cast<uint32_t>(nb)) atomicExch(&refused, 1);
  __syncthreads();
  if (refused) {
    if (threadIdx.x == 0) *status = kStaticRefused;
    return;
  }
  if (threadIdx.x == 0) *status = 0;
  // The caller's layout in: what every call must set afresh, since the array keeps the last
  // call's contents (the records' pad entries included, as unpack_bodies leaves them).
  for (int s = threadIdx.x; s < nb; s += blockDim.x) {
    for (int k = 0; k < 3; k++) {
      B.vw[8 * s + k] = Bi.velocity[3 * s + k];
      B.vw[8 * s + 3 + k] = Bi.angular[3 * s + k];
      B.pq[8 * s + k] = Bi.position[3 * s + k];
      B.st[4 * s + k] = Bi.start[3 * s + k];
      B.tc[4 * s + k] = Bi.tumbled[3 * s + k];
      B.pr[12 * s + k] = Bi.inertia[3 * s + k];
      B.pr[12 * s + 3 + k] = Bi.inv_inertia[3 * s + k];
      B.pr[12 * s + 6 + k] = Bi.dims[3 * s + k];
    }
    B.vw[8 * s + 6] = 0; B.vw[8 * s + 7] = 0;
    B.pq[8 * s + 3] = 0;
    B.st[4 * s + 3] = 0;
    for (int k = 0; k < 4; k++) { B.pq[8 * s + 4 + k] = Bi.rotation[4 * s + k]; B.sq[4 * s + k] = Bi.start_q[4 * s + k]; }
    B.tc[4 * s + 3] = Bi.ceiling[s];
    B.pr[12 * s + 9] = Bi.damping[s];
    B.pr[12 * s + 10] = Bi.angular_damping[s];
    B.pr[12 * s + 11] = Bi.gravity_scale[s];
    B.mi[8 * s] = Bi.inv_mass[s];
    for (int k = 0; k < 6; k++) B.mi[8 * s + 1 + k] = Bi.inv_i[6 * s + k];
    B.mi[8 * s + 7] = 0;
    uint32_t f = static_cast<uint32_t>(Bi.type[s]) & bg::F_TYPE;
    f |= (static_cast<uint32_t>(Bi.shape[s]) & 3u) << bg::F_SHAPE_SHIFT;
    if (Bi.frozen[s]) f |= bg::F_FROZEN;
    if (Bi.framed[s]) f |= bg::F_FRAMED;
    f |= (static_cast<uint32_t>(Bi.lock[s]) & 7u) << bg::F_LOCK_SHIFT;
    if (Bi.joint_head[s] != 0) f |= bg::F_JOINTED;
    if (Bi.awake[s]) f |= bg::F_AWAKE;
    B.fl[s] = f;
    B.head[s] = 0x7fffffff;
  }
  for (int i = threadIdx.x; i < na; i += blockDim.x) B.awake_list[i] = Bi.awake_list[i];
  for (int m = threadIdx.x; m < nr; m += blockDim.x) {
    R.row[m] = Ri.row[m];
    R.a[m] = Ri.a[m];
    R.b[m] = Ri.b[m];
    R.points[m] = Ri.points[m];
    for (int c = 0; c < 3; c++) {
      R.n[c * cap + m] = Ri.normal[3 * m + c];
      R.t1[c * cap + m] = Ri.t1[3 * m + c];
      R.t2[c * cap + m] = Ri.t2[3 * m + c];
      R.anchorA[c * cap + m] = 0;
      R.anchorB[c * cap + m] = 0;
    }
    R.friction[m] = Ri.friction[m];
    R.restitution[m] = Ri.restitution[m];
    R.tolerance[m] = Ri.tolerance[m];
    R.patch[m] = Ri.patch[m];
    R.gap[m] = Ri.gap[m];
    R.sliding[m] = 0;
    for (int k = 0; k < bg::P; k++) {
      R.maxni[k * cap + m] = Ri.max_normal_impulse[bg::P * m + k];
      R.relvel[k * cap + m] = Ri.relative_velocity[bg::P * m + k];
      R.separation[k * cap + m] = Ri.separation[bg::P * m + k];
      R.ni[k * cap + m] = Ri.normal_impulse[bg::P * m + k];
      for (int c = 0; c < 3; c++) {
        R.point[(k * 3 + c) * cap + m] = Ri.point[12 * m + 3 * k + c];
        R.shift[(k * 3 + c) * cap + m] = Ri.shift[12 * m + 3 * k + c];
      }
    }
    R.ti1[m] = Ri.tangent_impulse1[m]; R.ti2[m] = Ri.tangent_impulse2[m];
    R.ri1[m] = Ri.roll_impulse1[m]; R.ri2[m] = Ri.roll_impulse2[m];
    R.si[m] = Ri.spin_impulse[m]; R.drift1[m] = Ri.drift1[m]; R.drift2[m] = Ri.drift2[m];
  }
  __syncthreads();
  bg::WorldDesc w = {};
  w.nbodies = nb;
  w.nawake = na;
  w.nrows = nr;
  w.solved = Ri.solved;
  for (int k = 0; k < bg::NSTARTS; k++) w.starts[k] = Ri.starts[k];
  w.gravity[0] = gx; w.gravity[1] = gy; w.gravity[2] = gz;
  bg::StageParams p = {};
  p.B = B;
  p.R = R;
  p.worlds = nullptr;
  p.nworlds = 1;
  p.dt = dt;
  p.substeps = substeps;
  p.soft = soft;
  p.status = status;
  p.budget = kDefaultBudget;
  p.chunks = nullptr;
  p.nchunks = 0;
  bg::BlockTeam t;
  bg::solve_stage(p, w, t);
  __syncthreads();
  // The written columns back into the caller's arrays.
  for (int s = threadIdx.x; s < nb; s += blockDim.x) {
    for (int k = 0; k < 3; k++) {
      Bi.velocity[3 * s + k] = B.vw[8 * s + k];
      Bi.angular[3 * s + k] = B.vw[8 * s + 3 + k];
      Bi.position[3 * s + k] = B.pq[8 * s + k];
      Bi.start[3 * s + k] = B.st[4 * s + k];
      Bi.tumbled[3 * s + k] = B.tc[4 * s + k];
    }
    for (int k = 0; k < 4; k++) { Bi.rotation[4 * s + k] = B.pq[8 * s + 4 + k]; Bi.start_q[4 * s + k] = B.sq[4 * s + k]; }
    Bi.ceiling[s] = B.tc[4 * s + 3];
    for (int k = 0; k < 6; k++) Bi.inv_i[6 * s + k] = B.mi[8 * s + 1 + k];
  }
  for (int m = threadIdx.x; m < nr; m += blockDim.x) {
    for (int k = 0; k < bg::P; k++) {
      Ri.normal_impulse[bg::P * m + k] = R.ni[k * cap + m];
      Ri.max_normal_impulse[bg::P * m + k] = R.maxni[k * cap + m];
      Ri.relative_velocity[bg::P * m + k] = R.relvel[k * cap + m];
    }
    Ri.tangent_impulse1[m] = R.ti1[m]; Ri.tangent_impulse2[m] = R.ti2[m];
    Ri.roll_impulse1[m] = R.ri1[m]; Ri.roll_impulse2[m] = R.ri2[m];
    Ri.spin_impulse[m] = R.si[m]; Ri.drift1[m] = R.drift1[m]; Ri.drift2[m] = R.drift2[m];
    Ri.gap[m] = R.gap[m];
    Ri.sliding[m] = R.sliding[m];
    for (int c = 0; c < 3; c++) {
      if (Ri.anchor_a) Ri.anchor_a[3 * m + c] = R.anchorA[c * cap + m];
      if (Ri.anchor_b) Ri.anchor_b[3 * m + c] = R.anchorB[c * cap + m];
    }
  }
}

// Whether every column the static stage reads or writes is given (anchor_a / anchor_b may be NULL).
bool static_columns_given(const bg_bodies* B, const bg_rows* R) {
  const bool bodies = B->capacity == 0 ||
      (B->awake != nullptr && B->position != nullptr && B->rotation != nullptr && B->velocity != nullptr &&
       B->angular != nullptr && B->tumbled != nullptr && B->ceiling != nullptr && B->start != nullptr &&
       B->start_q != nullptr && B->inv_i != nullptr && B->inv_mass != nullptr && B->inertia != nullptr &&
       B->inv_inertia != nullptr && B->dims != nullptr && B->damping != nullptr && B->angular_damping != nullptr &&
       B->gravity_scale != nullptr && B->type != nullptr && B->shape != nullptr && B->frozen != nullptr &&
       B->framed != nullptr && B->lock != nullptr && B->joint_head != nullptr);
  const bool awake = B->awake_count == 0 || B->awake_list != nullptr;
  const bool rows = R->count == 0 ||
      (R->row != nullptr && R->a != nullptr && R->b != nullptr && R->points != nullptr && R->normal != nullptr &&
       R->t1 != nullptr && R->t2 != nullptr && R->friction != nullptr && R->restitution != nullptr &&
       R->tolerance != nullptr && R->patch != nullptr && R->separation != nullptr && R->point != nullptr &&
       R->shift != nullptr && R->normal_impulse != nullptr && R->tangent_impulse1 != nullptr &&
       R->tangent_impulse2 != nullptr && R->roll_impulse1 != nullptr && R->roll_impulse2 != nullptr &&
       R->spin_impulse != nullptr && R->drift1 != nullptr && R->drift2 != nullptr && R->gap != nullptr &&
       R->max_normal_impulse != nullptr && R->relative_velocity != nullptr && R->sliding != nullptr);
  return bodies && awake && rows;
}

}  // namespace

extern "C" int32_t bg_solve_step_static(const bg_bodies* bodies, const bg_rows* rows, const bg_step* step, void* stream) {
  if (bodies == nullptr || rows == nullptr || step == nullptr) return BG_EINVAL;
  // The same checks bg_solve_step makes of the counts and colour starts; the index columns are
  // device memory, so the kernel checks those before it writes anything.
  if (bodies->capacity < 0 || bodies->capacity > BG_STATIC_MAX_BODIES || bodies->awake_count < 0 ||
      bodies->awake_count > bodies->capacity || rows->count < 0 || rows->count > BG_STATIC_MAX_ROWS ||
      rows->solved < 0 || starts_problem(rows->count, rows->starts, rows->solved) != nullptr ||
      !static_columns_given(bodies, rows) || !(step->dt > 0) || step->substeps < 1)
    return BG_EINVAL;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) return BG_ECUDA;
  void* base = nullptr;
  {
    // First call on this device: the array's device address, looked up with the device current.
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if (g_static_addr[device] == nullptr) {
      void* ptr = nullptr;
      if (cudaGetSymbolAddress(&ptr, g_static_scratch) != cudaSuccess || ptr == nullptr) return BG_ECUDA;
      g_static_addr[device] = ptr;
    }
    base = g_static_addr[device];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  StaticIn in{*bodies, *rows};
  stage_static<<<1, kBlockThreads, 0, s>>>(in, static_cast<unsigned char*>(base), step->dt, step->substeps,
                                           make_soft(step->dt / step->substeps), step->gravity[0], step->gravity[1],
                                           step->gravity[2]);
  if (cudaGetLastError() != cudaSuccess) return BG_ECUDA;
  int32_t status = 0;
  if (cudaMemcpyAsync(&status, base, sizeof status, cudaMemcpyDeviceToHost, s) != cudaSuccess) return BG_ECUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return BG_ECUDA;
  return status == 0 ? BG_OK : status == kStaticRefused ? BG_EINVAL : BG_ETIMEOUT;
}

// ---- the narrowphase on the device (bg_collide) -------------------------------------------
//
// One thread a pair, running the same narrowphase source the host side of the step runs
// (host/collide_impl.hpp, the reference's src/collide.js restated, compiled here for sm_100a with
// -fmad=false, so the manifolds match the host's bit for bit).  The pairs are first put in order of
// their two shapes' kinds (a counting sort on the device), so each warp runs one of the six pair
// functions: box-box's face clipping, capsule-box's and the rest diverge only where their own
// branches do.

namespace {

constexpr int kCollideThreads = 128;
constexpr int kPairClasses = 6;   // sphere-sphere, sphere-capsule, sphere-box, capsule-capsule, capsule-box, box-box

struct CollideParams {
  const double *p, *q, *dims, *gscale;
  const uint8_t *shape, *type;
  const int32_t *a, *b;
  const double *margin, *tol;
  int32_t n;
  double gravity[3];
  int32_t* counts;   // kPairClasses pairs per class, then kPairClasses cursors
  int32_t* order;    // pairs in class order
  const uint8_t* skip;   // per pair, or NULL: 1 for a pair whose manifold is already known
  uint8_t* points;
  double *normal, *point, *separation;
  uint32_t* pid;
};

__device__ __forceinline__ int kind_of(uint8_t shape) {
  return shape == BG_SPHERE ? bearing::K_SPHERE : shape == BG_CAPSULE ? bearing::K_CAPSULE : bearing::K_BOX;
}

// The pair's class: its two kinds, lower first, as collide() dispatches them (src/collide.js:225-242).
__device__ __forceinline__ int pair_class(const CollideParams& c, int i) {
  int x = kind_of(c.shape[c.a[i]]), y = kind_of(c.shape[c.b[i]]);
  if (x > y) { const int t = x; x = y; y = t; }
  return x == 0 ? y : x == 1 ? 2 + y : 5;
}

__global__ void collide_count(CollideParams c) {
  __shared__ int local[kPairClasses];
  if (threadIdx.x < kPairClasses) local[threadIdx.x] = 0;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < c.n; i += gridDim.x * blockDim.x)
    if (c.skip == nullptr || c.skip[i] == 0) atomicAdd(&local[pair_class(c, i)], 1);
  __syncthreads();
  if (threadIdx.x < kPairClasses && local[threadIdx.x] > 0) atomicAdd(&c.counts[threadIdx.x], local[threadIdx.x]);
}

// Each class's first place in `order` (the cursors the scatter moves on).
__global__ void collide_starts(CollideParams c) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int at = 0;
  for (int k = 0; k < kPairClasses; k++) {
    c.counts[kPairClasses + k] = at;
    at += c.counts[k];
  }
}

// Each block places a chunk of pairs at a time: a place in the block's share of each class from a
// shared-memory count, and one global add per class a block for the share itself (the order
// within a class changes no manifold: each pair's is its own).
__global__ void collide_scatter(CollideParams c) {
  __shared__ int local[kPairClasses], base[kPairClasses];
  for (int i0 = blockIdx.x * blockDim.x; i0 < c.n; i0 += gridDim.x * blockDim.x) {
    if (threadIdx.x < kPairClasses) local[threadIdx.x] = 0;
    __syncthreads();
    const int i = i0 + threadIdx.x;
    int cls = -1, at = 0;
    if (i < c.n && (c.skip == nullptr || c.skip[i] == 0)) {
      cls = pair_class(c, i);
      at = atomicAdd(&local[cls], 1);
    }
    __syncthreads();
    if (threadIdx.x < kPairClasses)
      base[threadIdx.x] = local[threadIdx.x] > 0 ? atomicAdd(&c.counts[kPairClasses + threadIdx.x], local[threadIdx.x]) : 0;
    __syncthreads();
    if (cls >= 0) c.order[base[cls] + at] = i;
    __syncthreads();
  }
}

// load(): src/contact.js:1244-1276, for boxes, spheres and capsules, with the axes of
// src/core/math.js:222-227.
__device__ void load_shape(const CollideParams& c, int slot, bearing::Shape& s) {
  const double* d = c.dims + 3 * slot;
  const uint8_t shape = c.shape[slot];
  if (shape == BG_SPHERE) {
    s.kind = bearing::K_SPHERE;
    s.half[0] = d[0]; s.half[1] = 0; s.half[2] = 0;
  } else if (shape == BG_CAPSULE) {
    s.kind = bearing::K_CAPSULE;
    s.half[0] = d[0]; s.half[1] = (d[1] - 2 * d[0]) * 0.5; s.half[2] = 0;
  } else {
    s.kind = bearing::K_BOX;
    s.half[0] = d[0] * 0.5; s.half[1] = d[1] * 0.5; s.half[2] = d[2] * 0.5;
  }
  for (int k = 0; k < 3; k++) s.center[k] = c.p[3 * slot + k];
  const double scale = c.type[slot] == BG_DYNAMIC ? c.gscale[slot] : 0;
  for (int k = 0; k < 3; k++) s.weight[k] = c.gravity[k] * scale;
  const double* q = c.q + 4 * slot;
  const double x = q[0], y = q[1], z = q[2], w = q[3];
  double* ax = s.axes;
  ax[0] = 1 - 2 * (y * y + z * z); ax[1] = 2 * (x * y + z * w); ax[2] = 2 * (x * z - y * w);
  ax[3] = 2 * (x * y - z * w); ax[4] = 1 - 2 * (x * x + z * z); ax[5] = 2 * (y * z + x * w);
  ax[6] = 2 * (x * z + y * w); ax[7] = 2 * (y * z - x * w); ax[8] = 1 - 2 * (x * x + y * y);
}

__global__ void __launch_bounds__(kCollideThreads) collide_pairs(CollideParams c) {
  int n = c.n;   // the pairs sorted into `order`: all of them, or those not skipped
  if (c.skip != nullptr) {
    n = 0;
    for (int k = 0; k < kPairClasses; k++) n += c.counts[k];
  }
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int i = c.order[j];
    bearing::Shape sa, sb;
    bearing::Manifold mf;
    load_shape(c, c.a[i], sa);
    load_shape(c, c.b[i], sb);
    const int count = bearing::collideT<double>(sa, sb, c.margin[i], c.tol[i], mf);
    c.points[i] = static_cast<uint8_t>(count);
    for (int k = 0; k < 3; k++) c.normal[3 * i + k] = count > 0 ? mf.normal[k] : 0.0;
    for (int k = 0; k < bg::P; k++) {
      const bool used = k < count;
      for (int e = 0; e < 3; e++) c.point[3 * (bg::P * i + k) + e] = used ? mf.points[3 * k + e] : 0.0;
      c.separation[bg::P * i + k] = used ? mf.separations[k] : 0.0;
      c.pid[bg::P * i + k] = used ? mf.ids[k] : 0u;
    }
  }
}

// bg_collide's arrays for nb slots and np pairs, carved from `base` (NULL: only measures).
struct CollideLayout {
  double *p, *q, *dims, *gscale;
  uint8_t *shape, *type;
  int32_t *a, *b, *counts, *order;
  double *margin, *tol;
  uint8_t* points;
  double *normal, *point, *separation;
  uint32_t* pid;
  size_t bytes;
};

CollideLayout collide_layout(unsigned char* base, size_t nb, size_t np) {
  Carve k{base};
  CollideLayout L;
  L.p = k.take<double>(3 * nb); L.q = k.take<double>(4 * nb); L.dims = k.take<double>(3 * nb);
  L.gscale = k.take<double>(nb); L.shape = k.take<uint8_t>(nb); L.type = k.take<uint8_t>(nb);
  L.a = k.take<int32_t>(np); L.b = k.take<int32_t>(np); L.margin = k.take<double>(np); L.tol = k.take<double>(np);
  L.counts = k.take<int32_t>(2 * kPairClasses); L.order = k.take<int32_t>(np);
  L.points = k.take<uint8_t>(np); L.normal = k.take<double>(3 * np); L.point = k.take<double>(3 * bg::P * np);
  L.separation = k.take<double>(bg::P * np); L.pid = k.take<uint32_t>(bg::P * np);
  L.bytes = k.end;
  return L;
}

}  // namespace

extern "C" {

int32_t bg_collide(bg_ctx* c, const bg_bodies* B, const double* gravity, const bg_pairs* P, bg_manifolds* out) {
  if (c == nullptr) return BG_EINVAL;
  if (B == nullptr || gravity == nullptr || P == nullptr || out == nullptr) {
    set_error(c, "bg_collide: bodies, gravity, pairs or out is NULL");
    return BG_EINVAL;
  }
  const int64_t nb = B->capacity, np = P->count;
  if (nb < 0 || np < 0) {
    set_error(c, "bg_collide: capacity %d, pairs %d", B->capacity, P->count);
    return BG_EINVAL;
  }
  if (np == 0) return BG_OK;
  if (P->a == nullptr || P->b == nullptr || P->margin == nullptr || P->tolerance == nullptr || out->points == nullptr ||
      out->normal == nullptr || out->point == nullptr || out->separation == nullptr || out->pid == nullptr ||
      B->position == nullptr || B->rotation == nullptr || B->dims == nullptr || B->shape == nullptr ||
      B->type == nullptr || B->gravity_scale == nullptr) {
    set_error(c, "bg_collide: a column is NULL");
    return BG_EINVAL;
  }
  // every index is checked before anything is copied: a pair's slots among the bodies', and the
  // shapes it reads boxes, spheres or capsules
  for (int64_t i = 0; i < np; i++) {
    const int32_t a = P->a[i], b = P->b[i];
    if (a < 0 || a >= nb || b < 0 || b >= nb) {
      set_error(c, "bg_collide: pair %lld has slots %d, %d of %lld", static_cast<long long>(i), a, b,
                static_cast<long long>(nb));
      return BG_EINVAL;
    }
    for (const int32_t s : {a, b})
      if (B->shape[s] != BG_BOX && B->shape[s] != BG_SPHERE && B->shape[s] != BG_CAPSULE) {
        set_error(c, "bg_collide: slot %d is not a box, sphere or capsule", s);
        return BG_EUNSUPPORTED;
      }
  }
  cudaSetDevice(c->device);
  bg_ctx::Narrow& d = c->nw;
  if (d.block == nullptr || static_cast<size_t>(nb) > d.bodies || static_cast<size_t>(np) > d.pairs) {
    cudaStreamSynchronize(c->stream);
    if (d.block) cudaFree(d.block);
    d.block = nullptr;
    d.bodies = grown(d.bodies, static_cast<size_t>(nb));
    d.pairs = grown(d.pairs, static_cast<size_t>(np));
    void* block = nullptr;
    if (cudaMalloc(&block, collide_layout(nullptr, d.bodies, d.pairs).bytes) != cudaSuccess) {
      cudaGetLastError();
      d.bodies = d.pairs = 0;
      set_error(c, "bg_collide: cudaMalloc failed");
      return BG_ENOMEM;
    }
    d.block = static_cast<unsigned char*>(block);
  }
  if (d.begin == nullptr) {
    cudaEventCreate(&d.begin);
    cudaEventCreate(&d.end);
  }
  const CollideLayout L = collide_layout(d.block, d.bodies, d.pairs);
  const size_t b8 = static_cast<size_t>(nb) * sizeof(double), p8 = static_cast<size_t>(np) * sizeof(double);
  const size_t p4 = static_cast<size_t>(np) * sizeof(int32_t);
  cudaStream_t st = c->stream;
  bool ok = true;
  auto h2d = [&](void* dst, const void* src, size_t bytes) {
    ok = ok && cuda_ok(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st), "bg_collide upload");
  };
  h2d(L.p, B->position, 3 * b8); h2d(L.q, B->rotation, 4 * b8); h2d(L.dims, B->dims, 3 * b8);
  h2d(L.gscale, B->gravity_scale, b8); h2d(L.shape, B->shape, static_cast<size_t>(nb)); h2d(L.type, B->type, static_cast<size_t>(nb));
  h2d(L.a, P->a, p4); h2d(L.b, P->b, p4); h2d(L.margin, P->margin, p8); h2d(L.tol, P->tolerance, p8);
  ok = ok && cuda_ok(c, cudaMemsetAsync(L.counts, 0, 2 * kPairClasses * sizeof(int32_t), st), "bg_collide");
  if (!ok) return BG_ECUDA;
  CollideParams k;
  k.p = L.p; k.q = L.q; k.dims = L.dims; k.gscale = L.gscale; k.shape = L.shape; k.type = L.type;
  k.a = L.a; k.b = L.b; k.margin = L.margin; k.tol = L.tol; k.n = static_cast<int32_t>(np);
  for (int e = 0; e < 3; e++) k.gravity[e] = gravity[e];
  k.counts = L.counts; k.order = L.order; k.points = L.points; k.normal = L.normal; k.point = L.point;
  k.separation = L.separation; k.pid = L.pid; k.skip = nullptr;
  const int sweep = std::max(1, std::min(static_cast<int>((np + 255) / 256), 4 * c->sms));
  collide_count<<<sweep, 256, 0, st>>>(k);
  collide_starts<<<1, 32, 0, st>>>(k);
  collide_scatter<<<sweep, 256, 0, st>>>(k);
  const int blocks = static_cast<int>(std::min<int64_t>((np + kCollideThreads - 1) / kCollideThreads, 64 * c->sms));
  cudaEventRecord(d.begin, st);
  collide_pairs<<<blocks, kCollideThreads, 0, st>>>(k);
  cudaEventRecord(d.end, st);
  d.timed = true;
  c->last_launches += 4;
  if (!cuda_ok(c, cudaGetLastError(), "bg_collide launch")) return BG_ECUDA;
  auto d2h = [&](void* dst, const void* src, size_t bytes) {
    ok = ok && cuda_ok(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st), "bg_collide download");
  };
  d2h(out->points, L.points, static_cast<size_t>(np)); d2h(out->normal, L.normal, 3 * p8);
  d2h(out->point, L.point, 3 * bg::P * p8); d2h(out->separation, L.separation, bg::P * p8);
  d2h(out->pid, L.pid, bg::P * p4);
  ok = ok && cuda_ok(c, cudaStreamSynchronize(st), "bg_collide");
  return ok ? BG_OK : BG_ECUDA;
}

double bg_last_collide_ms(bg_ctx* c) {
  if (c == nullptr || !c->nw.timed) return -1;
  float ms = 0;
  if (cudaEventSynchronize(c->nw.end) != cudaSuccess || cudaEventElapsedTime(&ms, c->nw.begin, c->nw.end) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return ms;
}

}  // extern "C"

// ---- the colouring on the device (bg_colour) -----------------------------------------------

namespace {

struct ColourLayout {
  int32_t *a, *b, *deg, *off, *cursor, *list, *rank, *colour, *order, *starts, *status, *tiles;
  int32_t *keys[2], *vals[2], *rcounts, *colour_counts;
  uint8_t *type, *frozen;
  uint32_t* used;
  unsigned int* done;
  size_t bytes;
};

ColourLayout colour_layout(unsigned char* base, size_t nb, size_t n) {
  Carve k{base};
  ColourLayout L;
  const size_t tiles = (n + bgcol::kRadixThreads - 1) / bgcol::kRadixThreads;
  L.a = k.take<int32_t>(n); L.b = k.take<int32_t>(n);
  L.type = k.take<uint8_t>(nb); L.frozen = k.take<uint8_t>(nb);
  // zeroed together before each call: deg, cursor, used, done, colour_counts, status
  L.deg = k.take<int32_t>(nb); L.cursor = k.take<int32_t>(nb); L.used = k.take<uint32_t>(nb);
  L.done = k.take<unsigned int>(nb); L.colour_counts = k.take<int32_t>(bgcol::kRuns); L.status = k.take<int32_t>(1);
  L.off = k.take<int32_t>(nb + 1); L.list = k.take<int32_t>(2 * n); L.rank = k.take<int32_t>(2 * n);
  L.colour = k.take<int32_t>(n); L.order = k.take<int32_t>(n); L.starts = k.take<int32_t>(bgcol::kStarts);
  for (int j = 0; j < 2; j++) { L.keys[j] = k.take<int32_t>(n); L.vals[j] = k.take<int32_t>(n); }
  L.rcounts = k.take<int32_t>(bgcol::kBuckets * tiles + 1);
  L.tiles = k.take<int32_t>(std::max(nb, bgcol::kBuckets * tiles) / bgcol::kTile + 2);
  L.bytes = k.end;
  return L;
}

// The colouring's block, grown (by doubling) to hold nb slots and n manifolds.
bool colour_block(bg_ctx* c, size_t nb, size_t n) {
  bg_ctx::Colouring& d = c->col;
  if (d.block != nullptr && nb <= d.bodies && n <= d.rows) return true;
  cudaStreamSynchronize(c->stream);
  if (d.block) cudaFree(d.block);
  d.block = nullptr;
  d.bodies = grown(d.bodies, nb);
  d.rows = grown(d.rows, n);
  void* block = nullptr;
  if (cudaMalloc(&block, colour_layout(nullptr, d.bodies, d.rows).bytes) != cudaSuccess) {
    cudaGetLastError();
    d.bodies = d.rows = 0;
    return false;
  }
  d.block = static_cast<unsigned char*>(block);
  return true;
}

// Exclusive scan of in[0..n) into out[0..n] (out[n] the total) on the stream, across blocks (n > 0;
// `tiles` holds n / kTile + 2 entries).  in and out may be the same array.
void scan_into(cudaStream_t st, const int32_t* in, int32_t* out, int n, int32_t* tiles) {
  const int ntiles = (n + bgcol::kTile - 1) / bgcol::kTile;
  bgcol::col_tile_sums<<<ntiles, bgcol::kScanThreads, 0, st>>>(in, n, tiles);
  bgcol::col_scan<<<1, bgcol::kScanThreads, 0, st>>>(tiles, tiles, ntiles);
  bgcol::col_tile_scan<<<ntiles, bgcol::kScanThreads, 0, st>>>(in, out, n, tiles);
}

// colour() and arrange()'s order for p.n manifolds over p.nb slots, queued on the context's
// stream (p's arrays zeroed as colour_layout() says; `tiles` holds max(nb, kBuckets * p.tiles) / kTile + 2).
bool colour_kernels(bg_ctx* c, bgcol::ColourParams& p, int32_t* tiles) {
  cudaStream_t st = c->stream;
  const int64_t n = p.n, nb = p.nb;
  const int rows_grid = std::max(1, std::min(static_cast<int>((n + 255) / 256), 8 * c->sms));
  const int body_grid = std::max(1, std::min(static_cast<int>((nb + 255) / 256), 8 * c->sms));
  bgcol::col_degrees<<<rows_grid, 256, 0, st>>>(p);
  scan_into(st, p.deg, p.off, static_cast<int>(nb), tiles);
  bgcol::col_fill<<<rows_grid, 256, 0, st>>>(p);
  bgcol::col_ranks<<<body_grid, 256, 0, st>>>(p);
  {
    void* args[] = {&p};
    if (!cuda_ok(c, cudaLaunchCooperativeKernel(reinterpret_cast<void*>(bgcol::col_colour), dim3(c->sms), dim3(256),
                                                args, 0, st), "col_colour launch"))
      return false;
  }
  // arrange()'s order: the stable radix sort by (colour, b), 8 bits a pass
  bgcol::col_keys<<<rows_grid, 256, 0, st>>>(p);
  int bits = 1;
  while ((static_cast<int64_t>(1) << bits) <= static_cast<int64_t>(bgcol::kRuns) * nb) bits++;
  const int passes = (bits + 7) / 8;
  for (int pass = 0; pass < passes; pass++) {
    bgcol::col_radix_count<<<p.tiles, bgcol::kRadixThreads, 0, st>>>(p, pass & 1, 8 * pass);
    scan_into(st, p.rcounts, p.rcounts, bgcol::kBuckets * p.tiles, tiles);
    bgcol::col_radix_place<<<p.tiles, bgcol::kRadixThreads, 0, st>>>(p, pass & 1, 8 * pass, pass + 1 == passes);
  }
  bgcol::col_starts<<<1, 32, 0, st>>>(p);
  c->last_launches += 9 + 5 * passes;
  return cuda_ok(c, cudaGetLastError(), "colour launch");
}

}  // namespace

extern "C" {

int32_t bg_colour(bg_ctx* c, const bg_bodies* B, int32_t count, const int32_t* a, const int32_t* b, int32_t* colour,
                  int32_t* order, int32_t* starts, int32_t* solved) {
  if (c == nullptr) return BG_EINVAL;
  if (B == nullptr || starts == nullptr || solved == nullptr || count < 0 || B->capacity < 0) {
    set_error(c, "bg_colour: bodies, starts or solved is NULL, or a count is negative");
    return BG_EINVAL;
  }
  const int64_t n = count, nb = B->capacity;
  if (n > 0 && (a == nullptr || b == nullptr || colour == nullptr || order == nullptr || B->type == nullptr ||
                B->frozen == nullptr)) {
    set_error(c, "bg_colour: a column is NULL");
    return BG_EINVAL;
  }
  if (static_cast<int64_t>(bgcol::kRuns) * nb + 1 > INT32_MAX || 2 * n > INT32_MAX) {
    set_error(c, "bg_colour: too many slots or manifolds");
    return BG_EINVAL;
  }
  for (int64_t f = 0; f < n; f++)
    if (a[f] < 0 || a[f] >= nb || b[f] < 0 || b[f] >= nb || a[f] == b[f]) {
      set_error(c, "bg_colour: manifold %lld has slots %d, %d of %lld", static_cast<long long>(f), a[f], b[f],
                static_cast<long long>(nb));
      return BG_EINVAL;
    }
  std::fill(starts, starts + BG_STARTS, 0);
  *solved = 0;
  if (n == 0) return BG_OK;
  int32_t any_frozen = 0;
  for (int64_t x = 0; x < nb && !any_frozen; x++) any_frozen = B->frozen[x] != 0;
  cudaSetDevice(c->device);
  bg_ctx::Colouring& d = c->col;
  if (!colour_block(c, static_cast<size_t>(nb), static_cast<size_t>(n))) {
    set_error(c, "bg_colour: cudaMalloc failed");
    return BG_ENOMEM;
  }
  if (d.begin == nullptr) {
    cudaEventCreate(&d.begin);
    cudaEventCreate(&d.end);
  }
  // laid out for this call's sizes (the block holds at least that much)
  const ColourLayout L = colour_layout(d.block, static_cast<size_t>(nb), static_cast<size_t>(n));
  cudaStream_t st = c->stream;
  bool ok = cuda_ok(c, cudaMemcpyAsync(L.a, a, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st), "bg_colour") &&
            cuda_ok(c, cudaMemcpyAsync(L.b, b, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st), "bg_colour") &&
            cuda_ok(c, cudaMemcpyAsync(L.type, B->type, static_cast<size_t>(nb), cudaMemcpyHostToDevice, st), "bg_colour") &&
            cuda_ok(c, cudaMemcpyAsync(L.frozen, B->frozen, static_cast<size_t>(nb), cudaMemcpyHostToDevice, st), "bg_colour");
  const size_t zero = reinterpret_cast<unsigned char*>(L.off) - reinterpret_cast<unsigned char*>(L.deg);
  ok = ok && cuda_ok(c, cudaMemsetAsync(L.deg, 0, zero, st), "bg_colour");
  if (!ok) return BG_ECUDA;
  bgcol::ColourParams p;
  p.n = static_cast<int32_t>(n); p.nb = static_cast<int32_t>(nb); p.a = L.a; p.b = L.b; p.type = L.type;
  p.frozen = L.frozen; p.any_frozen = any_frozen; p.deg = L.deg; p.off = L.off; p.cursor = L.cursor; p.list = L.list;
  p.rank = L.rank; p.used = L.used; p.done = L.done; p.colour = L.colour; p.order = L.order; p.starts = L.starts;
  p.status = L.status; p.budget = c->budget;
  for (int j = 0; j < 2; j++) { p.keys[j] = L.keys[j]; p.vals[j] = L.vals[j]; }
  p.rcounts = L.rcounts; p.colour_counts = L.colour_counts;
  p.tiles = static_cast<int32_t>((n + bgcol::kRadixThreads - 1) / bgcol::kRadixThreads);
  cudaEventRecord(d.begin, st);
  if (!colour_kernels(c, p, L.tiles)) return BG_ECUDA;
  cudaEventRecord(d.end, st);
  d.timed = true;
  if (!cuda_ok(c, cudaGetLastError(), "bg_colour launch")) return BG_ECUDA;
  int32_t status = 0;
  ok = cuda_ok(c, cudaMemcpyAsync(&status, L.status, sizeof status, cudaMemcpyDeviceToHost, st), "bg_colour") &&
       cuda_ok(c, cudaStreamSynchronize(st), "bg_colour");
  if (!ok) return BG_ECUDA;
  if (status != 0) {
    set_error(c, "bg_colour: a wait ran past its budget");
    return BG_ETIMEOUT;
  }
  ok = cuda_ok(c, cudaMemcpyAsync(colour, L.colour, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st), "bg_colour") &&
       cuda_ok(c, cudaMemcpyAsync(order, L.order, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st), "bg_colour") &&
       cuda_ok(c, cudaMemcpyAsync(starts, L.starts, sizeof(int32_t) * BG_STARTS, cudaMemcpyDeviceToHost, st), "bg_colour") &&
       cuda_ok(c, cudaStreamSynchronize(st), "bg_colour");
  if (!ok) return BG_ECUDA;
  *solved = starts[BG_RESTING];
  return BG_OK;
}

double bg_last_colour_ms(bg_ctx* c) {
  if (c == nullptr || !c->col.timed) return -1;
  float ms = 0;
  if (cudaEventSynchronize(c->col.end) != cudaSuccess || cudaEventElapsedTime(&ms, c->col.begin, c->col.end) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return ms;
}

}  // extern "C"

// ---- a step's contacts on the device (bg_contact_step) -------------------------------------
//
// One call runs the step's contact pipeline on the context's stream: the narrowphase over the
// pair list (bg_collide's kernels), the rows emitted and warm-started from the contact memory
// (contact.cuh), colour() and arrange() (colour.cuh), the solve order and the grid's dataflow
// tables (contact.cuh, what order_rows() works out on the host for bg_solve_step), the solve
// stage, and store()/touched() into the other bank of contact memory.  The host waits on the
// device twice: for the number of rows (the colouring's launch sizes), and for the colour starts
// and the number of runs (the stage's launch parameters).

namespace {

// Where the pairs and the materials land in the upload block, after the bodies.
struct ContactIn {
  const int32_t *a = nullptr, *b = nullptr, *memory = nullptr;
  const double *margin = nullptr, *tol = nullptr, *friction = nullptr, *restitution = nullptr, *size = nullptr;
  const double* reach = nullptr;
};

Plan plan_contact_in(bg_ctx* c, const bg_bodies* B, const bg_materials* M, const bg_contact_pairs* CP, size_t nb,
                     size_t np, size_t na, unsigned char* base, ContactIn& in) {
  Plan P = plan_in(c, B, nullptr, nb, 0, na, base);
  const bg_pairs* L = CP ? &CP->list : nullptr;
  in.a = P.in<int32_t>(L ? L->a : nullptr, np, "pairs.a");
  in.b = P.in<int32_t>(L ? L->b : nullptr, np, "pairs.b");
  in.margin = P.in<double>(L ? L->margin : nullptr, np, "pairs.margin");
  in.tol = P.in<double>(L ? L->tolerance : nullptr, np, "pairs.tolerance");
  in.memory = P.in<int32_t>(CP ? CP->memory : nullptr, np, "pairs.memory");
  in.friction = P.in<double>(M ? M->friction : nullptr, nb, "materials.friction");
  in.restitution = P.in<double>(M ? M->restitution : nullptr, nb, "materials.restitution");
  in.size = P.in<double>(M ? M->size : nullptr, nb, "materials.size");
  const bool reuse = CP != nullptr && CP->reuse != 0;
  in.reach = P.in<double>(M && reuse ? M->reach : nullptr, reuse || CP == nullptr ? nb : 0, "materials.reach");
  return P;
}

// The call's scratch for nb slots and np pairs (so at most np rows), carved from `base` (NULL:
// only measures).
struct ContactLayout {
  int32_t *counts, *corder;        // the narrowphase's class sort
  uint8_t* points;                 // the manifolds, per pair
  double *normal, *point, *separation;
  uint32_t* pid;
  int32_t *rowof, *scan_tiles;     // np + 1 found rows, and the scan's tile sums
  bgct::FoundRows r;               // the rows in found order
  int32_t *ocounts, *groups, *chunk_base;   // the solve order
  int32_t *off, *cursor, *list;    // each body's solved rows (the dataflow's ranks)
  uint8_t* touching;
  int32_t* points_solved;
  uint8_t* kept;                   // per pair: its manifold reused
  size_t bytes;
};

ContactLayout contact_layout(unsigned char* base, size_t nb, size_t np) {
  Carve k{base};
  ContactLayout L;
  const size_t tiles = (np + bgct::kOrderThreads - 1) / bgct::kOrderThreads;
  L.counts = k.take<int32_t>(2 * kPairClasses); L.corder = k.take<int32_t>(np);
  L.points = k.take<uint8_t>(np); L.normal = k.take<double>(3 * np); L.point = k.take<double>(3 * bg::P * np);
  L.separation = k.take<double>(bg::P * np); L.pid = k.take<uint32_t>(bg::P * np);
  L.rowof = k.take<int32_t>(np + 1); L.scan_tiles = k.take<int32_t>(std::max(np, nb) / bgcol::kTile + 2);
  bgct::FoundRows& r = L.r;
  r.row = k.take<int32_t>(np); r.a = k.take<int32_t>(np); r.b = k.take<int32_t>(np); r.pair = k.take<int32_t>(np);
  r.points = k.take<uint8_t>(np); r.pid = k.take<uint32_t>(bg::P * np);
  r.normal = k.take<double>(3 * np); r.t1 = k.take<double>(3 * np); r.t2 = k.take<double>(3 * np);
  r.friction = k.take<double>(np); r.restitution = k.take<double>(np); r.tolerance = k.take<double>(np);
  r.patch = k.take<double>(np); r.separation = k.take<double>(bg::P * np); r.point = k.take<double>(3 * bg::P * np);
  r.shift = k.take<double>(3 * bg::P * np); r.ni = k.take<double>(bg::P * np);
  r.ti1 = k.take<double>(np); r.ti2 = k.take<double>(np); r.ri1 = k.take<double>(np); r.ri2 = k.take<double>(np);
  r.si = k.take<double>(np); r.drift1 = k.take<double>(np); r.drift2 = k.take<double>(np);
  r.maxni = k.take<double>(bg::P * np); r.relvel = k.take<double>(bg::P * np); r.gap = k.take<double>(np);
  L.ocounts = k.take<int32_t>(bgct::kKeys * tiles + 1);
  L.groups = k.take<int32_t>(bgct::kKeys + 1); L.chunk_base = k.take<int32_t>(bgct::kKeys + 1);
  L.off = k.take<int32_t>(nb + 1); L.cursor = k.take<int32_t>(nb); L.list = k.take<int32_t>(2 * np);
  L.touching = k.take<uint8_t>(np); L.points_solved = k.take<int32_t>(1); L.kept = k.take<uint8_t>(np);
  L.bytes = k.end;
  return L;
}

// One bank of contact memory for `cap` records, carved from `base` (NULL: only measures).
bgct::Memory bank_at(unsigned char* base, size_t cap, size_t* bytes = nullptr) {
  Carve k{base};
  bgct::Memory m;
  m.points = k.take<uint8_t>(cap); m.pid = k.take<uint32_t>(bg::P * cap); m.ni = k.take<double>(bg::P * cap);
  m.friction = k.take<double>(3 * cap); m.twist = k.take<double>(3 * cap); m.slip = k.take<double>(3 * cap);
  m.touching = k.take<uint8_t>(cap); m.cached = k.take<uint8_t>(cap); m.cache_points = k.take<uint8_t>(cap);
  m.pose = k.take<double>(7 * cap); m.loss = k.take<double>(cap); m.local_normal = k.take<double>(3 * cap);
  m.local = k.take<double>(6 * bg::P * cap); m.cache_id = k.take<uint32_t>(bg::P * cap);
  if (bytes) *bytes = k.end;
  return m;
}

size_t bank_bytes(size_t cap) {
  size_t n = 0;
  bank_at(nullptr, cap, &n);
  return n;
}

bgct::Memory bank(const bg_ctx::Contact& d, int which) {
  return bank_at(d.banks + static_cast<size_t>(which) * bank_bytes(d.bank_cap), d.bank_cap);
}

// The scratch block and the banks, grown (by doubling) for nb slots and np pairs; a grown pair of
// banks takes the last call's records with it.
bool contact_blocks(bg_ctx* c, size_t nb, size_t np) {
  bg_ctx::Contact& d = c->ct;
  if (d.block == nullptr || nb > d.bodies || np > d.pairs) {
    cudaStreamSynchronize(c->stream);
    if (d.block) cudaFree(d.block);
    d.block = nullptr;
    d.bodies = grown(d.bodies, nb);
    d.pairs = grown(d.pairs, np);
    void* block = nullptr;
    if (cudaMalloc(&block, contact_layout(nullptr, d.bodies, d.pairs).bytes) != cudaSuccess) {
      cudaGetLastError();
      d.bodies = d.pairs = 0;
      set_error(c, "bg_contact_step: cudaMalloc failed");
      return false;
    }
    d.block = static_cast<unsigned char*>(block);
  }
  if (d.banks == nullptr || np > d.bank_cap) {
    const size_t cap = grown(d.bank_cap, np);
    void* banks = nullptr;
    if (cudaMalloc(&banks, 2 * bank_bytes(cap)) != cudaSuccess) {
      cudaGetLastError();
      set_error(c, "bg_contact_step: cudaMalloc failed");
      return false;
    }
    bool ok = true;
    if (d.banks != nullptr && d.count > 0) {
      const bgct::Memory from = bank(d, d.current), to = bank_at(static_cast<unsigned char*>(banks), cap);
      const size_t n = static_cast<size_t>(d.count);
      auto copy = [&](void* dst, const void* src, size_t bytes) {
        ok = ok && cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c->stream) == cudaSuccess;
      };
      copy(to.points, from.points, n); copy(to.pid, from.pid, sizeof(uint32_t) * bg::P * n);
      copy(to.ni, from.ni, sizeof(double) * bg::P * n); copy(to.friction, from.friction, sizeof(double) * 3 * n);
      copy(to.twist, from.twist, sizeof(double) * 3 * n); copy(to.slip, from.slip, sizeof(double) * 3 * n);
      copy(to.touching, from.touching, n); copy(to.cached, from.cached, n); copy(to.cache_points, from.cache_points, n);
      copy(to.pose, from.pose, sizeof(double) * 7 * n); copy(to.loss, from.loss, sizeof(double) * n);
      copy(to.local_normal, from.local_normal, sizeof(double) * 3 * n);
      copy(to.local, from.local, sizeof(double) * 6 * bg::P * n); copy(to.cache_id, from.cache_id, sizeof(uint32_t) * bg::P * n);
      ok = ok && cudaStreamSynchronize(c->stream) == cudaSuccess;
    }
    if (!ok) {
      cudaGetLastError();
      cudaFree(banks);
      set_error(c, "bg_contact_step: the contact memory could not be moved");
      return false;
    }
    if (d.banks) cudaFree(d.banks);
    d.banks = static_cast<unsigned char*>(banks);
    d.bank_cap = cap;
    d.current = 0;
  }
  if (d.summary == nullptr) {
    void* h = nullptr;
    if (cudaHostAlloc(&h, 4096, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      set_error(c, "bg_contact_step: cudaHostAlloc failed");
      return false;
    }
    d.summary = static_cast<int32_t*>(h);
  }
  if (d.ev[0] == nullptr)
    for (cudaEvent_t& e : d.ev) cudaEventCreate(&e);
  return true;
}

// What the host checks before anything is copied: every index a kernel addresses memory with.
int contact_problem(bg_ctx* c, const bg_bodies* B, const bg_materials* M, const bg_contact_pairs* CP,
                    const bg_step* step) {
  if (B == nullptr || M == nullptr || CP == nullptr || step == nullptr) {
    set_error(c, "bg_contact_step: bodies, materials, pairs, step or out is NULL");
    return BG_EINVAL;
  }
  if (!(step->dt > 0) || step->substeps < 1) {
    set_error(c, "step: dt must be positive and substeps at least 1");
    return BG_EINVAL;
  }
  const int64_t nb = B->capacity, np = CP->list.count, na = B->awake_count;
  if (nb < 0 || na < 0 || na > nb || np < 0) {
    set_error(c, "bg_contact_step: negative or inconsistent counts");
    return BG_EINVAL;
  }
  if (static_cast<int64_t>(bgcol::kRuns) * nb + 1 > INT32_MAX || 2 * np + 64 > INT32_MAX) {
    set_error(c, "bg_contact_step: too many slots or pairs");
    return BG_EINVAL;
  }
  if (np > 0 && (CP->list.a == nullptr || CP->list.b == nullptr || CP->list.margin == nullptr ||
                 CP->list.tolerance == nullptr || CP->memory == nullptr)) {
    set_error(c, "bg_contact_step: a pair column is NULL");
    return BG_EINVAL;
  }
  if (nb > 0 && (B->shape == nullptr || B->frozen == nullptr || B->inv_mass == nullptr)) {
    set_error(c, "bg_contact_step: bodies.shape, frozen and inv_mass must be given");
    return BG_EINVAL;
  }
  if (na > 0 && B->awake_list == nullptr) {
    set_error(c, "bg_contact_step: bodies.awake_list must be given");
    return BG_EINVAL;
  }
  // The pairs are checked in chunks on the host pool; the first bad pair in list order is reported.
  const int32_t records = c->ct.count;
  constexpr int64_t kChunk = 16384;
  const int chunks = static_cast<int>((np + kChunk - 1) / kChunk);
  std::vector<int64_t> first_bad(static_cast<size_t>(chunks), -1);
  pool_of(c)->run(chunks, [&](int k) {
    for (int64_t i = k * kChunk; i < std::min(np, (k + 1) * kChunk); i++) {
      const int32_t a = CP->list.a[i], b = CP->list.b[i], j = CP->memory[i];
      bool bad = a < 0 || a >= nb || b < 0 || b >= nb || a == b || j < -1 || j >= records;
      if (!bad)
        for (const int32_t s : {a, b}) bad = bad || (B->shape[s] != BG_BOX && B->shape[s] != BG_SPHERE && B->shape[s] != BG_CAPSULE);
      if (bad) {
        first_bad[static_cast<size_t>(k)] = i;
        return;
      }
    }
  });
  for (const int64_t i : first_bad) {
    if (i < 0) continue;
    const int32_t a = CP->list.a[i], b = CP->list.b[i], j = CP->memory[i];
    if (a < 0 || a >= nb || b < 0 || b >= nb || a == b) {
      set_error(c, "bg_contact_step: pair %lld has slots %d, %d of %lld", static_cast<long long>(i), a, b,
                static_cast<long long>(nb));
      return BG_EINVAL;
    }
    for (const int32_t s : {a, b})
      if (B->shape[s] != BG_BOX && B->shape[s] != BG_SPHERE && B->shape[s] != BG_CAPSULE) {
        set_error(c, "bg_contact_step: slot %d is not a box, sphere or capsule", s);
        return BG_EUNSUPPORTED;
      }
    set_error(c, "bg_contact_step: pair %lld names contact record %d of %d", static_cast<long long>(i), j, records);
    return BG_EINVAL;
  }
  for (int64_t i = 0; i < na; i++)
    if (static_cast<uint32_t>(B->awake_list[i]) >= static_cast<uint32_t>(nb)) {
      set_error(c, "bg_contact_step: bodies.awake_list entry %lld is not one of the %lld slots", static_cast<long long>(i),
                static_cast<long long>(nb));
      return BG_EINVAL;
    }
  return BG_OK;
}

}  // namespace

extern "C" {

int32_t bg_contact_step(bg_ctx* c, const bg_bodies* B, const bg_materials* M, const bg_contact_pairs* CP,
                        const bg_step* step, bg_contact_result* out) {
  if (c == nullptr) return BG_EINVAL;
  if (out == nullptr) {
    set_error(c, "bg_contact_step: out is NULL");
    return BG_EINVAL;
  }
  int rc = contact_problem(c, B, M, CP, step);
  if (rc != BG_OK) return rc;
  const int nb = B->capacity, np = CP->list.count, na = B->awake_count;
  int32_t any_frozen = 0;
  for (int x = 0; x < nb && !any_frozen; x++) any_frozen = B->frozen[x] != 0;
  cudaSetDevice(c->device);
  c->last_launches = 0;
  c->uploaded = false;
  bg_ctx::Contact& d = c->ct;
  ContactIn in;
  const size_t in_need = plan_contact_in(c, nullptr, nullptr, nullptr, static_cast<size_t>(nb), static_cast<size_t>(np),
                                         static_cast<size_t>(na), nullptr, in).end;
  if (!ensure(c, nb, std::max(np, 1), na, 1, 0, in_need)) return BG_ENOMEM;
  if (!contact_blocks(c, static_cast<size_t>(nb), static_cast<size_t>(np))) return BG_ENOMEM;
  const ContactLayout L = contact_layout(d.block, static_cast<size_t>(nb), static_cast<size_t>(np));
  const bgct::Memory old = bank(d, d.current), next = bank(d, 1 - d.current);
  c->nbodies = nb;
  c->nawake = na;
  c->nworlds = 1;
  c->batch = false;
  rc = upload_plan(c, plan_contact_in(c, B, M, CP, static_cast<size_t>(nb), static_cast<size_t>(np),
                                      static_cast<size_t>(na), c->d_in, in));
  if (rc != BG_OK) return rc;
  cudaStream_t st = c->stream;
  int32_t* sum = d.summary;
  auto fetch = [&](void* dst, const void* src, size_t bytes, const char* what) {
    return cuda_ok(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st), what);
  };
  const int sweep = std::max(1, std::min((np + 255) / 256, 8 * c->sms));
  const bool reuse = CP->reuse != 0;
  bgct::Poses poses;
  poses.p = c->bin.position; poses.q = c->bin.rotation; poses.v = c->bin.velocity; poses.w = c->bin.angular;
  poses.dims = c->bin.dims; poses.reach = in.reach; poses.gscale = c->bin.gravity_scale; poses.type = c->bin.type;
  poses.shape = c->bin.shape; poses.joint_head = c->bin.joint_head;
  for (int k = 0; k < 3; k++) poses.gravity[k] = step->gravity[k];
  poses.dt = step->dt;
  // the kept manifolds that still hold, then the narrowphase, as bg_collide runs it, for the rest
  cudaEventRecord(d.ev[0], st);
  if (np > 0) {
    if (reuse) {
      bgct::ReuseParams rp;
      rp.np = np; rp.a = in.a; rp.b = in.b; rp.margin = in.margin; rp.tol = in.tol; rp.memory = in.memory;
      rp.s = poses; rp.old = old; rp.kept = L.kept; rp.points = L.points; rp.normal = L.normal; rp.point = L.point;
      rp.separation = L.separation; rp.pid = L.pid;
      bgct::ct_reuse<<<sweep, 256, 0, st>>>(rp);
      c->last_launches += 1;
    }
    if (!cuda_ok(c, cudaMemsetAsync(L.counts, 0, 2 * kPairClasses * sizeof(int32_t), st), "bg_contact_step")) return BG_ECUDA;
    CollideParams k;
    k.p = c->bin.position; k.q = c->bin.rotation; k.dims = c->bin.dims; k.gscale = c->bin.gravity_scale;
    k.shape = c->bin.shape; k.type = c->bin.type;
    k.a = in.a; k.b = in.b; k.margin = in.margin; k.tol = in.tol; k.n = np;
    for (int e = 0; e < 3; e++) k.gravity[e] = step->gravity[e];
    k.counts = L.counts; k.order = L.corder; k.points = L.points; k.normal = L.normal; k.point = L.point;
    k.separation = L.separation; k.pid = L.pid; k.skip = reuse ? L.kept : nullptr;
    collide_count<<<sweep, 256, 0, st>>>(k);
    collide_starts<<<1, 32, 0, st>>>(k);
    collide_scatter<<<sweep, 256, 0, st>>>(k);
    const int blocks = std::min((np + kCollideThreads - 1) / kCollideThreads, 64 * c->sms);
    collide_pairs<<<blocks, kCollideThreads, 0, st>>>(k);
    c->last_launches += 4;
  }
  cudaEventRecord(d.ev[1], st);
  // the rows: which pairs touch, and their found rows (the host waits for the count)
  bgct::EmitParams e;
  e.np = np; e.a = in.a; e.b = in.b; e.tol = in.tol; e.memory = in.memory;
  e.points = L.points; e.normal = L.normal; e.point = L.point; e.separation = L.separation; e.pid = L.pid;
  e.friction = in.friction; e.restitution = in.restitution; e.size = in.size; e.type = c->bin.type;
  e.rowof = L.rowof; e.old = old; e.r = L.r;
  e.reuse = reuse ? 1 : 0; e.kept = L.kept; e.next = next; e.s = poses;
  int nrows = 0;
  if (np > 0) {
    bgct::ct_flags<<<sweep, 256, 0, st>>>(e);
    scan_into(st, L.rowof, L.rowof, np, L.scan_tiles);
    c->last_launches += 4;
    if (!fetch(sum, L.rowof + np, sizeof(int32_t), "bg_contact_step") ||
        !cuda_ok(c, cudaStreamSynchronize(st), "bg_contact_step"))
      return BG_ECUDA;
    nrows = sum[0];
  }
  c->nrows = nrows;
  int32_t starts[bg::NSTARTS] = {0};
  int32_t nchunks = 0;
  if (nrows > 0) {
    const int rgrid = std::max(1, std::min((nrows + 255) / 256, 8 * c->sms));
    bgct::ct_emit<<<sweep, 256, 0, st>>>(e);
    // colour() and arrange()'s order, on the found rows
    if (!colour_block(c, static_cast<size_t>(nb), static_cast<size_t>(nrows))) {
      set_error(c, "bg_contact_step: cudaMalloc failed");
      return BG_ENOMEM;
    }
    const ColourLayout CL = colour_layout(c->col.block, static_cast<size_t>(nb), static_cast<size_t>(nrows));
    const size_t zero = reinterpret_cast<unsigned char*>(CL.off) - reinterpret_cast<unsigned char*>(CL.deg);
    if (!cuda_ok(c, cudaMemsetAsync(CL.deg, 0, zero, st), "bg_contact_step")) return BG_ECUDA;
    bgcol::ColourParams p;
    p.n = nrows; p.nb = nb; p.a = L.r.a; p.b = L.r.b; p.type = c->bin.type; p.frozen = c->bin.frozen;
    p.any_frozen = any_frozen; p.deg = CL.deg; p.off = CL.off; p.cursor = CL.cursor; p.list = CL.list;
    p.rank = CL.rank; p.used = CL.used; p.done = CL.done; p.colour = CL.colour; p.order = CL.order;
    p.starts = CL.starts; p.status = CL.status; p.budget = c->budget;
    for (int j = 0; j < 2; j++) { p.keys[j] = CL.keys[j]; p.vals[j] = CL.vals[j]; }
    p.rcounts = CL.rcounts; p.colour_counts = CL.colour_counts;
    p.tiles = (nrows + bgcol::kRadixThreads - 1) / bgcol::kRadixThreads;
    if (!colour_kernels(c, p, CL.tiles)) return BG_ECUDA;
    bgct::ct_rest<<<rgrid, 256, 0, st>>>(L.r, CL.colour, nrows);
    // the solve order and its runs
    bgct::OrderParams op;
    op.n = nrows; op.tiles = (nrows + bgct::kOrderThreads - 1) / bgct::kOrderThreads;
    op.order = CL.order; op.colour = CL.colour; op.points = L.r.points; op.counts = L.ocounts;
    op.perm = c->perm_dev; op.iperm = c->iperm_dev; op.groups = L.groups; op.chunks = c->chunks_dev;
    op.chunk_base = L.chunk_base;
    bgct::ct_order_count<<<op.tiles, bgct::kOrderThreads, 0, st>>>(op);
    scan_into(st, L.ocounts, L.ocounts, bgct::kKeys * op.tiles, L.scan_tiles);
    bgct::ct_order_place<<<op.tiles, bgct::kOrderThreads, 0, st>>>(op);
    bgct::ct_order_runs<<<1, bgct::kRunThreads, 0, st>>>(op);
    bgct::ct_order_chunks<<<rgrid, 256, 0, st>>>(op);
    c->last_launches += 9;
    if (!cuda_ok(c, cudaGetLastError(), "bg_contact_step launch")) return BG_ECUDA;
    // the host waits for what the stage's launch needs
    if (!fetch(sum, CL.starts, sizeof(int32_t) * bg::NSTARTS, "bg_contact_step") ||
        !fetch(sum + 64, L.chunk_base + bgct::kKeys, sizeof(int32_t), "bg_contact_step") ||
        !fetch(sum + 65, CL.status, sizeof(int32_t), "bg_contact_step") ||
        !cuda_ok(c, cudaStreamSynchronize(st), "bg_contact_step"))
      return BG_ECUDA;
    if (sum[65] != 0) {
      set_error(c, "bg_contact_step: a colouring wait ran past its budget; the step is lost");
      return BG_ETIMEOUT;
    }
    for (int k = 0; k < bg::NSTARTS; k++) starts[k] = sum[k];
    nchunks = sum[64];
  }
  const int solved = starts[bg::RESTING_RUN];
  // the world the stage solves, and the grid's dataflow tables
  bg::WorldDesc w = {};
  w.body0 = 0; w.nbodies = nb; w.awake0 = 0; w.nawake = na; w.row0 = 0; w.nrows = nrows; w.solved = solved;
  for (int k = 0; k < bg::NSTARTS; k++) w.starts[k] = starts[k];
  for (int k = 0; k < 3; k++) w.gravity[k] = step->gravity[k];
  c->worlds.assign(1, w);
  {
    std::vector<int32_t> bo = {0, nb}, ao = {0, na}, ro = {0, nrows};
    rc = upload_worlds(c, bo, ao, ro);
    if (rc != BG_OK) return rc;
  }
  const size_t nb4 = sizeof(int32_t) * static_cast<size_t>(std::max(nb, 1));
  if (!cuda_ok(c, cudaMemsetAsync(c->deg_dev, 0, nb4, st), "bg_contact_step") ||
      !cuda_ok(c, cudaMemsetAsync(L.cursor, 0, nb4, st), "bg_contact_step") ||
      !cuda_ok(c, cudaMemsetAsync(c->body_world_dev, 0, nb4, st), "bg_contact_step"))
    return BG_ECUDA;
  if (nrows > 0) {
    bgct::FlowParams f;
    f.solved = solved; f.nrows = nrows; f.nb = nb; f.perm = c->perm_dev; f.a = L.r.a; f.b = L.r.b;
    f.inv_mass = c->bin.inv_mass; f.deg = c->deg_dev; f.off = L.off; f.cursor = L.cursor; f.list = L.list;
    f.rank = c->rank_dev;
    const int rgrid = std::max(1, std::min((nrows + 255) / 256, 8 * c->sms));
    const int bgrid = std::max(1, std::min((nb + 255) / 256, 8 * c->sms));
    bgct::ct_flow_degrees<<<rgrid, 256, 0, st>>>(f);
    scan_into(st, c->deg_dev, L.off, nb, L.scan_tiles);
    bgct::ct_flow_fill<<<rgrid, 256, 0, st>>>(f);
    bgct::ct_flow_ranks<<<bgrid, 256, 0, st>>>(f);
    c->last_launches += 6;
  }
  c->nchunks = nchunks;
  c->chunks.clear();
  c->bruns.clear();
  c->brun_rows.clear();
  // the found rows in the caller's row layout are what the stage's unpack reads
  RowStage& q = c->rin;
  q.row = L.r.row; q.a = L.r.a; q.b = L.r.b; q.points = L.r.points; q.normal = L.r.normal; q.t1 = L.r.t1;
  q.t2 = L.r.t2; q.friction = L.r.friction; q.restitution = L.r.restitution; q.tolerance = L.r.tolerance;
  q.patch = L.r.patch; q.separation = L.r.separation; q.point = L.r.point; q.shift = L.r.shift;
  q.normal_impulse = L.r.ni; q.ti1 = L.r.ti1; q.ti2 = L.r.ti2; q.ri1 = L.r.ri1; q.ri2 = L.r.ri2; q.si = L.r.si;
  q.drift1 = L.r.drift1; q.drift2 = L.r.drift2;
  c->maxni_in = L.r.maxni;
  c->relvel_in = L.r.relvel;
  c->gap_in = L.r.gap;
  c->uploaded = true;
  rc = unpack(c);
  if (rc != BG_OK) return rc;
  rc = launch_stage(c, step);
  if (rc != BG_OK) return rc;
  // store() and touched(), into the other bank
  if (!cuda_ok(c, cudaMemsetAsync(L.points_solved, 0, sizeof(int32_t), st), "bg_contact_step")) return BG_ECUDA;
  if (np > 0) {
    bgct::KeepParams kp;
    kp.np = np; kp.solved = solved; kp.points = L.points; kp.rowof = L.rowof; kp.memory = in.memory;
    kp.iperm = c->iperm_dev; kp.pid = L.r.pid; kp.R = c->R; kp.old = old; kp.next = next; kp.touching = L.touching;
    kp.points_solved = L.points_solved; kp.reuse = reuse ? 1 : 0;
    bgct::ct_keep<<<sweep, 256, 0, st>>>(kp);
    c->last_launches += 1;
  }
  cudaEventRecord(d.ev[3], st);
  // the bodies back, with each pair's count and flag
  plan_out(c, nullptr, nullptr, static_cast<size_t>(nb), 0, c->d_out);
  {
    const int blocks = std::max(1, std::min(4 * c->sms, (nb + kUnpackThreads - 1) / kUnpackThreads));
    pack_bodies<<<blocks, kUnpackThreads, 0, st>>>(c->B, c->bout, nb);
    c->last_launches += 1;
  }
  if (!cuda_ok(c, cudaGetLastError(), "bg_contact_step launch")) return BG_ECUDA;
  if (!fetch(sum + 66, L.points_solved, sizeof(int32_t), "bg_contact_step")) return BG_ECUDA;
  rc = download_columns(c, B, nullptr);
  if (rc != BG_OK) return rc;
  if (np > 0 && ((out->points != nullptr && !fetch(out->points, L.points, static_cast<size_t>(np), "bg_contact_step")) ||
                 (out->touching != nullptr && !fetch(out->touching, L.touching, static_cast<size_t>(np), "bg_contact_step")) ||
                 !cuda_ok(c, cudaStreamSynchronize(st), "bg_contact_step")))
    return BG_ECUDA;
  // the records the next call reads are this call's
  d.current = 1 - d.current;
  d.count = np;
  d.timed = true;
  out->rows = nrows;
  out->solved = solved;
  out->points_solved = sum[66];
  for (int k = 0; k < bg::NSTARTS; k++) out->starts[k] = starts[k];
  return BG_OK;
}

int32_t bg_last_contact_ms(bg_ctx* c, double* ms) {
  if (c == nullptr || ms == nullptr || !c->ct.timed) return BG_EINVAL;
  const bg_ctx::Contact& d = c->ct;
  float t[4] = {0, 0, 0, 0};
  if (cudaEventSynchronize(d.ev[3]) != cudaSuccess || cudaEventElapsedTime(&t[0], d.ev[0], d.ev[1]) != cudaSuccess ||
      cudaEventElapsedTime(&t[1], d.ev[1], c->stage_begin) != cudaSuccess ||
      cudaEventElapsedTime(&t[2], c->stage_begin, c->stage_end) != cudaSuccess ||
      cudaEventElapsedTime(&t[3], c->stage_end, d.ev[3]) != cudaSuccess) {
    cudaGetLastError();
    return BG_ECUDA;
  }
  for (int k = 0; k < 4; k++) ms[k] = t[k];
  return BG_OK;
}

int32_t bg_contact_records(const bg_ctx* c) { return c == nullptr ? BG_EINVAL : c->ct.count; }

int32_t bg_contact_forget(bg_ctx* c) {
  if (c == nullptr) return BG_EINVAL;
  c->ct.count = 0;
  return BG_OK;
}

}  // extern "C"
