// Device-side layout of the solve stage's state.
//
// Bodies are stored by slot as small records sized to 32-byte sectors, so a row's gather of its
// two bodies touches the fewest sectors, and a sweep over the awake bodies still reads them
// contiguously:
//   vw[8 s]   vx vy vz wx wy wz . .        read and written by warm, solve, relax, restitution
//   mi[8 s]   invMass, invI xx xy xz yy yz zz .   (invI worked out each step by inertias)
//   pq[8 s]   px py pz . qx qy qz qw      read by solve, written by move
//   st[4 s]   start x y z .               start snapshot
//   sq[4 s]   startQ x y z w
//   tc[4 s]   tumbled x y z, ceiling      tumble() state
//   pr[12 s]  inertia(3) invInertia(3) dims(3) damping angularDamping gravityScale
//   fl[s]     flags: type 0-1, shape 2-3, frozen 4, framed 5, lock 6-8, jointed 9, awake 10
// Rows are stored column by column ("component-major"): scalar column c of row m at
// col[c * cap + m], so the 32 threads of a warp working on 32 consecutive rows read 32
// consecutive doubles of each column.  Point columns hold column (k * C + c) for point k.
#pragma once

#include <stdint.h>

namespace bg {

constexpr int P = 4;
constexpr int J = 12;
constexpr int FJ = 24;
constexpr int NCOLOURS = 32;
constexpr int OVERFLOW_RUN = 32;
constexpr int RESTING_RUN = 33;
constexpr int NSTARTS = 35;

// Body flag bits.
constexpr uint32_t F_TYPE = 3u;
constexpr int F_SHAPE_SHIFT = 2;
constexpr uint32_t F_FROZEN = 1u << 4;
constexpr uint32_t F_FRAMED = 1u << 5;
constexpr int F_LOCK_SHIFT = 6;
constexpr uint32_t F_JOINTED = 1u << 9;
constexpr uint32_t F_AWAKE = 1u << 10;

struct BodiesDev {
  double* vw;
  double* mi;
  double* pq;
  double* st;
  double* sq;
  double* tc;
  double* pr;
  uint32_t* fl;
  int32_t* awake_list;   // global slots of the awake bodies, world after world
  int32_t* head;         // restitution's per-body scratch (see restitution())
  int32_t* deg;          // rows that move this body in a pass (0 for a body the solve never moves)
  unsigned int* done;    // rows done on this body so far in the stage (the grid's dataflow)
};

struct RowsDev {
  int64_t cap;           // column stride
  int32_t* a;            // global slots
  int32_t* b;
  uint8_t* points;
  int32_t* row;          // found order -> global row, world after world
  double* n;             // 3 columns
  double* t1;            // 3
  double* t2;            // 3
  double* friction;
  double* restitution;
  double* tolerance;
  double* patch;
  double* separation;    // 4
  double* point;         // 12 (k*3+c)
  double* shift;         // 12
  double* ni;            // 4 normal impulses
  double* ti1;
  double* ti2;
  double* ri1;
  double* ri2;
  double* si;
  double* drift1;
  double* drift2;
  double* gap;
  double* maxni;         // 4
  double* relvel;        // 4
  uint8_t* sliding;
  double* anchorA;       // 3
  double* anchorB;       // 3
  // worked out once a step by prepare
  double* la;            // 12
  double* lb;            // 12
  double* adjusted;      // 4
  double* now;           // 4
  double* normalMass;    // 4
  double* lever;         // 4
  double* jac;           // 48 (k*12+c)
  double* K;             // 16
  double* fjac;          // 24
  double* tm;            // 3
  double* rm1;
  double* rm2;
  double* sm;
  // restitution's work lists
  int32_t* active;       // found indices of bouncy rows, compacted
  int32_t* pending;
  // the row's place among the rows on each of its bodies, in solve order (-1: a body the solve
  // never moves, so nothing to wait for)
  int32_t* rank_a;
  int32_t* rank_b;
};

// One world's share of the arrays.
struct WorldDesc {
  int32_t body0;         // first slot
  int32_t nbodies;
  int32_t awake0;        // first entry in awake_list
  int32_t nawake;
  int32_t row0;          // first row
  int32_t nrows;         // Contacts.count
  int32_t solved;
  int32_t starts[NSTARTS];
  double gravity[3];
};

struct Soft {
  double biasRate, massScale, impulseScale;
};

struct StageParams {
  BodiesDev B;
  RowsDev R;
  const WorldDesc* worlds;
  int32_t nworlds;
  double dt;
  int32_t substeps;
  Soft soft;
  // the grid barrier's arrival count and the step's status word (0 ok; 1 a wait ran past its
  // budget)
  unsigned int* bar_count;
  int32_t* status;
  int32_t* block_counts;  // per-block counts for restitution's compaction
  long long budget;
  // The grid's pass schedule: runs of rows (start, length), colour after colour, each within
  // one colour (or one row of the overflow); warp w takes runs w, w + warps, ... in order.
  const int2* chunks;
  int32_t nchunks;
  // The order CTAs take the worlds of a batch in (largest first), or NULL for 0, 1, 2, ...
  const int32_t* world_order;
  // A batch on the grid: each body's world, and the awake entries of every world together.
  const int32_t* body_world;
  int32_t nawake_total;
  // ... and its runs, drawn across worlds: run c is rows brun_rows[bruns[c].x ...][bruns[c].y]
  // (one colour and one point count; each world's overflow rows last, one a run).
  const int32_t* brun_rows;
  const int2* bruns;
  int32_t nbruns;
};

}  // namespace bg
