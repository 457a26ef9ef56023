/*
 * bearing_gpu.h - the C ABI of the B200 contact-solve library (libbearing_gpu.so).
 *
 * It takes the place of Bearing's worker threads (src/core/jobs.js, src/worker.js) for one
 * block of World.step: src/world.js:962-1032, the "solve stage".  In order, each step:
 *
 *   inertias        src/contact.js:1302-1310, 1493-1549   world inverse inertia per awake body
 *   start snapshot  src/world.js:964-974                  start / startQ of every awake body
 *   prepare         src/contact.js:1346-1445               per-row levers, masses, anchors, block K
 *   makeSoft        src/contact.js:1591-1597               soft-contact constants for h = dt/substeps
 *   substeps x N    src/world.js:1011-1024
 *     accelerate    src/world.js:1495-1530
 *     warm start    src/contact.js:1604-1663               colour by colour
 *     solve (bias)  src/contact.js:1782-2090               colour by colour, overflow in row order
 *     move          src/world.js:1533-1563, 2739-2834      incl. tumble() / untwist()
 *     relax         src/contact.js:1782-2090 (bias=false)
 *   restitution     src/contact.js:2229-2251               in found order (rows.row)
 *   slipped         src/contact.js:1122-1182               the drift half of store(); keep() stays on host
 *
 * The caller (the host side of World.step: broadphase, narrowphase, colouring in
 * src/graph.js:105-185) hands over the step's manifolds already laid out colour by colour,
 * with the reference's own column meanings (src/contact.js:184-248, src/graph.js:78-83).
 * Every array is plain FP64 / int32 / uint8 host memory owned by the caller.  The library owns
 * device memory, one CUDA stream and its kernels per context; two contexts never share state.
 *
 * Arithmetic is IEEE FP64 with no contraction (built with -fmad=false), in the reference's
 * operation order, so results are bit-identical to the reference's CPU solve over the same rows.
 *
 * Return codes: BG_OK (0) or a negative BG_E* code; bg_last_error() says why.  A failed
 * validation (BG_EINVAL) writes none of the caller's arrays and runs no kernel: the counts, the
 * colour starts and every index the caller passes are checked first (each row's a and b among
 * its world's slots, points 1..BG_POINTS, row[] a permutation of the world's rows, each awake
 * entry among the world's slots); a refused upload leaves the context with nothing uploaded.
 * A device wait that runs past its budget returns BG_ETIMEOUT, which the caller treats as
 * src/core/jobs.js:384-391 treats a lost step: fall back to the CPU.
 */
#ifndef BEARING_GPU_H
#define BEARING_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Points per manifold: src/contact.js:128 (P). */
#define BG_POINTS 4
/* Colours and the runs after them: src/graph.js:67-71 (COLOURS, OVERFLOW, RESTING). */
#define BG_COLOURS 32
#define BG_OVERFLOW 32
#define BG_RESTING 33
/* Length of rows.starts: src/contact.js:161 (COLOURS + 3). */
#define BG_STARTS 35

#define BG_OK 0
#define BG_EINVAL (-1)
#define BG_ECUDA (-2)
#define BG_ETIMEOUT (-3)
#define BG_ENOMEM (-4)
#define BG_EUNSUPPORTED (-5)
#define BG_EFAULT (-6)

/* bg_create flags */
#define BG_FLAG_NONE 0u
/* Reserved (accepted, no effect).  Every transfer already takes the fastest route by itself: a
 * column in page-locked host memory (cudaHostAlloc'd, or registered by the caller or through
 * bg_register_host) is copied to and
 * from directly; any other column goes through the library's own pinned staging, gathered and
 * scattered by a pool of host threads. */
#define BG_FLAG_PIN_HOST 1u
/* Run single worlds on the persistent grid (the default for a single world). */
#define BG_FLAG_GRID 2u
/* Run single worlds on one CTA (the path batched worlds take) instead of the grid. */
#define BG_FLAG_BLOCK 4u

/* World body type codes: src/world.js TYPES (dynamic 0, static 1, kinematic 2, character 3). */
#define BG_DYNAMIC 0
#define BG_STATIC 1
/* World shape codes: src/world.js:63 (box 0, sphere 1, capsule 2, hull 3, compound 4, mesh 5). */
#define BG_BOX 0
#define BG_SPHERE 1
#define BG_CAPSULE 2

typedef struct bg_ctx bg_ctx;

/*
 * Per-body columns, indexed by slot as World keeps them (src/world.js:228-311).  `capacity`
 * slots; vectors are packed (3 per slot, quaternions 4 per slot as x y z w).
 */
typedef struct bg_bodies {
  int32_t capacity;            /* slots in every per-body array */
  int32_t awake_count;         /* World._awakeCount */
  const int32_t* awake_list;   /* World._awakeList: the awake slots */
  const uint8_t* awake;        /* World._awake: 1 while awake (slipped() reads it) */
  /* read and written */
  double* position;            /* 3 per slot */
  double* rotation;            /* 4 per slot */
  double* velocity;            /* 3 per slot */
  double* angular;             /* 3 per slot */
  double* tumbled;             /* 3 per slot: world.js _tumbled */
  double* ceiling;             /* 1 per slot: world.js _ceiling */
  /* written */
  double* start;               /* 3 per slot: position as the step began (awake slots) */
  double* start_q;             /* 4 per slot */
  double* inv_i;               /* 6 per slot: world inverse inertia xx xy xz yy yz zz */
  /* read only */
  const double* inv_mass;      /* 1 */
  const double* inertia;       /* 3: principal moments */
  const double* inv_inertia;   /* 3 */
  const double* dims;          /* 3: box size; sphere radius; capsule radius, height */
  const double* damping;       /* 1 */
  const double* angular_damping; /* 1 */
  const double* gravity_scale; /* 1 */
  const uint8_t* type;         /* BG_DYNAMIC, BG_STATIC, ... */
  const uint8_t* shape;        /* BG_BOX, BG_SPHERE, BG_CAPSULE */
  const uint8_t* frozen;       /* World._frozen: nonzero frozen */
  const uint8_t* framed;       /* World._framed */
  const uint8_t* lock;         /* World._lock: bit k, no turning about world axis k */
  const int32_t* joint_head;   /* World._jointHead: nonzero for a jointed body */
} bg_bodies;

/*
 * One step's manifolds (src/contact.js Contacts), rows in colour order: colour k is rows
 * starts[k] .. starts[k+1]-1, the overflow starts[32] .. starts[33]-1, the resting run
 * starts[33] .. count-1 (not solved).  Point columns hold BG_POINTS entries per row,
 * vectors 3 per row or per point, as in the reference.
 */
typedef struct bg_rows {
  int32_t count;               /* Contacts.count */
  int32_t solved;              /* Contacts.solved == starts[33] */
  int32_t starts[BG_STARTS];   /* Contacts.starts */
  const int32_t* row;          /* found order -> row (Contacts.row), count entries */
  const int32_t* a;
  const int32_t* b;
  const uint8_t* points;       /* 1..4 */
  const double* normal;        /* 3 per row, from a to b */
  const double* t1;            /* 3 per row: basis() */
  const double* t2;            /* 3 per row */
  const double* friction;
  const double* restitution;
  const double* tolerance;
  const double* patch;
  const double* separation;    /* 4 per row */
  const double* point;         /* 12 per row */
  const double* shift;         /* 12 per row */
  /* read and written: warm-start impulses in, the step's impulses out */
  double* normal_impulse;      /* 4 per row */
  double* tangent_impulse1;
  double* tangent_impulse2;
  double* roll_impulse1;
  double* roll_impulse2;
  double* spin_impulse;
  double* drift1;              /* carried slip in, slipped() slip out */
  double* drift2;
  /* written */
  double* gap;                 /* least separation as the last pass saw it */
  double* max_normal_impulse;  /* 4 per row */
  double* relative_velocity;   /* 4 per row */
  /* written, and read after the stage by nothing but slipped() (src/contact.js:1125-1160), which
   * runs on the device: each may be NULL, and is then not copied back */
  uint8_t* sliding;
  double* anchor_a;            /* 3 per row */
  double* anchor_b;            /* 3 per row */
} bg_rows;

typedef struct bg_step {
  double dt;                   /* World.step(dt) */
  int32_t substeps;            /* World._substeps (8 by default) */
  double gravity[3];           /* World._gravity */
} bg_step;

/*
 * A batch of independent worlds solved in one launch.  bg_bodies and bg_rows then hold every
 * world's arrays end to end; these offsets say where each world's are.  Row columns' a and b,
 * awake_list entries and row[] entries are local to their world.
 */
typedef struct bg_worlds {
  int32_t count;               /* worlds */
  const int32_t* body_offset;  /* count+1: world w's slots are [body_offset[w], body_offset[w+1]) */
  const int32_t* awake_offset; /* count+1: into bodies.awake_list */
  const int32_t* row_offset;   /* count+1: into the row columns */
  const int32_t* starts;       /* BG_STARTS per world, local row numbers */
  const double* gravity;       /* 3 per world, or NULL for bg_step.gravity */
} bg_worlds;

/* Creates a context on CUDA device `device`.  NULL on failure (no device, no memory). */
bg_ctx* bg_create(int32_t device, uint32_t flags);
/* Frees every device buffer, stream and graph of the context. */
void bg_destroy(bg_ctx* ctx);
/* The last error's text for this context ("" if none).  Valid until the next call on ctx. */
const char* bg_last_error(const bg_ctx* ctx);
/* Version of the ABI: (major << 16) | minor. */
uint32_t bg_version(void);

/*
 * One solve stage end to end: uploads the bodies and rows, runs the solve stage on the device,
 * and downloads every written column.  Replaces src/world.js:962-1032 (inertias .. restitution,
 * plus the drift half of store()).  Synchronous.
 */
int32_t bg_solve_step(bg_ctx* ctx, const bg_bodies* bodies, const bg_rows* rows, const bg_step* step);

/* The same three parts, separately.  bg_upload and bg_solve are asynchronous on the context's
 * stream; bg_download synchronises.  bg_solve may be called again after bg_restore without a new
 * upload: bg_upload keeps a pristine device copy of what it uploaded. */
int32_t bg_upload(bg_ctx* ctx, const bg_bodies* bodies, const bg_rows* rows);
int32_t bg_restore(bg_ctx* ctx);
int32_t bg_solve(bg_ctx* ctx, const bg_step* step);
int32_t bg_download(bg_ctx* ctx, const bg_bodies* bodies, const bg_rows* rows);

/* Batched worlds: one CTA per small world (or every world on the persistent grid), the same solve
 * stage, one launch for all.  bg_batch_solve_step moves a large batch in groups of whole worlds
 * (bg_set_batch_groups): each group is copied in while the one before it solves, and its results
 * copied back while the next solves.  A batch split so leaves nothing uploaded on the context
 * (bg_restore and bg_batch_solve then return BG_EINVAL until the next upload). */
int32_t bg_batch_solve_step(bg_ctx* ctx, const bg_bodies* bodies, const bg_rows* rows,
                            const bg_worlds* worlds, const bg_step* step);
int32_t bg_batch_upload(bg_ctx* ctx, const bg_bodies* bodies, const bg_rows* rows, const bg_worlds* worlds);
int32_t bg_batch_solve(bg_ctx* ctx, const bg_step* step);
int32_t bg_batch_download(bg_ctx* ctx, const bg_bodies* bodies, const bg_rows* rows);

/*
 * Page-locks the caller's own long-lived columns (cudaHostRegister), so that the copies of every
 * later call go straight between them and the device, with no gather through the library's
 * staging block.  A Bearing World keeps its columns in typed arrays that live until they grow
 * (src/world.js:228-311, src/contact.js:196-248); this is the call a World makes once, and again
 * after either grows.  Every non-NULL column of `bodies` is registered for bodies->capacity slots
 * (awake_list: capacity entries) and of `rows` for `row_capacity` rows (>= rows->count: the
 * columns' allocated length).  Columns that share pages are registered as one range.  A call
 * replaces the ranges this context registered before (waiting for its stream first); a range
 * that CUDA reports as registered already (by another context, say) is left to its owner.
 * bg_unregister_host releases them, as does bg_destroy.  Until then the memory must stay
 * allocated: free or move it only after either.  A column that a call's copy would read or write
 * past its registered range (rows grew past row_capacity) is staged as if never registered.
 * Results never depend on it.
 */
int32_t bg_register_host(bg_ctx* ctx, const bg_bodies* bodies, const bg_rows* rows, int32_t row_capacity);
int32_t bg_unregister_host(bg_ctx* ctx);
/* Bytes this context holds page-locked by bg_register_host (0 if none). */
int64_t bg_registered_bytes(const bg_ctx* ctx);

/* The context's CUDA stream (a cudaStream_t), for callers that time or order work on it. */
void* bg_stream(bg_ctx* ctx);
/* Kernel launches issued since the last bg_upload / bg_restore (for launch accounting). */
int32_t bg_last_launches(const bg_ctx* ctx);
/* Device time, in milliseconds, of the last solve-stage kernel (CUDA events recorded around it
 * on the context's stream); synchronises.  Negative if none has run. */
double bg_last_stage_ms(bg_ctx* ctx);
/* Grid barriers each colour pass waits at, and the spin budget (iterations) of each wait.
 * 0 restores the default.  A wait past its budget makes the step return BG_ETIMEOUT. */
int32_t bg_set_wait_budget(bg_ctx* ctx, int64_t iterations);
/* How batched solves run (no counterpart in the reference: a Bearing World steps alone): one CTA of
 * 32, 64, 128 or 256 threads a world, or BG_BATCH_ON_GRID, every world on the persistent grid as
 * one flow.  0 (the default) tunes it on the next bg_batch_solve / bg_batch_solve_step: each
 * candidate solves the uploaded batch once, timed, from the same input, and the fastest is kept
 * for the context's later batched solves.  Results never depend on it. */
#define BG_BATCH_ON_GRID 1
int32_t bg_set_block_threads(bg_ctx* ctx, int32_t threads);
/* What batched solves use now (0 until tuned). */
int32_t bg_block_threads(const bg_ctx* ctx);
/* How many groups of whole worlds bg_batch_solve_step splits a batch into, 1 to
 * BG_MAX_BATCH_GROUPS (1: never split), or 0 (the default): one group per 131,072 rows when the
 * row columns are in page-locked memory, per 262,144 rows otherwise, and a smaller batch unsplit.
 * A group never holds less than one world.  Results never depend on it. */
#define BG_MAX_BATCH_GROUPS 8
int32_t bg_set_batch_groups(bg_ctx* ctx, int32_t groups);

/*
 * The adjoint of the solve stage: Bearing itself has no derivatives; this is the backward pass a
 * differentiable World takes through src/world.js:962-1032.  Given a step's input (the same
 * structures bg_solve_step takes, for one world or, with `worlds`, a batch) and the adjoints of a
 * loss with respect to the step's results, it computes the adjoints with respect to the step's
 * input.  It recomputes the step on the device, recording what each pass read, then sweeps the
 * passes in reverse, replaying each row and body from its record: the derivative is the one of the
 * step's own active set (the points each block LCP pushed, the friction cone's Newton rounds, the
 * clamps that held, the branches of tumble and untwist), so it equals a finite difference wherever
 * no decision of the step changes.  The recomputed results are written into the step's written
 * columns as bg_solve_step writes them.
 *
 * Results (adjoints of a loss) have the layout of the columns they belong to.  Body seeds and
 * results: position 3, rotation 4, velocity 3, angular 3, tumbled 3, ceiling 1 per slot; bodies
 * that do not move (inverse mass 0) are constants of the step, and their results are 0.  Row seeds
 * (the step's results): normal_impulse 4, tangent_impulse1/2, roll_impulse1/2, spin_impulse,
 * drift1/2 per row.  Row results (the step's input): the same impulses and drift as carried in,
 * and normal 3, t1 3, t2 3, friction 1, restitution 1, separation 4, point 12 per row.
 * Scope: dynamic and static boxes, spheres and capsules, without locks, freezing or joints; other
 * worlds return BG_EUNSUPPORTED.  Synchronous.
 */
typedef struct bg_body_grads {
  double* position;
  double* rotation;
  double* velocity;
  double* angular;
  double* tumbled;
  double* ceiling;
} bg_body_grads;

typedef struct bg_row_grads {
  double* normal_impulse;
  double* tangent_impulse1;
  double* tangent_impulse2;
  double* roll_impulse1;
  double* roll_impulse2;
  double* spin_impulse;
  double* drift1;
  double* drift2;
  double* normal;              /* results only */
  double* t1;
  double* t2;
  double* friction;
  double* restitution;
  double* separation;
  double* point;
} bg_row_grads;

int32_t bg_backward(bg_ctx* ctx, const bg_bodies* bodies, const bg_rows* rows, const bg_worlds* worlds,
                    const bg_step* step, const bg_body_grads* body_seed, const bg_row_grads* row_seed,
                    bg_body_grads* body_grad, bg_row_grads* row_grad);
/* The most tape nodes one replay of the last bg_backward recorded (each thread's tape holds
 * BG_TAPE_NODES), and the device time in milliseconds of its kernel. */
#define BG_TAPE_NODES 4096
int32_t bg_backward_tape_peak(const bg_ctx* ctx);
double bg_backward_ms(bg_ctx* ctx);
/* The bytes the last bg_backward's kernel moves by its design (records written by the recompute
 * and read by the replays, each replay's prepared terms and the adjoints it reads and writes):
 * the numerator of its roofline. */
int64_t bg_backward_bytes(const bg_ctx* ctx);

/*
 * The solve stage without allocating: no counterpart in the reference.
 *
 * For callers that may not allocate device memory themselves: a host runtime (a game engine's,
 * or a JavaScript embedding's) that keeps every device buffer in a pool of its own and hands
 * this library only pointers into it, or a per-frame loop that cannot afford the device-wide
 * synchronisation a cudaMalloc may bring.  The caller passes the same structures as
 * bg_solve_step, but every array they point to is DEVICE memory the caller owns; the written
 * columns are written back into those arrays.  The stage runs in one CTA on `stream` (a
 * cudaStream_t; NULL for the default stream) and the call returns when it is done.
 *
 * Its working memory is one fixed device array inside this library, of about 4 MiB, which every
 * GPU that loads the library holds until the process exits; so a world may have at most
 * BG_STATIC_MAX_BODIES slots and BG_STATIC_MAX_ROWS rows, and larger ones are refused with
 * BG_EINVAL (use bg_solve_step for those).  The first call on a device looks up that array's
 * device address with the device current, in the device's primary context (the CUDA runtime's
 * own), and keeps it for later calls on that device; do not call this again on a device after
 * cudaDeviceReset.  All calls share the one array: calls that overlap on the GPU (other streams,
 * other host threads) race, so run them one after another.  Each call synchronises `stream`
 * before it returns (it reads the kernel's status back), so no call can be captured into a CUDA
 * graph.  It calls no cudaMalloc or cudaFree.
 * The counts and colour starts are checked on the host as bg_solve_step checks them; the index
 * columns (device memory) are checked by the kernel before it writes anything.  Either refusal
 * returns BG_EINVAL and leaves the caller's arrays untouched.  Otherwise it returns BG_OK,
 * BG_ECUDA, or BG_ETIMEOUT as bg_solve_step does; there is no context, so no bg_last_error text.
 */
#define BG_STATIC_MAX_BODIES 512
#define BG_STATIC_MAX_ROWS 2048
int32_t bg_solve_step_static(const bg_bodies* bodies, const bg_rows* rows, const bg_step* step, void* stream);

/*
 * The narrowphase on the device, for spheres, capsules and boxes: what src/contact.js narrow()
 * asks of src/collide.js collide(a, b, margin, tolerance) for each pair whose boxes meet
 * (src/contact.js:296-368, src/collide.js:204-1229), one pair a thread.  Each pair's manifold has
 * the reference's normal (from a to b), points, separations and feature ids, bit for bit; a pair
 * that does not touch has 0 points.  Entries past a pair's point count are 0.
 * Reads bodies' capacity, position, rotation, dims, shape, type and gravity_scale (the rest may be
 * NULL); a body's axes are worked out from its rotation as src/core/math.js:222-227 does, and its
 * weight (the direction reducePoints() leans on, src/collide.js:1151-1178) is gravity times its
 * gravity scale for a dynamic body, 0 otherwise.  Synchronous.
 */
typedef struct bg_pairs {
  int32_t count;
  const int32_t* a;            /* each pair's slots, as narrow() hands them to collide() */
  const int32_t* b;
  const double* margin;        /* motion[a] + motion[b] + tolerance (src/contact.js:351) */
  const double* tolerance;     /* min(size[a], size[b]) * PIXEL (src/contact.js:316) */
} bg_pairs;

typedef struct bg_manifolds {
  uint8_t* points;             /* 0..BG_POINTS per pair */
  double* normal;              /* 3 per pair */
  double* point;               /* 3 * BG_POINTS per pair */
  double* separation;          /* BG_POINTS per pair */
  uint32_t* pid;               /* BG_POINTS per pair */
} bg_manifolds;

int32_t bg_collide(bg_ctx* ctx, const bg_bodies* bodies, const double* gravity, const bg_pairs* pairs,
                   bg_manifolds* out);
/* Device time in milliseconds of the last bg_collide's kernel (synchronises; negative if none). */
double bg_last_collide_ms(bg_ctx* ctx);

/*
 * The constraint-graph colouring on the device (src/graph.js:105-214), exactly: colour() gives each
 * manifold the lowest colour none of the manifolds found before it on its moving bodies holds
 * (OVERFLOW when all 32 are held, RESTING between frozen or static bodies), and arrange()'s row
 * order puts them colour by colour, each colour's by b's slot, ties in found order.
 * In: bodies' capacity, type and frozen (the rest may be NULL); the step's `count` manifolds in the
 * order narrow() found them, a[f] and b[f] (slots).  Out: colour[f]; order[o], the found index of
 * the manifold row o holds (c.order); starts[BG_STARTS] (Contacts.starts); *solved, the rows
 * before the resting run.  Synchronous; a wait past its budget returns BG_ETIMEOUT.
 */
int32_t bg_colour(bg_ctx* ctx, const bg_bodies* bodies, int32_t count, const int32_t* a, const int32_t* b,
                  int32_t* colour, int32_t* order, int32_t* starts, int32_t* solved);
/* Device time in milliseconds of the last bg_colour's kernels (synchronises; negative if none). */
double bg_last_colour_ms(bg_ctx* ctx);

/*
 * A step's contacts on the device, from the pair list to the stored contact memory.  For each pair
 * of the list the narrowphase (as bg_collide); for each pair that touches, a row, emitted, given its
 * tangent basis and warm-started from the pair's remembered contact (src/contact.js:889-921 emit,
 * 1283-1292 basis, 999-1036 carry); the rows coloured and ordered (src/graph.js:105-214, as
 * bg_colour) and the resting ones set aside (src/contact.js:1318-1329 rest); the solve stage (as
 * bg_solve_step); then each solved row's impulses stored into its pair's memory (src/contact.js:
 * 1067-1115 store/keep) and each pair's touching flag (2178-2213).  Replaces src/contact.js
 * narrow()'s find/emit/carry (296-368), colour/arrange, the solve stage (src/world.js:962-1032)
 * and store/touched.  The rows never leave the device: the bodies and the pair list go to it, the
 * bodies' written columns (as bg_solve_step writes them) and each pair's point count and touching
 * flag come back.  bodies: every column bg_solve_step reads, and those bg_collide reads.  gravity
 * is step->gravity.  Synchronous.
 *
 * The contact memory (src/pairs.js:50-58: a pair's remembered point ids and normal impulses, and its
 * friction, twist and slip) lives in the context, one record per pair of the last call's list.
 * pairs->memory[i] names pair i's record: its index in the list the previous bg_contact_step on this
 * context took, or -1 for a pair with nothing remembered (new, or forgotten since).  Each call
 * leaves one record per pair of its own list for the next: what store() keeps of a solved row, the
 * record the pair had for a resting row (store() skips those), nothing for a pair apart.
 * Refused with BG_EINVAL before anything is copied: a pair's slot out of range or both slots
 * equal, a shape that is not a box, sphere or capsule, a memory index outside [-1, records),
 * an awake entry out of range.
 */
typedef struct bg_materials {
  const double* friction;      /* per slot: World._friction */
  const double* restitution;   /* per slot: World._restitution */
  const double* size;          /* per slot: World._size (a row's patch, src/contact.js:906) */
  const double* reach;         /* per slot: World._reach (read only with reuse on) */
} bg_materials;

typedef struct bg_contact_pairs {
  bg_pairs list;               /* the pairs whose boxes meet, in pair order (src/contact.js:312-327) */
  const int32_t* memory;       /* per pair: its record in the previous call's list, or -1 */
  int32_t reuse;               /* nonzero: a pair whose record keeps a manifold reuses it while
                                  the bodies barely move (src/contact.js:388-595 reused/keeps) and
                                  a fresh manifold is kept (remember); records hold the manifolds */
} bg_contact_pairs;

typedef struct bg_contact_result {
  uint8_t* points;             /* per pair, or NULL: its manifold's point count (0: apart) */
  uint8_t* touching;           /* per pair, or NULL: touched()'s flag (0 for a pair apart) */
  int32_t rows;                /* Contacts.count */
  int32_t solved;              /* rows before the resting run */
  int32_t points_solved;       /* contact points of the solved rows */
  int32_t starts[BG_STARTS];   /* Contacts.starts */
} bg_contact_result;

int32_t bg_contact_step(bg_ctx* ctx, const bg_bodies* bodies, const bg_materials* materials,
                        const bg_contact_pairs* pairs, const bg_step* step, bg_contact_result* out);
/* Device time in milliseconds of the last bg_contact_step's parts (synchronises): ms[0] the
 * narrowphase, ms[1] rows, colours and order, ms[2] the solve stage, ms[3] store and touched.
 * BG_EINVAL if there was none. */
int32_t bg_last_contact_ms(bg_ctx* ctx, double* ms);
/* Records the context holds for the next bg_contact_step (the last call's list length). */
int32_t bg_contact_records(const bg_ctx* ctx);
/* Forgets every record: the next call's memory entries must all be -1. */
int32_t bg_contact_forget(bg_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* BEARING_GPU_H */
