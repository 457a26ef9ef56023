/*
 * bearing_world.h - the host side of World.step, around the solve stage (libbearing_host.so).
 *
 * Bearing's World (src/world.js) runs its broadphase, narrowphase and colouring on the CPU and
 * hands the solve stage (src/world.js:962-1032) to whatever runs it.  This library is that
 * host side for worlds of boxes, spheres and capsules: bodies by slot as World keeps them,
 * fat-box pair finding, the pair list with its warm-start memory (src/pairs.js), the
 * narrowphase (src/collide.js), emit/carry (src/contact.js:889-1036), the colouring and row
 * layout (src/graph.js:105-214), then store/keep (src/contact.js:1067-1115) and the transforms
 * (src/world.js:1040-1057) after the solve.  The solve stage itself is a pluggable function
 * with the signature of bg_solve_step (bearing_gpu.h): the GPU library, or any other.
 *
 * Not covered (a world using them is refused): hulls, compounds, meshes, heightfields, joints,
 * characters, sensors, sleeping islands and the time-of-impact sweep.  The contact-reuse cache
 * (src/contact.js:388-595) is an option (bw_options.reuse), off by default.
 */
#ifndef BEARING_WORLD_H
#define BEARING_WORLD_H

#include <stdint.h>

#include "bearing_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bw_world bw_world;

/* World options (src/world.js:82, 314-395): gravity, substeps. */
typedef struct bw_options {
  double gravity[3];
  int32_t substeps;
  int32_t reuse;               /* nonzero: keep touching pairs' manifolds and reuse them while the
                                  bodies barely move against each other (src/contact.js:388-595) */
} bw_options;

/* addBody's spec for a box, sphere or capsule (src/world.js:190-221 defaults). */
typedef struct bw_body {
  int32_t type;          /* BG_DYNAMIC or BG_STATIC (kinematic: 2) */
  int32_t shape;         /* BG_BOX, BG_SPHERE, BG_CAPSULE */
  double size[3];        /* box */
  double radius;         /* sphere, capsule */
  double height;         /* capsule, caps included */
  double density;        /* kg/m^3, used unless mass > 0 */
  double mass;           /* kg, 0: from density */
  double friction;
  double restitution;
  double damping;
  double angular_damping;
  double gravity_scale;
  double position[3];
  double rotation[4];    /* x y z w, normalised on the way in (src/core/check.js:106-117) */
  double velocity[3];
  double angular[3];
} bw_body;

/* The solve stage the world calls each step: bg_solve_step's signature with a user pointer. */
typedef int32_t (*bw_solver)(void* user, const bg_bodies* bodies, const bg_rows* rows, const bg_step* step);

/* Counters of the last step (for benchmarks and tests). */
typedef struct bw_stats {
  int32_t bodies;        /* slots in use */
  int32_t awake;
  int32_t pairs;
  int32_t rows;          /* manifolds (Contacts.count) */
  int32_t solved;        /* rows before the resting run */
  int32_t points;        /* contact points over the solved rows */
  int32_t colours;       /* colours used (non-empty), overflow excluded */
  int32_t overflow;      /* rows in the overflow colour */
  int64_t step;          /* steps taken */
} bw_stats;

bw_world* bw_create(const bw_options* options);
void bw_destroy(bw_world* world);
const char* bw_last_error(const bw_world* world);

/* Adds a body; returns its slot, or a negative BG_E* code. */
int32_t bw_add_body(bw_world* world, const bw_body* body);

/* World.workers (src/world.js:501-524): how many threads besides the caller's the step's host side
 * may use for its walk over the pairs when their boxes meet on another device; -1,
 * the reference's 'auto' and the default, is the machine's cores up to 16.  Results are the same
 * bits whatever it is.  BG_EINVAL below -1. */
int32_t bw_set_workers(bw_world* world, int32_t workers);

/* The solve stage to call; NULL restores none (bw_step then fails with BG_EUNSUPPORTED). */
int32_t bw_set_solver(bw_world* world, bw_solver solver, void* user);

/* The narrowphase on another device: fn (bg_collide's signature, with `user` for its context) is
 * handed each step's pairs whose boxes meet and returns their manifolds, which the step then
 * emits and carries as it would its own (src/contact.js:312-327).  NULL (the default) runs the
 * host's own.  The rows, their order and the pairs' memory are the same either way. */
typedef int32_t (*bw_narrowphase)(void* user, const bg_bodies* bodies, const double* gravity, const bg_pairs* pairs,
                                  bg_manifolds* out);
int32_t bw_set_narrowphase(bw_world* world, bw_narrowphase fn, void* user);

/* The whole contact side of a step on another device: fn (bg_contact_step's signature, with `user`
 * for its context) is handed the bodies, their materials and the step's pairs whose boxes meet, with
 * each pair's contact record from the previous call, and runs the narrowphase, the rows, colouring,
 * the solve stage and store() there (src/contact.js:296-368, 889-1115, 2178-2213; src/graph.js:
 * 105-214; src/world.js:962-1032).  The host keeps the pair list (src/pairs.js) and forgets the
 * pairs fn reports apart.  The step's rows then never reach the host: bw_rows_view shows none, and
 * bw_begin_step is refused.  Set it before the first step (BG_EINVAL after); NULL (the default)
 * keeps the host's rows and bw_set_solver's solve stage. */
typedef int32_t (*bw_contact_solver)(void* user, const bg_bodies* bodies, const bg_materials* materials,
                                     const bg_contact_pairs* pairs, const bg_step* step, bg_contact_result* out);
int32_t bw_set_contact_step(bw_world* world, bw_contact_solver fn, void* user);

/* A whole World.step(dt): bw_begin_step, the solver, bw_end_step. */
int32_t bw_step(bw_world* world, double dt);

/* The step up to the solve stage: bounds, pairs, narrowphase, emit/carry, colour, rest.
 * After it, bw_bodies_view / bw_rows_view describe the solve stage's input. */
int32_t bw_begin_step(bw_world* world, double dt);
/* The step after the solve stage: store/keep, touching, transforms. */
int32_t bw_end_step(bw_world* world);

/* Views of the world's own columns (valid until the next bw_* call that changes sizes). */
int32_t bw_bodies_view(bw_world* world, bg_bodies* out);
int32_t bw_rows_view(bw_world* world, bg_rows* out);
int32_t bw_step_params(const bw_world* world, bg_step* out);

/*
 * Many worlds stepped together (no reference counterpart: a Bearing World steps alone).  The
 * batch does each world's host side on `threads` CPU threads, then lays every world's solve-stage
 * input end to end, as bg_batch_solve_step (bearing_gpu.h) takes it; bw_batch_end_step hands each
 * world its part of the result back and finishes its step.  The worlds stay owned by the caller.
 */
typedef struct bw_batch bw_batch;
bw_batch* bw_batch_create(bw_world* const* worlds, int32_t count);
void bw_batch_destroy(bw_batch* batch);
int32_t bw_batch_begin_step(bw_batch* batch, double dt, int32_t threads);
int32_t bw_batch_views(bw_batch* batch, bg_bodies* bodies, bg_rows* rows, bg_worlds* worlds, bg_step* step);
int32_t bw_batch_end_step(bw_batch* batch, int32_t threads);

/*
 * What the host side of a step knows of each row beyond the solve stage's columns: for the
 * adjoint's replay of the row's narrowphase, emit, basis and carry (src/contact.js:889-1036), and
 * for the tests' checker, which recomputes them.  Filled after bw_begin_step, per row in the rows'
 * (colour) order; the row's pair is rows.a / rows.b.
 */
typedef struct bw_row_memory {
  uint32_t* pid;          /* 4 per row: each point's feature id (Contacts.pid) */
  double* margin;         /* 1 per row: the narrowphase margin, motion[a] + motion[b] + tolerance */
  uint8_t* remembered;    /* 1 per row: points the pair remembered from the last step (0: none carried) */
  uint32_t* memory_pid;   /* 4 per row: those points' feature ids */
  double* memory;         /* BW_MEMORY per row: normalImpulse[4], friction[3], twist[3], slip[3], 3 unused */
} bw_row_memory;
#define BW_MEMORY 16
int32_t bw_row_memory_get(const bw_world* world, bw_row_memory* out);
/* The same for a batch after bw_batch_begin_step, rows end to end as bw_batch_views lays them. */
int32_t bw_batch_row_memory(const bw_batch* batch, bw_row_memory* out);

/* The pairs the last bw_begin_step's narrowphase handed to collide() (src/contact.js:351-356:
 * those whose boxes met), in the order it took them, with the margin and tolerance it passed:
 * views into the world's own arrays, valid until its next step.  bw_collide_pairs runs the host's
 * narrowphase (the one the step itself uses) over any such list, with the bodies' current poses:
 * what bg_collide does on the device. */
int32_t bw_narrow_pairs(const bw_world* world, bg_pairs* out);
/* The host's colouring (src/graph.js:105-170, what each step's colour() runs) over any list of
 * manifolds in found order: bg_colour's arguments and results, on the CPU. */
int32_t bw_colour_rows(const bg_bodies* bodies, int32_t count, const int32_t* a, const int32_t* b, int32_t* colour,
                       int32_t* order, int32_t* starts, int32_t* solved);
int32_t bw_collide_pairs(const bg_bodies* bodies, const double* gravity, const bg_pairs* pairs, bg_manifolds* out,
                         int32_t threads);

/* A deep copy of a world (its bodies, pairs with their memory, broadphase and step count), for
 * checkpoints; bw_destroy frees it.  NULL if out of memory.  bw_copy makes dst a copy of src. */
bw_world* bw_clone(const bw_world* world);
int32_t bw_copy(bw_world* dst, const bw_world* src);

/*
 * The host side's share of a step's adjoint (bg_backward, bearing_gpu.h, is the solve stage's),
 * for one world or, with `worlds`, a batch laid out as bw_batch_views lays it.  Both run after the
 * step's bw_begin_step state is known again (the rows, and the bw_row_memory of that step).
 *
 * bw_keep_backward: the reverse of keep() (src/contact.js:1091-1115).  From the adjoints of what
 * each solved row left in its pair's memory (memory_grad, BW_MEMORY per row: normalImpulse[4],
 * friction[3], twist[3], slip[3]) to those of the row's results: it writes row_grad's impulses
 * and drift (the seeds bg_backward takes) and adds to row_grad's normal, t1 and t2.
 *
 * bw_narrow_backward: the reverse of each row's narrowphase (src/collide.js, for spheres, capsules
 * and boxes), emit (src/contact.js:889-921), basis (1283-1292) and carry (999-1036).  From the
 * adjoints of the rows' input (row_grad, as bg_backward leaves them) it adds those of each body's
 * position (3) and rotation (4) into position_grad / rotation_grad (moving bodies only), those of
 * each body's friction and restitution (World._friction / _restitution, given per slot in
 * `friction` / `restitution`) into friction_grad / restitution_grad, and writes those of the
 * memory each row carried in into memory_grad (BW_MEMORY per row; 0 where nothing was carried).
 * Returns BG_EFAULT if a row's replayed narrowphase does not find the rows' own points (the step
 * is not the one the rows came from).  `threads`: host threads over whole worlds.
 */
int32_t bw_keep_backward(const bg_rows* rows, const bg_worlds* worlds, const double* memory_grad, bg_row_grads* row_grad);
int32_t bw_narrow_backward(const bg_bodies* bodies, const bg_rows* rows, const bg_worlds* worlds,
                           const bw_row_memory* memory, const double* gravity, const double* friction,
                           const double* restitution, const bg_row_grads* row_grad, double* position_grad,
                           double* rotation_grad, double* friction_grad, double* restitution_grad, double* memory_grad,
                           int32_t threads);

/* Each slot's friction and restitution (World._friction, _restitution: what emit() mixes per
 * pair), copied into arrays of bw_stats.bodies entries. */
int32_t bw_materials(const bw_world* world, double* friction, double* restitution);

/* World.transforms: 7 floats per slot (position, rotation x y z w). */
const float* bw_transforms(const bw_world* world);
int32_t bw_stats_get(const bw_world* world, bw_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* BEARING_WORLD_H */
