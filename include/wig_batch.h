/*
 * wig_batch.h — C ABI of a batch of liquid worlds stepped together
 * (worldinagrain_b200).
 *
 * No counterpart in the reference, whose Simulation holds one world.  A
 * batch holds many independent worlds of any sizes, each in the reference's
 * buffer layouts (include/wig_fluid.h), in one packed device allocation; a
 * step of any subset of them runs each of the liquid's passes as ONE launch
 * over all the listed worlds (work lists written on the device), the CG
 * iterations in one CUDA-graph WHILE loop that runs while any world has not
 * converged.  A world's results are bit-for-bit those of stepping it alone
 * (wig_fluid_step's fast form): no arithmetic depends on its neighbours in
 * the batch.
 *
 * Lanes: a batch has WIG_BATCH_LANES independent step lanes, each with its
 * own work lists and graphs, so two steps of disjoint subsets may be in
 * flight at once on two streams (a serving loop admits new requests into
 * one lane while the other runs).  A world must not be in two steps in
 * flight at once.
 *
 * Same error convention as wig_fluid.h: 0 or a negative WIG_E_*, and
 * wig_fluid_last_error() for the message.
 */
#ifndef WIG_BATCH_H
#define WIG_BATCH_H

#include "wig_fluid.h"

#ifdef __cplusplus
extern "C" {
#endif

#define WIG_BATCH_LANES 2u
#define WIG_BATCH_MAX_WORLDS 65536u

typedef struct wig_batch wig_batch;

/* Device bytes one world of shape d holds in a batch (its seven buffers and
 * the fast form's scratch), for admission under a memory budget. */
int wig_batch_world_bytes(const wig_world_desc* d, uint64_t* out);

/* Creates a batch of n worlds (descs[n]) on the current CUDA device with
 * element table elems[n_elems]; every world's buffers zeroed. */
int wig_batch_create(const wig_world_desc* descs, uint32_t n, const wig_elem* elems, uint32_t n_elems,
                     wig_batch** out);

uint32_t wig_batch_worlds(const wig_batch* b);
int wig_batch_layout(const wig_batch* b, uint32_t world, wig_world_layout* out);
int wig_batch_buffers_of(wig_batch* b, uint32_t world, wig_fluid_buffers* out);

/* Host <-> device copies of one world's buffer (which as in
 * wig_fluid_upload), complete on return. */
int wig_batch_upload(wig_batch* b, uint32_t world, int which, const void* host, uint64_t offset, uint64_t bytes,
                     void* stream);
int wig_batch_download(wig_batch* b, uint32_t world, int which, void* host, uint64_t offset, uint64_t bytes,
                       void* stream);

/* One liquid step of the `count` distinct worlds listed, on lane `lane`,
 * asynchronous on `stream`: P[i] is worlds[i]'s Params; world_flags[i] (or
 * 0 for all when null) its own WIG_STEP_BOOKKEEPING_ONLY, WIG_STEP_VISCOUS,
 * WIG_STEP_SHIFTED_SET / _FIRST; flags (WIG_STEP_TOLERANCE,
 * WIG_STEP_F64_DOTS, WIG_STEP_SYNC_STATS), max_cycles (<= 64) and tolerance
 * apply to all.  The fast form only (no WIG_STEP_PLAIN / _PERSISTENT). */
int wig_batch_step(wig_batch* b, uint32_t lane, const uint32_t* worlds, uint32_t count, const wig_params* P,
                   const uint32_t* world_flags, uint32_t max_cycles, uint32_t flags, double tolerance, void* stream);

/* The listed worlds' statistics from their last steps (waits for the
 * streams those steps ran on).  launches: the kernels of that batch step. */
int wig_batch_read_stats(wig_batch* b, const uint32_t* worlds, uint32_t count, wig_fluid_stats* out);

/* One step as wig_batch_step, launched pass by pass with CUDA events around
 * each launch; ms_out / calls_out as in wig_fluid_step_profile.
 * Synchronous. */
int wig_batch_step_profile(wig_batch* b, uint32_t lane, const uint32_t* worlds, uint32_t count, const wig_params* P,
                           const uint32_t* world_flags, uint32_t max_cycles, uint32_t flags, double tolerance,
                           void* stream, float* ms_out, uint32_t* calls_out);

void wig_batch_destroy(wig_batch* b);

/* Serving: a batch whose worlds hold no device memory until admitted.
 * wig_batch_admit allocates one world's memory (zeroed; the host uploads
 * its state after) from the device's stream-ordered pool; wig_batch_evict
 * returns it (download the state first; the world's step counter and tiling
 * parity carry on when it is admitted again).  Only admitted worlds step.
 * wig_batch_resident_bytes: the admitted worlds' bytes. */
int wig_batch_create_deferred(const wig_world_desc* descs, uint32_t n, const wig_elem* elems, uint32_t n_elems,
                              wig_batch** out);
int wig_batch_admit(wig_batch* b, uint32_t world, void* stream);
int wig_batch_evict(wig_batch* b, uint32_t world, void* stream);
uint64_t wig_batch_resident_bytes(const wig_batch* b);

/* Pooled serving: each lane gets a pool of `bytes` that lends every world
 * of a step on that lane its per-step memory (its `parts` particle buffer,
 * which the step refills, its `cg` buffer, which the step writes before any
 * pass reads it, and the fast form's scratch); an admitted world then holds
 * only its persistent buffers, `field` without its coarse levels (copies of
 * field stop there; copies of parts and cg are refused).  Set both lanes'
 * pools before admitting any world.  A step whose worlds' per-step memory
 * exceeds the lane's pool is refused (WIG_E_OOM).
 * wig_batch_world_bytes_split gives a world's persistent and per-step bytes. */
int wig_batch_set_lane_pool(wig_batch* b, uint32_t lane, uint64_t bytes);
int wig_batch_world_bytes_split(const wig_world_desc* d, uint64_t* persistent, uint64_t* transient);

/* Launch shapes of the fast form, none of which changes a result bit of
 * the FP32 forms (every kernel's arithmetic and order are the same whichever
 * CTA does a unit; in the mixed form COARSE_CELLS also decides which levels
 * stay FP32 on chip rather than stored in 16 bits): what an autotuner may
 * choose per batch.
 *   COARSE_CELLS: the one-CTA coarse kernel takes a world's levels from its
 *     first level of at most this many cells (1 .. 4096; a world with no
 *     such level above its coarsest: from the coarsest), the tile kernels
 *     the levels above it: the depth of the V-cycle's on-chip part.  A
 *     batch of one world takes up to 16384: from a level of more than 4096
 *     cells its coarse levels run on a cluster of 8 CTAs (WIG_E_ARG when
 *     they do not fit its shared memory);
 *   LEVEL_PER_SM, CG_PER_SM, RELAX_PER_SM: CTAs a multiprocessor (1 .. 64)
 *     of the level tile kernels, of the three CG kernels, of the fine
 *     relaxation.
 * Defaults: COARSE_CELLS 4096, LEVEL_PER_SM 8, CG_PER_SM 8, RELAX_PER_SM 16;
 * for a batch of one world, as every wig_fluid handle is: COARSE_CELLS 2048,
 * LEVEL_PER_SM 32, CG_PER_SM 4, RELAX_PER_SM 64.
 * No step of the batch may be in flight; the lanes' graphs are recaptured
 * at their next step. */
enum wig_launch_knob {
    WIG_LAUNCH_COARSE_CELLS = 0,
    WIG_LAUNCH_LEVEL_PER_SM = 1,
    WIG_LAUNCH_CG_PER_SM = 2,
    WIG_LAUNCH_RELAX_PER_SM = 3,
    WIG_LAUNCH_KNOBS = 4
};
int wig_batch_set_launch(wig_batch* b, uint32_t knob, uint32_t value);
int wig_batch_get_launch(const wig_batch* b, uint32_t knob, uint32_t* value);

#ifdef __cplusplus
}
#endif

#endif /* WIG_BATCH_H */
