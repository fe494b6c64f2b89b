/* kratos_b200 -- C ABI of the B200 (sm_100a) hydro / ideal-MHD step.
 *
 * The library replaces the device side of Kratos's dynamics module: the
 * per-stage `integrate` driver that dynamics::base_t::enroll builds
 * (src/modules/dynamics/dynamics.h:51-103), run once per RK stage by
 * dynamics::base_t::step (src/modules/dynamics/dynamics.cpp:37-42), together
 * with the policy kernels it launches:
 *   cons2prim + CFL dt       hydro/eos/adiabatic.h:211-258, mhd/eos/adiabatic.h:127-234
 *   ghost fill (same level)  hydro/boundary/comm_functions.h:306-483,
 *                            mhd/boundary/comm_functions.h:433-815
 *   level jumps (hydro SMR)  hydro/boundary/comm_functions.h:329-505,
 *                            hydro/integrator/integrator.h:343-382
 *   PLM + HLLC / HLLD flux   prototypes/integrator.h:14-32 flux_kernel,
 *                            hydro/reconstruct/plm.h, hydro/riemann/hllc.h,
 *                            mhd/riemann/hlld.h
 *   RK2 conserved update     hydro/integrator/integrator.h:241-265,
 *                            hydro/integrator/rk2.h:20-41
 *   CT edge EMF + face B     mhd/integrator/integrator.h:191-462, mhd/integrator/rk2.h:20-63
 *   dt reduction             mesh/cycle/cycle.cpp:77-115
 * The host side (mesh, parameter files, snapshots, problem generators) calls
 * it with plain pointers; no torch or CUDA types cross this boundary.
 *
 * Conventions
 *   - Blocks: a uniform mesh of nb[0] x nb[1] x nb[2] blocks of n[0] x n[1] x
 *     n[2] cells, numbered lexicographically (x fastest); a statically refined
 *     mesh (kr_ctx_create_refined) numbers its blocks level by level.
 *     A sharded context (n_ranks > 1, below) holds a subset of them.
 *   - Host state arrays use the reference's per-block layouts (dat_3d_t,
 *     src/mesh/types/dat_3d.h:153-156, field index fastest), blocks in
 *     ascending global id:
 *       u  : [block][n2][n1][n0][nw]   nw = 5 (hydro) or 8 (MHD), no ghosts
 *       bf : [block][n2+5][n1+5][n0+5][3]  face B on the (n+1)^3 lattice with
 *            2 ghost layers (as the snapshot's field_bf_field)
 *   - Return codes: 0 success, negative on error; kr_last_error() describes
 *     the last error of a context (or of kr_ctx_create when ctx is NULL).
 *   - Threading: one host thread per context; one context per GPU.
 */
#ifndef KRATOS_B200_H
#define KRATOS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KR_ABI_VERSION 7

/* [boundary] kinds per side (hydro/boundary/phys_functors.h:11-91): an axis is
 * periodic only when both its sides are KR_BC_PER. */
enum kr_bc_t
{
    KR_BC_PER  = 0,            /* periodic                                       */
    KR_BC_OUT  = 1,            /* outflow: zero gradient, inflow velocity clamped */
    KR_BC_REF  = 2,            /* reflect: mirror, normal velocity negated        */
    KR_BC_FRE  = 3,            /* free: zero gradient                             */
    KR_BC_FIXD = 4             /* fixed: ghosts = w_fix (the [init] medium)       */
};

/* Riemann solver selection ([b200] riemann). */
enum kr_riemann_t
{
    KR_RIEMANN_DEFAULT = 0,    /* HLLC (hydro) / HLLD (MHD), as the reference     */
    KR_RIEMANN_HLLE    = 1,    /* two-wave HLLE everywhere (MHD only)            */
    KR_RIEMANN_LEARNED = 2     /* MLP face selector: HLLE where predicted safe,  */
                               /* HLLD elsewhere (MHD only)                      */
};

/* Time integrator ([b200] integrator). */
enum kr_integrator_t
{
    KR_INTEGRATOR_RK2 = 0,     /* Heun / SSP-RK2, the reference's rk2_t:          */
                               /*   U* = U + dt L(U), U' = (U + U*) / 2 + dt/2 L(U*) */
    KR_INTEGRATOR_VL2 = 1      /* van Leer predictor-corrector with CT (Stone &   */
                               /*   Gardiner 2009, New Astron. 14, 139; no        */
                               /*   reference counterpart): U* = U + dt/2 L1(U)    */
                               /*   with donor-cell states, U' = U + dt L(U*)      */
};

/* Step configuration.  Physics keys mirror the reference's [dynamics] and
 * [cycle] parameters (prototypes/eos.h:43-56, cycle.cpp:30-65). */
typedef struct
{
    int    abi_version;        /* KR_ABI_VERSION                                 */
    int    mhd;                /* 0: hydro (PLM+HLLC), 1: ideal MHD (PLM+HLLD+CT) */
    int    precision;          /* 2: FP64 throughout; 1: FP32 reconstruction and */
                               /*    Riemann, FP64 state / CT update / dt / c2p  */
    int    riemann;            /* enum kr_riemann_t                              */
    int    nb[ 3 ];            /* blocks per axis                                */
    int    n [ 3 ];            /* cells per block per axis (each >= 4)           */
    double x_min[ 3 ], x_max[ 3 ];
    double gamma, cfl, rho_floor, tmp_floor;
    double dt_init;            /* [cycle] dt_init (0: unset)                     */
    double dt_expand;          /* [cycle] dt_expand                              */
    int    device;             /* CUDA device ordinal                            */
    int    bc[ 6 ];            /* enum kr_bc_t for x-, x+, y-, y+, z-, z+       */
    double w_fix[ 5 ];         /* KR_BC_FIXD primitive state: rho, p, v0..2       */
    double b_fix[ 3 ];         /* KR_BC_FIXD magnetic field (MHD): [init] b0      */
    int    flags;              /* KR_FLAG_* bits                                 */
    int    n_ranks;            /* ranks sharing the mesh (0 or 1: not sharded)   */
    int    rank;               /* this context's rank, 0 <= rank < n_ranks       */
    int    sel_period;         /* learned mode: the network runs at stage 0 of   */
                               /* every sel_period-th step; the other stages    */
                               /* reuse its per-face choices (0 or 1: every step)*/
    int    integrator;         /* enum kr_integrator_t                           */
    int    reserved[ 2 ];
} kr_cfg;

/* kr_cfg.flags (bit 0, value 1, is reserved and ignored) */
#define KR_FLAG_HALO_ALL 2     /* route every neighbour copy, same-rank ones     */
                               /* included, through the halo exchange            */
                               /* (verification of the pack / exchange / unpack) */
#define KR_FLAG_BOXES    4     /* MHD, one rank, periodic: the nb[0] blocks are  */
                               /* independent periodic boxes, each the unit cube */
                               /* of n cells with its own CFL dt and time        */
                               /* (kr_init_boxes, kr_box_times); nb[1] = nb[2] = 1 */
#define KR_FLAG_UNFUSED  8     /* MHD, uniform mesh: run stage 0's cell and CT   */
                               /* updates and stage 1's cons -> prim as three    */
                               /* launches instead of one fused launch (the same */
                               /* arithmetic; a check).  Fused by default in the */
                               /* FP64 step and in kr_batch launches; the FP32   */
                               /* step always runs the three launches            */

typedef struct kr_ctx kr_ctx;

/* Fill a configuration with the reference's defaults: gamma 1.66667, cfl 0.3,
 * floors 1e-9, dt_expand 2, FP64, default Riemann solver, unit cube. */
void        kr_cfg_default( kr_cfg * cfg );

kr_ctx *    kr_ctx_create ( const kr_cfg * cfg );
void        kr_ctx_destroy( kr_ctx * ctx );
const char* kr_last_error ( const kr_ctx * ctx );

/* Static mesh refinement (hydro, one rank) -------------------------------
 * A region is one [refine_region*] section of the parameter file
 * (meshgen.cpp:111-160 load_refinement): every level-`level` block holding a
 * point of the box x_min..x_max is created, together with its ancestors and
 * their neighbours, so adjacent blocks differ by at most one level
 * (tree.cpp:139-232 insert).  The context's blocks are the tree's leaves,
 * numbered level by level and lexicographically (x fastest) inside a level;
 * every block has n cells, a level-L block a cell size 2^-L of the root's.
 * Each stage fills the ghosts across a level jump (restriction of the fine
 * side, prolongation with minmod slopes of the coarse side,
 * hydro/boundary/comm_functions.h:329-447) and corrects the coarse cells
 * next to a refined side with the area-averaged fine flux
 * (comm_functions.h:469-505, hydro/integrator/integrator.h:343-382).
 * With no region of level >= 1 this is kr_ctx_create.  Host state arrays hold
 * the blocks in this order; kr_block_info gives each block's level and
 * logical position (reg[3 b + a], at its level) and returns the count. */
typedef struct
{
    int    level;
    double x_min[ 3 ], x_max[ 3 ];
} kr_region;

kr_ctx *    kr_ctx_create_refined( const kr_cfg * cfg, int n_regions, const kr_region * regions );
int         kr_block_info        ( kr_ctx * ctx, int * level, int * reg );

/* Optional: run on a caller-owned stream (a cudaStream_t passed as void*). */
int kr_set_stream( kr_ctx * ctx, void * stream );

/* Seeded workload initial state into the device state (host-built, uploaded):
 * "shock" (hydro), "ot" or "turb" (MHD; decaying supersonic turbulence). */
int kr_init_problem( kr_ctx * ctx, const char * name, uint64_t seed );

/* Batched independent boxes (no reference counterpart as one launch: the
 * reference runs each box as its own mesh).  kr_box_params: the parameters
 * of box `box` of a seeded batch (problems.h kr_box_params): out[0] edge
 * length in cells, out[1..7] rho, p, velocity amplitude, beta, B_x, B_y, B_z.
 * kr_init_boxes: block b of a KR_FLAG_BOXES context (or the one block of a
 * periodic one-block MHD context) becomes box box_ids[b]; every box must have
 * the context's edge length.  kr_box_times: each block's time, last dt and
 * steps (arrays of kr_block_info's count; null entries skipped). */
int kr_box_params( uint64_t seed, int box, double gamma, double * out8 );
int kr_init_boxes( kr_ctx * ctx, uint64_t seed, const int * box_ids );
int kr_box_times( kr_ctx * ctx, double * t, double * dt_last, long long * n_steps );

/* Host <-> device state transfers (layouts above).  bf is ignored for hydro.
 * kr_get_state writes the cell-centred face-averaged B into u's slots 5..7. */
int kr_set_state( kr_ctx * ctx, const double * u, const double * bf );
int kr_get_state( kr_ctx * ctx, double * u, double * bf );

/* Advance n_steps Heun steps on the device (enqueued; returns without waiting).
 * Time and dt stay on the device until kr_get_time. */
int kr_step( kr_ctx * ctx, int n_steps );

/* Wait for the context's stream; read time, last dt, next dt bound, steps. */
int kr_get_time( kr_ctx * ctx, double * t, double * dt_last, double * dt_bound,
                 long long * n_steps_done );
/* Set time and the dt bound the next step starts from (restart). */
int kr_set_time( kr_ctx * ctx, double t, double dt_bound );

/* Sticky device status word: 0 ok; bit 0 non-finite or non-positive dt; bit 1
 * a NaN velocity in the state (stage 0's cons -> prim; the density and
 * pressure floors heal NaN density and pressure, as the reference's do); bit 2
 * an exchange index outside its block's arrays on a refined MHD mesh (the
 * access was skipped). */
int kr_status( kr_ctx * ctx );

/* Number of kernel launches kr_step enqueues per step (instrumentation). */
int kr_launches_per_step( kr_ctx * ctx );

/* Run one step eagerly (outside the captured graph) with CUDA events around
 * every kernel and return the step's milliseconds per kernel kind in ms[0..6]:
 * c2p, ghost, flux z, flux y, flux x, emf, update (both stages summed; where
 * stage 0's update and stage 1's c2p are fused, they count as update).
 * The step advances the state like kr_step.  n_kinds must be >= 7. */
int kr_profile_step( kr_ctx * ctx, int n_kinds, double * ms );

/* Diagnostics on the device state: max |div B| over owned cells (MHD) and the
 * domain totals of mass, momentum and energy (5 doubles). */
int kr_diagnostics( kr_ctx * ctx, double * max_div_b, double * totals5 );

/* ---- Learned HLLE/HLLD face selector (MHD).  No reference counterpart: the
 * reference always solves HLLD (mhd/riemann/hlld.h).  A 16 -> 32 -> 32 -> 1 MLP
 * (ReLU) predicts per face whether the cheap HLLE flux is within tolerance of
 * HLLD; with riemann = KR_RIEMANN_LEARNED the flux sweep evaluates it with BF16
 * tensor-core MMAs (FP32 accumulate) at stage 0 of every sel_period-th step.
 * A face that only its own block computes uses HLLE when every such face of its
 * warp (32 consecutive faces of the sweep) has logit > threshold; a face that a
 * neighbouring block computes too (block sides, the edge EMFs' ghost lines)
 * uses HLLE when its own logit is > threshold, which every block holding it
 * evaluates identically, so every face gets one flux.  HLLD elsewhere; the
 * choice holds until the next evaluation.  Parameters: 1633 floats, W1[16][32],
 * b1[32], W2[32][32], b2[32], W3[32], b3, row-major [in][out]. */

/* Upload selector parameters and the logit threshold to a context. */
int kr_set_selector( kr_ctx * ctx, const float * params, float threshold );

/* Faces evaluated and faces given HLLE since the last reset
 * (learned mode; counted when the network runs). */
int kr_selector_stats( kr_ctx * ctx, long long * faces, long long * cheap, int reset );

/* Run n_steps ordinary steps while logging about one face in `stride` (per
 * axis, stage and step; seeded) as a training sample: out[k*17 + 0..15] the
 * selector features, out[k*17 + 16] the face's HLLE-HLLD flux gap in units of
 * its flux scales.  At most max_samples are kept; *n_out receives the count. */
int kr_selector_collect( kr_ctx * ctx, int n_steps, unsigned stride, uint64_t seed,
                         long long max_samples, float * out, long long * n_out );

/* Selector network on the GPU, with the project's own kernels.  X: [n][16]
 * features, Y: [n] labels (1 = HLLE safe).  Loss: class-weighted binary
 * cross-entropy on the logit, weight 1 for y = 1 and wneg for y = 0.
 * kr_mlp_init: He-initialised parameters; kr_mlp_grad: mean loss and mean
 * gradient (one forward / backward pass); kr_mlp_train: Adam over mini-batches
 * of consecutive samples, params in/out; kr_mlp_infer: logits through the BF16
 * tensor-core path of the flux sweep.  Errors: kr_learn_last_error(). */
int         kr_mlp_param_count( void );
void        kr_mlp_init ( float * params, uint64_t seed );
int         kr_mlp_grad ( const float * X, const float * Y, long long n, const float * params,
                          float wneg, float * grad, double * loss, int device );
int         kr_mlp_train( const float * X, const float * Y, long long n, float * params,
                          int epochs, int batch, float lr, float wneg, double * loss, int device );
int         kr_mlp_infer( const float * X, long long n, const float * params, float * logits,
                          int device );
const char* kr_learn_last_error( void );

/* Allocation-free cons -> prim and CFL dt for ONE block, on device pointers.
 * No counterpart in the reference: it exists for callers that cannot allocate
 * device memory (code that runs under another framework's memory pool, or
 * where cudaMalloc is not allowed), so the one kernel it launches keeps its
 * scratch (per-CTA dt minima and a completion counter) in a fixed array inside
 * the library instead of asking for memory.  Limit: blocks of at most
 * 4,194,304 cells (16384 CTAs of 256 threads, 128 KiB of scratch, held by every
 * GPU that loads the library until the process exits); larger blocks return -2
 * with the reason in kr_last_error(NULL).  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress) -- make that first call
 * before any stream capture.  All calls share the array: calls that overlap on
 * the GPU race and must be serialised by the caller.
 *   cfg   : abi_version (KR_ABI_VERSION, else -1), mhd, n[3] (each >= 4,
 *           else -1), x_min/x_max (one block covering the box), gamma, cfl,
 *           rho_floor, tmp_floor; nb and precision are ignored
 *   u     : device, conserved state [5][n2][n1][n0] (rho, E, m0..2); read
 *           only: the density and pressure floors apply to w alone, u is not
 *           healed (the engine's step writes healed rho / E back into U)
 *   bf    : device, face B [3][n2+5][n1+5][n0+5] (MHD only, else may be NULL)
 *   w     : device output, primitives [nw][n2+4][n1+4][n0+4], interior written
 *           (nw = 8 MHD: rho, p, v0..2, B_cc0..2; 5 hydro)
 *   dt_out: device output, one double: cfl * min over cells of dx / signal speed
 *   stream: cudaStream_t (NULL: legacy default stream)
 * Returns 0, or a negative code (enqueued work is asynchronous on `stream`). */
int kr_c2p_dt_noalloc( const kr_cfg * cfg, const double * u, const double * bf,
                       double * w, double * dt_out, void * stream );

/* ---- Batched launch over blocks of uneven sizes (no reference counterpart as
 * one launch: the reference runs each box as its own mesh and launches per
 * block, src/modules/dynamics/dynamics.h:51-103).  A batch joins up to 6
 * KR_FLAG_BOXES contexts (one per box edge length; same device, precision,
 * solver, dt_expand and sel_period) so that every kernel kind of the step runs
 * as one persistent launch over all their blocks: its CTAs walk a work list of
 * the CTA tiles of every block (bigger blocks first), with the per-group
 * arguments in the kernel's parameter space, and give the per-context steps'
 * results bit for bit.  One CUDA graph per step (14 launches, 20 with the
 * learned selector: stage 0's update and stage 1's c2p fused; 16 and 22 for
 * contexts made with KR_FLAG_UNFUSED), on the first context's stream.  The contexts stay owned
 * by the caller and must outlive the batch; their state, times and selector
 * calls work as before.
 *   kr_batch_step       : n_steps Heun steps of every box (enqueued)
 *   kr_batch_set_grid / kr_batch_get_grid : CTAs of each launch kind (8 kinds:
 *                         c2p stage 0, c2p stage 1, flux sweeps, the network's
 *                         sweep, edge EMF, conserved update, face update, and
 *                         stage 0's fused update + c2p; 0 = one CTA per work
 *                         item); returns the kind count
 *   kr_batch_autotune   : times 1, 2, 4 and 8 waves of resident CTAs and one
 *                         CTA per item for every kind (two eager steps each,
 *                         on a copy of the state, restored), keeps each kind's
 *                         fastest and appends "<key> | c2p0=.. .." to
 *                         cache_path (NULL: no cache); a line of the same
 *                         key (device, SM count,
 *                         precision, solver, sizes and counts) is reused
 *                         instead.  Returns 1 when cached, 0 when tuned.
 *   kr_batch_profile_step: one step run eagerly with CUDA events around every
 *                         launch; ms[k] = milliseconds of launch kind k (the
 *                         grid order above), n_kinds >= 8.  The step advances
 *                         the state like kr_batch_step. */
typedef struct kr_batch kr_batch;
kr_batch *  kr_batch_create           ( kr_ctx * const * ctxs, int n );
void        kr_batch_destroy          ( kr_batch * batch );
const char* kr_batch_last_error       ( const kr_batch * batch );
int         kr_batch_step             ( kr_batch * batch, int n_steps );
int         kr_batch_launches_per_step( kr_batch * batch );
int         kr_batch_get_grid         ( kr_batch * batch, int * grid );
int         kr_batch_set_grid         ( kr_batch * batch, const int * grid );
int         kr_batch_autotune         ( kr_batch * batch, const char * cache_path, int * grid_out );
int         kr_batch_profile_step     ( kr_batch * batch, int n_kinds, double * ms );

/* ---- Sharding over ranks: one context per GPU.
 * The reference distributes blocks over MPI ranks (mesh/meshgen/meshgen.cpp:
 * 166-247), fills ghosts from other ranks' blocks through MPI messages
 * (hydro/boundary/keeper.cpp:86-185, mhd/boundary/keeper.h:189-324) and
 * reduces dt over ranks (cycle.cpp:77-95).  Here, with cfg.n_ranks > 1, the
 * nb[0] x nb[1] x nb[2] global blocks are split into n_ranks boxes of whole
 * blocks by recursive coordinate bisection (largest extent first, ties to the
 * outer axis); a context holds the blocks of cfg.rank in ascending global
 * (lexicographic) id, and kr_set_state / kr_get_state / kr_init_problem /
 * kr_diagnostics work on those blocks only.  Per stage the ghost values a
 * block needs from another rank's block -- the 2-layer primitive box of each
 * of the 26 directions and, for MHD, the face-B strips of the 6 face
 * directions -- are packed into one send buffer grouped by peer, exchanged
 * with grouped NCCL send / receive inside the step's CUDA graph, and unpacked
 * into the ghost zones; after stage 0's CFL reduction an NCCL all-reduce(min)
 * makes dt global.  NCCL is loaded at run time (libnccl.so.2).
 *
 * kr_shard_owner : host only (no device needed).  owner[g] = rank of global
 *                  block g for every block; returns the number of blocks of
 *                  cfg->rank, or < 0 (kr_last_error(NULL)) if the mesh has
 *                  fewer blocks than ranks along the bisection.
 * kr_halo_counts : host only.  Words exchanged per stage with every peer p:
 *                  send[2p] primitive words (the step's arithmetic type),
 *                  send[2p+1] face-B words (double); recv likewise.  Arrays of
 *                  2 * n_ranks entries.  Peer p = rank: same-rank copies, only
 *                  with KR_FLAG_HALO_ALL.
 * kr_shard_blocks: global ids of the context's blocks (gid may be NULL);
 *                  returns their number.
 * kr_comm_unique_id / kr_comm_init: ncclGetUniqueId on one rank, the 128
 *                  bytes shared by the caller (e.g. a torch.distributed
 *                  broadcast), then ncclCommInitRank(n_ranks, rank) on every
 *                  rank's context (collective; call before the first step).
 *                  kr_step on a sharded context without a communicator fails.
 * kr_group_step  : all n_ranks contexts of one mesh driven from one process
 *                  (ctxs[r] of rank r, same device): the exchange becomes
 *                  device copies between the contexts and the dt minimum a
 *                  kernel over their scalars, all on ctxs[0]'s stream
 *                  (synchronous).  For running a sharded mesh on one GPU. */
int kr_shard_owner   ( const kr_cfg * cfg, int * owner );
int kr_halo_counts   ( const kr_cfg * cfg, long long * send, long long * recv );
int kr_shard_blocks  ( kr_ctx * ctx, int * gid );
int kr_comm_unique_id( unsigned char id[ 128 ] );
int kr_comm_init     ( kr_ctx * ctx, const unsigned char id[ 128 ] );
int kr_group_step    ( kr_ctx * const * ctxs, int n, int n_steps );

#ifdef __cplusplus
}
#endif
#endif
