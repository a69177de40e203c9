/*
 * fdfault_b200 -- C ABI of the B200 time-stepping path for fdfault problems.
 *
 * The reference solver (edaub/fdfault) advances a problem with
 *   problem::problem(const char* filename)        src/problem.cpp:16
 *   problem::solve()                               src/problem.cpp:136
 *   domain::do_rk_stage(dt, stage, t, rk)          src/domain.hpp:26, src/domain.cpp:228
 * and keeps its state in fields::f/df (src/fields.hpp:58-59) and the friction
 * arrays of interface/friction (src/interface.hpp:66-73, src/friction.hpp:23-26),
 * which its output units read through friend access (src/outputunit.cpp:771-889).
 * The entry points below replace those calls: the state lives in GPU memory,
 * every stage runs as sm_100a kernels, and the host sees plain pointers and
 * sizes.  Every function returns 0 on success or a negative error code (no
 * C++ exception crosses the boundary); fdf_last_error() gives the message.
 * A handle may be used from one host thread at a time.
 */
#ifndef FDFAULT_B200_H
#define FDFAULT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fdf_handle fdf_handle;

/* precision of the field storage and stencil arithmetic */
#define FDF_PRECISION_FP64 0 /* FP64, the reference's operation order (bit-identical results) */
#define FDF_PRECISION_FP32 1 /* FP32 fields, metrics and stencil; FP64 friction, slip and time */

/* error codes */
#define FDF_ERR_ARG (-1)     /* invalid argument */
#define FDF_ERR_INPUT (-2)   /* problem file or side file rejected */
#define FDF_ERR_CUDA (-3)    /* CUDA runtime error */
#define FDF_ERR_SOLVER (-4)  /* device status: Newton failure, STZ melting, non-finite values */

/* geometry selectors for fdf_get_geometry */
#define FDF_GEOM_X 0      /* node coordinates, comp 0..ndim-1 */
#define FDF_GEOM_METRIC 1 /* d xi_l / d x_m, comp l*ndim+m */
#define FDF_GEOM_JAC 2    /* Jacobian */

/* fault array selectors for fdf_get_fault / fdf_set_fault (friction.hpp:23-26,
 * interface.hpp:66-73, stz.cpp:160-162, front.hpp) */
#define FDF_FAULT_U 0        /* slip magnitude */
#define FDF_FAULT_DU 1       /* RK register of slip */
#define FDF_FAULT_V 2        /* slip rate magnitude */
#define FDF_FAULT_S 3        /* shear traction magnitude */
#define FDF_FAULT_SN 4       /* normal traction */
#define FDF_FAULT_UX 5       /* slip components, (ndim-1) planes */
#define FDF_FAULT_DUX 6      /* RK register of slip components */
#define FDF_FAULT_VX 7       /* slip-rate components */
#define FDF_FAULT_SX 8       /* shear traction components */
#define FDF_FAULT_STATE 9    /* STZ effective temperature */
#define FDF_FAULT_DSTATE 10  /* RK register of the state */
#define FDF_FAULT_DSTATEDT 11/* state rate */
#define FDF_FAULT_TFRONT 12  /* rupture time (-1 before rupture) */

/* Replaces problem::problem (src/problem.cpp:16-84) including
 * domain::domain (src/domain.cpp:19-153): reads the .in file and its side
 * files, builds grid, metrics, normals, friction parameters and the time
 * step on device `device`. */
int fdf_create(const char* infile, int precision, int device, fdf_handle** out);

/* Releases all device memory of the problem. */
void fdf_destroy(fdf_handle* h);

/* ints[0..15]: ndim, mode, nx, ny, nz, nfields, nfieldsp, nifaces, nstages,
 *              nt, sbporder, nblocks x, y, z, plastic, rkorder
 * dbls[0..2]: dt, ttot, cfl  (problem::set_time_step, src/problem.cpp:94-134) */
int fdf_get_info(fdf_handle* h, int* ints, double* dbls);

/* Replaces domain::do_rk_stage (src/domain.cpp:228-305): one Runge-Kutta
 * stage with time step dt at step time t. */
int fdf_do_rk_stage(fdf_handle* h, double dt, int stage, double t);

/* Runs nsteps steps of the problem::solve loop body (src/problem.cpp:151-168):
 * all stages, the absolute-stress output round trip and the front update,
 * without writing output files. */
int fdf_step(fdf_handle* h, int nsteps);

/* Replaces problem::solve (src/problem.cpp:136-192): runs the remaining
 * steps, writes the output units and the rupture fronts. */
int fdf_solve(fdf_handle* h);

/* Stage `stage` of the current step as fdf_step runs it (the loop body of
 * src/problem.cpp:151-168 split at its domain::do_rk_stage calls); the last
 * stage advances the step counter.  Stages come in order 0, 1, ...; an x
 * slab exchanges its ghost planes between two calls. */
int fdf_step_stage(fdf_handle* h, int stage);

/* Multi-GPU x slabs.  The reference splits its domain across MPI ranks
 * (src/cartesian.cpp:88-165) and swaps ghost planes after every stage
 * (fields::exchange_neighbors, src/fields.cpp:276-291, called from
 * src/domain.cpp:228-305).  Here each process updates the global x planes
 * [x0, x1) of its own copy of the grid (3D; volume kernel 0 or 3; no
 * dissipation; each cut at least 16 planes inside an x block) and steps with
 * fdf_step_stage; after each stage it packs its edge planes for its
 * neighbours and unpacks theirs into its ghost planes.  (0, nx) is the whole
 * domain again.  fdf_step and fdf_solve refuse a slab. */
int fdf_set_x_range(fdf_handle* h, int x0, int x1);
/* planes: ghost planes per side (sbporder - 1); count: elements of one side's
 * exchange buffer; elem_bytes: 8 (FP64 problem) or 4 (FP32). */
int fdf_ghost_info(fdf_handle* h, int* planes, long long* count, int* elem_bytes);
/* side 0: the slab's first `planes` planes into dst (for the lower
 * neighbour); side 1: its last ones (for the upper neighbour).  dst and src
 * are device buffers of `count` elements, ordered on the handle's stream. */
int fdf_pack_ghosts(fdf_handle* h, int side, void* dst);
/* side 0: src into the ghost planes below x0; side 1: into those from x1. */
int fdf_unpack_ghosts(fdf_handle* h, int side, const void* src);
/* First global node lo[3] and node counts n[3] of block `block` (blocks in
 * the order of the input file's block list). */
int fdf_get_block(fdf_handle* h, int block, int* lo, int* n);
/* Interface `iface`: its normal direction (0 x, 1 y, 2 z), the minus-side
 * face's first global node lo[3] and the face's node counts n[2]; fault node
 * (a, b) lies at lo + a along the first other direction and + b along the
 * second (x before y before z). */
int fdf_get_interface(fdf_handle* h, int iface, int* direction, int* lo, int* n);
/* Launch on the caller's CUDA stream (own = 0; e.g. the stream a collective
 * library waits on) or the handle's own stream again (own = 1).  Waits for
 * the work already queued first.  The caller's stream must outlive its use
 * by the handle (set own = 1 before destroying it), and fdf_step, which
 * captures CUDA graphs on the stream, needs one other than the legacy
 * default stream. */
int fdf_set_stream(fdf_handle* h, int own, void* stream);

/* Index of the next step to run. */
int fdf_get_step(fdf_handle* h, int* step);
int fdf_set_step(fdf_handle* h, int step);

/* Field component comp (reference numbering, src/outputunit.cpp:123-156 /
 * 193-204) in the reference's node order (i, j, k; k fastest), n = nx*ny*nz
 * values.  absolute=1 adds the initial stress to stress components, as the
 * output units see them. */
int fdf_get_field(fdf_handle* h, int comp, int absolute, double* out);

/* Same values as fdf_get_field, without any device allocation, for callers
 * that may not allocate device memory once running (a service that sizes its
 * GPU memory up front, or code under an external memory budget), whereas
 * fdf_get_field may grow a scratch buffer with cudaMalloc.  The component is
 * gathered into one fixed static device buffer of FDF_NOALLOC_MAX_VALUES
 * doubles (8 MiB, held by every GPU that loads the library until exit), then
 * copied to `out`.  No counterpart in the reference (which has no device
 * memory).  Fields larger than the buffer are rejected with FDF_ERR_ARG.  The
 * first call on a device looks up the buffer's device address (make it before
 * any stream capture).  The buffer is shared by every handle on the device:
 * calls that overlap on the GPU (from several host threads, or on several
 * handles of one device) race on it and may return each other's values;
 * serialise them. */
#define FDF_NOALLOC_MAX_VALUES 1048576
int fdf_get_field_noalloc(fdf_handle* h, int comp, int absolute, double* out);
int fdf_set_field(fdf_handle* h, int comp, const double* in);

/* RK rate register df (src/fields.hpp:59) */
int fdf_get_rate(fdf_handle* h, int comp, double* out);
int fdf_set_rate(fdf_handle* h, int comp, const double* in);

/* Coordinates, metric and Jacobian (src/fields.hpp:60-62). */
int fdf_get_geometry(fdf_handle* h, int which, int comp, double* out);

/* Number of values of a fault array of interface iface (0 if absent). */
int fdf_fault_count(fdf_handle* h, int iface, int which, long long* n);
int fdf_get_fault(fdf_handle* h, int iface, int which, double* out);
/* Queues the same copy as fdf_get_fault behind the work already queued on the
 * handle and returns without waiting: `out` holds the values once a later
 * fdf_synchronize returns, and must stay valid until then.  The array is
 * snapshotted on the device (into a ring of at least 64 MB allocated by the
 * first call) and copied to `out` on a second stream, so with page-locked
 * `out` the copy overlaps the steps queued after it.  For reading a step's
 * fault output every step without stalling the next step, in the way the
 * reference's output units read the friction arrays after each step
 * (src/outputunit.cpp:771-889). */
int fdf_get_fault_async(fdf_handle* h, int iface, int which, double* out);
int fdf_set_fault(fdf_handle* h, int iface, int which, const double* in);

/* Waits for all queued device work; returns FDF_ERR_SOLVER if a kernel set
 * a status bit (Newton failure, melting, non-finite values). */
int fdf_synchronize(fdf_handle* h);

/* Device time of nsteps steps (CUDA events on the solver's stream), ms. */
int fdf_time_steps(fdf_handle* h, int nsteps, double* ms);

/* Per-kernel timing: with profiling on, each volume-kernel launch (kernel 0)
 * and each stage's interface kernels (kernel 1) are bracketed by CUDA events
 * on the solver's stream; read returns total milliseconds and launches. */
int fdf_profile(fdf_handle* h, int on);
int fdf_profile_read(fdf_handle* h, int kernel, double* total_ms, long long* launches);

/* fdf_step and fdf_time_steps run each step by replaying a captured CUDA
 * graph of one step (one graph per field-buffer parity) when per-launch
 * profiling is off (default on=1); fdf_solve, which writes output units
 * between steps, launches stage by stage.  Results are identical to the
 * launch-by-launch path (the stage time comes from a device step counter). */
int fdf_use_graphs(fdf_handle* h, int on);

/* Choose between the tiled FP32 volume kernel (default) and the
 * one-thread-per-node kernel for FP32 problems; active=1 if the tiled kernel
 * will run. */
int fdf_use_fast_kernel(fdf_handle* h, int on, int* active);

/* FP32 volume kernel by kind: 0 one thread per node (reference operation
 * order), 1 tiled (3D blocks of at least 8 x 32 in y x z, and 2D elastic
 * blocks at least 32 nodes wide in y), 2 staged (3D only: planes brought into
 * shared memory by TMA tensor copies), 3 register window (the default: 3D
 * blocks of the same sizes as kind 1, the x stencil window in registers and
 * every plane of a tile staged by TMA tensor copies; plastic stages add the
 * return map in separate passes, dissipative stages run kind 0; for 2D problems it selects the tiled 2D kernel like
 * kind 1).  active = the kind that will run (0 where the chosen one does not
 * apply to the problem: FP64 problems and problems with a heterogeneous
 * material file always run kind 0). */
int fdf_set_volume_kernel(fdf_handle* h, int kind, int* active);

/* Polls of each bounded wait for staged data in the TMA-staged volume kernels
 * (kinds 2 and 3); polls = 0 restores the built-in limit (2^22).  A wait that
 * runs out makes its CTA record FDF_ERR_TIMEOUT in the device status word
 * (reported by the next fdf_synchronize as FDF_ERR_SOLVER), wait with a fixed
 * generous limit for its own copies still in flight, and return; the fields of
 * that stage are then incomplete.  With polls = 1 every wait is a single
 * immediate test; with polls < 0 every such wait gives up at once, so a test
 * can exercise this path deterministically.  No reference counterpart: the
 * reference has no device waits. */
int fdf_set_wait_limit(fdf_handle* h, long long polls);

/* Nodes and bulk modulus of the Drucker-Prager return map (plastic problems).
 * Rule 0, the default, is the reference's block::calc_plastic
 * (src/block.cpp:442-589) as it runs: the function declares `double k` and
 * then an `int k` z-loop index, so the bulk modulus K = lambda + 2/3 G it
 * computes lands in the loop index.  The return map therefore gets trunc(K),
 * and the z loop continues at trunc(K) + 1: every node in 2D, and in 3D the
 * first z node of each column of a block (more with a heterogeneous material
 * whose trunc(K) + 1 falls inside the block).  Where that loop would never
 * end (3D blocks reaching z index trunc(K) + 1, e.g. nz > 54 for the usual
 * lambda = G = 32.04) stepping under rule 0 fails with FDF_ERR_SOLVER and a
 * message naming the loop.  Rule 1 applies the return map at every node with
 * the exact K, the evident intent of that code; it has no reference result to
 * match.  Changing the rule drops captured step graphs. */
#define FDF_PLASTIC_REFERENCE 0
#define FDF_PLASTIC_EVERY_NODE 1
int fdf_set_plastic_rule(fdf_handle* h, int rule);

/* FP64 energy diagnostics of an elastic problem, accumulated on the device
 * whatever the field precision, in the diagonal norm H of the SBP operator
 * (H D + D^T H = diag(-1, 0, ..., 0, 1); its first entry is the reference's
 * boundary norm h0, src/fd.cpp:119-120):
 *   out[0] kinetic energy  sum w J rho |v|^2 / 2,
 *   out[1] strain energy   sum w J sigma:S:sigma / 2   (w = H_i H_j H_k dxi dxeta dzeta),
 *   out[2] (with_rate) dE/dt = sum w J (rho v.L_v + sigma:S:L_sigma) under the
 *          semi-discrete operator L at the current state, volume terms, outer
 *          SATs and interfaces together; L(f) is obtained by a stage evaluation
 *          that leaves fields, slip and state unchanged and leaves dt L(f) in
 *          the rate register (fdf_get_rate); call it between steps,
 *   out[3] (with_rate) sum of the magnitudes of those rate terms (a scale),
 *   out[4] frictional power of all interfaces: minus-side face area element
 *          times traction . slip rate, from the fault arrays,
 *   out[5..7] zero.
 * Plastic problems are rejected.  No reference counterpart: the reference has
 * no energy diagnostics. */
int fdf_energy(fdf_handle* h, int with_rate, double out[8]);

/* Algorithmic bytes moved per node per stage by the volume kernel. */
int fdf_bytes_per_node_stage(fdf_handle* h, long long* bytes);

/* Message of the last failed call on h (or of the last failed fdf_create when
 * h is null). */
/* ---- STZ friction with a learned Newton initial guess (no counterpart in
 * the reference, whose solve always starts at the bracket midpoint,
 * src/utilities.cpp:89-179 called from src/stz.cpp:296-303).
 *
 * A 6 -> 64 -> 64 -> 1 ReLU network (BF16 weights and activations, FP32
 * accumulation) predicts t = log(s/(1-s))/20, s = (mu - muy)/(phi/|sn| - muy),
 * for every STZ fault node from the node's traction, normal stress, state
 * and parameters; the
 * bracketed Newton iteration starts at that mu and falls back to the plain
 * midpoint start when the guess is outside the bracket or does not converge.
 * Parameters are one flat FP32 vector of FDF_MLP_NPARAM values:
 * W1[64][6], b1[64], W2[64][64], b2[64], W3[64], b3. */
#define FDF_MLP_NPARAM 4673
int fdf_stz_set_learned(fdf_handle* h, int on);

/* Start of the STZ Newton solve, for judging the learned start against other
 * ways of cutting iterations: 0 bracket midpoint with the reference's
 * derivative (the reference, src/utilities.cpp:97 and src/stz.cpp:479; the
 * default), 1 the learned start (as fdf_stz_set_learned 1), 2 warm start from
 * each node's previous converged mu (the previous stage's root; the midpoint
 * where none is known or it leaves the bracket), 3 bracket midpoint with the
 * exact derivative of the slip-rate law instead of the reference's (whose sign
 * of the mu_y term makes the iteration converge linearly).  Modes 1-3 converge
 * to the same roots within the Newton tolerance, not bit for bit. */
int fdf_stz_set_start(fdf_handle* h, int mode);
/* counters of the Newton solves: [0] solves, [1] iterations, [2] solves that
 * started at the bracket midpoint (plain, or a rejected guess) */
int fdf_stz_set_counting(fdf_handle* h, int on);
int fdf_stz_read_counts(fdf_handle* h, long long* counts, int reset);
/* solver-generated training samples, one row of 8 floats per converged
 * Newton solve: the 6 network inputs, the target t and the converged mu;
 * capacity 0 stops collecting.  fdf_stz_samples copies min(count, max_rows)
 * rows and returns the number collected (capped at the capacity).  The target
 * column holds t = log(s/(1-s))/20. */
int fdf_stz_collect(fdf_handle* h, long long capacity);
int fdf_stz_samples(fdf_handle* h, float* out, long long max_rows, long long* count);
int fdf_mlp_init(fdf_handle* h, unsigned long long seed);
int fdf_mlp_set_params(fdf_handle* h, const float* params);
int fdf_mlp_get_params(fdf_handle* h, float* params);
/* network outputs y[n] for inputs x[n][6]; force_thread=1 uses the per-thread
 * path instead of the tensor-core warp path */
int fdf_mlp_infer(fdf_handle* h, const float* x, long long n, float* y, int force_thread);
/* gradient of 0.5*mean((y - t)^2) with respect to the parameters */
int fdf_mlp_gradients(fdf_handle* h, const float* x, const float* t, long long n, float* grads, double* loss);
/* Adam training on the collected samples (a tenth held out) */
int fdf_mlp_train(fdf_handle* h, int epochs, int batch, float lr, unsigned long long seed, double* train_loss,
                  double* val_loss);

/* ---- Batched ensemble of independent problems (no counterpart in the
 * reference, which runs one problem per process).
 *
 * All members run in FP32 (fields) with FP64 friction, share the Runge-Kutta
 * order, are elastic and use locked, frictionless or slip-weakening
 * interfaces.  Each stage of all members is a few batched volume launches
 * (2D members whose blocks are at least 32 nodes wide in y: the tiled 2D
 * kernel, one launch per SBP order and mode present; all others: the
 * one-thread-per-node kernel) and one batched interface launch, each over a
 * work list; step counters and field-buffer parities live on the device, and
 * chunks of 16 steps replay one captured CUDA graph.  A member's results are
 * bit-identical to running it alone in FP32 with the same volume kernel
 * (fdf_set_volume_kernel 1 for the first kind, 0 for the second).  Members
 * step min(nsteps, nt - step) steps. */
typedef struct fdf_ensemble fdf_ensemble;
int fdf_ensemble_create(const char* const* infiles, int n, int device, fdf_ensemble** out);
void fdf_ensemble_destroy(fdf_ensemble* e);
int fdf_ensemble_size(fdf_ensemble* e, int* n);
/* a handle on member i for the per-problem read functions (fdf_get_field,
 * fdf_get_fault, fdf_get_info ...); release it with fdf_destroy, which leaves
 * the member to the ensemble.  Stepping it directly desynchronises it. */
int fdf_ensemble_member(fdf_ensemble* e, int member, fdf_handle** out);
int fdf_ensemble_run(fdf_ensemble* e, int nsteps);
int fdf_ensemble_time_steps(fdf_ensemble* e, int nsteps, double* ms);
/* times `steps` real steps with each candidate CTA size and tile size, keeps
 * the fastest (tiling never changes results); `tile` is the node count of a
 * work item (the tiled 2D kernel takes tile / 32 rows of a 32-column tile) */
int fdf_ensemble_autotune(fdf_ensemble* e, int steps, int* threads, long long* tile);
int fdf_ensemble_set_config(fdf_ensemble* e, int threads, long long tile);
int fdf_ensemble_use_graph(fdf_ensemble* e, int on);
/* sum over members of nodes x stages: node-stage updates per ensemble step */
int fdf_ensemble_node_stages(fdf_ensemble* e, long long* per_step);
/* reads and clears every member's status word; FDF_ERR_SOLVER if one is set */
int fdf_ensemble_check_status(fdf_ensemble* e);
const char* fdf_ensemble_last_error(fdf_ensemble* e);

const char* fdf_last_error(fdf_handle* h);

#ifdef __cplusplus
}
#endif

#endif
