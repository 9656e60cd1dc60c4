/*
 * vxr.h — the C ABI of the B200-native rigid-body step.
 *
 * A drop-in for the reference's per-step pipeline (sibarum/vexelray-sim-rigid). Each entry point names the
 * reference interface it replaces, by path inside that project:
 *   gui  = vexelray-sim-rigid-gui/src/main/java/dev/vexelray/sim/rigid/gui/
 *   core = vexelray-sim-rigid-core/src/main/java/dev/vexelray/sim/rigid/
 *
 * Plain pointers and sizes only. Host buffers are caller-owned and copied in or out before the call returns;
 * the library owns all device memory of a world. One world = one host thread (as the reference: "not
 * thread-safe: one stepper, one thread", core/sphere/SphereStepper.java:19) and one CUDA stream of its own.
 * Every entry point returns a status (VXR_OK or an error below); vxr_box_error() gives the text of the last
 * error of a world.
 */
#ifndef VXR_H
#define VXR_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The reference throws IllegalArgumentException for bad parameters or sizes
 * (core/box/Boxes.java:212-226, core/box/BoxStep.java:82-85) and IllegalStateException for a pass that never
 * ends (core/sphere/SphereStepper.java:86-88); soft failures it counts in its reports. */
#define VXR_OK 0
#define VXR_EINVAL 1     /* bad argument: IllegalArgumentException in the reference */
#define VXR_ECAPACITY 2  /* more candidate pairs than the world's pair capacity */
#define VXR_EROUNDS 3    /* the device colouring did not finish within its wave limit */
#define VXR_ENONFINITE 4 /* non-finite state */
#define VXR_ETIMEOUT 5   /* a device wait (grid barrier) ran out: the step stopped, the GPU stays usable */
#define VXR_ECUDA 6      /* a CUDA call failed */

#define VXR_PARAM_COUNT 18   /* core/box/Boxes.java:101 */
#define VXR_SHOWN_STRIDE 20  /* core/box/Boxes.java:781 */
#define VXR_SLOTS 32         /* core/box/BoxBroad.java:60 */
#define VXR_MOST_ROUNDS 32   /* core/box/BoxStep.java:45 */
#define VXR_BOX_SHAPE 0.0f   /* core/box/Boxes.java:154 */
#define VXR_SPHERE_SHAPE 1.0f

/* The broad phase's grid: nx * ny * nz cubic cells of side `cell` from the origin
 * (core/sphere/SphereGrid.java:11-36). */
typedef struct {
    int32_t nx, ny, nz;
    float cell;
} vxr_grid;

/* A world's shape, fixed at creation: the reference's BoxStep(boxes, substeps, sweeps, symmetric, grid)
 * (core/box/BoxStep.java:81-162). */
typedef struct {
    int32_t bodies;
    int32_t substeps;
    int32_t sweeps;      /* sweeps of the solve and as many of the relax per substep */
    int32_t symmetric;   /* every other sweep backwards */
    vxr_grid grid;       /* nx = 0: no grid (a lone body, or bodies that never meet) */
    int32_t reach_cells; /* neighbourhood half-width in cells; 0 or 1 = the reference's 27 cells. Cells narrower
                            than the reference's rule (core/box/BoxBroad.java:66-68) need 2 or more. */
    int32_t max_pairs;   /* candidate/touching pair capacity; 0 = bodies * 32, the reference's slot count */
    int32_t device;      /* CUDA device ordinal */
    int32_t schedule;    /* 0: a grid-wide barrier after every round (default); 1: dependency-driven, each pair or
                            wall item waiting only for its own bodies. Both keep the reference's per-body order of
                            operations and give the same results. */
    int32_t solve_blocks_per_sm; /* blocks of the solve kernel an SM runs; 0 = as many as fit (the autotuner's knob) */
} vxr_box_config;

/* What a step took: core/box/BoxStepper.java:40 (Report), plus the totals over a vxr_box_step call. */
typedef struct {
    int32_t touching;  /* pairs whose manifolds have points (last step) */
    int32_t points;    /* their points */
    int32_t rounds;    /* rounds the touching pairs were coloured into */
    int32_t unplaced;  /* touching pairs left unsolved: every round had one of their bodies */
    int32_t unlisted;  /* partners the broad phase found and had no slot for */
    int32_t most_rounds;
    int64_t unplaced_total;
    int64_t unlisted_total;
    int32_t status;
    int32_t steps;
} vxr_box_report;

/* Version string of the library. */
const char* vxr_version(void);

/* The 18 parameter words as f32 bits: replaces Boxes.params(h, gx, gy, gz, sx, sy, sz, muStatic, muKinetic,
 * margin, muRolling) (core/box/Boxes.java:212-234), softness by Boxes.softness (:242-251). */
int32_t vxr_box_make_params(double h, double gx, double gy, double gz, double sx, double sy, double sz,
                            double mu_static, double mu_kinetic, double margin, double mu_rolling, int32_t* out18);

/* The grid over the walled box: replaces BoxBroad.grid (core/box/BoxBroad.java:66-68). */
int32_t vxr_box_make_grid(double sx, double sy, double sz, double widest_half_diagonal, double margin,
                          vxr_grid* out);

typedef struct vxr_box_world vxr_box_world;

/* A world on the GPU: replaces new BoxStep(...) + new BoxSimulation(context, step)
 * (core/box/BoxStep.java:81-162, gui/BoxSimulation.java:34-50). NULL on failure, *status says why. */
vxr_box_world* vxr_box_create(const vxr_box_config* config, int32_t* status);

/* Releases the world: replaces BoxSimulation.close (gui/BoxSimulation.java:183-188). */
void vxr_box_destroy(vxr_box_world* world);

/* The text of the world's last error. */
const char* vxr_box_error(const vxr_box_world* world);

/* Starts from a state: replaces BoxSimulation.start(x, y, z, u, v, w, spin[3][], q[4][], half[3][], shape, im,
 * params) (gui/BoxSimulation.java:77-108). Each array holds `bodies` floats; spin is the angular velocity in the
 * world's frame, turned into the angular momentum the body keeps (BoxDiagnostics.momentum, in doubles). Clears
 * every impulse, as the reference's runner.clear() does. */
int32_t vxr_box_start(vxr_box_world* world, const float* x, const float* y, const float* z, const float* u,
                      const float* v, const float* w, const float* const* spin3, const float* const* q4,
                      const float* const* half3, const float* shape, const float* im, const int32_t* params18);

/* Starts from a state given as the 18 fields x y z u v w lx ly lz qx qy qz qw im hx hy hz shape (angular
 * momentum, as core/box/BoxStep.java keeps it; the reference's test fixture writes these buffers directly,
 * vexelray-sim-rigid-core/src/test/java/dev/vexelray/sim/rigid/box/BoxScene.java:141-166). Clears every impulse. */
int32_t vxr_box_load_state(vxr_box_world* world, const float* const* fields18, const int32_t* params18);
/* Both starts refuse a state holding a NaN or an infinity with VXR_ENONFINITE and load nothing: such a state is
 * what the reference's diagnostics flag as broken (core/sphere/SphereDiagnostics.java:48-50). */

/* New parameters from the next step on: replaces BoxSimulation.params (gui/BoxSimulation.java:111-113). */
int32_t vxr_box_params(vxr_box_world* world, const int32_t* params18);

/* `steps` steps, waited for: replaces BoxSimulation.stepAndWait (gui/BoxSimulation.java:115-142), which runs
 * BoxStepper.step (core/box/BoxStepper.java:56-100). The report is the last step's, with totals. */
int32_t vxr_box_step(vxr_box_world* world, int32_t steps, vxr_box_report* report);

/* `steps` steps enqueued on the world's stream, not waited for; vxr_box_sync waits and reports. Replaces the
 * non-waiting SphereSimulation.step (gui/SphereSimulation.java:191-193) for boxes. */
int32_t vxr_box_step_async(vxr_box_world* world, int32_t steps);
int32_t vxr_box_sync(vxr_box_world* world, vxr_box_report* report);

/* The world's CUDA stream (a cudaStream_t), for a caller that times or orders work against it. */
void* vxr_box_stream(vxr_box_world* world);

/* The state read back into 13 caller arrays x y z u v w lx ly lz qx qy qz qw: replaces BoxSimulation.state
 * (gui/BoxSimulation.java:153-160). */
int32_t vxr_box_state(vxr_box_world* world, float* const* out13);
/* The same read-back without waiting: the state after the steps enqueued so far is split into slot `slot` (0 or 1)
 * on the device and copied into out13 on a stream of its own, so the next steps run while it travels. The arrays
 * must stay valid, and should be pinned, until vxr_box_state_wait(world, slot) returns; a slot is reused only after
 * its copy before has finished. Reads of this kind, one a step into alternating slots, hide the copies behind the
 * steps. */
int32_t vxr_box_state_async(vxr_box_world* world, float* const* out13, int32_t slot);
/* Waits until slot `slot`'s last copy is in the caller's arrays. */
int32_t vxr_box_state_wait(vxr_box_world* world, int32_t slot);

/* The last step's `shown`, 20 floats a body: replaces BoxSimulation.readShown (gui/BoxSimulation.java:163-165). */
int32_t vxr_box_read_shown(vxr_box_world* world, float* out);

/* The last step's touching pairs in slot order (the order BoxStepper reads `contacts`,
 * core/box/BoxStepper.java:71-90): first and second body, point count, the manifold in the reference's 40-word
 * layout (core/box/BoxContact.java:85-96) and the impulses in its 28-word layout (core/box/BoxPairs.java:48-50).
 * Any output may be NULL. Returns the number of touching pairs, or minus a status. */
int32_t vxr_box_touching(vxr_box_world* world, int32_t* first, int32_t* second, int32_t* points, float* manifold40,
                         float* impulses28, int32_t capacity);

/* The last step's candidate pairs (the broad phase's listed slots, core/box/BoxBroad.java:103-164), sorted
 * (first, second) flat. Returns their number, or minus a status. */
int32_t vxr_box_candidates(vxr_box_world* world, int32_t* pairs, int32_t capacity);

/* The wall impulses in the reference's layout: lambda 48 floats a body, rub 144, roll 144
 * (core/box/Boxes.java:142-147). Any output may be NULL. */
int32_t vxr_box_walls(vxr_box_world* world, float* lambda48, float* rub144, float* roll144);

/* How many dependency waves the last step's colouring took. */
int32_t vxr_box_colour_waves(vxr_box_world* world);

/* Measurement and iteration switches, from the next step on: residual = 1 gathers each sweep's residual (below);
 * cold_start = 1 starts every step's pair impulses from zero instead of carrying them (BoxPairs.carry,
 * core/box/BoxPairs.java:191-267) — the plain solver with no warm start, for comparison; sweeps (1 .. the count the
 * world was created with; 0 = that count) sets the sweeps of the solve and of the relax a substep runs, as the
 * reference's BoxStep sweeps (core/box/BoxStep.java:49-50); tolerance > 0 (with residual = 1, barrier schedule) stops a
 * substep's solve sweeps, and its relax sweeps, once a sweep's residual is at or below it. */
int32_t vxr_box_measure(vxr_box_world* world, int32_t residual, int32_t cold_start, int32_t sweeps, float tolerance);

/* How the substeps are scheduled, from the next step on; no reference counterpart, the results are the same either
 * way (the reference's per-body order, core/box/BoxStep.java:199-231). enable = 1 (the default): the connected
 * components of the placed touching pairs of at most 256 bodies are solved whole by one thread block each (several
 * components a block, up to 511 bodies, held in shared memory for the step), their rounds apart by block barriers,
 * and bodies in no placed pair by a thread each; only larger components go through the grid-wide phases. enable = 0: every body goes through the grid-wide phases. A measuring tolerance
 * (vxr_box_measure) runs every body through the grid-wide phases whatever this says. */
/* The longest a device-wide wait of a step (a grid barrier, a dependency wait) may last, from the next step on; ns
 * <= 0 restores the default of 2 s. A wait that runs out stops the step: the call returns VXR_ETIMEOUT and the GPU
 * stays usable (the world's state is then part-way through a step; load a state before stepping again). No
 * reference counterpart: the reference's host waits on its runner (core/box/BoxStepper.java:62). */
int32_t vxr_box_wait_limit(vxr_box_world* world, int64_t ns);

int32_t vxr_box_islands(vxr_box_world* world, int32_t enable);

/* Which kernel lists the broad phase's candidates, from the next step on; no reference counterpart, the pairs are the
 * same either way (BoxBroad.list, core/box/BoxBroad.java:103-164). tiled = 0 (the default): a thread a body walks its
 * 27 cells in global memory. tiled = 1: a block takes a run of 16 cells along x and stages their 27-cell
 * neighbourhoods in shared memory; where they are crowded a warp lists a body, testing 32 candidates at once with a
 * ballot compaction in the walk's order and a bitonic sort of the first 32 found, and where they are sparse a thread
 * lists a body from the staged copy. Measured on the large mixed scene the per-thread walk is the faster (0.23 against
 * 0.32-0.35 ms a step early in the drop, 0.62 against 0.63-0.66 ms on the landed pile), so it is the default.
 * Batched scenes and widened neighbourhoods always use the per-thread walk. */
int32_t vxr_box_list_kernel(vxr_box_world* world, int32_t tiled);

/* How the last step was scheduled: out5 = [bodies through the grid-wide phases, bodies in small components (island
 * blocks), bodies in no placed pair (a thread each), island groups, bodies of the largest component]. With islands
 * off: [bodies, 0, 0, 0, 0]. */
int32_t vxr_box_paths(vxr_box_world* world, int32_t* out5);

/* The last step's per-sweep residuals, substep by substep: the warm sweep, the solve sweeps, the relax sweeps
 * (substeps * (2 sweeps + 1) values). A sweep's residual is the largest positional correction its updates made at any
 * contact point, h k (|change of the normal impulse| + |change of the tangential impulse|) in metres, k the point's
 * generalised inverse mass along the normal: zero when the Gauss-Seidel solve has converged. The reference has no
 * residual; this is the measure "iterations to residual" counts in. used (may be NULL) receives 2 substeps ints: the
 * solve and the relax sweeps each substep ran. Returns the count of residuals, or minus a status. */
int32_t vxr_box_residuals(vxr_box_world* world, float* out, int32_t capacity, int32_t* used);
/* The same residuals in two parts, each the largest correction at a contact of one kind: pairs (between two bodies)
 * and walls (a body against the box); vxr_box_residuals gives the larger of the two, and a substep's sweeps stop
 * when both are within the tolerance. Either pointer may be NULL. Returns the count a part, or minus a status. */
int32_t vxr_box_residual_parts(vxr_box_world* world, float* pairs, float* walls, int32_t capacity);

/* Kernels this world's steps have launched since creation (each step launches the same number; reading the
 * state back is not counted). */
long long vxr_box_launches(vxr_box_world* world);

/* Per-phase device time: with enable = 1 each following step records CUDA events on the world's stream around
 * its broad phase, narrow phase (with the carry), colouring and solve; phase_ms4 receives the milliseconds
 * summed since the last call (resolved at vxr_box_sync), and the sums restart. The reference reports one GPU
 * time a step from Vulkan timestamps (gui/BoxSimulation.java:140-141). */
int32_t vxr_box_profile(vxr_box_world* world, int32_t enable, double* phase_ms4);

/* Phase trace of the solve: with enable = 1 each following step's solve kernel records, at the end of every
 * phase, (phase code << 48) | device nanoseconds, where the code is kind | sweep << 4 | round << 8 (kinds: 0 start,
 * 1 velocities, 2 walls, 3 positions, 4 a round of pairs, 5 the wall list). out receives the last traced step's
 * entries; returns their number, or minus a status. */
int32_t vxr_box_trace(vxr_box_world* world, int32_t enable, int64_t* out, int32_t capacity);

/* Activity of the last step: touching pairs, their points, bodies in a touching pair or holding a wall impulse,
 * and wall contact records held. */
int32_t vxr_box_activity(vxr_box_world* world, int64_t* out4);

/* The narrow phase alone over a caller's pair list: replaces the collide pass BoxContact.collide
 * (core/box/BoxContact.java:136-246) as the reference's BoxContactTest runs it. fields18 as for
 * vxr_box_load_state; pairs = first, second, ... (second -1: an empty slot); manifold40 receives 40 floats a pair. */
int32_t vxr_collide(int32_t bodies, const float* const* fields18, const int32_t* params18, int32_t npairs,
                    const int32_t* pairs, float* manifold40);

/* The broad phase with no allocation. No counterpart in the reference: it exists for callers that cannot allocate
 * device memory while they step bodies — a host that owns all device memory through its own pool, or code that
 * must not allocate (an allocation synchronises the device) between the launches it is recording or under a
 * frame deadline. It runs the same bin, stable counting sort, neighbourhood list and compaction kernels as a
 * world's step and writes the candidate pairs, sorted by (first, second), to the caller's device arrays first_out
 * and second_out (capacity entries each). All its scratch lives in one array of about 6 MiB in this library's
 * device memory, which every GPU that loads the library holds until the process exits; nothing is allocated.
 *   Limits: at most 16384 bodies and 262144 grid cells a call; beyond them the call returns VXR_ECAPACITY and does
 *   nothing.
 *   reach_cells: the neighbourhood's half-width in cells, 0 or 1 for the 27 cells, at most the grid's widest side
 *   (max of nx, ny, nz: a wider reach finds no more pairs); a negative or wider value returns VXR_EINVAL.
 *   fields11: device pointers to x y z qx qy qz qw hx hy hz shape (bodies floats each).
 *   result3: a device array that receives [candidate pairs found (may exceed capacity), partners beyond 32 slots,
 *   VXR_OK or VXR_ECAPACITY (more pairs than capacity: the first capacity are written)].
 *   stream: the cudaStream_t to run on (NULL: the default stream); the call does not wait.
 * Every call looks up the array's address on the current device (cudaGetSymbolAddress, which allocates nothing), so
 * the address stays right after cudaDeviceReset. The first call on a device may load the library's kernels onto it
 * and should come before any stream capture. Every call shares the array and it keeps the last call's contents:
 * calls whose work overlaps on the GPU (other streams, other host threads) race, so order them on one stream. */
int32_t vxr_box_broadphase_static(int32_t bodies, const float* const* fields11, vxr_grid grid, int32_t reach_cells,
                                  float margin, int32_t* first_out, int32_t* second_out, int32_t capacity,
                                  int32_t* result3, void* stream);

/* ---- Batched scenes -----------------------------------------------------------------------------------------------
 * Many independent scenes stepped as one world: no reference counterpart (the reference runs one BoxStep a scene,
 * core/box/BoxStep.java:81-162). Bodies are numbered scene after scene; each scene has its own grid (cells in one
 * key space, end to end, so no body meets another scene's) and its own gravity, walls and friction. The substep,
 * margin, softness and push are one for the batch. Every scene's step is the one a world of that scene alone would
 * take, bit for bit: greedy colouring gives each scene's pairs the rounds they get alone. */
typedef struct {
    int32_t scenes;
    const int32_t* bodies;   /* [scenes] bodies of each scene */
    const vxr_grid* grids;   /* [scenes] each scene's grid (vxr_box_make_grid over its own walls) */
    int32_t substeps, sweeps, symmetric, max_pairs, device, schedule, solve_blocks_per_sm;
} vxr_batch_config;

vxr_box_world* vxr_box_create_batch(const vxr_batch_config* config, int32_t* status);
/* Each scene's 18 parameter words ([scenes * 18], as vxr_box_make_params makes them); VXR_EINVAL where a scene's
 * substep, margin, softness or push differs from scene 0's. Needed before a batch's first step. vxr_box_params on a
 * batch gives every scene the same words. */
int32_t vxr_box_scene_params(vxr_box_world* world, const int32_t* params);
/* The batch's scene count (0 for a single scene); first_body (scenes + 1 entries, may be null) receives each
 * scene's first body and the total. */
int32_t vxr_box_scenes(const vxr_box_world* world, int32_t* first_body);

/* Diagnostics computed on the GPU where the state lies: BoxDiagnostics.of (core/box/BoxDiagnostics.java:18-43:
 * kinetic energy with the spin's 1/2 L.w, momentum, angular momentum about the origin, in doubles), the potential
 * energy against each body's gravity, the deepest overlap at the last step's contact points (their gaps measured
 * again from the present poses), the farthest any body reaches past a wall, the fastest body, and whether any state
 * word is not finite. */
typedef struct {
    double kinetic, rotational, potential, momentum[3], angular[3];
    double max_penetration, max_wall_penetration, max_speed;  /* metres, metres, metres a second */
    int32_t broken, pad;
} vxr_box_diag;
int32_t vxr_box_diagnostics(vxr_box_world* world, vxr_box_diag* out);

/* The positional complementarity error (metres) at each contact point of the last step, from the state at its end:
 * the larger of h max(0, -(vn + max(gap, 0) / h)) (for a point within the margin: how deep the relative normal
 * velocity would close within a substep beyond the gap) and max(0, -gap) (the overlap). No reference counterpart:
 * the reference has no residual; this is the measure a solve's quality is judged by. out receives 4 rows a touching
 * pair (round order), -1 past a pair's point count. Returns the row count (out NULL: only the count), or minus a
 * status. */
int32_t vxr_box_contact_errors(vxr_box_world* world, float* out, int32_t capacity);

/* `pairs` x 2 steps as replays of one CUDA graph holding two whole steps, enqueued without waiting (vxr_box_sync
 * waits and reports). The first call captures the graph; changing the parameters, the measuring switches or the
 * state captures it again at the next call. Profiling and tracing must be off. */
int32_t vxr_box_step_graph(vxr_box_world* world, int32_t pairs);

/* ---- The learned warm start's network ---------------------------------------------------------------------------
 * No reference counterpart: the reference warm-starts a contact with the impulses it took last step
 * (core/box/BoxPairs.java:191-267). This is a 16 -> 64 -> 64 -> 2 multilayer perceptron with SiLU activations, BF16
 * weights and activations, FP32 accumulation, run and trained by this library's tcgen05 kernels; it predicts a
 * contact's starting normal and friction impulse from 16 local features (vxr_box_features gives them). Parameters are
 * FP32 masters in the order w1 [16][64], b1 [64], w2 [64][64], b2 [64], w3 [64][2], b3 [2]. */
#define VXR_MLP_PARAMS 5378
typedef struct vxr_mlp vxr_mlp;
/* A network with He-initialised weights from `seed`, on `device`. */
vxr_mlp* vxr_mlp_create(int32_t device, uint64_t seed, int32_t* status);
void vxr_mlp_destroy(vxr_mlp* net);
const char* vxr_mlp_error(const vxr_mlp* net);
/* Parameters and the inputs' normalisation (x - mean) * inv_std; any pointer may be null (kept). Setting the
 * parameters restarts Adam. */
int32_t vxr_mlp_set(vxr_mlp* net, const float* params, const float* mean16, const float* inv_std16);
int32_t vxr_mlp_get(vxr_mlp* net, float* params, float* mean16, float* inv_std16);
/* Forward over `rows` host rows of 16 features: out2 receives (normal, friction) a row. */
int32_t vxr_mlp_forward(vxr_mlp* net, const float* features, int32_t rows, float* out2);
/* The gradients of the loss sum over rows |y - t|^2 / rows at the current parameters (no update), and the loss. */
int32_t vxr_mlp_gradients(vxr_mlp* net, const float* features, const float* targets, int32_t rows, float* grads,
                          float* loss);
/* Adam (beta 0.9, 0.999, eps 1e-8) at learning rate lr over `epochs` shuffled passes of minibatches of `batch`
 * rows; the normalisation is set from the training features first. epoch_loss (may be null) receives each epoch's
 * mean minibatch loss. */
int32_t vxr_mlp_train(vxr_mlp* net, const float* features, const float* targets, int32_t rows, int32_t epochs,
                      int32_t batch, float lr, uint64_t seed, float* epoch_loss);

/* The learned warm start in a box world. mode 0: off (the reference's carried impulses); 1: each step gathers 16
 * features a contact point at its start and the impulses its solve reached (vxr_box_features reads them); 2: each
 * step starts every contact point from `net`'s predicted normal and friction impulse instead of the carried ones;
 * 3: only the points that carried nothing (new contacts) start from the prediction, the others keep theirs.
 * Features: gap, relative normal and tangential speed, the two inverse masses, the two inverse inertias along the
 * normal, the carried normal and friction impulse, the two bodies' touching pair counts, the feature kind one-hot
 * (face of first, face of second, edge, sphere) and the normal's vertical component; impulses (carried, targets and
 * predictions) in units of the pair's effective mass x |g| x h. */
int32_t vxr_box_learned(vxr_box_world* world, vxr_mlp* net, int32_t mode);
/* A measurement: the following steps run only their first `count` substeps (the broad and narrow phase, the carry
 * and the colouring as in a whole step, then `count` substeps of the solve); 0 or the world's substep count restores
 * whole steps. solve_only = 1: the last of them skips its relax sweeps. With the learned warm start's gathering
 * (mode 1), the targets are then the impulses the first substeps reached: with solve_only, what the last one's solve
 * sweeps reached, the impulses that solve would start from to need no sweep. No reference counterpart. */
int32_t vxr_box_first_substeps(vxr_box_world* world, int32_t count, int32_t solve_only);
/* A measurement of what a perfect predictor could gain: the next step starts its contact points from what
 * `answers` (a world that gathers targets, mode 1) reached in its last step, point for point, in place of the carried
 * impulses (fresh_only = 1: only the points that carried nothing). whole = 0: the scaled normal and friction impulse
 * the network predicts (vxr_box_features' targets), applied as its predictions are; whole = 1: the whole impulse
 * records (normal, friction vector and rolling impulse of every point) and, unless fresh_only, the walls' records.
 * The points are matched by touching pair, so the two worlds must be twins: the same state and carried pairs before
 * that step (load the same state into both and step them alike). Everything is copied at the call, so `answers` may
 * be stepped or destroyed afterwards; vxr_box_learned(world, NULL, 0) ends it. No reference counterpart. */
int32_t vxr_box_learned_given(vxr_box_world* world, const vxr_box_world* answers, int32_t fresh_only, int32_t whole);
/* The last step's gathered rows, one a contact point: features16 (rows x 16) and targets2 (rows x 2), the first
 * `capacity` rows written; *rows receives their number. */
int32_t vxr_box_features(vxr_box_world* world, float* features16, float* targets2, int32_t capacity, int32_t* rows);

/* ---- The sphere package: XPBD spheres (core/sphere/) ------------------------------------------------------------
 * The reference's SphereSimulation (gui/SphereSimulation.java:33-295) over SphereStep and SphereStepper. A call of
 * steps is one persistent kernel: every pass of every substep, and Gauss-Seidel's run until done with the
 * stepper's batch sizing, happen on the device with no host wait between them. */

#define VXR_SPHERE_PARAM_COUNT 13       /* core/sphere/Spheres.java:141 */
#define VXR_SPHERE_SHOWN_STRIDE 40      /* core/sphere/Spheres.java:1654 */
#define VXR_SPHERE_FIELDS 24            /* core/sphere/Spheres.java:240-241 */
#define VXR_MOST_LISTED_SPHERES 46340   /* core/sphere/Spheres.java:787 */
#define VXR_SPHERE_ONE_BLOCK 8192       /* scenes up to this many spheres run on one block or one cluster */
#define VXR_SPHERE_CLUSTER_FROM 256     /* ... on a cluster from this many spheres (by default) */
#define VXR_SPHERE_CLUSTER 8            /* ... of this many blocks */
#define VXR_SPHERE_CLUSTER_WIDE_FROM 2048  /* ... and from this many spheres */
#define VXR_SPHERE_CLUSTER_WIDE 16     /* ... of this many */
/* How a pass solves (SphereStep.Solve, core/sphere/SphereStep.java:37-43). */
#define VXR_JACOBI 0
#define VXR_GAUSS_SEIDEL_BY_CONTACT 1   /* run until every contact is solved (SphereStepper) */
#define VXR_FIXED_ROUNDS 2              /* the same with `rounds` rounds a pass and no friction rounds (step()) */

typedef struct vxr_sphere_world vxr_sphere_world;

/* SphereStep(spheres, substeps, iterations, grid, solve, rounds, contactsPerSphere)
 * (core/sphere/SphereStep.java:115-131). */
typedef struct {
    int32_t spheres;
    int32_t substeps;
    int32_t iterations;
    int32_t solve;                /* VXR_JACOBI, VXR_GAUSS_SEIDEL_BY_CONTACT or VXR_FIXED_ROUNDS */
    int32_t rounds;               /* VXR_FIXED_ROUNDS: rounds a pass (SphereStep.ROUNDS = 32) */
    int32_t contacts_per_sphere;  /* list places a sphere; 0 = 6 (SphereStep.CONTACTS_PER_SPHERE) */
    vxr_grid grid;                /* nx = 0: every pair (Jacobi only) */
    int32_t device;
    int32_t blocks;               /* 0: up to VXR_SPHERE_ONE_BLOCK spheres one block (a cluster of
                                     VXR_SPHERE_CLUSTER from VXR_SPHERE_CLUSTER_FROM, of VXR_SPHERE_CLUSTER_WIDE
                                     from VXR_SPHERE_CLUSTER_WIDE_FROM), else enough for the list */
    int32_t cluster;              /* 2 to 16: the step runs on one thread-block cluster of this many blocks (one an
                                     SM), its passes separated by the cluster's barrier; 0: as `blocks` says */
} vxr_sphere_config;

/* SphereStepper.Report(waits, rounds, mostRounds, unlisted) (core/sphere/SphereStepper.java:40-47) of the call's
 * last step, and the same summed over the call's steps (most rounds: the largest). `waits` counts the batches of
 * rounds the reference's host would have waited for; here no host wait happens inside a call. */
typedef struct {
    int32_t waits, rounds, most_rounds, unlisted;
    int64_t waits_total, rounds_total;
    int32_t most_rounds_total;
    int32_t status;
    int64_t unlisted_total;
    int32_t listed;               /* the last substep's list length (contactCount[LISTED]) */
    int32_t pad;
} vxr_sphere_report;

/* Spheres.params (core/sphere/Spheres.java:212-228): 13 float words as int bits into out13; VXR_EINVAL where the
 * reference throws IllegalArgumentException. */
int32_t vxr_sphere_make_params(double h, double gx, double gy, double gz, double sx, double sy, double sz,
                               double omega, int32_t averaged, double restitution, double mu_static,
                               double mu_kinetic, double mu_rolling, int32_t* out13);
/* SphereGrid.covering(sx, sy, sz, widest) (core/sphere/SphereGrid.java:21-26). */
int32_t vxr_sphere_make_grid(double sx, double sy, double sz, double widest, vxr_grid* out);

/* new SphereStep(...) + new SphereSimulation(context, step) (gui/SphereSimulation.java:62-97). NULL on failure,
 * with the reason in *status. */
vxr_sphere_world* vxr_sphere_create(const vxr_sphere_config* config, int32_t* status);
/* SphereSimulation.close() (gui/SphereSimulation.java:288-295). */
void vxr_sphere_destroy(vxr_sphere_world* world);
const char* vxr_sphere_error(const vxr_sphere_world* world);

/* SphereSimulation.start(x, y, z, u, v, w, r, im, params) (gui/SphereSimulation.java:154-178): every buffer cleared,
 * these written, every orientation the identity, the picture's before and after both this state; friction on
 * when the parameters have any (Spheres.rubs). */
int32_t vxr_sphere_start(vxr_sphere_world* world, const float* x, const float* y, const float* z, const float* u,
                         const float* v, const float* w, const float* r, const float* im, const int32_t* params13);
/* The test fixture's start (ctest/sphere/Scene.java:122-158): every buffer cleared, then any of the 24 fields
 * (Spheres.SPHERE order: x y z u v w r im cx cy cz dx dy dz ax ay az tx ty tz qx qy qz qw; a null entry leaves it
 * zero, qw one) and the parameters; the picture's buffer zero. */
int32_t vxr_sphere_load_state(vxr_sphere_world* world, const float* const* fields24, const int32_t* params13);
/* Both starts refuse a state holding a NaN or an infinity with VXR_ENONFINITE and load nothing: such a state is
 * what the reference's diagnostics flag as broken (core/sphere/SphereDiagnostics.java:48-50). */
/* SphereSimulation.params(int[]) (gui/SphereSimulation.java:181-184): from the next step on. */
int32_t vxr_sphere_params(vxr_sphere_world* world, const int32_t* params13);
/* SphereStepper.friction(boolean) (core/sphere/SphereStepper.java:106-112): whether passes run friction rounds. */
int32_t vxr_sphere_friction(vxr_sphere_world* world, int32_t on);
/* The rounds a Gauss-Seidel pass run until done may take before the step stops with VXR_EROUNDS, "a pass is still
 * open" (core/sphere/SphereStepper.java:79,86-88); 0 (the default) is the reference's limit, the list's capacity
 * plus two cycles of rounds. Each round solves at least the open contact of highest priority, so an honest pass
 * never reaches the default; a lower limit makes a pass that needs more rounds an error, as the reference's test
 * does with a runner that never closes (ctest/sphere/SphereStepperTest.java:163-166). */
int32_t vxr_sphere_round_limit(vxr_sphere_world* world, int32_t rounds);

/* SphereSimulation.stepAndWait() (gui/SphereSimulation.java:196-199): `steps` steps, waiting for them. */
int32_t vxr_sphere_step(vxr_sphere_world* world, int32_t steps, vxr_sphere_report* report);
/* SphereSimulation.step() (gui/SphereSimulation.java:191-193): enqueued without waiting; vxr_sphere_sync waits. */
int32_t vxr_sphere_step_async(vxr_sphere_world* world, int32_t steps);
int32_t vxr_sphere_sync(vxr_sphere_world* world, vxr_sphere_report* report);
/* The world's cudaStream_t. */
void* vxr_sphere_stream(vxr_sphere_world* world);

/* SphereSimulation.state() (gui/SphereSimulation.java:256-260): x y z u v w ax ay az into out9 (null entries
 * skipped). */
int32_t vxr_sphere_state(vxr_sphere_world* world, float* const* out9);
/* Any one of the 24 fields (Scene.floats, ctest/sphere/Scene.java:207-210). */
int32_t vxr_sphere_field(vxr_sphere_world* world, int32_t field, float* out);
/* SphereSimulation.readShown() (gui/SphereSimulation.java:266-268): 40 floats a sphere. */
int32_t vxr_sphere_read_shown(vxr_sphere_world* world, float* out);
/* The last substep's contact list in list order, for inspection: pairs (lower, higher), the pass that solved each,
 * and its 7 impulse words (normal, tangential 3, angular 3); *listed receives its length (the first `capacity`
 * entries are written). */
int32_t vxr_sphere_contacts(vxr_sphere_world* world, int32_t* ab, int32_t* done, float* impulses7,
                            int32_t capacity, int32_t* listed);
/* The walls' impulses, 21 floats a sphere (Spheres.WALL_IMPULSE_WORDS, core/sphere/Spheres.java:952). */
int32_t vxr_sphere_walls(vxr_sphere_world* world, float* out);
/* contactCount: listed, missed, longest (core/sphere/Spheres.java:797-804). */
int32_t vxr_sphere_counts(vxr_sphere_world* world, int32_t* out3);
/* SphereDiagnostics.of (core/sphere/SphereDiagnostics.java:34-83) computed on the GPU: the deepest overlap between
 * two spheres over the smaller radius (searched in each sphere's grid neighbourhood as the last substep sorted them,
 * every pair without a grid), the farthest past a wall over the radius, kinetic energy with spin, the spin's part,
 * potential energy (-gy y), momentum, angular momentum about the origin, the fastest speed, non-finite state. */
typedef struct {
    double kinetic, rotational, potential, momentum[3], angular[3];
    double max_overlap, max_wall, max_speed;
    int32_t broken, pad;
} vxr_sphere_diag;
int32_t vxr_sphere_diagnostics(vxr_sphere_world* world, vxr_sphere_diag* out);

/* Blocks the world's kernel runs on (a cluster chosen by default that the GPU cannot place falls back to 8 blocks,
 * then to one: this says which was taken), and kernels its steps have launched (reading the state back is not
 * counted). */
int32_t vxr_sphere_blocks(const vxr_sphere_world* world);
int64_t vxr_sphere_launches(const vxr_sphere_world* world);

/* ---- The picture's hand-off: a ring of finished steps ------------------------------------------------------------
 * The reference's ShownRing (gui/ShownRing.java:37-177) with device buffers for its three slots: one the reader's
 * front, one ready (the newest finished step it has not taken), the rest free, the next step kept in one of them. A
 * slot's CUDA event stands for the reference's timeline value; a reader's stream waits on it (vxr_ring_wait) before it
 * reads the slot. A new simulation installs a new generation; the old one is retired once the reader has taken from
 * the new, and freed when the writer collects it (vxr_ring_retired). Thread-safe: one writer thread, one reader. */
#define VXR_RING_SPHERES 0   /* VXR_SPHERE_SHOWN_STRIDE floats a body (ShownRing.Shape.SPHERES) */
#define VXR_RING_BOXES 1     /* VXR_SHOWN_STRIDE floats a body */
typedef struct vxr_ring vxr_ring;
/* ShownRing.Frame (gui/ShownRing.java:88-96), with where its slot lies and the event to wait on. */
typedef struct {
    int64_t generation, step, finished_ns, words;
    int32_t slot, shape, bodies, pad;
    double extent[3];
    const float* data;  /* device pointer of the slot */
    void* event;        /* cudaEvent_t: the slot's contents are complete once it has fired */
} vxr_frame;
vxr_ring* vxr_ring_create(int32_t device);
void vxr_ring_destroy(vxr_ring* ring);
const char* vxr_ring_error(const vxr_ring* ring);
/* ShownRing.install: a generation of `bodies` bodies of `shape` in a box of extent3; returns its id (from 1) or
 * minus a status. bodies = 0: the roles alone, no buffers (for a caller that keeps its own). */
int64_t vxr_ring_install(vxr_ring* ring, int32_t shape, int32_t bodies, const double* extent3);
/* ShownRing.back: the slot the next step is kept in. */
int32_t vxr_ring_back(vxr_ring* ring);
/* ShownRing.publish: the step kept in back() is finished. */
int32_t vxr_ring_publish(vxr_ring* ring, int64_t step, int64_t finished_ns);
/* The writer's keep (Spheres.keep / Boxes.keep and publish): `words` floats of `shown` (a device pointer, e.g.
 * vxr_box_shown_device) copied into the back slot on `stream`, the slot's event recorded after it, then published. */
int32_t vxr_ring_keep(vxr_ring* ring, const float* shown, int64_t words, void* stream, int64_t step);
/* ShownRing.take: the newest finished step as the front (or the front as it was); returns 1 before any step has been
 * published, VXR_OK otherwise. */
int32_t vxr_ring_take(vxr_ring* ring, vxr_frame* out);
/* The reader's stream waits for the frame's slot to be complete. */
int32_t vxr_ring_wait(const vxr_frame* frame, void* stream);
/* The frame's slot copied to host memory once it is complete (frame->words floats): the picture handed to a reader
 * on another device, as ShownSlots.on reads it (gui/ShownSlots.java:35-156). */
int32_t vxr_ring_read(const vxr_frame* frame, float* out);
/* ShownRing.retired: generations the reader has moved past, each once; their slots are freed here. Returns how many,
 * their ids in ids (capacity entries at most). */
int32_t vxr_ring_retired(vxr_ring* ring, int64_t* ids, int32_t capacity);
/* The generations still live (not freed), the current one included. */
int32_t vxr_ring_live(vxr_ring* ring, int64_t* ids, int32_t capacity);
/* The world's resident `shown` (RigidSimulation.shown, gui/RigidSimulation.java:33-37): its device address, and its
 * length in floats into *words. */
const float* vxr_box_shown_device(vxr_box_world* world, int64_t* words);
const float* vxr_sphere_shown_device(vxr_sphere_world* world, int64_t* words);

/* ---- The picture: one ray a pixel against every body, into a headless RGB buffer -----------------------------------
 * The reference's fragment shaders as CUDA: Picture.java (camera ray, sky, checkered floor, light), SphereShader.java
 * (squashed spheres painted in octants) and BoxShader.java (slab test, edge band, sphere-shaped bodies). The push
 * constants of Picture.push (gui/Picture.java:202-216), as f32: */
typedef struct {
    float eye[3], right[3], up[3], forward[3]; /* right, up, forward unit length */
    float aspect;  /* width / height */
    float alpha;   /* how far between the last two steps to show the bodies, 0 to 1 */
    float extent[3];
    float squash;  /* spheres only: 0 not squashed, 1.5 overlaps just closed */
} vxr_camera;
/* `count` bodies of `shape` (VXR_RING_SPHERES / VXR_RING_BOXES) from `shown` (a device pointer, e.g. a ring
 * frame's data or vxr_*_shown_device) drawn into rgb (device, width * height * 3 floats, row 0 the top) on `stream`.
 * Pixel (i, j) is the one at uv ((i + 0.5) / width, (j + 0.5) / height). */
int32_t vxr_picture(int32_t shape, const float* shown, int32_t count, const vxr_camera* camera, int32_t width,
                    int32_t height, float* rgb, void* stream);
/* The same from and into host memory (a picture for a file or a reader without a device). */
int32_t vxr_picture_host(int32_t shape, const float* shown_host, int32_t count, const vxr_camera* camera,
                         int32_t width, int32_t height, float* rgb_host);

#ifdef __cplusplus
}
#endif

#endif /* VXR_H */
