// The box/mixed-body step on one B200: broad phase, narrow phase, warm-start carry, colouring and the
// coloured soft-step solve, all on the device, one stream per world, no host round trip inside a step.
//
// The step the reference runs (paths inside sibarum/vexelray-sim-rigid, core =
// vexelray-sim-rigid-core/src/main/java/dev/vexelray/sim/rigid/):
//   core/box/BoxStep.java:141-158  collide list: keep, bin, sort, list, collide, carry, counts
//   core/box/BoxStepper.java:56-100    host wait, greedy colouring, rounds written, substeps run
//   core/box/BoxStep.java:199-231  per substep: velocities, WARM sweep, sweeps x SOLVE, positions, sweeps x RELAX;
//                                  each sweep every round of pairs then the walls (reversed: walls first)
// Here the same passes run as device kernels in one stream. What changes is the layout and the scheduling:
//   * body state is five float4 arrays (pose+im, turn, half+shape, velocity, angular momentum);
//   * the 32 slots per body are compacted into a candidate list sorted by (first, second), the slot order;
//   * only touching pairs carry manifolds' solve data and impulses, double-buffered so "keep" is a swap;
//   * the host's greedy colouring becomes a device colouring that reproduces it exactly (a pair's round is the
//     least round free of the rounds of the lower-numbered pairs sharing a body, computed in dependency waves);
//   * all substeps of a step run in one cooperative kernel, a bounded grid barrier between phases;
//   * wall contacts that hold no impulse and whose body is far from every wall are skipped without loading
//     their records (a per-body bit mask says which records are nonzero).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "body_math.cuh"
#include "grid_sync.cuh"
#include "narrow.cuh"
#include "scan.cuh"
#include "vxr.h"

namespace vxr {

constexpr int SLOTS = 32;
constexpr int MOST_ROUNDS = 32;
constexpr int WALL_RECORDS = 48;
constexpr int SHOWN_STRIDE = 20;
constexpr int THREADS = 256;
constexpr int SOLVE_THREADS = 256;
// Within a round, pairs are grouped by kind so a warp's lanes take the same path: two spheres, a sphere and a box,
// then two boxes by point count (1 to 4).
constexpr int PAIR_KINDS = 6;
constexpr int BUCKETS = (MOST_ROUNDS + 1) * PAIR_KINDS;
// Pairs are bucketed by path, then round, then kind: path 0 the pairs the grid phases solve (bodies of a component
// too large for one block, and every unplaced pair), path 1 the pairs of the small components the island blocks solve.
constexpr int ALL_BUCKETS = 2 * BUCKETS;
// Islands: connected components of the placed touching pairs. A component of at most ISLAND_MOST bodies is solved
// whole by one block, its bodies in shared memory, its rounds apart by block barriers; larger ones go through the grid
// phases. Components are packed into groups in order of their roots: a group takes components until `base` bodies
// have been placed, so it holds at most base + ISLAND_MOST - 1 bodies. The base is chosen each step so that the island
// blocks take one group each where the small components' bodies allow it (group_base_of).
constexpr int ISLAND_MOST = 256;
constexpr int GROUP_BASE_LEAST = 256;
constexpr int GROUP_CAP = 640;  // a group's bodies in a block's shared memory (44 KB, under the 48 KB of static memory)
constexpr int GROUP_ROUNDS = MOST_ROUNDS;                // placed pairs only
constexpr int GROUP_LISTS = GROUP_ROUNDS * PAIR_KINDS;  // a group's pairs listed by (round, kind)
constexpr int ISLAND_THREADS = 256;                      // a block a group

// Bodies placed before a group's components stop: the small components' bodies shared evenly by the island blocks,
// at least GROUP_BASE_LEAST and at most GROUP_CAP - ISLAND_MOST (a group then holds at most GROUP_CAP - 1 bodies).
// With 107,445 such bodies and 296 blocks (the large scene early in its drop) that is 363: 296 groups, where a base of
// 256 made 420 and left 124 blocks two groups in turn.
__host__ __device__ inline int group_base_of(int island_bodies, int blocks) {
    const int even = (island_bodies + (blocks > 0 ? blocks : 1) - 1) / (blocks > 0 ? blocks : 1);
    return even < GROUP_BASE_LEAST ? GROUP_BASE_LEAST : (even > GROUP_CAP - ISLAND_MOST ? GROUP_CAP - ISLAND_MOST : even);
}

// ------------------------------------------------------------------------------------------------------------
// Device buffers of a world.
struct Bodies {
    float4 *pose, *turn, *half, *vel, *mom;  // (x, y, z, im), (qx, qy, qz, qw), (hx, hy, hz, shape), (u, v, w, 0), (L, 0)
    float4* inv;  // inverse principal moments (Boxes.inverseInertia), fixed once the bodies are loaded
};

struct Manifolds {  // the narrow phase's output, by candidate pair (the current step's)
    float4* head;  // [cap] normal, point count
    float* axis;   // [cap] the winning axis
    float4* pa;    // [cap * 4] anchor on the first body, depth
    float4* pb;    // [cap * 4] anchor on the second body
};

// One generation of the touching pairs, in round order (the order the solve reads them), with everything the
// solve needs and the impulses they carry. The step before's generation is what the carry reads.
struct PairGen {
    int* tstart;     // [n+1] first touching pair of each body, in slot order
    int* tb;         // [cap] second body of touching pair t (slot order)
    int* pos;        // [cap] round-order position of touching pair t
    int4* pair;      // [cap] by position: first, second, point count, packed round ranks (k_order)
    float4* normal;  // [cap] by position: normal, winning axis
    int* pstart;     // [cap] by position: where its points begin in the point arrays below
    // The point arrays hold a pair's points at pstart[position] + point, packed: a pair of one point takes one
    // entry, so the lanes of a warp, holding neighbouring positions, read neighbouring entries.
    float4* pa;      // [cap * 4] by point: anchor on first, depth
    float4* pb;      // [cap * 4] by point: anchor on second
    float4* imp;     // [cap * 4] by point: normal impulse, tangential impulse
    float4* impr;    // [cap * 4] by point: rolling impulse
    float4* prepA;   // [cap * 4] by point, this half-substep: anchor on first in the world's frame, gap
    float4* prepB;   // [cap * 4] by point, this half-substep: anchor on second in the world's frame, k normal
};

struct Counters {  // device-side counts of a step
    int candidates;     // candidate pairs listed
    int touching;       // touching pairs
    int points;         // their points
    int rounds;         // rounds used
    int unplaced;       // touching pairs with no round
    int unlisted;       // partners found beyond the 32 slots
    int status;         // ST_*
    int colour_waves;   // dependency waves the colouring took
    int abort;
    unsigned int bar_count, bar_gen;
    int remaining[3];
    int trace_len;
    int grid_rounds;  // rounds the grid phases' pairs (path 0) use
    int grid_n;       // bodies the grid phases move (components beyond a warp)
    int free_n;       // bodies in no placed pair
    int work;         // the island kernel's work counter
    int largest;      // bodies of the largest component
    int all_grid;     // a component too large for a block: every body through the grid phases
};

struct Totals {  // accumulated over the steps of one vxr_box_step call
    int last[5];
    int most_rounds;
    long long unplaced, unlisted;
    int status;
    int steps;
};

}  // namespace vxr

using namespace vxr;

struct vxr_box_world {
    int n = 0, substeps = 1, sweeps = 1, symmetric = 0;
    int nx = 1, ny = 1, nz = 1, has_grid = 0, reach_cells = 1;
    float cell = 1.0f;
    int cap = 0;  // candidate / touching capacity
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    Params params{};
    std::string error;
    int sms = 148;
    int solve_blocks = 0, colour_blocks = 0, island_blocks = 0;
    float last_ms = 0.0f;

    Bodies b{};
    float4* wall = nullptr;              // [n * 48] wall records: normal impulse, tangential impulse
    float4* wroll = nullptr;             // [n * 6] sphere rolling impulse against each wall
    unsigned long long* wmask = nullptr;  // [n] bit k: wall record k nonzero; bit 48 + w: roll record w nonzero
    float* shown = nullptr;              // [n * 20]

    int cells = 1;
    int *keys = nullptr, *cell_count = nullptr, *cell_start = nullptr, *cell_fill = nullptr;
    int *order_tmp = nullptr, *order = nullptr;
    float4* reach = nullptr;  // world half-extents of each body (BoxBroad.reach)
    int *partner = nullptr, *found = nullptr, *kept = nullptr, *cand_start = nullptr;
    int *cand_a = nullptr, *cand_b = nullptr;
    int *tcount = nullptr;
    int *scan_tiles = nullptr;
    Manifolds man{};
    int *ta = nullptr, *tcand = nullptr;    // this step's touching pairs in slot order: first body, candidate
    float4 *imp_t = nullptr, *impr_t = nullptr;  // carried impulses in slot order, before the round order
    PairGen gen[2]{};
    int cur = 0;  // gen[cur] is this step's, gen[cur ^ 1] the step before's
    int* wall_list = nullptr;    // [n] bodies near a wall or holding a wall impulse, rebuilt twice a substep
    int* wall_count = nullptr;   // [4 * substeps] their counts (spheres, boxes)
    int* version = nullptr;      // [n] items each body has done in the current block of sweeps
    int* listed = nullptr;       // [n] on the current wall list
    unsigned* body_colours = nullptr;  // [n] rounds each body has a pair in
    int schedule = 0;
    int measure = 0;                   // gather each sweep's residual
    int active_sweeps = 0;             // sweeps a substep runs (at most `sweeps`, the count it was created with)
    float tolerance = 0.0f;            // > 0: stop a substep's sweeps once the residual is this or less
    int* used = nullptr;               // [2 substeps] sweeps each half-substep ran
    int cold = 0;                      // start every step's pair impulses from zero (no carry)
    unsigned* residual = nullptr;      // [substeps * (2 sweeps + 1)]
    unsigned long long* trace = nullptr;  // phase end times of the last traced step
    int trace_cap = 0, tracing = 0;
    int *colour = nullptr, *inc_count = nullptr, *inc_start = nullptr, *inc_fill = nullptr, *inc_list = nullptr;
    int *round_count = nullptr, *round_start = nullptr, *round_fill = nullptr;  // by (round, kind) bucket
    int* bucket_start = nullptr;
    int *bucket_most = nullptr, *bucket_pstart = nullptr;  // by bucket: most points of a pair, first point
    // islands (connected components of the placed touching pairs), rebuilt every step
    int islands = 1;                  // small components solved by warps (0: every body through the grid phases)
    int list_tiled = 0;               // the broad phase's list by tiles of cells staged in shared memory
    unsigned long long wait_limit_ns = 2000000000ull;  // the longest a device-wide wait may last
    int groups_max = 0;               // groups the bodies can fill
    int *parent = nullptr;            // [n] union-find parent
    int *comp = nullptr;              // [n] each body's component: its root
    int *isl_size = nullptr;          // [n] bodies of the component rooted here
    int *isl_key = nullptr;           // [n] a small component's body count at its root, 0 elsewhere
    int *isl_offset = nullptr;        // [n + 1] their exclusive sum: where each small component's bodies begin
    int *isl_fill = nullptr;          // [n] bodies of the component placed so far
    int *body_group = nullptr;        // [n] a small component's group; -1 in no placed pair; -2 on the grid phases
    int *body_local = nullptr;        // [n] its place in the group
    int *group_body = nullptr;        // [groups_max * GROUP_CAP] each group's bodies
    int *group_count = nullptr;       // [groups_max]
    int *group_base = nullptr;        // [groups_max] the place of each group's first component
    int *gr_count = nullptr, *gr_start = nullptr, *gr_fill = nullptr;  // by (group, round, kind)
    int2* ilist = nullptr;            // [cap] island pairs by (group, round, kind): round-order position, local ids
    int *grid_list = nullptr, *free_list = nullptr;  // [n] bodies of the grid phases; bodies in no placed pair
    Counters* counters = nullptr;
    Totals* totals = nullptr;
    Totals* host_totals = nullptr;  // pinned
    float* pinned = nullptr;        // pinned staging for state transfers
    float* state13 = nullptr;       // [13 n] the state split into fields, for vxr_box_state
    // vxr_box_state_async: two slots of split fields, copied out on their own stream while the next step runs
    float* state_slot[2] = {nullptr, nullptr};
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t slot_split[2] = {nullptr, nullptr}, slot_copied[2] = {nullptr, nullptr};
    size_t pinned_bytes = 0;
    std::vector<void*> allocations;
    long long launches = 0;  // kernels this world has launched
    // phase timing: events around the broad phase, the narrow phase, the colouring and the solve of each step
    int profile = 0;
    std::vector<cudaEvent_t> events;  // 5 a step while profiling
    int events_used = 0;
    double phase_ms[4] = {0, 0, 0, 0};
    long long* activity = nullptr;  // device scratch for vxr_box_activity
    float* errors = nullptr;        // vxr_box_contact_errors' rows
    int err_rows = 0;
    // batched scenes (vxr_box_create_batch): each scene's parameter words and grid, each body's scene
    int scenes = 0;
    int scene_params_set = 0;
    Params* scene_params = nullptr;  // [scenes]
    int* body_scene = nullptr;       // [n]
    int4* scene_grid = nullptr;      // [scenes] nx, ny, nz, first key
    float* scene_cell = nullptr;     // [scenes]
    std::vector<int> scene_first;    // [scenes + 1] first body of each scene
    // a captured pair of steps (vxr_box_step_graph)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    long long graph_launches = 0;  // kernels in the captured pair of steps
    int capturing = 0;
    // the learned warm start: 0 off, 1 gather features and targets, 2 start from the network's impulses (3: new
    // contacts only), 4 start from given impulses held in lpred (5: new contacts only), 6 start from given whole
    // impulse records (7: new contacts only)
    int learn_mode = 0;
    int first_substeps = 0;  // a measurement: steps run only their first substeps (0: all)
    int solve_only = 0;      // ... and the last of them skips its relax sweeps
    vxr_mlp* learn_net = nullptr;
    float *lfeat = nullptr, *lpred = nullptr, *ltarget = nullptr;  // [cap * 4 rows] x 16, 2, 2
    float* lgiven = nullptr;  // [cap * 4 rows] x 2: given starts by touching pair (slot order), not by position
    float4 *lgiven_imp = nullptr, *lgiven_impr = nullptr;  // [cap * 4]: whole impulse records by touching pair
};

// The network's forward over rows counted on the device (mlp.cu).
int vxr_mlp_forward_device(vxr_mlp* net, const float* feats, const int* rows_dev, int rows_mult, int rows_max,
                           float* out, cudaStream_t stream);

namespace {

#define VXR_CUDA(call)                                                                                 \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) {                                                                       \
            fail(w, std::string(#call) + ": " + cudaGetErrorString(e_));                               \
            return VXR_ECUDA;                                                                          \
        }                                                                                              \
    } while (0)

int fail(vxr_box_world* w, const std::string& why) {
    if (w) w->error = why;
    return VXR_ECUDA;
}

template <typename T>
int alloc(vxr_box_world* w, T** p, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) {
        w->error = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        return VXR_ECUDA;
    }
    w->allocations.push_back(q);
    *p = (T*)q;
    return VXR_OK;
}

// ------------------------------------------------------------------------------------------------------------
// Broad phase kernels (BoxBroad.java).

struct GridDims {
    int nx, ny, nz;
    float cell;
    int reach;  // neighbourhood half-width in cells
};

// Batched scenes: each body's scene, and each scene's grid (nx, ny, nz, first key) and cell side. The scenes' grids
// lie end to end in one key space, so a body's neighbourhood never leaves its own scene. Null for a single scene.
struct SceneGrids {
    const int* body_scene;
    const int4* grid;
    const float* cell;
};

// The grid a body is binned and searched in: the world's, or its scene's (with that scene's first key).
__device__ __forceinline__ void grid_of(const GridDims& g, const SceneGrids& sg, int s, int& nx, int& ny, int& nz,
                                        int& base, float& cell) {
    nx = g.nx, ny = g.ny, nz = g.nz, base = 0, cell = g.cell;
    if (sg.body_scene) {
        const int sc = sg.body_scene[s];
        const int4 d = sg.grid[sc];
        nx = d.x, ny = d.y, nz = d.z, base = d.w, cell = sg.cell[sc];
    }
}

// bin :74-89, and reach :196-227 for the list.
__global__ void k_bin(int n, GridDims g, SceneGrids sg, const float4* __restrict__ pose,
                      const float4* __restrict__ turn, const float4* __restrict__ half, int* __restrict__ keys,
                      float4* __restrict__ reach, int* __restrict__ cell_count) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 p = pose[s];
    const float at[3] = {p.x, p.y, p.z};
    int gx, gy, gz, base;
    float cell;
    grid_of(g, sg, s, gx, gy, gz, base, cell);
    const int cells[3] = {gx, gy, gz};
    int c[3];
#pragma unroll
    for (int a = 0; a < 3; a++) c[a] = (int)fmaxf(0.0f, fminf((float)(cells[a] - 1), floorf(at[a] / cell)));
    const int key = base + (c[0] + cells[0] * (c[1] + cells[1] * c[2]));
    keys[s] = key;
    atomicAdd(&cell_count[key], 1);
    const float4 q = turn[s];
    const float4 h = half[s];
    const float x = q.x, y = q.y, z = q.z, w = q.w;
    const float r[3][3] = {{1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y - z * w), 2.0f * (x * z + y * w)},
                           {2.0f * (x * y + z * w), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z - x * w)},
                           {2.0f * (x * z - y * w), 2.0f * (y * z + x * w), 1.0f - 2.0f * (x * x + y * y)}};
    float out[3];
#pragma unroll
    for (int a = 0; a < 3; a++) out[a] = (h.x * fabsf(r[a][0]) + h.y * fabsf(r[a][1])) + h.z * fabsf(r[a][2]);
    if (h.w > 0.5f) out[0] = out[1] = out[2] = h.x;
    reach[s] = make_float4(out[0], out[1], out[2], 0.0f);
}

__global__ void k_scatter(int n, const int* __restrict__ keys, const int* __restrict__ cell_start,
                          int* __restrict__ cell_fill, int* __restrict__ order_tmp) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int key = keys[s];
    order_tmp[cell_start[key] + atomicAdd(&cell_fill[key], 1)] = s;
}

// The counting sort made stable: each body's place in its cell is the number of its cell's bodies with a
// lower index, whatever order the atomic scatter left.
__global__ void k_stable(int n, const int* __restrict__ keys, const int* __restrict__ cell_start,
                         const int* __restrict__ order_tmp, int* __restrict__ order) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int key = keys[s];
    const int start = cell_start[key], end = cell_start[key + 1];
    int rank = 0;
    for (int j = start; j < end; j++) rank += order_tmp[j] < s;
    order[start + rank] = s;
}

// list :103-164 with around :230-252: the higher-numbered bodies near s, the first 32 found kept in ascending
// order, and how many were found. With reach > 1 (cells narrower than the reference's rule) the neighbourhood
// widens to (2 reach + 1)^3 cells; at reach 1 it is the reference's 27, visited in its order.
__global__ void k_list(int n, GridDims g, SceneGrids sg, float margin, const float4* __restrict__ pose,
                       const float4* __restrict__ reach, const int* __restrict__ keys,
                       const int* __restrict__ cell_start, const int* __restrict__ order, int* __restrict__ partner,
                       int* __restrict__ found_out, int* __restrict__ kept_out, Counters* counters) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 ps = pose[s];
    const float4 rs = reach[s];
    const float centre[3] = {ps.x, ps.y, ps.z};
    const float rch[3] = {rs.x, rs.y, rs.z};
    int slot[SLOTS];
    int found = 0;
    int gx, gy, gz, base;
    float cell_side;
    grid_of(g, sg, s, gx, gy, gz, base, cell_side);
    const int key = keys[s] - base;
    const int ix = key % gx, iy = (key / gx) % gy, iz = key / (gx * gy);
    const int side = 2 * g.reach + 1;
    const int around = side * side * side;
    for (int nn = 0; nn < around; nn++) {
        const int jx = ix + (nn % side - g.reach);
        const int jy = iy + ((nn / side) % side - g.reach);
        const int jz = iz + (nn / (side * side) - g.reach);
        if (!(jx >= 0 && jx < gx && jy >= 0 && jy < gy && jz >= 0 && jz < gz)) continue;
        const int cell = base + (jx + gx * (jy + gy * jz));
        const int end = cell_start[cell + 1];
        for (int k = cell_start[cell]; k < end; k++) {
            const int o = order[k];
            if (!(o > s)) continue;
            const float4 po = pose[o];
            const float4 ro = reach[o];
            const bool close = !(fabsf(po.x - centre[0]) > (rch[0] + ro.x) + margin) &&
                               !(fabsf(po.y - centre[1]) > (rch[1] + ro.y) + margin) &&
                               !(fabsf(po.z - centre[2]) > (rch[2] + ro.z) + margin);
            if (!close) continue;
            if (found < SLOTS) {
                int place = found;
                while (place > 0) {
                    const int before = slot[place - 1];
                    if (before > o) {
                        slot[place] = before;
                        place--;
                    } else {
                        break;
                    }
                }
                slot[place] = o;
            }
            found++;
        }
    }
    const int kept = found < SLOTS ? found : SLOTS;
    for (int m = 0; m < kept; m++) partner[(long)s * SLOTS + m] = slot[m];
    found_out[s] = found;
    kept_out[s] = kept;
    if (found > SLOTS) atomicAdd(&counters->unlisted, found - SLOTS);
}

// The broad phase's list over a tile of cells (BoxBroad.list :103-164 with around :230-252, reach one cell): a block
// takes TILE_X consecutive cells of one x-row and stages the bodies of their 27-cell neighbourhoods (nine runs of
// the sorted order, one for each (y, z) row: cells along x have consecutive keys) in shared memory, each with its
// centre and its world half-extents. A warp then takes one of the tile's own bodies at a time. Its 32 lanes test 32
// of the body's candidates at once, in the reference's visiting order (the nine rows in turn, each row's three cells
// x-first, each cell in sorted order); a ballot marks the close ones and each found body moves to the lane of its
// place in the found order (popc and __fns over the ballot). The first 32 found, sorted ascending across the lanes
// (bitonic), are the body's slots: the reference's insertion into 32 ascending slots of what it finds, in its order.
// A neighbourhood too large to stage is read from global memory by the same warps.
constexpr int TILE_X = 16;
constexpr int STAGE_CAP = 1280;  // staged bodies a block

__device__ __forceinline__ int bitonic_ascending(int v, int lane) {
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const int other = __shfl_xor_sync(0xffffffffu, v, j);
            const bool up = (lane & k) == 0, lower = (lane & j) == 0;
            v = (lower == up) ? min(v, other) : max(v, other);
        }
    }
    return v;
}

__global__ void __launch_bounds__(256) k_list_tiled(GridDims g, float margin, const float4* __restrict__ pose,
                                                    const float4* __restrict__ reach, const int* __restrict__ keys,
                                                    const int* __restrict__ cell_start, const int* __restrict__ order,
                                                    int* __restrict__ partner, int* __restrict__ found_out,
                                                    int* __restrict__ kept_out, Counters* counters) {
    __shared__ float4 spose[STAGE_CAP], sreach[STAGE_CAP];  // reach .w: the body's index, as bits
    __shared__ int row_base[10];        // staged rows' first places (the last: the total)
    __shared__ int row_first[9];        // each row's first cell key (the staged column xs0), -1 if outside the grid
    __shared__ int staged;              // 1 when the neighbourhood fits in shared memory
    __shared__ int col_start[9][TILE_X + 3];  // staged place where each staged column's cell begins (and the end)
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int tiles_x = (nx + TILE_X - 1) / TILE_X;
    const int tile = blockIdx.x;
    const int tx = tile % tiles_x, iy = (tile / tiles_x) % ny, iz = tile / (tiles_x * ny);
    const int x0 = tx * TILE_X, x1 = min(x0 + TILE_X, nx) - 1;  // the tile's own cells, inclusive
    const int own_lo = cell_start[x0 + nx * (iy + ny * iz)], own_hi = cell_start[x1 + nx * (iy + ny * iz) + 1];
    if (own_lo == own_hi) return;  // no body to list (block-uniform)
    const int xs0 = max(x0 - 1, 0), xs1 = min(x1 + 1, nx - 1);  // the staged columns
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    if (threadIdx.x < 32) {  // the nine rows' runs: their lengths, scanned across the first lanes
        int len = 0, first = -1;
        if (lane < 9) {
            const int jy = iy + (lane % 3 - 1), jz = iz + (lane / 3 - 1);
            if (jy >= 0 && jy < ny && jz >= 0 && jz < nz) {
                first = xs0 + nx * (jy + ny * jz);
                len = cell_start[first + (xs1 - xs0) + 1] - cell_start[first];
            }
        }
        int sum = len;
#pragma unroll
        for (int o = 1; o < 16; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, sum, o);
            if (lane >= o) sum += y;
        }
        if (lane < 9) {
            row_base[lane] = sum - len;
            row_first[lane] = first;
        }
        if (lane == 8) {
            row_base[9] = sum;
            staged = sum <= STAGE_CAP ? 1 : 0;
        }
    }
    __syncthreads();
    const int use_shared = staged;
    if (use_shared) {
        for (int r = 0; r < 9; r++) {
            const int first = row_first[r];
            if (first < 0) continue;
            const int g0 = cell_start[first], base = row_base[r], len = row_base[r + 1] - base;
            for (int i = threadIdx.x; i < len; i += blockDim.x) {
                const int o = order[g0 + i];
                const float4 p = pose[o], q = reach[o];
                spose[base + i] = p;
                sreach[base + i] = make_float4(q.x, q.y, q.z, __int_as_float(o));
            }
            for (int c = threadIdx.x; c <= xs1 - xs0 + 1; c += blockDim.x)
                col_start[r][c] = base + (cell_start[first + c] - g0);
        }
    }
    __syncthreads();
    // A sparse neighbourhood (few candidates a body: about 3 x the staged bodies over the staged columns) would leave
    // most of a warp's lanes idle; then each thread lists one of the tile's bodies itself, walking the staged runs in
    // the same order and keeping its first 32 found in ascending slots as the reference inserts them.
    if (use_shared && 3 * row_base[9] < 24 * (xs1 - xs0 + 1)) {
        for (int i = own_lo + threadIdx.x; i < own_hi; i += blockDim.x) {
            const int s = order[i];
            const float4 ps = pose[s], rs = reach[s];
            const int cx_lo = max(keys[s] % nx - 1, 0) - xs0, cx_hi = min(keys[s] % nx + 1, nx - 1) - xs0;
            int slot[SLOTS];
            int found = 0;
            for (int r = 0; r < 9; r++) {
                if (row_first[r] < 0) continue;
                const int end = col_start[r][cx_hi + 1];
                for (int k = col_start[r][cx_lo]; k < end; k++) {
                    const float4 ro = sreach[k];
                    const int o = __float_as_int(ro.w);
                    if (!(o > s)) continue;
                    const float4 po = spose[k];
                    const bool close = !(fabsf(po.x - ps.x) > (rs.x + ro.x) + margin) &&
                                       !(fabsf(po.y - ps.y) > (rs.y + ro.y) + margin) &&
                                       !(fabsf(po.z - ps.z) > (rs.z + ro.z) + margin);
                    if (!close) continue;
                    if (found < SLOTS) {
                        int place = found;
                        while (place > 0 && slot[place - 1] > o) {
                            slot[place] = slot[place - 1];
                            place--;
                        }
                        slot[place] = o;
                    }
                    found++;
                }
            }
            const int kept = found < SLOTS ? found : SLOTS;
            for (int m = 0; m < kept; m++) partner[(long)s * SLOTS + m] = slot[m];
            found_out[s] = found;
            kept_out[s] = kept;
            if (found > SLOTS) atomicAdd(&counters->unlisted, found - SLOTS);
        }
        return;
    }
    for (int i = own_lo + warp; i < own_hi; i += warps) {
        const int s = order[i];
        const float4 ps = pose[s], rs = reach[s];
        const int ix = keys[s] % nx;
        // this body's nine runs: for row r, the cells ix-1 .. ix+1 inside the grid; lo in staged places (or global
        // order places), and the runs' lengths scanned so every lane can map a candidate's number to its run
        int lo = 0, len = 0;
        if (lane < 9) {
            const int first = row_first[lane];
            if (first >= 0) {
                const int c_lo = first + (max(ix - 1, 0) - xs0), c_hi = first + (min(ix + 1, nx - 1) - xs0);
                const int a = cell_start[c_lo], b = cell_start[c_hi + 1];
                len = b - a;
                lo = use_shared ? row_base[lane] + (a - cell_start[first]) : a;
            }
        }
        int end = len;
#pragma unroll
        for (int o = 1; o < 16; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, end, o);
            if (lane >= o) end += y;
        }
        // every lane holds the nine runs' ends, places and lengths
        int run_end[9], run_lo[9], run_len[9];
#pragma unroll
        for (int k = 0; k < 9; k++) {
            run_end[k] = __shfl_sync(0xffffffffu, end, k);
            run_lo[k] = __shfl_sync(0xffffffffu, lo, k);
            run_len[k] = __shfl_sync(0xffffffffu, len, k);
        }
        const int total = run_end[8];
        int found = 0, mine = 0x7fffffff;  // lane f holds the f-th body found, while f < 32
        for (int base = 0; base < total; base += 32) {
            const int f = base + lane;
            bool close = false;
            int o = 0;
            if (f < total) {
                int at = 0;
                bool seen = false;
#pragma unroll
                for (int k = 0; k < 9; k++) {  // the run this candidate falls in: the first whose end passes f
                    if (!seen && f < run_end[k]) {
                        at = run_lo[k] + (f - (run_end[k] - run_len[k]));
                        seen = true;
                    }
                }
                float4 po, ro;
                if (use_shared) {
                    po = spose[at];
                    ro = sreach[at];
                    o = __float_as_int(ro.w);
                } else {
                    o = order[at];
                    po = pose[o];
                    ro = reach[o];
                }
                close = o > s && !(fabsf(po.x - ps.x) > (rs.x + ro.x) + margin) &&
                        !(fabsf(po.y - ps.y) > (rs.y + ro.y) + margin) &&
                        !(fabsf(po.z - ps.z) > (rs.z + ro.z) + margin);
            }
            const unsigned hits = __ballot_sync(0xffffffffu, close);
            const int got = __popc(hits);
            // lane d takes the (d - found)-th hit of this batch, while d < 32
            const int want = lane - found;
            const int src = (want >= 0 && want < got) ? (int)__fns(hits, 0, want + 1) : lane;
            const int moved = __shfl_sync(0xffffffffu, o, src);
            if (want >= 0 && want < got) mine = moved;
            found += got;
        }
        const int kept = min(found, SLOTS);
        const int sorted = kept > 1 ? bitonic_ascending(mine, lane) : mine;  // kept is the same in every lane
        if (lane < kept) partner[(long)s * SLOTS + lane] = sorted;
        if (lane == 0) {
            found_out[s] = found;
            kept_out[s] = kept;
            if (found > SLOTS) atomicAdd(&counters->unlisted, found - SLOTS);
        }
    }
}

__global__ void k_candidates(int n, int cap, const int* __restrict__ kept, const int* __restrict__ cand_start,
                             const int* __restrict__ partner, int* __restrict__ cand_a, int* __restrict__ cand_b,
                             Counters* counters) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0) {
        const int total = cand_start[n];
        counters->candidates = total;
        if (total > cap) atomicCAS(&counters->status, ST_OK, ST_CAPACITY);
    }
    if (s >= n) return;
    const int base = cand_start[s];
    const int k = kept[s];
    for (int m = 0; m < k; m++) {
        if (base + m < cap) {
            cand_a[base + m] = s;
            cand_b[base + m] = partner[(long)s * SLOTS + m];
        }
    }
}

// ------------------------------------------------------------------------------------------------------------
// Narrow phase: one thread per candidate pair (BoxContact.collide).
__global__ void __launch_bounds__(128) k_collide(const int* __restrict__ cand_start_n, int cap, float margin,
                                                 const int* __restrict__ cand_a, const int* __restrict__ cand_b,
                                                 const float4* __restrict__ pose, const float4* __restrict__ turn,
                                                 const float4* __restrict__ half, float4* __restrict__ head,
                                                 float* __restrict__ axis, float4* __restrict__ pa,
                                                 float4* __restrict__ pb) {
    const int total = min(*cand_start_n, cap);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < total; c += gridDim.x * blockDim.x) {
        const int a = cand_a[c], b = cand_b[c];
        Manifold m;
        collide_pair(pose[a], turn[a], half[a], pose[b], turn[b], half[b], margin, m);
        head[c] = make_float4(m.normal[0], m.normal[1], m.normal[2], (float)m.count);
        axis[c] = m.axis;
        for (int i = 0; i < m.count; i++) {
            pa[(long)c * MOST_POINTS + i] = make_float4(m.a[i][0], m.a[i][1], m.a[i][2], m.depth[i]);
            pb[(long)c * MOST_POINTS + i] = make_float4(m.b[i][0], m.b[i][1], m.b[i][2], 0.0f);
        }
    }
}

// Per body: how many of its candidates touch.
__global__ void k_touch_count(int n, int cap, const int* __restrict__ cand_start, const float4* __restrict__ head,
                              int* __restrict__ tcount) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int k = 0;
    const int end = min(cand_start[s + 1], cap);
    for (int c = cand_start[s]; c < end; c++) k += head[c].w > 0.0f;
    tcount[s] = k;
}

// The touching list in slot order (BoxBroad.counts :174-188 and the order BoxStepper reads it in).
__global__ void k_touch_list(int n, int cap, const int* __restrict__ cand_start, const int* __restrict__ cand_b,
                             const float4* __restrict__ head, const int* __restrict__ tstart, int* __restrict__ ta,
                             int* __restrict__ tb, int* __restrict__ tcand, Counters* counters) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0) counters->touching = tstart[n];
    if (s >= n) return;
    int t = tstart[s];
    int points = 0;
    const int end = min(cand_start[s + 1], cap);
    for (int c = cand_start[s]; c < end; c++) {
        const float cnt = head[c].w;
        if (cnt > 0.0f) {
            ta[t] = s;
            tb[t] = cand_b[c];
            tcand[t] = c;
            points += (int)cnt;
            t++;
        }
    }
    if (points) atomicAdd(&counters->points, points);
}

// BoxPairs.carry :191-267: each new point takes the impulses of the nearest point of the same pair the step
// before (anchor on the first body within 5% of its smallest half-extent), one point to one point always. The
// pair the step before is found among its first body's touching pairs by the partner, as the reference finds its
// slot; pairs that did not touch then carried nothing, as their slots held no points.
__global__ void k_carry(const int* __restrict__ touching_n, const int* __restrict__ ta, const int* __restrict__ tb,
                        const int* __restrict__ tcand, const Manifolds m, const PairGen was,
                        const float4* __restrict__ half, float4* __restrict__ imp_t, float4* __restrict__ impr_t) {
    const int total = *touching_n;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int s = ta[t], partner = tb[t];
        const int c = tcand[t];
        const int count = (int)m.head[c].w;
        int old = -1;
        for (int u = was.tstart[s]; u < was.tstart[s + 1]; u++)
            if (was.tb[u] == partner) old = u;
        int before = 0;
        long wbase = 0;
        if (old >= 0) {
            const long op = was.pos[old];
            before = was.pair[op].z;
            wbase = was.pstart[op];
        }
        const float4 h = half[s];
        const float smallest = fminf(h.x, fminf(h.y, h.z));
        const float reach = (0.05f * smallest) * (0.05f * smallest);
        for (int point = 0; point < MOST_POINTS; point++) {
            float4 t0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), t1 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (point < count) {
                const float4 anchor = m.pa[(long)c * MOST_POINTS + point];
                float nearest = reach;
                for (int o = 0; o < MOST_POINTS; o++) {
                    if (!(o < before)) continue;
                    const float4 then = was.pa[wbase + o];
                    const float gap[3] = {anchor.x - then.x, anchor.y - then.y, anchor.z - then.z};
                    const float d2 = dot3(gap, gap);
                    if (d2 < nearest) {
                        nearest = d2;
                        t0 = was.imp[wbase + o];
                        t1 = was.impr[wbase + o];
                    }
                }
            }
            if (point == 0 && count == 1 && before == 1) {
                t0 = was.imp[wbase];
                t1 = was.impr[wbase];
            }
            imp_t[(long)t * MOST_POINTS + point] = t0;
            impr_t[(long)t * MOST_POINTS + point] = t1;
        }
    }
}

// ------------------------------------------------------------------------------------------------------------
// Colouring (BoxStepper.java:71-90), reproduced exactly on the device.
//
// The host's greedy pass puts each touching pair, in slot order, into the first of 32 rounds holding neither of
// its bodies. So a pair's round is the least round not used by the lower-numbered touching pairs that share a
// body with it (unplaced pairs use none); it depends on those pairs alone. Waves of the cooperative kernel below
// give every pair whose lower-numbered neighbours all have rounds its round, until none is left.

__global__ void k_inc_count(const int* __restrict__ touching_n, const int* __restrict__ ta,
                            const int* __restrict__ tb, int* __restrict__ inc_count) {
    const int total = *touching_n;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        atomicAdd(&inc_count[ta[t]], 1);
        atomicAdd(&inc_count[tb[t]], 1);
    }
}

__global__ void k_inc_fill(const int* __restrict__ touching_n, const int* __restrict__ ta,
                           const int* __restrict__ tb, const int* __restrict__ inc_start, int* __restrict__ inc_fill,
                           int* __restrict__ inc_list) {
    const int total = *touching_n;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int a = ta[t], b = tb[t];
        inc_list[inc_start[a] + atomicAdd(&inc_fill[a], 1)] = t;
        inc_list[inc_start[b] + atomicAdd(&inc_fill[b], 1)] = t;
    }
}

__device__ __forceinline__ bool lower_rounds(int t, int body, const int* inc_start, const int* inc_list,
                                             const int* colour, unsigned int& used) {
    for (int k = inc_start[body]; k < inc_start[body + 1]; k++) {
        const int u = inc_list[k];
        if (u < t) {
            const int cu = *(volatile const int*)&colour[u];
            if (cu < 0) return false;
            if (cu < MOST_ROUNDS) used |= 1u << cu;
        }
    }
    return true;
}

__global__ void __launch_bounds__(THREADS) k_colour(const int* __restrict__ touching_n, const int* __restrict__ ta,
                                                    const int* __restrict__ tb, const int* __restrict__ inc_start,
                                                    const int* __restrict__ inc_list, int* colour,
                                                    Counters* counters, GridBarrier bar) {
    const int total = *touching_n;
    const int threads = gridDim.x * blockDim.x;
    const int me = blockIdx.x * blockDim.x + threadIdx.x;
    // Each thread takes a contiguous run of pairs, so a body's consecutive pairs resolve in one wave.
    const int per = (total + threads - 1) / threads;
    const int lo = me * per, hi = min(total, lo + per);
    __shared__ int left_block;
    unsigned int epoch = 0;
    for (int wave = 0;; wave++) {
        if (threadIdx.x == 0) left_block = 0;
        __syncthreads();
        int left = 0;
        for (int t = lo; t < hi; t++) {
            if (colour[t] >= 0) continue;
            unsigned int used = 0u;
            if (lower_rounds(t, ta[t], inc_start, inc_list, colour, used) &&
                lower_rounds(t, tb[t], inc_start, inc_list, colour, used)) {
                const int r = used == 0xffffffffu ? MOST_ROUNDS : __ffs(~used) - 1;
                *(volatile int*)&colour[t] = r;
            } else {
                left++;
            }
        }
        if (left) atomicAdd(&left_block, left);
        __syncthreads();
        if (threadIdx.x == 0 && left_block) atomicAdd(&counters->remaining[wave % 3], left_block);
        if (!grid_sync(bar, epoch)) return;
        const int remaining = *(volatile int*)&counters->remaining[wave % 3];
        if (blockIdx.x == 0 && threadIdx.x == 0) counters->remaining[(wave + 2) % 3] = 0;
        if (remaining == 0) {
            if (me == 0) counters->colour_waves = wave + 1;
            return;
        }
        if (wave > total + 1) {
            if (me == 0) atomicCAS(&counters->status, ST_OK, ST_ROUNDS);
            return;
        }
    }
}


// ------------------------------------------------------------------------------------------------------------
// Islands. Two bodies joined by a chain of placed pairs form one component; bodies of different components share no
// pair and no wall record, so what a component's bodies go through in a step depends on that component alone. The
// reference's order of operations is a per-body order (each body: its pairs in round order, then its walls, sweep
// by sweep), so a component may be solved apart from the others, by one block with block barriers between its rounds,
// and give every bit the grid phases give. Components are found by union-find over the placed pairs (unplaced pairs
// are never solved, so they join nothing).

__device__ __forceinline__ int uf_find(int* parent, int x) {
    int p = *(volatile int*)&parent[x];
    while (p != x) {
        const int up = *(volatile int*)&parent[p];
        if (up != p) *(volatile int*)&parent[x] = up;  // halve the path: up is an ancestor of x
        x = p;
        p = up;
    }
    return x;
}

__global__ void k_uf_init(int n, int* __restrict__ parent, int* __restrict__ size, int* __restrict__ fill) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    parent[s] = s;
    size[s] = 0;
    fill[s] = 0;
}

// Each placed pair joins its bodies' components: the larger root is hooked under the smaller, so every parent is
// at most its child and no chain can loop.
__global__ void k_uf_link(const int* __restrict__ touching_n, const int* __restrict__ ta, const int* __restrict__ tb,
                          const int* __restrict__ colour, int* parent) {
    const int total = *touching_n;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int c = colour[t];
        if (c < 0 || c >= MOST_ROUNDS) continue;
        int a = uf_find(parent, ta[t]), b = uf_find(parent, tb[t]);
        while (a != b) {
            const int hi = max(a, b), lo = min(a, b);
            const int was = atomicCAS(&parent[hi], hi, lo);
            if (was == hi) break;
            a = uf_find(parent, was);
            b = uf_find(parent, lo);
        }
    }
}

// Every body's root (the links are done: parents only read), and each component's body count.
__global__ void k_uf_flatten(int n, const int* __restrict__ parent, int* __restrict__ comp, int* __restrict__ size) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int r = s;
    for (int p = parent[r]; p != r; p = parent[r]) r = p;
    comp[s] = r;
    atomicAdd(&size[r], 1);
}

// The largest component's body count.
__global__ void k_largest(int n, const int* __restrict__ root, const int* __restrict__ size, Counters* counters) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n && root[s] == s && size[s] > 1) atomicMax(&counters->largest, size[s]);
}

// Which path each body takes: a component of one body (no placed pair) alone, a component of at most ISLAND_MOST
// bodies in a group. Where any component is larger, every body goes through the grid phases: their phase count is
// set by the rounds alone, so the small components cost them nothing more there, while beside them the island
// blocks would only lengthen the step. A small component's root keys the packing.
__global__ void k_classify(int n, const int* __restrict__ root, const int* __restrict__ size, int* __restrict__ key,
                           int* __restrict__ body_group, int* __restrict__ grid_list, int* __restrict__ free_list,
                           Counters* counters) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int r = root[s];
    const int m = size[r];
    int k = 0;
    if (*(volatile const int*)&counters->largest > ISLAND_MOST) {
        body_group[s] = -2;
        if (s == 0) counters->all_grid = 1;
    } else if (m == 1) {
        body_group[s] = -1;
        free_list[atomicAdd(&counters->free_n, 1)] = s;
    } else {
        body_group[s] = -3;  // a small component's: its group comes from k_assign
        if (r == s) k = m;
    }
    key[s] = k;
}

// Where each group's bodies begin: the place of its first component (a component that began in the group before may
// reach past its group's boundary, so a group's places start at its own first component, not there).
__global__ void k_group_base(int n, const int* __restrict__ root, const int* __restrict__ size,
                             const int* __restrict__ offset, const int* __restrict__ body_group,
                             int* __restrict__ group_base, int blocks) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n || root[s] != s || body_group[s] == -2) return;
    const int m = size[s];
    if (m == 1) return;
    const int at = offset[s];
    atomicMin(&group_base[at / group_base_of(offset[n], blocks)], at);
}

// A small component's bodies: the group its root's place falls in, and places in that group one after another from
// the group's first (the group's components lie end to end: its places are 0 .. its body count - 1).
__global__ void k_assign(int n, const int* __restrict__ root, const int* __restrict__ size,
                         const int* __restrict__ offset, const int* __restrict__ group_base, int* __restrict__ fill,
                         int* __restrict__ body_group, int* __restrict__ body_local, int* __restrict__ group_body,
                         int* __restrict__ group_count, int blocks) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int r = root[s];
    const int m = size[r];
    if (m == 1 || body_group[s] == -2) return;
    const int at = offset[r];
    const int g = at / group_base_of(offset[n], blocks);
    const int local = (at - group_base[g]) + atomicAdd(&fill[r], 1);
    body_group[s] = g;
    body_local[s] = local;
    group_body[(long)g * GROUP_CAP + local] = s;
    atomicMax(&group_count[g], local + 1);
}

__device__ __forceinline__ int pair_kind(float shapeA, float shapeB, int count) {
    const bool sa = shapeA > 0.5f, sb = shapeB > 0.5f;
    if (sa && sb) return 0;
    if (sa || sb) return 1;
    return 1 + min(max(count, 1), 4);
}

// A pair's path: 1 where its first body is in a small component's group (its second then is too), else 0. Without
// islands (body_group null) every pair takes the grid phases.
__device__ __forceinline__ int path_of(const int* body_group, int a, int c) {
    return body_group != nullptr && c < MOST_ROUNDS && body_group[a] >= 0 ? 1 : 0;
}

__global__ void k_round_count(const int* __restrict__ touching_n, const int* __restrict__ colour,
                              int* __restrict__ round_count, int* __restrict__ bucket_most, Counters* counters,
                              const int* __restrict__ ta, const int* __restrict__ tb,
                              unsigned* __restrict__ body_colours, const int* __restrict__ tcand,
                              const float4* __restrict__ head, const float4* __restrict__ half,
                              const int* __restrict__ body_group, int* __restrict__ gr_count) {
    const int total = *touching_n;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        int c = colour[t];
        if (c < 0 || c > MOST_ROUNDS) {  // never coloured: the colouring stopped early
            atomicCAS(&counters->status, ST_OK, ST_ROUNDS);
            c = MOST_ROUNDS;
        }
        const int count = (int)head[tcand[t]].w;
        const int kind = pair_kind(half[ta[t]].w, half[tb[t]].w, count);
        const int path = path_of(body_group, ta[t], c);
        const int bucket = path * BUCKETS + c * PAIR_KINDS + kind;
        atomicAdd(&round_count[bucket], 1);
        atomicMax(&bucket_most[bucket], min(max(count, 1), MOST_POINTS));
        if (path == 1) atomicAdd(&gr_count[(body_group[ta[t]] * GROUP_ROUNDS + c) * PAIR_KINDS + kind], 1);
        if (c < MOST_ROUNDS) {
            atomicMax(&counters->rounds, c + 1);
            if (path == 0) atomicMax(&counters->grid_rounds, c + 1);
            atomicOr(&body_colours[ta[t]], 1u << c);
            atomicOr(&body_colours[tb[t]], 1u << c);
        } else {
            atomicAdd(&counters->unplaced, 1);
        }
    }
}

// The touching pairs gathered into round order: rounds 0..31, then the unplaced, each pair with its manifold and
// carried impulses next to it, so a solve phase reads one contiguous record per pair. Within a round the order is
// the atomic fill's: the pairs of a round share no body, so their order does not change any result.
__global__ void k_order(const int* __restrict__ touching_n, const int* __restrict__ colour,
                        const int* __restrict__ bucket_start, const int* __restrict__ bucket_most,
                        const int* __restrict__ bucket_pstart, int* __restrict__ round_fill, const int* __restrict__ ta,
                        const int* __restrict__ tcand, const Manifolds m, const float4* __restrict__ imp_t,
                        const float4* __restrict__ impr_t, PairGen now,
                        const unsigned* __restrict__ body_colours, const float4* __restrict__ half,
                        const int* __restrict__ body_group, const int* __restrict__ body_local,
                        const int* __restrict__ gr_start, int* __restrict__ gr_fill, int2* __restrict__ ilist) {
    const int total = *touching_n;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        int c = colour[t];
        if (c < 0 || c > MOST_ROUNDS) c = MOST_ROUNDS;
        const int kind = pair_kind(half[ta[t]].w, half[now.tb[t]].w, (int)m.head[tcand[t]].w);
        const int path = path_of(body_group, ta[t], c);
        const int bucket = path * BUCKETS + c * PAIR_KINDS + kind;
        const int rank = atomicAdd(&round_fill[bucket], 1);
        const int p = bucket_start[bucket] + rank;
        const long first = bucket_pstart[bucket] + (long)rank * bucket_most[bucket];
        now.pos[t] = p;
        now.pstart[p] = (int)first;
        if (path == 1) {  // the island list: by (group, round, kind), each pair's position and its bodies' places
            const int gr = (body_group[ta[t]] * GROUP_ROUNDS + c) * PAIR_KINDS + kind;
            ilist[gr_start[gr] + atomicAdd(&gr_fill[gr], 1)] =
                make_int2(p, body_local[ta[t]] | body_local[now.tb[t]] << 16);
        }
        const int cd = tcand[t];
        const float4 head = m.head[cd];
        const int count = (int)head.w;
        // For the dependency schedule: each body's rank of this pair among its rounds, and its pair count.
        const int a = ta[t], b = now.tb[t];
        const unsigned ma = body_colours[a], mb = body_colours[b];
        const unsigned below = c < MOST_ROUNDS ? (1u << c) - 1u : 0xffffffffu;
        const unsigned packed = (unsigned)__popc(ma & below) | (unsigned)__popc(mb & below) << 8 |
                                (unsigned)__popc(ma) << 16 | (unsigned)__popc(mb) << 24;
        now.pair[p] = make_int4(a, b, count, (int)packed);
        now.normal[p] = make_float4(head.x, head.y, head.z, m.axis[cd]);
        for (int i = 0; i < count && i < MOST_POINTS; i++) {
            now.pa[first + i] = m.pa[(long)cd * MOST_POINTS + i];
            now.pb[first + i] = m.pb[(long)cd * MOST_POINTS + i];
            now.imp[first + i] = imp_t[(long)t * MOST_POINTS + i];
            now.impr[first + i] = impr_t[(long)t * MOST_POINTS + i];
        }
    }
}

// Where each bucket's points begin: its pairs take `most` entries each (every pair of a box-box bucket has the
// same point count, and sphere pairs have one point, so the points are packed). One thread: ALL_BUCKETS entries.
__global__ void k_bucket_points(const int* __restrict__ round_count, const int* __restrict__ bucket_most,
                                int* __restrict__ bucket_pstart) {
    if (threadIdx.x != 0) return;
    int at = 0;
    for (int b = 0; b < ALL_BUCKETS; b++) {
        bucket_pstart[b] = at;
        at += round_count[b] * bucket_most[b];
    }
    bucket_pstart[ALL_BUCKETS] = at;
}

// Where each round begins: its first bucket's start.
__global__ void k_round_starts(const int* __restrict__ bucket_start, int* __restrict__ round_start) {
    // The grid phases' rounds (path 0, which comes first): r * PAIR_KINDS <= BUCKETS for r <= 33.
    const int r = threadIdx.x;
    if (r <= MOST_ROUNDS + 1) round_start[r] = bucket_start[r * PAIR_KINDS];
}

// ------------------------------------------------------------------------------------------------------------
// The substeps: one cooperative kernel, a grid barrier between phases.

struct SolveArgs {
    int n;
    Bodies b;
    float4* wall;
    float4* wroll;
    unsigned long long* wmask;
    int* wall_list;   // bodies that may touch a wall until positions next change, rebuilt twice a substep
    int* wall_count;  // [4 * substeps] their counts: spheres, boxes for each half-substep
    PairGen pairs;
    const int* round_start;
    Counters* counters;
    int* version;                  // [n] items of each body done in this block of sweeps (dependency schedule)
    int* listed;                   // [n] 1 where the body is on this half-substep's wall list
    const unsigned* body_colours;  // [n] the rounds of each body's pairs, one bit each
    int schedule;                  // 0: a grid barrier after every round; 1: dependency-driven
    unsigned* residual;            // [substeps * (2 sweeps + 1)] per-sweep residual (f32 bits), null: not measured;
                                   // the pairs' part here, the walls' part wall_split words on
    int wall_split;                // where the walls' part of the residual begins
    int solve_only;                // the last substep skips its relax sweeps (a measurement of the solve's impulses)
    float tolerance;               // > 0: a substep's solve (relax) sweeps stop once a sweep's residual is this or less
    int* used;                     // [2 substeps] solve and relax sweeps each substep ran
    int substeps, sweeps, symmetric;
    Params params;
    const Params* scene_params;  // batched scenes: each scene's words (gravity, walls, friction differ); else null
    const int* body_scene;       // [n] each body's scene; else null
    GridBarrier bar;
    unsigned long long* trace;  // null: not traced
    int trace_cap;
    const int* grid_list;  // the bodies the grid phases move (the rest are the island kernel's); null: every body
    const int* grid_n;     // their count (device)
};

// The i-th body of the grid phases, and how many there are.
__device__ __forceinline__ bool listed_grid(const SolveArgs& A) {
    return A.grid_list && !*(volatile const int*)&A.counters->all_grid;
}
__device__ __forceinline__ int grid_bodies(const SolveArgs& A) {
    return listed_grid(A) ? *(volatile const int*)A.grid_n : A.n;
}
__device__ __forceinline__ int grid_body(const SolveArgs& A, int i) { return listed_grid(A) ? A.grid_list[i] : i; }

// Body state a solve phase reads and writes goes through L2 (ld/st .cg): under the dependency schedule one
// body's consecutive items can run on different SMs.
__device__ __forceinline__ void load_held(Held& h, const Bodies& b, int s) {
    h.load(__ldcg(&b.pose[s]), __ldcg(&b.turn[s]), __ldg(&b.half[s]), __ldcg(&b.vel[s]), __ldcg(&b.mom[s]),
           __ldg(&b.inv[s]));
}
__device__ __forceinline__ void store_held(const Held& h, const Bodies& b, int s) {
    __stcg(&b.vel[s], make_float4(h.velocity[0], h.velocity[1], h.velocity[2], 0.0f));
    __stcg(&b.mom[s], make_float4(h.momentum[0], h.momentum[1], h.momentum[2], 0.0f));
}

__device__ __forceinline__ void list_wall_body(const SolveArgs& A, int s, float4 pose, int slot);

// Boxes.positions :299-342 for one moving body: x += h v; the turn by the angular velocity at the half step.
__device__ __forceinline__ void move_body(float4& p, float4& turn, float4 v, float4 l, float4 inv, float h) {
    p.x = p.x + h * v.x;
    p.y = p.y + h * v.y;
    p.z = p.z + h * v.z;
    {
        const float4 tq = turn;
        const float q[4] = {tq.x, tq.y, tq.z, tq.w};
        const float momentum[3] = {l.x, l.y, l.z};
        const float inverse[3] = {inv.x, inv.y, inv.z};
        float omega[3], mid[4], omega_mid[3], end[4];
        {
            const float c[4] = {-q[0], -q[1], -q[2], q[3]};
            const float tw = twice_of(q);
            float own[3], scaled[3];
            rotate_by(c, tw, momentum, own);
            for (int a = 0; a < 3; a++) scaled[a] = inverse[a] * own[a];
            rotate_by(q, tw, scaled, omega);
        }
        const float half_h = 0.5f * h;
        turned(q, omega, half_h, mid);
        {
            const float c[4] = {-mid[0], -mid[1], -mid[2], mid[3]};
            const float tw = twice_of(mid);
            float own[3], scaled[3];
            rotate_by(c, tw, momentum, own);
            for (int a = 0; a < 3; a++) scaled[a] = inverse[a] * own[a];
            rotate_by(mid, tw, scaled, omega_mid);
        }
        turned(q, omega_mid, h, end);
        turn = make_float4(end[0], end[1], end[2], end[3]);
    }
}

// Boxes.positions :299-342, and the body listed for the relax sweeps' walls from where it now is.
__device__ __forceinline__ void phase_positions(const SolveArgs& A, int slot) {
    const int stride = gridDim.x * blockDim.x;
    if (blockIdx.x == 0 && threadIdx.x == 0) A.counters->bar_gen = 0u;  // the dependency schedule's ticket
    const float h = A.params.w[P_H];
    const int count = grid_bodies(A);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        const int s = grid_body(A, i);
        float4 p = __ldcg(&A.b.pose[s]);
        const float im = p.w;
        A.version[s] = 0;
        A.listed[s] = 0;
        if (!(im > 0.0f)) continue;
        float4 turn = __ldcg(&A.b.turn[s]);
        move_body(p, turn, __ldcg(&A.b.vel[s]), __ldcg(&A.b.mom[s]), __ldg(&A.b.inv[s]), h);
        __stcg(&A.b.pose[s], p);
        __stcg(&A.b.turn[s], turn);
        list_wall_body(A, s, p, slot);
    }
}

// v[i] for a runtime i without indexing a local array (which would move the array to local memory).
__device__ __forceinline__ float pick3(const float* v, int i) { return i == 0 ? v[0] : (i == 1 ? v[1] : v[2]); }

// A body's scene in a batch, or -1 in a single scene; and a parameter word of that scene (the world's words for
// -1). In a batch the substep, margin, softness and push are one for every scene; gravity, walls and friction are
// the scene's own.
__device__ __forceinline__ int scene_of(const SolveArgs& A, int s) { return A.body_scene ? __ldg(&A.body_scene[s]) : -1; }
__device__ __forceinline__ float word_of(const SolveArgs& A, int sc, int i) {
    return sc < 0 ? A.params.w[i] : __ldg(&A.scene_params[sc].w[i]);
}

// Wall, roll and contact-point records: a record one thread alone reads and writes for a whole step (OWN, the island
// kernel's) goes through L1 with plain accesses; one that consecutive items of a step may take on different SMs (the
// grid phases') goes through L2 (ld/st .cg).
template <bool OWN, class T>
__device__ __forceinline__ T ld_rec(const T* p) {
    if (OWN) return *p;
    return __ldcg(p);
}
template <bool OWN, class T>
__device__ __forceinline__ void st_rec(T* p, T v) {
    if (OWN) *p = v;
    else __stcg(p, v);
}

// Which walls a body may touch: bit w set where the body's bounding sphere comes within the margin of wall w
// (a bound that holds through f32 rounding: every corner's gap to a wall not in the set exceeds the margin).
__device__ __forceinline__ unsigned near_walls(float4 pose, float4 hw, float margin, const float* extent) {
    const float r = hw.w > 0.5f ? hw.x : sqrtf((hw.x * hw.x + hw.y * hw.y) + hw.z * hw.z);
    const float bound = r * 1.01f + 1e-3f + margin;
    const float at[3] = {pose.x, pose.y, pose.z};
    unsigned near = 0u;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        if (!(at[a] - bound > 0.0f)) near |= 1u << (2 * a);
        if (!((extent[a] - at[a]) - bound > 0.0f)) near |= 1u << (2 * a + 1);
    }
    return near;
}

// The bodies the walls' sweeps must visit until positions next change: near a wall, or holding a wall impulse.
// The order of the list does not matter: each body's walls touch that body alone.
__device__ __forceinline__ void list_wall_body(const SolveArgs& A, int s, float4 pose, int slot) {
    const float4 hw = __ldg(&A.b.half[s]);
    const int sc = scene_of(A, s);
    const float extent[3] = {word_of(A, sc, P_SX), word_of(A, sc, P_SY), word_of(A, sc, P_SZ)};
    const bool list = __ldcg(&A.wmask[s]) != 0ull || near_walls(pose, hw, A.params.w[P_MARGIN], extent) != 0u;
    if (list) {  // spheres from the front of the list, boxes from the back: a warp's bodies take the same path
        if (hw.w > 0.5f) A.wall_list[atomicAdd(&A.wall_count[2 * slot], 1)] = s;
        else A.wall_list[A.n - 1 - atomicAdd(&A.wall_count[2 * slot + 1], 1)] = s;
    }
    A.listed[s] = list ? 1 : 0;
}

__device__ __forceinline__ void phase_velocities_and_list(const SolveArgs& A, int slot) {
    const int stride = gridDim.x * blockDim.x;
    if (blockIdx.x == 0 && threadIdx.x == 0) A.counters->bar_gen = 0u;  // the dependency schedule's ticket
    const float h = A.params.w[P_H];
    const int count = grid_bodies(A);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        const int s = grid_body(A, i);
        const float4 pose = A.b.pose[s];
        A.version[s] = 0;
        A.listed[s] = 0;
        if (!(pose.w > 0.0f)) continue;
        float4 v = __ldcg(&A.b.vel[s]);
        const int sc = scene_of(A, s);
        v.x = v.x + h * word_of(A, sc, P_GX);
        v.y = v.y + h * word_of(A, sc, P_GY);
        v.z = v.z + h * word_of(A, sc, P_GZ);
        __stcg(&A.b.vel[s], v);
        list_wall_body(A, s, pose, slot);
    }
}

// Boxes.walls :357-416 for one body held in registers: its corners (a sphere: its nearest point) against the six
// walls. A wall the body is far from, with no impulse held against it, is skipped: its contacts would neither
// start nor apply. Returns whether anything was applied (the caller then stores the body).
template <bool OWN = false>
__device__ __forceinline__ bool walls_of(const SolveArgs& A, Held& box, int s, int sweep, bool reverse,
                                         unsigned* track = nullptr) {
    const Params& P = A.params;
    const float margin = P.w[P_MARGIN];
    const int sc = scene_of(A, s);
    const float extent[3] = {word_of(A, sc, P_SX), word_of(A, sc, P_SY), word_of(A, sc, P_SZ)};
    const float mu_rolling = word_of(A, sc, P_MU_ROLLING);
    unsigned long long mask = ld_rec<OWN>(&A.wmask[s]);
    const float4 pose = make_float4(box.at[0], box.at[1], box.at[2], box.im);
    const float4 hw = make_float4(box.half[0], box.half[1], box.half[2], box.shape);
    const bool sphere = hw.w > 0.5f;
    const unsigned near = sweep == WARM ? 0u : near_walls(pose, hw, margin, extent);
    unsigned held_walls = 0u;
#pragma unroll
    for (int wl = 0; wl < 6; wl++) {
        const unsigned long long bits = (0xffull << (8 * wl)) | (1ull << (48 + wl));
        if (mask & bits) held_walls |= 1u << wl;
    }
    const unsigned visit = near | held_walls;
    if (visit == 0u) return false;
    Soft soft(P, true);
    if (sc >= 0) {
        soft.mu_static = word_of(A, sc, P_MU_STATIC);
        soft.mu_kinetic = word_of(A, sc, P_MU_KINETIC);
    }
    bool touched = false, box_corners = false;
    for (int order = 0; order < 6 && !box_corners; order++) {
        const int wall = reverse ? 5 - order : order;
        if (!((visit >> wall) & 1u)) continue;
        const int axis = wall / 2;
        const bool high = wall % 2 == 1;
        float n[3];
        for (int a = 0; a < 3; a++) n[a] = a == axis ? (high ? -1.0f : 1.0f) : 0.0f;
        if (sphere) {
            float r[3];
            for (int a = 0; a < 3; a++) r[a] = -(box.half[0] * n[a]);
            const float reach = pick3(box.at, axis) + pick3(r, axis);
            const float gap = high ? pick3(extent, axis) - reach : reach;
            const int bit = wall * 8, rbit = 48 + wall;
            const bool held = (mask >> bit) & 1ull, rolled = (mask >> rbit) & 1ull;
            const bool need = held || (sweep != WARM && gap < margin);
            float4 rec = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            const long at = (long)s * WALL_RECORDS + wall * 8;
            if (need) {
                rec = held ? ld_rec<OWN>(&A.wall[at]) : rec;
                contact<false>(sweep, gap, n, box, nullptr, box, r, rec, soft, -1.0f, track);
                if (sweep != WARM) {
                    st_rec<OWN>(&A.wall[at], rec);
                    mask = nonzero_bits(rec) ? (mask | (1ull << bit)) : (mask & ~(1ull << bit));
                }
                touched = true;
            }
            if (rolled || (sweep != WARM && nonzero_bits(rec))) {
                float4 rr = rolled ? ld_rec<OWN>(&A.wroll[(long)s * 6 + wall]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                roll<false>(sweep, box, box, box.half[0], rec.x, rr, mu_rolling);
                if (sweep != WARM) {
                    st_rec<OWN>(&A.wroll[(long)s * 6 + wall], rr);
                    mask = nonzero_bits(rr) ? (mask | (1ull << rbit)) : (mask & ~(1ull << rbit));
                }
                touched = true;
            }
        } else {
            box_corners = true;
        }
    }
    if (box_corners) {
        // A box: first which corners run, wall by wall in the sweep's order and corner by corner in it (a held
        // corner always; another, outside the warm sweep, where its wall is near and its gap is under the margin),
        // then those corners alone, in that order. Whether a corner runs depends only on the pose, which the walls
        // do not change, and on its own held bit, which only its own turn changes, so the order and every result
        // are the reference's. Lanes of a warp then solve their k-th corners together, whichever corners they are.
        unsigned long long todo = 0ull;
        for (int order = 0; order < 6; order++) {
            const int wall = reverse ? 5 - order : order;
            if (!((visit >> wall) & 1u)) continue;
            const unsigned held_bits = (unsigned)((mask >> (wall * 8)) & 0xffull);
            todo |= (unsigned long long)held_bits << (wall * 8);
            if (sweep == WARM || !((near >> wall) & 1u)) continue;
            const int axis = wall / 2;
            const bool high = wall % 2 == 1;
            for (int c = 0; c < 8; c++) {
                if ((held_bits >> c) & 1u) continue;
                float offset[3], r[3];
                for (int a = 0; a < 3; a++) offset[a] = box.half[a] * (2.0f * (float)((c >> a) & 1) - 1.0f);
                rotate_by(box.q, box.twice, offset, r);
                const float reach = pick3(box.at, axis) + pick3(r, axis);
                const float gap = high ? pick3(extent, axis) - reach : reach;
                if (gap < margin) todo |= 1ull << (wall * 8 + c);
            }
        }
        // the corners in the sweep's order: walls ascending and corners ascending, or both descending
        int bit = -1;
        auto next_bit = [&](unsigned long long left) {
            if (left == 0ull) return -1;
            return reverse ? 63 - __clzll((long long)left) : __ffsll((long long)left) - 1;
        };
        bit = next_bit(todo);
        float4 ahead = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (bit >= 0 && ((mask >> bit) & 1ull)) ahead = ld_rec<OWN>(&A.wall[(long)s * WALL_RECORDS + bit]);
        while (bit >= 0) {
            todo &= ~(1ull << bit);
            const int wall = bit / 8, c = bit % 8;
            const bool held = (mask >> bit) & 1ull;
            const float4 loaded = held ? ahead : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            const int after = next_bit(todo);
            if (after >= 0 && ((mask >> after) & 1ull)) ahead = ld_rec<OWN>(&A.wall[(long)s * WALL_RECORDS + after]);
            const int axis = wall / 2;
            const bool high = wall % 2 == 1;
            float n[3];
            for (int a = 0; a < 3; a++) n[a] = a == axis ? (high ? -1.0f : 1.0f) : 0.0f;
            float offset[3], r[3];
            for (int a = 0; a < 3; a++) offset[a] = box.half[a] * (2.0f * (float)((c >> a) & 1) - 1.0f);
            rotate_by(box.q, box.twice, offset, r);
            const float reach = pick3(box.at, axis) + pick3(r, axis);
            const float gap = high ? pick3(extent, axis) - reach : reach;
            float4 rec = loaded;
            contact<false>(sweep, gap, n, box, nullptr, box, r, rec, soft, -1.0f, track);
            if (sweep != WARM) {
                st_rec<OWN>(&A.wall[(long)s * WALL_RECORDS + bit], rec);
                mask = nonzero_bits(rec) ? (mask | (1ull << bit)) : (mask & ~(1ull << bit));
            }
            touched = true;
            bit = after;
        }
    }
    if (touched) st_rec<OWN>(&A.wmask[s], mask);
    return touched;
}

// Boxes.walls :357-416 over the listed bodies, each loaded afresh (its angular velocity from its angular
// momentum, as the reference's walls kernel loads it).
// The list's runs of 32 are dealt to the blocks in turn (as a round's pairs are), so the boxes, listed at its
// end and the heavier work, spread over every SM.
__device__ __forceinline__ void phase_walls(const SolveArgs& A, int sweep, bool reverse, int slot,
                                            unsigned* track) {
    const int runs = gridDim.x * (blockDim.x >> 5);
    const int run = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;
    const int spheres = *(volatile int*)&A.wall_count[2 * slot], boxes = *(volatile int*)&A.wall_count[2 * slot + 1];
    for (int k = run * 32 + (threadIdx.x & 31); k < spheres + boxes; k += runs * 32) {
        const int s = A.wall_list[k < spheres ? k : A.n - 1 - (k - spheres)];
        Held box;
        load_held(box, A.b, s);
        if (walls_of(A, box, s, sweep, reverse, track)) store_held(box, A.b, s);
    }
}

// BoxPairs.solve :64-151 for the pair at round-order position k: its whole manifold in turn, both bodies loaded
// once and stored once.
// fill: the first sweep of a substep's half (positions fixed until the next positions phase): each point's anchors
// in the world's frame, its gap and its normal's generalised inverse mass are worked out and kept; the later
// sweeps of that half read them back (the same values the reference works out again every sweep).
// solve_points: the pair's points with both bodies held (loaded by the caller, stored after).
template <bool OWN = false>
__device__ __forceinline__ void solve_points(const SolveArgs& A, long k, int4 rec4, Held& first, Held& second,
                                             int sweep, bool reverse, bool fill, unsigned* track) {
    const Params& P = A.params;
    const float4 head = __ldg(&A.pairs.normal[k]);
    const int ia = rec4.x, count = rec4.z;
    Soft soft(P, false);
    if (first.im == 0.0f || second.im == 0.0f) {
        soft.bias = P.w[P_STATIC_BIAS];
        soft.mass_scale = P.w[P_STATIC_MASS_SCALE];
        soft.impulse_scale = P.w[P_STATIC_IMPULSE_SCALE];
    }
    const int sc = scene_of(A, ia);
    float mu_rolling = P.w[P_MU_ROLLING];
    if (sc >= 0) {
        soft.mu_static = word_of(A, sc, P_MU_STATIC);
        soft.mu_kinetic = word_of(A, sc, P_MU_KINETIC);
        mu_rolling = word_of(A, sc, P_MU_ROLLING);
    }
    const float n[3] = {head.x, head.y, head.z};
    const bool anySphere = first.sphere() || second.sphere();
    // The points in turn (backward: last to first). Past the first sweep of a half, each point's kept terms and
    // impulses are loaded while the point before it is solved: their addresses depend on the pair alone, and no
    // point writes another's records.
    const long base = __ldg(&A.pairs.pstart[k]);
    float4 next_a = make_float4(0.0f, 0.0f, 0.0f, 0.0f), next_b = next_a, next_imp = next_a;
    if (!fill && count > 0) {
        const long at0 = base + (reverse ? count - 1 : 0);
        next_a = ld_rec<OWN>(&A.pairs.prepA[at0]);
        next_b = ld_rec<OWN>(&A.pairs.prepB[at0]);
        next_imp = ld_rec<OWN>(&A.pairs.imp[at0]);
    }
    for (int order = 0; order < MOST_POINTS; order++) {
        const int slot = reverse ? MOST_POINTS - 1 - order : order;
        if (!(slot < count)) continue;
        const long at = base + slot;
        float rA[3], rB[3], gap, kn;
        float4 rec;
        if (fill) {
            if (first.sphere()) {
                for (int a = 0; a < 3; a++) rA[a] = first.half[0] * n[a];
            } else {
                const float4 qa = __ldg(&A.pairs.pa[at]);
                const float anchorA[3] = {qa.x, qa.y, qa.z};
                rotate_by(first.q, first.twice, anchorA, rA);
            }
            if (second.sphere()) {
                for (int a = 0; a < 3; a++) rB[a] = -(second.half[0] * n[a]);
            } else {
                const float4 qb = __ldg(&A.pairs.pb[at]);
                const float anchorB[3] = {qb.x, qb.y, qb.z};
                rotate_by(second.q, second.twice, anchorB, rB);
            }
            gap = ((second.at[0] + rB[0]) - (first.at[0] + rA[0])) * n[0] +
                  ((second.at[1] + rB[1]) - (first.at[1] + rA[1])) * n[1];
            gap = gap + ((second.at[2] + rB[2]) - (first.at[2] + rA[2])) * n[2];
            kn = mass_along<true>(first, rA, second, rB, n);
            st_rec<OWN>(&A.pairs.prepA[at], make_float4(rA[0], rA[1], rA[2], gap));
            st_rec<OWN>(&A.pairs.prepB[at], make_float4(rB[0], rB[1], rB[2], kn));
            rec = ld_rec<OWN>(&A.pairs.imp[at]);
        } else {
            const float4 pa = next_a, pb = next_b;
            rec = next_imp;
            const int later = reverse ? slot - 1 : slot + 1;
            if (later >= 0 && later < count) {
                const long at1 = base + later;
                next_a = ld_rec<OWN>(&A.pairs.prepA[at1]);
                next_b = ld_rec<OWN>(&A.pairs.prepB[at1]);
                next_imp = ld_rec<OWN>(&A.pairs.imp[at1]);
            }
            rA[0] = pa.x; rA[1] = pa.y; rA[2] = pa.z; gap = pa.w;
            rB[0] = pb.x; rB[1] = pb.y; rB[2] = pb.z; kn = pb.w;
        }
        contact<true>(sweep, gap, n, first, rA, second, rB, rec, soft, kn, track);
        if (sweep != WARM) st_rec<OWN>(&A.pairs.imp[at], rec);
        if (anySphere) {
            float radius = second.half[0];
            if (first.sphere()) radius = first.half[0];
            if (first.sphere() && second.sphere())
                radius = (first.half[0] * second.half[0]) / (first.half[0] + second.half[0]);
            float4 rr = ld_rec<OWN>(&A.pairs.impr[at]);
            roll<true>(sweep, first, second, radius, rec.x, rr, mu_rolling);
            if (sweep != WARM) st_rec<OWN>(&A.pairs.impr[at], rr);
        }
    }
}

__device__ __forceinline__ void solve_pair(const SolveArgs& A, long k, int4 rec4, int sweep, bool reverse, bool fill,
                                           unsigned* track) {
    Held first, second;
    load_held(first, A.b, rec4.x);
    load_held(second, A.b, rec4.y);
    solve_points(A, k, rec4, first, second, sweep, reverse, fill, track);
    store_held(first, A.b, rec4.x);
    store_held(second, A.b, rec4.y);
}

// One round of pairs that share no body (the barrier schedule). A round's pairs lie in kind order (sphere pairs
// first, box pairs by point count last); its runs of 32 are dealt to the blocks in turn, so the heavy runs at the
// round's end spread over every SM instead of crowding a few, and each warp's pairs stay of one kind. Which
// thread solves a pair of a round changes no result: the round's pairs share no body.
__device__ __forceinline__ void phase_round(const SolveArgs& A, int sweep, bool reverse, int r, bool fill,
                                            unsigned* track) {
    const long runs = (long)gridDim.x * (blockDim.x >> 5);
    const long run = (long)(threadIdx.x >> 5) * gridDim.x + blockIdx.x;
    const int lo = A.round_start[r], hi = A.round_start[r + 1];
    for (long k = lo + run * 32 + (threadIdx.x & 31); k < hi; k += runs * 32)
        solve_pair(A, k, __ldg(&A.pairs.pair[k]), sweep, reverse, fill, track);
}

// Waits until every listed body has done exactly `want` items of this block. A bounded wait: past the limit it
// raises the abort and status words and returns false.
__device__ __forceinline__ bool wait_versions(const SolveArgs& A, int a, int wantA, int b, int wantB) {
    const volatile int* va = A.version + a;
    const volatile int* vb = A.version + (b < 0 ? a : b);
    if (*va == wantA && (b < 0 || *vb == wantB)) { __threadfence(); return true; }
    const unsigned long long start = global_ns();
    for (unsigned spins = 1;; spins++) {
        if (spins > 64) __nanosleep(32);
        if (*va == wantA && (b < 0 || *vb == wantB)) { __threadfence(); return true; }
        if ((spins & 63u) == 0u) {
            if (*(volatile int*)A.bar.abort) return false;
            if (global_ns() - start > A.bar.limit_ns) {
                atomicExch(A.bar.abort, 1);
                atomicCAS(A.bar.status, ST_OK, ST_TIMEOUT);
                return false;
            }
        }
    }
}

// A block of sweeps under the dependency schedule: every pair of every sweep, and the walls of every listed body,
// as items in the reference's order (sweep by sweep; within a sweep the rounds, then the walls; backward, the
// walls, then the rounds last to first). Each body counts the items it has done; an item runs once each of its
// bodies has done exactly the items that precede it in that body's own sequence of the reference's order:
//   per sweep a body has deg pair items (one per round it is in, in round order) and, if listed, one walls item.
// So the per-body order of operations, and every result, is the reference's; only unrelated bodies overlap.
// Items are handed out in increasing order, so the lowest unfinished item always has all it waits on done and a
// running warp holding it: the schedule cannot stall while every block is resident (a cooperative launch).
__device__ __forceinline__ bool block_of_sweeps(const SolveArgs& A, int first_kind, int sweeps, int rounds,
                                                int slot, int sweep0) {
    const int placed = A.round_start[rounds];
    const int spheres = *(volatile int*)&A.wall_count[2 * slot];
    const int walls = spheres + *(volatile int*)&A.wall_count[2 * slot + 1];
    const long per = (long)placed + walls;
    const long total = per * sweeps;
    // Warps take runs of 32 items from a ticket, in increasing order (the lowest unfinished item is always held
    // by a running warp).
    unsigned int* ticket = &A.counters->bar_gen;  // zeroed by the phase before the block
    for (;;) {
        long base = 0;
        if ((threadIdx.x & 31) == 0) base = atomicAdd(ticket, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total) break;
        const long i = base + (threadIdx.x & 31);
        if (i >= total) continue;
        const int w = (int)(i / per);
        const int j = (int)(i - (long)w * per);
        const int kind = w == 0 ? first_kind : (first_kind == WARM ? SOLVE : first_kind);
        const int sw = first_kind == WARM ? w - 1 : w;  // index among the block's SOLVE or RELAX sweeps
        const bool reverse = kind != WARM && A.symmetric && sw % 2 == 1;
        const bool is_pair = reverse ? j >= walls : j < placed;
        if (is_pair) {
            const long k = reverse ? (long)placed - 1 - (j - walls) : j;
            const int4 rec4 = __ldg(&A.pairs.pair[k]);
            const unsigned packed = (unsigned)rec4.w;
            const int rankA = packed & 255u, rankB = (packed >> 8) & 255u;
            const int degA = (packed >> 16) & 255u, degB = packed >> 24;
            const int lA = A.listed[rec4.x], lB = A.listed[rec4.y];
            const int wantA = w * (degA + lA) + (reverse ? lA + (degA - 1 - rankA) : rankA);
            const int wantB = w * (degB + lB) + (reverse ? lB + (degB - 1 - rankB) : rankB);
            if (!wait_versions(A, rec4.x, wantA, rec4.y, wantB)) return false;
            solve_pair(A, k, rec4, kind, reverse, w == 0, A.residual ? A.residual + sweep0 + w : nullptr);
            __threadfence();
            *(volatile int*)&A.version[rec4.x] = wantA + 1;
            *(volatile int*)&A.version[rec4.y] = wantB + 1;
        } else {
            const int wk = reverse ? j : j - placed;
            const int s = A.wall_list[wk < spheres ? wk : A.n - 1 - (wk - spheres)];
            const int deg = __popc(A.body_colours[s]);
            const int want = w * (deg + 1) + (reverse ? 0 : deg);
            if (!wait_versions(A, s, want, -1, 0)) return false;
            Held box;
            load_held(box, A.b, s);
            if (walls_of(A, box, s, kind, reverse, A.residual ? A.residual + sweep0 + w + A.wall_split : nullptr))
                store_held(box, A.b, s);
            __threadfence();
            *(volatile int*)&A.version[s] = want + 1;
        }
    }
    return true;
}

// Phase codes of the trace: kind | sweep << 4 | one-block run << 7 | round << 8.
enum : int { TR_START = 0, TR_VELOCITIES = 1, TR_WALLS = 2, TR_POSITIONS = 3, TR_ROUND = 4, TR_WALL_LIST = 5,
            TR_BLOCK = 6 };

struct Tracer {
    unsigned long long* out;
    int cap, len;
    __device__ __forceinline__ void mark(int code) {
        if (out && blockIdx.x == 0 && threadIdx.x == 0 && len < cap)
            out[len++] = ((unsigned long long)code << 48) | (global_ns() & 0xffffffffffffull);
    }
};

// Rounds of at most this many pairs (one a thread of a block) are run by one block, without grid barriers.
constexpr int SMALL_ROUND = SOLVE_THREADS;

// One sweep (BoxStep.sweep :217-231): every round of pairs, then the walls; backward, the walls first and the
// rounds last to first.
__device__ __forceinline__ bool sweep_all(const SolveArgs& A, Tracer& tr, unsigned int& epoch, int kind, bool reverse,
                                          int rounds, int slot, bool fill, int index) {
    unsigned* track = A.residual ? A.residual + index : nullptr;
    unsigned* wtrack = A.residual ? A.residual + index + A.wall_split : nullptr;
    if (reverse) {
        phase_walls(A, kind, true, slot, wtrack);
        if (!grid_sync(A.bar, epoch)) return false;
        tr.mark(TR_WALLS | kind << 4);
    }
    for (int order = 0; order < rounds;) {
        const int r = reverse ? rounds - 1 - order : order;
        if (A.round_start[r + 1] - A.round_start[r] > SMALL_ROUND) {
            phase_round(A, kind, reverse, r, fill, track);
            if (!grid_sync(A.bar, epoch)) return false;
            tr.mark(TR_ROUND | kind << 4 | r << 8);
            order++;
            continue;
        }
        // A run of small rounds: block 0 alone, a block barrier between them (each round's pairs are at most one a
        // thread), one grid barrier after the run. The other blocks wait at that barrier; the per-body order of
        // operations is the same. Every block reads the same round sizes, so every block takes the same path.
        int end = order;
        while (end < rounds) {
            const int q = reverse ? rounds - 1 - end : end;
            if (A.round_start[q + 1] - A.round_start[q] > SMALL_ROUND) break;
            end++;
        }
        if (blockIdx.x == 0) {
            for (int o = order; o < end; o++) {
                const int q = reverse ? rounds - 1 - o : o;
                const int lo = A.round_start[q], hi = A.round_start[q + 1];
                for (int k = lo + threadIdx.x; k < hi; k += blockDim.x)
                    solve_pair(A, k, __ldg(&A.pairs.pair[k]), kind, reverse, fill, track);
                __syncthreads();
                tr.mark(TR_ROUND | kind << 4 | 1 << 7 | q << 8);  // bit 7: a round of a one-block run
            }
        }
        if (!grid_sync(A.bar, epoch)) return false;
        order = end;
    }
    if (!reverse) {
        phase_walls(A, kind, false, slot, wtrack);
        if (!grid_sync(A.bar, epoch)) return false;
        tr.mark(TR_WALLS | kind << 4);
    }
    return true;
}

// Whether a substep's sweeps may stop after sweep `index`: its residual is at or below the tolerance. Every block
// reads the same word after the grid barrier, so every block decides the same.
__device__ __forceinline__ bool converged(const SolveArgs& A, int index) {
    if (!(A.tolerance > 0.0f) || !A.residual) return false;
    const float pairs = __uint_as_float(*(volatile unsigned*)&A.residual[index]);
    const float walls = __uint_as_float(*(volatile unsigned*)&A.residual[index + A.wall_split]);
    return pairs <= A.tolerance && walls <= A.tolerance;
}

__global__ void __launch_bounds__(SOLVE_THREADS, 2) k_solve(SolveArgs A) {
    const int rounds = *(volatile int*)&A.counters->grid_rounds;
    if (A.grid_list && grid_bodies(A) == 0) {  // every body is the island kernel's: nothing for the grid phases
        if (A.used && blockIdx.x == 0 && threadIdx.x == 0)
            for (int sub = 0; sub < A.substeps; sub++) {
                A.used[2 * sub] = A.sweeps;
                A.used[2 * sub + 1] = A.solve_only && sub == A.substeps - 1 ? 0 : A.sweeps;
            }
        return;
    }
    Tracer tr{A.trace, A.trace_cap, 0};
    unsigned int epoch = 0;
    tr.mark(TR_START);
    const int stride = 2 * A.sweeps + 1;  // residual words a substep
    for (int sub = 0; sub < A.substeps; sub++) {
        phase_velocities_and_list(A, 2 * sub);
        if (!grid_sync(A.bar, epoch)) return;
        tr.mark(TR_VELOCITIES);
        int solved = A.sweeps, relaxed = A.sweeps;
        if (A.schedule == 1) {
            if (!block_of_sweeps(A, WARM, 1 + A.sweeps, rounds, 2 * sub, sub * stride)) return;
            if (!grid_sync(A.bar, epoch)) return;
            tr.mark(TR_BLOCK | SOLVE << 4);
        } else {
            const int base = sub * stride;
            if (!sweep_all(A, tr, epoch, WARM, false, rounds, 2 * sub, true, base)) return;
            for (int sw = 0; sw < A.sweeps; sw++) {
                if (!sweep_all(A, tr, epoch, SOLVE, A.symmetric && sw % 2 == 1, rounds, 2 * sub, false, base + 1 + sw))
                    return;
                if (converged(A, base + 1 + sw)) {
                    solved = sw + 1;
                    break;
                }
            }
        }
        phase_positions(A, 2 * sub + 1);
        if (!grid_sync(A.bar, epoch)) return;
        tr.mark(TR_POSITIONS);
        if (A.solve_only && sub == A.substeps - 1) {
            relaxed = 0;
        } else if (A.schedule == 1) {
            if (!block_of_sweeps(A, RELAX, A.sweeps, rounds, 2 * sub + 1, sub * stride + 1 + A.sweeps)) return;
            if (!grid_sync(A.bar, epoch)) return;
            tr.mark(TR_BLOCK | RELAX << 4);
        } else {
            const int base = sub * stride + 1 + A.sweeps;
            for (int sw = 0; sw < A.sweeps; sw++) {
                if (!sweep_all(A, tr, epoch, RELAX, A.symmetric && sw % 2 == 1, rounds, 2 * sub + 1, sw == 0,
                               base + sw))
                    return;
                if (converged(A, base + sw)) {
                    relaxed = sw + 1;
                    break;
                }
            }
        }
        if (A.used && blockIdx.x == 0 && threadIdx.x == 0) {
            A.used[2 * sub] = solved;
            A.used[2 * sub + 1] = relaxed;
        }
    }
    if (A.trace && blockIdx.x == 0 && threadIdx.x == 0) A.counters->trace_len = tr.len;
}


// ------------------------------------------------------------------------------------------------------------
// The island kernel: whole substeps of the small components, a block a group, the group's bodies held in shared memory
// for the step; and the bodies in no placed pair, a thread each. Every operation is the one the grid phases make, in
// each body's order (velocities; the warm sweep and the solve sweeps, each its rounds then its walls, or backward the
// walls then the rounds; positions; the relax sweeps), so the results are theirs to the bit. As in the grid phases, a
// round's pairs lie in kind order and the walls' bodies are listed spheres first and boxes last, so a warp's lanes
// mostly take one path.

struct IslandArgs {
    const int* group_body;   // [groups * GROUP_CAP]
    const int* group_count;  // [groups]
    const int* gr_start;     // [groups * GROUP_LISTS + 1] each (group, round, kind)'s first entry of ilist
    const int2* ilist;       // position, local ids of first | second << 16
    const int* free_list;    // bodies in no placed pair
    const int* island_n;     // bodies in small components
    int* work;               // items handed out: groups, then runs of ISLAND_THREADS lone bodies
};

struct GroupBodies {  // a block's group, for the step
    float4 pose[GROUP_CAP], turn[GROUP_CAP], vel[GROUP_CAP], mom[GROUP_CAP];
    int id[GROUP_CAP];
    short wall_list[GROUP_CAP];  // bodies the walls' sweeps visit until positions next change: spheres, then boxes
    int wall_count[2];           // spheres (from the front), boxes (from the back)
    unsigned present;            // the rounds the group has pairs in
    int item;
};

__device__ __forceinline__ void load_local(Held& h, const GroupBodies& G, const Bodies& b, int i) {
    const int s = G.id[i];
    h.load(G.pose[i], G.turn[i], __ldg(&b.half[s]), G.vel[i], G.mom[i], __ldg(&b.inv[s]));
}
__device__ __forceinline__ void store_local(const Held& h, GroupBodies& G, int i) {
    G.vel[i] = make_float4(h.velocity[0], h.velocity[1], h.velocity[2], 0.0f);
    G.mom[i] = make_float4(h.momentum[0], h.momentum[1], h.momentum[2], 0.0f);
}

// Whether the walls' sweeps visit a body until positions next change: as list_wall_body decides.
__device__ __forceinline__ bool wall_listed(const SolveArgs& A, int s, float4 pose, float4 hw) {
    const int sc = scene_of(A, s);
    const float extent[3] = {word_of(A, sc, P_SX), word_of(A, sc, P_SY), word_of(A, sc, P_SZ)};
    return __ldcg(&A.wmask[s]) != 0ull || near_walls(pose, hw, A.params.w[P_MARGIN], extent) != 0u;
}

__device__ __forceinline__ void group_list_wall(GroupBodies& G, int i, float4 hw) {
    if (hw.w > 0.5f) G.wall_list[atomicAdd(&G.wall_count[0], 1)] = (short)i;
    else G.wall_list[GROUP_CAP - 1 - atomicAdd(&G.wall_count[1], 1)] = (short)i;
}

__device__ __forceinline__ void group_velocities(const SolveArgs& A, GroupBodies& G, int nb, float h) {
    if (threadIdx.x == 0) G.wall_count[0] = G.wall_count[1] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        const int s = G.id[i];
        const float4 pose = G.pose[i];
        if (!(pose.w > 0.0f)) continue;
        float4 v = G.vel[i];
        const int sc = scene_of(A, s);
        v.x = v.x + h * word_of(A, sc, P_GX);
        v.y = v.y + h * word_of(A, sc, P_GY);
        v.z = v.z + h * word_of(A, sc, P_GZ);
        G.vel[i] = v;
        const float4 hw = __ldg(&A.b.half[s]);
        if (wall_listed(A, s, pose, hw)) group_list_wall(G, i, hw);
    }
    __syncthreads();
}

__device__ __forceinline__ void group_positions(const SolveArgs& A, GroupBodies& G, int nb, float h) {
    if (threadIdx.x == 0) G.wall_count[0] = G.wall_count[1] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        const int s = G.id[i];
        float4 p = G.pose[i];
        if (!(p.w > 0.0f)) continue;
        float4 turn = G.turn[i];
        move_body(p, turn, G.vel[i], G.mom[i], __ldg(&A.b.inv[s]), h);
        G.pose[i] = p;
        G.turn[i] = turn;
        const float4 hw = __ldg(&A.b.half[s]);
        if (wall_listed(A, s, p, hw)) group_list_wall(G, i, hw);
    }
    __syncthreads();
}

__device__ __forceinline__ void group_walls(const SolveArgs& A, GroupBodies& G, int kind, bool reverse,
                                            unsigned* track) {
    const int spheres = G.wall_count[0], listed = spheres + G.wall_count[1];
    for (int k = threadIdx.x; k < listed; k += blockDim.x) {
        const int i = G.wall_list[k < spheres ? k : GROUP_CAP - 1 - (k - spheres)];
        Held box;
        load_local(box, G, A.b, i);
        if (walls_of<true>(A, box, G.id[i], kind, reverse, track)) store_local(box, G, i);
    }
}

// One sweep of a group: its rounds in order, a block barrier after each (a round's pairs share no body), then the
// walls; backward, the walls first and the rounds last to first.
__device__ __forceinline__ void group_sweep(const SolveArgs& A, const IslandArgs& I, GroupBodies& G, const int* gs,
                                            int kind, bool reverse, bool fill, int index) {
    unsigned* track = A.residual ? A.residual + index : nullptr;
    unsigned* wtrack = A.residual ? A.residual + index + A.wall_split : nullptr;
    if (reverse) {
        group_walls(A, G, kind, true, wtrack);
        __syncthreads();
    }
    for (unsigned left = G.present; left;) {
        const int r = reverse ? 31 - __clz(left) : __ffs(left) - 1;
        left &= ~(1u << r);
        const int hi = gs[(r + 1) * PAIR_KINDS];
        for (int idx = gs[r * PAIR_KINDS] + threadIdx.x; idx < hi; idx += blockDim.x) {
            const int2 e = __ldg(&I.ilist[idx]);
            const int la = e.y & 0xffff, lb = e.y >> 16;
            Held first, second;
            load_local(first, G, A.b, la);
            load_local(second, G, A.b, lb);
            solve_points<true>(A, e.x, __ldg(&A.pairs.pair[e.x]), first, second, kind, reverse, fill, track);
            store_local(first, G, la);
            store_local(second, G, lb);
        }
        __syncthreads();
    }
    if (!reverse) {
        group_walls(A, G, kind, false, wtrack);
        __syncthreads();
    }
}

__device__ __forceinline__ void run_group(const SolveArgs& A, const IslandArgs& I, GroupBodies& G, int g) {
    const int nb = I.group_count[g];
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        const int s = I.group_body[(long)g * GROUP_CAP + i];
        G.id[i] = s;
        G.pose[i] = __ldcg(&A.b.pose[s]);
        G.turn[i] = __ldcg(&A.b.turn[s]);
        G.vel[i] = __ldcg(&A.b.vel[s]);
        G.mom[i] = __ldcg(&A.b.mom[s]);
    }
    const int* gs = I.gr_start + (long)g * GROUP_LISTS;
    if (threadIdx.x < 32) {
        const int r = threadIdx.x;
        const unsigned present = __ballot_sync(0xffffffffu, gs[(r + 1) * PAIR_KINDS] > gs[r * PAIR_KINDS]);
        if (r == 0) G.present = present;
    }
    __syncthreads();
    const float h = A.params.w[P_H];
    const int stride = 2 * A.sweeps + 1;  // residual words a substep
    for (int sub = 0; sub < A.substeps; sub++) {
        group_velocities(A, G, nb, h);
        const int base = sub * stride;
        group_sweep(A, I, G, gs, WARM, false, true, base);
        for (int sw = 0; sw < A.sweeps; sw++)
            group_sweep(A, I, G, gs, SOLVE, A.symmetric && sw % 2 == 1, false, base + 1 + sw);
        group_positions(A, G, nb, h);
        if (A.solve_only && sub == A.substeps - 1) continue;
        const int relax = base + 1 + A.sweeps;
        for (int sw = 0; sw < A.sweeps; sw++)
            group_sweep(A, I, G, gs, RELAX, A.symmetric && sw % 2 == 1, sw == 0, relax + sw);
    }
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        const int s = G.id[i];
        __stcg(&A.b.pose[s], G.pose[i]);
        __stcg(&A.b.turn[s], G.turn[i]);
        __stcg(&A.b.vel[s], G.vel[i]);
        __stcg(&A.b.mom[s], G.mom[i]);
    }
    __syncthreads();  // the shared memory is the next group's
}

// A body in no placed pair, all substeps in one thread: velocities, its walls in every sweep it is listed for,
// positions. A fixed body (no inverse mass) is neither moved nor listed.
__device__ __forceinline__ void walls_alone(const SolveArgs& A, int s, float4 pose, float4 turn, float4 hw, float4& vel,
                                            float4& mom, float4 inv, int kind, bool reverse, unsigned* track) {
    Held box;
    box.load(pose, turn, hw, vel, mom, inv);
    if (walls_of<true>(A, box, s, kind, reverse, track)) {
        vel = make_float4(box.velocity[0], box.velocity[1], box.velocity[2], 0.0f);
        mom = make_float4(box.momentum[0], box.momentum[1], box.momentum[2], 0.0f);
    }
}

__device__ __forceinline__ void run_alone(const SolveArgs& A, int s) {
    float4 pose = __ldcg(&A.b.pose[s]);
    if (!(pose.w > 0.0f)) return;
    float4 turn = __ldcg(&A.b.turn[s]), vel = __ldcg(&A.b.vel[s]), mom = __ldcg(&A.b.mom[s]);
    const float4 hw = __ldg(&A.b.half[s]), inv = __ldg(&A.b.inv[s]);
    const int sc = scene_of(A, s);
    const float h = A.params.w[P_H];
    const float g[3] = {word_of(A, sc, P_GX), word_of(A, sc, P_GY), word_of(A, sc, P_GZ)};
    const int stride = 2 * A.sweeps + 1;
    unsigned* res = A.residual ? A.residual + A.wall_split : nullptr;  // a lone body's only contacts are walls
    for (int sub = 0; sub < A.substeps; sub++) {
        vel.x = vel.x + h * g[0];
        vel.y = vel.y + h * g[1];
        vel.z = vel.z + h * g[2];
        const int base = sub * stride;
        if (wall_listed(A, s, pose, hw)) {
            walls_alone(A, s, pose, turn, hw, vel, mom, inv, WARM, false, res ? res + base : nullptr);
            for (int sw = 0; sw < A.sweeps; sw++)
                walls_alone(A, s, pose, turn, hw, vel, mom, inv, SOLVE, A.symmetric && sw % 2 == 1,
                            res ? res + base + 1 + sw : nullptr);
        }
        move_body(pose, turn, vel, mom, inv, h);
        if (!(A.solve_only && sub == A.substeps - 1) && wall_listed(A, s, pose, hw)) {
            const int relax = base + 1 + A.sweeps;
            for (int sw = 0; sw < A.sweeps; sw++)
                walls_alone(A, s, pose, turn, hw, vel, mom, inv, RELAX, A.symmetric && sw % 2 == 1,
                            res ? res + relax + sw : nullptr);
        }
    }
    __stcg(&A.b.pose[s], pose);
    __stcg(&A.b.turn[s], turn);
    __stcg(&A.b.vel[s], vel);
    __stcg(&A.b.mom[s], mom);
}

// Blocks take items from a counter: the groups first (the longer chains), then runs of lone bodies, one a thread.
__global__ void __launch_bounds__(ISLAND_THREADS, 2) k_islands(SolveArgs A, IslandArgs I) {
    __shared__ GroupBodies G;
    const int island = *I.island_n;
    const int base = group_base_of(island, gridDim.x);
    const int ngroups = (island + base - 1) / base;
    const int nfree = *(volatile const int*)&A.counters->free_n;
    const int items = ngroups + (nfree + ISLAND_THREADS - 1) / ISLAND_THREADS;
    for (;;) {
        if (threadIdx.x == 0) G.item = atomicAdd(I.work, 1);
        __syncthreads();
        const int item = G.item;
        __syncthreads();
        if (item >= items) break;
        if (item < ngroups) {
            run_group(A, I, G, item);
        } else {
            const int f = (item - ngroups) * ISLAND_THREADS + threadIdx.x;
            if (f < nfree) run_alone(A, I.free_list[f]);
        }
    }
}

// ------------------------------------------------------------------------------------------------------------
// The learned warm start (no reference counterpart): 16 features a contact point at the step's start, a network's
// starting impulses written in place of the carried ones, and after the solve the impulses it reached (the
// training targets). A row is (round-order position x 4 + point slot); rows past a pair's point count are zero.
// Impulses are scaled by the pair's effective mass x |g| x h, the impulse that holds that mass a substep.

constexpr int FEATURES = 16;

__device__ __forceinline__ float impulse_scale_of(const Params& P, const Params* scene_params, const int* body_scene,
                                                  int a, float im_sum) {
    float gx = P.w[P_GX], gy = P.w[P_GY], gz = P.w[P_GZ];
    if (body_scene) {
        const Params& S = scene_params[body_scene[a]];
        gx = S.w[P_GX], gy = S.w[P_GY], gz = S.w[P_GZ];
    }
    const float g = sqrtf(gx * gx + gy * gy + gz * gz);
    const float s = (g * P.w[P_H]) / fmaxf(im_sum, 1e-30f);
    return s > 0.0f ? s : 1.0f;
}

// A contact point's anchors in the world's frame, and its relative velocity (second's point minus first's).
__device__ __forceinline__ void point_of(const Held& A, const Held& B, const float* n, float4 pa, float4 pb, float* rA,
                                         float* rB, float* rel) {
    if (A.sphere()) {
        for (int k = 0; k < 3; k++) rA[k] = A.half[0] * n[k];
    } else {
        const float anchor[3] = {pa.x, pa.y, pa.z};
        rotate_by(A.q, A.twice, anchor, rA);
    }
    if (B.sphere()) {
        for (int k = 0; k < 3; k++) rB[k] = -(B.half[0] * n[k]);
    } else {
        const float anchor[3] = {pb.x, pb.y, pb.z};
        rotate_by(B.q, B.twice, anchor, rB);
    }
    float va[3], vb[3];
    A.point_velocity(rA, va);
    B.point_velocity(rB, vb);
    for (int k = 0; k < 3; k++) rel[k] = vb[k] - va[k];
}

__global__ void k_features(const int* __restrict__ touching_n, const PairGen now, const Bodies b,
                           const int* __restrict__ degree, Params P, const Params* __restrict__ scene_params,
                           const int* __restrict__ body_scene, float* __restrict__ feat) {
    const int total = *touching_n;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        const int4 rec = now.pair[k];
        const float4 nm = now.normal[k];
        const float n[3] = {nm.x, nm.y, nm.z};
        const int axis = (int)nm.w;
        Held A, B;
        A.load(b.pose[rec.x], b.turn[rec.x], b.half[rec.x], b.vel[rec.x], b.mom[rec.x], b.inv[rec.x]);
        B.load(b.pose[rec.y], b.turn[rec.y], b.half[rec.y], b.vel[rec.y], b.mom[rec.y], b.inv[rec.y]);
        const float s = impulse_scale_of(P, scene_params, body_scene, rec.x, A.im + B.im);
        float ia[3], ib[3];
        A.times_inverse_inertia(n, ia);
        B.times_inverse_inertia(n, ib);
        const float kind[4] = {axis < 3 ? 1.0f : 0.0f, axis >= 3 && axis < 6 ? 1.0f : 0.0f,
                               axis >= 6 && axis < 15 ? 1.0f : 0.0f, axis >= 15 ? 1.0f : 0.0f};
        for (int slot = 0; slot < MOST_POINTS; slot++) {
            float* f = feat + ((size_t)k * MOST_POINTS + slot) * FEATURES;
            if (slot >= rec.z) {
                for (int j = 0; j < FEATURES; j++) f[j] = 0.0f;
                continue;
            }
            const size_t at = (size_t)now.pstart[k] + slot;
            float rA[3], rB[3], rel[3];
            point_of(A, B, n, now.pa[at], now.pb[at], rA, rB, rel);
            float gap = 0.0f;
            for (int j = 0; j < 3; j++) gap += ((B.at[j] + rB[j]) - (A.at[j] + rA[j])) * n[j];
            const float vn = rel[0] * n[0] + rel[1] * n[1] + rel[2] * n[2];
            float vt2 = 0.0f;
            for (int j = 0; j < 3; j++) {
                const float t = rel[j] - vn * n[j];
                vt2 += t * t;
            }
            const float4 imp = now.imp[at];
            const float lt = sqrtf(imp.y * imp.y + imp.z * imp.z + imp.w * imp.w);
            f[0] = gap;
            f[1] = vn;
            f[2] = sqrtf(vt2);
            f[3] = A.im;
            f[4] = B.im;
            f[5] = n[0] * ia[0] + n[1] * ia[1] + n[2] * ia[2];
            f[6] = n[0] * ib[0] + n[1] * ib[1] + n[2] * ib[2];
            f[7] = imp.x / s;
            f[8] = lt / s;
            f[9] = (float)degree[rec.x];
            f[10] = (float)degree[rec.y];
            for (int j = 0; j < 4; j++) f[11 + j] = kind[j];
            f[15] = n[1];
        }
    }
}

// The network's starting impulses in place of the carried ones: normal max(0, p0) s; friction max(0, p1) s along
// the carried tangential impulse, or against the tangential slip where none is carried.
// fresh_only: only the points that carried nothing (contacts new this step, or carried at zero); the others keep
// their carried impulses.
__global__ void k_apply_learned(const int* __restrict__ touching_n, PairGen now, const Bodies b,
                                const float* __restrict__ pred, Params P, const Params* __restrict__ scene_params,
                                const int* __restrict__ body_scene, bool fresh_only) {
    const int total = *touching_n;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        const int4 rec = now.pair[k];
        const float4 nm = now.normal[k];
        const float n[3] = {nm.x, nm.y, nm.z};
        Held A, B;
        A.load(b.pose[rec.x], b.turn[rec.x], b.half[rec.x], b.vel[rec.x], b.mom[rec.x], b.inv[rec.x]);
        B.load(b.pose[rec.y], b.turn[rec.y], b.half[rec.y], b.vel[rec.y], b.mom[rec.y], b.inv[rec.y]);
        const float s = impulse_scale_of(P, scene_params, body_scene, rec.x, A.im + B.im);
        for (int slot = 0; slot < rec.z && slot < MOST_POINTS; slot++) {
            const size_t row = (size_t)k * MOST_POINTS + slot, at = (size_t)now.pstart[k] + slot;
            const float ln = fmaxf(0.0f, pred[2 * row] * s);
            const float lt = fmaxf(0.0f, pred[2 * row + 1] * s);
            const float4 old = now.imp[at];
            if (fresh_only && nonzero_bits(old)) continue;
            float dir[3] = {old.y, old.z, old.w};
            float len = sqrtf(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
            if (!(len > 1e-12f)) {
                float rA[3], rB[3], rel[3];
                point_of(A, B, n, now.pa[at], now.pb[at], rA, rB, rel);
                const float vn = rel[0] * n[0] + rel[1] * n[1] + rel[2] * n[2];
                for (int j = 0; j < 3; j++) dir[j] = -(rel[j] - vn * n[j]);
                len = sqrtf(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
            }
            const float c = len > 1e-12f ? lt / len : 0.0f;
            now.imp[at] = make_float4(ln, dir[0] * c, dir[1] * c, dir[2] * c);
        }
    }
}

// Given starts between twin worlds. A pair's round-order position within its round depends on the order in which
// threads reached it, so it can differ between two worlds in the same state; its touching index t (slot order: first
// body, then its partners in slot order) cannot. by_pair: rows by position -> rows by touching index (pos[t] is t's
// position); by_position: back, for the step that uses them.
__global__ void k_rows_by_pair(const int* __restrict__ touching_n, const int* __restrict__ pos,
                               const float* __restrict__ by_position, float* __restrict__ by_pair) {
    const int total = *touching_n;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const size_t from = (size_t)pos[t] * MOST_POINTS * 2, to = (size_t)t * MOST_POINTS * 2;
        for (int j = 0; j < MOST_POINTS * 2; j++) by_pair[to + j] = by_position[from + j];
    }
}

__global__ void k_rows_by_position(const int* __restrict__ touching_n, const int* __restrict__ pos,
                                   const float* __restrict__ by_pair, float* __restrict__ by_position) {
    const int total = *touching_n;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const size_t to = (size_t)pos[t] * MOST_POINTS * 2, from = (size_t)t * MOST_POINTS * 2;
        for (int j = 0; j < MOST_POINTS * 2; j++) by_position[to + j] = by_pair[from + j];
    }
}

// Whole impulse records between twin worlds, by touching index: a pair's points' normal and tangential impulse and
// rolling impulse as the answers' step left them (by_pair), then in place of the carried ones (apply; with
// fresh_only, only where nothing was carried).
__global__ void k_records_by_pair(const int* __restrict__ touching_n, const PairGen last, float4* __restrict__ imp,
                                  float4* __restrict__ impr) {
    const int total = *touching_n;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int p = last.pos[t];
        const size_t at = (size_t)last.pstart[p];
        const int count = min(last.pair[p].z, MOST_POINTS);
        for (int slot = 0; slot < count; slot++) {
            imp[(size_t)t * MOST_POINTS + slot] = last.imp[at + slot];
            impr[(size_t)t * MOST_POINTS + slot] = last.impr[at + slot];
        }
    }
}

__global__ void k_apply_records(const int* __restrict__ touching_n, PairGen now, const float4* __restrict__ imp,
                                const float4* __restrict__ impr, bool fresh_only) {
    const int total = *touching_n;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int p = now.pos[t];
        const size_t at = (size_t)now.pstart[p];
        const int count = min(now.pair[p].z, MOST_POINTS);
        for (int slot = 0; slot < count; slot++) {
            if (fresh_only && (nonzero_bits(now.imp[at + slot]) || nonzero_bits(now.impr[at + slot]))) continue;
            now.imp[at + slot] = imp[(size_t)t * MOST_POINTS + slot];
            now.impr[at + slot] = impr[(size_t)t * MOST_POINTS + slot];
        }
    }
}

// The impulses the step's solve reached, scaled: the training targets.
__global__ void k_targets(const int* __restrict__ touching_n, const PairGen now, const Bodies b, Params P,
                          const Params* __restrict__ scene_params, const int* __restrict__ body_scene,
                          float* __restrict__ target) {
    const int total = *touching_n;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        const int4 rec = now.pair[k];
        const float s = impulse_scale_of(P, scene_params, body_scene, rec.x, b.pose[rec.x].w + b.pose[rec.y].w);
        for (int slot = 0; slot < MOST_POINTS; slot++) {
            const size_t row = (size_t)k * MOST_POINTS + slot;
            float4 imp = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (slot < rec.z) imp = now.imp[(size_t)now.pstart[k] + slot];
            target[2 * row] = imp.x / s;
            target[2 * row + 1] = sqrtf(imp.y * imp.y + imp.z * imp.z + imp.w * imp.w) / s;
        }
    }
}

// ------------------------------------------------------------------------------------------------------------
// Diagnostics on the device (BoxDiagnostics.of, core/box/BoxDiagnostics.java:18-43, and the penetrations and
// potential energy a long run is judged by): reductions over the state where it lies, sums in doubles.

struct Diag {
    double kinetic, rotational, potential, momentum[3], angular[3];
    unsigned max_penetration, max_wall, max_speed;  // non-negative floats as bits
    int broken;
};

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void k_diag_bodies(int n, const Bodies b, Params P, const Params* __restrict__ scene_params,
                              const int* __restrict__ body_scene, Diag* d) {
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // kinetic, rotational, potential, momentum 3, angular 3
    float wall = 0.0f, speed = 0.0f;
    int broken = 0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        Held h;
        h.load(b.pose[s], b.turn[s], b.half[s], b.vel[s], b.mom[s], b.inv[s]);
        for (int k = 0; k < 3; k++)
            if (!isfinite(h.at[k]) || !isfinite(h.velocity[k]) || !isfinite(h.momentum[k]) || !isfinite(h.q[k]))
                broken = 1;
        const float v2 = h.velocity[0] * h.velocity[0] + h.velocity[1] * h.velocity[1] + h.velocity[2] * h.velocity[2];
        speed = fmaxf(speed, sqrtf(v2));
        float ext[3] = {P.w[P_SX], P.w[P_SY], P.w[P_SZ]}, g[3] = {P.w[P_GX], P.w[P_GY], P.w[P_GZ]};
        if (body_scene) {
            const Params& S = scene_params[body_scene[s]];
            for (int k = 0; k < 3; k++) ext[k] = S.w[P_SX + k], g[k] = S.w[P_GX + k];
        }
        // how far past a wall the body reaches: a sphere's surface, a box's corners
        if (h.sphere()) {
            for (int k = 0; k < 3; k++) wall = fmaxf(wall, fmaxf(h.half[0] - h.at[k], (h.at[k] + h.half[0]) - ext[k]));
        } else {
            for (int c = 0; c < 8; c++) {
                float off[3], r[3];
                for (int k = 0; k < 3; k++) off[k] = ((c >> k) & 1) ? h.half[k] : -h.half[k];
                rotate_by(h.q, h.twice, off, r);
                for (int k = 0; k < 3; k++) {
                    const float p = h.at[k] + r[k];
                    wall = fmaxf(wall, fmaxf(-p, p - ext[k]));
                }
            }
        }
        if (!(h.im > 0.0f)) continue;
        const double m = 1.0 / (double)h.im;
        double lw = 0.0;
        for (int k = 0; k < 3; k++) lw += (double)h.momentum[k] * (double)h.omega[k];
        const double vv = (double)h.velocity[0] * h.velocity[0] + (double)h.velocity[1] * h.velocity[1] +
                          (double)h.velocity[2] * h.velocity[2];
        acc[0] += 0.5 * m * vv + 0.5 * lw;
        acc[1] += 0.5 * lw;
        acc[2] += -m * ((double)g[0] * h.at[0] + (double)g[1] * h.at[1] + (double)g[2] * h.at[2]);
        for (int k = 0; k < 3; k++) acc[3 + k] += m * h.velocity[k];
        const double x = h.at[0], y = h.at[1], z = h.at[2], u = h.velocity[0], v = h.velocity[1], w = h.velocity[2];
        acc[6] += m * (y * w - z * v) + h.momentum[0];
        acc[7] += m * (z * u - x * w) + h.momentum[1];
        acc[8] += m * (x * v - y * u) + h.momentum[2];
    }
    for (int k = 0; k < 9; k++) acc[k] = warp_sum(acc[k]);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&d->kinetic, acc[0]);
        atomicAdd(&d->rotational, acc[1]);
        atomicAdd(&d->potential, acc[2]);
        for (int k = 0; k < 3; k++) {
            atomicAdd(&d->momentum[k], acc[3 + k]);
            atomicAdd(&d->angular[k], acc[6 + k]);
        }
    }
    atomicMax(&d->max_wall, __float_as_uint(fmaxf(wall, 0.0f)));
    atomicMax(&d->max_speed, __float_as_uint(speed));
    if (broken) atomicExch(&d->broken, 1);
}

// The deepest overlap at the last step's contact points, their gaps measured again from where the bodies are now.
__global__ void k_diag_contacts(const int* __restrict__ touching_n, const PairGen last, const Bodies b, Diag* d) {
    const int total = *touching_n;
    float deepest = 0.0f;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        const int4 rec = last.pair[k];
        const float4 nm = last.normal[k];
        const float n[3] = {nm.x, nm.y, nm.z};
        Held A, B;
        A.load(b.pose[rec.x], b.turn[rec.x], b.half[rec.x], b.vel[rec.x], b.mom[rec.x], b.inv[rec.x]);
        B.load(b.pose[rec.y], b.turn[rec.y], b.half[rec.y], b.vel[rec.y], b.mom[rec.y], b.inv[rec.y]);
        for (int slot = 0; slot < rec.z && slot < MOST_POINTS; slot++) {
            const size_t at = (size_t)last.pstart[k] + slot;
            float rA[3], rB[3], rel[3];
            point_of(A, B, n, last.pa[at], last.pb[at], rA, rB, rel);
            float gap = 0.0f;
            for (int j = 0; j < 3; j++) gap += ((B.at[j] + rB[j]) - (A.at[j] + rA[j])) * n[j];
            deepest = fmaxf(deepest, -gap);
        }
    }
    atomicMax(&d->max_penetration, __float_as_uint(fmaxf(deepest, 0.0f)));
}

// The positional complementarity error at each contact point of the last step, from the bodies' state at its end
// (no reference counterpart; the reference has no residual): the depth the relative normal velocity would close
// within a substep beyond what the gap allows, h max(0, -(vn + max(gap, 0) / h)) for a point within the margin, and
// the depth the bodies already overlap, max(0, -gap); the larger. A row is (round-order position x 4 + point slot);
// rows past a pair's point count are -1.
__global__ void k_contact_errors(const int* __restrict__ touching_n, const PairGen last, const Bodies b, Params P,
                                 float* __restrict__ out) {
    const int total = *touching_n;
    const float h = P.w[P_H], margin = P.w[P_MARGIN];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        const int4 rec = last.pair[k];
        const float4 nm = last.normal[k];
        const float n[3] = {nm.x, nm.y, nm.z};
        Held A, B;
        A.load(b.pose[rec.x], b.turn[rec.x], b.half[rec.x], b.vel[rec.x], b.mom[rec.x], b.inv[rec.x]);
        B.load(b.pose[rec.y], b.turn[rec.y], b.half[rec.y], b.vel[rec.y], b.mom[rec.y], b.inv[rec.y]);
        for (int slot = 0; slot < MOST_POINTS; slot++) {
            float e = -1.0f;
            if (slot < rec.z) {
                const size_t at = (size_t)last.pstart[k] + slot;
                float rA[3], rB[3], rel[3];
                point_of(A, B, n, last.pa[at], last.pb[at], rA, rB, rel);
                float gap = 0.0f;
                for (int j = 0; j < 3; j++) gap += ((B.at[j] + rB[j]) - (A.at[j] + rA[j])) * n[j];
                const float vn = rel[0] * n[0] + rel[1] * n[1] + rel[2] * n[2];
                const float closing = gap <= margin ? h * fmaxf(0.0f, -(vn + fmaxf(gap, 0.0f) / h)) : 0.0f;
                e = fmaxf(closing, fmaxf(0.0f, -gap));
            }
            out[(size_t)k * MOST_POINTS + slot] = e;
        }
    }
}

// Boxes.show :801-820.
__global__ void k_show(int n, const Bodies b, float* __restrict__ shown) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float* sh = shown + (long)s * SHOWN_STRIDE;
    const float4 p = b.pose[s], q = b.turn[s], h = b.half[s];
    sh[0] = sh[4];
    sh[1] = sh[5];
    sh[2] = sh[6];
    sh[4] = p.x;
    sh[5] = p.y;
    sh[6] = p.z;
    sh[8] = h.x;
    sh[9] = h.y;
    sh[10] = h.z;
    sh[12] = sh[16];
    sh[13] = sh[17];
    sh[14] = sh[18];
    sh[15] = sh[19];
    sh[16] = q.x;
    sh[17] = q.y;
    sh[18] = q.z;
    sh[19] = q.w;
    sh[3] = h.w;
}

__global__ void k_totals(const Counters* c, Totals* t) {
    t->last[0] = c->touching;
    t->last[1] = c->points;
    t->last[2] = c->rounds;
    t->last[3] = c->unplaced;
    t->last[4] = c->unlisted;
    t->most_rounds = max(t->most_rounds, c->rounds);
    t->unplaced += c->unplaced;
    t->unlisted += c->unlisted;
    if (t->status == ST_OK) t->status = c->status;
    t->steps += 1;
}

// Activity of the last step, for the solve's algorithmic byte count: bodies in a touching pair or holding a
// wall impulse, and wall records held.
__global__ void k_activity(int n, const int* __restrict__ inc_count, const unsigned long long* __restrict__ wmask,
                           long long* out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const unsigned long long m = wmask[s];
    const bool paired = inc_count != nullptr && inc_count[s] > 0;
    if (paired || m) atomicAdd((unsigned long long*)&out[0], 1ull);
    if (m) atomicAdd((unsigned long long*)&out[1], (unsigned long long)__popcll(m));
}

// Each body's inverse principal moments, once its half-extents, shape and inverse mass are loaded.
__global__ void k_inverse_inertia(int n, const float4* __restrict__ pose, const float4* __restrict__ half,
                                  float4* __restrict__ inv) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float i3[3];
    inverse_inertia(half[s], pose[s].w, i3);
    inv[s] = make_float4(i3[0], i3[1], i3[2], 0.0f);
}

// ------------------------------------------------------------------------------------------------------------
// Host orchestration.

int blocks_for(long n, int threads) { return (int)std::max<long>(1, (n + threads - 1) / threads); }

int launch_cooperative(vxr_box_world* w, const void* fn, int blocks, int threads, void** args) {
    cudaError_t e;
    if (w->capturing) {  // the form a stream capture records as a cooperative kernel node
        cudaLaunchConfig_t c = {};
        c.gridDim = dim3(blocks);
        c.blockDim = dim3(threads);
        c.stream = w->stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        c.attrs = attr;
        c.numAttrs = 1;
        e = cudaLaunchKernelExC(&c, fn, args);
    } else {
        e = cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(threads), args, 0, w->stream);
    }
    if (e != cudaSuccess) return fail(w, std::string("cooperative launch: ") + cudaGetErrorString(e));
    return VXR_OK;
}

GridBarrier barrier_of(vxr_box_world* w) {
    GridBarrier g;
    g.count = &w->counters->bar_count;
    g.generation = &w->counters->bar_gen;
    g.abort = &w->counters->abort;
    g.status = &w->counters->status;
    g.limit_ns = w->wait_limit_ns;  // 2 s unless set: far above any barrier's honest wait
    return g;
}

int mark(vxr_box_world* w, int which) {
    if (!w->profile) return VXR_OK;
    const int need = w->events_used + 1;
    while ((int)w->events.size() < need) {
        cudaEvent_t e;
        VXR_CUDA(cudaEventCreate(&e));
        w->events.push_back(e);
    }
    (void)which;
    VXR_CUDA(cudaEventRecord(w->events[w->events_used++], w->stream));
    return VXR_OK;
}

// Launches per step, counted as they are made.
#define LAUNCHED(k) (w->launches += (k))

// Words of one part of the residual record (the pairs' or the walls'): a word for each sweep of every substep.
int residual_half(const vxr_box_world* w) { return w->substeps * (2 * w->sweeps + 1); }

// Whether a step solves its small components by island blocks: on by default; off where a substep's sweep count
// depends on a residual over every contact (the measuring tolerance), which only the grid phases gather.
bool islands_on(const vxr_box_world* w) {
    return w->islands && w->has_grid && !(w->measure && w->tolerance > 0.0f);
}

// One whole step, enqueued on the world's stream.
int enqueue_step(vxr_box_world* w) {
    cudaStream_t st = w->stream;
    const int n = w->n;
    if (w->scenes > 0 && !w->scene_params_set) {
        w->error = "a batch of scenes needs its scenes' parameters (vxr_box_scene_params) before a step";
        return VXR_EINVAL;
    }
    int rc0 = mark(w, 0);
    if (rc0) return rc0;
    VXR_CUDA(cudaMemsetAsync(w->counters, 0, sizeof(Counters), st));
    VXR_CUDA(cudaMemsetAsync(w->wall_count, 0, sizeof(int) * 4 * w->substeps, st));
    PairGen& now = w->gen[w->cur];
    PairGen& was = w->gen[w->cur ^ 1];
    if (w->has_grid) {
        GridDims g{w->nx, w->ny, w->nz, w->cell, w->reach_cells};
        const float margin = w->params.w[P_MARGIN];
        VXR_CUDA(cudaMemsetAsync(w->cell_count, 0, sizeof(int) * w->cells, st));
        VXR_CUDA(cudaMemsetAsync(w->cell_fill, 0, sizeof(int) * w->cells, st));
        const SceneGrids sg{w->body_scene, w->scene_grid, w->scene_cell};
        k_bin<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, g, sg, w->b.pose, w->b.turn, w->b.half, w->keys, w->reach,
                                                         w->cell_count);
        exclusive_scan(w->cell_count, w->cell_start, w->cells, w->scan_tiles, st);
        k_scatter<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, w->keys, w->cell_start, w->cell_fill,
                                                             w->order_tmp);
        k_stable<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, w->keys, w->cell_start, w->order_tmp, w->order);
        if (w->list_tiled && !w->body_scene && w->reach_cells == 1) {  // the tiled list: a block a run of cells
            const int tiles = ((w->nx + TILE_X - 1) / TILE_X) * w->ny * w->nz;
            k_list_tiled<<<tiles, 256, 0, st>>>(g, margin, w->b.pose, w->reach, w->keys, w->cell_start, w->order,
                                                w->partner, w->found, w->kept, w->counters);
        } else {  // batched scenes' grids, or a neighbourhood wider than 27 cells: a thread a body
            k_list<<<blocks_for(n, 128), 128, 0, st>>>(n, g, sg, margin, w->b.pose, w->reach, w->keys, w->cell_start,
                                                      w->order, w->partner, w->found, w->kept, w->counters);
        }
        exclusive_scan(w->kept, w->cand_start, n, w->scan_tiles, st);
        k_candidates<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, w->cap, w->kept, w->cand_start, w->partner,
                                                                w->cand_a, w->cand_b, w->counters);
        LAUNCHED(4 + 3 + 3 + 1);  // bin, scatter, stable, list, two scans of three, candidates
        if (int rc = mark(w, 1)) return rc;
        const int cblocks = w->sms * 8;
        k_collide<<<cblocks, 128, 0, st>>>(w->cand_start + n, w->cap, margin, w->cand_a, w->cand_b, w->b.pose,
                                            w->b.turn, w->b.half, w->man.head, w->man.axis, w->man.pa, w->man.pb);
        k_touch_count<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, w->cap, w->cand_start, w->man.head,
                                                                 w->tcount);
        exclusive_scan(w->tcount, now.tstart, n, w->scan_tiles, st);
        k_touch_list<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, w->cap, w->cand_start, w->cand_b, w->man.head,
                                                                now.tstart, w->ta, now.tb, w->tcand, w->counters);
        const int tblocks = w->sms * 4;
        if (w->cold) {  // the plain solver from nothing: no impulse carried from the step before
            VXR_CUDA(cudaMemsetAsync(w->imp_t, 0, sizeof(float4) * (size_t)w->cap * MOST_POINTS, st));
            VXR_CUDA(cudaMemsetAsync(w->impr_t, 0, sizeof(float4) * (size_t)w->cap * MOST_POINTS, st));
        } else {
            k_carry<<<tblocks, THREADS, 0, st>>>(now.tstart + n, w->ta, now.tb, w->tcand, w->man, was, w->b.half,
                                                w->imp_t, w->impr_t);
        }
        LAUNCHED(1 + 1 + 3 + 1 + 1);  // collide, touch count, scan, touch list, carry
        if (int rc = mark(w, 2)) return rc;
        // colouring
        VXR_CUDA(cudaMemsetAsync(w->inc_count, 0, sizeof(int) * n, st));
        VXR_CUDA(cudaMemsetAsync(w->inc_fill, 0, sizeof(int) * n, st));
        VXR_CUDA(cudaMemsetAsync(w->colour, 0xff, sizeof(int) * w->cap, st));
        k_inc_count<<<tblocks, THREADS, 0, st>>>(now.tstart + n, w->ta, now.tb, w->inc_count);
        exclusive_scan(w->inc_count, w->inc_start, n, w->scan_tiles, st);
        k_inc_fill<<<tblocks, THREADS, 0, st>>>(now.tstart + n, w->ta, now.tb, w->inc_start, w->inc_fill,
                                               w->inc_list);
        {
            const int* tn = now.tstart + n;
            GridBarrier bar = barrier_of(w);
            void* args[] = {(void*)&tn, (void*)&w->ta, (void*)&now.tb, (void*)&w->inc_start, (void*)&w->inc_list,
                            (void*)&w->colour, (void*)&w->counters, (void*)&bar};
            int rc = launch_cooperative(w, (const void*)k_colour, w->colour_blocks, THREADS, args);
            if (rc) return rc;
        }
        // islands: the components of the placed pairs, the small ones packed into groups
        const bool isl = islands_on(w);
        if (isl) {
            const int* tn = now.tstart + n;
            k_uf_init<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, w->parent, w->isl_size, w->isl_fill);
            k_uf_link<<<tblocks, THREADS, 0, st>>>(tn, w->ta, now.tb, w->colour, w->parent);
            k_uf_flatten<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, w->parent, w->comp, w->isl_size);
            k_largest<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, w->comp, w->isl_size, w->counters);
            k_classify<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, w->comp, w->isl_size, w->isl_key,
                                                                  w->body_group, w->grid_list, w->free_list,
                                                                  w->counters);
            exclusive_scan(w->isl_key, w->isl_offset, n, w->scan_tiles, st);
            VXR_CUDA(cudaMemsetAsync(w->group_count, 0, sizeof(int) * w->groups_max, st));
            VXR_CUDA(cudaMemsetAsync(w->group_base, 0x7f, sizeof(int) * w->groups_max, st));
            k_group_base<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, w->comp, w->isl_size, w->isl_offset,
                                                                    w->body_group, w->group_base, w->island_blocks);
            k_assign<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, w->comp, w->isl_size, w->isl_offset,
                                                                w->group_base, w->isl_fill, w->body_group,
                                                                w->body_local, w->group_body, w->group_count,
                                                                w->island_blocks);
            VXR_CUDA(cudaMemsetAsync(w->gr_count, 0, sizeof(int) * (size_t)w->groups_max * GROUP_LISTS, st));
            VXR_CUDA(cudaMemsetAsync(w->gr_fill, 0, sizeof(int) * (size_t)w->groups_max * GROUP_LISTS, st));
            LAUNCHED(7 + 3);  // init, link, flatten, largest, classify, group base, assign, scan
        }
        VXR_CUDA(cudaMemsetAsync(w->round_count, 0, sizeof(int) * ALL_BUCKETS, st));
        VXR_CUDA(cudaMemsetAsync(w->bucket_most, 0, sizeof(int) * ALL_BUCKETS, st));
        VXR_CUDA(cudaMemsetAsync(w->round_fill, 0, sizeof(int) * ALL_BUCKETS, st));
        VXR_CUDA(cudaMemsetAsync(w->body_colours, 0, sizeof(unsigned) * n, st));
        const int* groups_of = isl ? w->body_group : nullptr;
        k_round_count<<<tblocks, THREADS, 0, st>>>(now.tstart + n, w->colour, w->round_count, w->bucket_most,
                                                  w->counters, w->ta,
                                                  now.tb, w->body_colours, w->tcand, w->man.head, w->b.half,
                                                  groups_of, w->gr_count);
        exclusive_scan(w->round_count, w->bucket_start, ALL_BUCKETS, w->scan_tiles, st);
        if (isl) {
            exclusive_scan(w->gr_count, w->gr_start, w->groups_max * GROUP_LISTS, w->scan_tiles, st);
            LAUNCHED(3);
        }
        k_round_starts<<<1, 64, 0, st>>>(w->bucket_start, w->round_start);
        k_bucket_points<<<1, 32, 0, st>>>(w->round_count, w->bucket_most, w->bucket_pstart);
        k_order<<<tblocks, THREADS, 0, st>>>(now.tstart + n, w->colour, w->bucket_start, w->bucket_most,
                                            w->bucket_pstart, w->round_fill, w->ta,
                                            w->tcand, w->man, w->imp_t, w->impr_t, now,
                                            w->body_colours, w->b.half, groups_of, w->body_local, w->gr_start,
                                            w->gr_fill, w->ilist);
        LAUNCHED(1 + 3 + 1 + 1 + 1 + 3 + 1 + 1 + 1);  // inc count, scan, inc fill, colour, round count, scan,
                                                    // starts, bucket points, order
        if (w->learn_mode > 0) {
            const int* tn = now.tstart + n;
            k_features<<<tblocks, THREADS, 0, st>>>(tn, now, w->b, w->inc_count, w->params, w->scene_params,
                                                    w->body_scene, w->lfeat);
            LAUNCHED(1);
            if (w->learn_mode >= 6) {
                k_apply_records<<<tblocks, THREADS, 0, st>>>(tn, now, w->lgiven_imp, w->lgiven_impr,
                                                             w->learn_mode == 7);
                LAUNCHED(1);
            } else if (w->learn_mode >= 2) {
                if (w->learn_mode <= 3) {
                    if (vxr_mlp_forward_device(w->learn_net, w->lfeat, tn, MOST_POINTS, w->cap * MOST_POINTS,
                                               w->lpred, st) != VXR_OK) {
                        w->error = "the learned warm start's network did not launch";
                        return VXR_ECUDA;
                    }
                    LAUNCHED(1);
                } else {
                    k_rows_by_position<<<tblocks, THREADS, 0, st>>>(tn, now.pos, w->lgiven, w->lpred);
                    LAUNCHED(1);
                }
                k_apply_learned<<<tblocks, THREADS, 0, st>>>(tn, now, w->b, w->lpred, w->params, w->scene_params,
                                                             w->body_scene,
                                                             w->learn_mode == 3 || w->learn_mode == 5);
                LAUNCHED(1);
            }
        }
    } else {
        if (int rc = mark(w, 1)) return rc;
        if (int rc = mark(w, 2)) return rc;
    }
    if (int rc = mark(w, 3)) return rc;
    {
        SolveArgs A;
        A.n = n;
        A.b = w->b;
        A.wall = w->wall;
        A.wroll = w->wroll;
        A.wmask = w->wmask;
        A.wall_list = w->wall_list;
        A.wall_count = w->wall_count;
        A.version = w->version;
        A.listed = w->listed;
        A.body_colours = w->body_colours;
        A.schedule = w->schedule;
        A.residual = w->measure ? w->residual : nullptr;
        A.wall_split = residual_half(w);
        A.solve_only = w->solve_only;
        if (w->measure)
            VXR_CUDA(cudaMemsetAsync(w->residual, 0, sizeof(unsigned) * 2 * residual_half(w), st));
        A.pairs = now;
        A.round_start = w->round_start;
        A.counters = w->counters;
        A.substeps = w->first_substeps > 0 ? w->first_substeps : w->substeps;
        A.sweeps = w->active_sweeps;
        A.tolerance = w->measure ? w->tolerance : 0.0f;
        A.used = w->used;
        A.symmetric = w->symmetric;
        A.params = w->params;
        A.scene_params = w->scene_params;
        A.body_scene = w->body_scene;
        A.bar = barrier_of(w);
        A.trace = w->tracing ? w->trace : nullptr;
        A.trace_cap = w->trace_cap;
        const bool isl = islands_on(w);
        A.grid_list = isl ? w->grid_list : nullptr;
        A.grid_n = isl ? &w->counters->grid_n : nullptr;
        if (isl) {  // the small components and the lone bodies, then the grid phases for the rest
            IslandArgs I;
            I.group_body = w->group_body;
            I.group_count = w->group_count;
            I.gr_start = w->gr_start;
            I.ilist = w->ilist;
            I.free_list = w->free_list;
            I.island_n = w->isl_offset + n;
            I.work = &w->counters->work;
            k_islands<<<w->island_blocks, ISLAND_THREADS, 0, st>>>(A, I);
            LAUNCHED(1);
        }
        VXR_CUDA(cudaMemsetAsync(&w->counters->bar_count, 0, 2 * sizeof(unsigned int), st));
        void* args[] = {(void*)&A};
        int rc = launch_cooperative(w, (const void*)k_solve, w->solve_blocks, SOLVE_THREADS, args);
        if (rc) return rc;
    }
    if (int rc = mark(w, 4)) return rc;
    if (w->has_grid && w->learn_mode == 1) {
        k_targets<<<w->sms * 4, THREADS, 0, st>>>(now.tstart + n, now, w->b, w->params, w->scene_params,
                                                  w->body_scene, w->ltarget);
        LAUNCHED(1);
    }
    k_show<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, w->b, w->shown);
    k_totals<<<1, 1, 0, st>>>(w->counters, w->totals);
    LAUNCHED(1 + 2);  // solve, show, totals
    VXR_CUDA(cudaGetLastError());
    if (w->has_grid) w->cur ^= 1;
    return VXR_OK;
}

// Forgets a captured pair of steps: what it baked in (parameters, the pair generation, switches) has changed.
void drop_graph(vxr_box_world* w) {
    if (w->graph_exec) cudaGraphExecDestroy(w->graph_exec);
    if (w->graph) cudaGraphDestroy(w->graph);
    w->graph_exec = nullptr;
    w->graph = nullptr;
}

// Every impulse, wall record and pair list back to zero, as the reference's runner.clear() leaves them.
int clear_dynamic(vxr_box_world* w) {
    cudaStream_t st = w->stream;
    const int n = w->n;
    VXR_CUDA(cudaMemsetAsync(w->wall, 0, sizeof(float4) * (size_t)n * WALL_RECORDS, st));
    VXR_CUDA(cudaMemsetAsync(w->wroll, 0, sizeof(float4) * (size_t)n * 6, st));
    VXR_CUDA(cudaMemsetAsync(w->wmask, 0, sizeof(unsigned long long) * n, st));
    VXR_CUDA(cudaMemsetAsync(w->shown, 0, sizeof(float) * (size_t)n * SHOWN_STRIDE, st));
    VXR_CUDA(cudaMemsetAsync(w->totals, 0, sizeof(Totals), st));
    if (w->has_grid)
        for (int g = 0; g < 2; g++) VXR_CUDA(cudaMemsetAsync(w->gen[g].tstart, 0, sizeof(int) * ((size_t)n + 1), st));
    w->cur = 0;
    drop_graph(w);
    return VXR_OK;
}

int ensure_pinned(vxr_box_world* w, size_t bytes) {
    if (w->pinned_bytes >= bytes) return VXR_OK;
    if (w->pinned) cudaFreeHost(w->pinned);
    w->pinned = nullptr;
    w->pinned_bytes = 0;
    VXR_CUDA(cudaMallocHost(&w->pinned, bytes));
    w->pinned_bytes = bytes;
    return VXR_OK;
}

// float4 array <- four host arrays (any may be null: then `fill`)
int upload4(vxr_box_world* w, float4* dst, const float* a, const float* b, const float* c, const float* d,
            float fill_d) {
    const int n = w->n;
    int rc = ensure_pinned(w, sizeof(float4) * (size_t)n);
    if (rc) return rc;
    float* p = w->pinned;
    for (int s = 0; s < n; s++) {
        p[4 * s + 0] = a ? a[s] : 0.0f;
        p[4 * s + 1] = b ? b[s] : 0.0f;
        p[4 * s + 2] = c ? c[s] : 0.0f;
        p[4 * s + 3] = d ? d[s] : fill_d;
    }
    VXR_CUDA(cudaMemcpyAsync(dst, p, sizeof(float4) * (size_t)n, cudaMemcpyHostToDevice, w->stream));
    VXR_CUDA(cudaStreamSynchronize(w->stream));
    return VXR_OK;
}

// x y z u v w lx ly lz qx qy qz qw, field after field.
__global__ void k_state13(int n, const Bodies b, float* __restrict__ out) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const float4 p = b.pose[s], v = b.vel[s], l = b.mom[s], q = b.turn[s];
        const float f[13] = {p.x, p.y, p.z, v.x, v.y, v.z, l.x, l.y, l.z, q.x, q.y, q.z, q.w};
#pragma unroll
        for (int k = 0; k < 13; k++) out[(size_t)k * n + s] = f[k];
    }
}

// Boxes.params / softness (Boxes.java:212-251), computed in double and rounded to f32 bits.
int32_t f32bits(double v) {
    float f = (float)v;
    int32_t i;
    std::memcpy(&i, &f, 4);
    return i;
}
void softness(double hertz, double zeta, double h, double* out) {
    if (hertz == 0) {
        out[0] = 0;
        out[1] = 1;
        out[2] = 0;
        return;
    }
    const double omega = 2 * M_PI * hertz;
    const double a1 = 2 * zeta + h * omega;
    const double a2 = h * omega * a1;
    const double a3 = 1 / (1 + a2);
    out[0] = omega / a1;
    out[1] = a2 * a3;
    out[2] = a3;
}

// BoxDiagnostics.momentum in doubles (BoxDiagnostics.java:46-53): L = R I Rᵀ ω.
void rotate_d(const double* q, const double* p, double* out) {
    const double t0 = 2 * (q[1] * p[2] - q[2] * p[1]), t1 = 2 * (q[2] * p[0] - q[0] * p[2]),
                 t2 = 2 * (q[0] * p[1] - q[1] * p[0]);
    const double t[3] = {t0, t1, t2};
    const double qt[3] = {q[1] * t[2] - q[2] * t[1], q[2] * t[0] - q[0] * t[2], q[0] * t[1] - q[1] * t[0]};
    for (int a = 0; a < 3; a++) out[a] = p[a] + q[3] * t[a] + qt[a];
}

}  // namespace

// ================================================================================================================
// C-ABI
extern "C" {

const char* vxr_version(void) { return "vxr-b200 0.1 (sm_100a)"; }

int32_t vxr_box_make_params(double h, double gx, double gy, double gz, double sx, double sy, double sz,
                            double mu_static, double mu_kinetic, double margin, double mu_rolling, int32_t* out) {
    if (!out) return VXR_EINVAL;
    if (!(mu_rolling >= 0) || std::isinf(mu_rolling)) return VXR_EINVAL;
    if (!(margin >= 0) || std::isinf(margin)) return VXR_EINVAL;
    if (!(h > 0) || !(sx > 0) || !(sy > 0) || !(sz > 0)) return VXR_EINVAL;
    if (!(mu_static >= 0) || !(mu_kinetic >= 0) || std::isinf(mu_static) || std::isinf(mu_kinetic)) return VXR_EINVAL;
    const double hertz = std::min(150.0, 0.25 / h);
    double soft[3], stiff[3];
    softness(hertz, 10.0, h, soft);
    softness(2 * hertz, 10.0, h, stiff);
    const double v[18] = {h, gx, gy, gz, sx, sy, sz, mu_static, mu_kinetic, margin, soft[0], soft[1], soft[2],
                          stiff[0], stiff[1], stiff[2], 3.0, mu_rolling};
    for (int k = 0; k < 18; k++) out[k] = f32bits(v[k]);
    return VXR_OK;
}

int32_t vxr_box_make_grid(double sx, double sy, double sz, double widest_half_diagonal, double margin,
                          vxr_grid* out) {
    if (!out) return VXR_EINVAL;
    const double widest = 2 * widest_half_diagonal + margin;
    if (!(widest > 0)) return VXR_EINVAL;
    out->nx = std::max(1, (int)std::ceil(sx / widest));
    out->ny = std::max(1, (int)std::ceil(sy / widest));
    out->nz = std::max(1, (int)std::ceil(sz / widest));
    out->cell = (float)widest;
    return VXR_OK;
}

vxr_box_world* vxr_box_create(const vxr_box_config* cfg, int32_t* status) {
    auto set = [&](int32_t s) {
        if (status) *status = s;
    };
    if (!cfg || cfg->bodies < 1 || cfg->substeps < 1 || cfg->sweeps < 1) {
        set(VXR_EINVAL);
        return nullptr;
    }
    vxr_box_world* w = new vxr_box_world();
    w->n = cfg->bodies;
    w->substeps = cfg->substeps;
    w->sweeps = cfg->sweeps;
    w->active_sweeps = cfg->sweeps;
    w->symmetric = cfg->symmetric ? 1 : 0;
    w->schedule = cfg->schedule == 1 ? 1 : 0;
    w->device = cfg->device;
    w->has_grid = (cfg->bodies > 1 && cfg->grid.nx > 0 && cfg->grid.ny > 0 && cfg->grid.nz > 0 && cfg->grid.cell > 0)
                      ? 1 : 0;
    if (w->has_grid) {
        w->nx = cfg->grid.nx;
        w->ny = cfg->grid.ny;
        w->nz = cfg->grid.nz;
        w->cell = cfg->grid.cell;
        w->reach_cells = cfg->reach_cells > 0 ? cfg->reach_cells : 1;
        long cells = (long)w->nx * w->ny * w->nz;
        if (cells > (1L << 30)) {
            set(VXR_EINVAL);
            delete w;
            return nullptr;
        }
        w->cells = (int)cells;
    }
    long cap = cfg->max_pairs > 0 ? cfg->max_pairs : (long)w->n * SLOTS;
    if (cap > (1L << 30)) cap = 1L << 30;
    w->cap = (int)cap;
    auto bad = [&](int rc) {
        set(rc);
        vxr_box_destroy(w);
        return (vxr_box_world*)nullptr;
    };
    if (cudaSetDevice(w->device) != cudaSuccess) return bad(VXR_ECUDA);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, w->device) != cudaSuccess) return bad(VXR_ECUDA);
    w->sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking) != cudaSuccess) return bad(VXR_ECUDA);
    cudaEventCreate(&w->ev0);
    cudaEventCreate(&w->ev1);
    const int n = w->n;
    int rc = 0;
    rc |= alloc(w, &w->b.pose, n);
    rc |= alloc(w, &w->b.turn, n);
    rc |= alloc(w, &w->b.half, n);
    rc |= alloc(w, &w->b.vel, n);
    rc |= alloc(w, &w->b.mom, n);
    rc |= alloc(w, &w->b.inv, n);
    rc |= alloc(w, &w->wall, (size_t)n * WALL_RECORDS);
    rc |= alloc(w, &w->wroll, (size_t)n * 6);
    rc |= alloc(w, &w->wmask, n);
    rc |= alloc(w, &w->shown, (size_t)n * SHOWN_STRIDE);
    rc |= alloc(w, &w->counters, 1);
    rc |= alloc(w, &w->totals, 1);
    // groups the bodies can fill: one for every GROUP_BASE_LEAST placed (the least base), plus the last part-filled one
    w->groups_max = n / GROUP_BASE_LEAST + 2;
    rc |= alloc(w, &w->scan_tiles,
                scan_tiles_for(std::max(std::max(n, w->cells), w->groups_max * GROUP_LISTS + 1)) + 1);
    rc |= alloc(w, &w->round_count, ALL_BUCKETS);
    rc |= alloc(w, &w->round_start, MOST_ROUNDS + 2);
    rc |= alloc(w, &w->bucket_start, ALL_BUCKETS + 1);
    rc |= alloc(w, &w->bucket_most, ALL_BUCKETS);
    rc |= alloc(w, &w->bucket_pstart, ALL_BUCKETS + 1);
    rc |= alloc(w, &w->wall_list, n);
    rc |= alloc(w, &w->wall_count, 4 * (size_t)w->substeps);
    rc |= alloc(w, &w->version, n);
    rc |= alloc(w, &w->listed, n);
    rc |= alloc(w, &w->body_colours, n);
    rc |= alloc(w, &w->residual, 2 * (size_t)residual_half(w));  // the pairs' part, then the walls'
    rc |= alloc(w, &w->used, 2 * (size_t)w->substeps);
    rc |= alloc(w, &w->round_fill, ALL_BUCKETS);
    if (w->has_grid) {
        rc |= alloc(w, &w->keys, n);
        rc |= alloc(w, &w->cell_count, w->cells);
        rc |= alloc(w, &w->cell_start, (size_t)w->cells + 1);
        rc |= alloc(w, &w->cell_fill, w->cells);
        rc |= alloc(w, &w->order_tmp, n);
        rc |= alloc(w, &w->order, n);
        rc |= alloc(w, &w->reach, n);
        rc |= alloc(w, &w->partner, (size_t)n * SLOTS);
        rc |= alloc(w, &w->found, n);
        rc |= alloc(w, &w->kept, n);
        rc |= alloc(w, &w->cand_start, (size_t)n + 1);
        rc |= alloc(w, &w->cand_a, w->cap);
        rc |= alloc(w, &w->cand_b, w->cap);
        rc |= alloc(w, &w->tcount, n);
        rc |= alloc(w, &w->man.head, w->cap);
        rc |= alloc(w, &w->man.axis, w->cap);
        rc |= alloc(w, &w->man.pa, (size_t)w->cap * MOST_POINTS);
        rc |= alloc(w, &w->man.pb, (size_t)w->cap * MOST_POINTS);
        rc |= alloc(w, &w->ta, w->cap);
        rc |= alloc(w, &w->tcand, w->cap);
        rc |= alloc(w, &w->imp_t, (size_t)w->cap * MOST_POINTS);
        rc |= alloc(w, &w->impr_t, (size_t)w->cap * MOST_POINTS);
        for (int g = 0; g < 2; g++) {
            PairGen& p = w->gen[g];
            rc |= alloc(w, &p.tstart, (size_t)n + 1);
            rc |= alloc(w, &p.tb, w->cap);
            rc |= alloc(w, &p.pos, w->cap);
            rc |= alloc(w, &p.pair, w->cap);
            rc |= alloc(w, &p.normal, w->cap);
            rc |= alloc(w, &p.pstart, w->cap);
            rc |= alloc(w, &p.pa, (size_t)w->cap * MOST_POINTS);
            rc |= alloc(w, &p.pb, (size_t)w->cap * MOST_POINTS);
            rc |= alloc(w, &p.imp, (size_t)w->cap * MOST_POINTS);
            rc |= alloc(w, &p.impr, (size_t)w->cap * MOST_POINTS);
            if (g == 0) {  // the prepared anchors live for one half-substep: one buffer serves both generations
                rc |= alloc(w, &p.prepA, (size_t)w->cap * MOST_POINTS);
                rc |= alloc(w, &p.prepB, (size_t)w->cap * MOST_POINTS);
            } else {
                p.prepA = w->gen[0].prepA;
                p.prepB = w->gen[0].prepB;
            }
        }
        rc |= alloc(w, &w->colour, w->cap);
        rc |= alloc(w, &w->inc_count, n);
        rc |= alloc(w, &w->inc_start, (size_t)n + 1);
        rc |= alloc(w, &w->inc_fill, n);
        rc |= alloc(w, &w->inc_list, (size_t)w->cap * 2);
        rc |= alloc(w, &w->parent, n);
        rc |= alloc(w, &w->comp, n);
        rc |= alloc(w, &w->isl_size, n);
        rc |= alloc(w, &w->isl_key, n);
        rc |= alloc(w, &w->isl_offset, (size_t)n + 1);
        rc |= alloc(w, &w->isl_fill, n);
        rc |= alloc(w, &w->body_group, n);
        rc |= alloc(w, &w->body_local, n);
        rc |= alloc(w, &w->group_body, (size_t)w->groups_max * GROUP_CAP);
        rc |= alloc(w, &w->group_count, w->groups_max);
        rc |= alloc(w, &w->group_base, w->groups_max);
        rc |= alloc(w, &w->gr_count, (size_t)w->groups_max * GROUP_LISTS);
        rc |= alloc(w, &w->gr_start, (size_t)w->groups_max * GROUP_LISTS + 1);
        rc |= alloc(w, &w->gr_fill, (size_t)w->groups_max * GROUP_LISTS);
        rc |= alloc(w, &w->ilist, w->cap);
        rc |= alloc(w, &w->grid_list, n);
        rc |= alloc(w, &w->free_list, n);
    }
    if (rc) return bad(VXR_ECUDA);
    if (cudaMallocHost(&w->host_totals, sizeof(Totals)) != cudaSuccess) return bad(VXR_ECUDA);
    // Occupancy of the cooperative kernels: every block must be resident at once.
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve, SOLVE_THREADS, 0);
    per_sm = std::max(1, per_sm);
    if (cfg->solve_blocks_per_sm > 0) per_sm = std::min(per_sm, (int)cfg->solve_blocks_per_sm);
    w->solve_blocks = per_sm * w->sms;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_colour, THREADS, 0);
    w->colour_blocks = std::max(1, per_sm) * w->sms;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_islands, ISLAND_THREADS, 0);
    w->island_blocks = std::max(1, per_sm) * w->sms;
    // Everything starts at zero, as the reference's buffers do; every orientation the identity.
    cudaStream_t st = w->stream;
    cudaMemsetAsync(w->b.pose, 0, sizeof(float4) * n, st);
    cudaMemsetAsync(w->b.vel, 0, sizeof(float4) * n, st);
    cudaMemsetAsync(w->b.mom, 0, sizeof(float4) * n, st);
    cudaMemsetAsync(w->b.half, 0, sizeof(float4) * n, st);
    cudaMemsetAsync(w->wall, 0, sizeof(float4) * (size_t)n * WALL_RECORDS, st);
    cudaMemsetAsync(w->wroll, 0, sizeof(float4) * (size_t)n * 6, st);
    cudaMemsetAsync(w->wmask, 0, sizeof(unsigned long long) * n, st);
    cudaMemsetAsync(w->shown, 0, sizeof(float) * (size_t)n * SHOWN_STRIDE, st);
    cudaMemsetAsync(w->counters, 0, sizeof(Counters), st);
    cudaMemsetAsync(w->totals, 0, sizeof(Totals), st);
    cudaMemsetAsync(w->round_start, 0, sizeof(int) * (MOST_ROUNDS + 2), st);
    cudaMemsetAsync(w->body_colours, 0, sizeof(unsigned) * n, st);
    cudaMemsetAsync(w->version, 0, sizeof(int) * n, st);
    cudaMemsetAsync(w->listed, 0, sizeof(int) * n, st);
    if (w->has_grid) {
        for (int g = 0; g < 2; g++) {
            cudaMemsetAsync(w->gen[g].tstart, 0, sizeof(int) * ((size_t)n + 1), st);
        }
    }
    if (upload4(w, w->b.turn, nullptr, nullptr, nullptr, nullptr, 1.0f)) return bad(VXR_ECUDA);
    if (cudaStreamSynchronize(st) != cudaSuccess) return bad(VXR_ECUDA);
    set(VXR_OK);
    return w;
}

void vxr_box_destroy(vxr_box_world* w) {
    if (!w) return;
    if (w->stream) cudaStreamSynchronize(w->stream);
    drop_graph(w);
    for (void* p : w->allocations) cudaFree(p);
    if (w->pinned) cudaFreeHost(w->pinned);
    if (w->host_totals) cudaFreeHost(w->host_totals);
    if (w->ev0) cudaEventDestroy(w->ev0);
    if (w->ev1) cudaEventDestroy(w->ev1);
    for (cudaEvent_t e : w->events) cudaEventDestroy(e);
    if (w->copy_stream) {
        cudaStreamSynchronize(w->copy_stream);
        for (int k = 0; k < 2; k++) {
            cudaEventDestroy(w->slot_split[k]);
            cudaEventDestroy(w->slot_copied[k]);
        }
        cudaStreamDestroy(w->copy_stream);
    }
    if (w->stream) cudaStreamDestroy(w->stream);
    delete w;
}

const char* vxr_box_error(const vxr_box_world* w) { return w ? w->error.c_str() : "no world"; }

int32_t vxr_box_params(vxr_box_world* w, const int32_t* params) {
    if (!w || !params) return VXR_EINVAL;
    if (w->scenes > 0) {  // a batch: the same words for every scene
        std::vector<int32_t> all((size_t)w->scenes * P_COUNT);
        for (int sc = 0; sc < w->scenes; sc++) std::memcpy(&all[(size_t)sc * P_COUNT], params, sizeof(int32_t) * P_COUNT);
        return vxr_box_scene_params(w, all.data());
    }
    drop_graph(w);
    std::memcpy(w->params.w, params, sizeof(float) * P_COUNT);
    return VXR_OK;
}

int32_t vxr_box_scene_params(vxr_box_world* w, const int32_t* params) {
    if (!w || !params) return VXR_EINVAL;
    if (w->scenes == 0) {
        w->error = "not a batch of scenes";
        return VXR_EINVAL;
    }
    // the words every scene shares: the substep, the margin, the softness and the push
    const int shared[] = {P_H, P_MARGIN, P_BIAS, P_MASS_SCALE, P_IMPULSE_SCALE, P_STATIC_BIAS, P_STATIC_MASS_SCALE,
                          P_STATIC_IMPULSE_SCALE, P_PUSH};
    for (int sc = 1; sc < w->scenes; sc++)
        for (int k : shared)
            if (params[(size_t)sc * P_COUNT + k] != params[k]) {
                w->error = "scene " + std::to_string(sc) + " differs from scene 0 in word " + std::to_string(k) +
                           " (the substep, margin, softness and push are one for a batch)";
                return VXR_EINVAL;
            }
    drop_graph(w);
    std::memcpy(w->params.w, params, sizeof(float) * P_COUNT);
    VXR_CUDA(cudaMemcpyAsync(w->scene_params, params, sizeof(Params) * w->scenes, cudaMemcpyHostToDevice, w->stream));
    VXR_CUDA(cudaStreamSynchronize(w->stream));
    w->scene_params_set = 1;
    return VXR_OK;
}

vxr_box_world* vxr_box_create_batch(const vxr_batch_config* cfg, int32_t* status) {
    auto set = [&](int32_t s) {
        if (status) *status = s;
    };
    if (!cfg || cfg->scenes < 1 || !cfg->bodies || !cfg->grids) {
        set(VXR_EINVAL);
        return nullptr;
    }
    long total = 0, cells = 0;
    for (int sc = 0; sc < cfg->scenes; sc++) {
        const vxr_grid g = cfg->grids[sc];
        if (cfg->bodies[sc] < 1 || g.nx < 1 || g.ny < 1 || g.nz < 1 || !(g.cell > 0)) {
            set(VXR_EINVAL);
            return nullptr;
        }
        total += cfg->bodies[sc];
        cells += (long)g.nx * g.ny * g.nz;
    }
    if (total < 2 || total > (1L << 28) || cells > (1L << 30)) {
        set(VXR_EINVAL);
        return nullptr;
    }
    vxr_box_config c = {};
    c.bodies = (int32_t)total;
    c.substeps = cfg->substeps;
    c.sweeps = cfg->sweeps;
    c.symmetric = cfg->symmetric;
    c.grid.nx = (int32_t)cells;  // one key space for every scene's grid, end to end
    c.grid.ny = 1;
    c.grid.nz = 1;
    c.grid.cell = 1.0f;
    c.reach_cells = 1;
    c.max_pairs = cfg->max_pairs;
    c.device = cfg->device;
    c.schedule = cfg->schedule;
    c.solve_blocks_per_sm = cfg->solve_blocks_per_sm;
    vxr_box_world* w = vxr_box_create(&c, status);
    if (!w) return nullptr;
    const int scenes = cfg->scenes;
    w->scenes = scenes;
    int rc = 0;
    rc |= alloc(w, &w->scene_params, scenes);
    rc |= alloc(w, &w->body_scene, w->n);
    rc |= alloc(w, &w->scene_grid, scenes);
    rc |= alloc(w, &w->scene_cell, scenes);
    if (rc) {
        set(VXR_ECUDA);
        vxr_box_destroy(w);
        return nullptr;
    }
    std::vector<int> body_scene(w->n);
    std::vector<int4> grid(scenes);
    std::vector<float> cell(scenes);
    w->scene_first.assign(scenes + 1, 0);
    int first = 0, base = 0;
    for (int sc = 0; sc < scenes; sc++) {
        const vxr_grid g = cfg->grids[sc];
        w->scene_first[sc] = first;
        for (int k = 0; k < cfg->bodies[sc]; k++) body_scene[first + k] = sc;
        first += cfg->bodies[sc];
        grid[sc] = make_int4(g.nx, g.ny, g.nz, base);
        cell[sc] = g.cell;
        base += g.nx * g.ny * g.nz;
    }
    w->scene_first[scenes] = first;
    if (cudaMemcpy(w->body_scene, body_scene.data(), sizeof(int) * w->n, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(w->scene_grid, grid.data(), sizeof(int4) * scenes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(w->scene_cell, cell.data(), sizeof(float) * scenes, cudaMemcpyHostToDevice) != cudaSuccess) {
        set(VXR_ECUDA);
        vxr_box_destroy(w);
        return nullptr;
    }
    set(VXR_OK);
    return w;
}

int32_t vxr_box_scenes(const vxr_box_world* w, int32_t* first_body) {
    if (!w) return -VXR_EINVAL;
    if (first_body)
        for (int sc = 0; sc <= w->scenes && w->scenes > 0; sc++) first_body[sc] = w->scene_first[sc];
    return w->scenes;
}

int32_t vxr_box_learned(vxr_box_world* w, vxr_mlp* net, int32_t mode) {
    if (!w || mode < 0 || mode > 3 || (mode >= 2 && !net)) return VXR_EINVAL;
    if (!w->has_grid) {
        w->error = "the learned warm start works on a world with a grid";
        return VXR_EINVAL;
    }
    if (mode > 0 && !w->lfeat) {
        const size_t rows = (size_t)w->cap * MOST_POINTS;
        if (alloc(w, &w->lfeat, rows * FEATURES) || alloc(w, &w->lpred, rows * 2) || alloc(w, &w->ltarget, rows * 2))
            return VXR_ECUDA;
    }
    drop_graph(w);
    w->learn_mode = mode;
    w->learn_net = net;
    return VXR_OK;
}

int32_t vxr_box_first_substeps(vxr_box_world* w, int32_t count, int32_t solve_only) {
    if (!w || count < 0 || count > w->substeps || (solve_only != 0 && solve_only != 1)) return VXR_EINVAL;
    drop_graph(w);
    w->first_substeps = count == w->substeps ? 0 : count;
    w->solve_only = count > 0 ? solve_only : 0;
    return VXR_OK;
}

int32_t vxr_box_learned_given(vxr_box_world* w, const vxr_box_world* answers, int32_t fresh_only, int32_t whole) {
    if (!w || !answers || answers == w || (fresh_only != 0 && fresh_only != 1) || (whole != 0 && whole != 1))
        return VXR_EINVAL;
    if (!w->has_grid || !answers->ltarget || answers->cap != w->cap || answers->device != w->device ||
        answers->n != w->n) {
        w->error = "given starts need a world of the same bodies and pair capacity on the same device that gathered "
                   "targets";
        return VXR_EINVAL;
    }
    cudaSetDevice(w->device);
    const size_t rows = (size_t)w->cap * MOST_POINTS;
    if (!w->lfeat) {
        if (alloc(w, &w->lfeat, rows * FEATURES) || alloc(w, &w->lpred, rows * 2) || alloc(w, &w->ltarget, rows * 2))
            return VXR_ECUDA;
    }
    if (!w->lgiven && alloc(w, &w->lgiven, rows * 2)) return VXR_ECUDA;
    VXR_CUDA(cudaStreamSynchronize(answers->stream));
    if (whole) {  // the answers' whole records: pairs by touching index; the walls' records as they are (all only)
        if (!w->lgiven_imp && (alloc(w, &w->lgiven_imp, rows) || alloc(w, &w->lgiven_impr, rows))) return VXR_ECUDA;
        const PairGen& done = answers->gen[answers->cur ^ 1];
        VXR_CUDA(cudaMemsetAsync(w->lgiven_imp, 0, sizeof(float4) * rows, w->stream));
        VXR_CUDA(cudaMemsetAsync(w->lgiven_impr, 0, sizeof(float4) * rows, w->stream));
        k_records_by_pair<<<w->sms * 4, THREADS, 0, w->stream>>>(done.tstart + answers->n, done, w->lgiven_imp,
                                                                 w->lgiven_impr);
        VXR_CUDA(cudaGetLastError());
        if (!fresh_only) {
            const size_t n = w->n;
            VXR_CUDA(cudaMemcpyAsync(w->wall, answers->wall, sizeof(float4) * n * WALL_RECORDS,
                                     cudaMemcpyDeviceToDevice, w->stream));
            VXR_CUDA(cudaMemcpyAsync(w->wroll, answers->wroll, sizeof(float4) * n * 6, cudaMemcpyDeviceToDevice,
                                     w->stream));
            VXR_CUDA(cudaMemcpyAsync(w->wmask, answers->wmask, sizeof(unsigned long long) * n,
                                     cudaMemcpyDeviceToDevice, w->stream));
        }
        VXR_CUDA(cudaStreamSynchronize(w->stream));
        drop_graph(w);
        w->learn_mode = fresh_only ? 7 : 6;
        w->learn_net = nullptr;
        return VXR_OK;
    }
    // the answers' last step, by touching index: rows of pairs the answers did not touch stay zero
    const PairGen& last = answers->gen[answers->cur ^ 1];
    VXR_CUDA(cudaMemsetAsync(w->lgiven, 0, sizeof(float) * rows * 2, w->stream));
    k_rows_by_pair<<<w->sms * 4, THREADS, 0, w->stream>>>(last.tstart + answers->n, last.pos, answers->ltarget,
                                                         w->lgiven);
    VXR_CUDA(cudaGetLastError());
    VXR_CUDA(cudaStreamSynchronize(w->stream));
    drop_graph(w);
    w->learn_mode = fresh_only ? 5 : 4;
    w->learn_net = nullptr;
    return VXR_OK;
}

int32_t vxr_box_features(vxr_box_world* w, float* features16, float* targets2, int32_t capacity, int32_t* rows) {
    if (!w || !rows) return VXR_EINVAL;
    if (!w->lfeat) {
        w->error = "no features gathered: vxr_box_learned(world, net, 1) first";
        return VXR_EINVAL;
    }
    VXR_CUDA(cudaStreamSynchronize(w->stream));
    Counters c;
    VXR_CUDA(cudaMemcpy(&c, w->counters, sizeof(Counters), cudaMemcpyDeviceToHost));
    const int touching = std::min(c.touching, w->cap);
    const PairGen& last = w->gen[w->cur ^ 1];  // the step just taken (the generations swapped after it)
    std::vector<int4> pair(touching);
    std::vector<float> f((size_t)touching * MOST_POINTS * FEATURES), t((size_t)touching * MOST_POINTS * 2);
    if (touching) {
        VXR_CUDA(cudaMemcpy(pair.data(), last.pair, sizeof(int4) * touching, cudaMemcpyDeviceToHost));
        VXR_CUDA(cudaMemcpy(f.data(), w->lfeat, sizeof(float) * f.size(), cudaMemcpyDeviceToHost));
        VXR_CUDA(cudaMemcpy(t.data(), w->ltarget, sizeof(float) * t.size(), cudaMemcpyDeviceToHost));
    }
    int k = 0;
    for (int p = 0; p < touching; p++)
        for (int slot = 0; slot < pair[p].z && slot < MOST_POINTS; slot++) {
            const size_t row = (size_t)p * MOST_POINTS + slot;
            if (k < capacity) {
                if (features16) std::memcpy(features16 + (size_t)k * FEATURES, &f[row * FEATURES], sizeof(float) * FEATURES);
                if (targets2) std::memcpy(targets2 + (size_t)k * 2, &t[row * 2], sizeof(float) * 2);
            }
            k++;
        }
    *rows = k;
    return VXR_OK;
}

int32_t vxr_box_contact_errors(vxr_box_world* w, float* out, int32_t capacity) {
    if (!w || capacity < 0) return -VXR_EINVAL;
    if (!w->has_grid) return 0;
    cudaSetDevice(w->device);
    const PairGen& last = w->gen[w->cur ^ 1];
    int touching = 0;
    if (cudaMemcpy(&touching, last.tstart + w->n, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return -fail(w, "reading the touching count");
    const int rows = touching * MOST_POINTS;
    if (!out) return rows;
    if (capacity < rows) return -VXR_EINVAL;
    if (rows == 0) return 0;
    if (w->err_rows < rows) {
        if (alloc(w, &w->errors, (size_t)rows)) return -VXR_ECUDA;
        w->err_rows = rows;
    }
    k_contact_errors<<<w->sms * 4, THREADS, 0, w->stream>>>(last.tstart + w->n, last, w->b, w->params, w->errors);
    if (cudaGetLastError() != cudaSuccess) return -fail(w, "contact errors kernel");
    if (cudaMemcpyAsync(out, w->errors, sizeof(float) * rows, cudaMemcpyDeviceToHost, w->stream) != cudaSuccess ||
        cudaStreamSynchronize(w->stream) != cudaSuccess)
        return -fail(w, "reading the contact errors");
    return rows;
}

int32_t vxr_box_diagnostics(vxr_box_world* w, vxr_box_diag* out) {
    if (!w || !out) return VXR_EINVAL;
    cudaSetDevice(w->device);
    Diag* d = nullptr;
    VXR_CUDA(cudaMallocAsync(&d, sizeof(Diag), w->stream));
    VXR_CUDA(cudaMemsetAsync(d, 0, sizeof(Diag), w->stream));
    k_diag_bodies<<<w->sms * 4, THREADS, 0, w->stream>>>(w->n, w->b, w->params, w->scene_params, w->body_scene, d);
    if (w->has_grid) {
        const PairGen& last = w->gen[w->cur ^ 1];
        k_diag_contacts<<<w->sms * 4, THREADS, 0, w->stream>>>(last.tstart + w->n, last, w->b, d);
    }
    VXR_CUDA(cudaGetLastError());
    Diag h;
    VXR_CUDA(cudaMemcpyAsync(&h, d, sizeof(Diag), cudaMemcpyDeviceToHost, w->stream));
    VXR_CUDA(cudaFreeAsync(d, w->stream));
    VXR_CUDA(cudaStreamSynchronize(w->stream));
    out->kinetic = h.kinetic;
    out->rotational = h.rotational;
    out->potential = h.potential;
    for (int k = 0; k < 3; k++) {
        out->momentum[k] = h.momentum[k];
        out->angular[k] = h.angular[k];
    }
    float f;
    std::memcpy(&f, &h.max_penetration, 4);
    out->max_penetration = f;
    std::memcpy(&f, &h.max_wall, 4);
    out->max_wall_penetration = f;
    std::memcpy(&f, &h.max_speed, 4);
    out->max_speed = f;
    out->broken = h.broken;
    out->pad = 0;
    return VXR_OK;
}

const float* vxr_box_shown_device(vxr_box_world* w, int64_t* words) {
    if (!w) return nullptr;
    if (words) *words = (int64_t)w->n * SHOWN_STRIDE;
    return w->shown;
}

int32_t vxr_box_step_graph(vxr_box_world* w, int32_t pairs) {
    if (!w || pairs < 0) return VXR_EINVAL;
    if (w->profile || w->tracing) {
        w->error = "a captured step records no profile or trace: switch them off first";
        return VXR_EINVAL;
    }
    cudaSetDevice(w->device);
    if (!w->graph_exec) {
        const long long before = w->launches;
        VXR_CUDA(cudaStreamBeginCapture(w->stream, cudaStreamCaptureModeThreadLocal));
        w->capturing = 1;
        int rc = enqueue_step(w);
        if (rc == VXR_OK) rc = enqueue_step(w);  // two steps: the pair generations come back to where they were
        w->capturing = 0;
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(w->stream, &g);
        w->launches = before;
        if (rc != VXR_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            if (rc == VXR_OK) w->error = std::string("stream capture: ") + cudaGetErrorString(e);
            return rc != VXR_OK ? rc : VXR_ECUDA;
        }
        w->graph = g;
        VXR_CUDA(cudaGraphInstantiate(&w->graph_exec, g, 0));
        size_t nodes = 0;
        cudaGraphGetNodes(g, nullptr, &nodes);
        w->graph_launches = 0;
        std::vector<cudaGraphNode_t> all(nodes);
        if (nodes) cudaGraphGetNodes(g, all.data(), &nodes);
        for (cudaGraphNode_t node : all) {
            cudaGraphNodeType t;
            if (cudaGraphNodeGetType(node, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) w->graph_launches++;
        }
    }
    for (int k = 0; k < pairs; k++) {
        VXR_CUDA(cudaGraphLaunch(w->graph_exec, w->stream));
        w->launches += w->graph_launches;
    }
    return VXR_OK;
}

// Whether every value of the given host arrays is finite (the state a step may start from).
bool all_finite(const float* const* fields, int count, int n) {
    for (int k = 0; k < count; k++)
        for (int s = 0; s < n; s++)
            if (!std::isfinite(fields[k][s])) return false;
    return true;
}

int32_t vxr_box_load_state(vxr_box_world* w, const float* const* f, const int32_t* params) {
    if (!w || !f) return VXR_EINVAL;
    for (int k = 0; k < 18; k++)
        if (!f[k]) return VXR_EINVAL;
    if (!all_finite(f, 18, w->n)) {
        w->error = "a non-finite value in the state: nothing was loaded";
        return VXR_ENONFINITE;
    }
    cudaSetDevice(w->device);
    int rc = clear_dynamic(w);
    if (rc) return rc;
    rc |= upload4(w, w->b.pose, f[0], f[1], f[2], f[13], 0.0f);
    rc |= upload4(w, w->b.vel, f[3], f[4], f[5], nullptr, 0.0f);
    rc |= upload4(w, w->b.mom, f[6], f[7], f[8], nullptr, 0.0f);
    rc |= upload4(w, w->b.turn, f[9], f[10], f[11], f[12], 1.0f);
    rc |= upload4(w, w->b.half, f[14], f[15], f[16], f[17], 0.0f);
    if (rc) return VXR_ECUDA;
    k_inverse_inertia<<<blocks_for(w->n, THREADS), THREADS, 0, w->stream>>>(w->n, w->b.pose, w->b.half, w->b.inv);
    VXR_CUDA(cudaGetLastError());
    if (params) vxr_box_params(w, params);
    return VXR_OK;
}

int32_t vxr_box_start(vxr_box_world* w, const float* x, const float* y, const float* z, const float* u,
                      const float* v, const float* wv, const float* const* spin, const float* const* q,
                      const float* const* half, const float* shape, const float* im, const int32_t* params) {
    if (!w || !x || !y || !z || !u || !v || !wv || !spin || !q || !half || !shape || !im || !params)
        return VXR_EINVAL;
    const int n = w->n;
    std::vector<float> l[3];
    for (int a = 0; a < 3; a++) l[a].assign(n, 0.0f);
    for (int s = 0; s < n; s++) {
        if (im[s] <= 0) continue;
        const double m = 1.0 / im[s];
        double moment[3];
        if (shape[s] > 0.5f) {
            const double mo = 0.4 * m * half[0][s] * half[0][s];
            moment[0] = moment[1] = moment[2] = mo;
        } else {
            const double hx = half[0][s], hy = half[1][s], hz = half[2][s];
            moment[0] = m * (hy * hy + hz * hz) / 3;
            moment[1] = m * (hx * hx + hz * hz) / 3;
            moment[2] = m * (hx * hx + hy * hy) / 3;
        }
        const double qq[4] = {q[0][s], q[1][s], q[2][s], q[3][s]};
        const double cq[4] = {-qq[0], -qq[1], -qq[2], qq[3]};
        const double om[3] = {spin[0][s], spin[1][s], spin[2][s]};
        double own[3], lb[3];
        rotate_d(cq, om, own);
        for (int a = 0; a < 3; a++) own[a] *= moment[a];
        rotate_d(qq, own, lb);
        for (int a = 0; a < 3; a++) l[a][s] = (float)lb[a];
    }
    const float* f[18] = {x, y, z, u, v, wv, l[0].data(), l[1].data(), l[2].data(), q[0], q[1], q[2], q[3],
                          im, half[0], half[1], half[2], shape};
    int rc = vxr_box_load_state(w, f, params);
    if (rc) return rc;
    // shown from the starting state (Boxes.shownAtStart :827-842)
    std::vector<float> shown((size_t)n * SHOWN_STRIDE, 0.0f);
    for (int s = 0; s < n; s++) {
        float* sh = &shown[(size_t)s * SHOWN_STRIDE];
        const float at[3] = {x[s], y[s], z[s]};
        for (int a = 0; a < 3; a++) {
            sh[0 + a] = sh[4 + a] = at[a];
            sh[8 + a] = half[a][s];
        }
        sh[3] = shape[s];
        for (int k = 0; k < 4; k++) sh[12 + k] = sh[16 + k] = q[k][s];
    }
    VXR_CUDA(cudaMemcpy(w->shown, shown.data(), sizeof(float) * shown.size(), cudaMemcpyHostToDevice));
    return VXR_OK;
}

int32_t vxr_box_step_async(vxr_box_world* w, int32_t steps) {
    if (!w || steps < 0) return VXR_EINVAL;
    cudaSetDevice(w->device);
    for (int k = 0; k < steps; k++) {
        int rc = enqueue_step(w);
        if (rc) return rc;
    }
    return VXR_OK;
}

int32_t vxr_box_sync(vxr_box_world* w, vxr_box_report* report) {
    if (!w) return VXR_EINVAL;
    VXR_CUDA(cudaMemcpyAsync(w->host_totals, w->totals, sizeof(Totals), cudaMemcpyDeviceToHost, w->stream));
    VXR_CUDA(cudaMemsetAsync(w->totals, 0, sizeof(Totals), w->stream));
    VXR_CUDA(cudaStreamSynchronize(w->stream));
    for (int e = 0; e + 4 < w->events_used; e += 5) {
        for (int k = 0; k < 4; k++) {
            float ms = 0.0f;
            VXR_CUDA(cudaEventElapsedTime(&ms, w->events[e + k], w->events[e + k + 1]));
            w->phase_ms[k] += ms;
        }
    }
    w->events_used = 0;
    const Totals& t = *w->host_totals;
    if (report) {
        report->touching = t.last[0];
        report->points = t.last[1];
        report->rounds = t.last[2];
        report->unplaced = t.last[3];
        report->unlisted = t.last[4];
        report->most_rounds = t.most_rounds;
        report->unplaced_total = t.unplaced;
        report->unlisted_total = t.unlisted;
        report->status = t.status;
        report->steps = t.steps;
    }
    switch (t.status) {
        case ST_OK: return VXR_OK;
        case ST_CAPACITY: w->error = "pair capacity exceeded"; return VXR_ECAPACITY;
        case ST_ROUNDS: w->error = "colouring did not finish"; return VXR_EROUNDS;
        case ST_TIMEOUT: w->error = "a grid barrier timed out"; return VXR_ETIMEOUT;
        default: w->error = "step failed"; return VXR_ECUDA;
    }
}

int32_t vxr_box_step(vxr_box_world* w, int32_t steps, vxr_box_report* report) {
    int rc = vxr_box_step_async(w, steps);
    if (rc) return rc;
    return vxr_box_sync(w, report);
}

void* vxr_box_stream(vxr_box_world* w) { return w ? (void*)w->stream : nullptr; }

int32_t vxr_box_state(vxr_box_world* w, float* const* out) {
    if (!w || !out) return VXR_EINVAL;
    cudaSetDevice(w->device);
    // the 13 fields split out of the float4 arrays on the device, then copied straight into the caller's arrays
    // (at the copy engine's full rate when they are pinned), one synchronisation for all
    if (!w->state13 && alloc(w, &w->state13, (size_t)13 * w->n)) return VXR_ECUDA;
    const int n = w->n;
    k_state13<<<blocks_for(n, THREADS), THREADS, 0, w->stream>>>(n, w->b, w->state13);  // not a step's launch
    for (int f = 0; f < 13; f++)
        if (out[f])
            VXR_CUDA(cudaMemcpyAsync(out[f], w->state13 + (size_t)f * n, sizeof(float) * (size_t)n,
                                     cudaMemcpyDeviceToHost, w->stream));
    VXR_CUDA(cudaStreamSynchronize(w->stream));
    return VXR_OK;
}

int32_t vxr_box_state_async(vxr_box_world* w, float* const* out, int32_t slot) {
    if (!w || !out || slot < 0 || slot > 1) return VXR_EINVAL;
    cudaSetDevice(w->device);
    const int n = w->n;
    if (!w->copy_stream) {
        if (alloc(w, &w->state_slot[0], (size_t)13 * n) || alloc(w, &w->state_slot[1], (size_t)13 * n))
            return VXR_ECUDA;
        VXR_CUDA(cudaStreamCreateWithFlags(&w->copy_stream, cudaStreamNonBlocking));
        for (int k = 0; k < 2; k++) {
            VXR_CUDA(cudaEventCreateWithFlags(&w->slot_split[k], cudaEventDisableTiming));
            VXR_CUDA(cudaEventCreateWithFlags(&w->slot_copied[k], cudaEventDisableTiming));
        }
    }
    // the slot's copy before is done before its fields are written again; the fields split after the steps enqueued
    // so far, then copied out on the copy stream while the world's stream goes on
    VXR_CUDA(cudaStreamWaitEvent(w->stream, w->slot_copied[slot], 0));
    k_state13<<<blocks_for(n, THREADS), THREADS, 0, w->stream>>>(n, w->b, w->state_slot[slot]);  // not a step's launch
    VXR_CUDA(cudaGetLastError());
    VXR_CUDA(cudaEventRecord(w->slot_split[slot], w->stream));
    VXR_CUDA(cudaStreamWaitEvent(w->copy_stream, w->slot_split[slot], 0));
    for (int f = 0; f < 13; f++)
        if (out[f])
            VXR_CUDA(cudaMemcpyAsync(out[f], w->state_slot[slot] + (size_t)f * n, sizeof(float) * (size_t)n,
                                     cudaMemcpyDeviceToHost, w->copy_stream));
    VXR_CUDA(cudaEventRecord(w->slot_copied[slot], w->copy_stream));
    return VXR_OK;
}

int32_t vxr_box_state_wait(vxr_box_world* w, int32_t slot) {
    if (!w || slot < 0 || slot > 1) return VXR_EINVAL;
    if (!w->copy_stream) return VXR_OK;
    cudaSetDevice(w->device);
    VXR_CUDA(cudaEventSynchronize(w->slot_copied[slot]));
    return VXR_OK;
}

int32_t vxr_box_read_shown(vxr_box_world* w, float* out) {
    if (!w || !out) return VXR_EINVAL;
    VXR_CUDA(cudaMemcpyAsync(out, w->shown, sizeof(float) * (size_t)w->n * SHOWN_STRIDE, cudaMemcpyDeviceToHost,
                             w->stream));
    VXR_CUDA(cudaStreamSynchronize(w->stream));
    return VXR_OK;
}

int32_t vxr_box_touching(vxr_box_world* w, int32_t* first, int32_t* second, int32_t* points, float* manifold,
                         float* impulses, int32_t capacity) {
    if (!w) return -VXR_EINVAL;
    if (!w->has_grid) return 0;
    VXR_CUDA(cudaStreamSynchronize(w->stream));
    const PairGen& g = w->gen[w->cur ^ 1];  // the last step's
    int P = 0;
    VXR_CUDA(cudaMemcpy(&P, g.tstart + w->n, sizeof(int), cudaMemcpyDeviceToHost));
    if (!first && !second && !points && !manifold && !impulses) return P;
    if (P > capacity) return -VXR_ECAPACITY;
    if (P == 0) return 0;
    std::vector<int> pos(P), pstart(P);
    std::vector<int4> pair(P);
    std::vector<float4> normal(P), pa((size_t)P * MOST_POINTS), pb((size_t)P * MOST_POINTS),
        imp((size_t)P * MOST_POINTS), impr((size_t)P * MOST_POINTS);
    VXR_CUDA(cudaMemcpy(pos.data(), g.pos, sizeof(int) * P, cudaMemcpyDeviceToHost));
    VXR_CUDA(cudaMemcpy(pair.data(), g.pair, sizeof(int4) * P, cudaMemcpyDeviceToHost));
    VXR_CUDA(cudaMemcpy(pstart.data(), g.pstart, sizeof(int) * P, cudaMemcpyDeviceToHost));
    VXR_CUDA(cudaMemcpy(normal.data(), g.normal, sizeof(float4) * P, cudaMemcpyDeviceToHost));
    VXR_CUDA(cudaMemcpy(pa.data(), g.pa, sizeof(float4) * pa.size(), cudaMemcpyDeviceToHost));
    VXR_CUDA(cudaMemcpy(pb.data(), g.pb, sizeof(float4) * pb.size(), cudaMemcpyDeviceToHost));
    VXR_CUDA(cudaMemcpy(imp.data(), g.imp, sizeof(float4) * imp.size(), cudaMemcpyDeviceToHost));
    VXR_CUDA(cudaMemcpy(impr.data(), g.impr, sizeof(float4) * impr.size(), cudaMemcpyDeviceToHost));
    for (int t = 0; t < P; t++) {
        const int p = pos[t];
        const int cnt = pair[p].z;
        if (first) first[t] = pair[p].x;
        if (second) second[t] = pair[p].y;
        if (points) points[t] = cnt;
        if (manifold) {
            float* m = manifold + (size_t)t * MANIFOLD_WORDS;
            std::memset(m, 0, sizeof(float) * MANIFOLD_WORDS);
            m[0] = normal[p].x;
            m[1] = normal[p].y;
            m[2] = normal[p].z;
            m[3] = (float)cnt;
            m[4] = normal[p].w;
            for (int i = 0; i < cnt && i < MOST_POINTS; i++) {
                float* q = m + M_POINTS + i * M_POINT_WORDS;
                const float4 a = pa[(size_t)pstart[p] + i], b = pb[(size_t)pstart[p] + i];
                q[0] = a.x;
                q[1] = a.y;
                q[2] = a.z;
                q[3] = b.x;
                q[4] = b.y;
                q[5] = b.z;
                q[6] = a.w;
            }
        }
        if (impulses) {
            float* r = impulses + (size_t)t * 28;
            std::memset(r, 0, sizeof(float) * 28);
            for (int i = 0; i < cnt && i < MOST_POINTS; i++) {
                const float4 a = imp[(size_t)pstart[p] + i], b = impr[(size_t)pstart[p] + i];
                r[7 * i + 0] = a.x;
                r[7 * i + 1] = a.y;
                r[7 * i + 2] = a.z;
                r[7 * i + 3] = a.w;
                r[7 * i + 4] = b.x;
                r[7 * i + 5] = b.y;
                r[7 * i + 6] = b.z;
            }
        }
    }
    return P;
}

int32_t vxr_box_trace(vxr_box_world* w, int32_t enable, int64_t* out, int32_t capacity) {
    if (!w) return -VXR_EINVAL;
    if (enable) drop_graph(w);
    int len = 0;
    if (out && w->trace) {
        Counters c;
        VXR_CUDA(cudaStreamSynchronize(w->stream));
        VXR_CUDA(cudaMemcpy(&c, w->counters, sizeof(Counters), cudaMemcpyDeviceToHost));
        len = std::min(c.trace_len, std::min(capacity, w->trace_cap));
        if (len > 0) VXR_CUDA(cudaMemcpy(out, w->trace, sizeof(int64_t) * len, cudaMemcpyDeviceToHost));
    }
    if (enable && !w->trace) {
        w->trace_cap = 1 << 16;
        if (alloc(w, &w->trace, w->trace_cap)) return -VXR_ECUDA;
    }
    w->tracing = enable ? 1 : 0;
    return len;
}

int32_t vxr_box_candidates(vxr_box_world* w, int32_t* pairs, int32_t capacity) {
    if (!w) return -VXR_EINVAL;
    if (!w->has_grid) return 0;
    VXR_CUDA(cudaStreamSynchronize(w->stream));
    int C = 0;
    VXR_CUDA(cudaMemcpy(&C, w->cand_start + w->n, sizeof(int), cudaMemcpyDeviceToHost));
    C = std::min(C, w->cap);
    if (!pairs) return C;
    if (C > capacity) return -VXR_ECAPACITY;
    std::vector<int> a(C), b(C);
    VXR_CUDA(cudaMemcpy(a.data(), w->cand_a, sizeof(int) * C, cudaMemcpyDeviceToHost));
    VXR_CUDA(cudaMemcpy(b.data(), w->cand_b, sizeof(int) * C, cudaMemcpyDeviceToHost));
    for (int c = 0; c < C; c++) {
        pairs[2 * c] = a[c];
        pairs[2 * c + 1] = b[c];
    }
    return C;
}

int32_t vxr_box_walls(vxr_box_world* w, float* lambda, float* rub, float* rollw) {
    if (!w) return VXR_EINVAL;
    const int n = w->n;
    std::vector<float4> rec((size_t)n * WALL_RECORDS), rr((size_t)n * 6);
    VXR_CUDA(cudaStreamSynchronize(w->stream));
    VXR_CUDA(cudaMemcpy(rec.data(), w->wall, sizeof(float4) * rec.size(), cudaMemcpyDeviceToHost));
    VXR_CUDA(cudaMemcpy(rr.data(), w->wroll, sizeof(float4) * rr.size(), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < rec.size(); i++) {
        if (lambda) lambda[i] = rec[i].x;
        if (rub) {
            rub[3 * i] = rec[i].y;
            rub[3 * i + 1] = rec[i].z;
            rub[3 * i + 2] = rec[i].w;
        }
    }
    if (rollw) {
        std::memset(rollw, 0, sizeof(float) * (size_t)n * 144);
        for (int s = 0; s < n; s++)
            for (int wl = 0; wl < 6; wl++) {
                const size_t at = ((size_t)s * WALL_RECORDS + wl * 8) * 3;
                rollw[at] = rr[(size_t)s * 6 + wl].x;
                rollw[at + 1] = rr[(size_t)s * 6 + wl].y;
                rollw[at + 2] = rr[(size_t)s * 6 + wl].z;
            }
    }
    return VXR_OK;
}

int32_t vxr_box_colour_waves(vxr_box_world* w) {
    if (!w) return -VXR_EINVAL;
    Counters c;
    if (cudaMemcpy(&c, w->counters, sizeof(Counters), cudaMemcpyDeviceToHost) != cudaSuccess) return -VXR_ECUDA;
    return c.colour_waves;
}

long long vxr_box_launches(vxr_box_world* w) { return w ? w->launches : -1; }

int32_t vxr_box_measure(vxr_box_world* w, int32_t residual, int32_t cold_start, int32_t sweeps, float tolerance) {
    if (!w || sweeps < 0 || sweeps > w->sweeps || !(tolerance >= 0.0f)) return VXR_EINVAL;
    drop_graph(w);
    w->measure = residual ? 1 : 0;
    w->cold = cold_start ? 1 : 0;
    w->active_sweeps = sweeps > 0 ? sweeps : w->sweeps;
    w->tolerance = tolerance;
    return VXR_OK;
}

int32_t vxr_box_wait_limit(vxr_box_world* w, int64_t ns) {
    if (!w) return VXR_EINVAL;
    drop_graph(w);
    w->wait_limit_ns = ns > 0 ? (unsigned long long)ns : 2000000000ull;
    return VXR_OK;
}

int32_t vxr_box_list_kernel(vxr_box_world* w, int32_t tiled) {
    if (!w || tiled < 0 || tiled > 1) return VXR_EINVAL;
    drop_graph(w);
    w->list_tiled = tiled;
    return VXR_OK;
}

int32_t vxr_box_islands(vxr_box_world* w, int32_t enable) {
    if (!w) return VXR_EINVAL;
    drop_graph(w);
    w->islands = enable ? 1 : 0;
    return VXR_OK;
}

int32_t vxr_box_residuals(vxr_box_world* w, float* out, int32_t capacity, int32_t* used) {
    if (!w) return -VXR_EINVAL;
    const int count = w->substeps * (2 * w->active_sweeps + 1);
    if (!out && !used) return count;
    if (out && capacity < count) return -VXR_ECAPACITY;
    VXR_CUDA(cudaStreamSynchronize(w->stream));
    if (out) {
        std::vector<float> walls(count);
        VXR_CUDA(cudaMemcpy(out, w->residual, sizeof(float) * count, cudaMemcpyDeviceToHost));
        VXR_CUDA(cudaMemcpy(walls.data(), w->residual + residual_half(w), sizeof(float) * count,
                            cudaMemcpyDeviceToHost));
        for (int k = 0; k < count; k++) out[k] = std::max(out[k], walls[k]);
    }
    if (used) VXR_CUDA(cudaMemcpy(used, w->used, sizeof(int) * 2 * w->substeps, cudaMemcpyDeviceToHost));
    return count;
}

int32_t vxr_box_residual_parts(vxr_box_world* w, float* pairs, float* walls, int32_t capacity) {
    if (!w) return -VXR_EINVAL;
    const int count = w->substeps * (2 * w->active_sweeps + 1);
    if (!pairs && !walls) return count;
    if (capacity < count) return -VXR_ECAPACITY;
    VXR_CUDA(cudaStreamSynchronize(w->stream));
    if (pairs) VXR_CUDA(cudaMemcpy(pairs, w->residual, sizeof(float) * count, cudaMemcpyDeviceToHost));
    if (walls)
        VXR_CUDA(cudaMemcpy(walls, w->residual + residual_half(w), sizeof(float) * count, cudaMemcpyDeviceToHost));
    return count;
}

int32_t vxr_box_profile(vxr_box_world* w, int32_t enable, double* phase_ms4) {
    if (!w) return VXR_EINVAL;
    if (enable) drop_graph(w);
    if (phase_ms4)
        for (int k = 0; k < 4; k++) phase_ms4[k] = w->phase_ms[k];
    for (int k = 0; k < 4; k++) w->phase_ms[k] = 0.0;
    w->profile = enable ? 1 : 0;
    return VXR_OK;
}

int32_t vxr_box_activity(vxr_box_world* w, int64_t* out4) {
    if (!w || !out4) return VXR_EINVAL;
    if (!w->activity) {
        if (alloc(w, &w->activity, 2)) return VXR_ECUDA;
    }
    VXR_CUDA(cudaMemsetAsync(w->activity, 0, 2 * sizeof(long long), w->stream));
    k_activity<<<blocks_for(w->n, THREADS), THREADS, 0, w->stream>>>(w->n, w->has_grid ? w->inc_count : nullptr,
                                                                      w->wmask, w->activity);
    long long host[2];
    VXR_CUDA(cudaMemcpyAsync(host, w->activity, sizeof(host), cudaMemcpyDeviceToHost, w->stream));
    Counters c;
    VXR_CUDA(cudaMemcpyAsync(&c, w->counters, sizeof(Counters), cudaMemcpyDeviceToHost, w->stream));
    VXR_CUDA(cudaStreamSynchronize(w->stream));
    out4[0] = c.touching;
    out4[1] = c.points;
    out4[2] = host[0];
    out4[3] = host[1];
    return VXR_OK;
}

int32_t vxr_box_paths(vxr_box_world* w, int32_t* out5) {
    if (!w || !out5) return VXR_EINVAL;
    int32_t* out4 = out5;
    Counters c;
    int island = 0;
    VXR_CUDA(cudaMemcpyAsync(&c, w->counters, sizeof(Counters), cudaMemcpyDeviceToHost, w->stream));
    if (w->has_grid)
        VXR_CUDA(cudaMemcpyAsync(&island, w->isl_offset + w->n, sizeof(int), cudaMemcpyDeviceToHost, w->stream));
    VXR_CUDA(cudaStreamSynchronize(w->stream));
    const bool isl = islands_on(w) && !c.all_grid;
    out4[0] = isl ? c.grid_n : w->n;
    out4[1] = isl ? island : 0;
    out4[2] = isl ? c.free_n : 0;
    out4[3] = isl ? (island + group_base_of(island, w->island_blocks) - 1) / group_base_of(island, w->island_blocks) : 0;
    out5[4] = islands_on(w) ? c.largest : 0;
    return VXR_OK;
}

// The narrow phase alone over a caller's pairs (BoxContact.collide :136-246): host buffers in and out.
int32_t vxr_collide(int32_t bodies, const float* const* f, const int32_t* params, int32_t npairs,
                    const int32_t* pairs, float* manifold) {
    if (bodies < 1 || !f || !params || npairs < 0 || !pairs || !manifold) return VXR_EINVAL;
    for (int k = 0; k < 18; k++)
        if (!f[k]) return VXR_EINVAL;
    for (int p = 0; p < 2 * npairs; p++)
        if (pairs[p] >= bodies || pairs[p] < -1) return VXR_EINVAL;
    vxr_box_config cfg{};
    cfg.bodies = bodies;
    cfg.substeps = 1;
    cfg.sweeps = 1;
    int32_t st = 0;
    vxr_box_world* w = vxr_box_create(&cfg, &st);
    if (!w) return st;
    int rc = vxr_box_load_state(w, f, params);
    std::vector<int> a(std::max(npairs, 1)), b(std::max(npairs, 1));
    for (int p = 0; p < npairs; p++) {
        a[p] = pairs[2 * p];
        b[p] = pairs[2 * p + 1];
    }
    int *da = nullptr, *db = nullptr, *dn = nullptr;
    float4 *head = nullptr, *pa = nullptr, *pb = nullptr;
    float* axis = nullptr;
    rc = rc ? rc : alloc(w, &da, npairs);
    rc = rc ? rc : alloc(w, &db, npairs);
    rc = rc ? rc : alloc(w, &dn, 1);
    rc = rc ? rc : alloc(w, &head, npairs);
    rc = rc ? rc : alloc(w, &axis, npairs);
    rc = rc ? rc : alloc(w, &pa, (size_t)npairs * MOST_POINTS);
    rc = rc ? rc : alloc(w, &pb, (size_t)npairs * MOST_POINTS);
    if (!rc && npairs > 0) {
        // a pair whose second is -1 is empty: count 0 (BoxContact.java:147-150)
        std::vector<int> na(a), nb(b);
        int live = 0;
        std::vector<int> where(npairs, -1);
        for (int p = 0; p < npairs; p++)
            if (b[p] >= 0 && a[p] >= 0) {
                na[live] = a[p];
                nb[live] = b[p];
                where[p] = live++;
            }
        cudaMemcpy(da, na.data(), sizeof(int) * npairs, cudaMemcpyHostToDevice);
        cudaMemcpy(db, nb.data(), sizeof(int) * npairs, cudaMemcpyHostToDevice);
        cudaMemcpy(dn, &live, sizeof(int), cudaMemcpyHostToDevice);
        k_collide<<<w->sms * 8, 128, 0, w->stream>>>(dn, npairs, w->params.w[P_MARGIN], da, db, w->b.pose,
                                                      w->b.turn, w->b.half, head, axis, pa, pb);
        std::vector<float4> h(npairs), A((size_t)npairs * MOST_POINTS), B((size_t)npairs * MOST_POINTS);
        std::vector<float> ax(npairs);
        if (cudaStreamSynchronize(w->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
            rc = VXR_ECUDA;
        } else {
            cudaMemcpy(h.data(), head, sizeof(float4) * npairs, cudaMemcpyDeviceToHost);
            cudaMemcpy(ax.data(), axis, sizeof(float) * npairs, cudaMemcpyDeviceToHost);
            cudaMemcpy(A.data(), pa, sizeof(float4) * A.size(), cudaMemcpyDeviceToHost);
            cudaMemcpy(B.data(), pb, sizeof(float4) * B.size(), cudaMemcpyDeviceToHost);
            for (int p = 0; p < npairs; p++) {
                float* m = manifold + (size_t)p * MANIFOLD_WORDS;
                std::memset(m, 0, sizeof(float) * MANIFOLD_WORDS);
                const int q = where[p];
                if (q < 0) continue;
                const int cnt = (int)h[q].w;
                m[0] = h[q].x;
                m[1] = h[q].y;
                m[2] = h[q].z;
                m[3] = h[q].w;
                m[4] = ax[q];
                for (int i = 0; i < cnt; i++) {
                    float* r = m + M_POINTS + i * M_POINT_WORDS;
                    const float4 u = A[(size_t)q * MOST_POINTS + i], v = B[(size_t)q * MOST_POINTS + i];
                    r[0] = u.x;
                    r[1] = u.y;
                    r[2] = u.z;
                    r[3] = v.x;
                    r[4] = v.y;
                    r[5] = v.z;
                    r[6] = u.w;
                }
            }
        }
    }
    vxr_box_destroy(w);
    return rc;
}

}  // extern "C"

// ================================================================================================================
// The broad phase with no allocation.
//
// Some callers cannot allocate device memory while they step bodies: a host that hands the library only memory
// from its own pool (a Java or game-engine host managing device memory itself), code running where an allocation
// would synchronise the device or is forbidden (inside a frame's command stream, between the launches a caller is
// recording into a CUDA graph, or under a real-time deadline). For them, one entry point runs the broad phase (bin,
// stable counting sort, neighbourhood list and compaction: the same kernels a world's step runs) with all its
// scratch in one array in this library's device memory, sized below, that every GPU which loads the library holds
// until the process exits. The caller passes the inputs and the outputs; the library allocates nothing.
namespace {

constexpr int STATIC_MAX_BODIES = 16384;
constexpr int STATIC_MAX_CELLS = 262144;

constexpr size_t pad256(size_t bytes) { return (bytes + 255) & ~size_t(255); }
// regions, in order: pose, turn, half, reach (float4 a body); keys, order_tmp, order, partner (32 a body), found,
// kept, cand_start (+1); cell_count, cell_fill, cell_start (+1); scan tiles; counters
constexpr size_t STATIC_F4 = pad256(sizeof(float4) * STATIC_MAX_BODIES);
constexpr size_t STATIC_N = pad256(sizeof(int) * STATIC_MAX_BODIES);
constexpr size_t STATIC_N1 = pad256(sizeof(int) * (STATIC_MAX_BODIES + 1));
constexpr size_t STATIC_PARTNER = pad256(sizeof(int) * STATIC_MAX_BODIES * SLOTS);
constexpr size_t STATIC_C = pad256(sizeof(int) * STATIC_MAX_CELLS);
constexpr size_t STATIC_C1 = pad256(sizeof(int) * (STATIC_MAX_CELLS + 1));
constexpr size_t STATIC_TILES = pad256(sizeof(int) * ((STATIC_MAX_CELLS + SCAN_TILE - 1) / SCAN_TILE + 1));
constexpr size_t STATIC_COUNTERS = pad256(sizeof(Counters));
constexpr size_t STATIC_BYTES = 4 * STATIC_F4 + 5 * STATIC_N + STATIC_N1 + STATIC_PARTNER + 2 * STATIC_C + STATIC_C1 +
                                STATIC_TILES + STATIC_COUNTERS;

}  // namespace

// The scratch of vxr_box_broadphase_static: about 6 MiB. Host code must not use this name as a device address; the
// address comes from cudaGetSymbolAddress on the current device, every call.
static __device__ __align__(256) unsigned char vxr_broadphase_scratch[STATIC_BYTES];

namespace {

struct StaticFields {
    const float *x, *y, *z, *qx, *qy, *qz, *qw, *hx, *hy, *hz, *shape;
};

__global__ void k_pack_static(int n, StaticFields f, float4* __restrict__ pose, float4* __restrict__ turn,
                              float4* __restrict__ half) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    pose[s] = make_float4(f.x[s], f.y[s], f.z[s], 0.0f);
    turn[s] = make_float4(f.qx[s], f.qy[s], f.qz[s], f.qw[s]);
    half[s] = make_float4(f.hx[s], f.hy[s], f.hz[s], f.shape[s]);
}

__global__ void k_static_result(int n, int capacity, const int* __restrict__ cand_start, const Counters* counters,
                                int32_t* __restrict__ result) {
    const int total = cand_start[n];
    result[0] = total;
    result[1] = counters->unlisted;
    result[2] = total > capacity ? VXR_ECAPACITY : VXR_OK;
}

}  // namespace

extern "C" int32_t vxr_box_broadphase_static(int32_t bodies, const float* const* fields11, vxr_grid grid,
                                             int32_t reach_cells, float margin, int32_t* first_out,
                                             int32_t* second_out, int32_t capacity, int32_t* result3,
                                             void* stream) {
    if (bodies < 1 || !fields11 || !first_out || !second_out || !result3 || capacity < 0 || !(margin >= 0.0f))
        return VXR_EINVAL;
    for (int k = 0; k < 11; k++)
        if (!fields11[k]) return VXR_EINVAL;
    if (grid.nx < 1 || grid.ny < 1 || grid.nz < 1 || !(grid.cell > 0.0f)) return VXR_EINVAL;
    // The reach: 0 or 1 is the 27 cells; wider than the grid's widest side finds no more pairs, and an unbounded one
    // would only lengthen every thread's walk.
    if (reach_cells < 0 || reach_cells > std::max(grid.nx, std::max(grid.ny, grid.nz))) return VXR_EINVAL;
    const long cells = (long)grid.nx * grid.ny * grid.nz;
    if (bodies > STATIC_MAX_BODIES || cells > STATIC_MAX_CELLS) return VXR_ECAPACITY;  // beyond the fixed scratch
    // The array's address on the current device, looked up every call (no allocation): a cached one would go stale
    // once cudaDeviceReset unloads the module.
    void* symbol = nullptr;
    if (cudaGetSymbolAddress(&symbol, vxr_broadphase_scratch) != cudaSuccess || !symbol) return VXR_ECUDA;
    unsigned char* at = (unsigned char*)symbol;
    auto take = [&](size_t bytes) {
        unsigned char* r = at;
        at += bytes;
        return r;
    };
    float4* pose = (float4*)take(STATIC_F4);
    float4* turn = (float4*)take(STATIC_F4);
    float4* half = (float4*)take(STATIC_F4);
    float4* reach = (float4*)take(STATIC_F4);
    int* keys = (int*)take(STATIC_N);
    int* order_tmp = (int*)take(STATIC_N);
    int* order = (int*)take(STATIC_N);
    int* partner = (int*)take(STATIC_PARTNER);
    int* found = (int*)take(STATIC_N);
    int* kept = (int*)take(STATIC_N);
    int* cand_start = (int*)take(STATIC_N1);
    int* cell_count = (int*)take(STATIC_C);
    int* cell_fill = (int*)take(STATIC_C);
    int* cell_start = (int*)take(STATIC_C1);
    int* tiles = (int*)take(STATIC_TILES);
    Counters* counters = (Counters*)take(STATIC_COUNTERS);
    cudaStream_t st = (cudaStream_t)stream;
    const int n = bodies;
    // What must start at zero (the array keeps the last call's contents): the cell counts and fills, the counters.
    if (cudaMemsetAsync(cell_count, 0, sizeof(int) * cells, st) != cudaSuccess) return VXR_ECUDA;
    if (cudaMemsetAsync(cell_fill, 0, sizeof(int) * cells, st) != cudaSuccess) return VXR_ECUDA;
    if (cudaMemsetAsync(counters, 0, sizeof(Counters), st) != cudaSuccess) return VXR_ECUDA;
    StaticFields f{fields11[0], fields11[1], fields11[2], fields11[3], fields11[4], fields11[5],
                   fields11[6], fields11[7], fields11[8], fields11[9], fields11[10]};
    GridDims g{grid.nx, grid.ny, grid.nz, grid.cell, reach_cells > 0 ? reach_cells : 1};  // 0: the 27 cells
    k_pack_static<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, f, pose, turn, half);
    const SceneGrids none{nullptr, nullptr, nullptr};
    k_bin<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, g, none, pose, turn, half, keys, reach, cell_count);
    exclusive_scan(cell_count, cell_start, (int)cells, tiles, st);
    k_scatter<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, keys, cell_start, cell_fill, order_tmp);
    k_stable<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, keys, cell_start, order_tmp, order);
    k_list<<<blocks_for(n, 128), 128, 0, st>>>(n, g, none, margin, pose, reach, keys, cell_start, order, partner, found,
                                              kept, counters);
    exclusive_scan(kept, cand_start, n, tiles, st);
    k_candidates<<<blocks_for(n, THREADS), THREADS, 0, st>>>(n, capacity, kept, cand_start, partner, first_out,
                                                            second_out, counters);
    k_static_result<<<1, 1, 0, st>>>(n, capacity, cand_start, counters, result3);
    return cudaGetLastError() == cudaSuccess ? VXR_OK : VXR_ECUDA;
}
