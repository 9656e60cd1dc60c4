// The sphere package on the GPU: XPBD spheres in a walled box, solved by Jacobi or by Gauss-Seidel over a contact
// list run until every contact is solved, with warm starts, friction, rolling resistance, walls, restitution and the
// picture's pressing. The reference builds it as IR kernels, one dispatch each, driven from the host with a wait per
// batch of rounds (core = vexelray-sim-rigid-core/src/main/java/dev/vexelray/sim/rigid/; core/sphere/Spheres.java,
// SphereStep.java, SphereStepper.java). Here a whole call of steps is ONE persistent kernel: every pass of every
// substep runs in order inside it, the until-done loop and its batch sizing included, with a barrier between passes
// (the block's own barrier when the scene fits one block, a bounded grid barrier when it does not).
//
// Each pass keeps the reference's arithmetic in its association order (build with --fmad=false and IEEE division
// and square root), so a pass computes the reference's f32 values. Two things are made deterministic that the
// reference leaves to the device: the sort is stable (within a cell, ascending index), and the contact list is
// made by a count, a scan and a fill in sphere order (the order a serial run of the reference's atomic append
// gives), so the list, its chains and every later pass are reproducible bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "grid_sync.cuh"
#include "vxr.h"

namespace vxr {
namespace sph {

// Spheres.params words (core/sphere/Spheres.java:141-155).
enum { H = 0, GX, GY, GZ, SX, SY, SZ, OMEGA, AVERAGED, RESTITUTION, MU_STATIC, MU_KINETIC, MU_ROLLING, P_COUNT };
constexpr float COINCIDENT = 1e-12f;   // Spheres.java:157
constexpr float LIST_MARGIN = 0.02f;   // Spheres.java:795
constexpr float INERTIA = 0.4f;        // Spheres.java:247
constexpr int MOST_KEPT = 32;          // Spheres.java:944
constexpr int NEAR_KEPT = 16;          // near partners a sphere's count keeps for the list's fill
constexpr int CYCLE = 48, BATCH = 8;   // SphereStep.java:53-59
constexpr int SHRINK_AFTER = 120;      // SphereStepper.java:53
constexpr int SHOWN = 40, PRESSED_BEFORE = 8, PRESSED_AFTER = 20, TURNED_BEFORE = 32, TURNED_AFTER = 36;
constexpr int LISTED = 0, MISSED = 1, LONGEST = 2;
constexpr int THREADS = 512;
static_assert(THREADS % 32 == 0, "spheres are dealt out to the blocks by whole warps");
constexpr int SLICES_MOST = 1024;
constexpr int STAGE_MOST = 200 * 1024;  // shared memory a block may give a staged walk (the SM has 227 KB a block)  // blocks of a shared scan: a GPU holds at most 2048 / THREADS blocks an SM

struct SParams {
    float w[P_COUNT];
};

// Per-sphere state, seven float4 arrays (112 B a sphere). The inverse mass rides with the constraint moves and the
// radius with the position, so a parting contact reads two float4 a sphere.
struct State {
    float4* pos;   // x y z r
    float4* disp;  // dx dy dz im: what the constraints moved it this substep, and its inverse mass
    float4* turn;  // tx ty tz -: what the constraints turned it this substep
    float4* vel;   // u v w -
    float4* spin;  // ax ay az -: angular velocity
    float4* q;     // orientation qx qy qz qw
    float4* cvel;  // cx cy cz -: Jacobi's move, then the velocity before the substep's velocity pass
};

// One generation of the contact list: this substep's, or the one kept from the substep before.
struct ListGen {
    int2* pair;    // [cap] lower sphere, higher sphere
    int* done;     // [cap] the pass that solved it
    int* next;     // [cap] the lower sphere's previous contact, or -1
    float4* imp;   // [2 cap] (normal, p), (q, -): what it has taken this substep
    int* head;     // [n] the lower sphere's last contact, or -1
    int* start;    // [n + 1] where the lower sphere's contacts begin: they take places start .. head, one after
                   // another, so its chain (head, next, ...) is that range from the top down
};

struct Counts {
    int count[3];     // LISTED, MISSED, LONGEST (Spheres.CONTACT_COUNT_WORDS)
    int open[2];      // Spheres.OPEN_WORDS
    int last[4];      // the last step's report: waits, rounds, most rounds, unlisted
    long long total[4];  // summed over the call (most rounds: the largest)
    int status;
    int abort;
    unsigned int bar_count;
    unsigned int bar_gen;
    int cur;          // the generation holding the current list
    int rounds_at;    // the rounds a pass had run when it was given up (status ST_ROUNDS)
    int pad[2];
};

struct Kernel {
    int n, cap, substeps, iterations, solve, rounds, gridded, nx, ny, nz, cells, friction, steps;
    int cluster;  // the blocks form one thread-block cluster: passes are separated by the cluster's barrier
    int limit;    // rounds a pass may take before it is an error (SphereStepper.step :79)
    float cell;
    SParams p;
    State s;
    float4* wall;      // [6 n]: per axis, (normal, p) and (q, -)
    float* shown;      // [40 n]
    int* keys;         // [n]
    int* order;        // [n]
    int* cell_count;   // [cells]
    int* cell_start;   // [cells + 1]
    int* claims;       // [3 n]
    int* list_count;   // [n]
    int* near;         // [n * NEAR_KEPT] each sphere's first near partners, in the walk's order
    int* part;         // [blocks] each block's slice total in a scan the blocks share
    int* scan_tmp;     // [max(cells, n) + 1] a shared scan's slice-local prefixes
    const float* weight;  // the inverse masses a neighbour walk reads, weight[o * wstride]
    int wstride;
    int stage;         // 1: each block stages a walk's reads in its shared memory (staged_kernel)
    ListGen gen[2];
    Counts* counts;
    int* opening;      // [iterations] the rounds each pass's opening batch runs (SphereStepper.opening)
    int* enough;       // [iterations]
    GridBarrier bar;
};

__device__ __forceinline__ float dotf(const float* x, const float* y) {
    return x[0] * y[0] + (x[1] * y[1] + x[2] * y[2]);
}

__device__ __forceinline__ void crossf(const float* x, const float* y, float* z) {
    z[0] = x[1] * y[2] - x[2] * y[1];
    z[1] = x[2] * y[0] - x[0] * y[2];
    z[2] = x[0] * y[1] - x[1] * y[0];
}

__device__ __forceinline__ float get(const float4& v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// Spheres.turn :1468-1493: q + 1/2 (angle, 0) (x) q, normalised.
__device__ __forceinline__ float4 turned(float4 was, const float* angle) {
    const float a0 = 0.5f * angle[0], a1 = 0.5f * angle[1], a2 = 0.5f * angle[2];
    float4 now;
    now.x = was.x + (a0 * was.w + (a1 * was.z - a2 * was.y));
    now.y = was.y + (a1 * was.w + (a2 * was.x - a0 * was.z));
    now.z = was.z + (a2 * was.w + (a0 * was.y - a1 * was.x));
    now.w = was.w - (a0 * was.x + (a1 * was.y + a2 * was.z));
    const float len2 = (now.x * now.x + now.y * now.y) + (now.z * now.z + now.w * now.w);
    const float inverse = 1.0f / sqrtf(fmaxf(len2, 1e-30f));
    return make_float4(now.x * inverse, now.y * inverse, now.z * inverse, now.w * inverse);
}

// A sphere as a pass holds it: loaded once, worked on in registers, stored once (Spheres.Held :542-569).
struct Held {
    int s;
    float at[3], displaced[3], turned[3];
    float r, im;
};

__device__ __forceinline__ Held load(const State& S, int s) {
    Held h;
    h.s = s;
    const float4 p = S.pos[s], d = S.disp[s], t = S.turn[s];
    h.at[0] = p.x, h.at[1] = p.y, h.at[2] = p.z, h.r = p.w;
    h.displaced[0] = d.x, h.displaced[1] = d.y, h.displaced[2] = d.z, h.im = d.w;
    h.turned[0] = t.x, h.turned[1] = t.y, h.turned[2] = t.z;
    return h;
}

__device__ __forceinline__ void store(const State& S, const Held& h) {
    S.pos[h.s] = make_float4(h.at[0], h.at[1], h.at[2], h.r);
    S.disp[h.s] = make_float4(h.displaced[0], h.displaced[1], h.displaced[2], h.im);
    S.turn[h.s] = make_float4(h.turned[0], h.turned[1], h.turned[2], 0.0f);
}

// Spheres.Impulse :490-522: normal, p (3), q (3), two float4 in memory.
struct Impulse {
    float normal, p[3], q[3];
};

__device__ __forceinline__ Impulse load_impulse(const float4* at) {
    const float4 a = at[0], b = at[1];
    Impulse t;
    t.normal = a.x, t.p[0] = a.y, t.p[1] = a.z, t.p[2] = a.w;
    t.q[0] = b.x, t.q[1] = b.y, t.q[2] = b.z;
    return t;
}

__device__ __forceinline__ void store_impulse(float4* at, const Impulse& t) {
    at[0] = make_float4(t.normal, t.p[0], t.p[1], t.p[2]);
    at[1] = make_float4(t.q[0], t.q[1], t.q[2], 0.0f);
}

__device__ __forceinline__ void clear_impulse(Impulse& t) {
    t.normal = 0.0f;
    for (int k = 0; k < 3; k++) t.p[k] = t.q[k] = 0.0f;
}

__device__ __forceinline__ float turns_per_impulse(float wv, float lever, float radius) {
    return (wv * lever) / (INERTIA * (radius * radius));
}

__device__ __forceinline__ float rubbing_of(const SParams& P) {
    return P.w[MU_STATIC] + (P.w[MU_KINETIC] + P.w[MU_ROLLING]);
}

// Spheres.rub :662-677 (o null: a wall).
__device__ __forceinline__ void rub(Held& a, float wa, float turnsA, Held* o, float wo, float turnsO, const float* n,
                                    const float* p) {
    float np[3];
    crossf(n, p, np);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float move = wa * p[k];
        a.at[k] = a.at[k] + move;
        a.displaced[k] = a.displaced[k] + move;
        a.turned[k] = a.turned[k] - turnsA * np[k];
        if (o) {
            const float back = wo * p[k];
            o->at[k] = o->at[k] - back;
            o->displaced[k] = o->displaced[k] - back;
            o->turned[k] = o->turned[k] - turnsO * np[k];
        }
    }
}

// Spheres.contactTravel :751-766.
__device__ __forceinline__ void contact_travel(const float4& vel, const float4& spin, const Held& s, float h,
                                               const float* n, float lever, int side, float* travel) {
    float turn[3], turnN[3];
    turn[0] = h * spin.x + s.turned[0];
    turn[1] = h * spin.y + s.turned[1];
    turn[2] = h * spin.z + s.turned[2];
    crossf(turn, n, turnN);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float centre = h * get(vel, k) + s.displaced[k];
        const float spun = lever * turnN[k];
        travel[k] = side > 0 ? centre + spun : centre - spun;
    }
}

// Spheres.friction :595-654 (o null: a wall).
__device__ __forceinline__ void friction(const SParams& P, Held& a, const float4& velA, const float4& spinA, float wa,
                                         float leverA, Held* o, const float4& velO, const float4& spinO, float wo,
                                         float leverO, const float* n, Impulse& taken) {
    const float muS = P.w[MU_STATIC], muK = P.w[MU_KINETIC];
    const float lambdaN = taken.normal;
    if (!(muS + muK > 0.0f)) return;
    const float h = P.w[H];
    const float la = leverA;
    float slip[3];
    contact_travel(velA, spinA, a, h, n, la, -1, slip);
    const float ia = wa;
    const float leverOverIa = turns_per_impulse(ia, la, a.r);
    float weight = ia + leverOverIa * la;
    float leverOverIo = 0.0f, io = 0.0f;
    if (o) {
        io = wo;
        const float lo = leverO;
        float other[3];
        contact_travel(velO, spinO, *o, h, n, lo, 1, other);
#pragma unroll
        for (int k = 0; k < 3; k++) slip[k] = slip[k] - other[k];
        leverOverIo = turns_per_impulse(io, lo, o->r);
        weight = weight + (io + leverOverIo * lo);
    }
    const float along = dotf(slip, n);
    float tangent[3];
#pragma unroll
    for (int k = 0; k < 3; k++) tangent[k] = slip[k] - along * n[k];
    if (!(weight > 0.0f)) return;
    const float takenAlong = dotf(taken.p, n);
    float before[3], whole[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        before[k] = taken.p[k] - takenAlong * n[k];
        whole[k] = before[k] - tangent[k] / weight;
    }
    const float size2 = dotf(whole, whole);
    const float holds = muS * lambdaN;
    if (size2 > holds * holds) {
        const float cut = fminf(1.0f, (muK * lambdaN) / sqrtf(size2));
#pragma unroll
        for (int k = 0; k < 3; k++) whole[k] = whole[k] * cut;
    }
    float p[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        p[k] = whole[k] - before[k];
        taken.p[k] = whole[k];
    }
    rub(a, ia, leverOverIa, o, io, leverOverIo, n, p);
}

// Spheres.roll :699-741 (o null: a wall).
__device__ __forceinline__ void roll(const SParams& P, Held& a, const float4& spinA, float wa, Held* o,
                                     const float4& spinO, float wo, float reach, Impulse& taken) {
    const float muR = P.w[MU_ROLLING];
    const float h = P.w[H];
    const float ra = a.r;
    const float ia = wa / (INERTIA * (ra * ra));
    float inverse = ia;
    float io = 0.0f;
    float against[3];
    against[0] = h * spinA.x + a.turned[0];
    against[1] = h * spinA.y + a.turned[1];
    against[2] = h * spinA.z + a.turned[2];
    if (o) {
        const float ro = o->r;
        io = wo / (INERTIA * (ro * ro));
        inverse = inverse + io;
        against[0] = against[0] - (h * spinO.x + o->turned[0]);
        against[1] = against[1] - (h * spinO.y + o->turned[1]);
        against[2] = against[2] - (h * spinO.z + o->turned[2]);
    }
    if (!(inverse > 0.0f)) return;
    float whole[3];
#pragma unroll
    for (int k = 0; k < 3; k++) whole[k] = taken.q[k] - against[k] / inverse;
    const float size2 = dotf(whole, whole);
    const float holds = (muR * reach) * taken.normal;
    if (size2 > holds * holds) {
        const float cut = fminf(1.0f, holds / sqrtf(size2));
#pragma unroll
        for (int k = 0; k < 3; k++) whole[k] = whole[k] * cut;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float change = whole[k] - taken.q[k];
        taken.q[k] = whole[k];
        a.turned[k] = a.turned[k] + ia * change;
        if (o) o->turned[k] = o->turned[k] - io * change;
    }
}

// Spheres.warm :448-481.
__device__ __forceinline__ void warm(Held& a, float wa, Held& o, float wo, const float* d, float d2, float reach,
                                     Impulse& taken) {
    const float dist = sqrtf(d2);
    float n[3];
#pragma unroll
    for (int k = 0; k < 3; k++) n[k] = d[k] / dist;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float push = taken.normal * n[k];
        const float ma = push * wa;
        const float mo = -(push * wo);
        a.at[k] = a.at[k] + ma;
        o.at[k] = o.at[k] + mo;
        a.displaced[k] = a.displaced[k] + ma;
        o.displaced[k] = o.displaced[k] + mo;
    }
    const float along = dotf(taken.p, n);
#pragma unroll
    for (int k = 0; k < 3; k++) taken.p[k] = taken.p[k] - along * n[k];
    const float share = dist / reach;
    const float ra = a.r, ro = o.r;
    const float turnsA = turns_per_impulse(wa, share * ra, ra);
    const float turnsO = turns_per_impulse(wo, share * ro, ro);
    rub(a, wa, turnsA, &o, wo, turnsO, n, taken.p);
    const float ia = wa / (INERTIA * (ra * ra));
    const float io = wo / (INERTIA * (ro * ro));
#pragma unroll
    for (int k = 0; k < 3; k++) {
        a.turned[k] = a.turned[k] + ia * taken.q[k];
        o.turned[k] = o.turned[k] - io * taken.q[k];
    }
}

// Spheres.contact :369-439: contact c of spheres ai and oi, parting (rubs 0) or rubbing.
__device__ void contact(const Kernel& K, float4* impulse, int ai, int oi, int pass, int rubs) {
    const State& S = K.s;
    Held ha = load(S, ai), ho = load(S, oi);
    float d[3];
#pragma unroll
    for (int k = 0; k < 3; k++) d[k] = ha.at[k] - ho.at[k];
    const float d2 = dotf(d, d);
    const float reach = ha.r + ho.r;
    const float wa = ha.im, wo = ho.im;
    const float wsum = wa + wo;
    const float listed = reach * (1.0f + LIST_MARGIN);
    if (!(d2 < listed * listed)) return;
    if (!(d2 > COINCIDENT)) return;
    if (!(wsum > 0.0f)) return;
    Impulse taken = load_impulse(impulse);
    if (rubs == 0) {
        if (pass == 1) {
            if (rubbing_of(K.p) > 0.0f) warm(ha, wa, ho, wo, d, d2, reach, taken);
            else clear_impulse(taken);
        }
#pragma unroll
        for (int k = 0; k < 3; k++) d[k] = ha.at[k] - ho.at[k];
        const float dist = sqrtf(fmaxf(dotf(d, d), COINCIDENT));
        const float depth = fmaxf(-(taken.normal * wsum), K.p.w[OMEGA] * (reach - dist));
        taken.normal = taken.normal + depth / wsum;
        const float kk = depth / (dist * wsum);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float step = kk * d[k];
            const float ma = step * wa;
            const float mo = -(step * wo);
            ha.at[k] = ha.at[k] + ma;
            ho.at[k] = ho.at[k] + mo;
            ha.displaced[k] = ha.displaced[k] + ma;
            ho.displaced[k] = ho.displaced[k] + mo;
        }
    } else {
        const float dist = sqrtf(d2);
        float n[3];
#pragma unroll
        for (int k = 0; k < 3; k++) n[k] = d[k] / dist;
        const float share = dist / reach;
        const float pairRadius = (ha.r * ho.r) / reach;
        const float4 velA = S.vel[ai], velO = S.vel[oi], spinA = S.spin[ai], spinO = S.spin[oi];
        roll(K.p, ha, spinA, wa, &ho, spinO, wo, pairRadius, taken);
        friction(K.p, ha, velA, spinA, wa, share * ha.r, &ho, velO, spinO, wo, share * ho.r, n, taken);
    }
    store_impulse(impulse, taken);
    store(S, ha);
    store(S, ho);
}

// Spheres.priority :1166-1168.
__device__ __forceinline__ int priority(int pair, int g) {
    return (int)(((unsigned)pair * 0x9E3779B1u + (unsigned)g * 0x632BE5ABu) & 0x7FFFFFFFu);
}

// Cell of a centre (Spheres.bin :1308-1323).
__device__ __forceinline__ int cell_key(const Kernel& K, float x, float y, float z) {
    const int c0 = (int)fmaxf(0.0f, fminf((float)(K.nx - 1), floorf(x / K.cell)));
    const int c1 = (int)fmaxf(0.0f, fminf((float)(K.ny - 1), floorf(y / K.cell)));
    const int c2 = (int)fmaxf(0.0f, fminf((float)(K.nz - 1), floorf(z / K.cell)));
    return c0 + K.nx * (c1 + K.ny * c2);
}

// Spheres.around :1207-1229: every sphere of s's cell and the 26 around it, each cell in the sort's order; with no
// grid, every sphere in index order.
// visit(o, pos[o]) for each (with WEIGHTS, visit(o, pos[o], disp[o].w): the inverse mass comes in the same batch).
// The spheres of a run are fetched four at a time, their order entries and then their positions each as one batch of
// independent loads, before the four are visited in turn: the same spheres in the same order, with one memory round
// trip a batch instead of two or three a sphere.
template <bool WEIGHTS = false, typename Visit>
__device__ __forceinline__ void around(const Kernel& K, int s, Visit visit) {
    const float4* pos = K.s.pos;
    if (!K.gridded) {
        for (int o = 0; o < K.n; o++) {
            if constexpr (WEIGHTS) visit(o, pos[o], K.weight[(size_t)o * K.wstride]);
            else visit(o, pos[o]);
        }
        return;
    }
    const int key = K.keys[s];
    const int ix = key % K.nx, iy = (key / K.nx) % K.ny, iz = key / (K.nx * K.ny);
    // The cells go x fastest, and x-neighbours have consecutive keys, so each row of up to three cells is one run
    // of the sort's order: nine runs, the same spheres in the same order as cell by cell.
    const int x0 = max(ix - 1, 0), x1 = min(ix + 1, K.nx - 1);
    for (int row = 0; row < 9; row++) {
        const int jy = iy + (row % 3 - 1), jz = iz + (row / 3 - 1);
        if (!(jy >= 0 && jy < K.ny && jz >= 0 && jz < K.nz)) continue;
        const int first = x0 + K.nx * (jy + K.ny * jz);
        const int end = K.cell_start[first + (x1 - x0) + 1];
        for (int k = K.cell_start[first]; k < end; k += 4) {
            const int m = min(4, end - k);
            int o0 = K.order[k], o1 = 0, o2 = 0, o3 = 0;
            if (m > 1) o1 = K.order[k + 1];
            if (m > 2) o2 = K.order[k + 2];
            if (m > 3) o3 = K.order[k + 3];
            float4 p0 = pos[o0], p1 = p0, p2 = p0, p3 = p0;
            if (m > 1) p1 = pos[o1];
            if (m > 2) p2 = pos[o2];
            if (m > 3) p3 = pos[o3];
            float w0 = 0.0f, w1 = 0.0f, w2 = 0.0f, w3 = 0.0f;
            if constexpr (WEIGHTS) {
                w0 = K.weight[(size_t)o0 * K.wstride];
                if (m > 1) w1 = K.weight[(size_t)o1 * K.wstride];
                if (m > 2) w2 = K.weight[(size_t)o2 * K.wstride];
                if (m > 3) w3 = K.weight[(size_t)o3 * K.wstride];
            }
            for (int j = 0; j < m; j++) {
                if constexpr (WEIGHTS) visit(o0, p0, w0);
                else visit(o0, p0);
                o0 = o1, o1 = o2, o2 = o3;
                p0 = p1, p1 = p2, p2 = p3;
                w0 = w1, w1 = w2, w2 = w3;
            }
        }
    }
}

// --- per-sphere passes ---------------------------------------------------------------------------------------

// Spheres.predict :269-295.
__device__ __forceinline__ void predict(const Kernel& K, int s) {
    const State& S = K.s;
    if (!(S.disp[s].w > 0.0f)) return;
    const float h = K.p.w[H];
    float4 p = S.pos[s], v = S.vel[s];
    const float4 w = S.spin[s];
    v.x = v.x + h * K.p.w[GX];
    p.x = p.x + h * v.x;
    v.y = v.y + h * K.p.w[GY];
    p.y = p.y + h * v.y;
    v.z = v.z + h * K.p.w[GZ];
    p.z = p.z + h * v.z;
    S.vel[s] = v;
    S.pos[s] = p;
    const float angle[3] = {h * w.x, h * w.y, h * w.z};
    S.q[s] = turned(S.q[s], angle);
}

// Spheres.warmWalls :890-939.
__device__ __forceinline__ void warm_walls(const Kernel& K, int s) {
    const State& S = K.s;
    Held held = load(S, s);
    if (!(held.im > 0.0f)) return;
    const float r = held.r, wv = held.im;
    const float turns = turns_per_impulse(wv, r, r);
    const float rubbing = rubbing_of(K.p);
#pragma unroll
    for (int axis = 0; axis < 3; axis++) {
        float4* rec = K.wall + 6 * (size_t)s + 2 * axis;
        Impulse taken = load_impulse(rec);
        const float reach = r * (1.0f + LIST_MARGIN);
        const float position = held.at[axis];
        float out = 0.0f;
        if (position < reach) out = 1.0f;
        if (position > K.p.w[SX + axis] - reach) out = -1.0f;
        if (!(rubbing > 0.0f && out != 0.0f)) {
            clear_impulse(taken);
        } else {
            const float push = (taken.normal * wv) * out;
            held.at[axis] = held.at[axis] + push;
            held.displaced[axis] = held.displaced[axis] + push;
            taken.p[axis] = 0.0f;
            float n[3] = {0.0f, 0.0f, 0.0f};
            n[axis] = out;
            rub(held, wv, turns, nullptr, 0.0f, 0.0f, n, taken.p);
#pragma unroll
            for (int k = 0; k < 3; k++) held.turned[k] = held.turned[k] + (turns * taken.q[k]) / r;
        }
        store_impulse(rec, taken);
    }
    store(S, held);
}

// Spheres.walls :1185-1198 = shift :1351-1418 with friction.
__device__ __forceinline__ void walls(const Kernel& K, int s) {
    const State& S = K.s;
    Held held = load(S, s);
    if (!(held.im > 0.0f)) return;
    const float r = held.r;
    const float4 vel = S.vel[s], spin = S.spin[s];
    const float4 none = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float c = 0.0f;
        const float moved = held.at[a] + c;
        const float high = K.p.w[SX + a] - r;
        float side = 1.0f;
        float into = r - moved;
        if (moved * 2.0f > K.p.w[SX + a]) {
            side = -1.0f;
            into = moved - high;
        }
        const float wv = held.im;
        float4* rec = K.wall + 6 * (size_t)s + 2 * a;
        Impulse taken = load_impulse(rec);
        float inside = fmaxf(r, fminf(high, moved));
        float push = fmaxf(into, 0.0f);
        if (!(into > 0.0f) && taken.normal > 0.0f) {
            push = fmaxf(into, -(taken.normal * wv));
            inside = moved + side * push;
        }
        taken.normal = taken.normal + push / wv;
        held.at[a] = inside;
        held.displaced[a] = held.displaced[a] + (c + (inside - moved));
        const float reach = r * LIST_MARGIN;
        float out = 0.0f;
        if (!(inside > r + reach)) out = 1.0f;
        if (!(inside < high - reach)) out = -1.0f;
        if (out != 0.0f) {
            float n[3] = {0.0f, 0.0f, 0.0f};
            n[a] = out;
            roll(K.p, held, spin, wv, nullptr, none, 0.0f, r, taken);
            friction(K.p, held, vel, spin, wv, r, nullptr, none, none, 0.0f, 0.0f, n, taken);
        }
        store_impulse(rec, taken);
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float high = K.p.w[SX + a] - r;
        const float inside = fmaxf(r, fminf(high, held.at[a]));
        held.displaced[a] = held.displaced[a] + (inside - held.at[a]);
        held.at[a] = inside;
    }
    store(S, held);
}

// Spheres.solve(grid) :302-347 / Solving :1245-1298: Jacobi's move into cx, cy, cz.
constexpr int CONTACTS_HELD = 16;  // a sphere's contacts a Jacobi walk lists before solving them

__device__ __forceinline__ void jacobi_solve(const Kernel& K, int s) {
    const State& S = K.s;
    const float4 me = S.pos[s];
    const float mine[3] = {me.x, me.y, me.z};
    const float rs = me.w, ws = S.disp[s].w;
    float sum[3] = {0.0f, 0.0f, 0.0f};
    float contacts = 0.0f;
    // Whether o touches s, and if so its share of the move: the same arithmetic in both passes below.
    auto touching = [&](float4 other, float wo, float* d, float& reach, float& wsum) {
        d[0] = mine[0] - other.x, d[1] = mine[1] - other.y, d[2] = mine[2] - other.z;
        const float d2 = d[0] * d[0] + (d[1] * d[1] + d[2] * d[2]);
        reach = rs + other.w;
        wsum = ws + wo;
        return d2 < reach * reach && d2 > COINCIDENT && wsum > 0.0f;
    };
    auto add = [&](const float* d, float reach, float wsum) {
        const float d2 = d[0] * d[0] + (d[1] * d[1] + d[2] * d[2]);
        const float dist = sqrtf(d2);
        const float share = ((reach - dist) * (ws / wsum)) / dist;
#pragma unroll
        for (int a = 0; a < 3; a++) sum[a] = sum[a] + share * d[a];
        contacts = contacts + 1.0f;
    };
    // First the walk lists the touching spheres in its order (a cheap test a candidate), then they are solved in
    // that order: the lanes of a warp, each walking its own sphere, then run the square root and the divisions once
    // a contact, not once for every candidate any lane finds touching. A sphere touching more than CONTACTS_HELD
    // walks again, solving as it goes.
    int held[CONTACTS_HELD];
    int count = 0;
    around<true>(K, s, [&](int o, float4 other, float wo) {
        if (o == s) return;
        float d[3], reach, wsum;
        if (!touching(other, wo, d, reach, wsum)) return;
        if (count < CONTACTS_HELD) held[count] = o;
        count++;
    });
    if (count <= CONTACTS_HELD) {
        for (int k = 0; k < count; k++) {
            const int o = held[k];
            float d[3], reach, wsum;
            touching(S.pos[o], K.weight[(size_t)o * K.wstride], d, reach, wsum);
            add(d, reach, wsum);
        }
    } else {
        around<true>(K, s, [&](int o, float4 other, float wo) {
            if (o == s) return;
            float d[3], reach, wsum;
            if (touching(other, wo, d, reach, wsum)) add(d, reach, wsum);
        });
    }
    const float omega = K.p.w[OMEGA];
    float scale = omega;
    if (K.p.w[AVERAGED] > 0.0f) scale = omega / fmaxf(contacts, 1.0f);
    S.cvel[s] = make_float4(scale * sum[0], scale * sum[1], scale * sum[2], 0.0f);
}

// Spheres.apply :1326-1342 (shift without friction).
__device__ __forceinline__ void jacobi_apply(const Kernel& K, int s) {
    const State& S = K.s;
    Held held = load(S, s);
    if (!(held.im > 0.0f)) return;
    const float r = held.r;
    const float4 move = S.cvel[s];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float c = get(move, a);
        const float moved = held.at[a] + c;
        const float high = K.p.w[SX + a] - r;
        const float inside = fmaxf(r, fminf(high, moved));
        held.at[a] = inside;
        const float push = inside - moved;
        held.displaced[a] = held.displaced[a] + (c + push);
    }
    store(S, held);
}

// Spheres.velocity :1430-1460.
__device__ __forceinline__ void velocity(const Kernel& K, int s) {
    const State& S = K.s;
    const float perH = 1.0f / K.p.w[H];
    const float4 was = S.vel[s], d = S.disp[s], t = S.turn[s], w = S.spin[s];
    S.cvel[s] = make_float4(was.x, was.y, was.z, 0.0f);
    S.vel[s] = make_float4(was.x + d.x * perH, was.y + d.y * perH, was.z + d.z * perH, was.w);
    S.disp[s] = make_float4(0.0f, 0.0f, 0.0f, d.w);
    S.spin[s] = make_float4(w.x + t.x * perH, w.y + t.y * perH, w.z + t.z * perH, w.w);
    S.turn[s] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float angle[3] = {t.x, t.y, t.z};
    S.q[s] = turned(S.q[s], angle);
}

// Spheres.bounce(grid) :1528-1627: the change into dx, dy, dz.
__device__ __forceinline__ void bounce(const Kernel& K, int s) {
    const State& S = K.s;
    const float e = K.p.w[RESTITUTION];
    const float4 me = S.pos[s];
    const float wa = S.disp[s].w;
    if (!(e > 0.0f && wa > 0.0f)) return;
    const float h = K.p.w[H];
    const float gx = K.p.w[GX], gy = K.p.w[GY], gz = K.p.w[GZ];
    const float resting = (2.0f * h) * sqrtf(gx * gx + (gy * gy + gz * gz));
    const float ra = me.w;
    const float mine[3] = {me.x, me.y, me.z};
    const float4 v4 = S.vel[s], c4 = S.cvel[s];
    const float vel[3] = {v4.x, v4.y, v4.z}, was[3] = {c4.x, c4.y, c4.z};
    float sum[3] = {0.0f, 0.0f, 0.0f};
    around(K, s, [&](int o, float4 other) {
        if (o == s) return;
        float d[3] = {mine[0] - other.x, mine[1] - other.y, mine[2] - other.z};
        const float d2 = d[0] * d[0] + (d[1] * d[1] + d[2] * d[2]);
        const float near = (ra + other.w) * (1.0f + LIST_MARGIN);
        const float wsum = wa + S.disp[o].w;
        if (!(d2 < near * near && d2 > COINCIDENT)) return;
        const float dist = sqrtf(d2);
        const float4 ov = S.vel[o], oc = S.cvel[o];
        float closing = 0.0f, parting = 0.0f;
        const float n0 = d[0] / dist, n1 = d[1] / dist, n2 = d[2] / dist;
        closing = closing + n0 * (was[0] - oc.x);
        parting = parting + n0 * (vel[0] - ov.x);
        closing = closing + n1 * (was[1] - oc.y);
        parting = parting + n1 * (vel[1] - ov.y);
        closing = closing + n2 * (was[2] - oc.z);
        parting = parting + n2 * (vel[2] - ov.z);
        if (closing < -resting) {
            const float k = ((-(e * closing) - parting) * wa) / (wsum * dist);
#pragma unroll
            for (int a = 0; a < 3; a++) sum[a] = sum[a] + k * d[a];
        }
    });
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float reach = ra * (1.0f + LIST_MARGIN);
        if (mine[a] < reach && was[a] < -resting) sum[a] = sum[a] + (-(e * was[a]) - vel[a]);
        if (mine[a] > K.p.w[SX + a] - reach && was[a] > resting) sum[a] = sum[a] + (-(e * was[a]) - vel[a]);
    }
    S.disp[s] = make_float4(sum[0], sum[1], sum[2], wa);
}

// Spheres.bounced :1633-1644.
__device__ __forceinline__ void bounced(const Kernel& K, int s) {
    const State& S = K.s;
    const float4 v = S.vel[s], d = S.disp[s];
    S.vel[s] = make_float4(v.x + d.x, v.y + d.y, v.z + d.z, v.w);
    S.disp[s] = make_float4(0.0f, 0.0f, 0.0f, d.w);
}

// Spheres.show(grid) :1697-1794.
__device__ __forceinline__ void show(const Kernel& K, int s) {
    const State& S = K.s;
    float* sh = K.shown + (size_t)s * SHOWN;
    const float4 me = S.pos[s];
    const float mine[3] = {me.x, me.y, me.z};
    const float rs = me.w;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        sh[a] = sh[4 + a];
        sh[4 + a] = mine[a];
    }
    sh[3] = rs;
    for (int k = 0; k < 12; k++) sh[PRESSED_BEFORE + k] = sh[PRESSED_AFTER + k];
    const float4 q = S.q[s];
    for (int k = 0; k < 4; k++) sh[TURNED_BEFORE + k] = sh[TURNED_AFTER + k];
    sh[TURNED_AFTER + 0] = q.x;
    sh[TURNED_AFTER + 1] = q.y;
    sh[TURNED_AFTER + 2] = q.z;
    sh[TURNED_AFTER + 3] = q.w;
    float flat[6] = {0, 0, 0, 0, 0, 0}, lean[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float low = rs - mine[a];
        const float high = (mine[a] + rs) - K.p.w[SX + a];
        if (low > 0.0f) {
            const float share = low / rs;
            flat[a] = flat[a] + share;
            lean[a] = lean[a] + -1.0f * share;
        }
        if (high > 0.0f) {
            const float share = high / rs;
            flat[a] = flat[a] + share;
            lean[a] = lean[a] + 1.0f * share;
        }
    }
    around(K, s, [&](int o, float4 other) {
        if (o == s) return;
        float d[3] = {other.x - mine[0], other.y - mine[1], other.z - mine[2]};
        const float d2 = dotf(d, d);
        const float reach = rs + other.w;
        if (!(d2 < reach * reach && d2 > COINCIDENT)) return;
        const float dist = sqrtf(d2);
        const float share = (reach - dist) / reach;
        const float g = share / d2;
        const float along = share / dist;
        flat[0] = flat[0] + g * (d[0] * d[0]);
        flat[1] = flat[1] + g * (d[1] * d[1]);
        flat[2] = flat[2] + g * (d[2] * d[2]);
        flat[3] = flat[3] + g * (d[0] * d[1]);
        flat[4] = flat[4] + g * (d[0] * d[2]);
        flat[5] = flat[5] + g * (d[1] * d[2]);
#pragma unroll
        for (int a = 0; a < 3; a++) lean[a] = lean[a] + along * d[a];
    });
    float* after = sh + PRESSED_AFTER;
    for (int k = 0; k < 6; k++) after[k] = flat[k];
    for (int a = 0; a < 3; a++) after[6 + a] = lean[a];
    after[9] = (flat[0] + flat[1]) + flat[2];
    after[10] = sqrtf(dotf(lean, lean));
}

// --- the contact list ----------------------------------------------------------------------------------------

// listContacts' first half: how many spheres of higher index are near sphere a (Spheres.listContacts :961-1022).
// listContacts' first half: how many higher-numbered spheres are near a. The first NEAR_KEPT of them, in the walk's
// order, are kept in K.near for the fill, which then needs no second walk.
__device__ __forceinline__ int count_near(const Kernel& K, int a) {
    const float4 me = K.s.pos[a];
    int found = 0;
    int* keep = K.near + (size_t)a * NEAR_KEPT;
    around(K, a, [&](int o, float4 other) {
        if (!(o > a)) return;
        const float d0 = me.x - other.x, d1 = me.y - other.y, d2v = me.z - other.z;
        const float d2 = d0 * d0 + (d1 * d1 + d2v * d2v);
        const float near = (me.w + other.w) * (1.0f + LIST_MARGIN);
        if (d2 < near * near) {
            if (found < NEAR_KEPT) keep[found] = o;
            found++;
        }
    });
    return found;
}

// listContacts' second half: sphere a's contacts written at the places the scan gave it, chained, each with the
// impulses the pair took in the substep before (found by walking a's kept chain, at most MOST_KEPT places).
__device__ __forceinline__ void fill_near(const Kernel& K, const ListGen& L, const ListGen& kept, int a, int first) {
    const float4 me = K.s.pos[a];
    int slot = first;
    int last = -1;
    // a's kept chain, at most MOST_KEPT places from its head: the places of that range, searched with independent
    // loads (each partner is listed once, so the place found is the one the walk down the chain finds)
    const int top = kept.head[a];
    const int bottom = top >= 0 ? max(kept.start[a], top - (MOST_KEPT - 1)) : 0;
    auto place = [&](int o) {
        const int at = slot++;
        if (!(at < K.cap)) return;
        L.pair[at] = make_int2(a, o);
        L.done[at] = 0;
        L.next[at] = last;
        last = at;
        float4 w0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), w1 = w0;
        for (int j = top; j >= bottom; j--) {
            if (__ldg(&kept.pair[j].y) == o) {
                w0 = kept.imp[2 * (size_t)j];
                w1 = kept.imp[2 * (size_t)j + 1];
                break;
            }
        }
        L.imp[2 * (size_t)at] = w0;
        L.imp[2 * (size_t)at + 1] = w1;
    };
    const int found = K.list_count[a];
    if (found <= NEAR_KEPT) {  // the partners the count kept, in the walk's order
        const int* keep = K.near + (size_t)a * NEAR_KEPT;
        for (int i = 0; i < found; i++) place(keep[i]);
    } else {  // more than were kept: the walk again, the same spheres in the same order
        around(K, a, [&](int o, float4 other) {
            if (!(o > a)) return;
            const float d0 = me.x - other.x, d1 = me.y - other.y, d2v = me.z - other.z;
            const float d2 = d0 * d0 + (d1 * d1 + d2v * d2v);
            const float near = (me.w + other.w) * (1.0f + LIST_MARGIN);
            if (!(d2 < near * near)) return;
            place(o);
        });
    }
    L.head[a] = last;
}

// The list places a thread owns for a substep (place gtid + j gsize for j < HELD_PLACES), their pairs held in
// registers from the list's fill to the substep's end, and which of them this pass has done: a round reads neither
// from memory. No other thread writes a place's pair or its done mark.
constexpr int HELD_PLACES = 2;
struct HeldPlaces {
    int2 pair[HELD_PLACES];
    unsigned done;
};

// One place of a dispatch: solve it if it won the dispatch before (its priority holds both spheres' claims), else
// clear the spheres' checks and claim them for this dispatch (and note the pass still open). Returns whether it was
// solved.
// checked_a, checked_b: the spheres' check words, read by the caller (the claim arrays a dispatch checks are not
// written while it runs, so they may be read ahead).
__device__ __forceinline__ bool contact_place(const Kernel& K, const ListGen& L, int c, int2 ab, int checks,
                                              int claims, int pass, int dispatch, int check_dispatch, int rubs,
                                              int checked_a, int checked_b, int* claimed, int* cleared, bool& open) {
    const int pair = ab.x * K.n + ab.y;
    int won = 0;
    if (checks > 0) {
        const int last = priority(pair, check_dispatch);
        if (checked_a == last && checked_b == last) won = 1;
    }
    if (won) {
        contact(K, L.imp + 2 * (size_t)c, ab.x, ab.y, pass, rubs);
        L.done[c] = pass;
        return true;
    }
    cleared[ab.x] = 0;
    cleared[ab.y] = 0;
    if (claims > 0) {
        open = true;
        const int mine = priority(pair, dispatch);
        atomicMax(&claimed[ab.x], mine);
        atomicMax(&claimed[ab.y], mine);
    } else {
        atomicAdd(&K.counts->count[MISSED], 1);
    }
    return false;
}

// Spheres.contactRound :1076-1133, one dispatch over the list. The winners of a dispatch share no sphere (each
// sphere's claim is held by one priority), so they solve in parallel with the result of any serial order.
__device__ __forceinline__ void contact_round(const Kernel& K, const ListGen& L, int listed, int checks, int claims,
                                              int pass, int dispatch, int mark, int check_dispatch, int rubs,
                                              const int* checked, int* claimed, int* cleared, int gtid, int gsize,
                                              HeldPlaces& mine) {
    if (gtid == 0) K.counts->open[1 - mark] = 0;
    bool open = false;
    // the held places' check words, all loaded before the first place is solved
    int check_a[HELD_PLACES], check_b[HELD_PLACES];
#pragma unroll
    for (int j = 0; j < HELD_PLACES; j++) {
        const bool live = checks > 0 && gtid + j * gsize < listed && !((mine.done >> j) & 1u);
        check_a[j] = live ? checked[mine.pair[j].x] : 0;
        check_b[j] = live ? checked[mine.pair[j].y] : 0;
    }
#pragma unroll
    for (int j = 0; j < HELD_PLACES; j++) {
        const int c = gtid + j * gsize;
        if (c < listed && !((mine.done >> j) & 1u) &&
            contact_place(K, L, c, mine.pair[j], checks, claims, pass, dispatch, check_dispatch, rubs, check_a[j],
                          check_b[j], claimed, cleared, open))
            mine.done |= 1u << j;
    }
    for (int c = gtid + HELD_PLACES * gsize; c < listed; c += gsize) {
        if (L.done[c] == pass) continue;
        const int2 ab = L.pair[c];
        contact_place(K, L, c, ab, checks, claims, pass, dispatch, check_dispatch, rubs,
                      checks > 0 ? checked[ab.x] : 0, checks > 0 ? checked[ab.y] : 0, claimed, cleared, open);
    }
    // one store a warp that left a place open, not one a place
    if (__any_sync(0xffffffffu, open) && (threadIdx.x & 31) == 0) K.counts->open[mark] = 1;
}

__device__ __forceinline__ int position(int k) { return k == 0 ? 0 : 1 + (k - 1) % CYCLE; }

// Exclusive scan of in[lo..hi) into out[lo..hi), starting from zero, by the threads of one block; returns the range's
// total to every thread.
__device__ int block_scan_range(const int* in, int* out, int lo, int hi) {
    __shared__ int warp_sums[32];
    const int m = hi - lo;
    const int per = (m + blockDim.x - 1) / blockDim.x;
    const int begin = lo + min(m, (int)threadIdx.x * per), end = min(hi, begin + per);
    int sum = 0;
    for (int i = begin; i < end; i++) sum += in[i];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int v = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        warp_sums[lane] = v;
    }
    __syncthreads();
    int run = (warp > 0 ? warp_sums[warp - 1] : 0) + x - sum;
    for (int i = begin; i < end; i++) {
        const int v = in[i];
        out[i] = run;
        run += v;
    }
    const int total = warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
    return total;
}

// The first half of a scan every block shares: block b scans its slice of in[0..m) into out, and posts the slice's
// total. After a barrier, scan_finish adds the totals of the slices before it; out[m] is the whole total.
__device__ __forceinline__ void scan_slices(const Kernel& K, const int* in, int* out, int m) {
    const int per = (m + gridDim.x - 1) / gridDim.x;
    const int lo = min(m, (int)blockIdx.x * per), hi = min(m, lo + per);
    const int total = block_scan_range(in, out, lo, hi);
    if (threadIdx.x == 0) K.part[blockIdx.x] = total;
}
// After the barrier that follows scan_slices: the slice totals' exclusive prefix in this block's shared memory
// (slice b's offset at offs[b], the whole at offs[gridDim.x]), summed by one warp.
__device__ __forceinline__ void slice_offsets(const Kernel& K, int* offs) {
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int carry = 0;
        for (int base = 0; base < (int)gridDim.x; base += 32) {
            const int b = base + lane;
            const int v = b < (int)gridDim.x ? *(const volatile int*)&K.part[b] : 0;
            int x = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (b < (int)gridDim.x) offs[b] = carry + x - v;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
        if (lane == 0) offs[gridDim.x] = carry;
    }
    __syncthreads();
}

// Element i of the scan scan_slices left slice-local in `local`: any slice's, in the same pass as the finish.
__device__ __forceinline__ int scan_value(const int* local, const int* offs, int i, int m) {
    const int per = (m + gridDim.x - 1) / gridDim.x;
    return local[i] + offs[i / per];
}

// The block's own slice of the scan made whole into `out` (out[m]: the whole, from the last block); returns the whole.
__device__ __forceinline__ int scan_finish(const int* local, const int* offs, int* out, int m) {
    const int per = (m + gridDim.x - 1) / gridDim.x;
    const int lo = min(m, (int)blockIdx.x * per), hi = min(m, lo + per);
    const int offset = offs[blockIdx.x];
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) out[i] = local[i] + offset;
    const int whole = offs[gridDim.x];
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[m] = whole;
    return whole;
}

__device__ __forceinline__ int read_int(const int* p) { return *(const volatile int*)p; }

// The cluster's hardware barrier, with release and acquire at cluster scope: every block's writes before it
// (global memory included) are seen by every block after it.
__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// The barrier between passes: the block's own when the kernel is one block, the cluster's when its blocks form
// one cluster, else the bounded grid barrier.
#define SYNC()                                                    \
    do {                                                          \
        if (gridDim.x == 1) {                                     \
            __syncthreads();                                      \
        } else if (K.cluster) {                                   \
            cluster_sync();                                       \
        } else if (!grid_sync(K.bar, epoch)) {                    \
            return;                                               \
        }                                                         \
    } while (0)

__device__ __forceinline__ unsigned shared_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// One bulk copy (the TMA engine, no multicast) from global memory into this block's shared memory, counted on `bar`;
// both addresses 16-byte aligned, `bytes` a multiple of 16.
__device__ __forceinline__ void bulk_to_shared(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(shared_addr(dst)), "l"(src), "r"(bytes), "r"(shared_addr(bar))
                 : "memory");
}

// Waits for phase `parity` of `bar` to complete, at most limit_ns; false when the wait ran out.
__device__ __forceinline__ bool bar_wait(unsigned long long* bar, unsigned parity, unsigned long long limit_ns) {
    const unsigned long long start = global_ns();
    unsigned spins = 0;
    for (;;) {
        unsigned done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(shared_addr(bar)), "r"(parity)
                     : "memory");
        if (done) return true;
        if (((++spins & 255u) == 0u || spins == 1u) && global_ns() - start > limit_ns) return false;
    }
}

// Bytes of a block's staged copy for n spheres over `cells` cells: positions and displacements (whose .w is the
// inverse mass) as float4, then the sort's order and the cell starts, each padded to 16 bytes.
__host__ __device__ constexpr long staged_bytes(long n, long cells) {
    return 32 * n + 4 * ((n + 3) & ~3L) + 4 * ((cells + 1 + 3) & ~3L);
}

// A neighbour walk's reads (positions, inverse masses, the sort's order, the cell starts), copied into the block's
// shared memory by bulk copies after the barrier that ended their writes, and K reading them from there: a pass that
// writes none of them walks shared memory instead of making its chain of loads from L2. The same values in the same
// order, so the same results. Without staging (a scene too large for it), or once a copy's wait has run out (the
// status word then says so), K itself. Every thread of the block calls it, right after a barrier.
struct Stage {
    unsigned long long* bar;  // the copies' mbarrier
    int* broken;              // nonzero once a wait ran out: the walks read global memory from then on
    unsigned parity;          // the phase the next copies complete
};

__device__ __forceinline__ Kernel staged_kernel(const Kernel& K, float4* smem, Stage& st) {
    Kernel KS = K;
    if (!K.stage || *st.broken) return KS;
    const int n = K.n;
    float4* spos = smem;
    float4* sdisp = spos + n;
    int* sorder = reinterpret_cast<int*>(sdisp + n);
    int* sstart = sorder + ((n + 3) & ~3);
    const unsigned order_bulk = 4u * (unsigned)(n & ~3), start_bulk = 4u * (unsigned)((K.cells + 1) & ~3);
    if (threadIdx.x == 0) {
        // the sources' writes (ordered before by the barrier) and this block's reads of the old copy, before the
        // copy engine's accesses
        asm volatile("fence.proxy.async.global;\n\tfence.proxy.async.shared::cta;" ::: "memory");
        const unsigned bytes = 32u * (unsigned)n + order_bulk + start_bulk;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(shared_addr(st.bar)), "r"(bytes)
                     : "memory");
        bulk_to_shared(spos, K.s.pos, 16u * (unsigned)n, st.bar);
        bulk_to_shared(sdisp, K.s.disp, 16u * (unsigned)n, st.bar);
        if (order_bulk) bulk_to_shared(sorder, K.order, order_bulk, st.bar);
        if (start_bulk) bulk_to_shared(sstart, K.cell_start, start_bulk, st.bar);
    }
    for (int i = (n & ~3) + threadIdx.x; i < n; i += blockDim.x) sorder[i] = K.order[i];  // the ragged ends
    for (int i = ((K.cells + 1) & ~3) + threadIdx.x; i <= K.cells; i += blockDim.x) sstart[i] = K.cell_start[i];
    bool ok = bar_wait(st.bar, st.parity, K.bar.limit_ns);
    if (!ok) ok = bar_wait(st.bar, st.parity, K.bar.limit_ns);  // the copies in flight, once more
    st.parity ^= 1u;
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) {
            *st.broken = 1;
            atomicCAS(&K.counts->status, ST_OK, ST_TIMEOUT);
        }
        __syncthreads();
        return KS;
    }
    KS.s.pos = spos;
    KS.order = sorder;
    KS.cell_start = sstart;
    KS.weight = reinterpret_cast<const float*>(sdisp) + 3;  // sdisp[o].w
    KS.wstride = 4;
    return KS;
}

// `steps` whole steps (SphereStep's pass list :184-196; SphereStepper.step :66-103 when run until done).
__global__ void __launch_bounds__(THREADS) k_sphere_steps(Kernel K) {
    extern __shared__ float4 staged[];
    __shared__ unsigned long long stage_bar;
    __shared__ int stage_broken;
    Stage stage{&stage_bar, &stage_broken, 0u};
    if (K.stage) {
        if (threadIdx.x == 0) {
            stage_broken = 0;
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(shared_addr(&stage_bar)) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
    }
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gsize = gridDim.x * blockDim.x;
    // Spheres (and cells) are dealt out a warp's run of 32 at a time, in turn to each block, so that every block has
    // a share when there are fewer spheres than threads: a permutation of 0 .. gsize - 1, as gtid is.
    const int stid = ((threadIdx.x >> 5) * gridDim.x + blockIdx.x) * 32 + (threadIdx.x & 31);
    const int n = K.n;
    unsigned int epoch = 0;
    int cur = read_int(&K.counts->cur);
    const bool gs = K.solve != 0;
    const int limit = K.limit;
    // Without restitution the bounce pass changes nothing, so neither it nor the barriers around it are needed.
    const bool bouncing = K.p.w[RESTITUTION] > 0.0f;
    __shared__ int offs[SLICES_MOST + 1];
    for (int step = 0; step < K.steps; step++) {
        if (gtid == 0) {
            for (int k = 0; k < 4; k++) K.counts->last[k] = 0;
        }
        for (int sub = 0; sub < K.substeps; sub++) {
            // predict; the cell of each centre, counted; the walls' warm start; every claim cleared
            for (int s = stid; s < n; s += gsize) {
                if (sub > 0) bounced(K, s);
                predict(K, s);
                if (K.gridded) {
                    const float4 p = K.s.pos[s];
                    const int key = cell_key(K, p.x, p.y, p.z);
                    K.keys[s] = key;
                    atomicAdd(&K.cell_count[key], 1);
                }
                if (gs) {
                    warm_walls(K, s);
                    K.claims[s] = 0;
                    K.claims[n + s] = 0;
                    K.claims[2 * n + s] = 0;
                }
            }
            if (gs && gtid == 0) {
                Counts* c = K.counts;
                c->count[LONGEST] = max(c->count[LONGEST], c->count[LISTED]);
            }
            SYNC();
            if (K.gridded) {
                scan_slices(K, K.cell_count, K.scan_tmp, K.cells);
                SYNC();
                // the scan made whole, and in the same pass a place in its cell for each sphere (each block adds the
                // slice offsets itself); the counts return to zero for the next substep
                slice_offsets(K, offs);
                scan_finish(K.scan_tmp, offs, K.cell_start, K.cells);
                for (int s = stid; s < n; s += gsize) {
                    const int key = K.keys[s];
                    K.order[scan_value(K.scan_tmp, offs, key, K.cells) + atomicSub(&K.cell_count[key], 1) - 1] = s;
                }
                SYNC();
                // within a cell, ascending index: the stable counting sort's order
                for (int c = stid; c < K.cells; c += gsize) {
                    const int begin = K.cell_start[c], end = K.cell_start[c + 1];
                    for (int i = begin + 1; i < end; i++) {
                        const int v = K.order[i];
                        int j = i - 1;
                        while (j >= begin && K.order[j] > v) {
                            K.order[j + 1] = K.order[j];
                            j--;
                        }
                        K.order[j + 1] = v;
                    }
                }
                SYNC();
            }
            int listed = 0;
            if (gs) {
                // the walks of the count and the fill read the staged copy (positions change in neither)
                const Kernel KS = staged_kernel(K, staged, stage);
                for (int a = stid; a < n; a += gsize) K.list_count[a] = count_near(KS, a);
                SYNC();
                int* start = K.gen[cur ^ 1].start;  // the new list's
                scan_slices(K, K.list_count, K.scan_tmp, n);
                SYNC();
                slice_offsets(K, offs);
                {
                    const int whole = scan_finish(K.scan_tmp, offs, start, n);
                    if (gtid == 0) K.counts->count[LISTED] = whole;
                }
                cur ^= 1;
                const ListGen L = K.gen[cur], kept = K.gen[cur ^ 1];
                for (int a = stid; a < n; a += gsize) fill_near(KS, L, kept, a, scan_value(K.scan_tmp, offs, a, n));
                SYNC();
                listed = min(read_int(&K.counts->count[LISTED]), K.cap);
            }
            const ListGen L = K.gen[cur];
            HeldPlaces mine;
            mine.done = 0u;
#pragma unroll
            for (int j = 0; j < HELD_PLACES; j++) {
                const int c = gtid + j * gsize;
                mine.pair[j] = gs && c < listed ? L.pair[c] : make_int2(0, 0);
            }
            for (int it = 0; it < K.iterations; it++) {
                if (K.solve == 0) {
                    {
                        const Kernel KS = staged_kernel(K, staged, stage);
                        for (int s = stid; s < n; s += gsize) jacobi_solve(KS, s);
                    }
                    SYNC();
                    if (it == K.iterations - 1) {  // the last: each sphere's velocity right after its move
                        for (int s = stid; s < n; s += gsize) {
                            jacobi_apply(K, s);
                            velocity(K, s);
                        }
                    } else {
                        for (int s = stid; s < n; s += gsize) jacobi_apply(K, s);
                        SYNC();
                    }
                    continue;
                }
                if (K.solve == 2) {
                    // rounds 0..R on dispatches counted over the substep's passes (SphereStep.byContact :216-262)
                    mine.done = 0u;
                    for (int k = 0; k <= K.rounds; k++) {
                        const int g = it * (K.rounds + 1) + k;
                        contact_round(K, L, listed, k == 0 ? 0 : 1, k == K.rounds ? 0 : 1, it + 1, g, g % 2, g - 1,
                                      0, K.claims + ((g + 2) % 3) * n, K.claims + (g % 3) * n,
                                      K.claims + ((g + 1) % 3) * n, gtid, gsize, mine);
                        SYNC();
                    }
                    for (int s = stid; s < n; s += gsize) walls(K, s);
                    SYNC();
                    continue;
                }
                // until done: the opening batch, then BATCH more while the last round left a contact open
                int k = read_int(&K.opening[it]);
                int waits = 0;
                int from = 0;
                mine.done = 0u;
                for (;;) {
                    for (int j = from; j < k; j++) {
                        const int p = position(j);
                        contact_round(K, L, listed, p == 0 ? 0 : 1, 1, it + 1, it * CYCLE + p % CYCLE, p % 2,
                                      it * CYCLE + max(p - 1, 0) % CYCLE, 0, K.claims + ((p + 2) % 3) * n,
                                      K.claims + (p % 3) * n, K.claims + ((p + 1) % 3) * n, gtid, gsize, mine);
                        SYNC();
                    }
                    waits++;
                    const int open = read_int(&K.counts->open[position(k - 1) % 2]);
                    SYNC();
                    if (open == 0) break;
                    if (k > limit) {
                        if (gtid == 0) {
                            K.counts->rounds_at = k;
                            atomicCAS(&K.counts->status, ST_OK, ST_ROUNDS);
                        }
                        return;
                    }
                    from = k;
                    k += BATCH;
                }
                if (K.friction) {
                    // the same dispatches again, rubbing (SphereStep.rubs :271-278)
                    mine.done = 0u;
                    for (int j = 0; j < k; j++) {
                        const int p = position(j);
                        contact_round(K, L, listed, p == 0 ? 0 : 1, 1, K.iterations + it + 1,
                                      it * CYCLE + p % CYCLE, p % 2, it * CYCLE + max(p - 1, 0) % CYCLE, 1,
                                      K.claims + ((p + 2) % 3) * n, K.claims + (p % 3) * n,
                                      K.claims + ((p + 1) % 3) * n, gtid, gsize, mine);
                        SYNC();
                    }
                }
                for (int s = stid; s < n; s += gsize) walls(K, s);
                if (gtid == 0) {
                    Counts* c = K.counts;
                    const int unlisted = max(0, c->count[LISTED] - K.cap);
                    c->last[0] += waits;
                    c->last[1] += k;
                    c->last[2] = max(c->last[2], k);
                    c->last[3] += unlisted;
                    c->total[0] += waits;
                    c->total[1] += k;
                    c->total[2] = max(c->total[2], (long long)k);
                    c->total[3] += unlisted;
                    // SphereStepper.adapt :118-126
                    if (k > K.opening[it]) {
                        K.opening[it] = min(k, CYCLE);
                        K.enough[it] = 0;
                    } else if (++K.enough[it] >= SHRINK_AFTER && K.opening[it] > BATCH) {
                        K.opening[it] -= BATCH;
                        K.enough[it] = 0;
                    }
                }
                SYNC();
            }
            if (K.solve != 0)
                for (int s = stid; s < n; s += gsize) velocity(K, s);
            if (bouncing) {  // bounce reads the neighbours' velocities
                SYNC();
                for (int s = stid; s < n; s += gsize) bounce(K, s);
                SYNC();
            } else if (sub == K.substeps - 1) {
                SYNC();  // the picture reads the neighbours' positions
            }
        }
        // the last substep's restitution added, then the picture's buffer (its walk reads the staged copy: neither
        // pass moves a sphere)
        {
            const Kernel KS = staged_kernel(K, staged, stage);
            for (int s = stid; s < n; s += gsize) {
                bounced(K, s);
                show(KS, s);
            }
        }
        SYNC();
    }
    if (gtid == 0) K.counts->cur = cur;
}

// SphereDiagnostics.of (core/sphere/SphereDiagnostics.java:34-83) on the device: each sphere's deepest overlap with
// the spheres of its neighbourhood (the grid's 27 cells as the last substep sorted them; every sphere without a grid),
// over the smaller radius; how far it reaches past a wall, over its radius; energies, momenta and the fastest speed,
// summed in doubles.
struct SDiag {
    double kinetic, rotational, potential, momentum[3], angular[3];
    unsigned max_overlap, max_wall, max_speed;
    int broken;
};

__global__ void k_sphere_diag(Kernel K, SDiag* d) {
    const State& S = K.s;
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    float overlap = 0.0f, wall = 0.0f, speed = 0.0f;
    int broken = 0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < K.n; s += gridDim.x * blockDim.x) {
        const float4 p = S.pos[s], v = S.vel[s], w = S.spin[s];
        const float im = S.disp[s].w, r = p.w;
        const float f[9] = {p.x, p.y, p.z, v.x, v.y, v.z, w.x, w.y, w.z};
        for (int k = 0; k < 9; k++)
            if (!isfinite(f[k])) broken = 1;
        around(K, s, [&](int o, float4 q) {
            if (!(o > s)) return;
            const double dx = (double)p.x - q.x, dy = (double)p.y - q.y, dz = (double)p.z - q.z;
            const double depth = (double)(r + q.w) - sqrt(dx * dx + dy * dy + dz * dz);
            overlap = fmaxf(overlap, (float)(depth / fmin((double)r, (double)q.w)));
        });
        const float at[3] = {p.x, p.y, p.z};
        for (int a = 0; a < 3; a++)
            wall = fmaxf(wall, fmaxf((r - at[a]) / r, ((at[a] + r) - K.p.w[SX + a]) / r));
        const double vv = (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z;
        speed = fmaxf(speed, (float)sqrt(vv));
        if (!(im > 0.0f)) continue;
        const double m = 1.0 / (double)im;
        const double inertia = 0.4 * m * r * r;
        const double spin2 = (double)w.x * w.x + (double)w.y * w.y + (double)w.z * w.z;
        acc[0] += 0.5 * m * vv + 0.5 * inertia * spin2;
        acc[1] += 0.5 * inertia * spin2;
        acc[2] += m * -(double)K.p.w[GY] * p.y;
        acc[3] += m * v.x;
        acc[4] += m * v.y;
        acc[5] += m * v.z;
        acc[6] += m * ((double)p.y * v.z - (double)p.z * v.y) + inertia * w.x;
        acc[7] += m * ((double)p.z * v.x - (double)p.x * v.z) + inertia * w.y;
        acc[8] += m * ((double)p.x * v.y - (double)p.y * v.x) + inertia * w.z;
    }
    for (int k = 0; k < 9; k++)
        for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&d->kinetic, acc[0]);
        atomicAdd(&d->rotational, acc[1]);
        atomicAdd(&d->potential, acc[2]);
        for (int k = 0; k < 3; k++) {
            atomicAdd(&d->momentum[k], acc[3 + k]);
            atomicAdd(&d->angular[k], acc[6 + k]);
        }
    }
    atomicMax(&d->max_overlap, __float_as_uint(fmaxf(overlap, 0.0f)));
    atomicMax(&d->max_wall, __float_as_uint(fmaxf(wall, 0.0f)));
    atomicMax(&d->max_speed, __float_as_uint(speed));
    if (broken) atomicExch(&d->broken, 1);
}

}  // namespace sph
}  // namespace vxr

using namespace vxr;
using namespace vxr::sph;

struct vxr_sphere_world {
    int n = 0, substeps = 1, iterations = 1, solve = 0, rounds = 32, cap = 0;
    int gridded = 0, nx = 1, ny = 1, nz = 1, cells = 1;
    float cell = 1.0f;
    int device = 0, sms = 148, blocks = 1, friction = 1, cluster = 0;
    cudaStream_t stream = nullptr;
    SParams params{};
    std::string error;
    State s{};
    float4* wall = nullptr;
    float* shown = nullptr;
    int *keys = nullptr, *order = nullptr, *cell_count = nullptr, *cell_start = nullptr;
    int* part = nullptr;  // [blocks] the blocks' slice totals of a shared scan
    int* scan_tmp = nullptr;  // [max(cells, n) + 1] the slice-local prefixes of a shared scan
    int stage_bytes = 0;      // each block's shared memory for a staged walk (0: the walks read global memory)
    int *claims = nullptr, *list_count = nullptr, *near = nullptr;
    ListGen gen[2]{};
    Counts* counts = nullptr;
    Counts* host_counts = nullptr;  // pinned
    int *opening = nullptr, *enough = nullptr;
    float* pinned = nullptr;
    float* state9 = nullptr;  // [9 n] the state split into fields, for vxr_sphere_state
    size_t pinned_bytes = 0;
    std::vector<void*> allocations;
    long long launches = 0;
    int pending = 0;  // a call of steps is in flight
    int round_limit = 0;  // rounds a pass may take; 0: the reference's, the list's capacity + 2 cycles
};

namespace {

int sfail(vxr_sphere_world* w, int code, const std::string& why) {
    if (w) w->error = why;
    return code;
}

#define SPH_CUDA(call)                                                                           \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) return sfail(w, VXR_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
int salloc(vxr_sphere_world* w, T** p, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return sfail(w, VXR_ECUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    w->allocations.push_back(q);
    *p = (T*)q;
    return VXR_OK;
}

int32_t f32bits(double v) {
    const float f = (float)v;
    int32_t b;
    std::memcpy(&b, &f, 4);
    return b;
}

float* staging(vxr_sphere_world* w, size_t bytes) {
    if (w->pinned_bytes < bytes) {
        if (w->pinned) cudaFreeHost(w->pinned);
        w->pinned = nullptr;
        w->pinned_bytes = 0;
        if (cudaMallocHost(&w->pinned, bytes) != cudaSuccess) return nullptr;
        w->pinned_bytes = bytes;
    }
    return w->pinned;
}

// The 24 fields of the reference (Spheres.SPHERE :240-241) as (array, component) of the float4 layout.
struct FieldAt {
    int array;  // 0 pos 1 disp 2 turn 3 vel 4 spin 5 q 6 cvel
    int comp;
};
const FieldAt FIELD_AT[24] = {{0, 0}, {0, 1}, {0, 2}, {3, 0}, {3, 1}, {3, 2}, {0, 3}, {1, 3},
                              {6, 0}, {6, 1}, {6, 2}, {1, 0}, {1, 1}, {1, 2}, {4, 0}, {4, 1},
                              {4, 2}, {2, 0}, {2, 1}, {2, 2}, {5, 0}, {5, 1}, {5, 2}, {5, 3}};

float4* array_of(vxr_sphere_world* w, int k) {
    float4* arrays[7] = {w->s.pos, w->s.disp, w->s.turn, w->s.vel, w->s.spin, w->s.q, w->s.cvel};
    return arrays[k];
}

// Writes the fields given (null: zero; qw: one), every other buffer cleared, as the reference's runner.clear()
// and constants leave them (SphereSimulation.start, gui/SphereSimulation.java:154-178).
int write_state(vxr_sphere_world* w, const float* const* fields24, const float* shown) {
    const int n = w->n;
    const size_t bytes = sizeof(float4) * (size_t)n * 7;
    float4* host = (float4*)staging(w, bytes);
    if (!host) return sfail(w, VXR_ECUDA, "pinned staging");
    std::memset(host, 0, bytes);
    for (int s = 0; s < n; s++) host[5 * (size_t)n + s].w = 1.0f;  // qw
    for (int f = 0; f < 24; f++) {
        if (!fields24 || !fields24[f]) continue;
        const FieldAt at = FIELD_AT[f];
        float* base = (float*)(host + (size_t)at.array * n);
        for (int s = 0; s < n; s++) base[4 * (size_t)s + at.comp] = fields24[f][s];
    }
    cudaStream_t st = w->stream;
    for (int a = 0; a < 7; a++)
        SPH_CUDA(cudaMemcpyAsync(array_of(w, a), host + (size_t)a * n, sizeof(float4) * n, cudaMemcpyHostToDevice, st));
    SPH_CUDA(cudaStreamSynchronize(st));
    SPH_CUDA(cudaMemsetAsync(w->wall, 0, sizeof(float4) * 6 * (size_t)n, st));
    if (shown)
        SPH_CUDA(cudaMemcpyAsync(w->shown, shown, sizeof(float) * SHOWN * (size_t)n, cudaMemcpyHostToDevice, st));
    else
        SPH_CUDA(cudaMemsetAsync(w->shown, 0, sizeof(float) * SHOWN * (size_t)n, st));
    SPH_CUDA(cudaMemsetAsync(w->claims, 0, sizeof(int) * 3 * (size_t)n, st));
    if (w->gridded) SPH_CUDA(cudaMemsetAsync(w->cell_count, 0, sizeof(int) * (size_t)w->cells, st));
    if (w->solve != 0) {
        for (int g = 0; g < 2; g++) {
            SPH_CUDA(cudaMemsetAsync(w->gen[g].head, 0xFF, sizeof(int) * (size_t)n, st));
            SPH_CUDA(cudaMemsetAsync(w->gen[g].start, 0, sizeof(int) * ((size_t)n + 1), st));
            SPH_CUDA(cudaMemsetAsync(w->gen[g].done, 0, sizeof(int) * (size_t)w->cap, st));
        }
    }
    SPH_CUDA(cudaMemsetAsync(w->counts, 0, sizeof(Counts), st));
    SPH_CUDA(cudaStreamSynchronize(st));
    return VXR_OK;
}

Kernel kernel_of(vxr_sphere_world* w, int steps) {
    Kernel K;
    K.n = w->n;
    K.cap = w->cap;
    K.substeps = w->substeps;
    K.iterations = w->iterations;
    K.solve = w->solve;
    K.rounds = w->rounds;
    K.gridded = w->gridded;
    K.nx = w->nx;
    K.ny = w->ny;
    K.nz = w->nz;
    K.cells = w->cells;
    K.friction = w->friction;
    K.steps = steps;
    K.cluster = w->cluster;
    K.limit = w->round_limit > 0 ? w->round_limit : w->cap + 2 * CYCLE;
    K.cell = w->cell;
    K.p = w->params;
    K.s = w->s;
    K.wall = w->wall;
    K.shown = w->shown;
    K.keys = w->keys;
    K.order = w->order;
    K.cell_count = w->cell_count;
    K.cell_start = w->cell_start;
    K.claims = w->claims;
    K.list_count = w->list_count;
    K.near = w->near;
    K.part = w->part;
    K.scan_tmp = w->scan_tmp;
    K.weight = reinterpret_cast<const float*>(w->s.disp) + 3;  // disp[o].w
    K.wstride = 4;
    K.stage = w->stage_bytes > 0;
    K.gen[0] = w->gen[0];
    K.gen[1] = w->gen[1];
    K.counts = w->counts;
    K.opening = w->opening;
    K.enough = w->enough;
    K.bar.count = &w->counts->bar_count;
    K.bar.generation = &w->counts->bar_gen;
    K.bar.abort = &w->counts->abort;
    K.bar.status = &w->counts->status;
    K.bar.limit_ns = 2000000000ull;  // 2 s: far above any barrier's honest wait
    return K;
}

int launch_steps(vxr_sphere_world* w, int steps) {
    Kernel K = kernel_of(w, steps);
    cudaStream_t st = w->stream;
    // the barrier's counter, the status and the call's totals start at zero; the list, its counts and the
    // generation carry over
    SPH_CUDA(cudaMemsetAsync(&w->counts->total, 0, sizeof(long long) * 4, st));
    SPH_CUDA(cudaMemsetAsync(&w->counts->status, 0, sizeof(int) * 4, st));
    void* args[] = {&K};
    cudaError_t e;
    if (w->blocks == 1) {
        e = cudaLaunchKernel((const void*)k_sphere_steps, dim3(1), dim3(THREADS), args, w->stage_bytes, st);
    } else if (w->cluster) {  // every block in one cluster: co-scheduled by the hardware, the cluster barrier between
        cudaLaunchConfig_t c = {};
        c.gridDim = dim3(w->blocks);
        c.blockDim = dim3(THREADS);
        c.dynamicSmemBytes = w->stage_bytes;
        c.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = w->blocks;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        c.attrs = attr;
        c.numAttrs = 1;
        e = cudaLaunchKernelExC(&c, (const void*)k_sphere_steps, args);
    } else {
        e = cudaLaunchCooperativeKernel((const void*)k_sphere_steps, dim3(w->blocks), dim3(THREADS), args,
                                        w->stage_bytes, st);
    }
    if (e != cudaSuccess) return sfail(w, VXR_ECUDA, std::string("sphere step launch: ") + cudaGetErrorString(e));
    w->launches++;
    SPH_CUDA(cudaMemcpyAsync(w->host_counts, w->counts, sizeof(Counts), cudaMemcpyDeviceToHost, st));
    w->pending = 1;
    return VXR_OK;
}

int finish(vxr_sphere_world* w, vxr_sphere_report* report) {
    if (!w->pending) {
        if (report) std::memset(report, 0, sizeof(*report));
        return VXR_OK;
    }
    w->pending = 0;
    SPH_CUDA(cudaStreamSynchronize(w->stream));
    const Counts& c = *w->host_counts;
    if (report) {
        report->waits = c.last[0];
        report->rounds = c.last[1];
        report->most_rounds = c.last[2];
        report->unlisted = c.last[3];
        report->waits_total = c.total[0];
        report->rounds_total = c.total[1];
        report->most_rounds_total = (int32_t)c.total[2];
        report->unlisted_total = c.total[3];
        report->status = c.status;
        report->listed = c.count[LISTED];
    }
    if (c.status == ST_ROUNDS)
        return sfail(w, VXR_EROUNDS, "a pass is still open after " + std::to_string(c.rounds_at) +
                                         " rounds, on a list of " + std::to_string(c.count[LISTED]));
    if (c.status == ST_TIMEOUT)
        return sfail(w, VXR_ETIMEOUT,
                     "a device wait ran out (a grid barrier's, or a staged copy's); the step stopped or walked global "
                     "memory from then on");
    if (c.status != ST_OK) return sfail(w, VXR_ECUDA, "device status " + std::to_string(c.status));
    return VXR_OK;
}

}  // namespace

extern "C" {

int32_t vxr_sphere_make_params(double h, double gx, double gy, double gz, double sx, double sy, double sz,
                               double omega, int32_t averaged, double restitution, double mu_static,
                               double mu_kinetic, double mu_rolling, int32_t* out) {
    if (!out) return VXR_EINVAL;
    for (double mu : {mu_static, mu_kinetic, mu_rolling})
        if (!(mu >= 0) || std::isinf(mu)) return VXR_EINVAL;
    if (!(restitution >= 0) || !(restitution <= 1)) return VXR_EINVAL;
    if (!(h > 0) || !(sx > 0) || !(sy > 0) || !(sz > 0) || !(omega > 0) || !(omega <= 1)) return VXR_EINVAL;
    const double v[13] = {h, gx, gy, gz, sx, sy, sz, omega, averaged ? 1.0 : 0.0, restitution, mu_static,
                          mu_kinetic, mu_rolling};
    for (int k = 0; k < 13; k++) out[k] = f32bits(v[k]);
    return VXR_OK;
}

int32_t vxr_sphere_make_grid(double sx, double sy, double sz, double widest, vxr_grid* out) {
    if (!out || !(widest > 0)) return VXR_EINVAL;
    out->nx = std::max(1, (int)std::ceil(sx / widest));
    out->ny = std::max(1, (int)std::ceil(sy / widest));
    out->nz = std::max(1, (int)std::ceil(sz / widest));
    out->cell = (float)widest;
    return VXR_OK;
}

void vxr_sphere_destroy(vxr_sphere_world* w) {
    if (!w) return;
    if (w->stream) cudaStreamSynchronize(w->stream);
    for (void* p : w->allocations) cudaFree(p);
    if (w->pinned) cudaFreeHost(w->pinned);
    if (w->host_counts) cudaFreeHost(w->host_counts);
    if (w->stream) cudaStreamDestroy(w->stream);
    delete w;
}

vxr_sphere_world* vxr_sphere_create(const vxr_sphere_config* cfg, int32_t* status) {
    auto set = [&](int32_t s) {
        if (status) *status = s;
    };
    if (!cfg || cfg->spheres < 1 || cfg->substeps < 1 || cfg->iterations < 1 || cfg->solve < 0 || cfg->solve > 2) {
        set(VXR_EINVAL);
        return nullptr;
    }
    const bool gridded = cfg->grid.nx > 0 && cfg->grid.ny > 0 && cfg->grid.nz > 0 && cfg->grid.cell > 0;
    const int per = cfg->contacts_per_sphere > 0 ? cfg->contacts_per_sphere : 6;
    // Gauss-Seidel needs the grid and orders at most MOST_LISTED_SPHERES (SphereStep.java:115-131)
    if ((cfg->solve != 0 && !gridded) || (cfg->solve != 0 && cfg->spheres > VXR_MOST_LISTED_SPHERES) ||
        (cfg->solve == 2 && cfg->rounds < 1) || (long)cfg->spheres * per > (1L << 30)) {
        set(VXR_EINVAL);
        return nullptr;
    }
    vxr_sphere_world* w = new vxr_sphere_world();
    w->n = cfg->spheres;
    w->substeps = cfg->substeps;
    w->iterations = cfg->iterations;
    w->solve = cfg->solve;
    w->rounds = cfg->solve == 2 ? cfg->rounds : 0;
    w->cap = w->n * per;
    w->device = cfg->device;
    w->gridded = gridded ? 1 : 0;
    if (gridded) {
        const long cells = (long)cfg->grid.nx * cfg->grid.ny * cfg->grid.nz;
        if (cells > (1L << 28)) {
            set(VXR_EINVAL);
            delete w;
            return nullptr;
        }
        w->nx = cfg->grid.nx;
        w->ny = cfg->grid.ny;
        w->nz = cfg->grid.nz;
        w->cell = cfg->grid.cell;
        w->cells = (int)cells;
    }
    auto bad = [&](int rc) {
        set(rc);
        vxr_sphere_destroy(w);
        return (vxr_sphere_world*)nullptr;
    };
    if (cudaSetDevice(w->device) != cudaSuccess) return bad(VXR_ECUDA);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, w->device) != cudaSuccess) return bad(VXR_ECUDA);
    w->sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking) != cudaSuccess) return bad(VXR_ECUDA);
    const int n = w->n;
    int rc = 0;
    rc |= salloc(w, &w->s.pos, n);
    rc |= salloc(w, &w->s.disp, n);
    rc |= salloc(w, &w->s.turn, n);
    rc |= salloc(w, &w->s.vel, n);
    rc |= salloc(w, &w->s.spin, n);
    rc |= salloc(w, &w->s.q, n);
    rc |= salloc(w, &w->s.cvel, n);
    rc |= salloc(w, &w->wall, 6 * (size_t)n);
    rc |= salloc(w, &w->shown, SHOWN * (size_t)n);
    rc |= salloc(w, &w->claims, 3 * (size_t)n);
    rc |= salloc(w, &w->counts, 1);
    rc |= salloc(w, &w->opening, w->iterations);
    rc |= salloc(w, &w->enough, w->iterations);
    if (gridded) {
        rc |= salloc(w, &w->keys, n);
        rc |= salloc(w, &w->order, n);
        rc |= salloc(w, &w->cell_count, w->cells);
        rc |= salloc(w, &w->cell_start, (size_t)w->cells + 1);
    }
    if (w->solve != 0) {
        rc |= salloc(w, &w->list_count, n);
        rc |= salloc(w, &w->near, (size_t)n * NEAR_KEPT);
        for (int g = 0; g < 2; g++) {
            rc |= salloc(w, &w->gen[g].start, (size_t)n + 1);
            rc |= salloc(w, &w->gen[g].pair, w->cap);
            rc |= salloc(w, &w->gen[g].done, w->cap);
            rc |= salloc(w, &w->gen[g].next, w->cap);
            rc |= salloc(w, &w->gen[g].imp, 2 * (size_t)w->cap);
            rc |= salloc(w, &w->gen[g].head, n);
        }
    }
    if (rc) return bad(VXR_ECUDA);
    if (cudaMallocHost(&w->host_counts, sizeof(Counts)) != cudaSuccess) return bad(VXR_ECUDA);
    // A staged walk's copy (positions, displacements, the sort's order, cell starts) where one block's shared
    // memory holds it: the 4,096-sphere pile takes 180 KB.
    if (w->gridded) {
        const size_t bytes = (size_t)staged_bytes(n, w->cells);
        if (bytes <= (size_t)STAGE_MOST &&
            cudaFuncSetAttribute(k_sphere_steps, cudaFuncAttributeMaxDynamicSharedMemorySize, STAGE_MOST) ==
                cudaSuccess)
            w->stage_bytes = (int)bytes;
        else
            cudaGetLastError();
    }
    // One block while the scene is small enough that a block's barrier beats a grid's; otherwise every SM.
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sphere_steps, THREADS, w->stage_bytes);
    const int most = std::max(1, per_sm) * w->sms;
    const long work = std::max<long>(n, w->solve != 0 ? 3L * n : n);
    int blocks = cfg->blocks > 0 ? cfg->blocks : (n <= VXR_SPHERE_ONE_BLOCK ? 1 : (int)((work + THREADS - 1) / THREADS));
    w->blocks = std::max(1, std::min(blocks, most));
    // By default a scene of VXR_SPHERE_CLUSTER_FROM spheres or more (that one block would run alone) runs on a
    // cluster of VXR_SPHERE_CLUSTER blocks: measured on the 1,024-sphere lattice at rest, 5.0 ms a step against
    // 9.4 ms on one block; 12 and 16 blocks gain nothing more.
    // From VXR_SPHERE_CLUSTER_WIDE_FROM spheres, VXR_SPHERE_CLUSTER_WIDE blocks: on the reference's 4,096-sphere
    // pile, 3.28 ms a step against 4.05 on 8 (Gauss-Seidel until done, friction on).
    // A cluster asked for by the caller must fit, or the world is refused; one chosen here falls back to 8 blocks,
    // then to one block, where the GPU cannot place it (shared under MPS, or with fewer SMs free). vxr_sphere_blocks
    // tells which was taken.
    auto cluster_fits = [&](int size) {
        if (size > 16) return false;
        if (size > 8 &&
            cudaFuncSetAttribute(k_sphere_steps, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        cudaLaunchConfig_t c = {};
        c.gridDim = dim3(size);
        c.blockDim = dim3(THREADS);
        c.dynamicSmemBytes = w->stage_bytes;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = size;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        c.attrs = attr;
        c.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, (const void*)k_sphere_steps, &c) != cudaSuccess || clusters < 1) {
            cudaGetLastError();
            return false;
        }
        return true;
    };
    int cluster = cfg->cluster;
    if (cluster > 1) {  // asked for: one thread-block cluster of `cluster` blocks (at most 16, one a SM)
        if (!cluster_fits(cluster)) return bad(VXR_EINVAL);
    } else if (cluster == 0 && cfg->blocks == 0 && n >= VXR_SPHERE_CLUSTER_FROM && n <= VXR_SPHERE_ONE_BLOCK) {
        cluster = n >= VXR_SPHERE_CLUSTER_WIDE_FROM ? VXR_SPHERE_CLUSTER_WIDE : VXR_SPHERE_CLUSTER;
        if (!cluster_fits(cluster)) cluster = cluster > VXR_SPHERE_CLUSTER && cluster_fits(VXR_SPHERE_CLUSTER)
                                                  ? VXR_SPHERE_CLUSTER : 1;
    }
    if (cluster > 1) {
        w->blocks = cluster;
        w->cluster = 1;
    }
    if (w->blocks > SLICES_MOST) return bad(VXR_EINVAL);
    if (salloc(w, &w->part, (size_t)std::max(w->blocks, 1)) != VXR_OK) return bad(VXR_ECUDA);
    if (salloc(w, &w->scan_tmp, (size_t)std::max(w->cells, n) + 1) != VXR_OK) return bad(VXR_ECUDA);
    // the stepper's batch sizing starts at BATCH a pass (SphereStepper.java:59-64)
    std::vector<int> batch(w->iterations, BATCH);
    if (cudaMemcpy(w->opening, batch.data(), sizeof(int) * w->iterations, cudaMemcpyHostToDevice) != cudaSuccess)
        return bad(VXR_ECUDA);
    if (cudaMemset(w->enough, 0, sizeof(int) * w->iterations) != cudaSuccess) return bad(VXR_ECUDA);
    if (write_state(w, nullptr, nullptr) != VXR_OK) return bad(VXR_ECUDA);
    set(VXR_OK);
    return w;
}

const char* vxr_sphere_error(const vxr_sphere_world* w) { return w ? w->error.c_str() : "no world"; }

static int rubs_of(const int32_t* params) {
    float f[13];
    std::memcpy(f, params, sizeof(f));
    return (f[MU_STATIC] + f[MU_KINETIC]) + f[MU_ROLLING] > 0.0f ? 1 : 0;
}

// Whether every value of the given host arrays (null ones skipped) is finite.
static bool finite_fields(const float* const* fields, int count, int n) {
    for (int k = 0; k < count; k++)
        if (fields[k])
            for (int s = 0; s < n; s++)
                if (!std::isfinite(fields[k][s])) return false;
    return true;
}

int32_t vxr_sphere_start(vxr_sphere_world* w, const float* x, const float* y, const float* z, const float* u,
                         const float* v, const float* wv, const float* r, const float* im, const int32_t* params) {
    if (!w || !x || !y || !z || !u || !v || !wv || !r || !im || !params) return sfail(w, VXR_EINVAL, "null argument");
    {
        const float* given[8] = {x, y, z, u, v, wv, r, im};
        if (!finite_fields(given, 8, w->n))
            return sfail(w, VXR_ENONFINITE, "a non-finite value in the state: nothing was loaded");
    }
    if (w->pending) finish(w, nullptr);
    const float* fields[24] = {x, y, z, u, v, wv, r, im};
    std::vector<float> shown((size_t)w->n * SHOWN, 0.0f);
    for (int s = 0; s < w->n; s++) {
        float* b = shown.data() + (size_t)s * SHOWN;
        b[0] = b[4] = x[s];
        b[1] = b[5] = y[s];
        b[2] = b[6] = z[s];
        b[3] = r[s];
        b[TURNED_BEFORE + 3] = b[TURNED_AFTER + 3] = 1.0f;
    }
    std::memcpy(w->params.w, params, sizeof(float) * P_COUNT);
    w->friction = rubs_of(params);
    return write_state(w, fields, shown.data());
}

int32_t vxr_sphere_load_state(vxr_sphere_world* w, const float* const* fields24, const int32_t* params) {
    if (!w || !fields24 || !params) return sfail(w, VXR_EINVAL, "null argument");
    if (!finite_fields(fields24, 24, w->n))
        return sfail(w, VXR_ENONFINITE, "a non-finite value in the state: nothing was loaded");
    if (w->pending) finish(w, nullptr);
    std::memcpy(w->params.w, params, sizeof(float) * P_COUNT);
    w->friction = rubs_of(params);
    return write_state(w, fields24, nullptr);
}

int32_t vxr_sphere_params(vxr_sphere_world* w, const int32_t* params) {
    if (!w || !params) return sfail(w, VXR_EINVAL, "null argument");
    std::memcpy(w->params.w, params, sizeof(float) * P_COUNT);
    w->friction = rubs_of(params);
    return VXR_OK;
}

int32_t vxr_sphere_round_limit(vxr_sphere_world* w, int32_t rounds) {
    if (!w || rounds < 0) return sfail(w, VXR_EINVAL, "a round limit is at least 0");
    w->round_limit = rounds;
    return VXR_OK;
}

int32_t vxr_sphere_friction(vxr_sphere_world* w, int32_t on) {
    if (!w) return VXR_EINVAL;
    w->friction = on ? 1 : 0;
    return VXR_OK;
}

int32_t vxr_sphere_step_async(vxr_sphere_world* w, int32_t steps) {
    if (!w || steps < 0) return sfail(w, VXR_EINVAL, "steps must be at least 0");
    if (w->pending) {
        const int rc = finish(w, nullptr);
        if (rc != VXR_OK) return rc;
    }
    if (steps == 0) return VXR_OK;
    if (cudaSetDevice(w->device) != cudaSuccess) return sfail(w, VXR_ECUDA, "cudaSetDevice");
    return launch_steps(w, steps);
}

int32_t vxr_sphere_sync(vxr_sphere_world* w, vxr_sphere_report* report) {
    if (!w) return VXR_EINVAL;
    return finish(w, report);
}

int32_t vxr_sphere_step(vxr_sphere_world* w, int32_t steps, vxr_sphere_report* report) {
    const int rc = vxr_sphere_step_async(w, steps);
    if (rc != VXR_OK) return rc;
    return finish(w, report);
}

void* vxr_sphere_stream(vxr_sphere_world* w) { return w ? (void*)w->stream : nullptr; }

// x y z u v w ax ay az, field after field.
__global__ void k_state9(int n, const float4* __restrict__ pos, const float4* __restrict__ vel,
                         const float4* __restrict__ spin, float* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 p = pos[s], v = vel[s], a = spin[s];
    const float f[9] = {p.x, p.y, p.z, v.x, v.y, v.z, a.x, a.y, a.z};
#pragma unroll
    for (int k = 0; k < 9; k++) out[(size_t)k * n + s] = f[k];
}

int32_t vxr_sphere_field(vxr_sphere_world* w, int32_t field, float* out) {
    if (!w || !out || field < 0 || field >= 24) return sfail(w, VXR_EINVAL, "field is 0 to 23");
    if (w->pending) {
        const int rc = finish(w, nullptr);
        if (rc != VXR_OK) return rc;
    }
    const FieldAt at = FIELD_AT[field];
    const int n = w->n;
    float4* host = (float4*)staging(w, sizeof(float4) * n);
    if (!host) return sfail(w, VXR_ECUDA, "pinned staging");
    SPH_CUDA(cudaMemcpyAsync(host, array_of(w, at.array), sizeof(float4) * n, cudaMemcpyDeviceToHost, w->stream));
    SPH_CUDA(cudaStreamSynchronize(w->stream));
    const float* f = (const float*)host;
    for (int s = 0; s < n; s++) out[s] = f[4 * (size_t)s + at.comp];
    return VXR_OK;
}

int32_t vxr_sphere_state(vxr_sphere_world* w, float* const* out9) {
    if (!w || !out9) return sfail(w, VXR_EINVAL, "null argument");
    if (w->pending) {
        const int rc = finish(w, nullptr);
        if (rc != VXR_OK) return rc;
    }
    // the 9 fields split out of the float4 arrays on the device, then copied straight into the caller's arrays
    // (at the copy engine's full rate when they are pinned), one synchronisation for all
    const int n = w->n;
    if (!w->state9 && salloc(w, &w->state9, (size_t)9 * n) != VXR_OK) return VXR_ECUDA;
    k_state9<<<(n + 255) / 256, 256, 0, w->stream>>>(n, w->s.pos, w->s.vel, w->s.spin, w->state9);  // not a step's
    for (int k = 0; k < 9; k++)
        if (out9[k])
            SPH_CUDA(cudaMemcpyAsync(out9[k], w->state9 + (size_t)k * n, sizeof(float) * (size_t)n,
                                     cudaMemcpyDeviceToHost, w->stream));
    SPH_CUDA(cudaStreamSynchronize(w->stream));
    return VXR_OK;
}

int32_t vxr_sphere_read_shown(vxr_sphere_world* w, float* out) {
    if (!w || !out) return sfail(w, VXR_EINVAL, "null argument");
    if (w->pending) {
        const int rc = finish(w, nullptr);
        if (rc != VXR_OK) return rc;
    }
    SPH_CUDA(cudaMemcpy(out, w->shown, sizeof(float) * SHOWN * (size_t)w->n, cudaMemcpyDeviceToHost));
    return VXR_OK;
}

int32_t vxr_sphere_contacts(vxr_sphere_world* w, int32_t* ab, int32_t* done, float* impulses, int32_t capacity,
                            int32_t* listed) {
    if (!w || !listed) return sfail(w, VXR_EINVAL, "null argument");
    if (w->pending) {
        const int rc = finish(w, nullptr);
        if (rc != VXR_OK) return rc;
    }
    Counts c;
    SPH_CUDA(cudaMemcpy(&c, w->counts, sizeof(Counts), cudaMemcpyDeviceToHost));
    const int k = w->solve == 0 ? 0 : std::min(c.count[LISTED], w->cap);
    *listed = k;
    const int m = std::min(k, std::max(0, capacity));
    if (m == 0) return VXR_OK;
    const ListGen& L = w->gen[c.cur];
    if (ab) SPH_CUDA(cudaMemcpy(ab, L.pair, sizeof(int2) * m, cudaMemcpyDeviceToHost));
    if (done) SPH_CUDA(cudaMemcpy(done, L.done, sizeof(int) * m, cudaMemcpyDeviceToHost));
    if (impulses) {
        std::vector<float4> tmp(2 * (size_t)m);
        SPH_CUDA(cudaMemcpy(tmp.data(), L.imp, sizeof(float4) * 2 * m, cudaMemcpyDeviceToHost));
        for (int i = 0; i < m; i++) {
            const float4 a = tmp[2 * i], b = tmp[2 * i + 1];
            float* o = impulses + 7 * (size_t)i;
            o[0] = a.x, o[1] = a.y, o[2] = a.z, o[3] = a.w, o[4] = b.x, o[5] = b.y, o[6] = b.z;
        }
    }
    return VXR_OK;
}

int32_t vxr_sphere_walls(vxr_sphere_world* w, float* out) {
    if (!w || !out) return sfail(w, VXR_EINVAL, "null argument");
    if (w->pending) {
        const int rc = finish(w, nullptr);
        if (rc != VXR_OK) return rc;
    }
    std::vector<float4> tmp(6 * (size_t)w->n);
    SPH_CUDA(cudaMemcpy(tmp.data(), w->wall, sizeof(float4) * tmp.size(), cudaMemcpyDeviceToHost));
    for (int s = 0; s < w->n; s++)
        for (int a = 0; a < 3; a++) {
            const float4 p = tmp[6 * (size_t)s + 2 * a], q = tmp[6 * (size_t)s + 2 * a + 1];
            float* o = out + 21 * (size_t)s + 7 * a;
            o[0] = p.x, o[1] = p.y, o[2] = p.z, o[3] = p.w, o[4] = q.x, o[5] = q.y, o[6] = q.z;
        }
    return VXR_OK;
}

int32_t vxr_sphere_counts(vxr_sphere_world* w, int32_t* out3) {
    if (!w || !out3) return sfail(w, VXR_EINVAL, "null argument");
    if (w->pending) {
        const int rc = finish(w, nullptr);
        if (rc != VXR_OK) return rc;
    }
    Counts c;
    SPH_CUDA(cudaMemcpy(&c, w->counts, sizeof(Counts), cudaMemcpyDeviceToHost));
    for (int k = 0; k < 3; k++) out3[k] = c.count[k];
    return VXR_OK;
}

int32_t vxr_sphere_blocks(const vxr_sphere_world* w) { return w ? w->blocks : 0; }

const float* vxr_sphere_shown_device(vxr_sphere_world* w, int64_t* words) {
    if (!w) return nullptr;
    if (w->pending) finish(w, nullptr);
    if (words) *words = (int64_t)w->n * SHOWN;
    return w->shown;
}

int32_t vxr_sphere_diagnostics(vxr_sphere_world* w, vxr_sphere_diag* out) {
    if (!w || !out) return sfail(w, VXR_EINVAL, "null argument");
    if (w->pending) {
        const int rc = finish(w, nullptr);
        if (rc != VXR_OK) return rc;
    }
    const Kernel K = kernel_of(w, 0);
    SDiag* d = nullptr;
    SPH_CUDA(cudaMallocAsync(&d, sizeof(SDiag), w->stream));
    SPH_CUDA(cudaMemsetAsync(d, 0, sizeof(SDiag), w->stream));
    k_sphere_diag<<<std::max(1, std::min((w->n + 255) / 256, 4 * w->sms)), 256, 0, w->stream>>>(K, d);
    SPH_CUDA(cudaGetLastError());
    SDiag h;
    SPH_CUDA(cudaMemcpyAsync(&h, d, sizeof(SDiag), cudaMemcpyDeviceToHost, w->stream));
    SPH_CUDA(cudaFreeAsync(d, w->stream));
    SPH_CUDA(cudaStreamSynchronize(w->stream));
    out->kinetic = h.kinetic;
    out->rotational = h.rotational;
    out->potential = h.potential;
    for (int k = 0; k < 3; k++) {
        out->momentum[k] = h.momentum[k];
        out->angular[k] = h.angular[k];
    }
    float f;
    std::memcpy(&f, &h.max_overlap, 4);
    out->max_overlap = f;
    std::memcpy(&f, &h.max_wall, 4);
    out->max_wall = f;
    std::memcpy(&f, &h.max_speed, 4);
    out->max_speed = f;
    out->broken = h.broken;
    out->pad = 0;
    return VXR_OK;
}

int64_t vxr_sphere_launches(const vxr_sphere_world* w) { return w ? w->launches : 0; }

}  // extern "C"
