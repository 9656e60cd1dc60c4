// CPU ORACLE — test infrastructure only, never part of the product path.
//
// A single-precision C++ restatement of the reference's box/mixed-body step (package
// dev.vexelray.sim.rigid.box of sibarum/vexelray-sim-rigid), one function per IR kernel, with the
// reference's own buffer layout (32 partner slots per body, 40-word manifolds, 28-word impulse records,
// 48/144/144 wall words per body) and its pass order. Every float expression keeps the reference's
// association order; build with -ffp-contract=off so no multiply-add is fused.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library.
//
// Files restated (paths inside the reference project):
//   core = vexelray-sim-rigid-core/src/main/java/dev/vexelray/sim/rigid/
//   core/box/Boxes.java       velocities :276-289, positions :299-342, walls :357-416, Soft :421-450,
//                             contact :462-542, roll :553-600, Moving :660-773, show :801-820,
//                             inverseInertia :854-871, turned :877-899, rotate :907-921
//   core/box/BoxContact.java  collide :136-246, sphereContact :267-329, nearest :336-385, Solid :390-422,
//                             Edge :427-500, Face :505-817
//   core/box/BoxPairs.java    solve :64-151, keep :164-182, carry :191-267
//   core/box/BoxBroad.java    bin :74-89, list :103-164, counts :174-188, reach :196-227, around :230-252
//   core/box/BoxStep.java     pass order :235-267
//   core/box/BoxStepper.java  greedy colouring :324-368
//
// The counting sort the reference calls (SupirVast CountingSort, dev.supirvast:vastir 0.2.3-SNAPSHOT, not
// vendored) is restated as a STABLE counting sort: within a cell, bodies in ascending index. The reference's
// own within-cell order is unpinned; the box path's results do not depend on it unless a body overflows
// its 32 slots.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#ifdef _OPENMP
#include <omp.h>
#define ORC_PARALLEL_FOR _Pragma("omp parallel for schedule(dynamic, 256)")
#else
#define ORC_PARALLEL_FOR
#endif

namespace {

// --- constants (Boxes.java :101-147, BoxContact.java :85-123, BoxPairs.java :48-50,158, BoxBroad :60) ---
enum {
    H = 0, GX, GY, GZ, SX, SY, SZ, MU_STATIC, MU_KINETIC, MARGIN, BIAS, MASS_SCALE, IMPULSE_SCALE,
    STATIC_BIAS, STATIC_MASS_SCALE, STATIC_IMPULSE_SCALE, PUSH_SPEED, MU_ROLLING, PARAM_COUNT
};
constexpr int CORNERS = 8, WALLS = 6, LAMBDA_WORDS = 48, RUB_WORDS = 144, ROLL_WORDS = 144;
constexpr int MANIFOLD_WORDS = 40, NORMAL = 0, COUNT = 3, AXIS = 4, POINTS = 8, POINT_WORDS = 8;
constexpr int ANCHOR_FIRST = 0, ANCHOR_SECOND = 3, DEPTH = 6, MOST_POINTS = 4;
constexpr int CANDIDATES = 24, CANDIDATE_WORDS = 4, SCRATCH_WORDS = CANDIDATES * CANDIDATE_WORDS;
constexpr float RELATIVE = 0.98f, ABSOLUTE = 0.01f, PARALLEL = 1e-10f, SAME = 1e-12f, SLACK = 1e-5f,
                OFF_LINE = 1e-4f;
constexpr int SPHERE_BOX = 15, SPHERE_SPHERE = 16;
constexpr int IMPULSE_WORDS = MOST_POINTS * 7, POINT_IMPULSE = 7;
constexpr float SAME_POINT = 0.05f;
constexpr int SLOTS = 32, MOST_ROUNDS = 32;
constexpr int SHOWN_STRIDE = 20, CENTRE_BEFORE = 0, CENTRE_AFTER = 4, SHAPE_AT = 3, HALF_AT = 8,
              TURNED_BEFORE = 12, TURNED_AFTER = 16;
enum Sweep { WARM = 0, SOLVE = 1, RELAX = 2 };

// --- vector building blocks, in the reference's association order -------------------------------------
inline float dot3(const float* a, const float* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }
inline void cross3(const float* x, const float* y, float* o) {
    float c0 = x[1] * y[2] - x[2] * y[1];
    float c1 = x[2] * y[0] - x[0] * y[2];
    float c2 = x[0] * y[1] - x[1] * y[0];
    o[0] = c0; o[1] = c1; o[2] = c2;
}
// Boxes.rotate :907-921: p + w t + q × t, t = 2 q × p / |q|².
inline void rotate(const float* q, const float* p, float* out) {
    float twice = 2.0f / ((q[0] * q[0] + q[1] * q[1]) + (q[2] * q[2] + q[3] * q[3]));
    float t[3];
    cross3(q, p, t);
    for (int a = 0; a < 3; a++) t[a] = twice * t[a];
    float qt[3];
    cross3(q, t, qt);
    float o[3];
    for (int a = 0; a < 3; a++) o[a] = p[a] + (q[3] * t[a] + qt[a]);
    out[0] = o[0]; out[1] = o[1]; out[2] = o[2];
}
inline void conjugate(const float* q, float* c) { c[0] = -q[0]; c[1] = -q[1]; c[2] = -q[2]; c[3] = q[3]; }
inline float fmaxj(float a, float b) { return std::fmax(a, b); }
inline float fminj(float a, float b) { return std::fmin(a, b); }
// BoxContact.sign :879-883: 1 where x is at least zero, -1 where it is less.
inline float signOf(float x) { return x < 0.0f ? -1.0f : 1.0f; }

// Boxes.turned :877-899.
inline void turned(const float* q, const float* omega, float dt, float* now) {
    float a[3];
    for (int k = 0; k < 3; k++) a[k] = (0.5f * dt) * omega[k];
    float r[4];
    for (int k = 0; k < 3; k++) {
        int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
        r[k] = q[k] + (a[k] * q[3] + (a[k1] * q[k2] - a[k2] * q[k1]));
    }
    r[3] = q[3] - (a[0] * q[0] + (a[1] * q[1] + a[2] * q[2]));
    float len2 = (r[0] * r[0] + r[1] * r[1]) + (r[2] * r[2] + r[3] * r[3]);
    float inverse = 1.0f / std::sqrt(fmaxj(len2, 1e-30f));
    for (int k = 0; k < 4; k++) now[k] = r[k] * inverse;
}

struct World;

// Boxes.inverseInertia :854-871.
inline void inverseInertia(float hx, float hy, float hz, float shape, float im, float* inverse) {
    float h2[3] = {hx * hx, hy * hy, hz * hz};
    for (int a = 0; a < 3; a++) inverse[a] = (3.0f * im) / (h2[(a + 1) % 3] + h2[(a + 2) % 3]);
    if (shape > 0.5f) {
        for (int a = 0; a < 3; a++) inverse[a] = im / (0.4f * h2[0]);
    }
}

// Boxes.Moving :660-773: a body as a velocity solve holds it, loaded once, stored once.
struct Moving {
    int s;
    float shape, im;
    float at[3], q[4], half[3], inverse[3], velocity[3], momentum[3], omega[3];

    void inverseInertiaTimes(const float* x, float* out) const {
        float c[4], own[3], scaled[3];
        conjugate(q, c);
        rotate(c, x, own);
        for (int a = 0; a < 3; a++) scaled[a] = inverse[a] * own[a];
        rotate(q, scaled, out);
    }
    bool isSphere() const { return shape > 0.5f; }
    float inverseMassAlong(const float* r, const float* n) const {
        float rn[3], t[3];
        cross3(r, n, rn);
        inverseInertiaTimes(rn, t);
        return im + dot3(rn, t);
    }
    void pointVelocity(const float* r, float* out) const {
        float turning[3];
        cross3(omega, r, turning);
        for (int a = 0; a < 3; a++) out[a] = velocity[a] + turning[a];
    }
    void apply(const float* r, const float* p) {
        for (int a = 0; a < 3; a++) velocity[a] = velocity[a] + im * p[a];
        float angular[3], turn[3];
        cross3(r, p, angular);
        inverseInertiaTimes(angular, turn);
        for (int a = 0; a < 3; a++) {
            momentum[a] = momentum[a] + angular[a];
            omega[a] = omega[a] + turn[a];
        }
    }
    void turn(const float* j) {
        float spin[3];
        inverseInertiaTimes(j, spin);
        for (int a = 0; a < 3; a++) {
            momentum[a] = momentum[a] + j[a];
            omega[a] = omega[a] + spin[a];
        }
    }
};

// Boxes.Soft :421-450.
struct Soft {
    float h, margin, bias, massScale, impulseScale, push, muStatic, muKinetic;
    Soft(const float* params, bool fixed) {
        h = params[H];
        margin = params[MARGIN];
        bias = params[fixed ? STATIC_BIAS : BIAS];
        massScale = params[fixed ? STATIC_MASS_SCALE : MASS_SCALE];
        impulseScale = params[fixed ? STATIC_IMPULSE_SCALE : IMPULSE_SCALE];
        push = params[PUSH_SPEED];
        muStatic = params[MU_STATIC];
        muKinetic = params[MU_KINETIC];
    }
    void stiffen(bool fixed, const float* params) {
        if (fixed) {
            bias = params[STATIC_BIAS];
            massScale = params[STATIC_MASS_SCALE];
            impulseScale = params[STATIC_IMPULSE_SCALE];
        }
    }
};

// Boxes.relative :615-626.
inline void relative(const Moving* first, const float* rA, const Moving& second, const float* rB, float* out) {
    float vb[3];
    second.pointVelocity(rB, vb);
    if (!first) { out[0] = vb[0]; out[1] = vb[1]; out[2] = vb[2]; return; }
    float va[3];
    first->pointVelocity(rA, va);
    for (int a = 0; a < 3; a++) out[a] = vb[a] - va[a];
}
inline float inverseMassAlong(const Moving* first, const float* rA, const Moving& second, const float* rB,
                              const float* n) {
    float k = second.inverseMassAlong(rB, n);
    return first ? k + first->inverseMassAlong(rA, n) : k;
}
inline void applyPair(Moving* first, const float* rA, Moving& second, const float* rB, const float* p) {
    second.apply(rB, p);
    if (first) {
        float back[3] = {-p[0], -p[1], -p[2]};
        first->apply(rA, back);
    }
}
inline void applyAngular(Moving* first, Moving& second, const float* j) {
    second.turn(j);
    if (first) {
        float back[3] = {-j[0], -j[1], -j[2]};
        first->turn(back);
    }
}

// Boxes.contact :462-542.
void contact(Sweep sweep, float gap, const float* n, Moving* first, const float* rA, Moving& second,
             const float* rB, float* normals, long normalAt, float* tangents, long tangentAt, const Soft& soft) {
    float normal = normals[normalAt];
    float tangent[3] = {tangents[tangentAt], tangents[tangentAt + 1], tangents[tangentAt + 2]};
    bool holding = normal > 0.0f || dot3(tangent, tangent) > 0.0f;
    if (sweep == WARM) {
        if (holding) {
            float p[3];
            for (int a = 0; a < 3; a++) p[a] = normal * n[a] + tangent[a];
            applyPair(first, rA, second, rB, p);
        }
        return;
    }
    if (!(gap < soft.margin || holding)) return;
    float k = inverseMassAlong(first, rA, second, rB, n);
    float rel[3];
    relative(first, rA, second, rB, rel);
    float closing = dot3(rel, n);
    float bias = 0.0f, massScale = 1.0f, impulseScale = 0.0f;
    if (gap > 0.0f) bias = gap / soft.h;
    if (sweep == SOLVE && !(gap > 0.0f)) {
        bias = fmaxj(soft.bias * gap, -soft.push);
        massScale = soft.massScale;
        impulseScale = soft.impulseScale;
    }
    float change = -((massScale / k) * (closing + bias)) - impulseScale * normal;
    float total = fmaxj(0.0f, normal + change);
    normals[normalAt] = total;
    float p[3];
    for (int a = 0; a < 3; a++) p[a] = (total - normal) * n[a];
    applyPair(first, rA, second, rB, p);

    float sliding[3];
    relative(first, rA, second, rB, sliding);
    float along = dot3(sliding, n);
    for (int a = 0; a < 3; a++) sliding[a] = sliding[a] - along * n[a];
    float whole[3] = {tangent[0], tangent[1], tangent[2]};
    float speed = std::sqrt(dot3(sliding, sliding));
    if (speed > 1e-12f) {
        float t[3];
        for (int a = 0; a < 3; a++) t[a] = sliding[a] / speed;
        float kt = inverseMassAlong(first, rA, second, rB, t);
        float stop = speed / kt;
        for (int a = 0; a < 3; a++) whole[a] = whole[a] - stop * t[a];
    }
    float size = std::sqrt(dot3(whole, whole));
    if (size > soft.muStatic * total) {
        float cut = (soft.muKinetic * total) / size;
        for (int a = 0; a < 3; a++) whole[a] = whole[a] * cut;
    }
    float rubbed[3];
    for (int a = 0; a < 3; a++) {
        tangents[tangentAt + a] = whole[a];
        rubbed[a] = whole[a] - tangent[a];
    }
    applyPair(first, rA, second, rB, rubbed);
}

// Boxes.roll :553-600.
void roll(Sweep sweep, Moving* first, Moving& second, float radius, const float* normals, long normalAt,
          float* rolls, long rollAt, const float* params) {
    float old[3] = {rolls[rollAt], rolls[rollAt + 1], rolls[rollAt + 2]};
    if (sweep == WARM) {
        applyAngular(first, second, old);
        return;
    }
    float muRolling = params[MU_ROLLING];
    float whole[3], turning[3];
    for (int a = 0; a < 3; a++) {
        whole[a] = old[a];
        float against = first ? first->omega[a] : 0.0f;
        turning[a] = second.omega[a] - against;
    }
    float speed = std::sqrt(dot3(turning, turning));
    if (speed > 1e-12f && muRolling > 0.0f) {
        float t[3];
        for (int a = 0; a < 3; a++) t[a] = turning[a] / speed;
        float it[3];
        second.inverseInertiaTimes(t, it);
        float k = dot3(t, it);
        if (first) {
            float jt[3];
            first->inverseInertiaTimes(t, jt);
            k = k + dot3(t, jt);
        }
        float stop = speed / k;
        for (int a = 0; a < 3; a++) whole[a] = whole[a] - stop * t[a];
    }
    float most = (muRolling * radius) * fmaxj(0.0f, normals[normalAt]);
    float size = std::sqrt(dot3(whole, whole));
    if (size > most) {
        float scale = most / size;
        for (int a = 0; a < 3; a++) whole[a] = whole[a] * scale;
    }
    float change[3];
    for (int a = 0; a < 3; a++) {
        rolls[rollAt + a] = whole[a];
        change[a] = whole[a] - old[a];
    }
    applyAngular(first, second, change);
}

// ------------------------------------------------------------------------------------------------------
// The world: the reference's buffers (BoxStep.java :81-162).
struct World {
    int n, substeps, sweeps, symmetric;
    int nx, ny, nz;
    float cell;
    int reach_cells = 1;  // neighbourhood half-width in cells: 1 is the reference's 27 cells
    int slots, width;
    std::vector<float> f[18];  // x y z u v w lx ly lz qx qy qz qw im hx hy hz shape
    float params[PARAM_COUNT];
    std::vector<float> lambda, rub, rollw, shown;
    std::vector<int> keys, order, starts;
    std::vector<int> pairs, pairsWas, contacts, rounds;
    std::vector<float> manifold, manifoldWas, impulses, impulsesWas;
    // the last step's report: touching, points, rounds, unplaced, unlisted
    int report[5];
};
enum { FX = 0, FY, FZ, FU, FV, FW, FLX, FLY, FLZ, FQX, FQY, FQZ, FQW, FIM, FHX, FHY, FHZ, FSHAPE };

Moving load(const World& w, int s, float im) {
    Moving m;
    m.s = s;
    m.im = im;
    m.shape = w.f[FSHAPE][s];
    for (int a = 0; a < 3; a++) {
        m.at[a] = w.f[FX + a][s];
        m.half[a] = w.f[FHX + a][s];
        m.velocity[a] = w.f[FU + a][s];
        m.momentum[a] = w.f[FLX + a][s];
    }
    for (int k = 0; k < 4; k++) m.q[k] = w.f[FQX + k][s];
    inverseInertia(w.f[FHX][s], w.f[FHY][s], w.f[FHZ][s], w.f[FSHAPE][s], im, m.inverse);
    m.inverseInertiaTimes(m.momentum, m.omega);
    return m;
}
void store(World& w, const Moving& m) {
    for (int a = 0; a < 3; a++) {
        w.f[FU + a][m.s] = m.velocity[a];
        w.f[FLX + a][m.s] = m.momentum[a];
    }
}

// Boxes.velocities :276-289.
void velocities(World& w) {
    const float* p = w.params;
    ORC_PARALLEL_FOR
    for (int s = 0; s < w.n; s++) {
        if (!(w.f[FIM][s] > 0.0f)) continue;
        float h = p[H];
        for (int a = 0; a < 3; a++) w.f[FU + a][s] = w.f[FU + a][s] + h * p[GX + a];
    }
}

// Boxes.positions :299-342.
void positions(World& w) {
    const float* p = w.params;
    ORC_PARALLEL_FOR
    for (int s = 0; s < w.n; s++) {
        float im = w.f[FIM][s];
        if (!(im > 0.0f)) continue;
        float h = p[H];
        for (int a = 0; a < 3; a++) w.f[FX + a][s] = w.f[FX + a][s] + h * w.f[FU + a][s];
        float q[4], momentum[3], inverse[3];
        for (int k = 0; k < 4; k++) q[k] = w.f[FQX + k][s];
        for (int a = 0; a < 3; a++) momentum[a] = w.f[FLX + a][s];
        inverseInertia(w.f[FHX][s], w.f[FHY][s], w.f[FHZ][s], w.f[FSHAPE][s], im, inverse);
        auto omegaAt = [&](const float* turn, float* out) {
            float c[4], own[3], scaled[3];
            conjugate(turn, c);
            rotate(c, momentum, own);
            for (int a = 0; a < 3; a++) scaled[a] = inverse[a] * own[a];
            rotate(turn, scaled, out);
        };
        float omega[3];
        omegaAt(q, omega);
        float halfH = 0.5f * h;
        float mid[4];
        turned(q, omega, halfH, mid);
        float omegaMid[3];
        omegaAt(mid, omegaMid);
        float end[4];
        turned(q, omegaMid, h, end);
        for (int k = 0; k < 4; k++) w.f[FQX + k][s] = end[k];
    }
}

// Boxes.walls :357-416.
void walls(World& w, Sweep sweep, bool reverse) {
    const float* params = w.params;
    ORC_PARALLEL_FOR
    for (int s = 0; s < w.n; s++) {
        float im = w.f[FIM][s];
        if (!(im > 0.0f)) continue;
        Moving box = load(w, s, im);
        Soft soft(params, true);
        long base = (long)s * LAMBDA_WORDS;
        float extent[3] = {params[SX], params[SY], params[SZ]};
        for (int order = 0; order < WALLS; order++) {
            int wall = reverse ? WALLS - 1 - order : order;
            int axis = wall / 2;
            bool high = wall % 2 == 1;
            int firstSlot = wall * CORNERS;
            float n[3];
            for (int a = 0; a < 3; a++) n[a] = a == axis ? (high ? -1.0f : 1.0f) : 0.0f;
            if (box.isSphere()) {
                float r[3];
                for (int a = 0; a < 3; a++) r[a] = -(box.half[0] * n[a]);
                long at = base + firstSlot;
                long tangentAt = at * 3;
                float reach = box.at[axis] + r[axis];
                float gap = high ? extent[axis] - reach : reach;
                contact(sweep, gap, n, nullptr, nullptr, box, r, w.lambda.data(), at, w.rub.data(), tangentAt, soft);
                roll(sweep, nullptr, box, box.half[0], w.lambda.data(), at, w.rollw.data(), tangentAt, params);
            } else {
                for (int k = 0; k < CORNERS; k++) {
                    int c = reverse ? CORNERS - 1 - k : k;
                    float offset[3], r[3];
                    for (int a = 0; a < 3; a++) {
                        int bit = (c / (1 << a)) % 2;
                        offset[a] = box.half[a] * (2.0f * (float)bit - 1.0f);
                    }
                    rotate(box.q, offset, r);
                    long at = base + firstSlot + c;
                    long tangentAt = at * 3;
                    float reach = box.at[axis] + r[axis];
                    float gap = high ? extent[axis] - reach : reach;
                    contact(sweep, gap, n, nullptr, nullptr, box, r, w.lambda.data(), at, w.rub.data(), tangentAt,
                            soft);
                }
            }
        }
        store(w, box);
    }
}

// Boxes.show :801-820.
void show(World& w) {
    for (int s = 0; s < w.n; s++) {
        long base = (long)s * SHOWN_STRIDE;
        float* sh = w.shown.data();
        for (int a = 0; a < 3; a++) {
            sh[base + CENTRE_BEFORE + a] = sh[base + CENTRE_AFTER + a];
            sh[base + CENTRE_AFTER + a] = w.f[FX + a][s];
            sh[base + HALF_AT + a] = w.f[FHX + a][s];
        }
        for (int k = 0; k < 4; k++) {
            sh[base + TURNED_BEFORE + k] = sh[base + TURNED_AFTER + k];
            sh[base + TURNED_AFTER + k] = w.f[FQX + k][s];
        }
        sh[base + SHAPE_AT] = w.f[FSHAPE][s];
    }
}

// ------------------------------------------------------------------------------------------------------
// The narrow phase (BoxContact.java).

struct Solid {  // BoxContact.Solid :390-422
    float centre[3], axes[3][3], half[3];
    void loadFrom(const float* const* f, int s) {
        for (int a = 0; a < 3; a++) {
            centre[a] = f[FX + a][s];
            half[a] = f[FHX + a][s];
        }
        float x = f[FQX][s], y = f[FQY][s], z = f[FQZ][s], w = f[FQW][s];
        axes[0][0] = 1.0f - 2.0f * (y * y + z * z);
        axes[0][1] = 2.0f * (x * y + z * w);
        axes[0][2] = 2.0f * (x * z - y * w);
        axes[1][0] = 2.0f * (x * y - z * w);
        axes[1][1] = 1.0f - 2.0f * (x * x + z * z);
        axes[1][2] = 2.0f * (y * z + x * w);
        axes[2][0] = 2.0f * (x * z + y * w);
        axes[2][1] = 2.0f * (y * z - x * w);
        axes[2][2] = 1.0f - 2.0f * (x * x + y * y);
    }
    void own(const float* point, float* out) const {
        float off[3] = {point[0] - centre[0], point[1] - centre[1], point[2] - centre[2]};
        float o0 = dot3(off, axes[0]), o1 = dot3(off, axes[1]), o2 = dot3(off, axes[2]);
        out[0] = o0; out[1] = o1; out[2] = o2;
    }
};

inline void writeNormal(float* m, const float* normal, float axis) {
    for (int x = 0; x < 3; x++) m[NORMAL + x] = normal[x];
    m[AXIS] = axis;
}
inline void writePoint(float* m, int at, const float* onFirst, const float* onSecond, float depth) {
    for (int x = 0; x < 3; x++) {
        m[at + ANCHOR_FIRST + x] = onFirst[x];
        m[at + ANCHOR_SECOND + x] = onSecond[x];
    }
    m[at + DEPTH] = depth;
}

struct Edge {  // BoxContact.Edge :427-500
    float normal[3] = {0, 0, 0}, onFirst[3] = {0, 0, 0}, alongFirst[3] = {0, 0, 0};
    float halfFirst = 0, onSecond[3] = {0, 0, 0}, alongSecond[3] = {0, 0, 0}, halfSecond = 0, axis = 0;
    void record(const Solid& first, const Solid& second, int k, int j, const float* ax, const float* d) {
        float toward = 1.0f;
        if (dot3(d, ax) < 0.0f) toward = -1.0f;
        for (int a = 0; a < 3; a++) {
            normal[a] = ax[a] * toward;
            onFirst[a] = first.centre[a];
            onSecond[a] = second.centre[a];
            alongFirst[a] = first.axes[k][a];
            alongSecond[a] = second.axes[j][a];
        }
        for (int m = 0; m < 3; m++) {
            if (m != k) {
                float sign = signOf(dot3(first.axes[m], normal));
                for (int a = 0; a < 3; a++) onFirst[a] = onFirst[a] + (sign * first.half[m]) * first.axes[m][a];
            }
            if (m != j) {
                float sign = signOf(dot3(second.axes[m], normal));
                for (int a = 0; a < 3; a++) onSecond[a] = onSecond[a] - (sign * second.half[m]) * second.axes[m][a];
            }
        }
        halfFirst = first.half[k];
        halfSecond = second.half[j];
        axis = (float)(6 + 3 * k + j);
    }
    void contact(const Solid& first, const Solid& second, float bestEdge, float* m) const {
        float w[3] = {onFirst[0] - onSecond[0], onFirst[1] - onSecond[1], onFirst[2] - onSecond[2]};
        float cos = dot3(alongFirst, alongSecond);
        float dA = dot3(alongFirst, w);
        float dB = dot3(alongSecond, w);
        float den = 1.0f - cos * cos;
        float s = (cos * dB - dA) / den;
        float u = (dB - cos * dA) / den;
        s = fmaxj(-halfFirst, fminj(halfFirst, s));
        u = fmaxj(-halfSecond, fminj(halfSecond, u));
        float pointFirst[3], pointSecond[3];
        for (int a = 0; a < 3; a++) {
            pointFirst[a] = onFirst[a] + s * alongFirst[a];
            pointSecond[a] = onSecond[a] + u * alongSecond[a];
        }
        writeNormal(m, normal, axis);
        float of[3], os[3];
        first.own(pointFirst, of);
        second.own(pointSecond, os);
        writePoint(m, POINTS, of, os, -bestEdge);
    }
};

struct Face {  // BoxContact.Face :505-817
    const Solid* first;
    const Solid* second;
    float flip, margin;
    float refCentre[3], n[3], u[3], w[3], hn, hu, hw, axis;
    float face[3], a[3], c[3], ha, hc;
    float* cand;  // this pair's candidates scratch (CANDIDATES x 4 floats)

    Face(const Solid& firstBox, const Solid& secondBox, bool fromSecond, const float* bestFaceAxis, float mg,
         float* scratch)
        : first(&firstBox), second(&secondBox), margin(mg), cand(scratch) {
        flip = 1.0f;
        float k = bestFaceAxis[0];
        const Solid* ref = &firstBox;
        const Solid* inc = &secondBox;
        if (fromSecond) {
            flip = -1.0f;
            k = bestFaceAxis[1];
            ref = &secondBox;
            inc = &firstBox;
        }
        for (int e = 0; e < 3; e++) refCentre[e] = ref->centre[e];
        axis = k + 1.5f * (1.0f - flip);
        for (int e = 0; e < 3; e++) n[e] = u[e] = w[e] = 0.0f;
        hn = hu = hw = 0.0f;
        for (int kk = 0; kk < 3; kk++) {
            int ku = (kk + 1) % 3, kw = (kk + 2) % 3;
            if (k > (float)kk - 0.5f && k < (float)kk + 0.5f) {
                for (int e = 0; e < 3; e++) {
                    n[e] = ref->axes[kk][e];
                    u[e] = ref->axes[ku][e];
                    w[e] = ref->axes[kw][e];
                }
                hn = ref->half[kk];
                hu = ref->half[ku];
                hw = ref->half[kw];
            }
        }
        float apart[3] = {inc->centre[0] - refCentre[0], inc->centre[1] - refCentre[1], inc->centre[2] - refCentre[2]};
        if (dot3(apart, n) < 0.0f) {
            for (int e = 0; e < 3; e++) n[e] = -n[e];
        }
        float most = -1.0f, faceAxis[3] = {0, 0, 0}, hf = 0.0f;
        for (int e = 0; e < 3; e++) a[e] = c[e] = 0.0f;
        ha = hc = 0.0f;
        for (int m = 0; m < 3; m++) {
            int ma = (m + 1) % 3, mc = (m + 2) % 3;
            float tt = std::fabs(dot3(inc->axes[m], n));
            if (tt > most) {
                most = tt;
                for (int e = 0; e < 3; e++) {
                    faceAxis[e] = inc->axes[m][e];
                    a[e] = inc->axes[ma][e];
                    c[e] = inc->axes[mc][e];
                }
                hf = inc->half[m];
                ha = inc->half[ma];
                hc = inc->half[mc];
            }
        }
        float facing = signOf(dot3(faceAxis, n));
        for (int e = 0; e < 3; e++) face[e] = inc->centre[e] - (facing * hf) * faceAxis[e];
    }

    void keep(int& count, bool when, const float* point, float depth) {
        float deep = depth;
        if (when && deep > -margin && count < CANDIDATES) {
            float* at = cand + count * CANDIDATE_WORDS;
            at[0] = point[0]; at[1] = point[1]; at[2] = point[2]; at[3] = deep;
            count++;
        }
    }

    void emit(const float* at, int& count, float* m) const {
        float incident[3] = {at[0], at[1], at[2]};
        float deep = at[3];
        float onFirstIsRef = 0.5f * (flip + 1.0f);
        float pointFirst[3], pointSecond[3];
        for (int x = 0; x < 3; x++) {
            float lift = deep * n[x];
            pointFirst[x] = incident[x] + onFirstIsRef * lift;
            pointSecond[x] = incident[x] + (1.0f - onFirstIsRef) * lift;
        }
        float of[3], os[3];
        first->own(pointFirst, of);
        second->own(pointSecond, os);
        writePoint(m, POINTS + count * POINT_WORDS, of, os, deep);
        count++;
    }

    void reduce(int found, int& count, float* m) const {
        int deepest = 0;
        float most = -1e30f;
        for (int k = 0; k < found; k++) {
            float d = cand[k * 4 + 3];
            if (d > most) { most = d; deepest = k; }
        }
        const float* pa = cand + deepest * 4;
        int farthest = -1;
        float far = SAME;
        for (int k = 0; k < found; k++) {
            const float* q = cand + k * 4;
            float gap[3] = {q[0] - pa[0], q[1] - pa[1], q[2] - pa[2]};
            float d2 = dot3(gap, gap);
            if (d2 > far) { far = d2; farthest = k; }
        }
        emit(cand + deepest * 4, count, m);
        if (farthest > -1) {
            const float* pb = cand + farthest * 4;
            float ab[3] = {pb[0] - pa[0], pb[1] - pa[1], pb[2] - pa[2]};
            int left = -1, right = -1;
            float mostLeft = OFF_LINE * far;
            float mostRight = -mostLeft;
            for (int k = 0; k < found; k++) {
                const float* q = cand + k * 4;
                float aq[3] = {q[0] - pa[0], q[1] - pa[1], q[2] - pa[2]};
                float cr[3];
                cross3(ab, aq, cr);
                float area = dot3(cr, n);
                if (area > mostLeft) { mostLeft = area; left = k; }
                if (area < mostRight) { mostRight = area; right = k; }
            }
            emit(cand + farthest * 4, count, m);
            if (left > -1) emit(cand + left * 4, count, m);
            if (right > -1) emit(cand + right * 4, count, m);
        }
    }

    void contact(int& count, float* m) {
        const float signs[4][2] = {{1, 1}, {-1, 1}, {-1, -1}, {1, -1}};
        const float wide = 1.0f + SLACK;
        float corner[4][3], cu[4], cw[4], depth[4];
        for (int e = 0; e < 4; e++) {
            for (int x = 0; x < 3; x++)
                corner[e][x] = face[x] + ((signs[e][0] * ha) * a[x] + (signs[e][1] * hc) * c[x]);
            float rel[3] = {corner[e][0] - refCentre[0], corner[e][1] - refCentre[1], corner[e][2] - refCentre[2]};
            cu[e] = dot3(rel, u);
            cw[e] = dot3(rel, w);
            depth[e] = hn - dot3(rel, n);
            bool inside = std::fabs(cu[e]) < hu * wide && std::fabs(cw[e]) < hw * wide;
            keep(count, inside, corner[e], depth[e]);
        }
        for (int e = 0; e < 4; e++) {
            int next = (e + 1) % 4;
            for (int line = 0; line < 4; line++) {
                bool acrossU = line < 2;
                float side = line % 2 == 0 ? 1.0f : -1.0f;
                float from = acrossU ? cu[e] : cw[e];
                float to = acrossU ? cu[next] : cw[next];
                float alongFrom = acrossU ? cw[e] : cu[e];
                float alongTo = acrossU ? cw[next] : cu[next];
                float limit = acrossU ? hu : hw;
                float bound = acrossU ? hw : hu;
                float span = to - from;
                if (std::fabs(span) > SAME) {
                    float s = (side * limit - from) / span;
                    float along = alongFrom + s * (alongTo - alongFrom);
                    bool within = s > -SLACK && s < wide && std::fabs(along) < bound * wide;
                    float point[3];
                    for (int x = 0; x < 3; x++) point[x] = corner[e][x] + s * (corner[next][x] - corner[e][x]);
                    float deep = depth[e] + s * (depth[next] - depth[e]);
                    keep(count, within, point, deep);
                }
            }
        }
        float off[3] = {face[0] - refCentre[0], face[1] - refCentre[1], face[2] - refCentre[2]};
        float fu = dot3(off, u), fw = dot3(off, w);
        float au = ha * dot3(a, u), aw = ha * dot3(a, w);
        float bu = hc * dot3(c, u), bw = hc * dot3(c, w);
        float det = au * bw - aw * bu;
        if (std::fabs(det) > SAME) {
            for (int e = 0; e < 4; e++) {
                float ru = signs[e][0] * hu - fu;
                float rw = signs[e][1] * hw - fw;
                float alpha = (ru * bw - rw * bu) / det;
                float beta = (au * rw - aw * ru) / det;
                bool inside = std::fabs(alpha) < wide && std::fabs(beta) < wide;
                float point[3];
                for (int x = 0; x < 3; x++) point[x] = face[x] + ((alpha * ha) * a[x] + (beta * hc) * c[x]);
                float rel[3] = {point[0] - refCentre[0], point[1] - refCentre[1], point[2] - refCentre[2]};
                keep(count, inside, point, hn - dot3(rel, n));
            }
        }
        float normal[3] = {n[0] * flip, n[1] * flip, n[2] * flip};
        writeNormal(m, normal, axis);
        int found = count;
        count = 0;
        if (found > 0) reduce(found, count, m);
    }
};

// BoxContact.nearest :336-385.
float nearest(const Solid& box, const float* p, float* towards, float* surface) {
    float off[3] = {p[0] - box.centre[0], p[1] - box.centre[1], p[2] - box.centre[2]};
    float local[3], held[3], outside[3];
    for (int k = 0; k < 3; k++) {
        local[k] = dot3(off, box.axes[k]);
        held[k] = fmaxj(-box.half[k], fminj(box.half[k], local[k]));
    }
    for (int k = 0; k < 3; k++) outside[k] = local[k] - held[k];
    float away = std::sqrt(dot3(outside, outside));
    float reach = away;
    if (away > 1e-9f) {
        for (int a = 0; a < 3; a++) {
            float dir = 0.0f, at = box.centre[a];
            for (int k = 0; k < 3; k++) {
                dir = dir + outside[k] * box.axes[k][a];
                at = at + held[k] * box.axes[k][a];
            }
            towards[a] = dir / away;
            surface[a] = at;
        }
    } else {
        float least = 1e30f;
        for (int k = 0; k < 3; k++) {
            float inward = box.half[k] - std::fabs(local[k]);
            if (inward < least) {
                least = inward;
                float side = signOf(local[k]);
                for (int a = 0; a < 3; a++) {
                    towards[a] = side * box.axes[k][a];
                    float at = box.centre[a];
                    for (int j = 0; j < 3; j++) {
                        float along = j == k ? side * box.half[k] : local[j];
                        at = at + along * box.axes[j][a];
                    }
                    surface[a] = at;
                }
            }
        }
        reach = -least;
    }
    return reach;
}

// BoxContact.sphereContact :267-329.
void sphereContact(const Solid& first, const Solid& second, float shapeA, float shapeB, float margin, float* m) {
    float n[3] = {0, 0, 0}, onFirst[3] = {0, 0, 0}, onSecond[3] = {0, 0, 0};
    float depth = 0.0f, axis = (float)SPHERE_BOX;
    bool sphereA = shapeA > 0.5f, sphereB = shapeB > 0.5f;
    if (sphereA && sphereB) {
        float d[3] = {second.centre[0] - first.centre[0], second.centre[1] - first.centre[1],
                      second.centre[2] - first.centre[2]};
        float length = std::sqrt(dot3(d, d));
        n[1] = 1.0f;
        if (length > 1e-9f) {
            for (int a = 0; a < 3; a++) n[a] = d[a] / length;
        }
        depth = (first.half[0] + second.half[0]) - length;
        for (int a = 0; a < 3; a++) {
            onFirst[a] = first.centre[a] + first.half[0] * n[a];
            onSecond[a] = second.centre[a] - second.half[0] * n[a];
        }
        axis = (float)SPHERE_SPHERE;
    }
    for (int which = 0; which < 2; which++) {
        bool sphereFirst = which == 0;
        const Solid& round = sphereFirst ? first : second;
        const Solid& box = sphereFirst ? second : first;
        bool only = sphereFirst ? (sphereA && !sphereB) : (sphereB && !sphereA);
        if (!only) continue;
        float towards[3] = {0, 0, 0}, surface[3] = {0, 0, 0};
        float reach = nearest(box, round.centre, towards, surface);
        float radius = round.half[0];
        depth = radius - reach;
        for (int a = 0; a < 3; a++) {
            float onSphere = round.centre[a] - radius * towards[a];
            if (sphereFirst) {
                n[a] = -towards[a];
                onFirst[a] = onSphere;
                onSecond[a] = surface[a];
            } else {
                n[a] = towards[a];
                onFirst[a] = surface[a];
                onSecond[a] = onSphere;
            }
        }
    }
    writeNormal(m, n, axis);
    float kept = 0.0f;
    if (depth > -margin) {
        float of[3], os[3];
        first.own(onFirst, of);
        second.own(onSecond, os);
        writePoint(m, POINTS, of, os, depth);
        kept = 1.0f;
    }
    m[COUNT] = kept;
}

// BoxContact.collide :136-246, for one pair (ia, partner) into manifold m, with scratch cand.
void collideOne(const float* const* f, const float* params, int ia, int partner, float* m, float* cand) {
    m[COUNT] = 0.0f;
    if (partner < 0) return;
    Solid first, second;
    first.loadFrom(f, ia);
    second.loadFrom(f, partner);
    float shapeA = f[FSHAPE][ia], shapeB = f[FSHAPE][partner];
    float margin = params[MARGIN];
    float d[3] = {second.centre[0] - first.centre[0], second.centre[1] - first.centre[1],
                  second.centre[2] - first.centre[2]};
    float parted = -1e30f;
    float bestFace[2] = {-1e30f, -1e30f}, bestFaceAxis[2] = {0.0f, 0.0f};
    const Solid* boxes[2] = {&first, &second};
    for (int side = 0; side < 2; side++) {
        const Solid& own = *boxes[side];
        const Solid& other = *boxes[1 - side];
        for (int k = 0; k < 3; k++) {
            float reach = own.half[k];
            for (int j = 0; j < 3; j++) reach = reach + other.half[j] * std::fabs(dot3(own.axes[k], other.axes[j]));
            float sep = std::fabs(dot3(d, own.axes[k])) - reach;
            parted = fmaxj(parted, sep);
            if (sep > bestFace[side]) {
                bestFace[side] = sep;
                bestFaceAxis[side] = (float)k;
            }
        }
    }
    float bestEdge = -1e30f;
    Edge edge;
    for (int k = 0; k < 3; k++) {
        for (int j = 0; j < 3; j++) {
            float across[3];
            cross3(first.axes[k], second.axes[j], across);
            float length2 = dot3(across, across);
            if (length2 > PARALLEL) {
                float length = std::sqrt(length2);
                float inv = 1.0f / length;
                float ax[3] = {across[0] * inv, across[1] * inv, across[2] * inv};
                float reach = 0.0f;
                for (int mm = 0; mm < 3; mm++)
                    reach = reach + (first.half[mm] * std::fabs(dot3(first.axes[mm], ax)) +
                                     second.half[mm] * std::fabs(dot3(second.axes[mm], ax)));
                float sep = std::fabs(dot3(d, ax)) - reach;
                parted = fmaxj(parted, sep);
                if (sep > bestEdge) {
                    bestEdge = sep;
                    edge.record(first, second, k, j, ax, d);
                }
            }
        }
    }
    float smallest = first.half[0];
    for (int b = 0; b < 2; b++)
        for (int k = 0; k < 3; k++) smallest = fminj(smallest, boxes[b]->half[k]);
    float slack = ABSOLUTE * smallest;
    bool fromSecond = bestFace[1] > RELATIVE * bestFace[0] + slack;
    float faceSep = fromSecond ? bestFace[1] : bestFace[0];
    bool byEdge = bestEdge > RELATIVE * faceSep + slack;
    int count = 0;
    bool touching = !(parted > margin);
    if (touching) {
        if (byEdge) {
            edge.contact(first, second, bestEdge, m);
            count = 1;
        } else {
            Face face(first, second, fromSecond, bestFaceAxis, margin, cand);
            face.contact(count, m);
        }
    }
    m[COUNT] = (float)count;
    if (shapeA > 0.5f || shapeB > 0.5f) sphereContact(first, second, shapeA, shapeB, margin, m);
}

const float* const* fields(const World& w, const float** buf) {
    for (int k = 0; k < 18; k++) buf[k] = w.f[k].data();
    return buf;
}

// ------------------------------------------------------------------------------------------------------
// The broad phase (BoxBroad.java).

// BoxBroad.reach :196-227: the body's half-extents in the world's frame, R_ak from q.
void reachOf(const World& w, int s, float* out) {
    float x = w.f[FQX][s], y = w.f[FQY][s], z = w.f[FQZ][s], ww = w.f[FQW][s];
    float r[3][3] = {{1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y - z * ww), 2.0f * (x * z + y * ww)},
                     {2.0f * (x * y + z * ww), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z - x * ww)},
                     {2.0f * (x * z - y * ww), 2.0f * (y * z + x * ww), 1.0f - 2.0f * (x * x + y * y)}};
    float half[3] = {w.f[FHX][s], w.f[FHY][s], w.f[FHZ][s]};
    for (int a = 0; a < 3; a++)
        out[a] = (half[0] * std::fabs(r[a][0]) + half[1] * std::fabs(r[a][1])) + half[2] * std::fabs(r[a][2]);
    if (w.f[FSHAPE][s] > 0.5f) {
        for (int a = 0; a < 3; a++) out[a] = half[0];
    }
}

// BoxBroad.bin :74-89 and a stable counting sort of the keys (SupirVast CountingSort's role).
void binAndSort(World& w) {
    int cells[3] = {w.nx, w.ny, w.nz};
    int total = w.nx * w.ny * w.nz;
    for (int s = 0; s < w.n; s++) {
        int c[3];
        for (int a = 0; a < 3; a++)
            c[a] = (int)fmaxj(0.0f, fminj((float)(cells[a] - 1), std::floor(w.f[FX + a][s] / w.cell)));
        w.keys[s] = c[0] + cells[0] * (c[1] + cells[1] * c[2]);
    }
    w.starts.assign(total + 1, 0);
    for (int s = 0; s < w.n; s++) w.starts[w.keys[s] + 1]++;
    for (int k = 0; k < total; k++) w.starts[k + 1] += w.starts[k];
    std::vector<int> fill(w.starts.begin(), w.starts.end() - 1);
    for (int s = 0; s < w.n; s++) w.order[fill[w.keys[s]]++] = s;
}

// BoxBroad.list :103-164 with around :230-252. With reach_cells r > 1 (cells narrower than BoxBroad.grid's rule,
// :66-68) the walk widens to the (2r + 1)^3 cells around, in the same x-fastest order; at r = 1 it is the reference's
// 27 cells in its order.
void list(World& w) {
    const float margin = w.params[MARGIN];
    ORC_PARALLEL_FOR
    for (int s = 0; s < w.n; s++) {
        long base = (long)s * SLOTS;
        for (int m = 0; m < SLOTS; m++) {
            w.pairs[2 * (base + m)] = s;
            w.pairs[2 * (base + m) + 1] = -1;
        }
        float centre[3] = {w.f[FX][s], w.f[FY][s], w.f[FZ][s]};
        float reach[3];
        reachOf(w, s, reach);
        int found = 0;
        int key = w.keys[s];
        int ix = key % w.nx, iy = (key / w.nx) % w.ny, iz = key / (w.nx * w.ny);
        const int r = w.reach_cells, side = 2 * r + 1;
        for (int nn = 0; nn < side * side * side; nn++) {
            int jx = ix + (nn % side - r), jy = iy + ((nn / side) % side - r), jz = iz + (nn / (side * side) - r);
            if (!(jx >= 0 && jx < w.nx && jy >= 0 && jy < w.ny && jz >= 0 && jz < w.nz)) continue;
            int cell = jx + w.nx * (jy + w.ny * jz);
            for (int k = w.starts[cell]; k < w.starts[cell + 1]; k++) {
                int o = w.order[k];
                if (!(o > s)) continue;
                float other[3];
                reachOf(w, o, other);
                bool close = true;
                for (int a = 0; a < 3; a++)
                    close = close && !(std::fabs(w.f[FX + a][o] - centre[a]) > (reach[a] + other[a]) + margin);
                if (!close) continue;
                if (found < SLOTS) {
                    int place = found;
                    while (place > 0) {
                        int before = w.pairs[2 * (base + place - 1) + 1];
                        if (before > o) {
                            w.pairs[2 * (base + place) + 1] = before;
                            place--;
                        } else {
                            break;
                        }
                    }
                    w.pairs[2 * (base + place) + 1] = o;
                }
                found++;
            }
        }
        w.contacts[2L * w.slots + s] = found;
    }
}

// BoxBroad.counts :174-188.
void counts(World& w) {
    ORC_PARALLEL_FOR
    for (long p = 0; p < w.slots; p++) {
        int partner = w.pairs[2 * p + 1];
        int count = (int)w.manifold[p * MANIFOLD_WORDS + COUNT];
        w.contacts[p] = count > 0 ? partner : -1;
        w.contacts[w.slots + p] = count;
    }
}

// BoxPairs.keep :164-182.
void keepPairs(World& w) {
    std::memcpy(w.manifoldWas.data(), w.manifold.data(), sizeof(float) * w.manifold.size());
    std::memcpy(w.impulsesWas.data(), w.impulses.data(), sizeof(float) * w.impulses.size());
    std::memcpy(w.pairsWas.data(), w.pairs.data(), sizeof(int) * w.pairs.size());
}

// BoxPairs.carry :191-267.
void carry(World& w) {
    ORC_PARALLEL_FOR
    for (long p = 0; p < w.slots; p++) {
        long out = p * MANIFOLD_WORDS;
        long held = p * IMPULSE_WORDS;
        int count = (int)w.manifold[out + COUNT];
        int partner = w.pairs[2 * p + 1];
        long first = (p / SLOTS) * SLOTS;
        long wasSlot = -1;
        for (int look = 0; look < SLOTS; look++) {
            int then = w.pairsWas[2 * (first + look) + 1];
            if (then == partner && !(partner < 0)) wasSlot = first + look;
        }
        long outWas = wasSlot * MANIFOLD_WORDS;
        long heldWas = wasSlot * IMPULSE_WORDS;
        int before = 0;
        if (!(wasSlot < 0)) before = (int)w.manifoldWas[outWas + COUNT];
        int ia = w.pairs[2 * p];
        float smallest = fminj(w.f[FHX][ia], fminj(w.f[FHY][ia], w.f[FHZ][ia]));
        float reach = (SAME_POINT * smallest) * (SAME_POINT * smallest);
        for (int point = 0; point < MOST_POINTS; point++) {
            float taken[POINT_IMPULSE] = {0, 0, 0, 0, 0, 0, 0};
            if (point < count) {
                const float* anchor = &w.manifold[out + POINTS + point * POINT_WORDS + ANCHOR_FIRST];
                float nearestD = reach;
                for (int old = 0; old < MOST_POINTS; old++) {
                    if (!(old < before)) continue;
                    const float* then = &w.manifoldWas[outWas + POINTS + old * POINT_WORDS + ANCHOR_FIRST];
                    float gap[3] = {anchor[0] - then[0], anchor[1] - then[1], anchor[2] - then[2]};
                    float d2 = dot3(gap, gap);
                    if (d2 < nearestD) {
                        nearestD = d2;
                        for (int q = 0; q < POINT_IMPULSE; q++)
                            taken[q] = w.impulsesWas[heldWas + POINT_IMPULSE * old + q];
                    }
                }
            }
            if (point == 0 && count == 1 && before == 1) {
                for (int q = 0; q < POINT_IMPULSE; q++) taken[q] = w.impulsesWas[heldWas + q];
            }
            for (int q = 0; q < POINT_IMPULSE; q++) w.impulses[held + POINT_IMPULSE * point + q] = taken[q];
        }
    }
}

// BoxPairs.solve :64-151, one round.
void solveRound(World& w, Sweep sweep, bool reverse, int round) {
    const float* params = w.params;
    long start = (long)round * w.width;
    ORC_PARALLEL_FOR
    for (int k = 0; k < w.width; k++) {
        int pair = w.rounds[start + k];
        if (pair < 0) continue;
        long out = (long)pair * MANIFOLD_WORDS;
        int count = (int)w.manifold[out + COUNT];
        if (!(count > 0)) continue;
        int ia = w.pairs[2L * pair], ib = w.pairs[2L * pair + 1];
        float imA = w.f[FIM][ia], imB = w.f[FIM][ib];
        Moving first = load(w, ia, imA);
        Moving second = load(w, ib, imB);
        Soft soft(params, false);
        soft.stiffen(imA == 0.0f || imB == 0.0f, params);
        float n[3] = {w.manifold[out + NORMAL], w.manifold[out + NORMAL + 1], w.manifold[out + NORMAL + 2]};
        long held = (long)pair * IMPULSE_WORDS;
        for (int order = 0; order < MOST_POINTS; order++) {
            int slot = reverse ? MOST_POINTS - 1 - order : order;
            if (!(slot < count)) continue;
            long where = out + POINTS + slot * POINT_WORDS;
            float rA[3], rB[3];
            rotate(first.q, &w.manifold[where + ANCHOR_FIRST], rA);
            rotate(second.q, &w.manifold[where + ANCHOR_SECOND], rB);
            if (first.isSphere())
                for (int a = 0; a < 3; a++) rA[a] = first.half[0] * n[a];
            if (second.isSphere())
                for (int a = 0; a < 3; a++) rB[a] = -(second.half[0] * n[a]);
            float gap = ((second.at[0] + rB[0]) - (first.at[0] + rA[0])) * n[0] +
                        ((second.at[1] + rB[1]) - (first.at[1] + rA[1])) * n[1];
            gap = gap + ((second.at[2] + rB[2]) - (first.at[2] + rA[2])) * n[2];
            long normalAt = held + POINT_IMPULSE * slot;
            long tangentAt = normalAt + 1;
            contact(sweep, gap, n, &first, rA, second, rB, w.impulses.data(), normalAt, w.impulses.data(), tangentAt,
                    soft);
            if (first.isSphere() || second.isSphere()) {
                float radius = second.half[0];
                if (first.isSphere()) radius = first.half[0];
                if (first.isSphere() && second.isSphere())
                    radius = (first.half[0] * second.half[0]) / (first.half[0] + second.half[0]);
                roll(sweep, &first, second, radius, w.impulses.data(), normalAt, w.impulses.data(), normalAt + 4,
                     params);
            }
        }
        store(w, first);
        store(w, second);
    }
}

// BoxStep.sweep :217-231.
void sweepAll(World& w, Sweep kind, bool reverse, int rounds) {
    if (reverse) walls(w, kind, true);
    for (int order = 0; order < rounds; order++) {
        int r = reverse ? rounds - 1 - order : order;
        solveRound(w, kind, reverse, r);
    }
    if (!reverse) walls(w, kind, false);
}

// BoxStepper.step :56-100 with the collide list (BoxStep :141-158) and the substeps (BoxStep.build :199-215).
void stepOnce(World& w) {
    int used = 0;
    for (int k = 0; k < 5; k++) w.report[k] = 0;
    if (w.slots > 0) {
        keepPairs(w);
        binAndSort(w);
        list(w);
        const float* buf[18];
        const float* const* f = fields(w, buf);
        const float* params = w.params;
        ORC_PARALLEL_FOR
        for (long p = 0; p < w.slots; p++) {
            float scratch[SCRATCH_WORDS];
            collideOne(f, params, w.pairs[2 * p], w.pairs[2 * p + 1], &w.manifold[p * MANIFOLD_WORDS], scratch);
        }
        carry(w);
        counts(w);
        // The host's greedy colouring (BoxStepper :330-362).
        std::vector<int> filled(MOST_ROUNDS, 0);
        std::vector<std::vector<char>> taken(MOST_ROUNDS, std::vector<char>(w.n, 0));
        std::fill(w.rounds.begin(), w.rounds.end(), -1);
        int touching = 0, points = 0, unplaced = 0;
        for (long p = 0; p < w.slots; p++) {
            int b = w.contacts[p];
            if (b < 0) continue;
            int a = (int)(p / SLOTS);
            touching++;
            points += w.contacts[w.slots + p];
            int r = 0;
            while (r < MOST_ROUNDS && (taken[r][a] || taken[r][b])) r++;
            if (r == MOST_ROUNDS) {
                unplaced++;
            } else {
                taken[r][a] = taken[r][b] = 1;
                w.rounds[(long)r * w.width + filled[r]++] = (int)p;
                used = std::max(used, r + 1);
            }
        }
        int unlisted = 0;
        for (int s = 0; s < w.n; s++) unlisted += std::max(0, w.contacts[2L * w.slots + s] - SLOTS);
        w.report[0] = touching;
        w.report[1] = points;
        w.report[2] = used;
        w.report[3] = unplaced;
        w.report[4] = unlisted;
    }
    for (int sub = 0; sub < w.substeps; sub++) {
        velocities(w);
        sweepAll(w, WARM, false, used);
        for (int sweep = 0; sweep < w.sweeps; sweep++) sweepAll(w, SOLVE, w.symmetric && sweep % 2 == 1, used);
        positions(w);
        for (int sweep = 0; sweep < w.sweeps; sweep++) sweepAll(w, RELAX, w.symmetric && sweep % 2 == 1, used);
    }
    show(w);
}

}  // namespace

// ------------------------------------------------------------------------------------------------------
// C interface for the test harness (ctypes).
extern "C" {

// fields: 0 x 1 y 2 z 3 u 4 v 5 w 6 lx 7 ly 8 lz 9 qx 10 qy 11 qz 12 qw 13 im 14 hx 15 hy 16 hz 17 shape
void orc_box_set_reach(void* h, int reach_cells) { ((World*)h)->reach_cells = reach_cells > 0 ? reach_cells : 1; }

void* orc_box_create(int n, int substeps, int sweeps, int symmetric, int nx, int ny, int nz, float cell,
                     int grid) {
    World* w = new World();
    w->n = n;
    w->substeps = substeps;
    w->sweeps = sweeps;
    w->symmetric = symmetric;
    w->nx = nx;
    w->ny = ny;
    w->nz = nz;
    w->cell = cell;
    w->slots = (n > 1 && grid) ? n * SLOTS : 0;
    w->width = std::max(1, n / 2);
    for (int k = 0; k < 18; k++) w->f[k].assign(n, 0.0f);
    w->f[FQW].assign(n, 1.0f);
    std::memset(w->params, 0, sizeof(w->params));
    w->lambda.assign((size_t)LAMBDA_WORDS * n, 0.0f);
    w->rub.assign((size_t)RUB_WORDS * n, 0.0f);
    w->rollw.assign((size_t)ROLL_WORDS * n, 0.0f);
    w->shown.assign((size_t)SHOWN_STRIDE * n, 0.0f);
    if (w->slots > 0) {
        w->keys.assign(n, 0);
        w->order.assign(n, 0);
        w->pairs.assign(2L * w->slots, 0);
        w->pairsWas.assign(2L * w->slots, 0);
        w->manifold.assign((size_t)MANIFOLD_WORDS * w->slots, 0.0f);
        w->manifoldWas.assign((size_t)MANIFOLD_WORDS * w->slots, 0.0f);
        w->impulses.assign((size_t)IMPULSE_WORDS * w->slots, 0.0f);
        w->impulsesWas.assign((size_t)IMPULSE_WORDS * w->slots, 0.0f);
        w->contacts.assign(2L * w->slots + n, 0);
        w->rounds.assign((size_t)MOST_ROUNDS * w->width, -1);
    }
    for (int k = 0; k < 5; k++) w->report[k] = 0;
    return w;
}
void orc_box_destroy(void* h) { delete (World*)h; }
void orc_box_set_field(void* h, int field, const float* values) {
    World* w = (World*)h;
    std::memcpy(w->f[field].data(), values, sizeof(float) * w->n);
}
void orc_box_get_field(void* h, int field, float* out) {
    World* w = (World*)h;
    std::memcpy(out, w->f[field].data(), sizeof(float) * w->n);
}
void orc_box_set_params(void* h, const int32_t* bits) {
    World* w = (World*)h;
    std::memcpy(w->params, bits, sizeof(w->params));
}
void orc_box_set_shown(void* h, const float* shown) {
    World* w = (World*)h;
    std::memcpy(w->shown.data(), shown, sizeof(float) * w->shown.size());
}
void orc_box_get_shown(void* h, float* out) {
    World* w = (World*)h;
    std::memcpy(out, w->shown.data(), sizeof(float) * w->shown.size());
}
void orc_box_step(void* h, int steps, int32_t* report) {
    World* w = (World*)h;
    for (int k = 0; k < steps; k++) stepOnce(*w);
    if (report)
        for (int k = 0; k < 5; k++) report[k] = w->report[k];
}
int orc_box_slots(void* h) { return ((World*)h)->slots; }
// Reference-layout buffers: 0 pairs (2*slots i32), 1 manifold (40*slots f32), 2 impulses (28*slots f32),
// 3 contacts (2*slots+n i32), 4 lambda (48n), 5 rub (144n), 6 roll (144n), 7 rounds (32*width i32)
long orc_box_buffer_words(void* h, int which) {
    World* w = (World*)h;
    switch (which) {
        case 0: return (long)w->pairs.size();
        case 1: return (long)w->manifold.size();
        case 2: return (long)w->impulses.size();
        case 3: return (long)w->contacts.size();
        case 4: return (long)w->lambda.size();
        case 5: return (long)w->rub.size();
        case 6: return (long)w->rollw.size();
        case 7: return (long)w->rounds.size();
    }
    return 0;
}
void* orc_box_buffer(void* h, int which) {
    World* w = (World*)h;
    switch (which) {
        case 0: return w->pairs.data();
        case 1: return w->manifold.data();
        case 2: return w->impulses.data();
        case 3: return w->contacts.data();
        case 4: return w->lambda.data();
        case 5: return w->rub.data();
        case 6: return w->rollw.data();
        case 7: return w->rounds.data();
    }
    return nullptr;
}

// The collide pass alone over a caller's pair list (BoxContactTest.collide :441-482): pairs[2p], pairs[2p+1].
void orc_collide(int bodies, const float* const* f18, const int32_t* param_bits, int npairs, const int32_t* pairs,
                 float* manifold) {
    float params[PARAM_COUNT];
    std::memcpy(params, param_bits, sizeof(params));
    (void)bodies;
    ORC_PARALLEL_FOR
    for (int p = 0; p < npairs; p++) {
        float scratch[SCRATCH_WORDS];
        collideOne(f18, params, pairs[2 * p], pairs[2 * p + 1], manifold + (long)p * MANIFOLD_WORDS, scratch);
    }
}

int orc_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
