// CPU ORACLE — test infrastructure only, never part of the product path.
//
// A single-precision C++ restatement of the reference's sphere package (dev.vexelray.sim.rigid.sphere of
// sibarum/vexelray-sim-rigid): XPBD with Gauss-Seidel over a contact list, run until every contact is solved, with
// warm starts, friction, rolling resistance, walls and restitution. One function per IR kernel, the reference's
// buffers, its pass order, and its association order; build with -ffp-contract=off.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library.
//
// Files restated (core = vexelray-sim-rigid-core/src/main/java/dev/vexelray/sim/rigid/):
//   core/sphere/Spheres.java   params :212-228, predict :269-295, contact :369-439, warm :448-481,
//                              Impulse :490-522, friction :595-654, rub :662-677, roll :699-741, turnsPerImpulse
//                              :743-745, contactTravel :751-766, clearContacts :829-844, keepContacts :859-878,
//                              warmWalls :890-939, listContacts :961-1022, contactRound :1076-1133, report
//                              :1146-1159, priority :1166-1168, walls :1185-1198, bin :1308-1323, shift :1351-1418,
//                              velocity :1430-1460, turn :1468-1493, bounce :1528-1627, bounced :1633-1644,
//                              show :1697-1794
//   core/sphere/SphereStep.java   byContact :271-315, cycle :324-352, opening/more/closing :363-420
//   core/sphere/SphereStepper.java  step :66-103, adapt :118-126
//
// The counting sort (SupirVast's CountingSort, absent) is stable here: within a cell, ascending index. The list's
// atomic append is made in invocation order; no result depends on the list's order (a pair's priority, not its
// place, decides its round; its warm start is found by its partner).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

namespace {

enum { H = 0, GX, GY, GZ, SX, SY, SZ, OMEGA, AVERAGED, RESTITUTION, MU_STATIC, MU_KINETIC, MU_ROLLING, PARAMS };
constexpr float COINCIDENT = 1e-12f;
constexpr float LIST_MARGIN = 0.02f;
constexpr float INERTIA = 0.4f;
constexpr int IMPULSE_WORDS = 7, WALL_IMPULSE_WORDS = 21;
constexpr int LISTED = 0, MISSED = 1, LONGEST = 2;
constexpr int MOST_KEPT = 32;
constexpr int CYCLE = 48, BATCH = 8, SHRINK_AFTER = 120;
constexpr int SHOWN_STRIDE = 40, PRESSED_BEFORE = 8, PRESSED_AFTER = 20, TURNED_BEFORE = 32, TURNED_AFTER = 36;

enum {
    FX = 0, FY, FZ, FU, FV, FW, FR, FIM, FCX, FCY, FCZ, FDX, FDY, FDZ, FAX, FAY, FAZ, FTX, FTY, FTZ, FQX, FQY, FQZ,
    FQW, FIELDS
};

struct World {
    int n, substeps, iterations, capacity;
    int solve;   // 0 Jacobi, 1 Gauss-Seidel over the contact list until done, 2 the same with fixed rounds
    int rounds;  // for solve 2: the rounds a pass
    bool gridded;
    int nx, ny, nz;
    float cell;
    float params[PARAMS];
    std::vector<float> f[FIELDS];
    std::vector<float> shown;
    std::vector<int> keys, order, starts;
    std::vector<int> claims[3];
    std::vector<int> contactA, contactB, contactDone, contactNext, contactHead, keptB, keptNext, keptHead;
    std::vector<float> contactImpulse, keptImpulse, wallImpulse;
    int contactCount[3] = {0, 0, 0};
    int open[2] = {0, 0};
    int friction = 1;
    std::vector<int> opening, enough;
    int report[4] = {0, 0, 0, 0};  // waits, rounds, most rounds, unlisted
};

inline float dotf(const float* x, const float* y) { return x[0] * y[0] + (x[1] * y[1] + x[2] * y[2]); }
inline void crossf(const float* x, const float* y, float* z) {
    float o[3];
    for (int k = 0; k < 3; k++) {
        int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
        o[k] = x[k1] * y[k2] - x[k2] * y[k1];
    }
    z[0] = o[0]; z[1] = o[1]; z[2] = o[2];
}

// Spheres.turn :1468-1493: q turned by the small rotation `angle`.
void turnQ(World& w, int s, const float* angle) {
    float a[3];
    for (int k = 0; k < 3; k++) a[k] = 0.5f * angle[k];
    float was[4] = {w.f[FQX][s], w.f[FQY][s], w.f[FQZ][s], w.f[FQW][s]};
    float now[4];
    for (int k = 0; k < 3; k++) {
        int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
        now[k] = was[k] + (a[k] * was[3] + (a[k1] * was[k2] - a[k2] * was[k1]));
    }
    now[3] = was[3] - (a[0] * was[0] + (a[1] * was[1] + a[2] * was[2]));
    float len2 = (now[0] * now[0] + now[1] * now[1]) + (now[2] * now[2] + now[3] * now[3]);
    float inverse = 1.0f / std::sqrt(std::fmax(len2, 1e-30f));
    for (int k = 0; k < 4; k++) w.f[FQX + k][s] = now[k] * inverse;
}

// Spheres.predict :269-295.
void predict(World& w) {
    const float* p = w.params;
    for (int s = 0; s < w.n; s++) {
        if (!(w.f[FIM][s] > 0.0f)) continue;
        float h = p[H];
        for (int a = 0; a < 3; a++) {
            float vel = w.f[FU + a][s] + h * p[GX + a];
            w.f[FU + a][s] = vel;
            w.f[FX + a][s] = w.f[FX + a][s] + h * vel;
        }
        float angle[3];
        for (int a = 0; a < 3; a++) angle[a] = h * w.f[FAX + a][s];
        turnQ(w, s, angle);
    }
}

// Spheres.bin :1308-1323 and a stable counting sort.
void binSort(World& w) {
    int cells[3] = {w.nx, w.ny, w.nz};
    int total = w.nx * w.ny * w.nz;
    for (int s = 0; s < w.n; s++) {
        int c[3];
        for (int a = 0; a < 3; a++)
            c[a] = (int)std::fmax(0.0f, std::fmin((float)(cells[a] - 1), std::floor(w.f[FX + a][s] / w.cell)));
        w.keys[s] = c[0] + cells[0] * (c[1] + cells[1] * c[2]);
    }
    w.starts.assign(total + 1, 0);
    for (int s = 0; s < w.n; s++) w.starts[w.keys[s] + 1]++;
    for (int k = 0; k < total; k++) w.starts[k + 1] += w.starts[k];
    std::vector<int> fill(w.starts.begin(), w.starts.end() - 1);
    for (int s = 0; s < w.n; s++) w.order[fill[w.keys[s]]++] = s;
}

// Spheres.around :1207-1229: every sphere in s's cell and the 26 around it, cell by cell, each cell in the sort's
// order; with no grid, every sphere in index order (the all-pairs loops of solve(), bounce() and show()).
template <typename Visit>
void around(const World& w, int s, Visit visit) {
    if (!w.gridded) {
        for (int o = 0; o < w.n; o++) visit(o);
        return;
    }
    int key = w.keys[s];
    int ix = key % w.nx, iy = (key / w.nx) % w.ny, iz = key / (w.nx * w.ny);
    for (int nn = 0; nn < 27; nn++) {
        int jx = ix + (nn % 3 - 1), jy = iy + ((nn / 3) % 3 - 1), jz = iz + (nn / 9 - 1);
        if (!(jx >= 0 && jx < w.nx && jy >= 0 && jy < w.ny && jz >= 0 && jz < w.nz)) continue;
        int cell = jx + w.nx * (jy + w.ny * jz);
        for (int k = w.starts[cell]; k < w.starts[cell + 1]; k++) visit(w.order[k]);
    }
}

// A sphere as a pass holds it (Spheres.Held :542-569).
struct Held {
    int s;
    float at[3], displaced[3], turned[3];
    bool turns;
};
Held load(const World& w, int s, bool turns) {
    Held h;
    h.s = s;
    h.turns = turns;
    for (int k = 0; k < 3; k++) {
        h.at[k] = w.f[FX + k][s];
        h.displaced[k] = w.f[FDX + k][s];
        h.turned[k] = turns ? w.f[FTX + k][s] : 0.0f;
    }
    return h;
}
void store(World& w, const Held& h) {
    for (int k = 0; k < 3; k++) {
        w.f[FX + k][h.s] = h.at[k];
        w.f[FDX + k][h.s] = h.displaced[k];
        if (h.turns) w.f[FTX + k][h.s] = h.turned[k];
    }
}

// Spheres.Impulse :490-522: normal, p (3), q (3).
struct Impulse {
    float* at;
    float normal, p[3], q[3];
    explicit Impulse(float* base) : at(base) {
        normal = base[0];
        for (int k = 0; k < 3; k++) {
            p[k] = base[1 + k];
            q[k] = base[4 + k];
        }
    }
    void clear() {
        normal = 0.0f;
        for (int k = 0; k < 3; k++) p[k] = q[k] = 0.0f;
    }
    void save() {
        at[0] = normal;
        for (int k = 0; k < 3; k++) {
            at[1 + k] = p[k];
            at[4 + k] = q[k];
        }
    }
};

inline float turnsPerImpulse(float wv, float lever, float radius) { return (wv * lever) / (INERTIA * (radius * radius)); }
inline float rubbingOf(const float* p) { return p[MU_STATIC] + (p[MU_KINETIC] + p[MU_ROLLING]); }

// Spheres.rub :662-677.
void rub(Held& a, float wa, float turnsA, Held* o, float wo, float turnsO, const float* n, const float* p) {
    float np[3];
    crossf(n, p, np);
    for (int k = 0; k < 3; k++) {
        float move = wa * p[k];
        a.at[k] = a.at[k] + move;
        a.displaced[k] = a.displaced[k] + move;
        a.turned[k] = a.turned[k] - turnsA * np[k];
        if (o) {
            float back = wo * p[k];
            o->at[k] = o->at[k] - back;
            o->displaced[k] = o->displaced[k] - back;
            o->turned[k] = o->turned[k] - turnsO * np[k];
        }
    }
}

// Spheres.contactTravel :751-766.
void contactTravel(const World& w, const Held& s, float h, const float* n, float lever, int side, float* travel) {
    float turn[3];
    for (int k = 0; k < 3; k++) turn[k] = h * w.f[FAX + k][s.s] + s.turned[k];
    float turnN[3];
    crossf(turn, n, turnN);
    for (int k = 0; k < 3; k++) {
        float centre = h * w.f[FU + k][s.s] + s.displaced[k];
        float spun = lever * turnN[k];
        travel[k] = side > 0 ? centre + spun : centre - spun;
    }
}

// Spheres.friction :595-654.
void friction(const World& w, Held& a, float wa, float leverA, Held* o, float wo, float leverO, const float* n,
              Impulse& taken) {
    const float* P = w.params;
    float muS = P[MU_STATIC], muK = P[MU_KINETIC];
    float lambdaN = taken.normal;
    if (!(muS + muK > 0.0f)) return;
    float h = P[H];
    float la = leverA;
    float slip[3];
    contactTravel(w, a, h, n, la, -1, slip);
    float ia = wa;
    float leverOverIa = turnsPerImpulse(ia, la, w.f[FR][a.s]);
    float weight = ia + leverOverIa * la;
    float leverOverIo = 0.0f, io = 0.0f;
    if (o) {
        io = wo;
        float lo = leverO;
        float other[3];
        contactTravel(w, *o, h, n, lo, 1, other);
        for (int k = 0; k < 3; k++) slip[k] = slip[k] - other[k];
        leverOverIo = turnsPerImpulse(io, lo, w.f[FR][o->s]);
        weight = weight + (io + leverOverIo * lo);
    }
    float along = dotf(slip, n);
    float tangent[3];
    for (int k = 0; k < 3; k++) tangent[k] = slip[k] - along * n[k];
    if (!(weight > 0.0f)) return;
    float takenAlong = dotf(taken.p, n);
    float before[3], whole[3];
    for (int k = 0; k < 3; k++) {
        before[k] = taken.p[k] - takenAlong * n[k];
        whole[k] = before[k] - tangent[k] / weight;
    }
    float size2 = dotf(whole, whole);
    float holds = muS * lambdaN;
    if (size2 > holds * holds) {
        float cut = std::fmin(1.0f, (muK * lambdaN) / std::sqrt(size2));
        for (int k = 0; k < 3; k++) whole[k] = whole[k] * cut;
    }
    float p[3];
    for (int k = 0; k < 3; k++) {
        p[k] = whole[k] - before[k];
        taken.p[k] = whole[k];
    }
    rub(a, ia, leverOverIa, o, io, leverOverIo, n, p);
}

// Spheres.roll :699-741.
void roll(const World& w, Held& a, float wa, Held* o, float wo, float reach, Impulse& taken) {
    const float* P = w.params;
    float muR = P[MU_ROLLING];
    float h = P[H];
    float ra = w.f[FR][a.s];
    float ia = wa / (INERTIA * (ra * ra));
    float inverse = ia;
    float io = 0.0f;
    float against[3];
    for (int k = 0; k < 3; k++) against[k] = h * w.f[FAX + k][a.s] + a.turned[k];
    if (o) {
        float ro = w.f[FR][o->s];
        io = wo / (INERTIA * (ro * ro));
        inverse = inverse + io;
        for (int k = 0; k < 3; k++) against[k] = against[k] - (h * w.f[FAX + k][o->s] + o->turned[k]);
    }
    if (!(inverse > 0.0f)) return;
    float whole[3];
    for (int k = 0; k < 3; k++) whole[k] = taken.q[k] - against[k] / inverse;
    float size2 = dotf(whole, whole);
    float holds = (muR * reach) * taken.normal;
    if (size2 > holds * holds) {
        float cut = std::fmin(1.0f, holds / std::sqrt(size2));
        for (int k = 0; k < 3; k++) whole[k] = whole[k] * cut;
    }
    for (int k = 0; k < 3; k++) {
        float change = whole[k] - taken.q[k];
        taken.q[k] = whole[k];
        a.turned[k] = a.turned[k] + ia * change;
        if (o) o->turned[k] = o->turned[k] - io * change;
    }
}

// Spheres.warm :448-481.
void warm(const World& w, Held& a, float wa, Held& o, float wo, const float* d, float d2, float reach, Impulse& taken) {
    float dist = std::sqrt(d2);
    float n[3];
    for (int k = 0; k < 3; k++) n[k] = d[k] / dist;
    for (int k = 0; k < 3; k++) {
        float push = taken.normal * n[k];
        float ma = push * wa;
        float mo = -(push * wo);
        a.at[k] = a.at[k] + ma;
        o.at[k] = o.at[k] + mo;
        a.displaced[k] = a.displaced[k] + ma;
        o.displaced[k] = o.displaced[k] + mo;
    }
    float along = dotf(taken.p, n);
    for (int k = 0; k < 3; k++) taken.p[k] = taken.p[k] - along * n[k];
    float share = dist / reach;
    float ra = w.f[FR][a.s], ro = w.f[FR][o.s];
    float turnsA = turnsPerImpulse(wa, share * ra, ra);
    float turnsO = turnsPerImpulse(wo, share * ro, ro);
    rub(a, wa, turnsA, &o, wo, turnsO, n, taken.p);
    float ia = wa / (INERTIA * (ra * ra));
    float io = wo / (INERTIA * (ro * ro));
    for (int k = 0; k < 3; k++) {
        a.turned[k] = a.turned[k] + ia * taken.q[k];
        o.turned[k] = o.turned[k] - io * taken.q[k];
    }
}

// Spheres.contact :369-439.
void contact(World& w, int c, int ai, int oi, float omega, int pass, int rubs) {
    Held ha = load(w, ai, true), ho = load(w, oi, true);
    float d[3];
    for (int k = 0; k < 3; k++) d[k] = ha.at[k] - ho.at[k];
    float d2 = dotf(d, d);
    float reach = w.f[FR][ai] + w.f[FR][oi];
    float wa = w.f[FIM][ai], wo = w.f[FIM][oi];
    float wsum = wa + wo;
    float listed = reach * (1.0f + LIST_MARGIN);
    if (!(d2 < listed * listed)) return;
    if (!(d2 > COINCIDENT)) return;
    if (!(wsum > 0.0f)) return;
    Impulse taken(&w.contactImpulse[(size_t)c * IMPULSE_WORDS]);
    if (rubs == 0) {
        float rubbing = rubbingOf(w.params);
        if (pass == 1) {
            if (rubbing > 0.0f) warm(w, ha, wa, ho, wo, d, d2, reach, taken);
            else taken.clear();
        }
        for (int k = 0; k < 3; k++) d[k] = ha.at[k] - ho.at[k];
        float dist = std::sqrt(std::fmax(dotf(d, d), COINCIDENT));
        float depth = std::fmax(-(taken.normal * wsum), omega * (reach - dist));
        taken.normal = taken.normal + depth / wsum;
        float kk = depth / (dist * wsum);
        for (int k = 0; k < 3; k++) {
            float step = kk * d[k];
            float ma = step * wa;
            float mo = -(step * wo);
            ha.at[k] = ha.at[k] + ma;
            ho.at[k] = ho.at[k] + mo;
            ha.displaced[k] = ha.displaced[k] + ma;
            ho.displaced[k] = ho.displaced[k] + mo;
        }
    } else {
        float dist = std::sqrt(d2);
        float n[3];
        for (int k = 0; k < 3; k++) n[k] = d[k] / dist;
        float share = dist / reach;
        float pairRadius = (w.f[FR][ai] * w.f[FR][oi]) / reach;
        roll(w, ha, wa, &ho, wo, pairRadius, taken);
        friction(w, ha, wa, share * w.f[FR][ai], &ho, wo, share * w.f[FR][oi], n, taken);
    }
    taken.save();
    store(w, ha);
    store(w, ho);
}

// Spheres.warmWalls :890-939.
void warmWalls(World& w) {
    const float* P = w.params;
    for (int s = 0; s < w.n; s++) {
        if (!(w.f[FIM][s] > 0.0f)) continue;
        float r = w.f[FR][s], wv = w.f[FIM][s];
        float turns = turnsPerImpulse(wv, r, r);
        Held held = load(w, s, true);
        float rubbing = rubbingOf(P);
        for (int axis = 0; axis < 3; axis++) {
            Impulse taken(&w.wallImpulse[(size_t)s * WALL_IMPULSE_WORDS + axis * IMPULSE_WORDS]);
            float reach = r * (1.0f + LIST_MARGIN);
            float position = held.at[axis];
            float out = 0.0f;
            if (position < reach) out = 1.0f;
            if (position > P[SX + axis] - reach) out = -1.0f;
            bool near = rubbing > 0.0f && out != 0.0f;
            if (!near) {
                taken.clear();
            } else {
                float push = (taken.normal * wv) * out;
                held.at[axis] = held.at[axis] + push;
                held.displaced[axis] = held.displaced[axis] + push;
                taken.p[axis] = 0.0f;
                float n[3] = {0.0f, 0.0f, 0.0f};
                n[axis] = out;
                rub(held, wv, turns, nullptr, 0.0f, 0.0f, n, taken.p);
                for (int k = 0; k < 3; k++) held.turned[k] = held.turned[k] + (turns * taken.q[k]) / r;
            }
            taken.save();
        }
        store(w, held);
    }
}

// Spheres.keepContacts :859-878 then clearContacts :829-844.
void keepAndClear(World& w) {
    int listed = std::min(w.contactCount[LISTED], w.capacity);
    for (int c = 0; c < listed; c++) {
        w.keptB[c] = w.contactB[c];
        w.keptNext[c] = w.contactNext[c];
        for (int k = 0; k < IMPULSE_WORDS; k++)
            w.keptImpulse[(size_t)c * IMPULSE_WORDS + k] = w.contactImpulse[(size_t)c * IMPULSE_WORDS + k];
    }
    for (int s = 0; s < w.n; s++) {
        w.keptHead[s] = w.contactHead[s];
        w.contactHead[s] = -1;
    }
    for (int k = 0; k < 3; k++) std::fill(w.claims[k].begin(), w.claims[k].end(), 0);
    w.contactCount[LONGEST] = std::max(w.contactCount[LONGEST], w.contactCount[LISTED]);
    w.contactCount[LISTED] = 0;
}

// Spheres.listContacts :961-1022.
void listContacts(World& w) {
    for (int a = 0; a < w.n; a++) {
        float mine[3] = {w.f[FX][a], w.f[FY][a], w.f[FZ][a]};
        float ra = w.f[FR][a];
        around(w, a, [&](int o) {
            if (!(o > a)) return;
            float d[3];
            for (int k = 0; k < 3; k++) d[k] = mine[k] - w.f[FX + k][o];
            float d2 = d[0] * d[0] + (d[1] * d[1] + d[2] * d[2]);
            float near = (ra + w.f[FR][o]) * (1.0f + LIST_MARGIN);
            if (!(d2 < near * near)) return;
            int slot = w.contactCount[LISTED]++;
            if (!(slot < w.capacity)) return;
            w.contactA[slot] = a;
            w.contactB[slot] = o;
            w.contactDone[slot] = 0;
            w.contactNext[slot] = w.contactHead[a];
            w.contactHead[a] = slot;
            float warmth[IMPULSE_WORDS] = {0, 0, 0, 0, 0, 0, 0};
            int j = w.keptHead[a];
            int walked = 0;
            while (j >= 0 && walked < MOST_KEPT) {
                if (w.keptB[j] == o) {
                    for (int k = 0; k < IMPULSE_WORDS; k++) warmth[k] = w.keptImpulse[(size_t)j * IMPULSE_WORDS + k];
                    walked = MOST_KEPT;
                }
                j = w.keptNext[j];
                walked++;
            }
            for (int k = 0; k < IMPULSE_WORDS; k++) w.contactImpulse[(size_t)slot * IMPULSE_WORDS + k] = warmth[k];
        });
    }
}

inline int32_t priority(int32_t pair, int32_t g) {
    uint32_t p = (uint32_t)pair * 0x9E3779B1u + (uint32_t)g * 0x632BE5ABu;
    return (int32_t)(p & 0x7FFFFFFFu);
}

// Spheres.contactRound :1076-1133, one dispatch. r = [checks, claims, pass, dispatch, mark, checks dispatch, rubs];
// claim arrays: checked, claimed, cleared.
void contactRound(World& w, const int* r, int checkedI, int claimedI, int clearedI) {
    int mark = r[4];
    w.open[1 - mark] = 0;
    int listed = std::min(w.contactCount[LISTED], w.capacity);
    std::vector<int>& checked = w.claims[checkedI];
    std::vector<int>& claimed = w.claims[claimedI];
    std::vector<int>& cleared = w.claims[clearedI];
    float omega = w.params[OMEGA];
    for (int c = 0; c < listed; c++) {
        int pass = r[2];
        if (w.contactDone[c] == pass) continue;
        int a = w.contactA[c], o = w.contactB[c];
        int32_t pair = a * w.n + o;
        int won = 0;
        if (r[0] > 0) {
            int32_t last = priority(pair, r[5]);
            if (checked[a] == last && checked[o] == last) won = 1;
        }
        if (won) {
            contact(w, c, a, o, omega, pass, r[6]);
            w.contactDone[c] = pass;
        } else {
            cleared[a] = 0;
            cleared[o] = 0;
            if (r[1] > 0) {
                w.open[mark] = 1;
                int32_t mine = priority(pair, r[3]);
                claimed[a] = std::max(claimed[a], mine);
                claimed[o] = std::max(claimed[o], mine);
            } else {
                w.contactCount[MISSED]++;
            }
        }
    }
}

inline int position(int k) { return k == 0 ? 0 : 1 + (k - 1) % CYCLE; }

// The round at cycle position p of pass `it` (SphereStep.cycle :324-352): rubs selects the friction rounds.
void cycleRound(World& w, int it, int p, bool rubs) {
    int dispatch = it * CYCLE + p % CYCLE;
    int checks = it * CYCLE + std::max(p - 1, 0) % CYCLE;
    int pass = rubs ? w.iterations + it + 1 : it + 1;
    int r[7] = {p == 0 ? 0 : 1, 1, pass, dispatch, p % 2, checks, rubs ? 1 : 0};
    contactRound(w, r, (p + 2) % 3, p % 3, (p + 1) % 3);
}

// Spheres.shift :1351-1418 with friction (Spheres.walls :1185-1198).
void walls(World& w) {
    const float* P = w.params;
    for (int s = 0; s < w.n; s++) {
        if (!(w.f[FIM][s] > 0.0f)) continue;
        float r = w.f[FR][s];
        Held held = load(w, s, true);
        for (int a = 0; a < 3; a++) {
            float c = 0.0f;
            float moved = held.at[a] + c;
            float high = P[SX + a] - r;
            float side = 1.0f;
            float into = r - moved;
            if (moved * 2.0f > P[SX + a]) {
                side = -1.0f;
                into = moved - high;
            }
            float wv = w.f[FIM][s];
            Impulse taken(&w.wallImpulse[(size_t)s * WALL_IMPULSE_WORDS + a * IMPULSE_WORDS]);
            float inside = std::fmax(r, std::fmin(high, moved));
            float push = std::fmax(into, 0.0f);
            if (!(into > 0.0f) && taken.normal > 0.0f) {
                push = std::fmax(into, -(taken.normal * wv));
                inside = moved + side * push;
            }
            taken.normal = taken.normal + push / wv;
            held.at[a] = inside;
            held.displaced[a] = held.displaced[a] + (c + (inside - moved));
            float reach = r * LIST_MARGIN;
            float out = 0.0f;
            if (!(inside > r + reach)) out = 1.0f;
            if (!(inside < high - reach)) out = -1.0f;
            if (out != 0.0f) {
                float n[3] = {0.0f, 0.0f, 0.0f};
                n[a] = out;
                roll(w, held, wv, nullptr, 0.0f, r, taken);
                friction(w, held, wv, r, nullptr, 0.0f, 0.0f, n, taken);
            }
            taken.save();
        }
        for (int a = 0; a < 3; a++) {
            float high = P[SX + a] - r;
            float inside = std::fmax(r, std::fmin(high, held.at[a]));
            held.displaced[a] = held.displaced[a] + (inside - held.at[a]);
            held.at[a] = inside;
        }
        store(w, held);
    }
}

// Spheres.solve :302-347 and Solving :1245-1298: Jacobi's move for every sphere into cx, cy, cz, from the positions
// before the pass.
void jacobiSolve(World& w) {
    const float* P = w.params;
    for (int s = 0; s < w.n; s++) {
        float mine[3] = {w.f[FX][s], w.f[FY][s], w.f[FZ][s]};
        float rs = w.f[FR][s], ws = w.f[FIM][s];
        float sum[3] = {0.0f, 0.0f, 0.0f};
        float contacts = 0.0f;
        around(w, s, [&](int o) {
            if (o == s) return;
            float d[3];
            for (int a = 0; a < 3; a++) d[a] = mine[a] - w.f[FX + a][o];
            float d2 = d[0] * d[0] + (d[1] * d[1] + d[2] * d[2]);
            float reach = rs + w.f[FR][o];
            float wsum = ws + w.f[FIM][o];
            if (!(d2 < reach * reach)) return;
            if (!(d2 > COINCIDENT)) return;
            if (!(wsum > 0.0f)) return;
            float dist = std::sqrt(d2);
            float share = ((reach - dist) * (ws / wsum)) / dist;
            for (int a = 0; a < 3; a++) sum[a] = sum[a] + share * d[a];
            contacts = contacts + 1.0f;
        });
        float omega = P[OMEGA];
        float scale = omega;
        if (P[AVERAGED] > 0.0f) scale = omega / std::fmax(contacts, 1.0f);
        for (int a = 0; a < 3; a++) w.f[FCX + a][s] = scale * sum[a];
    }
}

// Spheres.apply :1326-1342 (shift :1351-1418 without friction): the move, then projected inside the walls.
void jacobiApply(World& w) {
    const float* P = w.params;
    for (int s = 0; s < w.n; s++) {
        if (!(w.f[FIM][s] > 0.0f)) continue;
        float r = w.f[FR][s];
        Held held = load(w, s, false);
        for (int a = 0; a < 3; a++) {
            float c = w.f[FCX + a][s];
            float moved = held.at[a] + c;
            float high = P[SX + a] - r;
            float inside = std::fmax(r, std::fmin(high, moved));
            held.at[a] = inside;
            float push = inside - moved;
            held.displaced[a] = held.displaced[a] + (c + push);
        }
        store(w, held);
    }
}

// Spheres.velocity :1430-1460.
void velocity(World& w) {
    for (int s = 0; s < w.n; s++) {
        float perH = 1.0f / w.params[H];
        for (int a = 0; a < 3; a++) {
            float was = w.f[FU + a][s];
            w.f[FCX + a][s] = was;
            w.f[FU + a][s] = was + w.f[FDX + a][s] * perH;
            w.f[FDX + a][s] = 0.0f;
        }
        float angle[3];
        for (int a = 0; a < 3; a++) {
            float by = w.f[FTX + a][s];
            w.f[FAX + a][s] = w.f[FAX + a][s] + by * perH;
            w.f[FTX + a][s] = 0.0f;
            angle[a] = by;
        }
        turnQ(w, s, angle);
    }
}

// Spheres.bounce(grid) :1528-1627 and bounced :1633-1644.
void bounce(World& w) {
    const float* P = w.params;
    std::vector<float> change(3 * (size_t)w.n, 0.0f);
    for (int s = 0; s < w.n; s++) {
        float e = P[RESTITUTION];
        float wa = w.f[FIM][s];
        if (!(e > 0.0f && wa > 0.0f)) continue;
        float h = P[H];
        float gx = P[GX], gy = P[GY], gz = P[GZ];
        float resting = (2.0f * h) * std::sqrt(gx * gx + (gy * gy + gz * gz));
        float ra = w.f[FR][s];
        float mine[3], vel[3], was[3], sum[3] = {0, 0, 0};
        for (int a = 0; a < 3; a++) {
            mine[a] = w.f[FX + a][s];
            vel[a] = w.f[FU + a][s];
            was[a] = w.f[FCX + a][s];
        }
        around(w, s, [&](int o) {
            if (o == s) return;
            float d[3];
            for (int a = 0; a < 3; a++) d[a] = mine[a] - w.f[FX + a][o];
            float d2 = d[0] * d[0] + (d[1] * d[1] + d[2] * d[2]);
            float near = (ra + w.f[FR][o]) * (1.0f + LIST_MARGIN);
            float wsum = wa + w.f[FIM][o];
            if (!(d2 < near * near && d2 > COINCIDENT)) return;
            float dist = std::sqrt(d2);
            float closing = 0.0f, parting = 0.0f;
            for (int a = 0; a < 3; a++) {
                float n = d[a] / dist;
                closing = closing + n * (was[a] - w.f[FCX + a][o]);
                parting = parting + n * (vel[a] - w.f[FU + a][o]);
            }
            if (closing < -resting) {
                float k = ((-(e * closing) - parting) * wa) / (wsum * dist);
                for (int a = 0; a < 3; a++) sum[a] = sum[a] + k * d[a];
            }
        });
        for (int a = 0; a < 3; a++) {
            float reach = ra * (1.0f + LIST_MARGIN);
            if (mine[a] < reach && was[a] < -resting) sum[a] = sum[a] + (-(e * was[a]) - vel[a]);
            if (mine[a] > P[SX + a] - reach && was[a] > resting) sum[a] = sum[a] + (-(e * was[a]) - vel[a]);
        }
        for (int a = 0; a < 3; a++) change[(size_t)s * 3 + a] = sum[a];
    }
    // bounced: dx, dy, dz hold the change (zero where bounce did not write), added to the velocity
    for (int s = 0; s < w.n; s++)
        for (int a = 0; a < 3; a++) {
            w.f[FU + a][s] = w.f[FU + a][s] + change[(size_t)s * 3 + a];
            w.f[FDX + a][s] = 0.0f;
        }
}

// Spheres.show(grid) :1697-1794.
void show(World& w) {
    const float* P = w.params;
    std::vector<float> out((size_t)w.n * SHOWN_STRIDE);
    for (int s = 0; s < w.n; s++) {
        const float* sh = &w.shown[(size_t)s * SHOWN_STRIDE];
        float* o = &out[(size_t)s * SHOWN_STRIDE];
        std::memcpy(o, sh, sizeof(float) * SHOWN_STRIDE);
        float mine[3];
        for (int a = 0; a < 3; a++) {
            mine[a] = w.f[FX + a][s];
            o[a] = sh[4 + a];
            o[4 + a] = mine[a];
        }
        float rs = w.f[FR][s];
        o[3] = rs;
        for (int k = 0; k < 12; k++) o[PRESSED_BEFORE + k] = sh[PRESSED_AFTER + k];
        for (int k = 0; k < 4; k++) {
            o[TURNED_BEFORE + k] = sh[TURNED_AFTER + k];
            o[TURNED_AFTER + k] = w.f[FQX + k][s];
        }
        float flat[6] = {0, 0, 0, 0, 0, 0}, lean[3] = {0, 0, 0};
        for (int a = 0; a < 3; a++) {
            float low = rs - mine[a];
            float high = (mine[a] + rs) - P[SX + a];
            for (int side = 0; side < 2; side++) {
                float depth = side == 0 ? low : high;
                float sg = side == 0 ? -1.0f : 1.0f;
                if (depth > 0.0f) {
                    float share = depth / rs;
                    flat[a] = flat[a] + share;
                    lean[a] = lean[a] + sg * share;
                }
            }
        }
        around(w, s, [&](int ot) {
            if (ot == s) return;
            float d[3];
            for (int a = 0; a < 3; a++) d[a] = w.f[FX + a][ot] - mine[a];
            float d2 = dotf(d, d);
            float reach = rs + w.f[FR][ot];
            if (!(d2 < reach * reach && d2 > COINCIDENT)) return;
            float dist = std::sqrt(d2);
            float share = (reach - dist) / reach;
            float g = share / d2;
            float along = share / dist;
            const int pairs[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
            for (int k = 0; k < 6; k++) flat[k] = flat[k] + g * (d[pairs[k][0]] * d[pairs[k][1]]);
            for (int a = 0; a < 3; a++) lean[a] = lean[a] + along * d[a];
        });
        float* after = o + PRESSED_AFTER;
        for (int k = 0; k < 6; k++) after[k] = flat[k];
        for (int a = 0; a < 3; a++) after[6 + a] = lean[a];
        after[9] = (flat[0] + flat[1]) + flat[2];
        after[10] = std::sqrt(dotf(lean, lean));
    }
    w.shown.swap(out);
}

// One pass run until done (SphereStepper.step :75-96 with SphereStep.opening/more): parting rounds until no contact
// is open, then as many friction rounds, then the walls. Returns the rounds run.
int passUntilDone(World& w, int it) {
    int limit = w.capacity + 2 * CYCLE;
    int k = w.opening[it];
    for (int j = 0; j < k; j++) cycleRound(w, it, position(j), false);
    w.report[0]++;
    int open = w.open[position(k - 1) % 2];
    while (open != 0) {
        if (k > limit) throw std::runtime_error("a pass is still open past its round limit");
        for (int j = k; j < k + BATCH; j++) cycleRound(w, it, position(j), false);
        k += BATCH;
        w.report[0]++;
        open = w.open[position(k - 1) % 2];
    }
    return k;
}

// A fixed-rounds pass (SphereStep.byContact :216-262): rounds 0 to `rounds` on dispatches g counted over the
// substep's passes; the last checks and does not claim, so what it leaves open is counted missed.
void fixedPass(World& w, int it) {
    for (int k = 0; k <= w.rounds; k++) {
        int g = it * (w.rounds + 1) + k;
        int r[7] = {k == 0 ? 0 : 1, k == w.rounds ? 0 : 1, it + 1, g, g % 2, g - 1, 0};
        contactRound(w, r, (g + 2) % 3, g % 3, (g + 1) % 3);
    }
}

// One step (SphereStep's pass list :184-196, and SphereStepper.step :66-103 for a solve run until done).
void stepOnce(World& w) {
    w.report[0] = w.report[1] = w.report[2] = w.report[3] = 0;
    for (int sub = 0; sub < w.substeps; sub++) {
        predict(w);
        if (w.gridded) binSort(w);
        if (w.solve != 0) {
            warmWalls(w);
            keepAndClear(w);
            listContacts(w);
        }
        for (int it = 0; it < w.iterations; it++) {
            if (w.solve == 0) {
                jacobiSolve(w);
                jacobiApply(w);
                continue;
            }
            if (w.solve == 2) {
                fixedPass(w, it);
                walls(w);
                continue;
            }
            int k = passUntilDone(w, it);
            if (w.friction)
                for (int j = 0; j < k; j++) cycleRound(w, it, position(j), true);
            walls(w);
            w.report[1] += k;
            w.report[2] = std::max(w.report[2], k);
            w.report[3] += std::max(0, w.contactCount[LISTED] - w.capacity);
            // SphereStepper.adapt :118-126
            if (k > w.opening[it]) {
                w.opening[it] = std::min(k, CYCLE);
                w.enough[it] = 0;
            } else if (++w.enough[it] >= SHRINK_AFTER && w.opening[it] > BATCH) {
                w.opening[it] -= BATCH;
                w.enough[it] = 0;
            }
        }
        velocity(w);
        bounce(w);
    }
    show(w);
}

}  // namespace

extern "C" {

// fields: 0 x 1 y 2 z 3 u 4 v 5 w 6 r 7 im 8-10 cx cy cz 11-13 dx dy dz 14-16 ax ay az 17-19 tx ty tz 20-23 q
// solve: 0 Jacobi, 1 Gauss-Seidel over the contact list run until done, 2 the same with `rounds` rounds a pass.
// nx = 0: no grid (every pair; Jacobi only).
void* orc_sphere_create(int n, int substeps, int iterations, int solve, int rounds, int nx, int ny, int nz, float cell,
                        int per_sphere) {
    World* w = new World();
    w->n = n;
    w->substeps = substeps;
    w->iterations = iterations;
    w->solve = solve;
    w->rounds = rounds;
    w->gridded = nx > 0;
    if (!w->gridded) nx = ny = nz = 1;
    w->capacity = n * per_sphere;
    w->nx = nx;
    w->ny = ny;
    w->nz = nz;
    w->cell = cell;
    for (int k = 0; k < FIELDS; k++) w->f[k].assign(n, 0.0f);
    w->f[FQW].assign(n, 1.0f);
    std::memset(w->params, 0, sizeof(w->params));
    w->shown.assign((size_t)n * SHOWN_STRIDE, 0.0f);
    w->keys.assign(n, 0);
    w->order.assign(n, 0);
    for (int k = 0; k < 3; k++) w->claims[k].assign(n, 0);
    const int cap = w->capacity;
    w->contactA.assign(cap, 0);
    w->contactB.assign(cap, 0);
    w->contactDone.assign(cap, 0);
    w->contactNext.assign(cap, 0);
    w->keptB.assign(cap, 0);
    w->keptNext.assign(cap, 0);
    w->contactHead.assign(n, -1);
    w->keptHead.assign(n, 0);
    w->contactImpulse.assign((size_t)cap * IMPULSE_WORDS, 0.0f);
    w->keptImpulse.assign((size_t)cap * IMPULSE_WORDS, 0.0f);
    w->wallImpulse.assign((size_t)n * WALL_IMPULSE_WORDS, 0.0f);
    w->opening.assign(iterations, BATCH);
    w->enough.assign(iterations, 0);
    return w;
}
void orc_sphere_destroy(void* h) { delete (World*)h; }
void orc_sphere_set_field(void* h, int field, const float* v) {
    World* w = (World*)h;
    std::memcpy(w->f[field].data(), v, sizeof(float) * w->n);
}
void orc_sphere_get_field(void* h, int field, float* out) {
    World* w = (World*)h;
    std::memcpy(out, w->f[field].data(), sizeof(float) * w->n);
}
void orc_sphere_set_params(void* h, const int32_t* bits, int friction) {
    World* w = (World*)h;
    std::memcpy(w->params, bits, sizeof(w->params));
    w->friction = friction;
}
int orc_sphere_step(void* h, int steps, int32_t* report) {
    World* w = (World*)h;
    try {
        for (int k = 0; k < steps; k++) stepOnce(*w);
    } catch (const std::exception&) {
        return 3;
    }
    if (report)
        for (int k = 0; k < 4; k++) report[k] = w->report[k];
    return 0;
}
void orc_sphere_shown(void* h, float* out) {
    World* w = (World*)h;
    std::memcpy(out, w->shown.data(), sizeof(float) * w->shown.size());
}
// The last substep's contact list, sorted by (a, b), with each contact's 7 impulse words; returns its length.
int orc_sphere_contacts(void* h, int32_t* ab, float* impulses, int capacity) {
    World* w = (World*)h;
    int listed = std::min(w->contactCount[LISTED], w->capacity);
    if (!ab) return listed;
    std::vector<int> idx(listed);
    for (int c = 0; c < listed; c++) idx[c] = c;
    std::sort(idx.begin(), idx.end(), [&](int p, int q) {
        return w->contactA[p] != w->contactA[q] ? w->contactA[p] < w->contactA[q] : w->contactB[p] < w->contactB[q];
    });
    for (int k = 0; k < listed && k < capacity; k++) {
        ab[2 * k] = w->contactA[idx[k]];
        ab[2 * k + 1] = w->contactB[idx[k]];
        if (impulses)
            for (int q = 0; q < IMPULSE_WORDS; q++)
                impulses[(size_t)k * IMPULSE_WORDS + q] = w->contactImpulse[(size_t)idx[k] * IMPULSE_WORDS + q];
    }
    return listed;
}
// The list as it lies, in list order: pairs, done marks and impulses; returns its length.
int orc_sphere_list(void* h, int32_t* ab, int32_t* done, float* impulses, int capacity) {
    World* w = (World*)h;
    int listed = std::min(w->contactCount[LISTED], w->capacity);
    for (int c = 0; c < listed && c < capacity; c++) {
        ab[2 * c] = w->contactA[c];
        ab[2 * c + 1] = w->contactB[c];
        if (done) done[c] = w->contactDone[c];
        if (impulses)
            for (int q = 0; q < IMPULSE_WORDS; q++)
                impulses[(size_t)c * IMPULSE_WORDS + q] = w->contactImpulse[(size_t)c * IMPULSE_WORDS + q];
    }
    return listed;
}
void orc_sphere_set_shown(void* h, const float* v) {
    World* w = (World*)h;
    std::memcpy(w->shown.data(), v, sizeof(float) * w->shown.size());
}
void orc_sphere_walls(void* h, float* out) {
    World* w = (World*)h;
    std::memcpy(out, w->wallImpulse.data(), sizeof(float) * w->wallImpulse.size());
}
void orc_sphere_counts(void* h, int32_t* out3) {
    World* w = (World*)h;
    for (int k = 0; k < 3; k++) out3[k] = w->contactCount[k];
}

}  // extern "C"
