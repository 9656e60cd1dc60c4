// The picture of a step, as CUDA: one thread a pixel, one ray, tested against every body exactly, written into a
// headless RGB buffer. Restates the reference's fragment shaders (gui = vexelray-sim-rigid-gui/src/main/java/dev/
// vexelray/sim/rigid/gui/): Picture.java (the camera ray :58-77, sky and checkered floor :122-146, the light :153-176),
// SphereShader.java (a quadratic per sphere against a bounding sphere first :79-105, the sphere squashed by its
// pressing :123-176, its octants :186-214) and BoxShader.java (the bounding sphere :63-79, the slab test in the box's
// frame, a sphere-shaped body's quadratic, the face entered and the edge band :94-191, rotate :197-211). Each
// expression keeps the shader's association order; mix(x, y, a) is x (1 - a) + y a, clamp is min(max(.)).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "vxr.h"

namespace {

struct Cam {
    float eye[3], right[3], up[3], forward[3];
    float aspect, alpha, squash;
    float extent[3];
    int count, width, height;
};

// Picture.java constants (:23-40), as the shaders' f32 constants.
constexpr float TAN_HALF = 0.5f;
constexpr float CHECKER = 0.05f;
__constant__ float LIGHT[3];
__constant__ float SKY_LOW[3] = {0.16f, 0.17f, 0.19f};
__constant__ float SKY_HIGH[3] = {0.05f, 0.06f, 0.08f};
__constant__ float FLOOR_A[3] = {0.30f, 0.31f, 0.33f};
__constant__ float FLOOR_B[3] = {0.24f, 0.25f, 0.27f};
__constant__ float BODY_A[3] = {0.90f, 0.55f, 0.22f};
__constant__ float BODY_B[3] = {0.30f, 0.62f, 0.86f};
constexpr float PALE = 0.45f, MOST_SQUASH = 0.5f, EDGE = 0.06f, EDGE_LIGHT = 0.55f, PARALLEL = 1e-9f;
constexpr int SPHERE_STRIDE = 40, BOX_STRIDE = 20;
// Spheres.show's words (core/sphere/Spheres.java:1654-1675) and Boxes.show's (core/box/Boxes.java:781-799)
constexpr int PRESSED_BEFORE = 8, PRESSED_AFTER = 20, TURNED_BEFORE_S = 32, TURNED_AFTER_S = 36, TRACE = 9,
              LEAN = 6, LEAN_LENGTH = 10;
constexpr int CENTRE_BEFORE = 0, SHAPE = 3, CENTRE_AFTER = 4, HALF = 8, TURNED_BEFORE_B = 12, TURNED_AFTER_B = 16;

__device__ __forceinline__ float mixf(float x, float y, float a) { return x * (1.0f - a) + y * a; }
__device__ __forceinline__ float dot3(const float* a, const float* b) {
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}
__device__ __forceinline__ void cross(const float* x, const float* y, float* z) {
    z[0] = x[1] * y[2] - x[2] * y[1];
    z[1] = x[2] * y[0] - x[0] * y[2];
    z[2] = x[0] * y[1] - x[1] * y[0];
}

// The ray through pixel (i, j), unit length (Picture.Frame :58-77); the top row is uv.y = 0.
__device__ __forceinline__ void ray_of(const Cam& c, int i, int j, float* d) {
    const float u = ((float)i + 0.5f) / (float)c.width, v = ((float)j + 0.5f) / (float)c.height;
    const float px = ((u * 2.0f - 1.0f) * c.aspect) * TAN_HALF;
    const float py = (1.0f - v * 2.0f) * TAN_HALF;
    for (int a = 0; a < 3; a++) d[a] = c.forward[a] + (c.right[a] * px + c.up[a] * py);
    const float inverse = 1.0f / sqrtf(dot3(d, d));
    for (int a = 0; a < 3; a++) d[a] = d[a] * inverse;
}

// Picture.background :122-146.
__device__ __forceinline__ void background(const Cam& c, const float* d, float best, float* rgb) {
    const float up = fminf(fmaxf(d[1] * 0.5f + 0.5f, 0.0f), 1.0f);
    for (int a = 0; a < 3; a++) rgb[a] = mixf(SKY_LOW[a], SKY_HIGH[a], up);
    if (d[1] < -1e-4f) {
        const float t = -c.eye[1] / d[1];
        if (t < best) {
            const float fx = c.eye[0] + t * d[0], fz = c.eye[2] + t * d[2];
            if (fx > 0.0f && fx < c.extent[0] && fz > 0.0f && fz < c.extent[2]) {
                const float s = floorf(fx / CHECKER) + floorf(fz / CHECKER);
                const float odd = s - 2.0f * floorf(s / 2.0f);
                for (int a = 0; a < 3; a++) rgb[a] = mixf(FLOOR_A[a], FLOOR_B[a], odd);
            }
        }
    }
}

// Picture.shade :153-176.
__device__ __forceinline__ void shade(const float* d, float hit, float* n, float pale, float* rgb) {
    const float nl = 1.0f / sqrtf(dot3(n, n));
    for (int a = 0; a < 3; a++) n[a] = n[a] * nl;
    const float diffuse = fmaxf(0.0f, (n[0] * LIGHT[0] + n[1] * LIGHT[1]) + n[2] * LIGHT[2]);
    float h[3];
    for (int a = 0; a < 3; a++) h[a] = LIGHT[a] - d[a];
    const float hl = 1.0f / sqrtf(dot3(h, h));
    const float nh = fmaxf(0.0f, dot3(n, h) * hl);
    const float nh2 = nh * nh;
    const float nh8 = (nh2 * nh2) * (nh2 * nh2);
    const float spec = 0.35f * (nh8 * (nh8 * nh8));
    const float g = hit * 0.618034f;
    const float tint = g - floorf(g);
    const float light = 0.22f + 0.78f * diffuse;
    for (int a = 0; a < 3; a++) {
        const float colour = mixf(mixf(BODY_A[a], BODY_B[a], tint), 1.0f, pale);
        rgb[a] = colour * light + spec;
    }
}

// The symmetric m (xx, yy, zz, xy, xz, yz) times x (SphereShader.times :262-270).
__device__ __forceinline__ void times(const float* m, const float* x, float* y) {
    const int row[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
    for (int a = 0; a < 3; a++) y[a] = m[row[a][0]] * x[0] + (m[row[a][1]] * x[1] + m[row[a][2]] * x[2]);
}

// ---- a frame's bodies: what no pixel changes ---------------------------------------------------------------------
// For each body, once a frame: o = eye - its blended centre, the bounding sphere's radius R, and |o|^2 - R^2 (the
// part of the bounding test's discriminant no pixel changes), each computed as the shaders compute it, so the pixels'
// results are the same to the bit as computing them per pixel.

constexpr int TILE = 16, THREADS = TILE * TILE, LIST = 1024;

__device__ __forceinline__ float sphere_bound(const Cam& c, const float* s, float* gain_out, float* lift_out) {
    const float r = s[3];
    const float trace = mixf(s[PRESSED_BEFORE + TRACE], s[PRESSED_AFTER + TRACE], c.alpha);
    const float lean_length = mixf(s[PRESSED_BEFORE + LEAN_LENGTH], s[PRESSED_AFTER + LEAN_LENGTH], c.alpha);
    const float gain = fminf(c.squash, MOST_SQUASH / fmaxf(trace, 1e-9f));
    const float lift = fmaxf(0.0f, gain * (2.0f / 3.0f) - 1.0f);
    *gain_out = gain;
    *lift_out = lift;
    return r * (1.0f + 0.53f * (gain * trace)) + lift * (r * lean_length);
}

template <int SHAPE>
__global__ void k_picture_bodies(Cam c, const float* __restrict__ shown, float4* __restrict__ pre,
                                 float* __restrict__ reach) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.count) return;
    float o[3], cc, R;
    if (SHAPE == VXR_RING_SPHERES) {
        const float* s = shown + (size_t)k * SPHERE_STRIDE;
        for (int a = 0; a < 3; a++) o[a] = c.eye[a] - mixf(s[a], s[4 + a], c.alpha);
        float gain, lift;
        const float bound = sphere_bound(c, s, &gain, &lift);
        cc = dot3(o, o) - bound * bound;
        R = bound;
    } else {
        const float* s = shown + (size_t)k * BOX_STRIDE;
        float half[3];
        for (int a = 0; a < 3; a++) {
            o[a] = c.eye[a] - mixf(s[CENTRE_BEFORE + a], s[CENTRE_AFTER + a], c.alpha);
            half[a] = s[HALF + a];
        }
        const float reach2 = dot3(half, half);
        cc = dot3(o, o) - reach2;
        R = sqrtf(reach2);
    }
    pre[k] = make_float4(o[0], o[1], o[2], cc);
    reach[k] = R;
}

// ---- one body against one pixel's ray, past the bounding test ------------------------------------------------------

struct SphereHit {
    float best = 1e30f, hit = -1.0f;
    float normal[3] = {0, 0, 0}, local[3] = {0, 0, 0};
};

// SphereShader.squashed :158-214
__device__ __forceinline__ void squashed(const Cam& c, const float* __restrict__ shown, int k, const float* d,
                                         SphereHit& h) {
    const float* s = shown + (size_t)k * SPHERE_STRIDE;
    float ctr[3];
    for (int a = 0; a < 3; a++) ctr[a] = mixf(s[a], s[4 + a], c.alpha);
    const float r = s[3];
    float gain, lift;
    sphere_bound(c, s, &gain, &lift);
    float m[6];
    for (int q = 0; q < 6; q++) {
        const float pressed = gain * mixf(s[PRESSED_BEFORE + q], s[PRESSED_AFTER + q], c.alpha);
        m[q] = q < 3 ? 1.0f - pressed : -pressed;
    }
    const float adj[6] = {m[1] * m[2] - m[5] * m[5], m[0] * m[2] - m[4] * m[4], m[0] * m[1] - m[3] * m[3],
                          m[4] * m[5] - m[3] * m[2], m[3] * m[5] - m[4] * m[1], m[3] * m[4] - m[0] * m[5]};
    const float det = m[0] * adj[0] + (m[3] * adj[3] + m[4] * adj[4]);
    float cube = 1.0f - (3.0f - (m[0] + (m[1] + m[2]))) / 3.0f;
    for (int step = 0; step < 2; step++) cube = (2.0f * cube + det / (cube * cube)) / 3.0f;
    const float scale = cube / det;
    float inv[6];
    for (int q = 0; q < 6; q++) inv[q] = adj[q] * scale;
    float om[3];
    for (int a = 0; a < 3; a++) {
        const float moved = ctr[a] + (lift * r) * mixf(s[PRESSED_BEFORE + LEAN + a], s[PRESSED_AFTER + LEAN + a], c.alpha);
        om[a] = c.eye[a] - moved;
    }
    float os[3], ds[3];
    times(inv, om, os);
    times(inv, d, ds);
    const float aa = dot3(ds, ds), hh = dot3(os, ds);
    const float disc = hh * hh - aa * (dot3(os, os) - r * r);
    if (!(disc > 0.0f)) return;
    const float t = (-hh - sqrtf(disc)) / aa;
    if (!(t > 0.0f && t < h.best)) return;
    h.best = t;
    h.hit = (float)k;
    float u[3];
    for (int a = 0; a < 3; a++) {
        u[a] = os[a] + t * ds[a];
        h.local[a] = u[a];
    }
    times(inv, u, h.normal);
}

// SphereShader.fragmentSpirv's colour (:131-140) and turned (:225-253): the octant in the sphere's own frame, the
// orientation blended the short way round.
__device__ __forceinline__ void sphere_colour(const Cam& c, const float* __restrict__ shown, const float* d,
                                              SphereHit& h, float* rgb) {
    background(c, d, h.best, rgb);
    if (!(h.hit > -0.5f)) return;
    const float* s = shown + (size_t)(int)h.hit * SPHERE_STRIDE;
    const float* before = s + TURNED_BEFORE_S;
    const float* after = s + TURNED_AFTER_S;
    float way = 1.0f;
    if (dot3(before, after) + before[3] * after[3] < 0.0f) way = -1.0f;
    float q[3];
    for (int a = 0; a < 3; a++) q[a] = -mixf(before[a] * way, after[a], c.alpha);
    const float w = mixf(before[3] * way, after[3], c.alpha);
    float t[3], qt[3];
    cross(q, h.local, t);
    for (int a = 0; a < 3; a++) t[a] = 2.0f * t[a];
    cross(q, t, qt);
    float p[3];
    for (int a = 0; a < 3; a++) p[a] = h.local[a] + (w * t[a] + qt[a]);
    const float patch = (p[0] * p[1]) * p[2] > 0.0f ? PALE : 0.0f;
    shade(d, h.hit, h.normal, patch, rgb);
}

// BoxShader.rotate :197-211: p turned by q of any length.
__device__ __forceinline__ void rotate(const float* q, const float* p, float* out) {
    const float twice = 2.0f / ((q[0] * q[0] + q[1] * q[1]) + (q[2] * q[2] + q[3] * q[3]));
    float t[3], qt[3];
    cross(q, p, t);
    for (int a = 0; a < 3; a++) t[a] = twice * t[a];
    cross(q, t, qt);
    for (int a = 0; a < 3; a++) out[a] = p[a] + (q[3] * t[a] + qt[a]);
}

struct BoxHit {
    float best = 1e30f, hit = -1.0f, edged = 0.0f, pale = 0.0f;
    float normal[3] = {0, 0, 0};
};

// BoxShader.slabs :115-190; o is the eye less the box's blended centre.
__device__ __forceinline__ void slabs(const Cam& c, const float* __restrict__ shown, int k, const float* o,
                                      const float* d, BoxHit& h) {
    const float* s = shown + (size_t)k * BOX_STRIDE;
    float half[3];
    for (int a = 0; a < 3; a++) half[a] = s[HALF + a];
    const float* before = s + TURNED_BEFORE_B;
    const float* after = s + TURNED_AFTER_B;
    float way = 1.0f;
    if (dot3(before, after) + before[3] * after[3] < 0.0f) way = -1.0f;
    float q[4];
    for (int a = 0; a < 4; a++) q[a] = mixf(before[a] * way, after[a], c.alpha);
    const float inverse[4] = {-q[0], -q[1], -q[2], q[3]};
    float os[3], ds[3];
    rotate(inverse, o, os);
    rotate(inverse, d, ds);
    const float round = s[SHAPE];
    if (round > 0.5f) {
        const float hh = dot3(os, ds);
        const float cc = dot3(os, os) - half[0] * half[0];
        const float bdisc = hh * hh - dot3(ds, ds) * cc;
        if (bdisc > 0.0f) {
            const float t = (-hh - sqrtf(bdisc)) / dot3(ds, ds);
            if (t > 0.0f && t < h.best) {
                h.best = t;
                h.hit = (float)k;
                float own[3];
                for (int a = 0; a < 3; a++) own[a] = os[a] + t * ds[a];
                rotate(q, own, h.normal);
                h.edged = 0.0f;
                h.pale = (own[0] * own[1]) * own[2] > 0.0f ? 1.0f : 0.0f;
            }
        }
    }
    float enter = -1e30f, leave = 1e30f, face = 0.0f;
    for (int a = 0; a < 3; a++) {
        float step = ds[a];
        if (fabsf(step) < PARALLEL) step = PARALLEL;
        const float t1 = (-half[a] - os[a]) / step;
        const float t2 = (half[a] - os[a]) / step;
        const float near = fminf(t1, t2);
        leave = fminf(leave, fmaxf(t1, t2));
        if (near > enter) {
            enter = near;
            face = (float)a;
        }
    }
    if (enter < leave && enter > 0.0f && enter < h.best && !(round > 0.5f)) {
        h.best = enter;
        h.hit = (float)k;
        float own[3], gap[3];
        for (int a = 0; a < 3; a++) {
            const float on = (face > (float)a - 0.5f && face < (float)a + 0.5f) ? 1.0f : 0.0f;
            own[a] = -(on * ds[a]);
            const float p = os[a] + enter * ds[a];
            gap[a] = half[a] - fabsf(p);
        }
        rotate(q, own, h.normal);
        const float sum = (gap[0] + gap[1]) + gap[2];
        const float least = fminf(gap[0], fminf(gap[1], gap[2]));
        const float most = fmaxf(gap[0], fmaxf(gap[1], gap[2]));
        const float to_edge = (sum - least) - most;
        const float band = EDGE * fminf(half[0], fminf(half[1], half[2]));
        h.edged = to_edge < band ? 1.0f : 0.0f;
        h.pale = 0.0f;
    }
}

__device__ __forceinline__ void box_colour(const Cam& c, const float* d, BoxHit& h, float* rgb) {
    background(c, d, h.best, rgb);
    if (!(h.hit > -0.5f)) return;
    shade(d, h.hit, h.normal, PALE * h.pale, rgb);
    for (int a = 0; a < 3; a++) rgb[a] = rgb[a] * mixf(1.0f, EDGE_LIGHT, h.edged);
}

// ---- a tile of pixels ----------------------------------------------------------------------------------------------
// One block a 16 x 16 tile. The block first keeps, in ascending order, the bodies whose bounding sphere can meet a
// ray of the tile: those within R (plus a slack far above f32 rounding) of the inside of the four planes through the
// eye and the tile's corner rays. Every pixel then runs the shaders' loop over the kept bodies alone. A body left out
// is one whose bounding test fails at every pixel of the tile, so it changes nothing there: the picture is the one the
// shaders' loop over every body gives, to the bit.

// The side planes of the tile's rays, through the eye, inward: from the f32 corner rays, in doubles, so that the
// planes hold those rays exactly; a plane whose corner rays coincide (a tile one pixel wide or high) is left out.
__device__ void tile_planes(const Cam& c, int i0, int j0, int i1, int j1, float (*plane)[4]) {
    const int q = threadIdx.y * blockDim.x + threadIdx.x;
    if (q >= 4) return;
    float f[4][3];
    ray_of(c, i0, j0, f[0]);
    ray_of(c, i1, j0, f[1]);
    ray_of(c, i1, j1, f[2]);
    ray_of(c, i0, j1, f[3]);
    const float* x = f[q];
    const float* y = f[(q + 1) & 3];
    double n[3] = {(double)x[1] * y[2] - (double)x[2] * y[1], (double)x[2] * y[0] - (double)x[0] * y[2],
                   (double)x[0] * y[1] - (double)x[1] * y[0]};
    double inward = 0.0;
    for (int a = 0; a < 3; a++) inward += n[a] * ((double)f[0][a] + f[1][a] + f[2][a] + f[3][a]);
    const double len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    const double sign = inward < 0.0 ? -1.0 : 1.0;
    for (int a = 0; a < 3; a++) plane[q][a] = len > 0.0 ? (float)(sign * n[a] / len) : 0.0f;
    plane[q][3] = len > 0.0 ? 1.0f : 0.0f;
}

// Whether a body's bounding sphere can meet a ray inside the four planes: within R plus a slack of each plane's
// inside. Rounding in the pixels' f32 tests moves a ray's reach by far less than the slack (1e-6 relative at most).
__device__ __forceinline__ bool may_meet(float4 p, float R, const float (*plane)[4]) {
    const float len = sqrtf(p.x * p.x + p.y * p.y + p.z * p.z);
    const float slack = R + 1e-5f * (R + len + len * (len / fmaxf(R, 1e-20f)));
    bool keep = true;
    for (int q = 0; q < 4; q++) {
        if (plane[q][3] == 0.0f) continue;
        const float inside_by = -(p.x * plane[q][0] + p.y * plane[q][1] + p.z * plane[q][2]);
        if (inside_by < -slack) keep = false;
    }
    return keep;
}

// Block-wide ordered compaction: this thread's place among the kept of its block's chunk (warp by warp, lane by
// lane), and the chunk's kept count. Every thread of the block calls it; `tid` is its flat index in a block of
// THREADS (whatever the block's shape).
__device__ __forceinline__ int kept_before(bool keep, int tid, int* s_warp, int& total) {
    const int lane = tid & 31, warp = tid >> 5;
    const unsigned vote = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) s_warp[warp] = __popc(vote);
    __syncthreads();
    int before = 0;
    total = 0;
    for (int w = 0; w < THREADS / 32; w++) {
        const int n = s_warp[w];
        before += w < warp ? n : 0;
        total += n;
    }
    return before + __popc(vote & ((1u << lane) - 1u));
}

// Scenes of many bodies: one block a super-tile of SUPER x SUPER pixels keeps, in ascending order, the bodies that
// may meet a ray of it; its tiles then test only those. A super-tile's rays lie inside its corner rays' planes and
// hold every ray of its tiles, so a body left out here is one every tile of it would leave out. More than `cap`
// kept: the list is marked full and its tiles test every body.
constexpr int SUPER = 64, SUPER_FROM = 2048, SUPER_CAP = 16384;

__global__ void __launch_bounds__(THREADS) k_picture_super(Cam c, const float4* __restrict__ pre,
                                                           const float* __restrict__ reach, int* __restrict__ list,
                                                           int* __restrict__ list_n, int cap) {
    __shared__ float s_plane[4][4];
    __shared__ int s_warp[THREADS / 32];
    const int supers_x = (c.width + SUPER - 1) / SUPER;
    const int st = blockIdx.x;
    const int i0 = (st % supers_x) * SUPER, j0 = (st / supers_x) * SUPER;
    const int i1 = min(i0 + SUPER - 1, c.width - 1), j1 = min(j0 + SUPER - 1, c.height - 1);
    tile_planes(c, i0, j0, i1, j1, s_plane);
    __syncthreads();
    int* mine = list + (size_t)st * cap;
    int listed = 0;
    for (int base = 0; base < c.count; base += THREADS) {
        const int k = base + threadIdx.x;
        const bool keep = k < c.count && may_meet(pre[k], reach[k], s_plane);
        int total;
        const int at = listed + kept_before(keep, threadIdx.x, s_warp, total);
        if (keep && at < cap) mine[at] = k;
        listed += total;
        __syncthreads();  // s_warp is written again by the next chunk
    }
    if (threadIdx.x == 0) list_n[st] = listed;
}

template <int SHAPE>
__global__ void __launch_bounds__(THREADS) k_picture(Cam c, const float* __restrict__ shown,
                                                     const float4* __restrict__ pre, const float* __restrict__ reach,
                                                     const int* __restrict__ list, const int* __restrict__ list_n,
                                                     int cap, float* __restrict__ out) {
    __shared__ float4 s_pre[LIST];
    __shared__ int s_body[LIST];
    __shared__ float s_plane[4][4];
    __shared__ int s_warp[THREADS / 32];
    const int tid = threadIdx.y * TILE + threadIdx.x;
    const int i0 = blockIdx.x * TILE, j0 = blockIdx.y * TILE;
    const int i1 = min(i0 + TILE - 1, c.width - 1), j1 = min(j0 + TILE - 1, c.height - 1);
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
    const bool inside = i < c.width && j < c.height;
    float d[3];
    ray_of(c, min(i, c.width - 1), min(j, c.height - 1), d);
    tile_planes(c, i0, j0, i1, j1, s_plane);
    // the bodies to go through: the super-tile's list, or every body (no lists, or the list overflowed)
    const int* from = nullptr;
    int m = c.count;
    if (list) {
        const int st = (j0 / SUPER) * ((c.width + SUPER - 1) / SUPER) + i0 / SUPER;
        const int kept = list_n[st];
        if (kept <= cap) {
            from = list + (size_t)st * cap;
            m = kept;
        }
    }
    __syncthreads();
    SphereHit sh;
    BoxHit bh;
    int listed = 0;
    for (int base = 0; base < m; base += THREADS) {
        const int e = base + tid;
        bool keep = false;
        int k = 0;
        float4 p = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (e < m) {
            k = from ? from[e] : e;
            p = pre[k];
            keep = may_meet(p, reach[k], s_plane);
        }
        int total;
        const int at = listed + kept_before(keep, tid, s_warp, total);
        if (keep) {
            s_pre[at] = p;
            s_body[at] = k;
        }
        listed += total;
        __syncthreads();
        if (listed > LIST - THREADS || base + THREADS >= m) {
            if (inside) {
                for (int e = 0; e < listed; e++) {
                    const float4 v = s_pre[e];
                    const float o[3] = {v.x, v.y, v.z};
                    const float half = dot3(o, d);
                    const float disc = half * half - v.w;
                    if (!(disc > 0.0f)) continue;
                    const float root = sqrtf(disc);
                    const float best = SHAPE == VXR_RING_SPHERES ? sh.best : bh.best;
                    if (!(root - half > 0.0f && -half - root < best)) continue;
                    if (SHAPE == VXR_RING_SPHERES)
                        squashed(c, shown, s_body[e], d, sh);
                    else
                        slabs(c, shown, s_body[e], o, d, bh);
                }
            }
            listed = 0;
            __syncthreads();
        }
    }
    if (!inside) return;
    float rgb[3];
    if (SHAPE == VXR_RING_SPHERES)
        sphere_colour(c, shown, d, sh, rgb);
    else
        box_colour(c, d, bh, rgb);
    float* o = out + 3 * ((size_t)j * c.width + i);
    o[0] = rgb[0];
    o[1] = rgb[1];
    o[2] = rgb[2];
}

Cam cam_of(const vxr_camera* k, int count, int width, int height) {
    Cam c;
    for (int a = 0; a < 3; a++) {
        c.eye[a] = k->eye[a];
        c.right[a] = k->right[a];
        c.up[a] = k->up[a];
        c.forward[a] = k->forward[a];
        c.extent[a] = k->extent[a];
    }
    c.aspect = k->aspect;
    c.alpha = k->alpha;
    c.squash = k->squash;
    c.count = count;
    c.width = width;
    c.height = height;
    return c;
}

bool light_set = false;

int set_light() {
    if (light_set) return VXR_OK;
    // (0.35, 0.85, 0.4) normalised in doubles, then rounded (Picture.LIGHT :27)
    const double x = 0.35, y = 0.85, z = 0.4, len = std::sqrt(x * x + y * y + z * z);
    const float l[3] = {(float)(x / len), (float)(y / len), (float)(z / len)};
    if (cudaMemcpyToSymbol(LIGHT, l, sizeof(l)) != cudaSuccess) return VXR_ECUDA;
    light_set = true;
    return VXR_OK;
}

}  // namespace

extern "C" {

int32_t vxr_picture(int32_t shape, const float* shown, int32_t count, const vxr_camera* camera, int32_t width,
                    int32_t height, float* rgb, void* stream) {
    if (!shown || !camera || !rgb || count < 0 || width < 1 || height < 1) return VXR_EINVAL;
    if (shape != VXR_RING_SPHERES && shape != VXR_RING_BOXES) return VXR_EINVAL;
    if (set_light() != VXR_OK) return VXR_ECUDA;
    const Cam c = cam_of(camera, count, width, height);
    cudaStream_t st = (cudaStream_t)stream;
    const int supers = ((width + SUPER - 1) / SUPER) * ((height + SUPER - 1) / SUPER);
    const bool use_supers = count >= SUPER_FROM;
    const int cap = std::min(count, SUPER_CAP);
    float4* pre = nullptr;
    float* reach = nullptr;
    int *list = nullptr, *list_n = nullptr;
    if (count > 0) {
        // a frame's scratch from the stream-ordered pool: no synchronisation, nothing shared between streams
        size_t bytes = (size_t)count * (sizeof(float4) + sizeof(float));
        if (use_supers) bytes += (size_t)supers * (cap + 1) * sizeof(int);
        void* scratch = nullptr;
        if (cudaMallocAsync(&scratch, bytes, st) != cudaSuccess) return VXR_ECUDA;
        pre = (float4*)scratch;
        reach = (float*)(pre + count);
        if (use_supers) {
            list_n = (int*)(reach + count);
            list = list_n + supers;
        }
        const int blocks = (count + 255) / 256;
        if (shape == VXR_RING_SPHERES)
            k_picture_bodies<VXR_RING_SPHERES><<<blocks, 256, 0, st>>>(c, shown, pre, reach);
        else
            k_picture_bodies<VXR_RING_BOXES><<<blocks, 256, 0, st>>>(c, shown, pre, reach);
        if (use_supers) k_picture_super<<<supers, THREADS, 0, st>>>(c, pre, reach, list, list_n, cap);
    }
    const dim3 block(TILE, TILE), grid((width + TILE - 1) / TILE, (height + TILE - 1) / TILE);
    if (shape == VXR_RING_SPHERES)
        k_picture<VXR_RING_SPHERES><<<grid, block, 0, st>>>(c, shown, pre, reach, list, list_n, cap, rgb);
    else
        k_picture<VXR_RING_BOXES><<<grid, block, 0, st>>>(c, shown, pre, reach, list, list_n, cap, rgb);
    if (pre && cudaFreeAsync(pre, st) != cudaSuccess) return VXR_ECUDA;
    return cudaGetLastError() == cudaSuccess ? VXR_OK : VXR_ECUDA;
}

int32_t vxr_picture_host(int32_t shape, const float* shown_host, int32_t count, const vxr_camera* camera,
                         int32_t width, int32_t height, float* rgb_host) {
    if (!shown_host || !camera || !rgb_host || count < 0 || width < 1 || height < 1) return VXR_EINVAL;
    const size_t words = (size_t)count * (shape == VXR_RING_SPHERES ? SPHERE_STRIDE : BOX_STRIDE);
    const size_t pixels = (size_t)width * height * 3;
    float *s = nullptr, *o = nullptr;
    if (cudaMalloc(&s, sizeof(float) * std::max<size_t>(words, 1)) != cudaSuccess) return VXR_ECUDA;
    if (cudaMalloc(&o, sizeof(float) * pixels) != cudaSuccess) {
        cudaFree(s);
        return VXR_ECUDA;
    }
    int rc = VXR_OK;
    if (words && cudaMemcpy(s, shown_host, sizeof(float) * words, cudaMemcpyHostToDevice) != cudaSuccess) rc = VXR_ECUDA;
    if (rc == VXR_OK) rc = vxr_picture(shape, s, count, camera, width, height, o, nullptr);
    if (rc == VXR_OK && cudaMemcpy(rgb_host, o, sizeof(float) * pixels, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = VXR_ECUDA;
    cudaFree(s);
    cudaFree(o);
    return rc;
}

}  // extern "C"
