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

__global__ void k_picture_spheres(Cam c, const float* __restrict__ shown, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= c.width || j >= c.height) return;
    float d[3];
    ray_of(c, i, j, d);
    float best = 1e30f, hit = -1.0f;
    float normal[3] = {0, 0, 0}, local[3] = {0, 0, 0};
    for (int k = 0; k < c.count; k++) {
        const float* s = shown + (size_t)k * SPHERE_STRIDE;
        float ctr[3], o[3];
        for (int a = 0; a < 3; a++) {
            ctr[a] = mixf(s[a], s[4 + a], c.alpha);
            o[a] = c.eye[a] - ctr[a];
        }
        const float r = s[3];
        const float trace = mixf(s[PRESSED_BEFORE + TRACE], s[PRESSED_AFTER + TRACE], c.alpha);
        const float lean_length = mixf(s[PRESSED_BEFORE + LEAN_LENGTH], s[PRESSED_AFTER + LEAN_LENGTH], c.alpha);
        const float gain = fminf(c.squash, MOST_SQUASH / fmaxf(trace, 1e-9f));
        const float lift = fmaxf(0.0f, gain * (2.0f / 3.0f) - 1.0f);
        const float bound = r * (1.0f + 0.53f * (gain * trace)) + lift * (r * lean_length);
        const float half = dot3(o, d);
        const float disc = half * half - (dot3(o, o) - bound * bound);
        if (!(disc > 0.0f)) continue;
        const float root = sqrtf(disc);
        if (!(root - half > 0.0f && -half - root < best)) continue;
        // squashed :123-176
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
        const float disc2 = hh * hh - aa * (dot3(os, os) - r * r);
        if (!(disc2 > 0.0f)) continue;
        const float t = (-hh - sqrtf(disc2)) / aa;
        if (!(t > 0.0f && t < best)) continue;
        best = t;
        hit = (float)k;
        float u[3];
        for (int a = 0; a < 3; a++) {
            u[a] = os[a] + t * ds[a];
            local[a] = u[a];
        }
        times(inv, u, normal);
    }
    float rgb[3];
    background(c, d, best, rgb);
    if (hit > -0.5f) {
        // turned :186-214: the octant in the sphere's own frame, the orientation blended the short way round
        const float* s = shown + (size_t)(int)hit * SPHERE_STRIDE;
        const float* before = s + TURNED_BEFORE_S;
        const float* after = s + TURNED_AFTER_S;
        float way = 1.0f;
        if (dot3(before, after) + before[3] * after[3] < 0.0f) way = -1.0f;
        float q[3];
        for (int a = 0; a < 3; a++) q[a] = -mixf(before[a] * way, after[a], c.alpha);
        const float w = mixf(before[3] * way, after[3], c.alpha);
        float t[3], qt[3];
        cross(q, local, t);
        for (int a = 0; a < 3; a++) t[a] = 2.0f * t[a];
        cross(q, t, qt);
        float p[3];
        for (int a = 0; a < 3; a++) p[a] = local[a] + (w * t[a] + qt[a]);
        const float patch = (p[0] * p[1]) * p[2] > 0.0f ? PALE : 0.0f;
        shade(d, hit, normal, patch, rgb);
    }
    float* o = out + 3 * ((size_t)j * c.width + i);
    o[0] = rgb[0];
    o[1] = rgb[1];
    o[2] = rgb[2];
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

__global__ void k_picture_boxes(Cam c, const float* __restrict__ shown, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= c.width || j >= c.height) return;
    float d[3];
    ray_of(c, i, j, d);
    float best = 1e30f, hit = -1.0f, edged = 0.0f, pale = 0.0f;
    float normal[3] = {0, 0, 0};
    for (int k = 0; k < c.count; k++) {
        const float* s = shown + (size_t)k * BOX_STRIDE;
        float o[3], half[3];
        for (int a = 0; a < 3; a++) {
            o[a] = c.eye[a] - mixf(s[CENTRE_BEFORE + a], s[CENTRE_AFTER + a], c.alpha);
            half[a] = s[HALF + a];
        }
        const float reach2 = dot3(half, half);
        const float along = dot3(o, d);
        const float disc = along * along - (dot3(o, o) - reach2);
        if (!(disc > 0.0f)) continue;
        const float root = sqrtf(disc);
        if (!(root - along > 0.0f && -along - root < best)) continue;
        // slabs :94-191
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
                if (t > 0.0f && t < best) {
                    best = t;
                    hit = (float)k;
                    float own[3];
                    for (int a = 0; a < 3; a++) own[a] = os[a] + t * ds[a];
                    rotate(q, own, normal);
                    edged = 0.0f;
                    pale = (own[0] * own[1]) * own[2] > 0.0f ? 1.0f : 0.0f;
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
        if (enter < leave && enter > 0.0f && enter < best && !(round > 0.5f)) {
            best = enter;
            hit = (float)k;
            float own[3], gap[3];
            for (int a = 0; a < 3; a++) {
                const float on = (face > (float)a - 0.5f && face < (float)a + 0.5f) ? 1.0f : 0.0f;
                own[a] = -(on * ds[a]);
                const float p = os[a] + enter * ds[a];
                gap[a] = half[a] - fabsf(p);
            }
            rotate(q, own, normal);
            const float sum = (gap[0] + gap[1]) + gap[2];
            const float least = fminf(gap[0], fminf(gap[1], gap[2]));
            const float most = fmaxf(gap[0], fmaxf(gap[1], gap[2]));
            const float to_edge = (sum - least) - most;
            const float band = EDGE * fminf(half[0], fminf(half[1], half[2]));
            edged = to_edge < band ? 1.0f : 0.0f;
            pale = 0.0f;
        }
    }
    float rgb[3];
    background(c, d, best, rgb);
    if (hit > -0.5f) {
        shade(d, hit, normal, PALE * pale, rgb);
        for (int a = 0; a < 3; a++) rgb[a] = rgb[a] * mixf(1.0f, EDGE_LIGHT, edged);
    }
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
    const dim3 block(16, 16), grid((width + 15) / 16, (height + 15) / 16);
    cudaStream_t st = (cudaStream_t)stream;
    if (shape == VXR_RING_SPHERES)
        k_picture_spheres<<<grid, block, 0, st>>>(c, shown, rgb);
    else
        k_picture_boxes<<<grid, block, 0, st>>>(c, shown, rgb);
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
