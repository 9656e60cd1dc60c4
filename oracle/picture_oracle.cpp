// CPU ORACLE — test infrastructure only, never part of the product path.
//
// A single-precision C++ restatement of the reference's two fragment shaders, pixel by pixel, for the picture's
// parity tests: each expression in the shader's own association order, build with -ffp-contract=off. GLSL's
// mix(x, y, a) is taken as x (1 - a) + y a and clamp as min(max(.)); the reference holds no rendered pictures, so
// these choices are this restatement's and the parity it gives is unpinned against the reference's GPU.
//
// Files restated (gui = vexelray-sim-rigid-gui/src/main/java/dev/vexelray/sim/rigid/gui/):
//   gui/Picture.java       Frame (the ray) :87-107, background :122-147, shade :154-181, push :202-216,
//                          LIGHT :68 and the colours :70-75
//   gui/SphereShader.java  fragmentSpirv :99-141, squashed :158-214, turned :225-253, pressing :263-266, times
//                          :269-277; the shown words of core/sphere/Spheres.java:1653-1668
//   gui/BoxShader.java     fragmentSpirv :68-109, slabs :115-190, rotate :196-211; the shown words of
//                          core/box/Boxes.java:781-791
//
// Only tests/ and __graft_entry__.smoke() load this library.
#include <cmath>
#include <cstdint>

namespace {

typedef float V3[3];

struct Push {  // Picture.MEMBERS, in order
    float e[3], r[3], u[3], f[3];
    float aspect, alpha, count, sx, sy, sz, squash;
};

float light(int a) {
    const double x = 0.35, y = 0.85, z = 0.4;
    const double length = std::sqrt(x * x + y * y + z * z);
    const double l[3] = {x / length, y / length, z / length};
    return (float)l[a];
}

const double SKY_LOW[3] = {0.16, 0.17, 0.19}, SKY_HIGH[3] = {0.05, 0.06, 0.08};
const double FLOOR_A[3] = {0.30, 0.31, 0.33}, FLOOR_B[3] = {0.24, 0.25, 0.27};
const double BODY_A[3] = {0.90, 0.55, 0.22}, BODY_B[3] = {0.30, 0.62, 0.86};

inline float F(double x) { return (float)x; }
inline float mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }
inline float dot(const float* a, const float* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }
inline float fmin_(float a, float b) { return std::fmin(a, b); }
inline float fmax_(float a, float b) { return std::fmax(a, b); }

struct Frame {
    float eye[3], d[3], alpha, sx, sz, squash;
    int count;
};

// Picture.Frame: uv the pixel's centre, its top row v = 0.
Frame frame_of(const Push& p, float uvx, float uvy) {
    Frame fr;
    for (int a = 0; a < 3; a++) fr.eye[a] = p.e[a];
    fr.alpha = p.alpha;
    fr.count = (int)p.count;
    fr.sx = p.sx;
    fr.sz = p.sz;
    fr.squash = p.squash;
    const float px = ((uvx * F(2) - F(1)) * p.aspect) * F(0.5);
    const float py = (F(1) - uvy * F(2)) * F(0.5);
    for (int a = 0; a < 3; a++) fr.d[a] = p.f[a] + (p.r[a] * px + p.u[a] * py);
    const float inverse = F(1) / std::sqrt(dot(fr.d, fr.d));
    for (int a = 0; a < 3; a++) fr.d[a] = fr.d[a] * inverse;
    return fr;
}

void background(const Frame& fr, float best, float* rgb) {
    const float up = fmin_(fmax_(fr.d[1] * F(0.5) + F(0.5), F(0)), F(1));
    for (int a = 0; a < 3; a++) rgb[a] = mix(F(SKY_LOW[a]), F(SKY_HIGH[a]), up);
    if (fr.d[1] < F(-1e-4)) {
        const float t = -fr.eye[1] / fr.d[1];
        if (t < best) {
            const float fx = fr.eye[0] + t * fr.d[0];
            const float fz = fr.eye[2] + t * fr.d[2];
            if ((fx > F(0) && fx < fr.sx) && (fz > F(0) && fz < fr.sz)) {
                const float s = std::floor(fx / F(0.05)) + std::floor(fz / F(0.05));
                const float odd = s - F(2) * std::floor(s / F(2));
                for (int a = 0; a < 3; a++) rgb[a] = mix(F(FLOOR_A[a]), F(FLOOR_B[a]), odd);
            }
        }
    }
}

void shade(float* rgb, const Frame& fr, float hit, float* n, float pale) {
    const float nl = F(1) / std::sqrt(dot(n, n));
    for (int a = 0; a < 3; a++) n[a] = n[a] * nl;
    const float diffuse = fmax_(F(0), (n[0] * light(0) + n[1] * light(1)) + n[2] * light(2));
    float h[3];
    for (int a = 0; a < 3; a++) h[a] = light(a) - fr.d[a];
    const float hl = F(1) / std::sqrt(dot(h, h));
    const float nh = fmax_(F(0), dot(n, h) * hl);
    const float nh2 = nh * nh;
    const float nh8 = (nh2 * nh2) * (nh2 * nh2);
    const float spec = F(0.35) * (nh8 * (nh8 * nh8));
    const float g = hit * F(0.618034);
    const float tint = g - std::floor(g);
    const float lit = F(0.22) + F(0.78) * diffuse;
    for (int a = 0; a < 3; a++) {
        const float colour = mix(mix(F(BODY_A[a]), F(BODY_B[a]), tint), F(1), pale);
        rgb[a] = colour * lit + spec;
    }
}

void cross(const float* x, const float* y, float* out) {
    const float cx = x[1] * y[2] - x[2] * y[1];
    const float cy = x[2] * y[0] - x[0] * y[2];
    const float cz = x[0] * y[1] - x[1] * y[0];
    out[0] = cx;
    out[1] = cy;
    out[2] = cz;
}

// ---- spheres -------------------------------------------------------------------------------------------------------

const int S_STRIDE = 40, S_PRESSED_BEFORE = 8, S_PRESSED_AFTER = 20, S_TURNED_BEFORE = 32, S_TURNED_AFTER = 36;
const int S_FLATTENING = 0, S_LEAN = 6, S_TRACE = 9, S_LEAN_LENGTH = 10;

float pressing(const float* shown, int base, int word, float alpha) {
    return mix(shown[base + S_PRESSED_BEFORE + word], shown[base + S_PRESSED_AFTER + word], alpha);
}

void times(const float* m, const float* x, float* y) {
    static const int row[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
    for (int a = 0; a < 3; a++) y[a] = m[row[a][0]] * x[0] + (m[row[a][1]] * x[1] + m[row[a][2]] * x[2]);
}

void squashed(const float* shown, int k, int base, const float* c, float r, float gain, float lift, const Frame& fr,
              float& best, float& hit, float* normal, float* local) {
    float m[6];
    for (int j = 0; j < 6; j++) {
        const float pressed = gain * pressing(shown, base, S_FLATTENING + j, fr.alpha);
        m[j] = j < 3 ? F(1) - pressed : -pressed;
    }
    const float adj[6] = {m[1] * m[2] - m[5] * m[5], m[0] * m[2] - m[4] * m[4], m[0] * m[1] - m[3] * m[3],
                          m[4] * m[5] - m[3] * m[2], m[3] * m[5] - m[4] * m[1], m[3] * m[4] - m[0] * m[5]};
    const float det = m[0] * adj[0] + (m[3] * adj[3] + m[4] * adj[4]);
    float cube = F(1) - (F(3) - (m[0] + (m[1] + m[2]))) / F(3);
    for (int step = 0; step < 2; step++) cube = (F(2) * cube + det / (cube * cube)) / F(3);
    const float scale = cube / det;
    float inverse[6];
    for (int j = 0; j < 6; j++) inverse[j] = adj[j] * scale;
    float o[3];
    for (int a = 0; a < 3; a++) {
        const float moved = c[a] + (lift * r) * pressing(shown, base, S_LEAN + a, fr.alpha);
        o[a] = fr.eye[a] - moved;
    }
    float os[3], ds[3];
    times(inverse, o, os);
    times(inverse, fr.d, ds);
    const float aa = dot(ds, ds);
    const float hh = dot(os, ds);
    const float disc = hh * hh - aa * (dot(os, os) - r * r);
    if (disc > F(0)) {
        const float t = (-hh - std::sqrt(disc)) / aa;
        if (t > F(0) && t < best) {
            best = t;
            hit = (float)k;
            float u[3];
            for (int a = 0; a < 3; a++) {
                u[a] = os[a] + t * ds[a];
                local[a] = u[a];
            }
            float n[3];
            times(inverse, u, n);
            for (int a = 0; a < 3; a++) normal[a] = n[a];
        }
    }
}

float turned(const float* shown, float hit, float alpha, const float* local) {
    const int base = (int)hit * S_STRIDE;
    float before[4], after[4];
    for (int a = 0; a < 4; a++) {
        before[a] = shown[base + S_TURNED_BEFORE + a];
        after[a] = shown[base + S_TURNED_AFTER + a];
    }
    float way = F(1);
    if (dot(before, after) + before[3] * after[3] < F(0)) way = F(-1);
    float q[3];
    for (int a = 0; a < 3; a++) q[a] = -mix(before[a] * way, after[a], alpha);
    const float w = mix(before[3] * way, after[3], alpha);
    float t[3], qt[3], p[3];
    cross(q, local, t);
    for (int a = 0; a < 3; a++) t[a] = F(2) * t[a];
    cross(q, t, qt);
    for (int a = 0; a < 3; a++) p[a] = local[a] + (w * t[a] + qt[a]);
    return (p[0] * p[1]) * p[2];
}

void sphere_pixel(const Push& p, const float* shown, float uvx, float uvy, float* rgb) {
    const Frame fr = frame_of(p, uvx, uvy);
    const float squash = fr.squash;
    float best = F(1e30), hit = F(-1);
    float normal[3] = {0, 0, 0}, local[3] = {0, 0, 0};
    for (int k = 0; k < fr.count; k++) {
        const int base = k * S_STRIDE;
        float c[3], o[3];
        for (int a = 0; a < 3; a++) {
            c[a] = mix(shown[base + a], shown[base + 4 + a], fr.alpha);
            o[a] = fr.eye[a] - c[a];
        }
        const float r = shown[base + 3];
        const float trace = pressing(shown, base, S_TRACE, fr.alpha);
        const float lean_length = pressing(shown, base, S_LEAN_LENGTH, fr.alpha);
        const float gain = fmin_(squash, F(0.5) / fmax_(trace, F(1e-9)));
        const float lift = fmax_(F(0), gain * F(2.0 / 3) - F(1));
        const float bound = r * (F(1) + F(0.53) * (gain * trace)) + lift * (r * lean_length);
        const float half = dot(o, fr.d);
        const float disc = half * half - (dot(o, o) - bound * bound);
        if (disc > F(0)) {
            const float root = std::sqrt(disc);
            if (root - half > F(0) && -half - root < best)
                squashed(shown, k, base, c, r, gain, lift, fr, best, hit, normal, local);
        }
    }
    background(fr, best, rgb);
    if (hit > F(-0.5)) {
        float patch = F(0);
        if (turned(shown, hit, fr.alpha, local) > F(0)) patch = F(0.45);
        shade(rgb, fr, hit, normal, patch);
    }
}

// ---- boxes ---------------------------------------------------------------------------------------------------------

const int B_STRIDE = 20, B_CENTRE_BEFORE = 0, B_SHAPE = 3, B_CENTRE_AFTER = 4, B_HALF = 8, B_TURNED_BEFORE = 12,
          B_TURNED_AFTER = 16;

void rotate(const float* q, const float* p, float* out) {
    const float twice = F(2) / ((q[0] * q[0] + q[1] * q[1]) + (q[2] * q[2] + q[3] * q[3]));
    float t[3], qt[3];
    cross(q, p, t);
    for (int a = 0; a < 3; a++) t[a] = twice * t[a];
    cross(q, t, qt);
    for (int a = 0; a < 3; a++) out[a] = p[a] + (q[3] * t[a] + qt[a]);
}

void slabs(const float* shown, int k, int base, const float* o, const float* half, const Frame& fr, float& best,
           float& hit, float& edged, float& pale, float* normal) {
    float before[4], after[4];
    for (int j = 0; j < 4; j++) {
        before[j] = shown[base + B_TURNED_BEFORE + j];
        after[j] = shown[base + B_TURNED_AFTER + j];
    }
    float way = F(1);
    if (dot(before, after) + before[3] * after[3] < F(0)) way = F(-1);
    float q[4];
    for (int j = 0; j < 4; j++) q[j] = mix(before[j] * way, after[j], fr.alpha);
    const float inverse[4] = {-q[0], -q[1], -q[2], q[3]};
    float os[3], ds[3];
    rotate(inverse, o, os);
    rotate(inverse, fr.d, ds);

    const float round = shown[base + B_SHAPE];
    if (round > 0.5f) {
        const float hh = dot(os, ds);
        const float cc = dot(os, os) - half[0] * half[0];
        const float disc = hh * hh - dot(ds, ds) * cc;
        if (disc > F(0)) {
            const float t = (-hh - std::sqrt(disc)) / dot(ds, ds);
            if (t > F(0) && t < best) {
                best = t;
                hit = (float)k;
                float own[3], world[3];
                for (int a = 0; a < 3; a++) own[a] = os[a] + t * ds[a];
                rotate(q, own, world);
                for (int a = 0; a < 3; a++) normal[a] = world[a];
                edged = F(0);
                pale = F(0);
                if ((own[0] * own[1]) * own[2] > F(0)) pale = F(1);
            }
        }
    }

    float enter = F(-1e30), leave = F(1e30), face = F(0);
    for (int a = 0; a < 3; a++) {
        float step = ds[a];
        if (std::fabs(step) < F(1e-9)) step = F(1e-9);
        const float t1 = (-half[a] - os[a]) / step;
        const float t2 = (half[a] - os[a]) / step;
        const float near = fmin_(t1, t2);
        leave = fmin_(leave, fmax_(t1, t2));
        if (near > enter) {
            enter = near;
            face = F(a);
        }
    }
    if (((enter < leave && enter > F(0)) && enter < best) && !(round > 0.5f)) {
        best = enter;
        hit = (float)k;
        float own[3], gap[3];
        for (int a = 0; a < 3; a++) {
            float on = F(0);
            if (face > F(a - 0.5) && face < F(a + 0.5)) on = F(1);
            own[a] = -(on * ds[a]);
            const float pa = os[a] + enter * ds[a];
            gap[a] = half[a] - std::fabs(pa);
        }
        float world[3];
        rotate(q, own, world);
        for (int a = 0; a < 3; a++) normal[a] = world[a];
        const float sum = (gap[0] + gap[1]) + gap[2];
        const float least = fmin_(gap[0], fmin_(gap[1], gap[2]));
        const float most = fmax_(gap[0], fmax_(gap[1], gap[2]));
        const float to_edge = (sum - least) - most;
        const float band = F(0.06) * fmin_(half[0], fmin_(half[1], half[2]));
        edged = F(0);
        pale = F(0);
        if (to_edge < band) edged = F(1);
    }
}

void box_pixel(const Push& p, const float* shown, float uvx, float uvy, float* rgb) {
    const Frame fr = frame_of(p, uvx, uvy);
    float best = F(1e30), hit = F(-1), edged = F(0), pale = F(0);
    float normal[3] = {0, 0, 0};
    for (int k = 0; k < fr.count; k++) {
        const int base = k * B_STRIDE;
        float o[3], half[3];
        for (int a = 0; a < 3; a++) {
            const float c = mix(shown[base + B_CENTRE_BEFORE + a], shown[base + B_CENTRE_AFTER + a], fr.alpha);
            o[a] = fr.eye[a] - c;
            half[a] = shown[base + B_HALF + a];
        }
        const float reach2 = dot(half, half);
        const float along = dot(o, fr.d);
        const float disc = along * along - (dot(o, o) - reach2);
        if (disc > F(0)) {
            const float root = std::sqrt(disc);
            if (root - along > F(0) && -along - root < best)
                slabs(shown, k, base, o, half, fr, best, hit, edged, pale, normal);
        }
    }
    background(fr, best, rgb);
    if (hit > F(-0.5)) {
        shade(rgb, fr, hit, normal, F(0.45) * pale);
        for (int a = 0; a < 3; a++) rgb[a] = rgb[a] * mix(F(1), F(0.55), edged);
    }
}

}  // namespace

extern "C" {

// `push` is Picture.push's 19 floats; rgb gets rows row0 .. row0 + rows - 1 of the width x height picture (row 0 the
// top), width * rows * 3 floats. shape 0 spheres, 1 boxes.
void orc_picture(int shape, const float* shown, const float* push, int width, int height, int row0, int rows,
                 float* rgb) {
    Push p;
    const float* w = push;
    for (int a = 0; a < 3; a++) {
        p.e[a] = w[a];
        p.r[a] = w[3 + a];
        p.u[a] = w[6 + a];
        p.f[a] = w[9 + a];
    }
    p.aspect = w[12];
    p.alpha = w[13];
    p.count = w[14];
    p.sx = w[15];
    p.sy = w[16];
    p.sz = w[17];
    p.squash = w[18];
    for (int j = row0; j < row0 + rows; j++)
        for (int i = 0; i < width; i++) {
            const float uvx = ((float)i + 0.5f) / (float)width, uvy = ((float)j + 0.5f) / (float)height;
            float* out = rgb + 3 * ((long)(j - row0) * width + i);
            if (shape == 0)
                sphere_pixel(p, shown, uvx, uvy, out);
            else
                box_pixel(p, shown, uvx, uvy, out);
        }
}

}  // extern "C"
