// Per-body and per-contact arithmetic of the box/mixed soft step, on the device.
//
// Every expression keeps the association order of the reference's IR (paths inside sibarum/vexelray-sim-rigid,
// core = vexelray-sim-rigid-core/src/main/java/dev/vexelray/sim/rigid/): with --fmad=false and IEEE division and
// square root, each result is the same f32 the reference's kernels define.
//
//   rotate                 core/box/Boxes.java:907-921
//   turned                 core/box/Boxes.java:877-899
//   inverseInertia         core/box/Boxes.java:854-871
//   Moving (a held body)   core/box/Boxes.java:660-773
//   Soft                   core/box/Boxes.java:421-450
//   contact                core/box/Boxes.java:462-542
//   roll                   core/box/Boxes.java:553-600
#pragma once
#include <cstdint>

namespace vxr {

// Parameter words (Boxes.java:97-122).
enum : int {
    P_H = 0, P_GX, P_GY, P_GZ, P_SX, P_SY, P_SZ, P_MU_STATIC, P_MU_KINETIC, P_MARGIN, P_BIAS, P_MASS_SCALE,
    P_IMPULSE_SCALE, P_STATIC_BIAS, P_STATIC_MASS_SCALE, P_STATIC_IMPULSE_SCALE, P_PUSH, P_MU_ROLLING, P_COUNT
};
enum Sweep : int { WARM = 0, SOLVE = 1, RELAX = 2 };

struct Params {
    float w[P_COUNT];
};

__device__ __forceinline__ float dot3(const float* a, const float* b) {
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}
__device__ __forceinline__ void cross3(const float* x, const float* y, float* o) {
    const float c0 = x[1] * y[2] - x[2] * y[1];
    const float c1 = x[2] * y[0] - x[0] * y[2];
    const float c2 = x[0] * y[1] - x[1] * y[0];
    o[0] = c0;
    o[1] = c1;
    o[2] = c2;
}
// 2 / |q|², the factor every turn by q (or by its conjugate: the same squares) scales by.
__device__ __forceinline__ float twice_of(const float* q) {
    return 2.0f / ((q[0] * q[0] + q[1] * q[1]) + (q[2] * q[2] + q[3] * q[3]));
}

// p turned by q: p + w t + q × t with t = 2 q × p / |q|², the factor given.
__device__ __forceinline__ void rotate_by(const float* q, float twice, const float* p, float* out) {
    float t[3];
    cross3(q, p, t);
#pragma unroll
    for (int a = 0; a < 3; a++) t[a] = twice * t[a];
    float qt[3];
    cross3(q, t, qt);
    float o[3];
#pragma unroll
    for (int a = 0; a < 3; a++) o[a] = p[a] + (q[3] * t[a] + qt[a]);
    out[0] = o[0];
    out[1] = o[1];
    out[2] = o[2];
}
__device__ __forceinline__ void rotateq(const float* q, const float* p, float* out) { rotate_by(q, twice_of(q), p, out); }
__device__ __forceinline__ float sign_of(float x) { return x < 0.0f ? -1.0f : 1.0f; }

// q turned by omega for dt, first order, normalised.
__device__ __forceinline__ void turned(const float* q, const float* omega, float dt, float* now) {
    float a[3];
#pragma unroll
    for (int k = 0; k < 3; k++) a[k] = (0.5f * dt) * omega[k];
    float r[4];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
        r[k] = q[k] + (a[k] * q[3] + (a[k1] * q[k2] - a[k2] * q[k1]));
    }
    r[3] = q[3] - (a[0] * q[0] + (a[1] * q[1] + a[2] * q[2]));
    const float len2 = (r[0] * r[0] + r[1] * r[1]) + (r[2] * r[2] + r[3] * r[3]);
    const float inverse = 1.0f / sqrtf(fmaxf(len2, 1e-30f));
#pragma unroll
    for (int k = 0; k < 4; k++) now[k] = r[k] * inverse;
}

// Inverse principal moments: a box's 3 im / (b² + c²), a sphere's im / (0.4 r²).
__device__ __forceinline__ void inverse_inertia(const float4 half, float im, float* inverse) {
    const float h2[3] = {half.x * half.x, half.y * half.y, half.z * half.z};
#pragma unroll
    for (int a = 0; a < 3; a++) inverse[a] = (3.0f * im) / (h2[(a + 1) % 3] + h2[(a + 2) % 3]);
    if (half.w > 0.5f) {
#pragma unroll
        for (int a = 0; a < 3; a++) inverse[a] = im / (0.4f * h2[0]);
    }
}

// A body as a velocity solve holds it: pose read-only, velocity, angular momentum and angular velocity
// updated in registers and stored once.
struct Held {
    float at[3], q[4], half[3], inverse[3], velocity[3], momentum[3], omega[3];
    float im, shape, twice;

    __device__ __forceinline__ void times_inverse_inertia(const float* x, float* out) const {
        const float c[4] = {-q[0], -q[1], -q[2], q[3]};
        float own[3], scaled[3];
        rotate_by(c, twice, x, own);
#pragma unroll
        for (int a = 0; a < 3; a++) scaled[a] = inverse[a] * own[a];
        rotate_by(q, twice, scaled, out);
    }
    // inv: the body's inverse principal moments (inverse_inertia of its half-extents, shape and inverse mass)
    __device__ __forceinline__ void load(float4 pose, float4 turn, float4 halfw, float4 vel, float4 mom, float4 inv) {
        at[0] = pose.x; at[1] = pose.y; at[2] = pose.z; im = pose.w;
        q[0] = turn.x; q[1] = turn.y; q[2] = turn.z; q[3] = turn.w;
        half[0] = halfw.x; half[1] = halfw.y; half[2] = halfw.z; shape = halfw.w;
        velocity[0] = vel.x; velocity[1] = vel.y; velocity[2] = vel.z;
        momentum[0] = mom.x; momentum[1] = mom.y; momentum[2] = mom.z;
        inverse[0] = inv.x; inverse[1] = inv.y; inverse[2] = inv.z;
        twice = twice_of(q);
        times_inverse_inertia(momentum, omega);
    }
    __device__ __forceinline__ bool sphere() const { return shape > 0.5f; }
    __device__ __forceinline__ float mass_along(const float* r, const float* n) const {
        float rn[3], t[3];
        cross3(r, n, rn);
        times_inverse_inertia(rn, t);
        return im + dot3(rn, t);
    }
    __device__ __forceinline__ void point_velocity(const float* r, float* out) const {
        float turning[3];
        cross3(omega, r, turning);
#pragma unroll
        for (int a = 0; a < 3; a++) out[a] = velocity[a] + turning[a];
    }
    __device__ __forceinline__ void apply(const float* r, const float* p) {
#pragma unroll
        for (int a = 0; a < 3; a++) velocity[a] = velocity[a] + im * p[a];
        float angular[3], t[3];
        cross3(r, p, angular);
        times_inverse_inertia(angular, t);
#pragma unroll
        for (int a = 0; a < 3; a++) {
            momentum[a] = momentum[a] + angular[a];
            omega[a] = omega[a] + t[a];
        }
    }
    __device__ __forceinline__ void turn(const float* j) {
        float spin[3];
        times_inverse_inertia(j, spin);
#pragma unroll
        for (int a = 0; a < 3; a++) {
            momentum[a] = momentum[a] + j[a];
            omega[a] = omega[a] + spin[a];
        }
    }
};

struct Soft {
    float h, margin, bias, mass_scale, impulse_scale, push, mu_static, mu_kinetic;
    __device__ __forceinline__ Soft(const Params& p, bool fixed) {
        h = p.w[P_H];
        margin = p.w[P_MARGIN];
        bias = p.w[fixed ? P_STATIC_BIAS : P_BIAS];
        mass_scale = p.w[fixed ? P_STATIC_MASS_SCALE : P_MASS_SCALE];
        impulse_scale = p.w[fixed ? P_STATIC_IMPULSE_SCALE : P_IMPULSE_SCALE];
        push = p.w[P_PUSH];
        mu_static = p.w[P_MU_STATIC];
        mu_kinetic = p.w[P_MU_KINETIC];
    }
};

// The pair forms take a first body; the wall forms pass none (a fixed wall).
template <bool PAIR>
__device__ __forceinline__ void relative_velocity(const Held& first, const float* rA, const Held& second,
                                                  const float* rB, float* out) {
    float vb[3];
    second.point_velocity(rB, vb);
    if (!PAIR) {
        out[0] = vb[0]; out[1] = vb[1]; out[2] = vb[2];
        return;
    }
    float va[3];
    first.point_velocity(rA, va);
#pragma unroll
    for (int a = 0; a < 3; a++) out[a] = vb[a] - va[a];
}
template <bool PAIR>
__device__ __forceinline__ float mass_along(const Held& first, const float* rA, const Held& second, const float* rB,
                                            const float* n) {
    const float k = second.mass_along(rB, n);
    return PAIR ? k + first.mass_along(rA, n) : k;
}
template <bool PAIR>
__device__ __forceinline__ void apply_pair(Held& first, const float* rA, Held& second, const float* rB,
                                           const float* p) {
    second.apply(rB, p);
    if (PAIR) {
        const float back[3] = {-p[0], -p[1], -p[2]};
        first.apply(rA, back);
    }
}
template <bool PAIR>
__device__ __forceinline__ void apply_angular(Held& first, Held& second, const float* j) {
    second.turn(j);
    if (PAIR) {
        const float back[3] = {-j[0], -j[1], -j[2]};
        first.turn(back);
    }
}

// One contact point, one sweep. rec = (normal impulse, tangential impulse x, y, z), updated in place.
// Returns whether the record was touched (read and possibly written).
// k_given: the normal's generalised inverse mass when the caller has it (it depends only on the pose, so it is the
// same in every sweep of a substep's half); negative: computed here.
// track: where the sweep's residual is gathered (null: not measured). A point's share is the positional correction
// this sweep's update makes there, h k (|change of the normal impulse| + |change of the tangential impulse|): the
// solve has converged at the point when it is zero. Measuring changes no result.
template <bool PAIR>
__device__ __forceinline__ void contact(int sweep, float gap, const float* n, Held& first, const float* rA,
                                        Held& second, const float* rB, float4& rec, const Soft& soft,
                                        float k_given = -1.0f, unsigned* track = nullptr) {
    const float normal = rec.x;
    const float tangent[3] = {rec.y, rec.z, rec.w};
    const bool holding = normal > 0.0f || dot3(tangent, tangent) > 0.0f;
    if (sweep == WARM) {
        if (holding) {
            float p[3];
#pragma unroll
            for (int a = 0; a < 3; a++) p[a] = normal * n[a] + tangent[a];
            apply_pair<PAIR>(first, rA, second, rB, p);
        }
        return;
    }
    if (!(gap < soft.margin || holding)) return;
    const float k = k_given >= 0.0f ? k_given : mass_along<PAIR>(first, rA, second, rB, n);
    float rel[3];
    relative_velocity<PAIR>(first, rA, second, rB, rel);
    const float closing = dot3(rel, n);
    float bias = 0.0f, mass_scale = 1.0f, impulse_scale = 0.0f;
    if (gap > 0.0f) bias = gap / soft.h;
    if (sweep == SOLVE && !(gap > 0.0f)) {
        bias = fmaxf(soft.bias * gap, -soft.push);
        mass_scale = soft.mass_scale;
        impulse_scale = soft.impulse_scale;
    }
    const float change = -((mass_scale / k) * (closing + bias)) - impulse_scale * normal;
    const float total = fmaxf(0.0f, normal + change);
    float p[3];
#pragma unroll
    for (int a = 0; a < 3; a++) p[a] = (total - normal) * n[a];
    apply_pair<PAIR>(first, rA, second, rB, p);

    float sliding[3];
    relative_velocity<PAIR>(first, rA, second, rB, sliding);
    const float along = dot3(sliding, n);
#pragma unroll
    for (int a = 0; a < 3; a++) sliding[a] = sliding[a] - along * n[a];
    float whole[3] = {tangent[0], tangent[1], tangent[2]};
    const float speed = sqrtf(dot3(sliding, sliding));
    if (speed > 1e-12f) {
        float t[3];
#pragma unroll
        for (int a = 0; a < 3; a++) t[a] = sliding[a] / speed;
        const float kt = mass_along<PAIR>(first, rA, second, rB, t);
        const float stop = speed / kt;
#pragma unroll
        for (int a = 0; a < 3; a++) whole[a] = whole[a] - stop * t[a];
    }
    const float size = sqrtf(dot3(whole, whole));
    if (size > soft.mu_static * total) {
        const float cut = (soft.mu_kinetic * total) / size;
#pragma unroll
        for (int a = 0; a < 3; a++) whole[a] = whole[a] * cut;
    }
    float rubbed[3];
#pragma unroll
    for (int a = 0; a < 3; a++) rubbed[a] = whole[a] - tangent[a];
    rec = make_float4(total, whole[0], whole[1], whole[2]);
    apply_pair<PAIR>(first, rA, second, rB, rubbed);
    if (track) {
        const float moved = soft.h * k * (fabsf(total - normal) + sqrtf(dot3(rubbed, rubbed)));
        if (moved > 0.0f) atomicMax(track, __float_as_uint(moved));
    }
}

// Rolling resistance at one contact with a sphere in it; roll = the accumulated angular impulse (x, y, z).
template <bool PAIR>
__device__ __forceinline__ void roll(int sweep, Held& first, Held& second, float radius, float normal_now,
                                     float4& rollrec, float mu_rolling) {
    const float old[3] = {rollrec.x, rollrec.y, rollrec.z};
    if (sweep == WARM) {
        apply_angular<PAIR>(first, second, old);
        return;
    }
    float whole[3], turning[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        whole[a] = old[a];
        const float against = PAIR ? first.omega[a] : 0.0f;
        turning[a] = second.omega[a] - against;
    }
    const float speed = sqrtf(dot3(turning, turning));
    if (speed > 1e-12f && mu_rolling > 0.0f) {
        float t[3];
#pragma unroll
        for (int a = 0; a < 3; a++) t[a] = turning[a] / speed;
        float it[3];
        second.times_inverse_inertia(t, it);
        float k = dot3(t, it);
        if (PAIR) {
            float jt[3];
            first.times_inverse_inertia(t, jt);
            k = k + dot3(t, jt);
        }
        const float stop = speed / k;
#pragma unroll
        for (int a = 0; a < 3; a++) whole[a] = whole[a] - stop * t[a];
    }
    const float most = (mu_rolling * radius) * fmaxf(0.0f, normal_now);
    const float size = sqrtf(dot3(whole, whole));
    if (size > most) {
        const float scale = most / size;
#pragma unroll
        for (int a = 0; a < 3; a++) whole[a] = whole[a] * scale;
    }
    float change[3];
#pragma unroll
    for (int a = 0; a < 3; a++) change[a] = whole[a] - old[a];
    rollrec = make_float4(whole[0], whole[1], whole[2], 0.0f);
    apply_angular<PAIR>(first, second, change);
}

__device__ __forceinline__ bool nonzero_bits(float4 r) {
    return (__float_as_uint(r.x) | __float_as_uint(r.y) | __float_as_uint(r.z) | __float_as_uint(r.w)) != 0u;
}

}  // namespace vxr
