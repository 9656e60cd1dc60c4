// The narrow phase of one pair: separating axes over 15 axes with the face bias, the face manifold by clipping
// (up to 24 candidates reduced to 4), the edge contact, and the sphere–sphere / sphere–box contact.
//
// Restates core/box/BoxContact.java (core = vexelray-sim-rigid-core/src/main/java/dev/vexelray/sim/rigid/):
// collide :136-246, sphereContact :267-329, nearest :336-385, Solid :390-422, Edge :427-500, Face :505-817,
// in the same association order. One difference of form, none of result: a pair with a sphere in it skips the
// box test, since the sphere contact overwrites every word of the manifold the step reads (normal, axis, count
// and point 0).
#pragma once
#include "body_math.cuh"

namespace vxr {

constexpr int MANIFOLD_WORDS = 40, M_COUNT = 3, M_AXIS = 4, M_POINTS = 8, M_POINT_WORDS = 8;
constexpr int MOST_POINTS = 4, CANDIDATES = 24;
constexpr float RELATIVE = 0.98f, ABSOLUTE = 0.01f, PARALLEL = 1e-10f, SAME = 1e-12f, SLACK = 1e-5f,
                OFF_LINE = 1e-4f;
constexpr int SPHERE_BOX = 15, SPHERE_SPHERE = 16;

// A manifold as the device keeps it: the normal and count, then per point the anchor on each body and the
// depth. head = (nx, ny, nz, count), axis separately; pa[i] = (anchor on first, depth), pb[i] = (anchor on second,
// axis id in .w of point 0 only).
struct Manifold {
    float normal[3];
    float axis;
    int count;
    float a[MOST_POINTS][3], b[MOST_POINTS][3], depth[MOST_POINTS];
};

struct Solid {
    float centre[3], axes[3][3], half[3];
    __device__ __forceinline__ void load(float4 pose, float4 q, float4 hw) {
        centre[0] = pose.x; centre[1] = pose.y; centre[2] = pose.z;
        half[0] = hw.x; half[1] = hw.y; half[2] = hw.z;
        const float x = q.x, y = q.y, z = q.z, w = q.w;
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
    __device__ __forceinline__ void own(const float* point, float* out) const {
        const float off[3] = {point[0] - centre[0], point[1] - centre[1], point[2] - centre[2]};
        const float o0 = dot3(off, axes[0]), o1 = dot3(off, axes[1]), o2 = dot3(off, axes[2]);
        out[0] = o0; out[1] = o1; out[2] = o2;
    }
};

__device__ __forceinline__ void put_point(Manifold& m, int i, const float* of, const float* os, float depth) {
#pragma unroll
    for (int x = 0; x < 3; x++) {
        m.a[i][x] = of[x];
        m.b[i][x] = os[x];
    }
    m.depth[i] = depth;
}

struct EdgeRecord {
    float normal[3], onFirst[3], alongFirst[3], halfFirst, onSecond[3], alongSecond[3], halfSecond, axis;
    __device__ __forceinline__ void record(const Solid& first, const Solid& second, int k, int j, const float* ax,
                                           const float* d) {
        float toward = 1.0f;
        if (dot3(d, ax) < 0.0f) toward = -1.0f;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            normal[a] = ax[a] * toward;
            onFirst[a] = first.centre[a];
            onSecond[a] = second.centre[a];
            alongFirst[a] = first.axes[k][a];
            alongSecond[a] = second.axes[j][a];
        }
#pragma unroll
        for (int m = 0; m < 3; m++) {
            if (m != k) {
                const float sign = sign_of(dot3(first.axes[m], normal));
#pragma unroll
                for (int a = 0; a < 3; a++) onFirst[a] = onFirst[a] + (sign * first.half[m]) * first.axes[m][a];
            }
            if (m != j) {
                const float sign = sign_of(dot3(second.axes[m], normal));
#pragma unroll
                for (int a = 0; a < 3; a++) onSecond[a] = onSecond[a] - (sign * second.half[m]) * second.axes[m][a];
            }
        }
        halfFirst = first.half[k];
        halfSecond = second.half[j];
        axis = (float)(6 + 3 * k + j);
    }
    __device__ __forceinline__ void contact(const Solid& first, const Solid& second, float bestEdge,
                                            Manifold& m) const {
        const float w[3] = {onFirst[0] - onSecond[0], onFirst[1] - onSecond[1], onFirst[2] - onSecond[2]};
        const float cs = dot3(alongFirst, alongSecond);
        const float dA = dot3(alongFirst, w);
        const float dB = dot3(alongSecond, w);
        const float den = 1.0f - cs * cs;
        float s = (cs * dB - dA) / den;
        float u = (dB - cs * dA) / den;
        s = fmaxf(-halfFirst, fminf(halfFirst, s));
        u = fmaxf(-halfSecond, fminf(halfSecond, u));
        float pf[3], ps[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            pf[a] = onFirst[a] + s * alongFirst[a];
            ps[a] = onSecond[a] + u * alongSecond[a];
        }
#pragma unroll
        for (int a = 0; a < 3; a++) m.normal[a] = normal[a];
        m.axis = axis;
        float of[3], os[3];
        first.own(pf, of);
        second.own(ps, os);
        put_point(m, 0, of, os, -bestEdge);
    }
};

// The face contact: reference face of one body, incident face of the other, clipped into <= 24 candidates
// (kept in local memory), reduced to <= 4 points.
struct FaceClip {
    const Solid* first;
    const Solid* second;
    float flip, margin;
    float refCentre[3], n[3], u[3], w[3], hn, hu, hw, axis;
    float face[3], a[3], c[3], ha, hc;
    float cand[CANDIDATES][4];

    __device__ __forceinline__ void setup(const Solid& firstBox, const Solid& secondBox, bool fromSecond,
                                          const float* bestFaceAxis, float mg) {
        first = &firstBox;
        second = &secondBox;
        margin = mg;
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
#pragma unroll
        for (int e = 0; e < 3; e++) refCentre[e] = ref->centre[e];
        axis = k + 1.5f * (1.0f - flip);
#pragma unroll
        for (int e = 0; e < 3; e++) n[e] = u[e] = w[e] = 0.0f;
        hn = hu = hw = 0.0f;
#pragma unroll
        for (int kk = 0; kk < 3; kk++) {
            const int ku = (kk + 1) % 3, kw = (kk + 2) % 3;
            if (k > (float)kk - 0.5f && k < (float)kk + 0.5f) {
#pragma unroll
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
        const float apart[3] = {inc->centre[0] - refCentre[0], inc->centre[1] - refCentre[1],
                                inc->centre[2] - refCentre[2]};
        if (dot3(apart, n) < 0.0f) {
#pragma unroll
            for (int e = 0; e < 3; e++) n[e] = -n[e];
        }
        float most = -1.0f, faceAxis[3] = {0.0f, 0.0f, 0.0f}, hf = 0.0f;
#pragma unroll
        for (int e = 0; e < 3; e++) a[e] = c[e] = 0.0f;
        ha = hc = 0.0f;
#pragma unroll
        for (int m = 0; m < 3; m++) {
            const int ma = (m + 1) % 3, mc = (m + 2) % 3;
            const float tt = fabsf(dot3(inc->axes[m], n));
            if (tt > most) {
                most = tt;
#pragma unroll
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
        const float facing = sign_of(dot3(faceAxis, n));
#pragma unroll
        for (int e = 0; e < 3; e++) face[e] = inc->centre[e] - (facing * hf) * faceAxis[e];
    }

    __device__ __forceinline__ void keep(int& count, bool when, const float* point, float depth) {
        if (when && depth > -margin && count < CANDIDATES) {
            cand[count][0] = point[0];
            cand[count][1] = point[1];
            cand[count][2] = point[2];
            cand[count][3] = depth;
            count++;
        }
    }

    __device__ __forceinline__ void emit(int at, int& count, Manifold& m) const {
        const float deep = cand[at][3];
        const float onFirstIsRef = 0.5f * (flip + 1.0f);
        float pf[3], ps[3];
#pragma unroll
        for (int x = 0; x < 3; x++) {
            const float lift = deep * n[x];
            pf[x] = cand[at][x] + onFirstIsRef * lift;
            ps[x] = cand[at][x] + (1.0f - onFirstIsRef) * lift;
        }
        float of[3], os[3];
        first->own(pf, of);
        second->own(ps, os);
        put_point(m, count, of, os, deep);
        count++;
    }

    __device__ void reduce(int found, int& count, Manifold& m) const {
        int deepest = 0;
        float most = -1e30f;
        for (int k = 0; k < found; k++) {
            const float d = cand[k][3];
            if (d > most) {
                most = d;
                deepest = k;
            }
        }
        const float pa[3] = {cand[deepest][0], cand[deepest][1], cand[deepest][2]};
        int farthest = -1;
        float far = SAME;
        for (int k = 0; k < found; k++) {
            const float gap[3] = {cand[k][0] - pa[0], cand[k][1] - pa[1], cand[k][2] - pa[2]};
            const float d2 = dot3(gap, gap);
            if (d2 > far) {
                far = d2;
                farthest = k;
            }
        }
        emit(deepest, count, m);
        if (farthest > -1) {
            const float ab[3] = {cand[farthest][0] - pa[0], cand[farthest][1] - pa[1], cand[farthest][2] - pa[2]};
            int left = -1, right = -1;
            float mostLeft = OFF_LINE * far;
            float mostRight = -mostLeft;
            for (int k = 0; k < found; k++) {
                const float aq[3] = {cand[k][0] - pa[0], cand[k][1] - pa[1], cand[k][2] - pa[2]};
                float cr[3];
                cross3(ab, aq, cr);
                const float area = dot3(cr, n);
                if (area > mostLeft) {
                    mostLeft = area;
                    left = k;
                }
                if (area < mostRight) {
                    mostRight = area;
                    right = k;
                }
            }
            emit(farthest, count, m);
            if (left > -1) emit(left, count, m);
            if (right > -1) emit(right, count, m);
        }
    }

    __device__ void contact(int& count, Manifold& m) {
        const float signs[4][2] = {{1.0f, 1.0f}, {-1.0f, 1.0f}, {-1.0f, -1.0f}, {1.0f, -1.0f}};
        const float wide = 1.0f + SLACK;
        float corner[4][3], cu[4], cw[4], depth[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
#pragma unroll
            for (int x = 0; x < 3; x++)
                corner[e][x] = face[x] + ((signs[e][0] * ha) * a[x] + (signs[e][1] * hc) * c[x]);
            const float rel[3] = {corner[e][0] - refCentre[0], corner[e][1] - refCentre[1],
                                  corner[e][2] - refCentre[2]};
            cu[e] = dot3(rel, u);
            cw[e] = dot3(rel, w);
            depth[e] = hn - dot3(rel, n);
            const bool inside = fabsf(cu[e]) < hu * wide && fabsf(cw[e]) < hw * wide;
            keep(count, inside, corner[e], depth[e]);
        }
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int next = (e + 1) % 4;
#pragma unroll
            for (int line = 0; line < 4; line++) {
                const bool acrossU = line < 2;
                const float side = line % 2 == 0 ? 1.0f : -1.0f;
                const float from = acrossU ? cu[e] : cw[e];
                const float to = acrossU ? cu[next] : cw[next];
                const float alongFrom = acrossU ? cw[e] : cu[e];
                const float alongTo = acrossU ? cw[next] : cu[next];
                const float limit = acrossU ? hu : hw;
                const float bound = acrossU ? hw : hu;
                const float span = to - from;
                if (fabsf(span) > SAME) {
                    const float s = (side * limit - from) / span;
                    const float along = alongFrom + s * (alongTo - alongFrom);
                    const bool within = s > -SLACK && s < wide && fabsf(along) < bound * wide;
                    float point[3];
#pragma unroll
                    for (int x = 0; x < 3; x++) point[x] = corner[e][x] + s * (corner[next][x] - corner[e][x]);
                    const float deep = depth[e] + s * (depth[next] - depth[e]);
                    keep(count, within, point, deep);
                }
            }
        }
        const float off[3] = {face[0] - refCentre[0], face[1] - refCentre[1], face[2] - refCentre[2]};
        const float fu = dot3(off, u), fw = dot3(off, w);
        const float au = ha * dot3(a, u), aw = ha * dot3(a, w);
        const float bu = hc * dot3(c, u), bw = hc * dot3(c, w);
        const float det = au * bw - aw * bu;
        if (fabsf(det) > SAME) {
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const float ru = signs[e][0] * hu - fu;
                const float rw = signs[e][1] * hw - fw;
                const float alpha = (ru * bw - rw * bu) / det;
                const float beta = (au * rw - aw * ru) / det;
                const bool inside = fabsf(alpha) < wide && fabsf(beta) < wide;
                float point[3];
#pragma unroll
                for (int x = 0; x < 3; x++) point[x] = face[x] + ((alpha * ha) * a[x] + (beta * hc) * c[x]);
                const float rel[3] = {point[0] - refCentre[0], point[1] - refCentre[1], point[2] - refCentre[2]};
                keep(count, inside, point, hn - dot3(rel, n));
            }
        }
#pragma unroll
        for (int x = 0; x < 3; x++) m.normal[x] = n[x] * flip;
        m.axis = axis;
        const int found = count;
        count = 0;
        if (found > 0) reduce(found, count, m);
    }
};

__device__ __forceinline__ float nearest(const Solid& box, const float* p, float* towards, float* surface) {
    const float off[3] = {p[0] - box.centre[0], p[1] - box.centre[1], p[2] - box.centre[2]};
    float local[3], held[3], outside[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        local[k] = dot3(off, box.axes[k]);
        held[k] = fmaxf(-box.half[k], fminf(box.half[k], local[k]));
    }
#pragma unroll
    for (int k = 0; k < 3; k++) outside[k] = local[k] - held[k];
    const float away = sqrtf(dot3(outside, outside));
    float reach = away;
    if (away > 1e-9f) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            float dir = 0.0f, at = box.centre[a];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                dir = dir + outside[k] * box.axes[k][a];
                at = at + held[k] * box.axes[k][a];
            }
            towards[a] = dir / away;
            surface[a] = at;
        }
    } else {
        float least = 1e30f;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float inward = box.half[k] - fabsf(local[k]);
            if (inward < least) {
                least = inward;
                const float side = sign_of(local[k]);
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    towards[a] = side * box.axes[k][a];
                    float at = box.centre[a];
#pragma unroll
                    for (int j = 0; j < 3; j++) {
                        const float along = j == k ? side * box.half[k] : local[j];
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

__device__ __forceinline__ void sphere_contact(const Solid& first, const Solid& second, bool sphereA, bool sphereB,
                                               float margin, Manifold& m) {
    float n[3] = {0.0f, 0.0f, 0.0f}, onFirst[3] = {0.0f, 0.0f, 0.0f}, onSecond[3] = {0.0f, 0.0f, 0.0f};
    float depth = 0.0f, axis = (float)SPHERE_BOX;
    if (sphereA && sphereB) {
        const float d[3] = {second.centre[0] - first.centre[0], second.centre[1] - first.centre[1],
                            second.centre[2] - first.centre[2]};
        const float length = sqrtf(dot3(d, d));
        n[1] = 1.0f;
        if (length > 1e-9f) {
#pragma unroll
            for (int a = 0; a < 3; a++) n[a] = d[a] / length;
        }
        depth = (first.half[0] + second.half[0]) - length;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            onFirst[a] = first.centre[a] + first.half[0] * n[a];
            onSecond[a] = second.centre[a] - second.half[0] * n[a];
        }
        axis = (float)SPHERE_SPHERE;
    } else {
        const bool sphereFirst = sphereA;
        const Solid& round = sphereFirst ? first : second;
        const Solid& box = sphereFirst ? second : first;
        float towards[3] = {0.0f, 0.0f, 0.0f}, surface[3] = {0.0f, 0.0f, 0.0f};
        const float reach = nearest(box, round.centre, towards, surface);
        const float radius = round.half[0];
        depth = radius - reach;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const float onSphere = round.centre[a] - radius * towards[a];
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
#pragma unroll
    for (int a = 0; a < 3; a++) m.normal[a] = n[a];
    m.axis = axis;
    m.count = 0;
    if (depth > -margin) {
        float of[3], os[3];
        first.own(onFirst, of);
        second.own(onSecond, os);
        put_point(m, 0, of, os, depth);
        m.count = 1;
    }
}

// The manifold of one pair (BoxContact.collide :136-246).
__device__ __noinline__ void collide_pair(float4 poseA, float4 turnA, float4 halfA, float4 poseB, float4 turnB,
                                          float4 halfB, float margin, Manifold& m) {
    Solid first, second;
    first.load(poseA, turnA, halfA);
    second.load(poseB, turnB, halfB);
    m.count = 0;
    m.axis = 0.0f;
    m.normal[0] = m.normal[1] = m.normal[2] = 0.0f;
    const bool sphereA = halfA.w > 0.5f, sphereB = halfB.w > 0.5f;
    if (sphereA || sphereB) {
        sphere_contact(first, second, sphereA, sphereB, margin, m);
        return;
    }
    const float d[3] = {second.centre[0] - first.centre[0], second.centre[1] - first.centre[1],
                        second.centre[2] - first.centre[2]};
    float parted = -1e30f;
    float bestFace[2] = {-1e30f, -1e30f}, bestFaceAxis[2] = {0.0f, 0.0f};
#pragma unroll
    for (int side = 0; side < 2; side++) {
        const Solid& own = side == 0 ? first : second;
        const Solid& other = side == 0 ? second : first;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float reach = own.half[k];
#pragma unroll
            for (int j = 0; j < 3; j++) reach = reach + other.half[j] * fabsf(dot3(own.axes[k], other.axes[j]));
            const float sep = fabsf(dot3(d, own.axes[k])) - reach;
            parted = fmaxf(parted, sep);
            if (sep > bestFace[side]) {
                bestFace[side] = sep;
                bestFaceAxis[side] = (float)k;
            }
        }
    }
    float bestEdge = -1e30f;
    EdgeRecord edge;
#pragma unroll
    for (int e = 0; e < 3; e++) {
        edge.normal[e] = edge.onFirst[e] = edge.alongFirst[e] = edge.onSecond[e] = edge.alongSecond[e] = 0.0f;
    }
    edge.halfFirst = edge.halfSecond = edge.axis = 0.0f;
    for (int k = 0; k < 3; k++) {
        for (int j = 0; j < 3; j++) {
            float across[3];
            cross3(first.axes[k], second.axes[j], across);
            const float length2 = dot3(across, across);
            if (length2 > PARALLEL) {
                const float length = sqrtf(length2);
                const float inv = 1.0f / length;
                const float ax[3] = {across[0] * inv, across[1] * inv, across[2] * inv};
                float reach = 0.0f;
#pragma unroll
                for (int mm = 0; mm < 3; mm++)
                    reach = reach + (first.half[mm] * fabsf(dot3(first.axes[mm], ax)) +
                                     second.half[mm] * fabsf(dot3(second.axes[mm], ax)));
                const float sep = fabsf(dot3(d, ax)) - reach;
                parted = fmaxf(parted, sep);
                if (sep > bestEdge) {
                    bestEdge = sep;
                    edge.record(first, second, k, j, ax, d);
                }
            }
        }
    }
    float smallest = first.half[0];
#pragma unroll
    for (int k = 0; k < 3; k++) smallest = fminf(smallest, first.half[k]);
#pragma unroll
    for (int k = 0; k < 3; k++) smallest = fminf(smallest, second.half[k]);
    const float slack = ABSOLUTE * smallest;
    const bool fromSecond = bestFace[1] > RELATIVE * bestFace[0] + slack;
    const float faceSep = fromSecond ? bestFace[1] : bestFace[0];
    const bool byEdge = bestEdge > RELATIVE * faceSep + slack;
    if (parted > margin) return;
    if (byEdge) {
        edge.contact(first, second, bestEdge, m);
        m.count = 1;
    } else {
        FaceClip face;
        face.setup(first, second, fromSecond, bestFaceAxis, margin);
        int count = 0;
        face.contact(count, m);
        m.count = count;
    }
}

}  // namespace vxr
