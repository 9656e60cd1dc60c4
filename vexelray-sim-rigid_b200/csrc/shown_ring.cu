// Finished steps handed from the thread that steps to the thread that reads them, neither waiting for the other:
// the reference's ShownRing (vexelray-sim-rigid-gui/src/main/java/dev/vexelray/sim/rigid/gui/ShownRing.java:37-177)
// with device buffers for its slots. Three slots take three roles: the front (the one the reader reads), ready (the
// newest finished step not taken yet, or none) and the rest free, one of which the next step is kept in. A slot's
// CUDA event stands for the reference's timeline value: a reader's stream waits on it before it reads the slot.
// Generations: a new simulation brings new slots; the old ones are retired once the reader has taken from the new.
// Thread-safe: every call holds the ring's lock for a few field writes (and, for keep, two enqueued operations).
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "vxr.h"

namespace {

constexpr int SLOTS = 3;

struct Gen {
    long long id = 0;
    int shape = 0, bodies = 0;
    long long words = 0;
    double extent[3] = {0, 0, 0};
    float* slot[SLOTS] = {nullptr, nullptr, nullptr};
    cudaEvent_t done[SLOTS] = {nullptr, nullptr, nullptr};
};

void release(Gen* g) {
    if (!g) return;
    for (int k = 0; k < SLOTS; k++) {
        if (g->slot[k]) cudaFree(g->slot[k]);
        if (g->done[k]) cudaEventDestroy(g->done[k]);
    }
    delete g;
}

long long now_ns() {
    return (long long)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

}  // namespace

struct vxr_ring {
    std::mutex lock;
    int device = 0;
    long long next_id = 1;
    Gen* generation = nullptr;
    Gen* front_generation = nullptr;  // may be older than `generation`
    std::vector<Gen*> retired;         // moved past by the reader, not yet handed to the writer to free
    std::vector<Gen*> all;             // every generation not yet freed
    int front = -1, ready = -1, back = 0;
    long long steps[SLOTS] = {0, 0, 0}, finished[SLOTS] = {0, 0, 0};
    bool taken = false;
    vxr_frame frame{};
    std::string error;
};

namespace {

void describe(const vxr_ring* r, const Gen* g, int slot, vxr_frame* f) {
    f->generation = g->id;
    f->slot = slot;
    f->shape = g->shape;
    f->step = r->steps[slot];
    f->finished_ns = r->finished[slot];
    f->bodies = g->bodies;
    f->words = g->words;
    f->data = g->slot[slot];
    f->event = (void*)g->done[slot];
    for (int k = 0; k < 3; k++) f->extent[k] = g->extent[k];
}

// ShownRing.publish :136-147, the lock held.
void publish_locked(vxr_ring* r, long long step, long long finished) {
    r->steps[r->back] = step;
    r->finished[r->back] = finished;
    r->ready = r->back;
    for (int k = 0; k < SLOTS; k++) {
        if (k != r->ready && !(r->front_generation == r->generation && k == r->front)) {
            r->back = k;
            break;
        }
    }
}

void forget(vxr_ring* r, Gen* g) {
    for (size_t k = 0; k < r->all.size(); k++)
        if (r->all[k] == g) {
            r->all.erase(r->all.begin() + (long)k);
            break;
        }
}

}  // namespace

extern "C" {

vxr_ring* vxr_ring_create(int32_t device) {
    vxr_ring* r = new vxr_ring();
    r->device = device;
    return r;
}

void vxr_ring_destroy(vxr_ring* r) {
    if (!r) return;
    for (Gen* g : r->all) {
        if (g->bodies > 0) cudaSetDevice(r->device);
        release(g);
    }
    delete r;
}

const char* vxr_ring_error(const vxr_ring* r) { return r ? r->error.c_str() : "no ring"; }

int64_t vxr_ring_install(vxr_ring* r, int32_t shape, int32_t bodies, const double* extent3) {
    if (!r || bodies < 0 || (shape != VXR_RING_SPHERES && shape != VXR_RING_BOXES)) return -VXR_EINVAL;
    Gen* g = new Gen();
    g->shape = shape;
    g->bodies = bodies;
    g->words = (long long)bodies * (shape == VXR_RING_SPHERES ? VXR_SPHERE_SHOWN_STRIDE : VXR_SHOWN_STRIDE);
    if (extent3)
        for (int k = 0; k < 3; k++) g->extent[k] = extent3[k];
    if (bodies > 0) {  // a ring with no bodies keeps no buffers: its roles alone
        if (cudaSetDevice(r->device) != cudaSuccess) {
            delete g;
            return -VXR_ECUDA;
        }
        for (int k = 0; k < SLOTS; k++) {
            if (cudaMalloc(&g->slot[k], sizeof(float) * (size_t)g->words) != cudaSuccess ||
                cudaEventCreateWithFlags(&g->done[k], cudaEventDisableTiming) != cudaSuccess) {
                release(g);
                return -VXR_ECUDA;
            }
        }
    }
    std::lock_guard<std::mutex> hold(r->lock);
    g->id = r->next_id++;
    // ShownRing.install :119-128
    if (r->generation && r->generation != r->front_generation) r->retired.push_back(r->generation);
    r->generation = g;
    r->all.push_back(g);
    r->ready = -1;
    r->back = 0;
    for (int k = 0; k < SLOTS; k++) r->steps[k] = 0;
    return g->id;
}

int32_t vxr_ring_back(vxr_ring* r) {
    if (!r) return -VXR_EINVAL;
    std::lock_guard<std::mutex> hold(r->lock);
    return r->back;
}

int32_t vxr_ring_publish(vxr_ring* r, int64_t step, int64_t finished_ns) {
    if (!r) return VXR_EINVAL;
    std::lock_guard<std::mutex> hold(r->lock);
    if (!r->generation) return VXR_EINVAL;
    publish_locked(r, step, finished_ns);
    return VXR_OK;
}

int32_t vxr_ring_keep(vxr_ring* r, const float* shown, int64_t words, void* stream, int64_t step) {
    if (!r || !shown) return VXR_EINVAL;
    std::lock_guard<std::mutex> hold(r->lock);
    Gen* g = r->generation;
    if (!g || g->bodies == 0 || words != g->words) {
        r->error = "keep: no generation of this size installed";
        return VXR_EINVAL;
    }
    cudaSetDevice(r->device);
    cudaStream_t st = (cudaStream_t)stream;
    const int slot = r->back;
    if (cudaMemcpyAsync(g->slot[slot], shown, sizeof(float) * (size_t)words, cudaMemcpyDeviceToDevice, st) !=
            cudaSuccess ||
        cudaEventRecord(g->done[slot], st) != cudaSuccess) {
        r->error = "keep: the copy or its event did not enqueue";
        return VXR_ECUDA;
    }
    publish_locked(r, step, now_ns());
    return VXR_OK;
}

int32_t vxr_ring_take(vxr_ring* r, vxr_frame* out) {
    if (!r || !out) return VXR_EINVAL;
    std::lock_guard<std::mutex> hold(r->lock);
    // ShownRing.take :161-172
    if (r->ready >= 0) {
        if (r->front_generation && r->front_generation != r->generation) r->retired.push_back(r->front_generation);
        r->front = r->ready;
        r->front_generation = r->generation;
        r->ready = -1;
        describe(r, r->generation, r->front, &r->frame);
        r->taken = true;
    }
    if (!r->taken) return 1;  // nothing published yet
    *out = r->frame;
    return VXR_OK;
}

int32_t vxr_ring_wait(const vxr_frame* f, void* stream) {
    if (!f) return VXR_EINVAL;
    if (!f->event) return VXR_OK;
    return cudaStreamWaitEvent((cudaStream_t)stream, (cudaEvent_t)f->event, 0) == cudaSuccess ? VXR_OK : VXR_ECUDA;
}

int32_t vxr_ring_read(const vxr_frame* f, float* out) {
    if (!f || !out || !f->data) return VXR_EINVAL;
    if (f->event && cudaEventSynchronize((cudaEvent_t)f->event) != cudaSuccess) return VXR_ECUDA;
    return cudaMemcpy(out, f->data, sizeof(float) * (size_t)f->words, cudaMemcpyDeviceToHost) == cudaSuccess
               ? VXR_OK
               : VXR_ECUDA;
}

int32_t vxr_ring_retired(vxr_ring* r, int64_t* ids, int32_t capacity) {
    if (!r) return -VXR_EINVAL;
    std::vector<Gen*> out;
    {
        std::lock_guard<std::mutex> hold(r->lock);
        out.swap(r->retired);
        for (Gen* g : out) forget(r, g);
    }
    int n = 0;
    for (Gen* g : out) {
        if (ids && n < capacity) ids[n] = g->id;
        n++;
        if (g->bodies > 0) cudaSetDevice(r->device);
        release(g);  // no reader can still be reading it
    }
    return n;
}

int32_t vxr_ring_live(vxr_ring* r, int64_t* ids, int32_t capacity) {
    if (!r) return -VXR_EINVAL;
    std::lock_guard<std::mutex> hold(r->lock);
    // ShownRing.all :175-187, without handing anything to be freed: the generations still live, the current one included
    int n = 0;
    for (Gen* g : r->all) {
        if (ids && n < capacity) ids[n] = g->id;
        n++;
    }
    return n;
}

}  // extern "C"
