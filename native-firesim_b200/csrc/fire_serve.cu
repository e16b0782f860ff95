// fire_serve.cu -- independent scenes, batched sub-steps and a serving loop.
//
// The reference drives one process-wide scene.  Here every FireScene is a
// firesim::Scene with its own fields and stream, so the kernels of many
// scenes run side by side on the GPU, and a FireServer admits scenes as they
// arrive and steps all of them, one step per round, within a device-memory
// budget.  Scenes share nothing, so each scene's result is the same bits
// whether it runs alone or in a mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/fire_ext.h"
#include "fire_scene.h"

namespace firesim {
void setLastErrorMessage(const char* msg);
}  // namespace firesim

struct FireScene {
    std::unique_ptr<firesim::Scene> scene;
    int device = 0;
};

namespace {

bool fail(const std::string& msg) {
    firesim::setLastErrorMessage(msg.c_str());
    return false;
}

bool useDevice(int device) {
    const cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    return true;
}

std::unique_ptr<firesim::Scene> makeScene(int device, int fw, int fh, int nx, int ny, int nz, std::string& err) {
    auto scene = std::make_unique<firesim::Scene>();
    if (!scene->init(device, fw, fh, nx, ny, nz, err) || !scene->reset(err)) return nullptr;
    return scene;
}

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * static_cast<double>(v.size() - 1);
    const size_t lo = static_cast<size_t>(std::floor(pos));
    const size_t hi = std::min(v.size() - 1, lo + 1);
    return v[lo] + (v[hi] - v[lo]) * (pos - static_cast<double>(lo));
}

}  // namespace

// ---------------------------------------------------------------------------
// FireScene

extern "C" FireScene* fireSceneCreate(int device, int frameW, int frameH, int nx, int ny, int nz) {
    if (!useDevice(device)) return nullptr;
    std::string err;
    auto scene = makeScene(device, frameW, frameH, nx, ny, nz, err);
    if (!scene) {
        fail(err);
        return nullptr;
    }
    FireScene* h = new FireScene;
    h->scene = std::move(scene);
    h->device = device;
    return h;
}

extern "C" void fireSceneDestroy(FireScene* scene) {
    if (scene == nullptr) return;
    cudaSetDevice(scene->device);
    delete scene;
}

extern "C" size_t fireSceneDeviceBytes(const FireScene* scene) { return scene ? scene->scene->deviceBytes() : 0; }

extern "C" bool fireSceneSetPressureSolver(FireScene* scene, int iterations, float omega) {
    if (scene == nullptr) return fail("Scene handle was null.");
    std::string err;
    if (!scene->scene->setPressureSolver(iterations, omega, err)) return fail(err);
    return true;
}

extern "C" bool fireSceneSetPressureTolerance(FireScene* scene, double maxResidual, int checkEvery) {
    if (scene == nullptr) return fail("Scene handle was null.");
    std::string err;
    if (!scene->scene->setPressureTolerance(maxResidual, checkEvery, err)) return fail(err);
    return true;
}

extern "C" bool fireSceneSetPhysicsParams(FireScene* scene, const FirePhysicsParams* params) {
    if (scene == nullptr) return fail("Scene handle was null.");
    if (params == nullptr) return fail("Physics parameter pointer was null.");
    std::string err;
    if (!scene->scene->setPhysics(*params, err)) return fail(err);
    return true;
}

extern "C" bool fireSceneSetPressureMultigrid(FireScene* scene, int maxCycles, int preSmooth, int postSmooth) {
    if (scene == nullptr) return fail("Scene handle was null.");
    std::string err;
    if (!scene->scene->setPressureMultigrid(maxCycles, preSmooth, postSmooth, err)) return fail(err);
    return true;
}

extern "C" bool fireSceneSetHdrBuffer(FireScene* scene, void* devicePtr, size_t pitchBytes, int format) {
    if (scene == nullptr) return fail("Scene handle was null.");
    if (!useDevice(scene->device)) return false;
    std::string err;
    if (!scene->scene->registerHdrSlot(0, devicePtr, pitchBytes, format, err) || !scene->scene->setActiveSlot(0, err)) return fail(err);
    return true;
}

extern "C" bool fireSceneStep(FireScene* scene, const FireSettings* settings, int render) {
    if (scene == nullptr) return fail("Scene handle was null.");
    if (settings == nullptr) return fail("Settings pointer was null.");
    if (!useDevice(scene->device)) return false;
    std::string err;
    if (!scene->scene->frame(nullptr, *settings, nullptr, true, true, render != 0, err)) return fail(err);
    return true;
}

extern "C" bool fireSceneSynchronize(FireScene* scene) {
    if (scene == nullptr) return fail("Scene handle was null.");
    if (!useDevice(scene->device)) return false;
    std::string err;
    if (!scene->scene->synchronize(err)) return fail(err);
    return true;
}

extern "C" bool fireSceneGetStream(FireScene* scene, void** stream) {
    if (scene == nullptr || stream == nullptr) return fail("Scene handle or stream pointer was null.");
    *stream = scene->scene->stream;
    return true;
}

extern "C" bool fireSceneGetField(FireScene* scene, int field, void* host, size_t bytes) {
    if (scene == nullptr || host == nullptr) return fail("Scene handle or host pointer was null.");
    if (!useDevice(scene->device)) return false;
    std::string err;
    if (!scene->scene->synchronize(err) || !scene->scene->getField(field, host, bytes, err)) return fail(err);
    return true;
}

extern "C" bool fireBatchStep(FireScene* const* scenes, const FireSettings* settings, const int* render, int n) {
    if (n < 0 || (n > 0 && (scenes == nullptr || settings == nullptr))) return fail("fireBatchStep: null scene or settings array.");
    for (int i = 0; i < n; ++i) {
        if (!fireSceneStep(scenes[i], &settings[i], render ? render[i] : 0)) return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// FireServer

namespace {

struct InFlight {
    cudaEvent_t done;
    bool rendered;
};

struct Active {
    FireServeRequest req{};
    std::unique_ptr<firesim::Scene> scene;
    void* hdr = nullptr;
    size_t bytes = 0;
    int queued = 0;                 // steps queued so far
    cudaEvent_t last = nullptr;     // completion of the previous step (admission for the first)
    std::deque<InFlight> inflight;  // queued, not yet observed complete
    std::vector<cudaEvent_t> spare;
};

constexpr int kStepsInFlight = 2;

}  // namespace

using Shape = std::tuple<int, int, int, int, int>;  // nx, ny, nz, frameW, frameH

struct FireServer {
    int device = 0;
    size_t budget = 0;
    long long maxActiveVoxels = 0;
    std::vector<FireServeRequest> pending;  // sorted by arrival when the run starts
    std::map<Shape, size_t> bytesByShape;   // measured scene + frame bytes
    std::deque<std::unique_ptr<Active>> pool;  // finished scenes, oldest first
};

namespace {

cudaEvent_t takeEvent(Active& a) {
    if (!a.spare.empty()) {
        cudaEvent_t e = a.spare.back();
        a.spare.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void releaseActive(Active& a) {
    if (a.scene) cudaStreamSynchronize(a.scene->stream);
    for (InFlight& f : a.inflight) cudaEventDestroy(f.done);
    for (cudaEvent_t e : a.spare) cudaEventDestroy(e);
    if (a.last) cudaEventDestroy(a.last);
    a.inflight.clear();
    a.spare.clear();
    a.last = nullptr;
    if (a.hdr) cudaFree(a.hdr);
    a.hdr = nullptr;
    a.scene.reset();
}

size_t frameBytes(const FireServeRequest& r) { return static_cast<size_t>(r.frameW) * r.frameH * sizeof(float) * 4; }

Shape shapeOf(const FireServeRequest& r) { return std::make_tuple(r.nx, r.ny, r.nz, r.frameW, r.frameH); }

}  // namespace

extern "C" FireServer* fireServerCreate(int device, size_t budgetBytes) {
    if (!useDevice(device)) return nullptr;
    FireServer* s = new FireServer;
    s->device = device;
    s->budget = budgetBytes;
    return s;
}

extern "C" void fireServerDestroy(FireServer* server) {
    if (server == nullptr) return;
    cudaSetDevice(server->device);
    for (auto& a : server->pool) releaseActive(*a);
    delete server;
}

extern "C" bool fireServerSetLimits(FireServer* server, long long maxActiveVoxels) {
    if (server == nullptr || maxActiveVoxels < 0) return fail("fireServerSetLimits: null server or negative limit.");
    server->maxActiveVoxels = maxActiveVoxels;
    return true;
}

extern "C" bool fireServerSubmit(FireServer* server, const FireServeRequest* request) {
    if (server == nullptr || request == nullptr) return fail("fireServerSubmit: null server or request.");
    const FireServeRequest& r = *request;
    if (r.nx < 2 || r.ny < 2 || r.nz < 2 || r.frameW < 1 || r.frameH < 1 || r.steps < 1 || r.renderEvery < 0) {
        return fail("fireServerSubmit: invalid grid, frame, step count or render interval.");
    }
    std::string err;
    if (r.physics.mode != 0 && !firesim::validatePhysicsParams(r.physics, err)) return fail("fireServerSubmit: " + err);
    server->pending.push_back(r);
    return true;
}

extern "C" bool fireServerRun(FireServer* server, double maxSeconds, FireServeReport* report) {
    if (server == nullptr || report == nullptr) return fail("fireServerRun: null server or report.");
    if (!useDevice(server->device)) return false;
    std::stable_sort(server->pending.begin(), server->pending.end(),
                     [](const FireServeRequest& a, const FireServeRequest& b) { return a.arrivalSeconds < b.arrivalSeconds; });
    std::deque<FireServeRequest> waiting(server->pending.begin(), server->pending.end());
    server->pending.clear();
    FireServeReport rep{};
    rep.submitted = static_cast<int>(waiting.size());
    std::vector<double> stepMs, frameMs, queueMs;
    std::vector<std::unique_ptr<Active>> active;
    size_t inUse = 0;
    for (auto& p : server->pool) inUse += p->bytes;
    long long activeVoxels = 0;
    std::string err;
    bool ok = true;
    const auto t0 = std::chrono::steady_clock::now();
    auto now = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };

    while (ok && (!waiting.empty() || !active.empty())) {
        const double t = now();
        if (t > maxSeconds) break;
        // Admission: in arrival order, while the voxel limit and the budget hold.
        while (!waiting.empty() && waiting.front().arrivalSeconds <= t) {
            const FireServeRequest& r = waiting.front();
            const long long voxels = static_cast<long long>(r.nx) * r.ny * r.nz;
            if (server->maxActiveVoxels > 0 && !active.empty() && activeVoxels + voxels > server->maxActiveVoxels) break;
            const Shape shape = shapeOf(r);
            // A pooled scene of this shape is taken as it is.
            std::unique_ptr<Active> a;
            for (auto it = server->pool.begin(); it != server->pool.end(); ++it) {
                if (shapeOf((*it)->req) == shape) {
                    a = std::move(*it);
                    server->pool.erase(it);
                    break;
                }
            }
            if (!a) {
                // A new scene: make room by freeing pooled scenes, oldest first.
                const auto known = server->bytesByShape.find(shape);
                const size_t need = known != server->bytesByShape.end() ? known->second : 0;
                while (!server->pool.empty() && inUse + need > server->budget) {
                    inUse -= server->pool.front()->bytes;
                    releaseActive(*server->pool.front());
                    server->pool.pop_front();
                }
                if (known != server->bytesByShape.end() && inUse + need > server->budget && !active.empty()) break;
                a = std::make_unique<Active>();
                a->scene = makeScene(server->device, r.frameW, r.frameH, r.nx, r.ny, r.nz, err);
                if (!a->scene) {
                    ok = fail(err);
                    break;
                }
                if (cudaMalloc(&a->hdr, frameBytes(r)) != cudaSuccess) {
                    cudaGetLastError();
                    ok = fail("fireServerRun: cudaMalloc of a scene's HDR frame failed.");
                    break;
                }
                if (!a->scene->registerHdrSlot(0, a->hdr, static_cast<size_t>(r.frameW) * 16, FIRE_HDR_RGBA32F, err) ||
                    !a->scene->setActiveSlot(0, err)) {
                    ok = fail(err);
                    break;
                }
                a->bytes = a->scene->deviceBytes() + frameBytes(r);
                server->bytesByShape[shape] = a->bytes;
                if (inUse + a->bytes > server->budget && !active.empty()) {
                    // The first scene of this shape did not fit after all: give it back.
                    releaseActive(*a);
                    break;
                }
                inUse += a->bytes;
            } else {
                // A pooled scene starts like a new one: clocks and fields reset, frame cleared.
                if (!a->scene->reset(err) ||
                    cudaMemsetAsync(a->hdr, 0, frameBytes(a->req), a->scene->stream) != cudaSuccess) {
                    ok = fail(err.empty() ? std::string("fireServerRun: clearing a pooled scene failed.") : err);
                    break;
                }
            }
            a->req = r;
            a->queued = 0;
            if (r.sorIterations > 0 && !a->scene->setPressureSolver(r.sorIterations, r.sorOmega, err)) {
                ok = fail(err);
                break;
            }
            // The request's physics; its first step resets the fields in that physics.
            FirePhysicsParams physics = r.physics;
            if (physics.mode == 0) firesim::defaultPhysicsParams(physics, r.nx, r.ny, r.nz);
            if (!a->scene->setPhysics(physics, err)) {
                ok = fail(err);
                break;
            }
            a->last = takeEvent(*a);
            cudaEventRecord(a->last, a->scene->stream);
            activeVoxels += voxels;
            rep.deviceBytesPeak = std::max(rep.deviceBytesPeak, inUse);
            queueMs.push_back((t - r.arrivalSeconds) * 1e3);
            waiting.pop_front();
            active.push_back(std::move(a));
            rep.admittedPeak = std::max(rep.admittedPeak, static_cast<int>(active.size()));
        }
        if (!ok) break;
        // One round: every admitted scene with room in its queue takes its next step.
        bool progressed = false;
        for (auto& ap : active) {
            Active& a = *ap;
            if (a.queued >= a.req.steps || static_cast<int>(a.inflight.size()) >= kStepsInFlight) continue;
            FireSettings s = a.req.settings;
            s.reset = a.queued == 0 ? 1 : 0;
            const bool render = a.req.renderEvery > 0 && (a.queued % a.req.renderEvery) == a.req.renderEvery - 1;
            if (!a.scene->frame(nullptr, s, nullptr, true, true, render, err)) {
                ok = fail(err);
                break;
            }
            InFlight f{takeEvent(a), render};
            cudaEventRecord(f.done, a.scene->stream);
            a.inflight.push_back(f);
            ++a.queued;
            progressed = true;
        }
        if (!ok) break;
        // Completions, in order per scene.
        for (auto& ap : active) {
            Active& a = *ap;
            while (!a.inflight.empty() && cudaEventQuery(a.inflight.front().done) == cudaSuccess) {
                InFlight f = a.inflight.front();
                a.inflight.pop_front();
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, a.last, f.done);
                stepMs.push_back(ms);
                if (f.rendered) frameMs.push_back(ms);
                rep.voxelSteps += static_cast<double>(a.req.nx) * a.req.ny * a.req.nz;
                a.spare.push_back(a.last);
                a.last = f.done;
                progressed = true;
            }
        }
        // Finished scenes leave and free their memory.
        for (size_t i = 0; i < active.size();) {
            Active& a = *active[i];
            if (a.queued >= a.req.steps && a.inflight.empty()) {
                if (!a.scene->synchronize(err)) {
                    ok = fail(err);
                    break;
                }
                if (a.req.resultHeat && !a.scene->getField(FIRE_FIELD_HEAT, a.req.resultHeat,
                                                           static_cast<size_t>(a.req.nx) * a.req.ny * a.req.nz * sizeof(float), err)) {
                    ok = fail(err);
                    break;
                }
                if (a.req.resultHdr && cudaMemcpy(a.req.resultHdr, a.hdr, frameBytes(a.req), cudaMemcpyDeviceToHost) != cudaSuccess) {
                    ok = fail("fireServerRun: copy of a finished scene's frame failed.");
                    break;
                }
                activeVoxels -= static_cast<long long>(a.req.nx) * a.req.ny * a.req.nz;
                if (a.last) {
                    a.spare.push_back(a.last);
                    a.last = nullptr;
                }
                server->pool.push_back(std::move(active[i]));
                active.erase(active.begin() + static_cast<long>(i));
                ++rep.completed;
            } else {
                ++i;
            }
        }
        if (!ok) break;
        if (!progressed) {
            if (active.empty() && !waiting.empty()) {
                const double wait = waiting.front().arrivalSeconds - now();
                if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.001)));
            } else {
                std::this_thread::sleep_for(std::chrono::microseconds(20));
            }
        }
    }
    for (auto& ap : active) {
        inUse -= ap->bytes;
        releaseActive(*ap);
    }
    rep.seconds = now();
    rep.stepMsP50 = percentile(stepMs, 0.50);
    rep.stepMsP95 = percentile(stepMs, 0.95);
    rep.stepMsP99 = percentile(stepMs, 0.99);
    rep.stepMsMax = stepMs.empty() ? 0.0 : *std::max_element(stepMs.begin(), stepMs.end());
    rep.frameMsP50 = percentile(frameMs, 0.50);
    rep.frameMsP95 = percentile(frameMs, 0.95);
    rep.frameMsP99 = percentile(frameMs, 0.99);
    rep.queueMsP50 = percentile(queueMs, 0.50);
    rep.queueMsP99 = percentile(queueMs, 0.99);
    *report = rep;
    return ok;
}
