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

extern "C" bool fireSceneGetPressureStats(FireScene* scene, int* iterations, float* maxResidual, double* l2Residual) {
    if (scene == nullptr || iterations == nullptr || maxResidual == nullptr || l2Residual == nullptr) {
        return fail("fireSceneGetPressureStats: null scene or output pointer.");
    }
    if (!useDevice(scene->device)) return false;
    std::string err;
    if (!scene->scene->pressureStats(*iterations, *maxResidual, *l2Residual, err)) return fail(err);
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

namespace {

// A scene of the batched serving loop, created before the run for one shape
// (with its HDR frame and every buffer a batched step needs).
struct BatchedSlot {
    std::unique_ptr<firesim::Scene> scene;
    void* hdr = nullptr;
    size_t bytes = 0;
    bool busy = false;
};

}  // namespace

struct FireServer {
    int device = 0;
    size_t budget = 0;
    long long maxActiveVoxels = 0;
    double latencyTargetMs = 0.0;  // batched loop: admit while the predicted round time stays within it (0 = off)
    std::vector<FireServeRequest> pending;  // sorted by arrival when the run starts
    std::map<Shape, size_t> bytesByShape;   // measured scene + frame bytes
    std::deque<std::unique_ptr<Active>> pool;  // finished scenes, oldest first
    // The batched loop: its scenes by shape, and the runner that steps them.
    std::map<Shape, std::vector<std::unique_ptr<BatchedSlot>>> slots;
    std::unique_ptr<firesim::BatchRunner> runner;
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
    firesim::deviceFree(a.hdr);
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
    if (server->runner) server->runner->release();
    for (auto& kv : server->slots) {
        for (auto& slot : kv.second) {
            slot->scene->stream = slot->scene->ownStream();
            firesim::deviceFree(slot->hdr);
        }
    }
    delete server;
}

extern "C" bool fireServerSetLatencyTarget(FireServer* server, double roundMs) {
    if (server == nullptr || !(roundMs >= 0.0)) return fail("fireServerSetLatencyTarget: null server or negative target.");
    server->latencyTargetMs = roundMs;
    return true;
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
    if (r.multigridCycles < 0 || r.multigridCycles > 1000 || r.multigridPre < 0 || r.multigridPre > 8 || r.multigridPost < 0 ||
        r.multigridPost > 8 || !(r.pressureTolerance >= 0.0)) {
        return fail("fireServerSubmit: invalid multigrid cycles, smoothing sweeps or pressure tolerance.");
    }
    if (r.multigridCycles > 0 && (r.physics.mode != 1 || r.physics.pressureTop != 1)) {
        return fail("fireServerSubmit: multigrid needs the config physics with p = 0 on the top face (pressureTop 1).");
    }
    server->pending.push_back(r);
    return true;
}

namespace {

using EventRef = std::shared_ptr<CUevent_st>;

EventRef recordEvent(cudaStream_t stream) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    if (cudaEventRecord(e, stream) != cudaSuccess) {
        cudaEventDestroy(e);
        return nullptr;
    }
    return EventRef(e, [](cudaEvent_t ev) { cudaEventDestroy(ev); });
}

bool isBatchable(const FireServeRequest& r) { return r.physics.mode == 1 && r.physics.pressureTop == 1 && r.multigridCycles > 0; }

// The serving loop when every request uses the config physics with the
// multigrid projection: all admitted scenes advance together, one
// BatchRunner sub-step (one launch per stage over all of them) per round.
// Scenes are created before the clock starts, per shape as many as the
// active-cell limit lets run at once (within the budget), so the loop itself
// allocates nothing; a request whose shape has no free scene waits.  A
// round's step latency is the device time between the end of the scene's
// previous round (its admission, for its first step) and the end of this one.
bool runBatched(FireServer* server, std::deque<FireServeRequest>& waiting, double maxSeconds, FireServeReport& rep) {
    using firesim::BatchRunner;
    std::string err;
    if (!server->runner) {
        server->runner = std::make_unique<BatchRunner>();
        if (!server->runner->init(server->device, err)) {
            server->runner.reset();
            return fail("fireServerRun: " + err);
        }
    }
    BatchRunner& runner = *server->runner;
    // Scenes per shape before the run.
    std::map<Shape, int> demand;
    for (const FireServeRequest& r : waiting) ++demand[shapeOf(r)];
    size_t inUse = 0;
    for (auto& kv : server->slots)
        for (auto& slot : kv.second) inUse += slot->bytes;
    for (const auto& kv : demand) {
        const Shape& shape = kv.first;
        const long long cells = static_cast<long long>(std::get<0>(shape)) * std::get<1>(shape) * std::get<2>(shape);
        const long long cap = server->maxActiveVoxels > 0 ? std::max(1LL, server->maxActiveVoxels / cells) : kv.second;
        const int want = static_cast<int>(std::min<long long>({static_cast<long long>(kv.second), cap,
                                                                 static_cast<long long>(firesim::kBatchMaxScenes)}));
        auto& have = server->slots[shape];
        while (static_cast<int>(have.size()) < want) {
            const auto known = server->bytesByShape.find(shape);
            if (known != server->bytesByShape.end() && inUse + known->second > server->budget && !have.empty()) break;
            auto slot = std::make_unique<BatchedSlot>();
            slot->scene = makeScene(server->device, std::get<3>(shape), std::get<4>(shape), std::get<0>(shape), std::get<1>(shape),
                                    std::get<2>(shape), err);
            if (!slot->scene) return fail("fireServerRun: " + err);
            const size_t frame = static_cast<size_t>(std::get<3>(shape)) * std::get<4>(shape) * sizeof(float) * 4;
            if (firesim::deviceAlloc(&slot->hdr, frame, "served HDR frame") != cudaSuccess) {
                cudaGetLastError();
                return fail("fireServerRun: cudaMalloc of a scene's HDR frame failed.");
            }
            // Any request of the shape gives the buffers' sizes; its physics is set again at admission.
            const FireServeRequest* r0 = nullptr;
            for (const FireServeRequest& r : waiting) {
                if (shapeOf(r) == shape) {
                    r0 = &r;
                    break;
                }
            }
            firesim::Scene& sc = *slot->scene;
            if (!sc.setPhysics(r0->physics, err) ||
                !sc.setPressureMultigrid(r0->multigridCycles, r0->multigridPre > 0 ? r0->multigridPre : 2,
                                         r0->multigridPost > 0 ? r0->multigridPost : 2, err) ||
                !sc.setPressureTolerance(r0->pressureTolerance, 1, err) || !sc.prepareBatched(err) ||
                !sc.registerHdrSlot(0, slot->hdr, static_cast<size_t>(std::get<3>(shape)) * 16, FIRE_HDR_RGBA32F, err) ||
                !sc.setActiveSlot(0, err) || !sc.synchronize(err)) {
                firesim::deviceFree(slot->hdr);
                return fail("fireServerRun: " + err);
            }
            sc.stream = runner.stream();
            slot->bytes = sc.deviceBytes() + frame;
            server->bytesByShape[shape] = slot->bytes;
            inUse += slot->bytes;
            have.push_back(std::move(slot));
            if (inUse > server->budget) break;
        }
    }
    rep.deviceBytesPeak = std::max(rep.deviceBytesPeak, inUse);

    struct Live {
        FireServeRequest req{};
        BatchedSlot* slot = nullptr;
        int queued = 0, done = 0;
        EventRef last;  // end of its previous round (the start of its first round, for the first)
    };
    struct Round {
        EventRef start, done;
        long long voxels = 0;
        std::vector<Live*> members;
        std::vector<char> rendered;
    };
    constexpr int kRoundsInFlight = 2;
    std::vector<std::unique_ptr<Live>> live;
    std::deque<Round> rounds;
    std::vector<firesim::Scene*> members, lastMembers;
    std::vector<FireSettings> settings;
    std::vector<int> render;
    std::vector<double> stepMs, frameMs, queueMs;
    long long activeVoxels = 0;
    double msPerVoxel = 0.0;  // device time per cell of a round: a decaying peak over the rounds
    bool ok = true;
    const auto t0 = std::chrono::steady_clock::now();
    auto now = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    while (ok && (!waiting.empty() || !live.empty())) {
        const double t = now();
        if (t > maxSeconds) break;
        bool progressed = false;
        // Admission in arrival order, while the active-cell limit holds and a scene of the shape is free.
        while (!waiting.empty() && waiting.front().arrivalSeconds <= t && static_cast<int>(live.size()) < firesim::kBatchMaxScenes) {
            const FireServeRequest& r = waiting.front();
            const long long voxels = static_cast<long long>(r.nx) * r.ny * r.nz;
            if (server->maxActiveVoxels > 0 && !live.empty() && activeVoxels + voxels > server->maxActiveVoxels) break;
            // Latency target: the rounds' measured device time per cell predicts the round time.
            if (server->latencyTargetMs > 0.0 && msPerVoxel > 0.0 && !live.empty() &&
                static_cast<double>(activeVoxels + voxels) * msPerVoxel > server->latencyTargetMs) {
                break;
            }
            BatchedSlot* slot = nullptr;
            for (auto& sl : server->slots[shapeOf(r)]) {
                if (!sl->busy) {
                    slot = sl.get();
                    break;
                }
            }
            if (slot == nullptr) break;
            firesim::Scene& sc = *slot->scene;
            if (!sc.setPhysics(r.physics, err) ||
                !sc.setPressureMultigrid(r.multigridCycles, r.multigridPre > 0 ? r.multigridPre : 2, r.multigridPost > 0 ? r.multigridPost : 2,
                                         err) ||
                !sc.setPressureTolerance(r.pressureTolerance, 1, err)) {
                ok = fail("fireServerRun: " + err);
                break;
            }
            auto l = std::make_unique<Live>();
            l->req = r;
            l->slot = slot;
            l->last = recordEvent(runner.stream());
            if (!l->last) {
                ok = fail("fireServerRun: cudaEventRecord failed.");
                break;
            }
            slot->busy = true;
            activeVoxels += voxels;
            queueMs.push_back((t - r.arrivalSeconds) * 1e3);
            live.push_back(std::move(l));
            waiting.pop_front();
            rep.admittedPeak = std::max(rep.admittedPeak, static_cast<int>(live.size()));
            progressed = true;
        }
        if (!ok) break;
        // One round over every live scene with steps left to queue.
        if (static_cast<int>(rounds.size()) < kRoundsInFlight) {
            members.clear();
            settings.clear();
            render.clear();
            Round round;
            for (auto& lp : live) {
                Live& l = *lp;
                if (l.queued >= l.req.steps) continue;
                members.push_back(l.slot->scene.get());
                FireSettings st = l.req.settings;
                st.reset = l.queued == 0 ? 1 : 0;
                settings.push_back(st);
                const bool r = l.req.renderEvery > 0 && (l.queued % l.req.renderEvery) == l.req.renderEvery - 1;
                render.push_back(r ? 1 : 0);
                round.members.push_back(&l);
                round.rendered.push_back(r ? 1 : 0);
            }
            if (!members.empty()) {
                if (members != lastMembers) {
                    if (!runner.setScenes(members, err)) {
                        ok = fail("fireServerRun: " + err);
                        break;
                    }
                    lastMembers = members;
                }
                round.start = recordEvent(runner.stream());
                // A scene's first step is timed from the start of its first
                // round; the wait before it (behind the rounds in flight) is
                // its queue time, like the wait before admission.
                for (Live* l : round.members) {
                    if (l->queued == 0) l->last = round.start;
                }
                if (!runner.run(settings.data(), render.data(), err)) {
                    ok = fail("fireServerRun: " + err);
                    break;
                }
                round.done = recordEvent(runner.stream());
                for (Live* l : round.members) round.voxels += static_cast<long long>(l->req.nx) * l->req.ny * l->req.nz;
                if (!round.done) {
                    ok = fail("fireServerRun: cudaEventRecord failed.");
                    break;
                }
                for (Live* l : round.members) ++l->queued;
                rounds.push_back(std::move(round));
                progressed = true;
            }
        }
        // Completed rounds, in order.
        while (!rounds.empty() && cudaEventQuery(rounds.front().done.get()) == cudaSuccess) {
            Round& r = rounds.front();
            float roundMs = 0.0f;
            if (r.start && cudaEventElapsedTime(&roundMs, r.start.get(), r.done.get()) == cudaSuccess && r.voxels > 0) {
                // A decaying peak of the rounds' time per cell, so that the
                // admission plans for the dearer rounds (renders, more
                // multigrid cycles) rather than the mean.
                const double sample = roundMs / static_cast<double>(r.voxels);
                msPerVoxel = std::max(sample, 0.99 * msPerVoxel);
            }
            for (size_t i = 0; i < r.members.size(); ++i) {
                Live& l = *r.members[i];
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, l.last.get(), r.done.get());
                stepMs.push_back(ms);
                if (r.rendered[i]) frameMs.push_back(ms);
                rep.voxelSteps += static_cast<double>(l.req.nx) * l.req.ny * l.req.nz;
                l.last = r.done;
                ++l.done;
            }
            rounds.pop_front();
            progressed = true;
        }
        // Finished scenes leave; their scene is free for the next request of the shape.
        for (size_t i = 0; i < live.size();) {
            Live& l = *live[i];
            if (l.done < l.req.steps) {
                ++i;
                continue;
            }
            firesim::Scene& sc = *l.slot->scene;
            if (l.req.resultHeat && (!sc.synchronize(err) ||
                                     !sc.getField(FIRE_FIELD_HEAT, l.req.resultHeat,
                                                  static_cast<size_t>(l.req.nx) * l.req.ny * l.req.nz * sizeof(float), err))) {
                ok = fail("fireServerRun: " + err);
                break;
            }
            if (l.req.resultHdr &&
                cudaMemcpy(l.req.resultHdr, l.slot->hdr, frameBytes(l.req), cudaMemcpyDeviceToHost) != cudaSuccess) {
                ok = fail("fireServerRun: copy of a finished scene's frame failed.");
                break;
            }
            activeVoxels -= static_cast<long long>(l.req.nx) * l.req.ny * l.req.nz;
            l.slot->busy = false;
            live.erase(live.begin() + static_cast<long>(i));
            ++rep.completed;
            progressed = true;
        }
        if (!ok) break;
        if (!progressed) {
            if (live.empty() && !waiting.empty()) {
                const double wait = waiting.front().arrivalSeconds - now();
                if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.001)));
            } else {
                std::this_thread::sleep_for(std::chrono::microseconds(20));
            }
        }
    }
    if (cudaStreamSynchronize(runner.stream()) != cudaSuccess) ok = fail("fireServerRun: the batch stream failed.");
    if (ok && !runner.checkStatus(err)) ok = fail("fireServerRun: " + err);
    for (auto& l : live) l->slot->busy = false;
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
    return ok;
}

}  // namespace

extern "C" bool fireServerRun(FireServer* server, double maxSeconds, FireServeReport* report) {
    if (server == nullptr || report == nullptr) return fail("fireServerRun: null server or report.");
    if (!useDevice(server->device)) return false;
    const bool batched = !server->pending.empty() &&
                         std::all_of(server->pending.begin(), server->pending.end(), [](const FireServeRequest& r) { return isBatchable(r); });
    if (batched) {
        std::stable_sort(server->pending.begin(), server->pending.end(),
                         [](const FireServeRequest& a, const FireServeRequest& b) { return a.arrivalSeconds < b.arrivalSeconds; });
        std::deque<FireServeRequest> waiting(server->pending.begin(), server->pending.end());
        server->pending.clear();
        FireServeReport rep{};
        rep.submitted = static_cast<int>(waiting.size());
        const bool ok = runBatched(server, waiting, maxSeconds, rep);
        *report = rep;
        return ok;
    }
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
                if (firesim::deviceAlloc(&a->hdr, frameBytes(r), "served HDR frame") != cudaSuccess) {
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
            // The pressure solver of this request (a pooled scene keeps its previous one otherwise).
            const int pre = r.multigridPre > 0 ? r.multigridPre : 2, post = r.multigridPost > 0 ? r.multigridPost : 2;
            if (!a->scene->setPressureMultigrid(r.multigridCycles, pre, post, err) ||
                !a->scene->setPressureTolerance(r.pressureTolerance, r.multigridCycles > 0 ? 1 : 10, err)) {
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
