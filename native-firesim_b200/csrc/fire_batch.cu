// fire_batch.cu -- many scenes of the config physics stepped together, one
// launch per stage over all of them.
//
// fireBatchStep (fire_serve.cu) queues each scene's own launch sequence on
// its own stream, so a batch of 48 small scenes is ~10 launches per scene per
// sub-step and the small scenes' solves run side by side but each bound by
// its own latency.  BatchRunner instead queues, per sub-step, one upload of
// the scenes' step descriptors and then one launch per stage whose blocks
// cover every scene (fire_config.cu, batch*), with the whole pressure solve
// of every scene in one persistent multigrid launch (fire_mg.cu, mgSolve).
// Per element the kernels run the single-scene bodies, so every scene gives
// the same bits alone or in the batch.  The FireBatch C API and the serving
// loop (fire_serve.cu) are built on it.
//
// While a scene belongs to a FireBatch, its work (its resets, its field
// reads) runs on the batch's stream, so it stays ordered with the batch's
// launches; destroying the batch gives each scene its own stream back.
// Destroy the batch before its scenes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/fire_ext.h"
#include "fire_scene.h"

namespace firesim {

void setLastErrorMessage(const char* msg);

BatchRunner::~BatchRunner() { release(); }

void BatchRunner::release() {
    if (stream_ != nullptr) cudaStreamSynchronize(stream_);
    solver_.release();
    deviceFree(dScenes_);
    deviceFree(dPlan_);
    for (int k = 0; k < kRing; ++k) {
        if (host_[k] != nullptr) cudaFreeHost(host_[k]);
        if (copied_[k] != nullptr) cudaEventDestroy(copied_[k]);
        host_[k] = nullptr;
        copied_[k] = nullptr;
    }
    if (hostStatus_ != nullptr) cudaFreeHost(hostStatus_);
    if (stream_ != nullptr) cudaStreamDestroy(stream_);
    dScenes_ = nullptr;
    dPlan_ = nullptr;
    hostStatus_ = nullptr;
    stream_ = nullptr;
    scenes_.clear();
}

bool BatchRunner::init(int device, std::string& err) {
    device_ = device;
    const size_t staging = kBatchMaxScenes * sizeof(BatchScene) + sizeof(BatchPlan);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&hostStatus_), sizeof(unsigned), cudaHostAllocMapped);
    if (e == cudaSuccess) e = deviceAlloc(reinterpret_cast<void**>(&dScenes_), kBatchMaxScenes * sizeof(BatchScene), "batch scene table");
    if (e == cudaSuccess) e = deviceAlloc(reinterpret_cast<void**>(&dPlan_), sizeof(BatchPlan), "batch plan");
    for (int k = 0; k < kRing && e == cudaSuccess; ++k) {
        e = cudaHostAlloc(reinterpret_cast<void**>(&host_[k]), staging, cudaHostAllocDefault);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&copied_[k], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        err = std::string("batch: ") + cudaGetErrorString(e);
        release();
        return false;
    }
    *hostStatus_ = 0;
    return true;
}

bool BatchRunner::setScenes(const std::vector<Scene*>& scenes, std::string& err) {
    const int n = static_cast<int>(scenes.size());
    if (n > kBatchMaxScenes) {
        err = "batch: at most " + std::to_string(kBatchMaxScenes) + " scenes";
        return false;
    }
    if (n == 0) {
        scenes_.clear();
        return true;
    }
    const Scene& first = *scenes[0];
    std::vector<MgScene> mg(n);
    for (int i = 0; i < n; ++i) {
        const Scene& s = *scenes[i];
        if (!s.incrementalProjection()) {
            err = "batch: scene " + std::to_string(i) +
                  " is not the config physics with p = 0 on the top face and the multigrid solve (mode 1, pressureTop 1, multigrid cycles > 0)";
            return false;
        }
        if (s.multigridCycles() != first.multigridCycles() || s.multigridPre() != first.multigridPre() ||
            s.multigridPost() != first.multigridPost() || s.pressureTolerance() != first.pressureTolerance()) {
            err = "batch: the scenes' multigrid cycles, smoothing sweeps and tolerance must agree";
            return false;
        }
        if (!scenes[i]->multigridScene(mg[i], err)) return false;
    }
    if (!solver_.plan(device_, mg, first.multigridCycles(), first.multigridPre(), first.multigridPost(), first.pressureTolerance(), stream_,
                      err)) {
        return false;
    }
    scenes_ = scenes;
    return true;
}

bool BatchRunner::run(const FireSettings* settings, const int* render, std::string& err) {
    const int n = static_cast<int>(scenes_.size());
    if (n == 0) return true;
    // Validate before any scene's host state moves.
    for (int i = 0; i < n; ++i) {
        if (render != nullptr && render[i] != 0 && !scenes_[i]->hasHdrOutput()) {
            err = "scene " + std::to_string(i) + ": HDR output buffer slot is not registered.";
            return false;
        }
    }
    // The staging buffer of this sub-step: wait until its last copy has run.
    const int k = slot_;
    slot_ = (slot_ + 1) % kRing;
    cudaError_t e = cudaEventSynchronize(copied_[k]);
    if (e != cudaSuccess) {
        err = std::string("batch: waiting for a staging copy: ") + cudaGetErrorString(e);
        return false;
    }
    BatchScene* desc = reinterpret_cast<BatchScene*>(host_[k]);
    BatchPlan* plan = reinterpret_cast<BatchPlan*>(host_[k] + kBatchMaxScenes * sizeof(BatchScene));
    std::memset(plan, 0, sizeof(BatchPlan));
    plan->scenes = n;
    bool anyRender = false;
    for (int i = 0; i < n; ++i) {
        const bool r = render != nullptr && render[i] != 0;
        anyRender = anyRender || r;
        if (!scenes_[i]->batchStep(desc[i], settings[i], r, err)) {
            err = "scene " + std::to_string(i) + ": " + err;
            return false;
        }
        for (int sp = 0; sp < kBatchSpaces; ++sp) {
            const int perBlock = kBatchThreads * batchPerThread(sp);
            plan->start[sp][i + 1] = plan->start[sp][i] + (desc[i].count[sp] + perBlock - 1) / perBlock;
        }
    }
    cudaStream_t s = stream_;
    e = cudaMemcpyAsync(dScenes_, desc, n * sizeof(BatchScene), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dPlan_, plan, sizeof(BatchPlan), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaEventRecord(copied_[k], s);
    if (e != cudaSuccess) {
        err = std::string("batch: descriptor upload: ") + cudaGetErrorString(e);
        return false;
    }
    const BatchScene* dS = dScenes_;
    const BatchPlan* dP = dPlan_;
    unsigned long long launched = 0;
    auto go = [&](void (*kernel)(const BatchScene*, const BatchPlan*), int space) {
        const int blocks = plan->start[space][n];
        if (blocks > 0) {
            kernel<<<blocks, kBatchThreads, 0, s>>>(dS, dP);
            ++launched;
        }
    };
    go(batchAdvectVelocity, kBatchFaces);
    go(batchAdvectScalars, kBatchCells);
    go(batchVorticity, kBatchCells);
    go(batchCellForce, kBatchCells);
    go(batchApplyForces, kBatchFaces);
    go(batchPrepareIncrement, kBatchCells);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string("batch: stage launch: ") + cudaGetErrorString(e);
        return false;
    }
    if (!solver_.launch(s, hostStatus_, err)) return false;
    ++launched;
    go(batchSubtractIncrement, kBatchCells);
    if (anyRender) {
        go(batchTransmittance, kBatchLight);
        go(batchRaymarch, kBatchPixels);
        go(batchPackHdr, kBatchPixels);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string("batch: stage launch: ") + cudaGetErrorString(e);
        return false;
    }
    launches_ += launched;
    return true;
}

bool BatchRunner::checkStatus(std::string& err) {
    const unsigned st = *reinterpret_cast<volatile unsigned*>(hostStatus_);
    if (st == 0) return true;
    *hostStatus_ = 0;
    err = "multigrid solve: a grid barrier wait timed out in phase " + std::to_string(st & ~kMgStatusFlag);
    return false;
}

}  // namespace firesim

namespace {

bool fail(const std::string& msg) {
    firesim::setLastErrorMessage(msg.c_str());
    return false;
}

}  // namespace

struct FireBatch {
    firesim::BatchRunner runner;
    int device = 0;
};

extern "C" FireBatch* fireBatchCreate(FireScene* const* handles, int n) {
    if (handles == nullptr || n < 1 || n > firesim::kBatchMaxScenes) {
        fail("fireBatchCreate: 1 to " + std::to_string(firesim::kBatchMaxScenes) + " scene handles are needed.");
        return nullptr;
    }
    for (int i = 0; i < n; ++i) {
        if (handles[i] == nullptr) {
            fail("fireBatchCreate: a scene handle was null.");
            return nullptr;
        }
        if (handles[i]->device != handles[0]->device) {
            fail("fireBatchCreate: the scenes are on different devices.");
            return nullptr;
        }
        for (int j = 0; j < i; ++j) {
            if (handles[j] == handles[i]) {
                fail("fireBatchCreate: a scene appears twice.");
                return nullptr;
            }
        }
    }
    auto b = std::make_unique<FireBatch>();
    b->device = handles[0]->device;
    std::string err;
    if (!b->runner.init(b->device, err)) {
        fail("fireBatchCreate: " + err);
        return nullptr;
    }
    // The scenes' queued work first, then every scene runs on the batch stream.
    std::vector<firesim::Scene*> scenes;
    for (int i = 0; i < n; ++i) {
        firesim::Scene* s = handles[i]->scene.get();
        if (cudaStreamSynchronize(s->stream) != cudaSuccess) {
            fail("fireBatchCreate: a scene's stream failed.");
            return nullptr;
        }
        scenes.push_back(s);
    }
    for (firesim::Scene* s : scenes) s->stream = b->runner.stream();
    if (!b->runner.setScenes(scenes, err)) {
        for (firesim::Scene* s : scenes) s->stream = s->ownStream();
        fail("fireBatchCreate: " + err);
        return nullptr;
    }
    return b.release();
}

extern "C" void fireBatchDestroy(FireBatch* batch) {
    if (batch == nullptr) return;
    cudaSetDevice(batch->device);
    if (batch->runner.stream() != nullptr) cudaStreamSynchronize(batch->runner.stream());
    for (firesim::Scene* s : batch->runner.scenes()) s->stream = s->ownStream();
    batch->runner.release();
    delete batch;
}

extern "C" bool fireBatchRun(FireBatch* batch, const FireSettings* settings, const int* render) {
    if (batch == nullptr || settings == nullptr) return fail("fireBatchRun: null batch or settings.");
    if (cudaSetDevice(batch->device) != cudaSuccess) return fail("fireBatchRun: cudaSetDevice failed.");
    std::string err;
    if (!batch->runner.run(settings, render, err)) return fail("fireBatchRun: " + err);
    return true;
}

extern "C" bool fireBatchSynchronize(FireBatch* batch) {
    if (batch == nullptr) return fail("fireBatchSynchronize: null batch.");
    if (cudaSetDevice(batch->device) != cudaSuccess) return fail("fireBatchSynchronize: cudaSetDevice failed.");
    const cudaError_t e = cudaStreamSynchronize(batch->runner.stream());
    if (e != cudaSuccess) return fail(std::string("fireBatchSynchronize: ") + cudaGetErrorString(e));
    std::string err;
    if (!batch->runner.checkStatus(err)) return fail("fireBatchSynchronize: " + err);
    return true;
}

extern "C" bool fireBatchGetStream(FireBatch* batch, void** stream) {
    if (batch == nullptr || stream == nullptr) return fail("fireBatchGetStream: null batch or stream pointer.");
    *stream = batch->runner.stream();
    return true;
}

extern "C" bool fireBatchGetLaunchCount(FireBatch* batch, unsigned long long* count) {
    if (batch == nullptr || count == nullptr) return fail("fireBatchGetLaunchCount: null batch or count pointer.");
    *count = batch->runner.launches();
    return true;
}
