// fire_guard.cu -- deviceAlloc / deviceFree and the guard-zone checker of the
// FIRE_BOUNDS_CHECK build (the contract is in fire_guard.h).
#include "fire_guard.h"

#include <climits>
#include <cstdio>
#include <map>
#include <mutex>
#include <vector>

namespace firesim {

#ifndef FIRE_BOUNDS_CHECK

cudaError_t deviceAlloc(void** p, size_t bytes, const char* /*label*/) { return cudaMalloc(p, bytes); }

void deviceFree(void* p) {
    if (p != nullptr) cudaFree(p);
}

bool checkGuards(int& corrupted, std::string& report) {
    corrupted = -1;
    report = "bounds checks are compiled only into the FIRE_BOUNDS_CHECK build (libfiresim_b200_checked.so)";
    return true;
}

bool plantGuardByte(const char* /*label*/, size_t /*offset*/, std::string& err) {
    err = "plantGuardByte: bounds checks are compiled only into the FIRE_BOUNDS_CHECK build";
    return false;
}

#else

namespace {

struct Guarded {
    char* base = nullptr;  // the allocation: guard, payload, guard
    size_t bytes = 0;      // the payload
    int device = 0;
    std::string label;
};

std::mutex g_mutex;
std::map<void*, Guarded> g_live;     // keyed by the payload address
std::vector<std::string> g_freedBad;  // changed zones found when their buffer was freed

constexpr unsigned long long kClean = ULLONG_MAX;

// Lowest byte offset at or after `skip` in `zone` whose value is not 0xFF,
// or kClean.
__global__ void guardScan(const uint4* __restrict__ zone, size_t words, unsigned skip, unsigned long long* firstChanged) {
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < words; i += stride) {
        const uint4 v = zone[i];
        if ((v.x & v.y & v.z & v.w) == 0xFFFFFFFFu) continue;
        const unsigned part[4] = {v.x, v.y, v.z, v.w};
        for (int k = 0; k < 16; ++k) {
            const unsigned long long offset = static_cast<unsigned long long>(i) * 16ull + k;
            if (offset >= skip && ((part[k >> 2] >> (8 * (k & 3))) & 0xFFu) != 0xFFu) {
                atomicMin(firstChanged, offset);
                break;
            }
        }
    }
}

// Scans both zones of each buffer (on the current device); for each changed
// zone appends a description to `bad` and re-arms the zone.
cudaError_t scan(const std::vector<Guarded>& bufs, std::vector<std::string>& bad) {
    if (bufs.empty()) return cudaSuccess;
    unsigned long long* d = nullptr;
    const size_t zones = 2 * bufs.size();
    cudaError_t e = cudaMalloc(&d, zones * sizeof(unsigned long long));
    if (e != cudaSuccess) return e;
    e = cudaMemset(d, 0xFF, zones * sizeof(unsigned long long));
    for (size_t i = 0; i < bufs.size() && e == cudaSuccess; ++i) {
        const char* zone[2] = {bufs[i].base, bufs[i].base + kGuardBytes + bufs[i].bytes};
        for (int side = 0; side < 2; ++side) {
            // The payload's size need not be a multiple of 16: the after-zone is
            // scanned in 16-byte words from the boundary below its start, and the
            // kernel skips the leading bytes, which belong to the payload.
            const size_t lead = reinterpret_cast<size_t>(zone[side]) & 15;
            const uint4* start = reinterpret_cast<const uint4*>(zone[side] - lead);
            guardScan<<<64, 256>>>(start, kGuardBytes / 16, static_cast<unsigned>(lead), d + 2 * i + side);
        }
        e = cudaGetLastError();
    }
    std::vector<unsigned long long> first(zones, kClean);
    if (e == cudaSuccess) e = cudaMemcpy(first.data(), d, zones * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return e;
    for (size_t i = 0; i < bufs.size(); ++i) {
        for (int side = 0; side < 2; ++side) {
            if (first[2 * i + side] == kClean) continue;
            const char* zone = side == 0 ? bufs[i].base : bufs[i].base + kGuardBytes + bufs[i].bytes;
            const size_t lead = reinterpret_cast<size_t>(zone) & 15;
            char line[320];
            const long long offset = static_cast<long long>(first[2 * i + side]) - static_cast<long long>(lead);
            if (side == 0) {
                std::snprintf(line, sizeof(line), "'%s' (%zu bytes): write before its start, the farthest changed byte %lld bytes before it",
                              bufs[i].label.c_str(), bufs[i].bytes, static_cast<long long>(kGuardBytes) - offset);
            } else {
                std::snprintf(line, sizeof(line), "'%s' (%zu bytes): write past its end, first changed byte at end + %lld",
                              bufs[i].label.c_str(), bufs[i].bytes, offset < 0 ? 0ll : offset);
            }
            bad.push_back(line);
            e = cudaMemset(const_cast<char*>(zone), 0xFF, kGuardBytes);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

}  // namespace

cudaError_t deviceAlloc(void** p, size_t bytes, const char* label) {
    *p = nullptr;
    char* base = nullptr;
    const size_t total = bytes + 2 * kGuardBytes;
    cudaError_t e = cudaMalloc(&base, total);
    if (e != cudaSuccess) return e;
    // The fill runs on the legacy default stream; wait for it, so that work on
    // the library's non-blocking streams cannot start before it ends.
    e = cudaMemset(base, 0xFF, total);
    if (e == cudaSuccess) e = cudaStreamSynchronize(nullptr);
    if (e != cudaSuccess) {
        cudaFree(base);
        return e;
    }
    int device = 0;
    cudaGetDevice(&device);
    *p = base + kGuardBytes;
    std::lock_guard<std::mutex> lock(g_mutex);
    g_live[*p] = Guarded{base, bytes, device, label != nullptr ? label : "device buffer"};
    return cudaSuccess;
}

void deviceFree(void* p) {
    if (p == nullptr) return;
    Guarded g;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        auto it = g_live.find(p);
        if (it == g_live.end()) {
            cudaFree(p);
            return;
        }
        g = it->second;
        g_live.erase(it);
    }
    int device = 0;
    cudaGetDevice(&device);
    std::vector<std::string> bad;
    if (device == g.device && cudaDeviceSynchronize() == cudaSuccess && scan({g}, bad) == cudaSuccess && !bad.empty()) {
        std::lock_guard<std::mutex> lock(g_mutex);
        for (std::string& b : bad) g_freedBad.push_back("freed " + b);
    }
    cudaFree(g.base);
}

bool checkGuards(int& corrupted, std::string& report) {
    corrupted = 0;
    report.clear();
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        report = std::string("checkGuards: ") + cudaGetErrorString(e);
        return false;
    }
    std::vector<Guarded> bufs;
    std::vector<std::string> bad;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        for (const auto& kv : g_live) {
            if (kv.second.device == device) bufs.push_back(kv.second);
        }
        bad.swap(g_freedBad);
    }
    e = scan(bufs, bad);
    if (e != cudaSuccess) {
        report = std::string("checkGuards: ") + cudaGetErrorString(e);
        return false;
    }
    corrupted = static_cast<int>(bad.size());
    if (!bad.empty()) report = "bounds check: " + bad.front() + (bad.size() > 1 ? " (and " + std::to_string(bad.size() - 1) + " more)" : "");
    return true;
}

bool plantGuardByte(const char* label, size_t offset, std::string& err) {
    if (label == nullptr || offset >= kGuardBytes) {
        err = "plantGuardByte: a label and an offset below the guard size are required";
        return false;
    }
    char* at = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        for (const auto& kv : g_live) {
            if (kv.second.label == label) {
                at = kv.second.base + kGuardBytes + kv.second.bytes + offset;
                break;
            }
        }
    }
    if (at == nullptr) {
        err = std::string("plantGuardByte: no live buffer labelled '") + label + "'";
        return false;
    }
    cudaError_t e = cudaMemset(at, 0, 1);
    if (e == cudaSuccess) e = cudaStreamSynchronize(nullptr);
    if (e != cudaSuccess) {
        err = std::string("plantGuardByte: ") + cudaGetErrorString(e);
        return false;
    }
    return true;
}

#endif

}  // namespace firesim
