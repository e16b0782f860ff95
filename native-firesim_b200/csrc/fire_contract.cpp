// fire_contract.cpp -- the scene/emitter contract of native-firesim's worker.
//
// Before every frame the reference's worker copies its scene's emitter
// parameters into FireSettings (applySceneEmitterParams, src/main.cpp:433-447).
// It loads them once per scene (loadSceneEmitterParams, src/main.cpp:1397-1476)
// from assets/fire-scenes/<id>/scene.json and, for the mesh scenes 1 and 2,
// from emitter-mask.json beside it.  fireCudaApplySceneContract does the same
// for a headless caller.
//
// The reference reads those files with a small scanner, not a JSON parser: a
// key is found at its FIRST occurrence anywhere in the text (nested objects
// included), a number is strtof() after the next ':', an array or object is
// the bracket-balanced span after the key, and an array's numbers are every
// strtof() match in that span (src/main.cpp:1148-1264).  The contracts in the
// reference's assets depend on these rules (the gas burner's
// "heightBandMeters" is first found in "emitterHint", not in
// "derivedEmitter"), so they are kept here, in this file's own code.
#include <algorithm>
#include <array>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/fire_ext.h"

namespace firesim {
void setLastErrorMessage(const char* msg);
}  // namespace firesim

namespace {

// SceneEmitterParams and its defaults (src/main.cpp:173-183).
struct EmitterContract {
    float centerX = 0.0f;
    float centerZ = 0.0f;
    float heightNorm = 0.0f;
    float heightBandNorm = 0.06f;
    float radius = 0.48f;
    int burnerCount = 0;
    float burnerX[4] = {};
    float burnerY[4] = {};
    float burnerZ[4] = {};
};

std::string readFile(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return {};
    std::ostringstream ss;
    ss << in.rdbuf();
    return ss.str();
}

size_t keyPosition(const std::string& text, const char* key) { return text.find(std::string("\"") + key + "\""); }

bool numberAt(const std::string& text, const char* key, float& out) {
    const size_t at = keyPosition(text, key);
    if (at == std::string::npos) return false;
    const size_t colon = text.find(':', at + std::char_traits<char>::length(key) + 2);
    if (colon == std::string::npos) return false;
    const char* begin = text.c_str() + colon + 1;
    char* end = nullptr;
    const float v = std::strtof(begin, &end);
    if (end == begin) return false;
    out = v;
    return true;
}

// Bracket-balanced span that opens at the first `open` after the key.
std::string spanAt(const std::string& text, const char* key, char open, char close, bool skipStrings) {
    const size_t at = keyPosition(text, key);
    if (at == std::string::npos) return {};
    const size_t start = text.find(open, at);
    if (start == std::string::npos) return {};
    int depth = 0;
    bool inString = false, escaped = false;
    for (size_t i = start; i < text.size(); ++i) {
        const char c = text[i];
        if (skipStrings) {
            if (escaped) {
                escaped = false;
                continue;
            }
            if (c == '\\') {
                escaped = inString;
                continue;
            }
            if (c == '"') {
                inString = !inString;
                continue;
            }
            if (inString) continue;
        }
        if (c == open) {
            ++depth;
        } else if (c == close && --depth == 0) {
            return text.substr(start, i - start + 1);
        }
    }
    return {};
}

std::vector<float> numbersIn(const std::string& span) {
    std::vector<float> values;
    const char* p = span.c_str();
    while (*p != '\0') {
        char* end = nullptr;
        const float v = std::strtof(p, &end);
        if (end != p) {
            values.push_back(v);
            p = end;
        } else {
            ++p;
        }
    }
    return values;
}

std::array<float, 3> tripletAt(const std::string& text, const char* key, std::array<float, 3> fallback) {
    const std::vector<float> v = numbersIn(spanAt(text, key, '[', ']', false));
    return v.size() >= 3 ? std::array<float, 3>{v[0], v[1], v[2]} : fallback;
}

const char* assetIdOf(int scene) {
    switch (scene) {
        case 0: return "room";
        case 1: return "campfire";
        case 2: return "gas-burner-aver1";
        default: return "";
    }
}

// src/main.cpp:1397-1476.
EmitterContract loadContract(int scene, const std::string& fireScenesDir) {
    EmitterContract c;
    const std::string asset = assetIdOf(scene);
    const std::string dir = (fireScenesDir.empty() || asset.empty()) ? std::string() : fireScenesDir + "/" + asset;
    const std::string sceneText = dir.empty() ? std::string() : readFile(dir + "/scene.json");
    if (!sceneText.empty()) {
        const std::string emitterObject = spanAt(sceneText, "emitter", '{', '}', true);
        const std::string& src = emitterObject.empty() ? sceneText : emitterObject;
        const std::array<float, 3> center = tripletAt(src, "centerMeters", {0.0f, 0.02f, 0.0f});
        c.centerX = center[0];
        c.centerZ = center[2];
        c.heightNorm = (center[1] - 0.02f) / 2.03f;
        float v = 0.0f;
        if (numberAt(src, "radiusMeters", v)) c.radius = v;
        if (numberAt(src, "heightBandMeters", v)) c.heightBandNorm = v / 2.03f;
    } else if (scene == 1) {
        c.radius = 0.32f;
        c.heightNorm = (0.045f - 0.02f) / 2.03f;
        c.heightBandNorm = 0.20f / 2.03f;
    } else if (scene == 2) {
        c.radius = 0.24f;
        c.heightNorm = (0.138f - 0.02f) / 2.03f;
        c.heightBandNorm = 0.105f / 2.03f;
    }
    if (asset.empty() || scene == 0 || dir.empty()) return c;
    const std::string mask = readFile(dir + "/emitter-mask.json");
    if (mask.empty()) return c;
    const std::array<float, 3> shift = tripletAt(sceneText, "translationMeters", {0.0f, scene == 2 ? -0.24f : 0.0f, 0.0f});
    float v = 0.0f;
    if (numberAt(mask, "centerXMeters", v)) c.centerX = v;
    if (numberAt(mask, "centerZMeters", v)) c.centerZ = v;
    if (numberAt(mask, "centerYMeters", v)) {
        c.heightNorm = (v - 0.02f) / 2.03f;
    } else if (numberAt(mask, "worldHeightMeters", v)) {
        c.heightNorm = (v - 0.02f) / 2.03f;
    }
    if (numberAt(mask, "heightBandMeters", v)) c.heightBandNorm = v / 2.03f;
    if (numberAt(mask, "radiusMeters", v)) {
        c.radius = v;
    } else if (numberAt(mask, "radiusFraction", v)) {
        float width = 0.0f, depth = 0.0f;
        if (numberAt(mask, "width", width) && numberAt(mask, "depth", depth)) c.radius = v * std::max(width, depth);
    }
    const std::vector<float> burners = numbersIn(spanAt(mask, "burnerCentersMeters", '[', ']', false));
    c.burnerCount = static_cast<int>(std::min<size_t>(4, burners.size() / 3));
    for (int i = 0; i < c.burnerCount; ++i) {
        c.burnerX[i] = burners[3 * i + 0] + shift[0];
        c.burnerY[i] = burners[3 * i + 1] + shift[1];
        c.burnerZ[i] = burners[3 * i + 2] + shift[2];
    }
    if (scene == 2 && c.burnerCount > 0) c.heightNorm = (c.burnerY[0] - 0.02f) / 2.03f;
    return c;
}

}  // namespace

extern "C" bool fireCudaApplySceneContract(int sceneId, const char* fireScenesDir, FireSettings* settings) {
    if (settings == nullptr) {
        firesim::setLastErrorMessage("fireCudaApplySceneContract: settings pointer was null.");
        return false;
    }
    // applySceneEmitterParams (src/main.cpp:433-447) clamps the scene id.
    const int scene = std::max(0, std::min(2, sceneId));
    const EmitterContract c = loadContract(scene, fireScenesDir ? std::string(fireScenesDir) : std::string());
    settings->emitterCenterX = c.centerX;
    settings->emitterCenterZ = c.centerZ;
    settings->emitterHeightNorm = c.heightNorm;
    settings->emitterHeightBandNorm = c.heightBandNorm;
    settings->emitterRadius = c.radius;
    settings->burnerCenterCount = c.burnerCount;
    for (int i = 0; i < 4; ++i) {
        settings->burnerCenterX[i] = c.burnerX[i];
        settings->burnerCenterY[i] = c.burnerY[i];
        settings->burnerCenterZ[i] = c.burnerZ[i];
    }
    return true;
}
