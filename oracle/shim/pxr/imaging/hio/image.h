// Stand-in for HioImage (oracle build of the reference sources; test
// infrastructure). Images are float RGB buffers registered in memory by the
// harness under a path; OpenForReading returns them, unknown paths give null.
#pragma once
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "pxr/pxr.h"

PXR_NAMESPACE_OPEN_SCOPE

// The formats ImageTextureSamplerFactory distinguishes; registered images are Float32Vec3.
enum HioFormat {
    HioFormatInvalid = -1,
    HioFormatUNorm8, HioFormatUNorm8Vec2, HioFormatUNorm8Vec3, HioFormatUNorm8Vec4,
    HioFormatUNorm8srgb, HioFormatUNorm8Vec2srgb, HioFormatUNorm8Vec3srgb, HioFormatUNorm8Vec4srgb,
    HioFormatFloat16, HioFormatFloat16Vec2, HioFormatFloat16Vec3, HioFormatFloat16Vec4,
    HioFormatFloat32, HioFormatFloat32Vec2, HioFormatFloat32Vec3, HioFormatFloat32Vec4,
};

inline int HioGetComponentCount(HioFormat f) {
    switch (f) {
    case HioFormatUNorm8: case HioFormatUNorm8srgb: case HioFormatFloat16: case HioFormatFloat32: return 1;
    case HioFormatUNorm8Vec2: case HioFormatUNorm8Vec2srgb: case HioFormatFloat16Vec2: case HioFormatFloat32Vec2:
        return 2;
    case HioFormatUNorm8Vec3: case HioFormatUNorm8Vec3srgb: case HioFormatFloat16Vec3: case HioFormatFloat32Vec3:
        return 3;
    case HioFormatUNorm8Vec4: case HioFormatUNorm8Vec4srgb: case HioFormatFloat16Vec4: case HioFormatFloat32Vec4:
        return 4;
    default: return 0;
    }
}

class HioImage;
using HioImageSharedPtr = std::shared_ptr<HioImage>;

class HioImage {
  public:
    struct StorageSpec {
        int width = 0, height = 0, depth = 1;
        HioFormat format = HioFormatInvalid;
        bool flipped = false;
        void *data = nullptr;
    };
    static std::map<std::string, std::pair<int, int>> &Sizes() {
        static std::map<std::string, std::pair<int, int>> m;
        return m;
    }
    static std::map<std::string, std::vector<float>> &Pixels() {
        static std::map<std::string, std::vector<float>> m;
        return m;
    }
    static void Register(const std::string &path, int w, int h, const float *rgb) {
        Sizes()[path] = {w, h};
        Pixels()[path].assign(rgb, rgb + (size_t)w * h * 3);
    }
    static HioImageSharedPtr OpenForReading(const std::string &path) {
        auto it = Sizes().find(path);
        if (it == Sizes().end()) return nullptr;
        auto img = std::make_shared<HioImage>();
        img->_path = path;
        img->_w = it->second.first;
        img->_h = it->second.second;
        return img;
    }
    int GetWidth() const { return _w; }
    int GetHeight() const { return _h; }
    HioFormat GetFormat() const { return HioFormatFloat32Vec3; }
    bool Read(const StorageSpec &spec) {
        const auto &px = Pixels()[_path];
        std::memcpy(spec.data, px.data(), px.size() * sizeof(float));
        return true;
    }

  private:
    std::string _path;
    int _w = 0, _h = 0;
};

PXR_NAMESPACE_CLOSE_SCOPE
