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

enum HioFormat { HioFormatInvalid = -1, HioFormatFloat32Vec3 = 1 };

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
