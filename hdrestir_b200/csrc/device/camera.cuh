// GenerateCameraRay (scene/camera_ray.cpp:10-76): pinhole or thin-lens ray
// through inverse view/projection matrices in double precision, like the
// reference's GfMatrix4d::Transform, then narrowed to float.
#pragma once

#include "gf.cuh"
#include "rng.cuh"
#include "spectrum.cuh"

namespace hdr {

struct CameraParamsD {  // scene/camera_params.h:8-20
    int has_params;
    int enable_dof;
    int enable_exposure;
    float focal_length, f_stop, focus_distance;
    int bokeh_blades;
    float lens_distortion, iso, shutter_speed;
    float exposure_mult;  // GetExposureMultiplier, evaluated on the host
};

struct CameraD {
    double inv_view[16];
    double inv_proj[16];
    int width, height;
    CameraParamsD p;
    // non-null in a pass recorded into a CUDA graph: the frame index lives in device
    // memory there, so one recorded frame replays for any frame index
    const int *frame_slot;
};

// The frame index a kernel renders: its argument, or the value stored in the
// frame slot when the launch belongs to a recorded graph.
__device__ __forceinline__ int live_frame(const CameraD &c, int frame_arg) {
    return c.frame_slot ? *c.frame_slot : frame_arg;
}

struct RayF {
    V3 o, d;
};

__device__ __forceinline__ RayF camera_ray(const CameraD &c, float px, float py, MtStream &rng) {
    float ndc_x = (2.0f * px / (float)c.width) - 1.0f;
    float ndc_y = (2.0f * py / (float)c.height) - 1.0f;
    if (c.p.has_params && c.p.lens_distortion != 0.0f) {
        const float r2 = ndc_x * ndc_x + ndc_y * ndc_y;
        const float f = 1.0f + c.p.lens_distortion * r2;
        ndc_x *= f;
        ndc_y *= f;
    }
    const V3 origin = d3_to_f(m4d_transform(c.inv_view, D3{0.0, 0.0, 0.0}));
    const V3 near_cam = d3_to_f(m4d_transform(c.inv_proj, D3{(double)ndc_x, (double)ndc_y, -1.0}));
    if (!(c.p.has_params && c.p.enable_dof)) {
        const V3 near_world = d3_to_f(m4d_transform(c.inv_view, f3_to_d(near_cam)));
        return RayF{origin, normalized(near_world - origin)};
    }
    const float aperture = (c.p.focal_length / 10.0f) / (2.0f * c.p.f_stop);
    float lens_u, lens_v;
    const double kTwoPi = 2.0 * 3.14159265358979323846;  // 2.0f * M_PI in double
    if (c.p.bokeh_blades < 3) {
        const float r = sqrtf(rng.next_float());
        const float theta = (float)(kTwoPi * (double)rng.next_float());
        lens_u = r * HDR_COSF(theta);
        lens_v = r * HDR_SINF(theta);
    } else {
        const float theta = (float)(kTwoPi * (double)rng.next_float());
        const float r = sqrtf(rng.next_float());
        const float sector_angle = (float)(kTwoPi / (double)(float)c.p.bokeh_blades);
        const float sector = floorf(theta / sector_angle);
        const float angle_in_sector = theta - sector * sector_angle;
        const float dd = HDR_COSF(sector_angle / 2.0f) / HDR_COSF(sector_angle / 2.0f - angle_in_sector);
        lens_u = r * dd * HDR_COSF(theta);
        lens_v = r * dd * HDR_SINF(theta);
    }
    lens_u *= aperture;
    lens_v *= aperture;
    const V3 lens_cam{lens_u, lens_v, 0.0f};
    const V3 focal_cam = near_cam * c.p.focus_distance;
    const V3 lens_world = d3_to_f(m4d_transform(c.inv_view, f3_to_d(lens_cam)));
    const V3 focal_world = d3_to_f(m4d_transform(c.inv_view, f3_to_d(focal_cam)));
    return RayF{lens_world, normalized(focal_world - lens_world)};
}

}  // namespace hdr
