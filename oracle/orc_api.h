/*
 * CPU oracle entry points — TEST INFRASTRUCTURE (see orc_core.h).
 * Called through ctypes by tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg only.
 */
#ifndef HDR_ORACLE_API_H
#define HDR_ORACLE_API_H

#include "orc_core.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_TRACE 64

typedef struct {
    int max_depth, enable_subsurface, max_refl, max_refr, render_ibl_background;
    float roulette;
} orc_path_params;

typedef struct {
    int candidate_count, use_reservoir, skip_visibility, m_cap;
} orc_ris_params;

typedef struct {
    int ris; /* 0: PathTracePass (MIS), 1: RISPathTracePass */
    orc_path_params path;
    orc_ris_params ris_params;
} orc_frame_params;

/* WeightedReservoir<RISLightCandidate> of one pixel (reservoir.h:69-161) */
typedef struct {
    int has_sample, has_lc, light, origin, vis_tested, pdf_solid, m;
    float dir[3], color[3], normal[3];
    float dist, pdf, target, wsum, w;
    float tp[4];
} orc_reservoir;

/* per-pixel record of the primary RIS call, for bit-exact parity checks */
typedef struct {
    int n_candidates;
    int n_nee_idx;
    int nee_light[ORC_MAX_TRACE]; /* light index of each NEE candidate, -1 = none */
    int ris_choice;               /* standard-RIS winner index, -1 = none */
    int draws;
    float L[4];
    float lambda[4];
} orc_pixel_trace;

void orc_camera_ray(const hdr_camera *cam, const double *inv_view, const double *inv_proj, float px, float py,
                    orc_rng *r, float *out6);
void orc_raycast(const orc_scene *s, const hdr_camera *cam, int frame, hdr_gbuffer_texel *gbuf, int threads);
void orc_integrate(const orc_scene *s, const hdr_camera *cam, int frame, const orc_frame_params *fp,
                   hdr_gbuffer_texel *gbuf, float *color, orc_reservoir *res, orc_pixel_trace *trace, int threads);
/* the same passes restricted to image rows [y0, y1) (bounded CPU-baseline samples) */
void orc_raycast_band(const orc_scene *s, const hdr_camera *cam, int frame, hdr_gbuffer_texel *gbuf, int y0,
                      int y1, int threads);
void orc_integrate_band(const orc_scene *s, const hdr_camera *cam, int frame, const orc_frame_params *fp,
                        hdr_gbuffer_texel *gbuf, float *color, orc_reservoir *res, orc_pixel_trace *trace, int y0,
                        int y1, int threads);
void orc_accumulate(float *color, float *accum, int width, int height, int frame, int firefly);
void orc_accumulate_shader(float *color, float *accum, int width, int height, int frame, int firefly);
void orc_rng_floats(const uint32_t *seeds, int n, int count, float *out);
float orc_reservoir_known_answer(float weight, float phat, int candidates_per_frame);
void orc_trace_rays(const orc_scene *s, const float *rays, const float *tmax, int n, int any_hit,
                    hdr_gbuffer_texel *out);
int orc_scene_sky(const orc_scene *s, const float *dirs, int n, float *out, float *sun);

#ifdef __cplusplus
}
#endif
#endif
