/*
 * hdcx_oracle.h - C interface of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY: a CPU restatement of hdCodex's GLSL integrator
 * (src/gpu/vulkan_path_tracer.cpp:100-1891) and scene packing (:1961-2066,
 * :2604-2993). Only the tests, the smoke check and the benchmark's CPU
 * baseline load it, as the checker; the product never does.
 *
 * An oracle_tracer mirrors VulkanPathTracer's observable state: the packed
 * scene, the RGBA32F running mean of the last render size, and the fallback
 * up axis fixed by the first render (vulkan_path_tracer.cpp:3237-3241).
 */
#ifndef HDCX_ORACLE_H
#define HDCX_ORACLE_H

#include "hdcx.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_tracer oracle_tracer;

oracle_tracer* oracle_create(void);
void oracle_destroy(oracle_tracer* tracer);
/* Packs the snapshot and builds the CPU BVH (NULL clears the scene). */
int oracle_set_scene(oracle_tracer* tracer, const hdcx_scene_desc* scene);
int oracle_has_geometry(const oracle_tracer* tracer);
/* Fills a view of the packed scene (valid until the next set_scene). */
int oracle_packed_view(const oracle_tracer* tracer, hdcx_packed_scene* view);
/* Render(camera, w, h, sampleIndex, maxBounces, sampleCount) over the pixel
 * rectangle [x0, x1) x [y0, y1) (x1 = y1 = 0 means the whole image) with
 * `threads` worker threads (0 = all cores). rgba_out (w*h*4) receives the
 * running mean (pixels outside the rectangle keep their previous value);
 * xyz_out (w*h*3, optional) receives the FP64 XYZ sums. counters (optional)
 * receives extension, shadow and subsurface ray counts. Returns 1 if it
 * rendered, 0 when there was no geometry or a zero size. */
int oracle_render(oracle_tracer* tracer, const hdcx_camera* camera, uint32_t width,
                  uint32_t height, uint32_t sample_index, uint32_t max_bounces,
                  uint32_t sample_count, uint32_t x0, uint32_t y0, uint32_t x1,
                  uint32_t y1, int32_t threads, float* rgba_out, double* xyz_out,
                  uint64_t* counters);
/* Closest confirmed hit of every camera ray of sample `sample_number`
 * (0xffffffff = miss) and its distance. */
int oracle_trace_primary(oracle_tracer* tracer, const hdcx_camera* camera, uint32_t width,
                         uint32_t height, uint32_t sample_number, int32_t threads,
                         uint32_t* primitive_out, float* distance_out);

#ifdef __cplusplus
}
#endif

#endif
