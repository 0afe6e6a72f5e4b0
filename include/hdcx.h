/*
 * hdcx.h - C ABI of the B200 (sm_100a) spectral path-tracing backend for hdCodex.
 *
 * This is the drop-in boundary. Every entry point takes plain pointers, sizes and
 * POD structs; no C++ or torch types cross it. The C++ class
 * hdcodex::CudaPathTracer (include/hdcx/cuda_path_tracer.h) is a thin shim over
 * these calls with the same methods as the reference's hdcodex::VulkanPathTracer
 * (include/hdcodex/gpu/vulkan_path_tracer.h:26-52).
 *
 * Scene input mirrors the reference's scene ABI (include/hdcodex/core/
 * versioned_scene.h:17-274): meshes with face-corner UVs/normals and per-triangle
 * material ids, the compiled MaterialX closure fields of SceneMaterial, RGBA8 or
 * RGBA32F textures with UDIM tiles, and UsdLux-derived lights. Field names follow
 * the reference, in snake_case; defaults are given by hdcx_material_defaults() etc.
 *
 * Every function returns an hdcx_status. On a nonzero status the tracer's
 * hdcx_last_error() holds a one-line message (the reference throws
 * std::runtime_error on any Vulkan failure, vulkan_path_tracer.cpp:1894-1903).
 */
#ifndef HDCX_H
#define HDCX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define HDCX_API __declspec(dllexport)
#else
#define HDCX_API __attribute__((visibility("default")))
#endif

#define HDCX_ABI_VERSION 1u

/* Hard limits of the reference integrator (vulkan_path_tracer.cpp:22-29). */
#define HDCX_MAX_TEXTURES 256u
#define HDCX_MISSING_TEXTURE 0xffffffffu
#define HDCX_UDIM_TEXTURE_FLAG 0x80000000u
#define HDCX_UDIM_TILE_MASK 0x7fffffu
#define HDCX_MAX_PATH_BOUNCES 12u
#define HDCX_MAX_LIGHTS 64u

typedef enum hdcx_status {
    HDCX_OK = 0,
    HDCX_ERROR_INVALID_ARGUMENT = 1,
    HDCX_ERROR_CUDA = 2,
    HDCX_ERROR_OUT_OF_MEMORY = 3,
    HDCX_ERROR_NO_DEVICE = 4,
    HDCX_ERROR_UNSUPPORTED = 5,
    HDCX_ERROR_TIMEOUT = 6,
    HDCX_ERROR_INTERNAL = 7
} hdcx_status;

/* ShadingMode (include/hdcodex/core/shading_mode.h:9-13). Fused and Modular
 * select the same CUDA kernels; RasterPreview is rejected as the reference's
 * CreatePipeline rejects it (vulkan_path_tracer.cpp:2495-2498). */
typedef enum hdcx_shading_mode {
    HDCX_SHADING_FUSED = 0,
    HDCX_SHADING_MODULAR = 1,
    HDCX_SHADING_RASTER_PREVIEW = 2
} hdcx_shading_mode;

/* PathTracerCamera (vulkan_path_tracer.h:16-23). Row 0 of the image is the
 * lowerLeft edge; a pixel (x, y) looks along
 * lowerLeft + u*horizontal + v*vertical - origin. */
typedef struct hdcx_camera {
    float origin[3];
    float lower_left[3];
    float horizontal[3];
    float vertical[3];
} hdcx_camera;

/* SceneMesh (versioned_scene.h:17-34). Counts are element counts of the arrays. */
typedef struct hdcx_mesh_desc {
    const char* id;
    const float* positions;          /* 3 floats per vertex */
    uint64_t position_count;
    const uint32_t* indices;         /* 3 per triangle */
    uint64_t index_count;
    const float* texcoords;          /* 2 floats per triangulated face corner */
    uint64_t texcoord_count;
    const float* normals;            /* 3 floats per face corner; zero = geometric */
    uint64_t normal_count;
    const char* material_id;         /* NULL or "" = display-color fallback */
    const char* const* triangle_material_ids; /* optional, one per triangle */
    uint64_t triangle_material_id_count;
    float display_color[3];
} hdcx_mesh_desc;

/* Diffuse models of SceneMaterial::DiffuseModel (versioned_scene.h:37-42). */
#define HDCX_DIFFUSE_LAMBERT 0u
#define HDCX_DIFFUSE_OREN_NAYAR 1u
#define HDCX_DIFFUSE_BURLEY 2u
#define HDCX_DIFFUSE_OREN_NAYAR_ENERGY_COMPENSATED 3u

/* The compact path-closure fields of SceneMaterial (versioned_scene.h:117-188),
 * in the reference's declaration order. The MaterialX raster/SPIR-V members of
 * SceneMaterial are never read by the integrator and are not part of this ABI. */
typedef struct hdcx_material_desc {
    const char* id;
    float base_color[3];
    float base_color_texture_scale[3];
    float base_color_texture_bias[3];
    int32_t base_color_texture_channel;
    float emission[3];
    float transmission_color[3];
    float transmission_scatter[3];
    float specular_color[3];
    float coat_color[3];
    float sheen_color[3];
    float translucent_color[3];
    float subsurface_color[3];
    float subsurface_radius[3];
    uint32_t diffuse_model;
    float diffuse_weight;
    float diffuse_roughness;
    float metalness;
    float roughness;
    float roughness_v;
    float opacity;
    float emission_weight;
    float transmission;
    float transmission_depth;
    float transmission_scatter_anisotropy;
    float transmission_dispersion_scale;
    float transmission_dispersion_abbe_number;
    float index_of_refraction;
    float specular_weight;
    float coat;
    float coat_roughness;
    float coat_roughness_v;
    float coat_index_of_refraction;
    float sheen;
    float sheen_roughness;
    uint32_t sheen_mode;             /* 0 Conty-Kulla, 1 Zeltner */
    float translucent_weight;
    float subsurface;
    float subsurface_scale;
    float subsurface_scatter_anisotropy;
    int32_t thin_walled;
    int32_t normal_texture_flip_y;
    float normal_texture_scale;
    const char* base_color_texture;
    const char* metalness_texture;
    const char* roughness_texture;
    const char* diffuse_weight_texture;
    const char* diffuse_roughness_texture;
    const char* emission_texture;
    const char* opacity_texture;
    const char* normal_texture;
    const char* transmission_texture;
    const char* specular_texture;
    const char* specular_color_texture;
    const char* coat_texture;
    const char* coat_color_texture;
    const char* coat_roughness_texture;
    const char* sheen_texture;
    const char* sheen_color_texture;
    const char* sheen_roughness_texture;
    const char* translucent_weight_texture;
    const char* translucent_color_texture;
    const char* subsurface_texture;
    const char* subsurface_color_texture;
    const char* subsurface_radius_texture;
} hdcx_material_desc;

/* SceneTexture (versioned_scene.h:191-206): RGBA8 (optionally sRGB) or RGBA32F. */
typedef struct hdcx_texture_desc {
    const char* id;
    const char* udim_set_id;         /* non-empty for a UDIM tile */
    uint32_t udim_tile;
    uint32_t width;
    uint32_t height;
    int32_t srgb;
    const uint8_t* rgba;             /* width*height*4 bytes, or NULL */
    uint64_t rgba_count;
    const float* rgba_float;         /* width*height*4 floats, or NULL */
    uint64_t rgba_float_count;
} hdcx_texture_desc;

/* SceneLightType / DomeTextureFormat (versioned_scene.h:208-223). */
#define HDCX_LIGHT_DOME 0u
#define HDCX_LIGHT_RECT 1u
#define HDCX_LIGHT_DISK 2u
#define HDCX_LIGHT_SPHERE 3u
#define HDCX_LIGHT_CYLINDER 4u
#define HDCX_LIGHT_DISTANT 5u
#define HDCX_DOME_AUTOMATIC 0u
#define HDCX_DOME_LATLONG 1u
#define HDCX_DOME_MIRRORED_BALL 2u
#define HDCX_DOME_ANGULAR 3u
#define HDCX_DOME_CUBEMAP_VERTICAL_CROSS 4u

/* SceneLight (versioned_scene.h:225-266), in declaration order. */
typedef struct hdcx_light_desc {
    const char* id;
    uint32_t type;
    int32_t visible;
    float color[3];
    float temperature_color[3];
    float intensity;
    float exposure;
    float diffuse;
    float specular;
    int32_t normalize;
    const char* texture;
    uint32_t texture_format;
    float basis_x[3];
    float basis_y[3];
    float basis_z[3];
    float position[3];
    float axis_u[3];
    float axis_v[3];
    float width;
    float height;
    float radius;
    float length;
    float angle;
    float area;
    float shaping_focus;
    float shaping_focus_tint[3];
    float shaping_cone_angle;
    float shaping_cone_softness;
    int32_t shadow_enable;
    float shadow_color[3];
    float shadow_distance;
    float shadow_falloff;
    float shadow_falloff_gamma;
} hdcx_light_desc;

/* SceneSnapshot (versioned_scene.h:268-274). Arrays are taken in the given
 * order, exactly as SetScene takes a published snapshot (whose containers the
 * reference's VersionedScene fills in id order, versioned_scene.h:297-326). */
typedef struct hdcx_scene_desc {
    uint64_t revision;
    const hdcx_mesh_desc* meshes;
    uint64_t mesh_count;
    const hdcx_material_desc* materials;
    uint64_t material_count;
    const hdcx_texture_desc* textures;
    uint64_t texture_count;
    const hdcx_light_desc* lights;
    uint64_t light_count;
} hdcx_scene_desc;

/* An instancer: mesh `mesh_index` of the scene, given in object space, drawn
 * once per transform. No counterpart in the reference's scene ABI: its Hydra
 * mesh adapter flattens an instanced mesh into world-space copies before the
 * tracer sees it (mesh.cpp:955-1004). hdcx_set_scene_instanced renders the
 * scene exactly as hdcx_set_scene renders that flattened scene (same
 * triangles, ids, images), with one bottom-level BVH per instanced mesh under
 * a top-level BVH of instances instead of one BVH over every copy.
 * Transforms are affine 4x4 matrices, 16 doubles each, row-major in the
 * row-vector convention of the reference's Gf matrices (world = [p 1] M; the
 * translation in elements 12..14; column 3 must be (0, 0, 0, 1)). The
 * flattening, per instance in order and then per valid triangle: positions
 * ((x*m00 + y*m10) + z*m20) + m30 (likewise y, z) in binary64 rounded to
 * float; corner normals n' = n inverse(A) (A the upper 3x3, inverse by
 * cofactors / determinant) normalised in binary64 (divided by max(length,
 * 1e-10), zero when length <= 1e-12) and rounded; texcoords and per-triangle
 * materials copied. */
typedef struct hdcx_instancer_desc {
    uint64_t mesh_index;
    const double* transforms;
    uint64_t instance_count;
} hdcx_instancer_desc;

/* Device records, byte-identical to the reference's GpuMaterial (23 x 16 B,
 * vulkan_path_tracer.cpp:1907-1933) and GpuLight (14 x 16 B, :1935-1952). */
#define HDCX_GPU_MATERIAL_BYTES 368u
#define HDCX_GPU_LIGHT_BYTES 224u

/* Texel formats of a packed texture (the reference's VkFormat choice,
 * vulkan_path_tracer.cpp:2218-2221). */
#define HDCX_TEXEL_RGBA8_UNORM 0u
#define HDCX_TEXEL_RGBA8_SRGB 1u
#define HDCX_TEXEL_RGBA32F 2u

typedef struct hdcx_packed_texture {
    uint32_t width;
    uint32_t height;
    uint32_t format;                 /* HDCX_TEXEL_* */
    uint32_t reserved;
    const void* texels;              /* width*height*4 bytes or floats */
} hdcx_packed_texture;

/* The flattened scene in the integrator's device layout (the reference's
 * BuildScene output, vulkan_path_tracer.cpp:2604-2993). */
typedef struct hdcx_packed_scene {
    uint32_t vertex_count;
    uint32_t triangle_count;
    uint32_t material_count;
    uint32_t light_count;            /* authored lights (<= 64); buffer holds max(1, n) */
    uint32_t texture_count;
    uint32_t opaque;                 /* all materials opaque (vulkan_path_tracer.cpp:2609-2612) */
    const float* vertices;           /* 4 floats per vertex (xyz, w = 1) */
    const uint32_t* indices;         /* 3 per triangle */
    const uint32_t* triangle_materials;
    const float* texcoords;          /* 6 floats per triangle (face corners) */
    const float* normals;            /* 12 floats per triangle (corner xyz0) */
    const void* materials;           /* material_count * 368 B */
    const void* lights;              /* max(1, light_count) * 224 B */
    const float* emissive;           /* 4 floats per triangle: cdf, prob/area, area, 0 */
    const hdcx_packed_texture* textures;
} hdcx_packed_scene;

typedef struct hdcx_tracer hdcx_tracer;
typedef struct hdcx_packing hdcx_packing;

/* Per-render counters, filled by hdcx_get_stats after a render. */
typedef struct hdcx_render_stats {
    uint64_t spectral_paths;         /* pixels * spp * 3 */
    uint64_t extension_rays;         /* closest-hit rays (camera + bounces) */
    uint64_t shadow_rays;            /* any-hit visibility rays */
    uint64_t subsurface_rays;        /* opaque boundary rays of the SSS walk */
    double render_ms;                /* device time of the last render call */
    double extend_ms;                /* device time in closest-hit traversal */
    double shade_ms;                 /* device time in shading */
    double shadow_ms;                /* device time in shadow traversal */
    uint32_t waves;                  /* path waves the render was split into */
    uint32_t extend_launches;        /* closest-hit traversal launches */
    uint64_t kernel_launches;        /* kernels the render launched */
    uint64_t extension_node_visits;  /* wide nodes loaded by closest-hit rays (counting mode) */
    uint64_t extension_triangle_tests; /* triangle tests of closest-hit rays (counting mode) */
    uint64_t shadow_node_visits;     /* wide nodes loaded by shadow rays (counting mode) */
    uint64_t shadow_triangle_tests;  /* triangle tests of shadow rays (counting mode) */
} hdcx_render_stats;

/* One job of hdcx_render_batch: the arguments of one hdcx_render call and
 * the job's results. */
typedef struct hdcx_batch_job {
    hdcx_tracer* tracer;     /* the job renders this tracer's scene */
    hdcx_camera camera;
    uint32_t width;
    uint32_t height;
    uint32_t sample_index;
    uint32_t max_bounces;
    uint32_t sample_count;
    float* rgba_out;         /* width*height*4 floats (host or device), or NULL */
    int32_t written;         /* out: as hdcx_render's *written */
    hdcx_status status;      /* out: this job's status (hdcx_last_error(tracer) has the message) */
    double render_ms;        /* out: device time of the job on its tracer's stream */
} hdcx_batch_job;

/* Launch tuning of a tracer (hdcx_autotune, hdcx_set_tuning): paths per wave
 * and blocks of 128 threads per SM of the traversal and shade kernels. Images
 * do not depend on these values. */
typedef struct hdcx_tuning {
    uint64_t wave_paths;           /* 0 = automatic (up to 12,582,912) */
    uint32_t trace_blocks_per_sm;  /* default 16 */
    uint32_t shade_blocks_per_sm;  /* default 8 */
    double milliseconds;           /* hdcx_autotune: device time of the best configuration */
    double default_milliseconds;   /* hdcx_autotune: device time of the defaults */
    uint32_t candidates;           /* hdcx_autotune: configurations timed (0: taken from the cache) */
    uint32_t sort_hits;            /* 1: hits are shaded in material order (a counting sort per bounce); default 0 */
    uint32_t sort_rays;            /* 1: secondary rays are traced in direction order (a sort within chunks of
                                      1024 queue entries per bounce); default 0 */
} hdcx_tuning;

/* Profiling switches for hdcx_set_profiling. */
#define HDCX_PROFILE_STAGE_TIMES 1u      /* CUDA events around every extend/shade/shadow launch */
#define HDCX_PROFILE_COUNT_TRAVERSAL 2u  /* traversal kernels count node visits and triangle tests */

/* ---------------------------------------------------------------------------
 * Library and device probing
 * ------------------------------------------------------------------------- */

/* Returns HDCX_ABI_VERSION. */
HDCX_API uint32_t hdcx_abi_version(void);

/* Byte size of each ABI struct, indexed 0..7: camera, mesh, material, texture,
 * light, scene, packed_texture, packed_scene; 8: render_stats; 9: batch_job;
 * 10: nrc_config; 11: tuning.
 * Lets bindings check their struct mirrors. Returns the number of entries. */
HDCX_API uint32_t hdcx_abi_struct_sizes(uint64_t* sizes, uint32_t capacity);

/* Fills the reference defaults of SceneMaterial / SceneLight / SceneMesh
 * (versioned_scene.h:121-188, :225-266, :33). String members are set to NULL. */
HDCX_API void hdcx_material_defaults(hdcx_material_desc* material);
HDCX_API void hdcx_light_defaults(hdcx_light_desc* light);
HDCX_API void hdcx_mesh_defaults(hdcx_mesh_desc* mesh);

/* Replaces HdCodexRendererPlugin::IsSupported / ProbeVulkanDevices
 * (renderer_plugin.cpp:34-60, vulkan_context.h:10-60): *supported = 1 when a
 * CUDA device of compute capability 10.x is present. */
HDCX_API hdcx_status hdcx_probe_devices(int32_t* supported, int32_t* device_count);

/* Budget of the device memory the library may hold on `device`, in bytes (0:
 * no budget, the default). No counterpart in the reference, whose Vulkan
 * allocations are bounded only by the device. Every allocation of the
 * library (path arenas, scene and BVH buffers, the BVH build's temporaries,
 * radiance caches; not hdcx_render_static's static array) counts against it;
 * one that would exceed it fails like an exhausted device: the call returns
 * HDCX_ERROR_OUT_OF_MEMORY with a message, launches nothing for that call,
 * and the tracer stays usable. Allocations already made are kept when the
 * budget is lowered. Device ordinals 0..63. */
HDCX_API hdcx_status hdcx_set_device_memory_limit(int32_t device, uint64_t bytes);
/* Bytes the library holds on `device`, and its budget (0: none). */
HDCX_API hdcx_status hdcx_get_device_memory_usage(int32_t device, uint64_t* in_use, uint64_t* limit);

/* ---------------------------------------------------------------------------
 * Tracer lifetime (VulkanPathTracer constructor/destructor,
 * vulkan_path_tracer.cpp:3348-3350; render_delegate.cpp:113-132 constructs it)
 * ------------------------------------------------------------------------- */
HDCX_API hdcx_status hdcx_create(int32_t device, hdcx_tracer** tracer);
HDCX_API void hdcx_destroy(hdcx_tracer* tracer);

/* Message of the last failed call on this tracer ("" when none). */
HDCX_API const char* hdcx_last_error(const hdcx_tracer* tracer);

/* ---------------------------------------------------------------------------
 * Scene (VulkanPathTracer::SetScene, vulkan_path_tracer.cpp:3351-3354 ->
 * Impl::BuildScene :2604-3128)
 * ------------------------------------------------------------------------- */

/* Flattens, packs and uploads a snapshot and builds the BVH on the GPU.
 * scene == NULL clears the scene (HasGeometry becomes false). Synchronous. */
HDCX_API hdcx_status hdcx_set_scene(hdcx_tracer* tracer, const hdcx_scene_desc* scene);

/* Uploads an already packed scene (a caller that packs on its own side). */
HDCX_API hdcx_status hdcx_set_scene_packed(hdcx_tracer* tracer, const hdcx_packed_scene* scene);

/* hdcx_set_scene with instancers (hdcx_instancer_desc): the meshes they name
 * are given in object space and drawn once per transform. Same triangles,
 * flattened ids and images as hdcx_set_scene of the flattened scene; the
 * acceleration structure is two-level: one 8-wide BVH per instanced mesh
 * (object space) and one over the other triangles (world space), under a
 * top-level BVH of instances. Invalid or singular transforms give
 * HDCX_ERROR_INVALID_ARGUMENT. */
HDCX_API hdcx_status hdcx_set_scene_instanced(hdcx_tracer* tracer, const hdcx_scene_desc* scene,
                                              const hdcx_instancer_desc* instancers, uint64_t instancer_count);

/* Moves the object-space points of instancer `instancer` (its index in the
 * last hdcx_set_scene_instanced call; position_count = 3 x its point count)
 * for a deforming mesh: the flattened world vertices of all its instances and
 * the emissive-triangle CDF are recomputed, its bottom-level BVH is refitted
 * (same topology, boxes and quantisation recomputed level by level from the
 * leaves up) and the top-level BVH is rebuilt. Corner normals, texcoords and
 * materials are kept. Renders afterwards equal those of the flattened scene
 * with the moved points. */
HDCX_API hdcx_status hdcx_update_instancer_points(hdcx_tracer* tracer, uint64_t instancer, const float* positions,
                                                  uint64_t position_count);

/* Texture level of detail (not in the reference, whose sampler reads one
 * mip level, vulkan_path_tracer.cpp:2401-2423; README.md lists texture LOD as
 * future work). mode 0 (default): every lookup at level 0, the reference's
 * sampling. mode 1: the library builds a mip pyramid of every texture on the
 * GPU (2x2 means in linear RGBA32F, odd sizes reusing their last row or
 * column) and material textures are filtered trilinearly at the level ray
 * cones give (Akenine-Moller et al. 2019): a cone starts with the spread of a
 * camera pixel and follows smooth reflections and refractions; after any
 * other bounce lookups return to level 0. Light and dome textures and normal
 * maps stay at level 0. Images then differ from the reference's: less
 * texture aliasing and noise at low sample counts, slightly blurred
 * textures. Scenes set later get pyramids while the mode is on. */
HDCX_API hdcx_status hdcx_set_texture_lod(hdcx_tracer* tracer, uint32_t mode);
/* Copies mip level `level` (>= 1) of packed texture `texture` (RGBA32F,
 * width*height*4 floats; host or device memory; NULL only reports the size). */
HDCX_API hdcx_status hdcx_read_texture_level(hdcx_tracer* tracer, uint32_t texture, uint32_t level, float* rgba_out,
                                             uint64_t float_count, uint32_t* width, uint32_t* height);

/* Size and build cost of the current scene. */
typedef struct hdcx_scene_info {
    uint64_t triangles;      /* flattened triangles */
    uint64_t instances;      /* top-level leaves (0: a single-level scene) */
    uint64_t bottom_levels;  /* bottom-level BVHs */
    uint64_t bvh_bytes;      /* nodes and leaf triangle copies of every BVH */
    uint64_t scene_bytes;    /* every device buffer of the scene, BVHs included */
    double build_ms;         /* host wall time of the last set_scene: packing, upload, BVH builds */
    double bvh_build_ms;     /* of which the BVH builds */
} hdcx_scene_info;
HDCX_API hdcx_status hdcx_get_scene_info(const hdcx_tracer* tracer, hdcx_scene_info* info);

/* Packs a snapshot on the host without a device; the view stays valid until
 * hdcx_packing_destroy. Used to check the packing against the reference rules. */
HDCX_API hdcx_status hdcx_pack_scene(const hdcx_scene_desc* scene, hdcx_packing** packing);
/* hdcx_pack_scene with instancers: the packing of the flattened scene. */
HDCX_API hdcx_status hdcx_pack_scene_instanced(const hdcx_scene_desc* scene, const hdcx_instancer_desc* instancers,
                                               uint64_t instancer_count, hdcx_packing** packing);
HDCX_API const hdcx_packed_scene* hdcx_packing_view(const hdcx_packing* packing);
HDCX_API void hdcx_packing_destroy(hdcx_packing* packing);

/* VulkanPathTracer::HasGeometry (vulkan_path_tracer.cpp:3371). */
HDCX_API int32_t hdcx_has_geometry(const hdcx_tracer* tracer);

/* SetShadingMode / GetShadingMode (vulkan_path_tracer.cpp:3355-3362).
 * RasterPreview returns HDCX_ERROR_UNSUPPORTED and keeps the current mode. */
HDCX_API hdcx_status hdcx_set_shading_mode(hdcx_tracer* tracer, int32_t mode);
HDCX_API int32_t hdcx_get_shading_mode(const hdcx_tracer* tracer);

/* ---------------------------------------------------------------------------
 * Rendering (VulkanPathTracer::Render, vulkan_path_tracer.cpp:3363-3370 ->
 * Impl::Trace :3230-3306)
 * ------------------------------------------------------------------------- */

/* Traces sample_count samples per pixel starting at sample_index and updates
 * the device running mean exactly like the reference's accumulation
 * (vulkan_path_tracer.cpp:1886-1890): pixel = (prev*sample_index + batch) /
 * (sample_index + sample_count), alpha = 1. sample_index == 0 restarts.
 * max_bounces is clamped to [1, 12]. When rgba_out is not NULL the whole
 * RGBA32F image (width*height*4 floats, row 0 = bottom) is copied into it.
 * With no geometry or a zero size nothing is traced and *written = 0
 * (the reference returns an empty vector, :3235); otherwise *written = 1.
 * Device memory: the path state of a wave (about 359 bytes per path) lives in
 * a per-device pool of arenas, not in the tracer: a call checks out a free
 * arena (at most eight per device; when all are busy it waits for one) and
 * grows it to its wave, and the arenas are freed with the device's last
 * tracer. Tracers that render one after another therefore share one arena.
 * Automatic waves take at most three quarters of the free device memory plus
 * what the arena holds. A tracer in radiance-cache mode keeps path state of
 * its own. */
HDCX_API hdcx_status hdcx_render(hdcx_tracer* tracer, const hdcx_camera* camera,
                                 uint32_t width, uint32_t height,
                                 uint32_t sample_index, uint32_t max_bounces,
                                 uint32_t sample_count, float* rgba_out,
                                 int32_t* written);

/* The interactive preview of HdCodexRenderPass::_Execute (render_pass.cpp:
 * 191-208) on the device: renders at half resolution (ceil(width/2) x
 * ceil(height/2)) from sample 0 with two bounces and one sample per pixel,
 * exactly as hdcx_render would (the running mean restarts at that size), then
 * upscales the image to width x height by nearest neighbour on the GPU, with
 * the reference's UpscaleNearest rule (render_pass.cpp:45-68: source pixel =
 * min(size - 1, destination * size / destination size)), where the reference
 * upscales on the CPU. When rgba_out is not NULL the upscaled RGBA32F image
 * (width*height*4 floats; host or device memory) is copied into it; it also
 * stays on the device (hdcx_device_preview). *written as hdcx_render. */
HDCX_API hdcx_status hdcx_render_preview(hdcx_tracer* tracer, const hdcx_camera* camera,
                                         uint32_t width, uint32_t height, float* rgba_out,
                                         int32_t* written);
/* Device pointer of the last upscaled preview (valid until the next preview
 * of a larger size, or destroy). */
HDCX_API hdcx_status hdcx_device_preview(hdcx_tracer* tracer, const float** device_rgba);

/* hdcx_render without waiting: where the reference blocks on a fence and then
 * copies the whole image (vulkan_path_tracer.cpp:3287-3305), this enqueues the
 * render and the read-back of its running mean and returns a ticket at once.
 * The render runs on the tracer's stream; the image is copied to device
 * staging there, and from it to a pinned host buffer of the tracer on a
 * second stream, so the copy of frame n overlaps the rendering of frame n+1.
 * Two frames may be in flight: a call whose slot still holds the frame two
 * tickets back completes that frame first (and gives up its image). Frames
 * complete in ticket order. Same images, counters and running-mean rules as
 * hdcx_render; hdcx_render, hdcx_render_preview, hdcx_render_static,
 * hdcx_render_batch, hdcx_read_aovs and hdcx_set_scene complete pending frames
 * first. A frame with no geometry or a zero size writes nothing. */
HDCX_API hdcx_status hdcx_render_async(hdcx_tracer* tracer, const hdcx_camera* camera,
                                       uint32_t width, uint32_t height,
                                       uint32_t sample_index, uint32_t max_bounces,
                                       uint32_t sample_count, uint64_t* ticket);
/* Waits for the frame `ticket` (and every earlier pending frame) and gives
 * its image: *host_rgba points at width*height*4 floats in pinned host memory
 * owned by the tracer, valid until the hdcx_render_async call two tickets
 * later (or destroy); *written = 0 and *host_rgba = NULL for a frame that
 * wrote nothing. hdcx_get_stats then describes the frame. A ticket no longer
 * held gives HDCX_ERROR_INVALID_ARGUMENT. */
HDCX_API hdcx_status hdcx_wait_render(hdcx_tracer* tracer, uint64_t ticket, const float** host_rgba,
                                      int32_t* written);

/* Device AOVs written by every render (hdcx_render, _async, _batch,
 * _preview's half-resolution render) once enabled: per pixel of the render,
 * the flattened primitive index of the closest accepted primary hit
 * (0xffffffff: miss) and its distance along the normalised camera ray (0 on a
 * miss), for the render's first sample sample_index: the hdcx_trace_primary
 * result for that sample, without a separate call. No counterpart in the
 * reference, whose render buffer holds colour only (render_buffer.cpp:114-129).
 * Either flag enables both; 0 disables them. */
#define HDCX_AOV_PRIMITIVE_ID 1u
#define HDCX_AOV_DEPTH 2u
HDCX_API hdcx_status hdcx_set_aovs(hdcx_tracer* tracer, uint32_t flags);
/* Copies the last render's AOVs (pixel_count >= width*height; host or device
 * destinations; either may be NULL). */
HDCX_API hdcx_status hdcx_read_aovs(hdcx_tracer* tracer, uint32_t* primitive_out, float* depth_out,
                                    uint64_t pixel_count);

/* hdcx_render for callers that cannot allocate device memory. No counterpart
 * in the reference: VulkanPathTracer has no entry point of this kind.
 *
 * Who needs it: a plugin running inside a host application that reserves the
 * GPU's memory for itself and gives plugins no allocator, and interactive
 * loops that cannot afford the device-wide synchronisation cudaFree (and often
 * cudaMalloc) implies. hdcx_render allocates path state and per-pixel sums on
 * its first call and whenever the image size grows; this entry point calls no
 * allocator (no cudaMalloc, no cudaFree, no allocating library routine).
 *
 * Same integrator and results as hdcx_render, except where the image lives:
 * the running mean is the caller's device buffer `rgba_device`
 * (width*height*4 floats, 16-byte aligned), read when sample_index > 0 and
 * written on every call, in place of the tracer's own accumulation buffer
 * (which this call neither reads nor writes; hdcx_read_rgba, hdcx_read_xyz and
 * hdcx_get_stats are not updated). The caller's earlier work on rgba_device
 * must have finished before the call; the call returns once the image is
 * written.
 *
 * The scratch (the path state of one wave of 65,536 paths and the per-pixel
 * sums of one frame) is one static device array of 62,063,104 bytes inside
 * the library, which every GPU that loads the library keeps until the process
 * exits. Images above 1,048,576 pixels (width*height) are rejected with
 * HDCX_ERROR_INVALID_ARGUMENT and a message, and so is a tracer with a
 * radiance cache attached (this entry point has no cache mode, whose training
 * buffers it would have to allocate). The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture. All calls on a
 * device share the array, which keeps the last call's contents, so calls whose
 * GPU work overlapped would race: the library holds a per-device lock for the
 * whole call, GPU work included. With no geometry or a zero size nothing is
 * traced and *written = 0; otherwise *written = 1. */
HDCX_API hdcx_status hdcx_render_static(hdcx_tracer* tracer, const hdcx_camera* camera,
                                        uint32_t width, uint32_t height,
                                        uint32_t sample_index, uint32_t max_bounces,
                                        uint32_t sample_count, float* rgba_device,
                                        int32_t* written);

/* Renders several jobs, each exactly as hdcx_render would (same images, same
 * running means, same counters), with their kernels overlapping on the GPU:
 * every job runs on its own tracer's stream, all jobs are launched before any
 * is waited for. No counterpart in the reference, whose caller renders one
 * delegate at a time; it replaces a serial loop of Render calls over many
 * scenes (a farm of small shots, turntables, look-development variants).
 * Each tracer appears in at most one job (HDCX_ERROR_INVALID_ARGUMENT
 * otherwise). Tracers may live on different devices. Per-stage times are not
 * recorded for batched jobs. Path state: the jobs of a device are dealt,
 * largest first, to up to four lanes that run concurrently, one path arena
 * (see hdcx_render) per lane; the jobs of a lane run one after another on its
 * arena. A lane holds waves of its largest job's paths, at most 50,331,648
 * paths and at most an equal share of `path_budget` paths of path state per
 * device (0: half of the device's free memory at the call), never below
 * 1,048,576 paths; a wave size set with hdcx_set_wave_size bounds its own
 * job's waves. A batch takes the arenas that are free and waits only while it
 * holds none. Jobs in radiance-cache mode render on their own tracers' path
 * state. Returns HDCX_OK when every job
 * succeeded, else the first failing job's status; each job's own status is in
 * its `status`. */
HDCX_API hdcx_status hdcx_render_batch(hdcx_batch_job* jobs, uint32_t count, uint64_t path_budget);

/* hdcx_render_batch with options. HDCX_BATCH_CUDA_GRAPH: the kernels of all
 * jobs (each on its tracer's stream) are captured into one CUDA graph and
 * launched at once. The device keeps the executable graph between calls: a
 * batch with the same launch topology as the last one (same jobs, sizes and
 * wave counts) updates it in place (cudaGraphExecUpdate) instead of
 * instantiating a new one. Every job's render_ms is then its own device time
 * from its first to its last kernel inside the graph (jobs overlap, so these
 * do not add up to the batch's time). A batch that cannot be captured (jobs
 * on several devices, a job in radiance-cache mode) runs as hdcx_render_batch
 * does. Same images either way. */
#define HDCX_BATCH_CUDA_GRAPH 1u
HDCX_API hdcx_status hdcx_render_batch_ex(hdcx_batch_job* jobs, uint32_t count, uint64_t path_budget, uint32_t flags);
/* Batch graphs of `device` so far: instantiated anew, and updated in place. */
HDCX_API hdcx_status hdcx_get_batch_graph_stats(int32_t device, uint64_t* instantiations, uint64_t* updates);

/* Copies the current device RGBA32F accumulation (width*height*4 floats). */
HDCX_API hdcx_status hdcx_read_rgba(hdcx_tracer* tracer, float* rgba_out, uint64_t float_count);

/* Copies the FP64 per-pixel CIE XYZ sums (width*height*3 doubles) and the
 * number of samples they hold. The mean XYZ is sum / samples. For every sample
 * the three lanes add (cie(lambda) * 400/106.856895 * radiance) / 3, the XYZ
 * the reference's sensor (vulkan_path_tracer.cpp:172-179) feeds its sRGB matrix. */
HDCX_API hdcx_status hdcx_read_xyz(hdcx_tracer* tracer, double* xyz_out,
                                   uint64_t double_count, uint64_t* samples);

/* Device pointer of the RGBA32F accumulation buffer (valid until the next
 * render with another size, set_scene or destroy). */
HDCX_API hdcx_status hdcx_device_rgba(hdcx_tracer* tracer, const float** device_rgba);

/* Primary-ray hit test for sample `sample_number`: writes for every pixel the
 * flattened primitive index of the closest accepted hit (0xffffffff = miss)
 * and its distance. All three wavelength lanes of a sample share the camera
 * ray (same seed and jitter, vulkan_path_tracer.cpp:1202-1213). */
HDCX_API hdcx_status hdcx_trace_primary(hdcx_tracer* tracer, const hdcx_camera* camera,
                                        uint32_t width, uint32_t height,
                                        uint32_t sample_number, uint32_t* primitive_out,
                                        float* distance_out);

/* Counters of the last render. */
HDCX_API hdcx_status hdcx_get_stats(const hdcx_tracer* tracer, hdcx_render_stats* stats);

/* Turns profiling on or off (HDCX_PROFILE_* bits); results are unchanged. */
HDCX_API hdcx_status hdcx_set_profiling(hdcx_tracer* tracer, uint32_t flags);

/* Number of paths resident per wave (0 = automatic). Larger waves use more
 * device memory for path state; results do not depend on it. */
HDCX_API hdcx_status hdcx_set_wave_size(hdcx_tracer* tracer, uint64_t paths_per_wave);

/* Current tuning of the tracer (milliseconds fields 0). */
HDCX_API hdcx_status hdcx_get_tuning(const hdcx_tracer* tracer, hdcx_tuning* tuning);
HDCX_API hdcx_status hdcx_set_tuning(hdcx_tracer* tracer, const hdcx_tuning* tuning);
/* Autotuner (no counterpart in the reference): times renders of this camera,
 * size, bounce budget and sample count over wave sizes and traversal/shade
 * grid sizes and the hit sort, one knob at a time from the defaults, keeps the fastest on the
 * tracer and returns it. Wave sizes of 1M to 48M paths are tried, the larger
 * ones while their path state (about 359 bytes per path) fits half of the free
 * device memory; a path arena grown for a candidate larger than the one kept
 * is released before it returns. Results are cached per device and workload shape
 * (triangles, pixels, samples, bounces, shading variant) for the process, so
 * a repeated call times nothing. The tuning renders overwrite the tracer's
 * accumulation: render with sample_index 0 afterwards. */
HDCX_API hdcx_status hdcx_autotune(hdcx_tracer* tracer, const hdcx_camera* camera, uint32_t width, uint32_t height,
                                   uint32_t max_bounces, uint32_t sample_count, hdcx_tuning* result);

/* ---------------------------------------------------------------------------
 * Neural radiance cache (no counterpart in the reference; the learned part of
 * the B200 build): a multiresolution hash-grid encoding of position (16
 * levels x 2 FP16 features, 2^log2_table_size entries per level) plus
 * direction, shading normal, roughness and wavelength, feeding a 64-wide MLP
 * with four ReLU hidden layers whose forward and backward passes run as BF16
 * tcgen05 tensor-core GEMMs with FP32 accumulation; FP32 Adam on the relative
 * L2 loss. A query record is HDCX_NRC_QUERY_FLOATS floats: position (3,
 * normalised to [0, 1]), direction (3), shading normal (3), roughness,
 * (wavelength - 380) / 400, 0. Query, target and output pointers of the
 * query/train/gradient calls are device memory.
 * ------------------------------------------------------------------------- */
#define HDCX_NRC_QUERY_FLOATS 12u
#define HDCX_NRC_WEIGHT_COUNT 17408u /* 4 x 64 x 64 + 16 x 64 FP32 weights, row-major [out][in] per layer */
#define HDCX_NRC_LEVELS 16u

typedef struct hdcx_nrc hdcx_nrc;

typedef struct hdcx_nrc_config {
    uint32_t log2_table_size;   /* entries per level = 2^n (default 19) */
    uint32_t base_resolution;   /* cells per axis of the coarsest level (default 16) */
    uint32_t finest_resolution; /* cells per axis of the finest level (default 2048) */
    float learning_rate;        /* Adam step size (default 1e-2) */
    float beta1;                /* default 0.9 */
    float beta2;                /* default 0.99 */
    float epsilon;              /* default 1e-8 */
    uint32_t seed;              /* initialisation seed */
} hdcx_nrc_config;

HDCX_API void hdcx_nrc_defaults(hdcx_nrc_config* config);
HDCX_API hdcx_status hdcx_nrc_create(int32_t device, const hdcx_nrc_config* config, hdcx_nrc** out);
HDCX_API void hdcx_nrc_destroy(hdcx_nrc* cache);
HDCX_API const char* hdcx_nrc_last_error(const hdcx_nrc* cache);
/* FP32 parameters of the hash table: levels x 2^log2_table_size x 2. */
HDCX_API uint64_t hdcx_nrc_grid_parameter_count(const hdcx_nrc* cache);
/* Cells per axis of each of the HDCX_NRC_LEVELS levels. */
HDCX_API hdcx_status hdcx_nrc_resolutions(const hdcx_nrc* cache, uint32_t* resolutions);
/* radiance[i] = the cache's prediction for query record i. */
HDCX_API hdcx_status hdcx_nrc_query(hdcx_nrc* cache, const float* queries, uint32_t count, float* radiance);
/* `steps` Adam steps on the batch; *mean_loss (host, optional) = the last
 * step's mean relative L2 loss. */
HDCX_API hdcx_status hdcx_nrc_train(hdcx_nrc* cache, const float* queries, const float* targets, uint32_t count,
                                    uint32_t steps, float* mean_loss);
/* Gradients of the mean loss of the batch, without an update, into host
 * arrays of HDCX_NRC_WEIGHT_COUNT and hdcx_nrc_grid_parameter_count floats
 * (either may be NULL). */
HDCX_API hdcx_status hdcx_nrc_gradients(hdcx_nrc* cache, const float* queries, const float* targets, uint32_t count,
                                        float* mlp_gradient, float* grid_gradient);
/* Failure-path check: runs the cache kernels' bounded tensor-core wait on an
 * mbarrier that nothing arrives at, for at most `polls` polls. The wait runs
 * out, the kernel records it and returns, and the call returns
 * HDCX_ERROR_TIMEOUT with a message; the device context stays usable. */
HDCX_API hdcx_status hdcx_nrc_check_wait_timeout(hdcx_nrc* cache, uint32_t polls);
/* Host copies of the FP32 parameters (either may be NULL). Setting them
 * resets the Adam state. */
HDCX_API hdcx_status hdcx_nrc_get_parameters(hdcx_nrc* cache, float* mlp, float* grid);
HDCX_API hdcx_status hdcx_nrc_set_parameters(hdcx_nrc* cache, const float* mlp, const float* grid);

/* Renders of `tracer` use the radiance cache (NULL: the plain integrator).
 * Paths stop at the first surface vertex after `prefix_bounces` bounces and
 * add throughput x the cache's prediction there; about `training_paths`
 * paths per wave (a deterministic subset by path identity) run the full
 * bounce budget, and the radiance each gathered after every vertex trains the
 * cache (`train_steps` Adam steps per wave) before the next wave. The cache
 * must live on the tracer's device; it is not owned by the tracer. Renders in
 * this mode synchronise with the host once per wave. */
HDCX_API hdcx_status hdcx_set_radiance_cache(hdcx_tracer* tracer, hdcx_nrc* cache, uint32_t prefix_bounces,
                                             uint32_t training_paths, uint32_t train_steps);
/* Path termination by spread (Mueller et al., "Real-time Neural Radiance
 * Caching for Path Tracing", 2021, sec. 3.4): with factor c > 0 a
 * cache-mode path also ends, and queries the cache, at the first vertex
 * where its spread a(x1..xn) = (sum_i sqrt(|x(i-1) - xi|^2 / (p(wi)
 * |cos(theta_i)|)))^2 exceeds c times the primary footprint |x0 - x1|^2 /
 * (4 pi |cos(theta_1)|); specular bounces add nothing, so specular chains
 * continue to a rough vertex. prefix_bounces stays the latest bounce. The
 * paper's c is 0.01; 0 (the default) ends paths by the prefix alone. No
 * counterpart in the reference (it has no radiance cache). */
HDCX_API hdcx_status hdcx_set_radiance_cache_spread(hdcx_tracer* tracer, float factor);
/* Totals since the cache was attached: queries answered, training samples
 * used, and the mean loss of the last training step. */
HDCX_API hdcx_status hdcx_get_radiance_cache_stats(const hdcx_tracer* tracer, uint64_t* queries, uint64_t* samples,
                                                   float* last_loss);

/* ---------------------------------------------------------------------------
 * Test support (failure detection). No counterpart in the reference.
 * ------------------------------------------------------------------------- */

/* Makes the tracer's BVH cyclic for a test of traversal-fault reporting: the
 * root node's internal children are redirected to the root itself and the
 * seven nodes after it (all in bounds, so nothing is read outside the node
 * array). Rays that enter the redirected child then revisit nodes until
 * their node budget or their stack runs out, which the traversal records;
 * the next hdcx_render returns HDCX_ERROR_INTERNAL ("traversal fault") and
 * the tracer stays usable. hdcx_set_scene rebuilds a valid BVH. Requires a
 * BVH of at least 8 nodes (else HDCX_ERROR_INVALID_ARGUMENT). */
HDCX_API hdcx_status hdcx_test_break_bvh(hdcx_tracer* tracer);

#ifdef __cplusplus
}
#endif

#endif /* HDCX_H */
