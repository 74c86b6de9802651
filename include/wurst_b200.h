/*
 * wurst_b200.h -- C ABI of the B200-native `nextevent_path_tracer`.
 *
 * Drop-in boundary for the reference's NEE+MIS integrator
 * (jamornsriwasansak/wurstrenderer). The reference exposes the path as a
 * Renderer plugin selected by name from a simple2 scene JSON and writes PFM
 * images; this header is the plain-C surface underneath that boundary, with
 * no C++ or torch types: plain pointers, sizes and status codes.
 *
 * Conventions: every function returns WR_OK (0) or a nonzero status and never
 * throws across the ABI; wr_last_error() describes the last failure on the
 * calling thread. Output buffers are owned by the caller. Each scene handle
 * owns one CUDA stream on the current device; a handle is not re-entrant (one
 * call at a time per handle), different handles may be used concurrently.
 * Images are W*H*3 doubles, row 0 = top, x fastest, RGB -- the layout of the
 * reference's Film / Fimage (src/common/film.h, src/common/floatimage.h).
 */
#ifndef WURST_B200_H
#define WURST_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define WR_ABI_VERSION 1

/* status codes */
#define WR_OK 0
#define WR_ERR_INVALID_ARGUMENT 1
#define WR_ERR_IO 2
#define WR_ERR_PARSE 3
#define WR_ERR_UNSUPPORTED 4
#define WR_ERR_CUDA 5
#define WR_ERR_OUT_OF_MEMORY 6
#define WR_ERR_TIMEOUT 7

typedef struct wr_scene wr_scene;

typedef struct wr_render_desc {
    int num_spp;             /* samples per pixel; <= 0 takes "num_spp" of the render entry (default 16) */
    int num_path_vertices;   /* <= 0 takes "num_path_vertices" of the render entry (default 10) */
    unsigned int seed;       /* selects the random streams; 0 is a valid seed */
    int render_index;        /* which "render" entry supplies the defaults */
    int queue_capacity;      /* wavefront slots; 0 = default (tuned) */
    int grid_trace;          /* persistent blocks of the traversal kernels; 0 = occupancy-derived */
    int grid_shade;          /* persistent blocks of shade / raygen; 0 = occupancy-derived */
    int use_graph;           /* 1: the whole render is one CUDA-graph launch (while-loop node over the
                                bounce iterations); 0: host-driven launches */
    int profile;             /* 0: off; 1: per-kernel CUDA-event timing (plain launches, extend and
                                shadow rays in separate kernels); 2: timing + traversal counters
                                (node visits, triangle tests); 3: as 2 with the fused schedule of
                                unprofiled renders (WR_K_EXTEND times the kernel that traces each
                                iteration's extend rays with the previous iteration's shadow rays,
                                WR_K_SHADOW the last iteration's shadow rays) */
    int trace_block;         /* threads per block of the traversal kernels: 64, 128 or 256; 0 = 128 */
    int integrator;          /* 0: the render entry's "integrator" (default nextevent_path_tracer);
                                1: nextevent_path_tracer; 2: primitive_path_tracer; 3: light_splatting */
    int guiding;             /* learned proposal (no counterpart in the reference; NEE+MIS only):
                                0: off (plain NEE+MIS);
                                1: train a fresh network online on the first guide_train_spp samples per
                                   pixel (in passes, Adam after each pass), use it for the remaining samples;
                                2: use the scene's current network as it is (no training) */
    int guide_train_spp;     /* samples per pixel of the training phase; 0 = 32 */
    int guide_pass_spp;      /* samples per pixel per training pass; 0 = about 2^22 paths per pass, at
                                least four passes */
    int guide_batch;         /* training records per Adam step; 0 = 16384 */
    int guide_steps;         /* Adam steps of the training phase, spread evenly over its passes; 0 = a
                                budget of about 18 % of the render's device time (estimated from the first
                                pass), 256 to 8192 steps */
    float guide_clamp;       /* loss weights are clamped at guide_clamp x their mean over the pass;
                                0 = 1000, < 0 = no clamp */
    int fetch_threshold;     /* traversal: a warp hands new rays to its idle lanes when fewer than this
                                many of its 32 lanes are still traversing; 1..32, 0 = 20 */
    int max_iterations;      /* debugging: lowers the wavefront's iteration bound (0 = the bound derived
                                from the work, (waves + 2) * (num_path_vertices + 2) + 64). A render
                                that has not drained when its bound is reached stops and returns
                                WR_ERR_TIMEOUT; the handle stays usable */
    float guide_lr;          /* Adam learning rate of the training phase; 0 = 1e-3 */
    int reserved[1];
} wr_render_desc;

typedef struct wr_render_stats {
    double render_ms;                 /* device time of the bounce loop + resolve */
    unsigned long long paths;         /* camera samples traced (W*H*spp) */
    unsigned long long iterations;    /* bookkeeping launches of the wavefront loop, the first
                                         wavefront's included (bounce iterations + 1) */
    unsigned int max_shadow_queue;    /* largest shadow-ray queue seen */
    unsigned int queue_capacity;      /* wavefront slots used */
    int grid_trace, grid_shade;       /* persistent blocks used */
    int trace_block;                  /* threads per traversal block used */
    unsigned long long kernel_launches;   /* kernels launched by the render */
    /* per-kernel totals, filled when desc.profile != 0 (index: WR_K_*) */
    double kernel_ms[8];
    unsigned long long kernel_count[8];   /* launches */
    unsigned long long kernel_items[8];   /* rays / paths processed */
    unsigned long long extend_node_visits, extend_tri_tests;   /* profile == 2 */
    unsigned long long shadow_node_visits, shadow_tri_tests;
    /* guided renders */
    unsigned long long guide_records;     /* training records collected */
    unsigned long long guide_steps;       /* Adam steps taken */
    double guide_train_ms;                /* device time of the training kernels */
    double guide_loss;                    /* mean loss of the last training pass */
    int guide_passes;                     /* render passes (training passes + the final one) */
    int reserved_stats;
} wr_render_stats;

#define WR_K_EXTEND 0
#define WR_K_SHADE 1
#define WR_K_RAYGEN 2
#define WR_K_SHADOW 3
#define WR_K_ADVANCE 4
#define WR_K_RESOLVE 5
#define WR_K_GUIDE 6      /* guiding-network inference over the wavefront */
#define WR_K_TRAIN 7      /* guiding-network training (gradient + Adam) */

typedef struct wr_scene_info {
    int width, height;                /* camera resolution */
    int num_spp, num_path_vertices;   /* of render entry 0 (defaults when absent) */
    unsigned long long num_triangles;
    int num_meshes, num_lights, has_envmap;
    int bvh_nodes, bvh_depth;
    double bvh_sah_cost;
    double build_ms;                  /* scene parse + BVH + upload + CDF build */
    int num_renders;
    int bvh_builder;                  /* WR_BVH_* used */
    double bvh_ms;                    /* BVH build time (device time for WR_BVH_DEVICE_LBVH) */
} wr_scene_info;

#define WR_BVH_HOST_SAH 0       /* binned SAH on the host, <= max_leaf triangles per leaf (default) */
#define WR_BVH_DEVICE_LBVH 1    /* linear BVH built on the device (Morton codes, radix sort, Karras 2012) */

#define WR_BVH_WIDTH_DEFAULT 2 /* bvh_width 0 selects this */
#define WR_MAX_LEAF_DEFAULT 2  /* max_leaf 0 selects this (binary and 8-wide trees) */
#define WR_SAH_PATCH_COST_DEFAULT 16 /* sah_patch_cost_milli 0 selects this many triangle tests */

typedef struct wr_scene_options {
    int bvh_builder;         /* WR_BVH_HOST_SAH or WR_BVH_DEVICE_LBVH */
    int max_leaf;            /* host SAH: triangles per leaf, 1..16 (0 = WR_MAX_LEAF_DEFAULT; at
                                most 3 for the 8-wide tree) */
    int bvh_width;           /* 2: binary BVH (64-byte nodes); 8: compressed 8-wide BVH (80-byte
                                nodes, 8-bit quantised child boxes, <= 3 triangles per leaf);
                                0: WR_BVH_WIDTH_DEFAULT */
    int sah_trav_cost_milli; /* host SAH: cost of one traversal step relative to one triangle
                                test, in thousandths, 1..100000 (0 = 1000) */
    int sah_patch_cost_milli;/* host SAH: cost of one Phong patch test relative to one triangle
                                test, in thousandths, 1..1000000 (0 = WR_SAH_PATCH_COST_DEFAULT) */
    int reserved[3];
} wr_scene_options;

/* Parses a simple2 scene JSON (Simple2Parser::Parse, src/sceneio/simple2parser.h:84-100),
 * loads its OBJ/MTL meshes and envmap, builds the BVH and the FP64 light /
 * environment CDFs, and uploads everything to the current CUDA device. */
int wr_scene_create(const char *scene_json_path, wr_scene **out);

/* Same with build options (opts may be NULL: defaults). */
int wr_scene_create_ex(const char *scene_json_path, const wr_scene_options *opts, wr_scene **out);

/* Same from JSON text (the --jsimple2parse path, src/main.cpp:12-15);
 * relative mesh paths resolve against base_dir (NULL: current directory). */
int wr_scene_create_from_json(const char *json_text, const char *base_dir, wr_scene **out);

void wr_scene_destroy(wr_scene *scene);

/* Host-only validation of a scene (no GPU needed): parses the JSON and its
 * meshes and builds the host SAH BVH as wr_scene_create does, fills `info`
 * (build_ms covers parse + BVH only) and uploads nothing. Phong tessellation
 * surfaces enter as their triangles (wr_scene_create bounds each patch). */
int wr_scene_inspect(const char *scene_json_path, wr_scene_info *info);

/* Same with build options (opts may be NULL: defaults; the host SAH builder only,
 * WR_ERR_UNSUPPORTED for WR_BVH_DEVICE_LBVH). */
int wr_scene_inspect_ex(const char *scene_json_path, const wr_scene_options *opts, wr_scene_info *info);

int wr_scene_get_info(const wr_scene *scene, wr_scene_info *info);

/* Replaces the camera with a simple2 "camera" JSON object
 * (ThinlensCamera::FromSimple2ParseJson, src/camera/thinlens.h:13-26). */
int wr_scene_set_camera_json(wr_scene *scene, const char *camera_json);

/* Renders with the NEE+MIS integrator ("nextevent_path_tracer",
 * PathNeeRenderer::render, src/renderer/pathnextevent.h:152-191), or, when the
 * render entry or desc->integrator selects it, with the BSDF-only
 * "primitive_path_tracer" (PrimitivePathRenderer::render,
 * src/renderer/primitivepath.h:60-101) or the light tracer "light_splatting"
 * (LightSplattingRenderer::render, src/renderer/lightsplatting.h:38-112), and
 * copies the W*H*3 image (base/spp + splat/(spp*W*H)) into host memory. desc may
 * be NULL (defaults). */
int wr_render(wr_scene *scene, const wr_render_desc *desc, double *out_rgb);

/* Same, writing the image to device memory (W*H*3 doubles on the scene's
 * device); no host copy. */
int wr_render_device(wr_scene *scene, const wr_render_desc *desc, double *out_rgb_device);

/* One render job of a batch (many cameras / resolutions / sample counts over one scene). */
typedef struct wr_job {
    const char *camera_json;   /* simple2 "camera" object of this job; NULL: the scene's camera */
    int num_spp;               /* <= 0: "num_spp" of the render entry */
    int num_path_vertices;     /* <= 0: "num_path_vertices" of the render entry */
    unsigned int seed;         /* random streams of this job (mixed with its index) */
    int reserved[3];
} wr_job;

/* Renders n jobs over the scene in one wavefront: every job is an independent
 * PathNeeRenderer::render with its own camera (src/renderer/pathnextevent.h:152-191),
 * but all their samples share the same queues, and with desc->use_graph the whole
 * bounce loop of all jobs is one CUDA-graph launch. desc supplies the wavefront
 * settings (its num_spp / num_path_vertices / seed are ignored). out_rgb receives the
 * images concatenated in job order (job j: W_j*H_j*3 doubles). */
int wr_render_batch(wr_scene *scene, const wr_job *jobs, int n, const wr_render_desc *desc, double *out_rgb);
int wr_render_batch_device(wr_scene *scene, const wr_job *jobs, int n, const wr_render_desc *desc,
                           double *out_rgb_device);

int wr_get_render_stats(const wr_scene *scene, wr_render_stats *stats);

/* No counterpart in the reference. wr_render_device without any allocation:
 * the wavefront and film scratch live in one fixed 10 MiB device array that
 * the library holds on every GPU it is loaded on, for callers that may not
 * allocate device memory while running (fixed memory budgets, or no implicit
 * synchronisation from cudaMalloc/cudaFree). Limits: films of at most 65,536
 * pixels (larger: WR_ERR_INVALID_ARGUMENT), a 32,768-path wavefront, plain
 * kernel launches (desc->queue_capacity, use_graph and profile are ignored).
 * The integrator is resolved as wr_render_device resolves it; the learned
 * proposal needs buffers of its own, so desc->guiding != 0 returns
 * WR_ERR_UNSUPPORTED. Every call clears and reuses the same array, so calls that
 * overlap on the GPU race; the first call on a device resolves the array's
 * address and should precede any stream capture. */
int wr_render_device_noalloc(wr_scene *scene, const wr_render_desc *desc, double *out_rgb_device);

/* Autotuner (no counterpart in the reference): times short renders of the
 * scene's camera at probe_spp samples per pixel over traversal block sizes
 * {64, 128, 256}, wavefront capacities {2^19 .. 2^22}, persistent-CTA counts
 * {1/2, 1} x the occupancy limit and ray-fetching thresholds {12 .. 28}
 * (coordinate descent, starting from `base`), and
 * writes the fastest settings into *best (other fields copied from base) and
 * its time per render into *best_ms. */
int wr_autotune(wr_scene *scene, const wr_render_desc *base, int probe_spp, wr_render_desc *best, double *best_ms);

/* The same search for a batch (no counterpart in the reference): each candidate is timed on
 * wr_render_batch over the n probe jobs (their cameras, spp and depths as given; a caller
 * usually passes a subset of its batch at reduced spp). */
int wr_autotune_batch(wr_scene *scene, const wr_job *jobs, int n, const wr_render_desc *base, wr_render_desc *best,
                      double *best_ms);

/* ---- Learned guiding proposal (no counterpart in the reference) ----
 * A 64-64-64-64-64-64 ReLU MLP (BF16 weights and activations, FP32 accumulation on
 * the tensor cores, FP32 master weights) maps 64 encoded inputs -- the hit position
 * normalised to the scene box, sin/cos(2^f pi p) for f = 0..5, the geometric normal
 * turned toward the outgoing direction, the outgoing direction, sin/cos(pi n),
 * sin/cos(pi wo), zeros and a constant 1 -- to 8 von Mises-Fisher lobes: axis
 * (outputs 5k..5k+2, normalised), sharpness softplus(5k+3) + 0.5, weight softmax(5k+4).
 * Unit 63 of every hidden layer is the constant 1, so column 63 is a bias.
 * Weights: WR_GUIDE_PARAMS floats, [layer][out][in]. One network per scene handle. */
#define WR_GUIDE_PARAMS 20480

/* Initialises the network with seeded uniform (Glorot) weights and clears Adam's state. */
int wr_guide_reset(wr_scene *scene, unsigned int seed);
int wr_guide_get_params(wr_scene *scene, float *params);
int wr_guide_set_params(wr_scene *scene, const float *params);
/* The position normalisation: feature = (p - lo) * inv_extent. */
int wr_guide_box(const wr_scene *scene, float lo[3], float inv_extent[3]);
/* Lobes for n rows of 9 floats (position, normal, outgoing direction), host memory:
 * 40 floats per row, 8 x (axis xyz, sharpness) then the 8 weights. */
int wr_guide_eval(wr_scene *scene, const float *rows, int n, float *lobes);
/* Gradient of sum_i -min(c_i, c_max) log q_i(direction_i) over n training records of
 * 20 floats (position, c, normal, -, outgoing, -, direction, -, throughput, -),
 * host memory, into grad (WR_GUIDE_PARAMS floats); *loss receives the summed loss
 * (may be NULL). The network is not changed. */
int wr_guide_gradient(wr_scene *scene, const float *records, int n, float c_max, float *grad, double *loss);
/* `steps` Adam steps (learning rate lr) on minibatches of `batch` records drawn in a
 * fixed shuffled order from the n records; loss_per_step (may be NULL) receives
 * each step's mean loss before its update. */
int wr_guide_train(wr_scene *scene, const float *records, int n, int steps, int batch, float lr,
                   double *loss_per_step);

/* Closest-hit queries (EmbreeAccel::intersectTriangleInfo,
 * src/accel/embreeaccel.h:425-464). rays: n x 8 floats
 * (ox, oy, oz, tnear, dx, dy, dz, tfar) in host memory. Outputs (host):
 * geom_id = Embree geomID (mesh attach order, -1 on a miss), prim_id =
 * triangle within the mesh, t = hit distance, uv = 2 floats per ray
 * (barycentric weights of vertices 1 and 2). uv may be NULL. */
int wr_trace_closest(wr_scene *scene, const float *rays, int n, int *geom_id, int *prim_id, float *t, float *uv);

/* Closest hits with the unit geometry normal at the hit (n x 3 floats): the
 * triangle's face normal, or on a Phong tessellation patch the patch normal
 * (PhongMeshGeometry::intersect, src/geometry/phongmesh.h:178-368, reported to the
 * renderer as Embree's Ng, src/accel/embreeaccel.h:101-127,419-420). Rays, ids and t
 * as wr_trace_closest. */
int wr_trace_hits(wr_scene *scene, const float *rays, int n, int *geom_id, int *prim_id, float *t, float *normal);

/* Occlusion queries (EmbreeAccel::isIntersect, src/accel/embreeaccel.h:336-351). */
int wr_trace_occluded(wr_scene *scene, const float *rays, int n, int *occluded);

/* Traversal statistics for a ray batch: totals of inner-node visits and
 * triangle tests (the counts that define the traversal kernel's algorithmic bytes). */
int wr_trace_stats(wr_scene *scene, const float *rays, int n, int any_hit, unsigned long long *node_visits,
                   unsigned long long *tri_tests);

/* PFM output in the reference's layout (FimageIo::SavePfmColor, src/common/floatimage.h:435-462). */
int wr_write_pfm(const char *path, const double *rgb, int width, int height);

/* Float image input as the scene loader reads environment maps (FimageIo::Load,
 * src/common/floatimage.h:379-404): .pfm, .hdr (Radiance RGBE) or .exr (one-part scanline
 * OpenEXR, HALF / FLOAT channels, uncompressed / RLE / ZIPS / ZIP). Writes the size; with rgb
 * non-NULL also width * height * 3 floats, row 0 = top (call once with NULL to size the buffer). */
int wr_read_image(const char *path, int *width, int *height, float *rgb);

/* Whole simple2 flow of the reference CLI (src/main.cpp:5-15,
 * src/sceneio/simple2parser.h:102-223): load the scene, render every
 * "nextevent_path_tracer" entry of "render" and write its "output" PFM next
 * to the scene JSON; "primitive_path_tracer" and "light_splatting" entries
 * likewise. Other integrators return WR_ERR_UNSUPPORTED. */
int wr_run_simple2(const char *scene_json_path);
int wr_run_jsimple2(const char *json_text);

/* Makes `device` the current CUDA device of the calling thread for this
 * library (scene handles remember the device they were created on). */
int wr_set_device(int device);

const char *wr_last_error(void);
int wr_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* WURST_B200_H */
