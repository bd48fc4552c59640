/* nrt.h -- C ABI of the B200 NURBS ray-intersection engine (libnrt.so).
 *
 * The engine keeps the pipeline of Frostbite16/rt-nurbs as a drop-in:
 *   knot-insertion Bezier decomposition  -> nrt_decompose / nrt_scene_create
 *   SAH BVH over patch bounding boxes     -> nrt_build_bvh_binary / nrt_scene_create
 *   per-ray traversal + rational Newton   -> nrt_intersect
 *   pinhole primary rays                  -> nrt_generate_camera_rays
 * Each entry point names the reference function it replaces (paths relative
 * to the reference project root).
 *
 * Conventions
 *  - Every function returns an nrt_status; on failure nrt_last_error() gives a
 *    message (thread-local, valid until the next call on that thread).
 *  - Device buffers are owned by the caller and passed as plain pointers.
 *  - Device work is enqueued on the caller's stream (cudaStream_t passed as
 *    void*, NULL = legacy default stream) and is asynchronous unless stated.
 *  - A scene handle may be used from one stream at a time.
 *  - Control points are weighted-homogeneous (w*x, w*y, w*z, w), float32,
 *    exactly as ParametricSurf::nurbsSurf (src/math/nurbs.h:17-22).
 */
#ifndef NRT_H
#define NRT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    NRT_OK = 0,
    NRT_ERR_INVALID = 1,      /* bad argument (null pointer, size, degree) */
    NRT_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    NRT_ERR_UNSUPPORTED = 3,  /* feature not available in this build / on this device */
    NRT_ERR_DEVICE = 4,       /* a kernel reported an error (see nrt_last_error) */
    NRT_ERR_NOMEM = 5         /* host or device allocation failed */
} nrt_status;

#define NRT_MAX_DEGREE 7

/* One NURBS surface: ParametricSurf::nurbsSurf (src/math/nurbs.h:17-22).
 * control_points: (n+1)*(m+1) points, index i*(m+1)+j, i along u.
 * u_knots: n+p+2 values, v_knots: m+q+2 values (clamped). */
typedef struct {
    const float* control_points;
    const float* u_knots;
    const float* v_knots;
    int n, m, p, q;
} nrt_nurbs_surface;

/* ------------------------------------------------------------------------
 * Decomposition.  Replaces BezierPatchOps::getPatch (src/math/bezier_patch.h:86-139)
 * with NurbsOps::decomposeSurface (src/math/nurbs.h:143-250), Algorithm A5.7,
 * for degrees up to NRT_MAX_DEGREE (the reference caps at 4, src/constants.h:31-32).
 * nrt_decompose_count gives nbU, nbV.  nrt_decompose writes nbU*nbV patches,
 * patch (i,j) at i*nbV+j, each (p+1)*(q+1) points with index r*(q+1)+c, r
 * along u, and ranges (u0,u1,v0,v1) per patch.  Host memory, synchronous.
 * The arithmetic is float in the reference's order of operations, so the
 * control points equal getPatch's bit for bit. */
int nrt_decompose_count(const nrt_nurbs_surface* surf, int* nbU, int* nbV);
int nrt_decompose(const nrt_nurbs_surface* surf, float* cp_out, float* ranges_out, int* nbU, int* nbV);

/* Curvature-driven refinement before decomposition: knots inserted along u,
 * then along v, as NurbsOps::curvatureRefinementU / curvatureRefinementV
 * (src/math/nurbs.h:289-486, applied in that order by src/core/main.cpp:100-102).
 * Each knot span gets floor(C * max|A_j| * span^1.5 / sqrt(mean |V_j|))
 * evenly spaced knots (NurbsOps::knotsToAdd, src/math/nurbs.h:254-281; V_j and
 * A_j the first- and second-derivative control vectors of the span,
 * maximised over the net's lines), inserted by Algorithm A5.1 (float, the
 * reference's order of operations).  C <= 0 leaves the surface unchanged.
 * nrt_refine_count gives (n, m) after refinement; nrt_refine_surface writes
 * the (n+1)*(m+1) points (index i*(m+1)+j) and the n+p+2 and m+q+2 knots.
 * Host, synchronous. */
int nrt_refine_count(const nrt_nurbs_surface* surf, float C, int* n_out, int* m_out);
int nrt_refine_surface(const nrt_nurbs_surface* surf, float C, float* cp_out, float* u_knots_out, float* v_knots_out,
                       int* n_out, int* m_out);
/* The same refinement computed on `device`, with the same bits: the counts by
 * one thread per (knot span, line of the net), the A5.1 insertions by one
 * thread per line (NurbsOps::curvatureRefinementU/V, src/math/nurbs.h:289-486,
 * with knotsToAdd :254-281 and curveKnotInsert :96-140).  Host input and
 * output; cp_out holds cap_points points, u_knots_out cap_u and v_knots_out
 * cap_v floats.  *n_out, *m_out are always set; when the outputs are too small
 * (or NULL) the call returns NRT_ERR_INVALID without writing them, so a
 * caller can size them and call again.  Synchronous. */
int nrt_refine_surface_device(const nrt_nurbs_surface* surf, float C, int device, float* cp_out, int64_t cap_points,
                              float* u_knots_out, int cap_u, float* v_knots_out, int cap_v, int* n_out, int* m_out);

/* Patch bounding boxes from the dehomogenised control points:
 * BezierPatchOps::bounds (src/math/bezier_patch.h:153-169).  boxes: 6 floats
 * per patch (min xyz, max xyz).  cp_offset[k] is the first point of patch k,
 * degrees[2k..2k+1] = (p, q). Host, synchronous. */
int nrt_patch_bounds(const float* cp, const int32_t* cp_offset, const int32_t* degrees, int n_patches, float* boxes);

/* Binary BVH in the reference's node layout (BVHNode, src/core/bvh.h:13-17):
 * node_bounds 6 floats, left_first, prim_count; inner nodes have prim_count 0
 * and children left_first, left_first+1.  order[k] = input index of the
 * primitive in leaf slot k (the reference reorders its patch array the same
 * way, src/core/bvh.h:167-175).  Arrays hold 2N-1 nodes; *n_nodes gets the
 * number used.  builder NRT_BVH_EXACT_SAH replaces BvhOps::buildBVH
 * (src/core/bvh.h:148-179) node for node (O(N^2) per level, for small N);
 * NRT_BVH_BINNED_SAH is the O(N log N) builder used for scenes (32 bins,
 * stable partition).  NRT_BVH_BINNED_SAH_DEVICE (scenes only) builds the
 * same tree on the device, together with the decomposition and the packing:
 * the scene it creates is bit-identical to NRT_BVH_BINNED_SAH's. */
enum { NRT_BVH_BINNED_SAH = 0, NRT_BVH_EXACT_SAH = 1, NRT_BVH_BINNED_SAH_DEVICE = 2 };
int nrt_build_bvh_binary(const float* boxes, int n, int builder, float* node_bounds, uint32_t* left_first,
                         uint32_t* prim_count, int32_t* order, int* n_nodes);

/* ------------------------------------------------------------------------
 * Scenes: decomposition + BVH + device upload in one call (the host pipeline
 * of src/core/main.cpp:104-149 / src/core/benchmark.cpp:163-186).  The scene
 * keeps its own device copy (each patch's points as (x, y) and (z, w) pair
 * arrays, 16-byte aligned, in patch-local coordinates; a 4-wide BVH).  Patch ids reported by
 * nrt_intersect are global patch indices in creation order: surface 0's
 * patches first, each surface in getPatch order. */
typedef struct nrt_scene nrt_scene;

typedef struct {
    int builder;        /* NRT_BVH_BINNED_SAH (default), NRT_BVH_EXACT_SAH, or
                           NRT_BVH_BINNED_SAH_DEVICE (whole build on the device) */
    int max_leaf;       /* patches per BVH leaf (1..8, default 1) */
    int device;         /* CUDA device ordinal */
    int64_t wavefront_chunk; /* rays per wavefront pass (0 = 2^23); bounds its scratch,
                                about 1.1 KB per ray, allocated on first use */
} nrt_build_opts;

int nrt_scene_create(const nrt_nurbs_surface* surfaces, int n_surfaces, const nrt_build_opts* opts,
                     nrt_scene** out);
/* Same from patches that are already decomposed (cp_offset/degrees as nrt_patch_bounds). */
int nrt_scene_create_from_patches(const float* cp, const int32_t* cp_offset, const int32_t* degrees, int n_patches,
                                  const nrt_build_opts* opts, nrt_scene** out);
int nrt_scene_destroy(nrt_scene* scene);

typedef struct {
    int n_patches;
    int n_surfaces;
    int n_nodes;        /* 4-wide BVH nodes */
    int bvh_depth;
    size_t device_bytes;
    int degree_hist[(NRT_MAX_DEGREE + 1) * (NRT_MAX_DEGREE + 1)]; /* patches per (p,q), index p*8+q */
} nrt_scene_info;
int nrt_scene_get_info(const nrt_scene* scene, nrt_scene_info* info);
/* Global patch index -> (surface, patch within the surface, u0,u1,v0,v1). Host copies. */
int nrt_scene_patch_table(const nrt_scene* scene, int32_t* surface_of, float* ranges);
/* Copies the scene's whole device arena (info.device_bytes bytes: BVH nodes,
 * packed patches and per-slot tables, counters) to host memory, for
 * inspection; `bytes` must be at least device_bytes.  Synchronous. */
int nrt_scene_copy_arena(const nrt_scene* scene, void* host_dst, size_t bytes);

/* ------------------------------------------------------------------------
 * Rays and hits: structure-of-arrays device buffers (SoAQueue::ray_queue,
 * src/gpu/soa.h:6-14, without the idx_interact slot: misses are patch = -1). */
typedef struct {
    const float *ox, *oy, *oz;
    const float *dx, *dy, *dz;
} nrt_rays;

typedef struct {
    float *ox, *oy, *oz;
    float *dx, *dy, *dz;
} nrt_rays_out;

/* Hit record per ray.  patch = -1 on a miss.  t is the distance along the ray
 * in units of |d| (the reference's t, src/gpu/intersect.cu:129-131, which
 * assumes |d| = 1), (u, v) are patch-local in [0,1].  Optional arrays may be
 * NULL: iters (Newton evaluations of the accepted solve), tests (patch tests
 * that ran Newton), geom (9 floats: S, dS/du, dS/dv in world space, as
 * surfaceInteraction's dpdu/dpdv, src/gpu/interact.h:6-21). */
typedef struct {
    int32_t* patch;
    float* t;
    float* u;
    float* v;
    int32_t* iters;
    int32_t* tests;
    float* geom;
} nrt_hits;

enum { NRT_INIT_MIDPOINT = 0, NRT_INIT_BILINEAR = 1, NRT_INIT_LEARNED = 2 };
enum { NRT_SCHED_PIXEL = 0, NRT_SCHED_WAVEFRONT = 1 };

typedef struct {
    int init_mode;        /* NRT_INIT_*: (0.5,0.5); the reference's bilinear guess
                             (src/math/bezier_patch.h:272-327); or the learned MLP */
    int max_iter;         /* Newton evaluations per (ray, patch); the reference uses 7 */
    float eps;            /* converged when |r1|+|r2| < eps; the reference uses 1e-4 */
    float det_eps;        /* |det J| below this takes the seeded pull step (1e-5) */
    float cond_fp64;      /* solve the 2x2 step in FP64 when cond(J) exceeds this; 0 = never */
    int fp64_final;       /* 1: one FP64 Newton step on the converged point */
    int hull_cull;        /* skip (ray, patch) tests that provably cannot converge (results
                             unchanged): 1 control points all on one side of a ray plane by
                             more than eps; 2 also each half net split at u or v = 1/2;
                             wavefront only: 3 an oriented-box test of each patch during
                             traversal, and no per-pair test after it (the fastest: the
                             per-pair tests cost more than the solves they remove once the
                             box test has run; the per-pixel schedule runs level 1 for it);
                             4 the box test, then the exact 2D hull of the plane residuals
                             and of both halves of the net split at u = 1/2, or at v = 1/2 */
    int schedule;         /* NRT_SCHED_PIXEL or NRT_SCHED_WAVEFRONT */
    int seed_offset;      /* added to the ray index to seed the singular-Jacobian pull */
    float flat_threshold; /* flat-skip in pixels (src/gpu/intersect.cu:104-123); 0 = off.  Both
                             schedules; the culls (hull_cull) can remove pairs that flat-skip
                             would accept, as the reference has no cull */
    float cam_k;          /* 0.5*H/tan(vfov/2), only used by flat-skip */
    int learned_iters;    /* NRT_INIT_LEARNED: evaluations from the network's guess before
                             falling back to plain Newton from (0.5,0.5); 0 = max_iter */
} nrt_intersect_opts;

/* Fill opts with the plain settings: midpoint init, 8 evaluations, eps 1e-6,
 * det_eps 1e-5, no FP64, no cull, per-pixel schedule. */
void nrt_default_opts(nrt_intersect_opts* opts);
/* The reference's settings (calculateIntersectWrapper, src/gpu/intersect.cu:199-220):
 * bilinear init, 7 evaluations, eps 1e-4, det_eps 1e-5. */
void nrt_reference_opts(nrt_intersect_opts* opts);

/* Closest hit for n rays.  Replaces calculateIntersectWrapper /
 * calculateIntersect (src/gpu/intersect.h:9-13, src/gpu/intersect.cu:20-220).
 * Asynchronous on `stream`; device buffers; n may be 0. */
int nrt_intersect(nrt_scene* scene, const nrt_rays* rays, int64_t n, const nrt_intersect_opts* opts,
                  const nrt_hits* hits, void* stream);

/* Intersection without any allocation, for callers that cannot allocate GPU
 * memory while they run: real-time or embedded loops with a fixed memory
 * budget, or code under a memory pool that owns the device.  No reference
 * counterpart: the reference has no scratch-free entry point (its kernel uses
 * no scratch at all, src/gpu/intersect.cu:20-194).
 * It runs the wavefront schedule (opts->schedule is ignored) with its scratch
 * in a fixed 64 MiB array inside libnrt.so, which every GPU that loads the
 * library holds until the process exits; rays go through in passes that fit
 * that array.  Scenes too large for it (about 5 million patches and more) are
 * rejected with NRT_ERR_INVALID.  The first call on a device looks the array
 * up (cudaGetSymbolAddress) and keeps its address for the life of the process;
 * after a cudaDeviceReset (or any other teardown of the device's primary
 * context) that address is stale and this entry point must not be called
 * again in the process.  The call synchronises `stream` once per round to read
 * the number of rays still traversing into a host word, so it must not be
 * called while `stream`, or any other stream of that device, is being captured
 * into a CUDA graph.  All calls share the one array, so calls whose work
 * overlaps on the GPU race: serialise them on one stream.  Rounds run with the
 * scene's round quotas (nrt_scene_set_tuning), as nrt_intersect does. */
int nrt_intersect_noalloc(nrt_scene* scene, const nrt_rays* rays, int64_t n, const nrt_intersect_opts* opts,
                          const nrt_hits* hits, void* stream);

/* Launch shapes of the wavefront schedule, per scene: the autotuner's knobs
 * (no reference counterpart; the reference has one fixed 16x16 launch,
 * src/gpu/intersect.cu:205-217).  In nrt_scene_set_tuning a field <= 0 keeps
 * its current value. */
typedef struct {
    int64_t step_blocks;     /* traversal kernel in the graph: persistent blocks of 128 threads whose
                                warps take 32 active rays at a time */
    int64_t scatter_blocks;  /* work-item scatter in the graph: persistent blocks of 256 threads */
    int32_t class_blocks;    /* blocks of 256 threads per degree-class Newton launch */
    int32_t graph;           /* 1: rounds run inside one CUDA graph with a device-side loop (no host
                                synchronisation); 2: host-driven rounds (one synchronisation each) */
    int64_t chunk;           /* rays per wavefront pass (bounds the scratch, about 1.1 KB per ray) */
    int32_t quota0;          /* candidates a ray emits in the first round, doubling per round ... */
    int32_t quota_max;       /* ... up to this many (<= 8); the default 4, then 8 */
    int32_t stage_nodes;     /* nodes of the top of the 4-wide tree (numbered breadth first, so 1, 5, 21,
                                85 and 341 are whole levels) that each traversal block copies into shared
                                memory and reads from there; 1 (the default: the root only) to 341 */
} nrt_wavefront_tuning;
int nrt_scene_get_tuning(const nrt_scene* scene, nrt_wavefront_tuning* out);
int nrt_scene_set_tuning(nrt_scene* scene, const nrt_wavefront_tuning* in);
/* Autotuner: times nrt_intersect (wavefront) on these rays and buffers under
 * candidate launch shapes, one knob at a time (coordinate descent over
 * traversal and scatter grids, class-launch blocks, round quotas, the
 * staged top of the tree and rays per pass; the graph/host-driven choice
 * stays as set), and keeps the
 * fastest on the scene.  *out gets it and
 * *best_ms its time per call (CUDA events, `reps` calls after one untimed
 * call).  Synchronous.  Results do not depend on the tuning. */
int nrt_autotune(nrt_scene* scene, const nrt_rays* rays, int64_t n, const nrt_intersect_opts* opts,
                 const nrt_hits* hits, int reps, nrt_wavefront_tuning* out, float* best_ms, void* stream);

/* Counters of the last nrt_intersect on this scene (synchronises the stream). */
typedef struct {
    uint64_t rays, box_tests, patch_candidates, patch_culled, newton_solves, newton_evals, fp64_solves,
        fp64_final_steps, hits, errors;
    uint64_t learned_solves;   /* solves started from the network's guess */
    uint64_t learned_fallbacks;/* of those, how many did not converge and fell back to plain Newton */
    uint64_t evals_by_degree[64];      /* Newton evaluations per (p,q), index p*8+q */
    uint64_t hull_tests_by_degree[64]; /* hull tests per (p,q) */
    uint64_t kernel_launches;          /* kernels launched by the last nrt_intersect (host count) */
    uint64_t rounds;                   /* wavefront rounds of the last nrt_intersect */
    double newton_kernel_ms;           /* with kernel timing on: device time of the per-class Newton
                                          launches of the last nrt_intersect (CUDA events) */
    uint64_t newton_kernel_launches;   /* with kernel timing on: how many such launches */
    uint64_t flat_skips;               /* (ray, patch) tests accepted by flat-skip without Newton
                                          (the reference's skip_count, src/gpu/intersect.cu:111) */
    uint64_t learned_converged;        /* learned solves that converged from the network's guess */
    uint64_t learned_fallback_converged; /* learned solves that fell back and then converged in plain
                                            Newton: with learned_converged, the pairs that have a root */
} nrt_counters;
int nrt_enable_counters(nrt_scene* scene, int enable);
/* Kernel timing for roofline measurement: while enabled, the wavefront runs
 * its rounds host-driven and brackets each round's per-class Newton launches
 * with CUDA events on the caller's stream; nrt_get_counters reports their
 * summed device time. */
int nrt_enable_kernel_timing(nrt_scene* scene, int enable);
int nrt_get_counters(nrt_scene* scene, nrt_counters* out, void* stream);

/* ------------------------------------------------------------------------
 * Pinhole camera rays.  Replaces calculateRaysWrapper / calculateRays<perspective>
 * (src/gpu/generateRaysKernel.cu:15-69, src/core/camera.h:63-174): eye, look,
 * up as Transform::lookAt; vertical (short-axis) field of view in degrees;
 * ray index (y*W + x)*spp + s; spp = 1 uses the pixel centre, spp > 1 jitters
 * with a seeded PCG hash.  Directions are unit length. */
typedef struct {
    float eye[3], look[3], up[3];
    float fov_deg;
    int width, height, spp;
    uint32_t seed;
} nrt_camera;
int nrt_generate_camera_rays(const nrt_camera* cam, const nrt_rays_out* out, void* stream);

/* Diffuse bounce rays from the hits of an nrt_intersect (no reference
 * counterpart: the reference traces primary rays only).  For every ray with
 * a hit, the shading normal normalize(dS/dv x dS/du) (the reference's normal,
 * src/gpu/testShading.cu:46) turned against the incoming ray, a
 * cosine-weighted direction about it from a PCG hash of (seed, ray index),
 * and the origin S + offset * normal.  hits->geom is required.  The output is
 * compacted in ray order: out[k], k < *n_out, with src_index[k] the input
 * ray.  scratch: device memory of nrt_bounce_scratch_bytes(n) bytes, or NULL
 * to let the call allocate and free it.  Synchronises `stream` (to return
 * *n_out). */
size_t nrt_bounce_scratch_bytes(int64_t n);
int nrt_generate_bounce_rays(const nrt_rays* rays, const nrt_hits* hits, int64_t n, uint32_t seed, float offset,
                             const nrt_rays_out* out, int32_t* src_index, int64_t* n_out, void* scratch,
                             void* stream);

/* ------------------------------------------------------------------------
 * Output stage (headless).  nrt_shade fills a float RGB framebuffer (SoA,
 * SoAQueue::frame_buffer, src/gpu/soa.h:22-26) from hits: mode 0 the hit mask
 * in red (redTestShading, src/gpu/testShading.cu:9-24), mode 1 the normal map
 * (n + 1) / 2 with n = normalize(dS/dv x dS/du) (normalsTestShading,
 * src/gpu/testShading.cu:27-55; needs hits->geom).  nrt_compare_hits gives per
 * ray, against a reference hit set, the hit-point distance in pixels
 * |P_ref - P_test| cam_k / t_ref and the normal angle in degrees (NaN unless
 * both hit) and a hit/miss mismatch flag, the error measures of the
 * reference's benchmark (src/core/benchmark.cpp:206-222).  Device buffers,
 * asynchronous.  nrt_write_ppm writes host RGB floats in [0,1] as a binary
 * PPM (src/core/benchmark.cpp:85-97). */
int nrt_shade(const nrt_hits* hits, int64_t n, int mode, float* r, float* g, float* b, void* stream);
int nrt_compare_hits(const nrt_rays* rays, const nrt_hits* ref, const nrt_hits* test, int64_t n, float cam_k,
                     float* px_err, float* deg_err, int32_t* mismatch, void* stream);
int nrt_write_ppm(const char* path, int width, int height, const float* r, const float* g, const float* b);

/* ------------------------------------------------------------------------
 * Learned initial guess (no reference counterpart: the reference starts every
 * solve from its bilinear guess, src/gpu/intersect.cu:102).  A 12-64-64-2
 * MLP with SiLU maps (ray, patch) features to a starting (u, v); BF16 tensor
 * cores, FP32 accumulation and FP32 master weights with Adam.  Parameters in
 * this order: W1[64][12], b1[64], W2[64][64], b2[64], W3[2][64], b3[2]. */
#define NRT_MLP_PARAMS 5122
typedef struct nrt_mlp nrt_mlp;
typedef struct {
    int epochs;        /* passes over the samples (20) */
    int batch;         /* samples per Adam step (>= 32) */
    float lr;          /* Adam learning rate (1e-3) */
    float beta1, beta2, eps; /* 0 = 0.9, 0.999, 1e-8 */
    uint32_t seed;     /* shuffling seed */
} nrt_train_opts;
size_t nrt_mlp_param_count(void);
int nrt_mlp_create(int device, uint32_t seed, nrt_mlp** out);   /* Glorot-uniform init */
int nrt_mlp_destroy(nrt_mlp* mlp);
int nrt_mlp_get_params(const nrt_mlp* mlp, float* host_params);  /* NRT_MLP_PARAMS floats */
int nrt_mlp_set_params(nrt_mlp* mlp, const float* host_params);
/* features: device n x 12 floats; out_uv: device n x 2 (unclamped network output). */
int nrt_mlp_forward(const nrt_mlp* mlp, const float* features, int64_t n, float* out_uv, void* stream);
/* Gradient of mean_i |y_i - t_i|^2 over the n rows (one batch), into host memory. */
int nrt_mlp_gradients(nrt_mlp* mlp, const float* features, const float* targets, int64_t n, float* host_grads,
                      float* host_loss, void* stream);
/* Adam training on device samples; host_epoch_loss (optional) gets the mean batch loss per epoch. */
int nrt_mlp_train(nrt_mlp* mlp, const float* features, const float* targets, int64_t n, const nrt_train_opts* opts,
                  float* host_epoch_loss, void* stream);
/* Versioned binary file with a CRC-32 (weights and Adam state). */
int nrt_mlp_save(const nrt_mlp* mlp, const char* path);
int nrt_mlp_load(const char* path, int device, nrt_mlp** out);
/* Copy the network into the scene; enables NRT_INIT_LEARNED for it. */
int nrt_scene_set_mlp(nrt_scene* scene, const nrt_mlp* mlp);
/* Run the wavefront intersection with `opts` (which must use the midpoint
 * guess) and record, for every solve, its 12 features and its converged
 * (u, v), or (-1, -1) when it did not converge: training pairs for the network.  features: device
 * capacity x 12, targets: device capacity x 2; *count gets the number of pairs
 * found (it may exceed capacity; only capacity are written).  Synchronous. */
int nrt_collect_training_data(nrt_scene* scene, const nrt_rays* rays, int64_t n, const nrt_intersect_opts* opts,
                              float* features, float* targets, int64_t capacity, int64_t* count, void* stream);

const char* nrt_last_error(void);
const char* nrt_version(void);

#ifdef __cplusplus
}
#endif
#endif /* NRT_H */
