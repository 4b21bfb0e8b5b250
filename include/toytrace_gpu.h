/*
 * toytrace_gpu.h -- C ABI of the B200 forward path tracer with next-event estimation.
 *
 * This is the drop-in boundary for ToyTrace's `--algo pt` rendering algorithm.  The
 * reference runs that algorithm as `ForwardPathTracer`, a `RenderingAlgo` subclass
 * (src/renderingalgorithms_pathtracing.cxx:59-75; interface in
 * src/renderingalgorithms_interface.hxx:13-30).  A host adapter (toytrace_gpu_algo.hpp)
 * implements that interface on top of the entry points below, so toytrace can select the
 * GPU tracer as one more algorithm name.
 *
 * Conventions
 *  - Every entry point returns a tt_status; nothing throws across the ABI.
 *  - All pointers in tt_scene_desc and in the batch calls are HOST pointers unless the
 *    function name ends in `_device`.
 *  - Spectra are binned: TT_NBINS bins of 10 nm between 370 and 730 nm, bin i centred at
 *    375 + 10 i nm (src/spectral.hxx:24-44).
 *  - Pixel ("unit") index = y * xres + x with y = 0 the BOTTOM row of the image, as in
 *    Camera::UnitToPixel (src/camera.hxx:22-29).  tt_generate_image flips rows the way
 *    framebuffer::ToImage does (src/renderbuffer.hxx:99-125).
 */
#ifndef TOYTRACE_GPU_H
#define TOYTRACE_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TT_NBINS 36
#define TT_ABI_VERSION 9

typedef int32_t tt_status;
enum {
  TT_OK = 0,
  TT_ERR_CUDA = 1,          /* a CUDA runtime call failed (message via tt_last_error) */
  TT_ERR_INVALID = 2,       /* bad argument or malformed scene */
  TT_ERR_CAPACITY = 3,      /* a fixed-size device structure overflowed */
  TT_ERR_LOOP_CAP = 4,      /* a bounded device loop (BVH stack, tracking) hit its cap */
  TT_ERR_INTERRUPTED = 5,   /* the pass was stopped by tt_request_stop */
  TT_ERR_NOT_READY = 6      /* tt_upload_scene has not run yet */
};

/* Shader kinds: the surface scatterers of src/shader.cxx. */
enum {
  TT_SHADER_DIFFUSE = 0,             /* DiffuseShader            shader.cxx:251-318 */
  TT_SHADER_SPECULAR_REFLECTIVE = 1, /* SpecularReflectiveShader shader.cxx:322-366 */
  TT_SHADER_SPECULAR_DIELECTRIC = 2, /* SpecularTransmissiveDielectricShader shader.cxx:378-630 */
  TT_SHADER_MICROFACET = 3,          /* MicrofacetShader (Beckmann, VNDF) shader.cxx:634-707 */
  TT_SHADER_GLOSSY_DIELECTRIC = 4,   /* GlossyTransmissiveDielectricShader (rough Beckmann
                                        interface, alpha and ior_ratio) shader.cxx:710-787 */
  TT_SHADER_SPECULAR_DENSE_DIELECTRIC = 5 /* SpecularDenseDielectricShader: a smooth coating with
                                        Schlick reflectivity specular_reflectivity over a Lambert
                                        base of the reflectance (shader.cxx:977-1081) */
};

/* A material = shader + optional area emitter + optional media on either side
 * (struct Material, src/scene.hxx:45-54).  A material with volume_boundary set has no
 * shader: its triangles only delimit media, are invisible to rays and live in a separate
 * acceleration structure (Scene::BuildAccelStructure's volume scene, scene.cxx:131-137). */
typedef struct tt_material {
  int32_t shader;                  /* TT_SHADER_* (ignored for volume boundaries) */
  float reflectance[TT_NBINS];     /* kr_d / kr_s per bin (diffuse, mirror, microfacet) */
  float alpha;                     /* Beckmann roughness (microfacet, glossy dielectric) */
  float ior_ratio;                 /* inside / outside IOR (dielectrics) */
  int32_t emissive;                /* nonzero: UniformAreaLight on every triangle */
  float emission[TT_NBINS];        /* UniformAreaLight spectrum (area power density;
                                      radiance = spectrum / 2pi, light.hxx:72-108) */
  int32_t medium_inside;           /* 1 + index of the medium behind the winding normal,
                                      0 = none (zero-initialised materials have no media) */
  int32_t medium_outside;          /* 1 + index of the medium the normal points into, 0 = none */
  int32_t volume_boundary;         /* nonzero: medium boundary only, no surface */
  int32_t diffuse_texture;         /* TT_SHADER_DIFFUSE: 1 + index of the tt_texture that multiplies
                                      the reflectance at the hit's texture coordinates
                                      (MaybeMultiplyTextureLookup, shader.cxx:17-27); 0 = none
                                      (also the dense dielectric's diffuse base) */
  float specular_reflectivity;     /* TT_SHADER_SPECULAR_DENSE_DIELECTRIC: reflectivity at normal
                                      incidence of the coating */
} tt_material;

/* An RGB texture (Texture, texture.hxx:15-117): linear RGB floats, width * height * 3, row 0 =
 * the TOP row of the image.  8-bit sRGB images are converted to linear by the caller
 * (Color::SRGBToLinear), as Texture::GetPixel does.  Lookups take the texel under the
 * coordinates wrapped to [0, 1) (UvToPixel, texture.hxx:37-55), no filtering. */
typedef struct tt_texture {
  int32_t width;
  int32_t height;
  const float* rgb;
} tt_texture;

/* Phase functions (src/phasefunctions.cxx). */
enum { TT_PHASE_UNIFORM = 0, TT_PHASE_RAYLEIGH = 1, TT_PHASE_HENYEY_GREENSTEIN = 2 };
enum {
  TT_MEDIUM_HOMOGENEOUS = 0,       /* HomogeneousMedium, shader.cxx:1234-1316 */
  TT_MEDIUM_ATMOSPHERE = 1         /* Atmosphere::Tabulated, atmosphere.cxx:18-126, 234-348 */
};

/* A participating medium.  Priority decides which of overlapping media is current
 * (MediumTracker, rendering_util.hxx:18-126); empty space has priority -1.
 *
 * TT_MEDIUM_HOMOGENEOUS: constant sigma_s, sigma_a per bin and per unit length, with the
 * phase function `phase` (phase_g for Henyey-Greenstein).
 *
 * TT_MEDIUM_ATMOSPHERE: a spherical planet's atmosphere with collision coefficients
 * tabulated over altitude (TabulatedConstituents + SphereGeometry, atmosphere.hxx:79-123),
 * lengths in km.  Altitude = distance to planet_center - planet_radius.  Row i of the
 * tables holds the coefficients per km at altitude table_h0 + i * table_dh, linearly
 * interpolated in between, clamped to row 0 below and zero above the last row.  Molecules
 * scatter with the Rayleigh phase function, aerosols with Henyey-Greenstein(phase_g)
 * (the reference hard-codes g = 0.7, atmosphere.cxx:26).  sigma_s, sigma_a and phase are
 * unused.  The tables are copied by tt_create. */
typedef struct tt_medium {
  int32_t kind;                    /* TT_MEDIUM_* */
  int32_t priority;
  float sigma_s[TT_NBINS];
  float sigma_a[TT_NBINS];
  int32_t phase;                   /* TT_PHASE_* */
  float phase_g;                   /* Henyey-Greenstein asymmetry */
  float planet_center[3];          /* atmosphere only, from here on */
  float planet_radius;
  int32_t table_size;              /* altitude rows, >= 2 */
  float table_h0;
  float table_dh;
  const float* sigma_t;            /* table_size x TT_NBINS, total extinction */
  const float* sigma_s_molecules;  /* table_size x TT_NBINS */
  const float* sigma_s_aerosols;   /* table_size x TT_NBINS */
} tt_medium;

/* Environmental lights: the members of TotalEnvironmentalRadianceField (light.hxx:292-304). */
enum {
  TT_ENV_DOME = 0,        /* DistantDomeLight   light.hxx:180-219: spectrum, dir = up     */
  TT_ENV_SUN = 1,         /* Sun                light.hxx:238-288: scalar = total power,
                             dir = direction the light travels, scalar2 = opening angle deg */
  TT_ENV_MAP = 2,         /* EnvMapLight        light.cxx:88-189: texture, dir = up      */
  TT_ENV_DIRECTIONAL = 3  /* DistantDirectionalLight light.hxx:146-177: spectrum, dir       */
};

typedef struct tt_env_light {
  int32_t kind;
  float spectrum[TT_NBINS];
  float dir[3];
  float scalar;
  float scalar2;
  int32_t tex_width;       /* TT_ENV_MAP: float RGB texture, row 0 = top row of the image */
  int32_t tex_height;
  const float* tex_rgb;    /* tex_width * tex_height * 3 floats (linear RGB) */
} tt_env_light;

/* PointLight (light.hxx:13-42): spectrum = total power, radiated uniformly. */
typedef struct tt_point_light {
  float spectrum[TT_NBINS];
  float pos[3];
} tt_point_light;

enum { TT_CAMERA_PINHOLE = 0, TT_CAMERA_FISHEYE = 1 };

/* PerspectiveCamera (camera.hxx:62-156): fov_deg is the HORIZONTAL full angle.
 * FisheyeHemisphereCamera (camera.hxx:159-232) ignores fov_deg. */
typedef struct tt_camera {
  int32_t kind;
  float pos[3];
  float dir[3];
  float up[3];
  float fov_deg;
  int32_t xres;
  int32_t yres;
} tt_camera;

/* Flat scene.  Triangles are numbered in the order given, spheres after them (sphere i
 * is primitive num_triangles + i); tt_intersect_batch reports these global indices.
 * normals may be NULL (flat shading: smooth normal = geometry normal, like
 * Mesh::MakeFlatNormals, primitive.cxx:18-46).  Spheres are the reference's analytic
 * Spheres geometry (primitive.hxx:94-136): surfaces, area lights or medium boundaries
 * depending on their material, with outward normals. */
typedef struct tt_scene_desc {
  uint32_t num_vertices;
  const float* vertices;        /* num_vertices * 3 */
  const float* normals;         /* num_vertices * 3 or NULL */
  uint32_t num_triangles;
  const uint32_t* indices;      /* num_triangles * 3 */
  const uint32_t* material_ids; /* num_triangles */
  uint32_t num_materials;
  const tt_material* materials;
  uint32_t num_env_lights;
  const tt_env_light* env_lights;
  uint32_t num_point_lights;
  const tt_point_light* point_lights;
  uint32_t num_media;
  const tt_medium* media;
  uint32_t num_spheres;
  const float* spheres;                /* num_spheres * 4: centre x, y, z, radius */
  const uint32_t* sphere_material_ids; /* num_spheres */
  tt_camera camera;
  const float* uvs;             /* num_vertices * 2 texture coordinates (Mesh::uvs), or NULL
                                   (all zero); a triangle hit interpolates them with its
                                   barycentrics; a sphere hit maps its normal to (phi / 2pi,
                                   theta / pi), y up (EmbreeAccelerator, embreeaccelerator.cxx:
                                   216-259) */
  uint32_t num_textures;
  const tt_texture* textures;
} tt_scene_desc;

enum { TT_SAMPLE_BOTH = 0, TT_SAMPLE_BSDF = 1, TT_SAMPLE_LIGHTS = 2 }; /* --pt-sample-mode */
/* --algo: the forward path tracer with NEE (pt, renderingalgorithms_pathtracing.cxx) or its
 * null-path variant (pt2, renderingalgorithms_pathtracing2.cxx). */
enum { TT_ALGO_PT = 0, TT_ALGO_PT2 = 1 };

/* RenderingParameters subset used by the path (src/scene.hxx:24-43). */
typedef struct tt_params {
  int32_t max_ray_depth;        /* --rd (reference default 25) */
  int32_t pt_sample_mode;       /* TT_SAMPLE_* */
  int32_t max_samples_per_pixel;/* --spp; <= 0 means unbounded (Run loops until stopped) */
  int32_t wave_paths;           /* paths resident per wavefront wave; 0 = default (2^27, halved
                                   while the device cannot hold it) */
  int32_t device;               /* CUDA device ordinal */
  int32_t algo;                 /* TT_ALGO_* */
  int32_t qmc;                  /* --qmc (RenderingParameters::qmc): Sobol points with per-pixel
                                   rotations instead of pseudo-random numbers; used by pt2 only
                                   (as in the reference), which then needs max_ray_depth <= 31 */
  int32_t sort_shading;         /* algo pt: 1 = from the second bounce on, before each shading
                                   launch the bounce's hit queue is partitioned by the hit's
                                   shading kind (escaped, volume, one key per shader), so that a
                                   warp shades one material kind; negative = the queue in
                                   traversal order; 0 (the default) = sorted in scenes without
                                   media whose surfaces use three or more shader kinds, else
                                   traversal order */
} tt_params;

typedef struct tt_ctx tt_ctx;

/* Per-context counters, accumulated since tt_reset_stats. */
typedef struct tt_stats {
  uint64_t paths;               /* camera samples started */
  uint64_t extension_rays;      /* closest-hit queries */
  uint64_t shadow_rays;         /* occlusion queries */
  uint64_t extend_launches;     /* closest-hit kernel launches */
  double extend_ms;             /* summed CUDA-event time of those launches (if profiling) */
  uint64_t shadow_launches;
  double shadow_ms;
  double pass_ms;               /* summed CUDA-event time of whole passes */
  uint64_t kernel_launches;     /* all kernels launched by render passes */
  uint64_t node_visits;         /* closest-hit traversal: BVH nodes visited (counting mode) */
  uint64_t tri_tests;           /* closest-hit traversal: triangles tested (counting mode) */
  uint64_t shadow_node_visits;  /* occlusion traversal, counting mode */
  uint64_t shadow_tri_tests;
  uint64_t counted_rays;
  uint32_t bvh_nodes;
  uint32_t bvh_node_bytes;
  uint32_t tri_bytes;
  uint32_t bvh_depth;
  uint64_t error_flags;         /* device error word (TT_ERR_* bits) */
  uint64_t guide_records;       /* training records collected (learned guiding) */
  uint64_t guide_steps;         /* Adam steps taken */
  double guide_loss;            /* mean loss of the last training step */
  double guide_train_ms;        /* summed CUDA-event time of training steps */
} tt_stats;

/* Queue lengths of the last wavefront wave of the last pass: for bounce b = 0..n-1,
 * out[3b] extension rays, out[3b+1] shadow rays, out[3b+2] finished paths.  Returns
 * TT_ERR_INVALID when n exceeds max_ray_depth + 1. */
tt_status tt_last_wave_queue_lengths(tt_ctx* ctx, int32_t* out, int32_t n);

/* Library/ABI version; lets a loader check it bound the right library. */
int32_t tt_abi_version(void);

/* RenderAlgorithmFactory + constructor (renderingalgorithms.cxx:27-42): validates and deep
 * copies the scene description; allocates nothing on the GPU yet.  The large arrays of the
 * copy (vertices, normals, indices, materials per triangle, texture coordinates, environment
 * maps) live in page-locked host memory from a process-wide pool (blocks of 1 MiB and more;
 * reused by later contexts after tt_destroy, up to 4 GiB kept; ordinary memory when the
 * CUDA runtime cannot pin), so that tt_upload_scene copies them by DMA. */
tt_status tt_create(const tt_scene_desc* scene, const tt_params* params, tt_ctx** out_ctx);

/* RenderingAlgo::InitializeScene + Scene::BuildAccelStructure (scene.cxx:116-141): builds
 * the BVH and uploads geometry, materials, lights and the framebuffer. */
tt_status tt_upload_scene(tt_ctx* ctx);

/* One pass of the SamplesPerPixelSchedule loop (renderingalgorithms_simplebase.hxx:125-157):
 * renders spp samples for every pixel into the accumulators.  seed selects the PCG32
 * stream family; samples are numbered consecutively across passes. */
tt_status tt_render_pass(tt_ctx* ctx, int32_t spp, uint64_t seed);

/* Same as tt_render_pass restricted to pixels [pixel_begin, pixel_end). */
tt_status tt_render_pass_range(tt_ctx* ctx, int32_t spp, uint64_t seed,
                               int32_t pixel_begin, int32_t pixel_end);

/* Render pass that allocates no memory.  No counterpart in the reference: it exists for
 * callers that cannot let a library call cudaMalloc at render time -- applications that
 * own all GPU memory through their own pool or a fixed budget, or code where an
 * allocation would synchronise the device and stall concurrent work.  The wavefront path
 * state lives in one static device array inside the library (about 14.7 MB, held by every
 * GPU that loads the library until the process exits) instead of memory the context
 * allocates.  The caller passes the outputs: d_accum and d_light_accum are device buffers
 * of xres*yres*3 floats to which the pass ADDS the unnormalised RGB sums of its samples and
 * the camera-vertex splats (already weighted by 1/(xres*yres)), like one pass of
 * tt_render_pass before it folds them into its own accumulators; sample numbers
 * sample_offset .. sample_offset+spp-1 select the same random streams tt_render_pass uses.
 * The context's own accumulators, counters and statistics are not touched.
 * Limits: at most 65,536 camera samples (spp x pixels in [pixel_begin, pixel_end)) per
 * call and max_ray_depth <= 1000, else TT_ERR_CAPACITY.  Calls on one device share the
 * static array: calls that overlap on the GPU race.  The call returns after the work has
 * finished on `stream` (a cudaStream_t; NULL = legacy default stream).  Its first call on
 * a device looks up the array's device address (cudaGetSymbolAddress) and must come before
 * any stream capture.  Requires tt_upload_scene (which allocates the scene) to have run.
 * The pass always renders unguided, also in a context with guiding enabled (the guide's
 * records and network inputs need buffers of their own), shades in traversal order whatever
 * sort_shading says (the sort needs buffers of its own too), and algo pt only
 * (TT_ERR_INVALID for pt2).  A stop requested before the call makes it return TT_ERR_INTERRUPTED without
 * rendering; a stop requested while it runs does not cut it short. */
tt_status tt_render_pass_noalloc(tt_ctx* ctx, int32_t spp, uint64_t seed, int32_t pixel_begin,
                                 int32_t pixel_end, uint64_t sample_offset, float* d_accum,
                                 float* d_light_accum, void* stream);

/* RenderingAlgo::RequestInterrupt / RequestFullStop: lock-free flag writes, callable from
 * any thread, also before the first pass.  A stop makes the running and all later
 * passes return TT_ERR_INTERRUPTED at the next wave boundary. */
tt_status tt_request_interrupt(tt_ctx* ctx);
tt_status tt_request_stop(tt_ctx* ctx);
/* Returns 1 and clears the flag if an interrupt was requested since the last poll. */
int32_t tt_poll_interrupt(tt_ctx* ctx);
int32_t tt_stop_requested(tt_ctx* ctx);

/* Linear RGB per pixel = accum / samples_per_pixel + light_accum * npix / splat_count,
 * exactly Spectral3ImageBuffer::ToImage before the clamp (renderbuffer.hxx:172-200).
 * rgb: npix*3 floats.  sample_counts (nullable): npix entries of samples per pixel. */
tt_status tt_read_framebuffer(tt_ctx* ctx, float* rgb_linear, uint64_t* sample_counts);

/* Raw accumulators for parity tests: accum and light_accum, npix*3 doubles each. */
tt_status tt_read_accumulators(tt_ctx* ctx, double* accum, double* light_accum,
                               uint64_t* samples_per_pixel, uint64_t* splat_count);

/* GenerateImage: 8-bit RGB, clamp to [0,1], sRGB unless linear, rows flipped
 * (framebuffer::ToImage, renderbuffer.hxx:99-125).  out: xres*yres*3 bytes. */
tt_status tt_generate_image(tt_ctx* ctx, int32_t linear_output, uint8_t* out_rgb8);

/* Clears accumulators and sample counters. */
tt_status tt_clear_framebuffer(tt_ctx* ctx);

/* Closest-hit queries (EmbreeAccelerator::FirstIntersection, embreeaccelerator.cxx:87-131).
 * rays: n * 8 floats (org xyz, tnear, dir xyz, tfar).  Outputs (n each): prim id or -1,
 * hit distance, barycentric u, v (hit = (1-u-v) v0 + u v1 + v v2). */
tt_status tt_intersect_batch(tt_ctx* ctx, const float* rays, int32_t n,
                             int32_t* prim_ids, float* t, float* u, float* v);
/* Occlusion queries (EmbreeAccelerator::IsOccluded, embreeaccelerator.cxx:284-304). */
tt_status tt_occluded_batch(tt_ctx* ctx, const float* rays, int32_t n, uint8_t* occluded);
/* Device-pointer variants; stream is a cudaStream_t (NULL = legacy default stream). */
tt_status tt_intersect_batch_device(tt_ctx* ctx, const float* d_rays, int32_t n,
                                    int32_t* d_prim_ids, float* d_t, float* d_u, float* d_v,
                                    void* stream);

/* Counting traversal over a ray batch: adds nodes visited and triangles tested to the
 * stats (for the algorithmic-bytes model of the closest-hit kernel). */
tt_status tt_count_traversal(tt_ctx* ctx, const float* rays, int32_t n);

/* BSDF sampling/evaluation on the device for the sampling tests
 * (ShaderScatterer fixture, tests_sampling.cxx:932-1046).  The surface lies in the
 * z = 0 plane with geometry and shading normal +z; wi: reverse incident direction
 * (pointing away from the surface).  lambda_idx: 3 bin indices.
 *   sample: out_dir n*3, out_value n*3, out_pdf n (negative = from a delta distribution).
 *   eval:   dirs n*3 in, out_value n*3, out_pdf n. */
tt_status tt_sample_bsdf_batch(tt_ctx* ctx, int32_t material, const float* wi,
                               const int32_t* lambda_idx, int32_t n, uint64_t seed,
                               float* out_dir, float* out_value, float* out_pdf);
tt_status tt_eval_bsdf_batch(tt_ctx* ctx, int32_t material, const float* wi,
                             const int32_t* lambda_idx, const float* dirs, int32_t n,
                             float* out_value, float* out_pdf);

/* Phase-function sampling/evaluation on the device for the sampling tests
 * (PhaseFunctionTests, tests_sampling.cxx:1202-1259): the phase function of medium `medium`
 * (index into tt_scene_desc.media) at a volume vertex at pos -- a homogeneous medium's own
 * function, or the atmosphere's SimpleCombined Rayleigh + Henyey-Greenstein mixture weighted
 * by the constituents' sigma_s at pos's altitude (phasefunctions.cxx:206-273).  wi: reverse
 * incident direction (the direction of travel is -wi).  Sample i draws from the PCG32 stream
 * (seed, i).  Outputs as the BSDF batch calls; value per selected wavelength, pdf. */
tt_status tt_sample_phase_batch(tt_ctx* ctx, int32_t medium, const float* pos, const float* wi,
                                const int32_t* lambda_idx, int32_t n, uint64_t seed,
                                float* out_dir, float* out_value, float* out_pdf);
tt_status tt_eval_phase_batch(tt_ctx* ctx, int32_t medium, const float* pos, const float* wi,
                              const int32_t* lambda_idx, const float* dirs, int32_t n,
                              float* out_value, float* out_pdf);

/* Device-side copy of the raw accumulators into caller-owned device buffers (npix*3
 * doubles each), ordered on `stream` (a cudaStream_t; NULL = legacy default stream).
 * Lets a multi-GPU caller reduce framebuffers with NCCL without a host round trip. */
tt_status tt_read_accumulators_device(tt_ctx* ctx, double* d_accum, double* d_light_accum, void* stream);

/* Profiling level: 0 off; 1 render passes time each closest-hit and shadow launch with
 * CUDA events on the launching stream and add the durations to the stats; 2 additionally
 * counts BVH nodes visited and triangles tested (slower; for the bytes-per-ray model). */
tt_status tt_set_profiling(tt_ctx* ctx, int32_t on);
tt_status tt_get_stats(tt_ctx* ctx, tt_stats* out);
tt_status tt_reset_stats(tt_ctx* ctx);

/* Last error message of this context (or of the last failed tt_create when ctx is NULL). */
tt_status tt_last_error(tt_ctx* ctx, char* buf, int32_t n);

/* ---- Learned path guiding ----------------------------------------------------------
 * The reference's guided path tracer (renderingalgorithms_pathtracing_guided.cxx) samples
 * non-delta surface vertices from a vMF mixture combined with the BSDF by one-sample MIS
 * (SampleWithBinaryMixtureDensity, :474-524), the mixtures being fitted per spatial cell
 * from radiance records (path_guiding.cxx).  Here a small MLP maps (position, normal,
 * outgoing direction) to an 8-lobe vMF mixture and to the probability of sampling it; it is
 * trained online on the paths' own records by BF16 tensor-core kernels.  These entry
 * points have no counterparts in the reference. */
typedef struct tt_guiding_params {
  int32_t enabled;              /* 1: guided sampling at diffuse and microfacet surfaces */
  int32_t train;                /* 1: collect records and train after every pass;
                                   2: collect records only (tt_guide_read_records) */
  float learning_rate;          /* Adam step size (0: 1e-3) */
  int32_t record_pool;          /* records kept across passes, a ring that overwrites the
                                   oldest (0: 65536); only records that carry light are kept */
  int32_t batch;                /* records per Adam step, drawn at random from the pool (0: 8192) */
  int32_t steps_per_pass;       /* Adam steps after each pass (0: 16) */
  int32_t max_depth;            /* guide the vertices of the first max_depth bounces only, BSDF
                                   sampling beyond (0: every bounce) */
  uint64_t seed;                /* weight initialisation */
  int32_t method;               /* TT_GUIDE_LEARNED (the network) or TT_GUIDE_TREE (the
                                   reference's kd-tree cells with vMF mixtures, below) */
  int32_t tree_subdivision;     /* TT_GUIDE_TREE: records per cell of the initial tree
                                   (--guide-subdiv-factor, scene.hxx:39; 0: 100) */
  int32_t tree_em_iters;        /* TT_GUIDE_TREE: 0 = the reference's incremental EM (a
                                   maximisation step every 10 x prior strength records, each
                                   on that chunk alone); k > 0 = k EM iterations per round over
                                   all of the round's records of the cell */
  int32_t network;              /* TT_GUIDE_LEARNED: the kernels that evaluate and train the
                                   network, TT_GUIDE_NET_TCGEN05 (tensor-memory accumulators,
                                   128-row tiles; a training step is one kernel) or
                                   TT_GUIDE_NET_MMA (warp-level mma.sync, 16-row tiles); both
                                   give the same network outputs, and gradients equal up to the
                                   rounding of BF16 hidden gradients */
  int32_t tree_distribution;    /* TT_GUIDE_TREE: the directional distribution of a cell,
                                   TT_TREE_VMF (8-lobe vMF mixture, the reference's MoVmf
                                   distribution) or TT_TREE_QUADTREE (the reference's active
                                   quadtree radiance distribution, fitted with the stochastic
                                   record filter) */
} tt_guiding_params;
enum { TT_GUIDE_LEARNED = 0, TT_GUIDE_TREE = 1 };
enum { TT_GUIDE_NET_TCGEN05 = 0, TT_GUIDE_NET_MMA = 1 };
enum { TT_TREE_VMF = 0, TT_TREE_QUADTREE = 1 };

/* Enables or disables guiding.  The network is created (He-uniform weights from `seed`) on
 * first use and keeps its trained weights while guiding is switched off and on again.  Until
 * its first training step (or tt_guide_set_params) the network is not sampled: guided
 * vertices draw from the BSDF alone, which keeps the first pass as good as unguided
 * rendering while it collects the first training records. */
tt_status tt_set_guiding(tt_ctx* ctx, const tt_guiding_params* params);
/* Number of network parameters (FP32 layout: per layer W[out][in] then b[out]). */
int32_t tt_guide_num_params(void);
tt_status tt_guide_get_params(tt_ctx* ctx, float* out, int32_t n);
tt_status tt_guide_set_params(tt_ctx* ctx, const float* in, int32_t n);
/* Network outputs (n x 48) for n rows of 96 input features (host buffers). */
tt_status tt_guide_forward_batch(tt_ctx* ctx, const float* features, int32_t n, float* out);
/* The same forward pass on the tcgen05 tensor cores (128-row tiles, accumulators in tensor
 * memory); TT_ERR_LOOP_CAP if a wait on the tensor cores timed out. */
tt_status tt_guide_forward_batch_tc(tt_ctx* ctx, const float* features, int32_t n, float* out);
/* Mean-loss gradient (tt_guide_num_params floats) and the loss for n training records of
 * 14 floats each: position in [0,1]^3, normal, outgoing direction, sampled direction,
 * BSDF pdf of the sampled direction, F/q (host buffers). */
tt_status tt_guide_gradient_batch(tt_ctx* ctx, const float* records, int32_t n, float* grad, float* loss);
/* The same mean-loss gradient over a mini-batch of n records drawn from a pool of pool_n
 * records (host buffer) the way the renderer's training steps draw theirs: record i of the
 * mini-batch is pool[h(seed ^ h(i)) mod pool_n], h the SplitMix64 finalizer, gathered on the
 * device by the gradient kernel itself. */
tt_status tt_guide_gradient_pool_batch(tt_ctx* ctx, const float* pool, int32_t pool_n, int32_t n, uint64_t seed,
                                       float* grad, float* loss);
/* `steps` Adam steps of size learning_rate on n training records (layout as above; host
 * buffer), the optimiser state carried over from earlier steps; *loss = the loss of the
 * last step's gradient (may be NULL). */
tt_status tt_guide_train_batch(tt_ctx* ctx, const float* records, int32_t n, int32_t steps, float learning_rate,
                               float* loss);
/* Copies up to max_records training records of the pool (14 floats each, layout above) to
 * `out`, *n = the number copied, and empties the pool. */
tt_status tt_guide_read_records(tt_ctx* ctx, float* out, int32_t max_records, int32_t* n);
/* Feature encoding of n points (position in [0,1]^3, normal, outgoing direction: 9 floats
 * each) into n x 96 features, as the renderer computes them. */
tt_status tt_guide_features_batch(tt_ctx* ctx, const float* points, int32_t n, float* features);

/* Tree guider (method TT_GUIDE_TREE): the guided tracer's spatial cells (PathGuiding,
 * path_guiding.cxx:347-813) with per-cell 8-lobe vMF mixtures (MoVmfRadianceDistribution,
 * path_guiding.hxx:63-190) fitted by incremental EM with a prior
 * (distribution_mixture_models.cxx:279-388), sampled against the BSDF with probability 0.5
 * (renderingalgorithms_pathtracing_guided.cxx:470).  After each training pass the pass's
 * records are fitted into the cells on the GPU (one warp per cell); the first round builds
 * the kd-tree from the records, later rounds split cells that received too many.
 * Cell and node counts, fitted rounds and records: */
tt_status tt_guide_tree_info(tt_ctx* ctx, int32_t* cells, int32_t* nodes, int32_t* rounds, int64_t* records);
/* Mixtures of the first max_cells cells, 40 floats each: weights[8], means[8][3],
 * concentrations[8]. */
tt_status tt_guide_tree_mixtures(tt_ctx* ctx, float* out, int32_t max_cells);
/* Cells of n normalised positions (3 floats each) in the current tree. */
tt_status tt_guide_tree_lookup_batch(tt_ctx* ctx, const float* points, int32_t n, int32_t* cells);
/* The fit of one cell on the device, for tests: n records of 4 floats (direction xyz,
 * weight) in the order given, starting from mixture_in / fit_in (NULL: the prior mixture
 * and an empty fit state of 36 floats: mean weight, its count, max record count, pending
 * count, pending sums), incremental (batch_iters = 0) or batch EM; writes the 40-float
 * mixture and the fit state. */
tt_status tt_vmf_fit_batch(const float* records, int32_t n, const float* mixture_in, const float* fit_in,
                           int32_t batch_iters, float* mixture_out, float* fit_out);
/* The initial kd-tree build over n points (3 floats each, host only, no device use): writes
 * each point's cell and *cells; min_points as --guide-subdiv-factor. */
tt_status tt_kdtree_build_batch(const float* points, int32_t n, int32_t min_points, int32_t* cell_of_point,
                                int32_t* cells);
/* Quadtree radiance distribution (tree_distribution = TT_TREE_QUADTREE; path_guiding.cxx:
 * 108-310, path_guiding_quadtree.cxx).  Directions map to the unit square by
 * u = atan2(y, x) / (2 pi) + 1/2, v = (z + 1) / 2; a node's children are the quadrants
 * 0 = (u < c, v < c), 1 = (u >= c, v < c), 2 = (u < c, v >= c), 3 = (u >= c, v >= c) of its
 * square; every parent precedes its children.  Sampling weights: leaves as fitted, inner
 * nodes the sums of their children.
 * A cell's current distribution: children (4 per node, -1 for a leaf) and sampling weights
 * of up to cap nodes, *num_nodes = its node count (TT_ERR_CAPACITY if above cap). */
tt_status tt_guide_tree_quadtree(tt_ctx* ctx, int32_t cell, int32_t cap, int32_t* children, float* weights,
                                 int32_t* num_nodes);
/* The quadtree fit on the host, for tests (no device use): InitialFit + Bake on the na
 * records A (unit directions, 3 floats each, and weights); with stage >= 1 then
 * IncrementalFit of the nb records B; with stage >= 2 then IterationUpdateAndBake.  Writes
 * children, sampling weights and the prior of up to cap nodes and *num_nodes. */
tt_status tt_quadtree_fit_batch(const float* dirs_a, const float* weights_a, int32_t na, const float* dirs_b,
                                const float* weights_b, int32_t nb, int32_t stage, int32_t cap, int32_t* children,
                                float* weights, float* prior, int32_t* num_nodes);
/* The device sampler of the tree-guided kernel on a given quadtree, for tests: n directions
 * drawn with the uniforms u[2i], u[2i+1] (hierarchical warping), their densities per unit
 * solid angle, and the density the guided kernel evaluates at the returned direction. */
tt_status tt_quadtree_sample_batch(const int32_t* children, const float* weights, int32_t num_nodes, const float* u,
                                   int32_t n, float* out_dir, float* out_pdf, float* out_pdf_eval);

/* ---- Multi-view batches ------------------------------------------------------------
 * No counterpart in the reference (it renders one camera per RenderingAlgo).  A batch of
 * views of the uploaded scene, each with its own camera, resolution and samples per pixel,
 * is rendered as one wavefront: the waves run over the concatenation of the views' pixel
 * and sample ranges, so many small views fill the GPU like one large frame.  The per-wave
 * launch sequence runs as one captured CUDA graph, replayed for every wave. */
typedef struct tt_view {
  tt_camera camera;
  int32_t spp;
} tt_view;

/* Renders views[0..n) and writes their linear RGB images (row 0 at the bottom, as
 * tt_read_framebuffer) one after the other into rgb (host; 3 * sum(xres * yres) floats).
 * View v uses the random streams of a single-camera tt_render_pass of that camera with
 * seed + v and sample numbers 0..spp-1.  The context's own framebuffer is not touched. */
tt_status tt_render_views(tt_ctx* ctx, const tt_view* views, int32_t n, uint64_t seed, float* rgb);

/* Completion time of every view of the last tt_render_views call, in ms after the batch
 * started on the device (CUDA events): a view is complete when the wave that holds its last
 * path has finished.  -1 for views a stop request left unfinished.  n must equal the last
 * batch's view count. */
tt_status tt_views_completion_ms(tt_ctx* ctx, float* out, int32_t n);

#define TT_TUNE_MAX 16
typedef struct tt_tune_result {
  int32_t wave_paths;           /* chosen paths per wave (queue capacity) */
  int32_t grid;                 /* chosen blocks per wavefront launch */
  double ms;                    /* probe time of the chosen configuration */
  int32_t candidates;
  int32_t candidate_wave[TT_TUNE_MAX];
  int32_t candidate_grid[TT_TUNE_MAX];
  double candidate_ms[TT_TUNE_MAX];
  int32_t block;                /* chosen threads per block of the wavefront launches */
  int32_t bvh_width;            /* chosen BVH layout: 4 (the device-built tree with four children
                                   per node, the default), 2 (binary: host-built trees) or 8
                                   (8-wide compressed) */
  int32_t candidate_block[TT_TUNE_MAX];
  int32_t candidate_width[TT_TUNE_MAX];
} tt_tune_result;

/* Autotuner: times one-sample probes of the batch over queue capacities (2^22, 2^24, 2^25,
 * 2^26 paths per wave) and launch widths (0.5, 1, 2 x the occupancy grid) with 256-thread
 * blocks on the default BVH layout; then, at the best of those, 128-thread blocks (twice the grid)
 * and the 8-wide compressed BVH (built on the host on first use, kept next to the default
 * one); and keeps the fastest configuration for this context's later passes. */
tt_status tt_autotune_views(tt_ctx* ctx, const tt_view* views, int32_t n, tt_tune_result* out);

void tt_destroy(tt_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* TOYTRACE_GPU_H */
