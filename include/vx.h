/*
 * vx.h - C ABI of libvx: B200-native ESVO voxel ray casting.
 *
 * Drop-in boundary for the reference's voxel ray-casting hot path
 * (Lint111/VBVS--VIXEN).  Each entry point names the reference interface it
 * replaces; paths are relative to the reference project's VIXEN/ directory.
 *
 * Conventions
 *  - Plain C types only.  A stream is passed as `void*` holding a
 *    cudaStream_t (NULL = legacy default stream).
 *  - Every call returns VX_OK or a negative vx_status; the message of the
 *    last error on the calling thread is in vx_last_error_string().  No C++
 *    exception crosses this boundary (the reference nodes throw
 *    std::runtime_error, ComputeDispatchNode.cpp:67,78,100,227).
 *  - A vx_scene's arrays are immutable after creation and it may be used
 *    from any host thread; device work is ordered on the stream given to
 *    each call.  Exception: vx_cast_shadow_rays keeps scratch in the scene,
 *    so its calls on one scene must not overlap on the GPU.
 *  - "_dev" pointers are device pointers (cudaMalloc / torch tensors) on the
 *    scene's device; "_host" pointers are host memory (pinned for best speed).
 */
#ifndef VX_H
#define VX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VX_ABI_VERSION 2

typedef enum vx_status {
    VX_OK = 0,
    VX_EINVAL = -1,     /* bad argument or malformed scene buffers */
    VX_ECUDA = -2,      /* a CUDA runtime call failed */
    VX_EOVERFLOW = -3,  /* a size is beyond a format limit */
    VX_ETIMEOUT = -4,   /* a bounded device-side wait gave up */
    VX_ENOMEM = -5,     /* host or device allocation failed */
    VX_ENOTFOUND = -6,  /* no CUDA device, or the library was built without one */
    VX_EIO = -7,        /* a file could not be opened, read or written */
    VX_EFORMAT = -8     /* a file is not in the expected format */
} vx_status;

/* ------------------------------------------------------------------------
 * Device data layout
 * --------------------------------------------------------------------- */

/* One octree node ("child descriptor"), 8 bytes.
 * Replaces ChildDescriptor (SVO/include/SVOTypes.h:36-117), whose 15-bit
 * childPointer is widened to 32 bits so scenes above 32,767 descriptors
 * keep the indices an unbounded reference would produce.
 *   child_ptr : index of the first child descriptor (children are stored
 *               contiguously, non-leaf children first, octant ascending)
 *   masks     : valid_mask (bits 0-7) | leaf_mask (bits 8-15)        */
typedef struct vx_node {
    uint32_t child_ptr;
    uint32_t masks;
} vx_node;

/* The OctreeConfig fields the traversal needs
 * (RenderGraph/src/Nodes/VoxelGridNode.cpp:36-66; filled at
 * CashSystem/src/VoxelSceneCacher.cpp:592-625). */
typedef struct vx_octree_config {
    float world_min[3];     /* rebuild() bounds (SVORebuild.cpp:228) */
    float world_max[3];
    int32_t max_levels;     /* userMaxLevels (octree depth), 1..23 */
    int32_t brick_depth;    /* brickDepthLevels; must be 3 (8^3 bricks) */
    int32_t bricks_per_axis;/* ceil(int(world size x) / 8) (SVORebuild.cpp:261-262) */
    int32_t reserved;
} vx_octree_config;

/* Brick colour payload kinds. */
typedef enum vx_color_kind {
    VX_COLOR_NONE = 0,
    VX_COLOR_RGBA8 = 1,  /* 512 x u32 per brick, voxel z*64+y*8+x (brickData layout,
                            VoxelSceneCacher.cpp:551-578) */
    VX_COLOR_DXT1 = 2,   /* 32 x u64 BC1 blocks per brick, block = voxel >> 4
                            (VoxelRayMarch_Compressed.comp:142-158) */
    VX_COLOR_MATERIAL = 3 /* 512 x u32 material words per brick, voxel z*64+y*8+x:
                            the reference's brickData (VoxelSceneCacher.cpp:551-587,
                            material id per voxel, 0 = empty).  A hit is coloured
                            getMaterialColor(word & 0xFF) (shaders/Materials.glsl:18-60,
                            VoxelRayMarch.comp:188-192); occupancy (brick_occ) must be
                            word != 0, the shader's test */
} vx_color_kind;

/* Host-side description of a scene: the buffers VoxelGridNode publishes
 * (RenderGraph/include/Data/Nodes/VoxelGridNodeConfig.h:68-125) in this
 * library's layout.  vx_scene_create copies them to the device. */
typedef struct vx_scene_desc {
    vx_octree_config config;
    const vx_node* nodes;          /* node_count descriptors, root at 0 */
    uint32_t node_count;
    uint32_t brick_count;
    const uint32_t* node_brick;    /* node_count: brick index field of each
                                      descriptor (leafToBrickView source,
                                      SVORebuild.cpp:569-574) */
    const uint32_t* grid_lookup;   /* bricks_per_axis^3, x fastest, brick index
                                      or 0xFFFFFFFF (brickGridLookup,
                                      VoxelSceneCacher.cpp:670-713) */
    const uint32_t* brick_coord;   /* brick_count: grid coordinate
                                      x | y<<10 | z<<20 */
    const uint32_t* brick_occ;     /* brick_count x 16 u32: occupancy bit of
                                      voxel i at word i>>5, bit i&31 */
    int32_t color_kind;            /* vx_color_kind */
    const void* brick_color;       /* RGBA8 or DXT1 payload, or NULL */
    const void* brick_normal;      /* NULL, or brick_count x 32 DXT normal
                                      blocks of 16 B {blockA, blockB}
                                      (COMPRESSED_NORMAL_BUFFER,
                                      SVORebuild.cpp:615-722); see
                                      vx_build_normals */
} vx_scene_desc;

/* Ray: origin and direction (need not be normalised; the cast normalises
 * like validateRayInput, SVOTraversal.cpp:238-259). 24 bytes. */
typedef struct vx_ray {
    float ox, oy, oz;
    float dx, dy, dz;
} vx_ray;

/* Hit flags (vx_hit.flags). */
#define VX_HIT_HIT          0x01u /* the ray hit a voxel */
#define VX_HIT_AXIS_MASK    0x06u /* entry-face normal axis (0 x, 1 y, 2 z) << 1 */
#define VX_HIT_NORMAL_NEG   0x08u /* normal component is -1 (else +1) */
#define VX_HIT_METHOD_MASK  0x30u /* brick lookup that found the brick (1 position,
                                     2 ray entry, 3 octant) << 4 */
#define VX_RAY_ITER_CAP     0x40u /* traversal stopped at the 500-iteration cap */
#define VX_RAY_INVALID      0x80u /* rejected by input validation */

/* Hit record, 16 bytes.  Replaces ISVOStructure::RayHit
 * (SVO/include/ISVOStructure.h:101-112): tMin -> t, entity -> (brick, voxel),
 * normal -> flags; tMax = t + 1 and hitPoint = origin + normalize(dir) * t
 * follow from these. */
typedef struct vx_hit {
    float t;          /* hit distance along the normalised direction, world units */
    uint32_t brick;   /* brick index, 0xFFFFFFFF on a miss (and on an LOD hit) */
    uint32_t node;    /* index of the parent descriptor at the leaf */
    uint16_t voxel;   /* voxel within the brick, z*64+y*8+x; 0xFFFF on a miss */
    uint8_t flags;    /* VX_HIT_* / VX_RAY_* */
    uint8_t scale;    /* RayHit::scale: max_levels - 1 for a voxel hit
                         (SVOBrickDDA.cpp:509), the cell's user scale for an
                         LOD hit, 0 on a miss */
} vx_hit;

/* Per-ray work counters (optional output, for algorithmic-byte accounting),
 * 16 bytes.  The first three are the reference traversal's counts (bounds:
 * iters <= 500, grid_reads <= 2 and dda_steps <= 24 per iteration); the
 * run_* fields are what the kernel executed, which is less when a ray is
 * caught in a repeating cycle before the iteration cap. */
typedef struct vx_ray_counters {
    uint16_t iters;           /* ESVO loop iterations */
    uint16_t grid_reads;      /* brickGridLookup reads */
    uint32_t dda_steps;       /* DDA occupancy tests */
    uint16_t run_iters;
    uint16_t run_grid_reads;
    uint32_t run_dda_steps;
} vx_ray_counters;

/* Camera push constants, 64 bytes: the PushConstants block of
 * shaders/VoxelRayMarch.comp:85-94 (fov in degrees, vertical). */
typedef struct vx_camera_pc {
    float camera_pos[3];  float time;
    float camera_dir[3];  float fov;
    float camera_up[3];   float aspect;
    float camera_right[3]; int32_t debug_mode;
} vx_camera_pc;

typedef struct vx_scene vx_scene;

/* ------------------------------------------------------------------------
 * Library
 * --------------------------------------------------------------------- */
int32_t vx_abi_version(void);
/* Message of the last failed call on this thread ("" if none). */
const char* vx_last_error_string(void);

/* ------------------------------------------------------------------------
 * Scene lifetime.  Replaces VoxelSceneCacher::UploadToGPU
 * (CashSystem/src/VoxelSceneCacher.cpp:719-891): one device allocation with
 * 256-byte aligned sub-buffers, owned by the scene.  The grid lookup entries
 * and brick coordinates are validated on the host before upload, so every
 * device read stays in bounds; child pointers are bounds-checked during
 * traversal exactly as executePushPhase does (SVOTraversal.cpp:352-354).
 * The scene lives on the device current at creation.
 * --------------------------------------------------------------------- */
int vx_scene_create(const vx_scene_desc* desc, vx_scene** out);
int vx_scene_destroy(vx_scene* scene);
/* Device bytes held by the scene. */
int vx_scene_device_bytes(const vx_scene* scene, uint64_t* out);

/* Bounds checks.  libvx_checked.so (make checked) is this library with every
 * device index into the scene arrays, the traversal stack and the batch's
 * scene table tested before its load; a failing test sets a bit (1 node, 2
 * brick grid, 4 brick, 8 voxel, 16 stack slot, 32 scene table) and the load
 * reads element 0 instead.  This call reports whether the loaded library is
 * that build and returns the bits set since the last call (clearing them)
 * after synchronising the device; the default build reports 0 / 0.  It stands
 * in for a memory checker where none can run. */
int vx_bounds_checks(int32_t* enabled, uint32_t* violations);

/* What a scene holds (for vx_scene_download and cache files). */
typedef struct vx_scene_info {
    vx_octree_config config;
    uint32_t node_count;
    uint32_t brick_count;
    int32_t color_kind;
    int32_t has_normals;
} vx_scene_info;
int vx_scene_info_get(const vx_scene* scene, vx_scene_info* out);
/* Copies the scene's device arrays into caller host buffers of the sizes
 * vx_scene_desc gives them (nodes: node_count x 2 u32; normals: brick_count
 * x 64 u64); any pointer may be NULL.  Synchronous. */
int vx_scene_download(const vx_scene* scene, uint32_t* nodes, uint32_t* node_brick, uint32_t* grid_lookup,
                      uint32_t* brick_coord, uint32_t* brick_occ, void* brick_color,
                      uint64_t* brick_normal);

/* ------------------------------------------------------------------------
 * Scene cache files.  Replaces VoxelSceneCacher::SerializeToFile /
 * DeserializeFromFile (CashSystem/src/VoxelSceneCacher.cpp:179-364).
 * VXSC: this library's format, every array of a scene exactly, with a
 * checksum.  VSCA version 1: the reference's format (one entry written;
 * reading picks entry `entry`): ESVO descriptors in ChildDescriptor layout
 * (child pointers must fit 15 bits), brickData material words (occupied = 1),
 * DXT1 colours, DXT normals, brickGridLookup, OctreeConfig.  Reading keeps the
 * brickData material words (occupancy = word != 0); writing stores a
 * VX_COLOR_MATERIAL scene's words as brickData (otherwise 1 per occupied
 * voxel).  A vx_cache holds the host arrays; vx_cache_desc exposes them for
 * vx_scene_create.
 * --------------------------------------------------------------------- */
typedef struct vx_cache vx_cache;
int vx_cache_write(const char* path, const vx_scene_desc* desc);
int vx_cache_read(const char* path, vx_cache** out);
int vx_cache_write_vsca(const char* path, const vx_scene_desc* desc, uint32_t scene_type,
                        uint32_t resolution, float density, uint32_t seed);
int vx_cache_read_vsca(const char* path, uint32_t entry, vx_cache** out);
int vx_cache_desc(const vx_cache* cache, vx_scene_desc* desc);
/* The same scene with the material words of a VSCA file's brickData as its
 * colour (VX_COLOR_MATERIAL): the uncompressed shader's colour source
 * (VoxelRayMarch.comp:188-192).  vx_cache_desc gives the file's DXT1 colours
 * when it has them and the material words otherwise.  VX_EINVAL when the
 * cache holds no material words (VXSC files of other colour kinds). */
int vx_cache_desc_materials(const vx_cache* cache, vx_scene_desc* desc);
int vx_cache_free(vx_cache* cache);
/* vx_scene_download + vx_cache_write, and vx_cache_read + vx_scene_create. */
int vx_scene_save(const vx_scene* scene, const char* path);
int vx_scene_load(const char* path, vx_scene** out);

/* Device scene builder: the arrays of vx_build_dense, index for index, built
 * on the current device from R^3 occupancy bits already in device memory
 * (bits_dev, layout of vx_build_dense, R a multiple of 64 up to 4096), written
 * straight into a new scene.  color_kind VX_COLOR_RGBA8 / VX_COLOR_DXT1 adds
 * the payload of vx_synth_rgba8 / vx_synth_dxt1 for color_seed; with_normals
 * adds the DXT normal payload of vx_build_normals.  Allocates its own scratch
 * and returns when the scene is complete. */
int vx_scene_create_dense_dev(const uint64_t* bits_dev, uint32_t R, int32_t max_levels,
                              int32_t color_kind, uint64_t color_seed, int32_t with_normals,
                              vx_scene** out, void* stream);

/* ------------------------------------------------------------------------
 * Ray casting.  Replaces LaineKarrasOctree::castRay
 * (SVO/src/SVOTraversal.cpp:189-196, castRayImpl :516-691, brick DDA
 * SVOBrickDDA.cpp:65-533) for a batch of rays, with identical results.
 * t_min / t_max clip the ray like castRay's tMin / tMax.
 * counters_dev and color_dev may be NULL.  color_dev receives, per ray, the
 * hit voxel's RGBA8 word (u32) for VX_COLOR_RGBA8 scenes, its material word
 * (u32) for VX_COLOR_MATERIAL scenes, or its decoded DXT1
 * texel (3 floats, DXT1ColorCompressor::decodeColorHead,
 * VoxelData/src/Compression/DXT1Compressor.cpp:14-36) for VX_COLOR_DXT1 scenes;
 * misses leave zeros.
 * --------------------------------------------------------------------- */
int vx_cast_rays(const vx_scene* scene, const vx_ray* rays_dev, uint32_t n,
                 float t_min, float t_max, vx_hit* hits_dev, void* color_dev,
                 vx_ray_counters* counters_dev, void* stream);

/* Same with host buffers: copies rays in, casts, copies hits (and colours)
 * out, and returns after the results are in host memory. */
int vx_cast_rays_host(const vx_scene* scene, const vx_ray* rays_host, uint32_t n,
                      float t_min, float t_max, vx_hit* hits_host, void* color_host,
                      void* stream);

/* Normalised DXT normal of each hit voxel (getCompressedVoxelNormal,
 * VoxelRayMarch_Compressed.comp:160-165): normals_dev gets n x 3 floats,
 * zeros for misses and LOD hits.  The scene needs a normal payload. */
int vx_hit_normals(const vx_scene* scene, const vx_hit* hits_dev, uint32_t n, float* normals_dev,
                   void* stream);

/* ------------------------------------------------------------------------
 * Screen-space LOD cut.  Replaces LaineKarrasOctree::castRayWithLOD /
 * castRayScreenSpaceLOD / castRayLOD (SVO/src/SVOTraversal.cpp:198-232, the
 * termination test :613-651) and LODParameters (SVO/include/SVOLOD.h:50-177).
 * Every processed child cell whose entry distance d satisfies
 * d * ray_dir_size + ray_orig_size >= cell size ends the ray with an LOD hit:
 * t = d, flags = VX_HIT_HIT with the +y normal, brick 0xFFFFFFFF, voxel
 * 0xFFFF, node = the parent descriptor of the cell, scale = the cell's user
 * scale (esvoToUserScale, LaineKarrasOctree.h:381-383); colour zeros.
 * ray_dir_size <= 0 disables the cut (results equal vx_cast_rays).
 * castRayLOD(bias) is {0, bias}; castRayScreenSpaceLOD(fovY, H) is
 * vx_lod_from_camera(fovY, H, 0).
 * --------------------------------------------------------------------- */
typedef struct vx_lod_params {
    float ray_orig_size;  /* cone diameter at the ray origin, world units */
    float ray_dir_size;   /* cone diameter growth per unit distance */
} vx_lod_params;

/* LODParameters::fromCameraWithNearPlane (near_plane = 0: fromCamera),
 * SVOLOD.h:83-119: ray_dir_size = 2 tan(fov_y / screen_height / 2),
 * ray_orig_size = near_plane * ray_dir_size.  Host arithmetic. */
int vx_lod_from_camera(float fov_y, int32_t screen_height, float near_plane, vx_lod_params* out);
/* LODParameters::withBias (SVOLOD.h:169-176): both sizes times 2^bias. */
int vx_lod_with_bias(const vx_lod_params* in, float bias, vx_lod_params* out);

int vx_cast_rays_lod(const vx_scene* scene, const vx_ray* rays_dev, uint32_t n,
                     float t_min, float t_max, const vx_lod_params* lod, vx_hit* hits_dev,
                     void* color_dev, vx_ray_counters* counters_dev, void* stream);
int vx_cast_rays_host_lod(const vx_scene* scene, const vx_ray* rays_host, uint32_t n,
                          float t_min, float t_max, const vx_lod_params* lod, vx_hit* hits_host,
                          void* color_host, void* stream);

/* ------------------------------------------------------------------------
 * Frame render.  Replaces ComputeDispatchNode's
 * vkCmdDispatch((W+7)/8,(H+7)/8,1) of VoxelRayMarch[_Compressed].comp
 * (RenderGraph/src/Nodes/ComputeDispatchNode.cpp:249-317) with the
 * swapchain image replaced by a headless device buffer: one primary ray per
 * pixel (RayGeneration.glsl:61-71), the cast above, and Lambert shading
 * (Lighting.glsl:19-28) or the sky colour on a miss.  image_dev: W*H RGBA8
 * (row-major, row 0 at the top), may be NULL; hits_dev / color_dev optional.
 * --------------------------------------------------------------------- */
int vx_render(const vx_scene* scene, const vx_camera_pc* pc, uint32_t width,
              uint32_t height, uint32_t* image_dev, vx_hit* hits_dev,
              void* color_dev, void* stream);

/* Primary rays of a camera exactly as vx_render generates them. */
int vx_camera_rays(const vx_camera_pc* pc, uint32_t width, uint32_t height,
                   vx_ray* rays_host);
int vx_camera_rays_dev(const vx_camera_pc* pc, uint32_t width, uint32_t height,
                       vx_ray* rays_dev, void* stream);

/* ------------------------------------------------------------------------
 * Batched form (no reference counterpart).  One persistent launch casts the
 * rays of many scenes: rays of scene i are rays[begin[i] .. begin[i+1]) of
 * one buffer (begin: count + 1 device u32, begin[0] = 0, begin[count] = n).
 * Hits are identical to vx_cast_rays on each scene.  Warps take tasks of
 * `rays_per_task` consecutive rays from a work counter the batch owns, so
 * calls on one batch must not overlap on the GPU.
 * --------------------------------------------------------------------- */
typedef struct vx_batch vx_batch;
typedef struct vx_batch_tuning {
    int32_t block;            /* 128 or 256 threads */
    int32_t rays_per_task;    /* multiple of 32 */
    int32_t stack_in_shared;  /* 1: traversal stack in shared memory, 0: in local memory */
    int32_t refill;           /* 0: each lane casts its rays of a task start to end;
                                 1..32: lanes advance one ESVO iteration per round and the
                                 warp deals new rays to idle lanes once this many are idle */
    int32_t budget;           /* refill 0 only.  0: none; 1..500: a ray still running after this
                                 many ESVO iterations is set aside, and a second launch casts the
                                 set-aside rays from the start (a warp otherwise waits for its
                                 longest ray).  Same results; the batch holds a list of n u32,
                                 allocated on the first call with a larger n (outside a capture:
                                 cast once before capturing by hand) */
} vx_batch_tuning;

int vx_batch_create(const vx_scene* const* scenes, uint32_t count, vx_batch** out);
int vx_batch_destroy(vx_batch* batch);
int vx_batch_set_tuning(vx_batch* batch, const vx_batch_tuning* tuning);
int vx_batch_get_tuning(const vx_batch* batch, vx_batch_tuning* tuning);
int vx_cast_batch(vx_batch* batch, const vx_ray* rays_dev, const uint32_t* begin_dev, uint32_t n,
                  float t_min, float t_max, vx_hit* hits_dev, vx_ray_counters* counters_dev,
                  void* stream);
/* Times every (block, rays_per_task, stack placement, refill, budget)
 * candidate on the given rays (3 calls each, best of the last 2), keeps the
 * fastest in the batch and returns it.  Writes hits_dev. */
int vx_batch_autotune(vx_batch* batch, const vx_ray* rays_dev, const uint32_t* begin_dev, uint32_t n,
                      vx_hit* hits_dev, void* stream, vx_batch_tuning* best, float* best_ms);

/* The batched cast without any device allocation.  No counterpart in the
 * reference.  For callers that cannot allocate device memory: an application
 * that owns a fixed device-memory budget, or a frame loop where cudaMalloc's
 * implicit device synchronisation is not acceptable.  Takes the scenes
 * directly (no vx_batch) and keeps its scratch -- the task counter and a copy
 * of the scene table -- in a static device array of VX_NOALLOC_SCRATCH_BYTES
 * that every device loading the library holds until exit; count above
 * VX_NOALLOC_MAX_SCENES is rejected (VX_EOVERFLOW).  The first call on a
 * device resolves the array's address and the launch shape; make that first
 * call before any stream capture.  Every call shares the one array: the call
 * rewrites the table and clears the counter on its stream (the table goes to
 * a one-block staging kernel as a launch parameter, so the call copies nothing
 * from host memory and does not wait on the stream), and calls that overlap on
 * the GPU race.  Uses block 256, 32 rays per task, stack in shared memory;
 * hits are identical to vx_cast_batch. */
#define VX_NOALLOC_MAX_SCENES 64
#define VX_NOALLOC_SCRATCH_BYTES 16384
int vx_cast_batch_noalloc(const vx_scene* const* scenes, uint32_t count, const vx_ray* rays_dev,
                          const uint32_t* begin_dev, uint32_t n, float t_min, float t_max,
                          vx_hit* hits_dev, void* stream);

/* Secondary rays from primary hits.  Bounce: 2 rays per primary ray (out:
 * 2n), origin = hit point + 1e-3 * normal (hit point = origin +
 * normalize(dir) * t), direction = a cosine-weighted hemisphere sample about
 * the normal from a fixed 4096-entry table (vx_bounce_table), chosen by a
 * hash of (seed, ray index, k).  Shadow: 1 ray per primary ray toward
 * light_dir.  Misses produce zero-direction rays, which a cast reports as
 * VX_RAY_INVALID. */
int vx_spawn_bounce_rays(const vx_ray* rays_dev, const vx_hit* hits_dev, uint32_t n, uint64_t seed,
                         vx_ray* out_dev, void* stream);
int vx_spawn_shadow_rays(const vx_ray* rays_dev, const vx_hit* hits_dev, uint32_t n,
                         const float light_dir[3], vx_ray* out_dev, void* stream);
int vx_bounce_table(float* out /* 4096 x 3 */);

/* The shadow pass of a frame in one call: for every primary ray i with a hit,
 * the shadow ray toward light_dir (vx_spawn_shadow_rays' ray), cast in
 * [t_min, t_max]; shadow_hits_dev[i] receives exactly what
 * vx_spawn_shadow_rays followed by vx_cast_rays over all n slots writes (the
 * invalid-ray record for primary misses, whose shadow rays have no
 * direction).  Only the rays of hits are cast: they are compacted on the
 * device first.  No reference counterpart (the reference's shaders trace no
 * secondary rays).  Uses scratch held by the scene (about 28 bytes per
 * primary ray, allocated on the first call and when n grows); calls on the
 * same scene that overlap on the GPU race on it. */
int vx_cast_shadow_rays(const vx_scene* scene, const vx_ray* rays_dev, const vx_hit* hits_dev, uint32_t n,
                        const float light_dir[3], float t_min, float t_max, vx_hit* shadow_hits_dev,
                        void* stream);

/* One frame as a CUDA graph: batched primary cast, bounce spawn, batched
 * bounce cast (bounce_begin = 2 x primary begin).  Capture needs a
 * non-default stream; launch replays it on any stream. */
int vx_batch_capture_frame(vx_batch* batch, const vx_ray* primary_dev, const uint32_t* primary_begin_dev,
                           uint32_t n, vx_hit* primary_hits_dev, vx_ray* bounce_dev,
                           const uint32_t* bounce_begin_dev, vx_hit* bounce_hits_dev, uint64_t seed,
                           void* stream);
/* The same frame with the bounce rays compacted: the bounce pass casts only
 * the 2 rays of every primary hit.  bounce_dev (2n rays of scratch) receives
 * them, 2h of them for h primary hits, per scene grouped by direction bin
 * (the octant and the order of the three axes by |d|: 48 bins); inside a
 * group chunk by chunk of 1024 primary rays of the scene, inside a chunk the
 * first bounce rays in primary order, then the second ones (the same order on
 * every launch).  The frame computes the per-scene offsets itself.  primary_begin_dev is read once, at
 * capture (it must run from 0 to n and not decrease).  bounce_hits_dev (2n records) ends up exactly as
 * with vx_batch_capture_frame: slot 2i + k holds bounce k of primary ray i,
 * and the slots of primary misses hold the invalid-ray record a cast writes
 * for their zero-direction rays.  Scratch of about 8n bytes is allocated at
 * capture time (the first capture, or a larger n). */
int vx_batch_capture_frame_compact(vx_batch* batch, const vx_ray* primary_dev, const uint32_t* primary_begin_dev,
                                   uint32_t n, vx_hit* primary_hits_dev, vx_ray* bounce_dev,
                                   vx_hit* bounce_hits_dev, uint64_t seed, void* stream);
int vx_batch_launch_frame(vx_batch* batch, void* stream);
/* The captured frame from host buffers: copies n primary rays in (into the
 * primary buffer the frame was captured with), replays the frame, copies the
 * n primary hits out while the bounce pass runs and the 2n bounce hits out
 * after it, and returns when every result is in host memory.  Pinned host
 * buffers let the copies run at full link speed. */
int vx_batch_launch_frame_host(vx_batch* batch, const vx_ray* primary_host, vx_hit* primary_hits_host,
                               vx_hit* bounce_hits_host, void* stream);
/* The frame of vx_batch_capture_frame_compact, captured as `parts` pieces
 * with a graph each: piece k casts the primary rays [k n / parts,
 * (k + 1) n / parts) of the frame (a piece may begin or end inside a scene)
 * and the bounce rays of their hits.  primary_hits_dev and bounce_hits_dev
 * end up exactly as with the whole frame (bounce directions follow the frame's
 * ray index); each piece compacts its bounce rays into its own range
 * bounce_dev[2 r0 .. 2 r1).  vx_batch_launch_frame replays the pieces in order,
 * the even ones on its stream and the odd ones on a stream of the batch, so
 * that one piece's kernels start while the previous piece's drain, and makes
 * its stream wait for both; vx_batch_launch_frame_host does the same and
 * overlaps the pieces with the copies: the rays of every piece go in on a
 * copy stream, piece k casts once its rays are in, and its primary and bounce
 * hits go out on a second copy stream once it is done, while the next pieces
 * cast.  vx_batch_frame_compaction returns
 * VX_EINVAL for such a frame.  Scratch: that of the compacted frame, per
 * piece. */
int vx_batch_capture_frame_parts(vx_batch* batch, const vx_ray* primary_dev, const uint32_t* primary_begin_dev,
                                 uint32_t n, vx_hit* primary_hits_dev, vx_ray* bounce_dev, vx_hit* bounce_hits_dev,
                                 uint64_t seed, uint32_t parts, void* stream);
/* Layout of a compacted frame after it has run: the compacted bounce rays of
 * scene s are bounce_dev[scene_begin[s] .. scene_begin[s + 1]) (count + 1 host
 * u32), and compacted ray j's record is bounce_hits_dev[map[j]] (map_host:
 * scene_begin[count] host u32).  Synchronous reads; any pointer may be NULL.
 * cbegin_dev / map_dev receive the device addresses of those arrays, valid
 * until the next capture. */
int vx_batch_frame_compaction(const vx_batch* batch, uint32_t* scene_begin, uint32_t* map_host,
                              const uint32_t** cbegin_dev, const uint32_t** map_dev);
/* Tuning of the bounce pass of a captured frame (default, or after a null
 * tuning: the batch's own).  Incoherent bounce rays favour other shapes than
 * camera rays: autotune each pass on its own rays.  Applies to later captures. */
int vx_batch_set_bounce_tuning(vx_batch* batch, const vx_batch_tuning* tuning);

/* ------------------------------------------------------------------------
 * Differentiable form (no reference counterpart).  The traversal is discrete
 * and not differentiated: the forward pass records each pixel's hit (the
 * vx_hit of the cast) and the backward pass replays it.  Attributes are FP32:
 *   VX_DIFF_VOXEL_RGB:      attr[(brick*512 + voxel)*3 + c], 3 floats per voxel
 *   VX_DIFF_DXT1_ENDPOINTS: attr[block*6 + 0..2] = e0, [block*6 + 3..5] = e1
 *                           per DXT1 block (block = brick*32 + voxel/16), with
 *                           the fixed 2-bit selectors idx[block]; texel =
 *                           w0*e0 + w1*e1, (w0,w1) = (1,0),(0,1),(2/3,1/3),(1/3,2/3)
 * Pixel of a hit = texel * (0.3 + max(n.L, 0) * 0.7) (Lighting.glsl:19-28);
 * a miss shows the sky colour.  image: W*H*3 floats, record: W*H vx_hit.
 * Backward: loss = sum (image - target)^2 over pixels and channels (added to
 * *loss_dev if not NULL); dL/dattr is ADDED to grad_dev (same layout as attr;
 * zero it first) with warp-aggregated atomics.
 * --------------------------------------------------------------------- */
#define VX_DIFF_VOXEL_RGB 0
#define VX_DIFF_DXT1_ENDPOINTS 1
int vx_diff_forward(const vx_scene* scene, const vx_camera_pc* pc, uint32_t width, uint32_t height,
                    int32_t kind, const float* attr_dev, const uint32_t* dxt_idx_dev, float* image_dev,
                    vx_hit* record_dev, void* stream);
/* The forward pass of `views` cameras in one launch (better filled than one
 * launch per view): image_dev and record_dev are view-major (view v's pixels
 * start at v * width * height); vx_diff_backward then takes all of them with
 * n = views * width * height.  views <= VX_DIFF_MAX_VIEWS. */
#define VX_DIFF_MAX_VIEWS 64
int vx_diff_forward_views(const vx_scene* scene, const vx_camera_pc* pcs, uint32_t views,
                          uint32_t width, uint32_t height, int32_t kind, const float* attr_dev,
                          const uint32_t* dxt_idx_dev, float* image_dev, vx_hit* record_dev,
                          void* stream);
int vx_diff_backward(uint32_t n, int32_t kind, const uint32_t* dxt_idx_dev, const vx_hit* record_dev,
                     const float* image_dev, const float* target_dev, float* grad_dev, float* loss_dev,
                     void* stream);

/* ------------------------------------------------------------------------
 * Host scene builder.  Replaces LaineKarrasOctree::rebuild
 * (SVO/src/SVORebuild.cpp:228-607) plus VoxelSceneCacher::BuildOctree /
 * BuildBrickGridLookup (VoxelSceneCacher.cpp:463-713) for a dense occupancy
 * grid with world bounds [0,R]^3: same brick order (Morton rank), same
 * descriptor order (BFS, non-leaf children first), same lookup table.
 * Input: R^3 occupancy bits, x fastest, 64 voxels per u64 word (R a multiple
 * of 64).  The result owns host arrays exposed through a vx_scene_desc.
 * --------------------------------------------------------------------- */
typedef struct vx_build vx_build;
int vx_build_dense(const uint64_t* occupancy_bits, uint32_t R, int32_t max_levels,
                   vx_build** out);
/* Fills desc with pointers into the build (valid until vx_build_free);
 * colour fields are left empty. */
int vx_build_desc(const vx_build* build, vx_scene_desc* desc);
int vx_build_free(vx_build* build);

/* DXT normal payload of bricks from their occupancy (16 u32 per brick, as
 * vx_scene_desc.brick_occ): the geometric normal of every voxel
 * (computeGeometricNormal, SVO/src/SVORebuild.cpp:145-193: central
 * difference of the brick's occupancy, outward), empty voxels (0,1,0), each
 * block of 16 encoded by DXTNormalCompressor::encodeBlockTyped
 * (DXT1Compressor.cpp:242-333), empty blocks {0,0} (SVORebuild.cpp:658-722).
 * out: brick_count x 32 x {blockA, blockB}.  The host form uses all host
 * threads; the device form (16-byte aligned buffers) is stream-ordered.
 * Both produce identical bits. */
int vx_build_normals(const uint32_t* brick_occ, uint32_t brick_count, uint64_t* out);
int vx_build_normals_dev(const uint32_t* brick_occ_dev, uint32_t brick_count, uint64_t* out_dev,
                         void* stream);

/* DXT1 colour payload of bricks from per-voxel colours (rgb: brick_count x
 * 512 x 3 floats, voxel z*64+y*8+x) and occupancy: empty voxels (0,0,0),
 * each block of 16 encoded by DXT1ColorCompressor::encodeBlockTyped
 * (DXT1Compressor.cpp:57-111), empty blocks 0 (SVORebuild.cpp:658-722).
 * out: brick_count x 32 u64, the layout of VX_COLOR_DXT1.  Host and device
 * forms produce identical bits. */
int vx_build_dxt1(const float* rgb, const uint32_t* brick_occ, uint32_t brick_count, uint64_t* out);
int vx_build_dxt1_dev(const float* rgb_dev, const uint32_t* brick_occ_dev, uint32_t brick_count,
                      uint64_t* out_dev, void* stream);

/* Per-voxel colours of material words for the DXT1 payload: rgb[3i..3i+2] =
 * MaterialIdToColor(words[i]) (SVO/src/SVORebuild.cpp:68-120, the colour the
 * reference's compressed payload is encoded from at :679-700; its ids 33-39
 * differ from the shader's getMaterialColor).  Feed the result to
 * vx_build_dxt1 / vx_build_dxt1_dev with the bricks' occupancy.  The host
 * form uses all host threads; both give identical bits. */
int vx_material_rgb(const uint32_t* words, uint64_t n, float* rgb);
int vx_material_rgb_dev(const uint32_t* words_dev, uint64_t n, float* rgb_dev, void* stream);

/* Converts reference-layout descriptors (64-bit ChildDescriptor,
 * SVOTypes.h:36-47: childPointer:15 far:1 valid:8 leaf:8 | brick:24 flags:8)
 * into vx_node + node_brick.  Far pointers are rejected (VX_EINVAL). */
int vx_nodes_from_reference(const uint64_t* ref_nodes, uint32_t n, vx_node* nodes,
                            uint32_t* node_brick);

/* ------------------------------------------------------------------------
 * Synthetic inputs (no reference counterpart; seeded, deterministic).
 * --------------------------------------------------------------------- */
/* Value-noise occupancy: lattice spacing `spacing` voxels, `octaves`
 * octaves (persistence 0.5, lacunarity 2), thresholded at the quantile that
 * leaves `fill` of the voxels solid; `shell` adds the one-voxel box shell.
 * out_bits: R^3/64 words.  Uses all host threads. */
int vx_synth_noise(uint32_t R, uint32_t spacing, uint32_t octaves, float fill,
                   uint64_t seed, int32_t shell, uint64_t* out_bits);
/* The same bits as vx_synth_noise, generated on the current device into
 * out_bits_dev (R <= 2048).  Allocates and frees its own scratch (the float
 * field and the lattice tables) and returns after the bits are written. */
int vx_synth_noise_dev(uint32_t R, uint32_t spacing, uint32_t octaves, float fill,
                       uint64_t seed, int32_t shell, uint64_t* out_bits_dev, void* stream);
/* Urban lattice: 32x32 blocks of pitch R/32 (block + street of max(1, R/256)
 * voxels: 8 at R = 2048), each a solid box of seeded height in [hmin, hmax]. */
int vx_synth_urban(uint32_t R, uint32_t hmin, uint32_t hmax, uint64_t seed,
                   uint64_t* out_bits);
/* Per-brick colour payloads keyed on brick grid coordinates (so they do not
 * depend on brick order): RGBA8 uniform per voxel, or DXT1 blocks with
 * uniform u32 head and index words. */
int vx_synth_rgba8(const uint32_t* brick_coord, uint32_t brick_count, uint64_t seed,
                   uint32_t* out);
int vx_synth_dxt1(const uint32_t* brick_coord, uint32_t brick_count, uint64_t seed,
                  uint64_t* out);

#ifdef __cplusplus
}
#endif

#endif /* VX_H */
