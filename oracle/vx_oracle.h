/*
 * vx_oracle.h - C interface of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a line-by-line CPU restatement of
 * the reference's octree rebuild (VIXEN/libraries/SVO/src/SVORebuild.cpp),
 * ray cast (VIXEN/libraries/SVO/src/SVOTraversal.cpp, SVOBrickDDA.cpp) and
 * DXT1 colour codec (VIXEN/libraries/VoxelData/src/Compression/DXT1Compressor.cpp).
 * Only tests, the smoke check and the CPU-baseline leg of the benchmark may
 * load it; the product library never links or calls it.
 *
 * Parity status: pinned to the reference's own code.  `make -C oracle ref`
 * compiles the reference's rebuild, castRay / castRayWithLOD, brick DDA and
 * rebuild payload encoders from its sources, with stand-ins for glm and
 * gaia-ecs (not installed here; oracle/ref_shim/), and tests/test_ref_pin.py
 * requires this restatement to give the same bits on the same voxels and
 * rays.  It is also held to the reference's behavioural tests (KATs in
 * tests/test_oracle_kat.py) and to golden vectors it generated itself.
 */
#ifndef VX_ORACLE_H
#define VX_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vxo_scene vxo_scene;

/* Hit record of the oracle (one per ray). */
typedef struct vxo_hit {
    float t;          /* RayHit::tMin  (SVOBrickDDA.cpp:506) */
    float t_exit;     /* RayHit::tMax  (SVOBrickDDA.cpp:507) */
    float hit_point[3];
    float normal[3];
    uint32_t brick;   /* brick-view index (Morton rank), 0xFFFFFFFF on miss */
    uint32_t node;    /* parent descriptor index at the leaf (SVOBrickDDA.cpp:77) */
    uint32_t voxel;   /* in-brick voxel index z*64+y*8+x, 0xFFFF on miss */
    int32_t key[3];   /* integer world position of the hit entity */
    int32_t scale;    /* RayHit::scale */
    uint32_t flags;   /* VX_HIT_* bits, same encoding as the product (vx.h) */
    uint32_t iters;   /* ESVO loop iterations */
    uint32_t grid_reads; /* brickGridLookup reads (position-based lookups) */
    uint32_t dda_steps;  /* DDA occupancy tests */
    uint32_t leaf_visits;
} vxo_hit;

/* Build from a list of integer voxel keys (world integer positions, as
 * MortonCode64::fromWorldPos would quantise them).  world_min/max are the
 * rebuild() bounds.  Returns NULL on error (message in err). */
vxo_scene* vxo_build_from_keys(const int32_t* keys_xyz, uint64_t n,
                               const float world_min[3], const float world_max[3],
                               int max_levels, int brick_depth,
                               char* err, int errlen);

/* Build from a dense occupancy bit grid of side R (x fastest, 64 voxels per
 * word, bit b of word w is voxel x = (w % (R/64))*64 + b).  World bounds are
 * [0,R]^3 as VoxelSceneCacher::BuildOctree uses (VoxelSceneCacher.cpp:521-522).
 * R must be a multiple of 64. */
vxo_scene* vxo_build_from_dense(const uint64_t* bits, int R, int max_levels,
                                int brick_depth, char* err, int errlen);

void vxo_free(vxo_scene* s);

uint32_t vxo_node_count(const vxo_scene* s);
uint32_t vxo_brick_count(const vxo_scene* s);
int32_t  vxo_bricks_per_axis(const vxo_scene* s);
uint32_t vxo_max_child_pointer(const vxo_scene* s);

/* Dump the octree in the product's device format (vx.h):
 * nodes: 2 u32 per descriptor {child_pointer, valid | leaf << 8};
 * node_brick: brick index field of every descriptor;
 * grid_lookup: bricks_per_axis^3 u32 (0xFFFFFFFF empty);
 * brick_coord: x | y<<10 | z<<20 per brick;
 * brick_occ: 16 u32 per brick, bit (i & 31) of word (i >> 5) for voxel i.
 * Any pointer may be NULL. */
void vxo_export(const vxo_scene* s, uint32_t* nodes, uint32_t* node_brick,
                uint32_t* grid_lookup, uint32_t* brick_coord, uint32_t* brick_occ);

/* castRay over n rays (6 floats each: origin, direction) with nthreads host
 * threads (<= 0: all hardware threads). */
void vxo_cast_rays(const vxo_scene* s, const float* rays, uint64_t n,
                   float t_min, float t_max, vxo_hit* out, int nthreads);

/* castRayWithLOD (SVOTraversal.cpp:198-232) with LODParameters {ray_orig_size,
 * ray_dir_size} (SVOLOD.h:50-177); ray_dir_size <= 0 is castRay.  A ray that
 * stops at the LOD cut is a hit with brick 0xFFFFFFFF, voxel 0xFFFF, normal
 * (0,1,0), scale = the cell's user scale and node = the parent descriptor. */
void vxo_cast_rays_lod(const vxo_scene* s, const float* rays, uint64_t n, float t_min, float t_max,
                       float ray_orig_size, float ray_dir_size, vxo_hit* out, int nthreads);

/* LODParameters::fromCameraWithNearPlane / fromCamera (near_plane = 0) and
 * withBias (SVOLOD.h:83-176); out = {rayOrigSize, rayDirSize}. */
void vxo_lod_from_camera(float fov_y, int32_t screen_height, float near_plane, float out[2]);
void vxo_lod_with_bias(const float in[2], float bias, float out[2]);

/* Same as vxo_cast_rays, but replaces the octree with hand-built descriptors
 * (test_octree_queries.cpp builds such octrees with setOctree()). */
vxo_scene* vxo_build_from_descriptors(const uint32_t* nodes, const uint32_t* node_brick,
                                      uint32_t node_count,
                                      const float world_min[3], const float world_max[3],
                                      int max_levels, int brick_depth);

/* DXT1 colour codec restatement (DXT1Compressor.cpp:14-130). */
void     vxo_dxt1_decode_head(uint32_t head, float ref[12]);
void     vxo_dxt1_decode_block(uint64_t block, float out[48]);
uint32_t vxo_dxt1_encode_head(const float c0[3], const float c1[3]);
uint64_t vxo_dxt1_encode_block(const float* colors, uint64_t valid_count,
                               const int32_t* indices);

/* Colour fetch of a hit, restating the compressed shader's addressing
 * (VoxelRayMarch_Compressed.comp:142-158): block = voxel >> 4, texel = voxel & 15. */
/* Seeded synthetic inputs of the benchmark frames (vx_oracle_synth.cpp): the
 * same bits as the product's vx_synth_noise / vx_synth_urban /
 * vx_bounce_table / vx_spawn_*_rays, computed without the product library.
 * threads = 0: all cores.  Return 0, or -1 on bad arguments. */
int vxo_synth_noise(uint32_t R, uint32_t spacing, uint32_t octaves, float fill, uint64_t seed, int32_t shell,
                    uint64_t* out, int threads);
int vxo_synth_urban(uint32_t R, uint32_t hmin, uint32_t hmax, uint64_t seed, uint64_t* out);
void vxo_bounce_table(float* out /* 4096 x 3 */);
/* Material colours: MaterialIdToColor (SVORebuild.cpp:68-120, the compressed
 * payload's source) and getMaterialColor (shaders/Materials.glsl:18-60, the
 * uncompressed shader's). */
void vxo_material_color_cpu(uint32_t id, float out[3]);
void vxo_material_color_shader(uint32_t id, float out[3]);
/* kind 0: 2 bounce rays per ray (out 2n x 6); kind 1: a shadow ray toward
 * light (out n x 6).  index: each ray's position in its frame (NULL: i). */
void vxo_spawn_rays(const float* rays, const vxo_hit* hits, const uint64_t* index, uint64_t n, int kind,
                    uint64_t seed, const float light[3], float* out);

/* Primary rays of a camera (VoxelRayMarch.comp:453-455, RayGeneration.glsl:61-71):
 * pc = the 64-byte push constants as 16 words; out: w*h x 6 floats, row-major
 * from the top row; uv_y (may be NULL): each pixel's uv.y. */
void vxo_camera_rays(const float pc[16], uint32_t w, uint32_t h, float* out, float* uv_y);
void vxo_hit_texel_dxt(const uint64_t* brick_dxt, uint32_t brick, uint32_t voxel, float out[3]);
void vxo_hit_texels_dxt(const uint64_t* brick_dxt, uint64_t n, const uint32_t* brick, const uint32_t* voxel,
                        float* out);

/* Lambert shading of a hit colour (Lighting.glsl:19-28) and the sky colour on
 * a miss (VoxelRayMarch.comp:493-499); returns RGBA8 like an UNORM imageStore. */
uint32_t vxo_shade(const float color[3], int hit, int normal_axis, int normal_neg, float uv_y);

/* DXT normal codec (DXTNormalCompressor, DXT1Compressor.cpp:168-354):
 * encode 16 normals (valid_count <= 16, indices may be NULL) into {blockA,
 * blockB}; decode the 16 unnormalised texels (Compression.glsl:158-177). */
void     vxo_dxtn_encode_block(const float* normals, uint64_t valid_count, const int32_t* indices,
                               uint64_t out[2]);
void     vxo_dxtn_decode_block(const uint64_t in[2], float out[48]);
uint32_t vxo_encode_raw_normal(const float n[3]);

/* Geometric normals of one brick's 512 voxels from its 16-word occupancy
 * (computeGeometricNormal, SVORebuild.cpp:145-193). */
void vxo_geometric_normals(const uint32_t* occ, float out[1536]);

/* DXT normal payload of brick_count bricks (SVORebuild.cpp:658-722):
 * 32 blocks x {blockA, blockB} per brick. */
void vxo_brick_normals(const uint32_t* occ, uint64_t brick_count, uint64_t* out, int nthreads);

/* DXT1 colour payload of brick_count bricks from per-voxel RGB (512 x 3
 * floats per brick) and occupancy (SVORebuild.cpp:658-722). */
void vxo_brick_dxt1(const float* rgb, const uint32_t* occ, uint64_t brick_count, uint64_t* out);

/* normalize(decodeDXTNormal) of a hit voxel (VoxelRayMarch_Compressed.comp:160-165). */
void vxo_hit_normal_dxt(const uint64_t* brick_nrm, uint32_t brick, uint32_t voxel, float out[3]);

/* Lighting with the decoded normal blended with the hit's entry-face normal:
 * normalize(n_dxt + face * 0.5) (VoxelRayMarch_Compressed.comp:242-256). */
uint32_t vxo_shade_dxt_normal(const float color[3], int hit, const float n_dxt[3], int normal_axis,
                              int normal_neg, float uv_y);

#ifdef __cplusplus
}
#endif

#endif
