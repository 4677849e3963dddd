/*
 * mpm_types.h — plain-C mirrors of the reference's GPU uniform / storage structs.
 *
 * Every struct here is byte-for-byte the layout the reference uploads with
 * queue.writeBuffer, so a host that already packs these (fluid-gpu.js,
 * diffuse-gpu.js) can hand the same bytes to the C ABI unchanged.
 * Sizes are checked with static asserts in the library and in the tests.
 */
#ifndef MPM_TYPES_H
#define MPM_TYPES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* config.js:11 — capacity of the wall uniform. */
#define MPM_MAX_WALLS 4
/* config.js:7 — default diffuse pool size (desktop). */
#define MPM_DIFFUSE_MAX_COUNT_DEFAULT 30000
/* shaders.js:5 — floor spring band (cells), baked into G2P. */
#define MPM_FLOOR_SPRING_BAND 3.0f

/* Params uniform, 80 B: shaders.js:27-49; packed by fluid-gpu.js:295-313. */
typedef struct mpm_params {
    uint32_t grid_X, grid_Y, grid_Z, particle_num;
    float dt, gravity, rest_density, stiffness, eos_power, viscosity;
    float hard_min, hard_max_x, hard_max_y, hard_max_z;
    float wall_min, wall_stiffness, lookahead_k;
    float _pad0, _pad1, _pad2;
} mpm_params;

/* One moving-wall OBB, 80 B: shaders.js:123-129. */
typedef struct mpm_wall {
    float center_cy[4];   /* xyz centre, w = cos(yaw)          */
    float lmin_sy[4];     /* xyz local min, w = sin(yaw)       */
    float lmax_cp[4];     /* xyz local max, w = cos(pitch)     */
    float vel_sp[4];      /* xyz linear velocity, w = sin(pitch) */
    float omega_pad[4];   /* xyz angular velocity               */
} mpm_wall;

/* WallParams uniform, 16 + 4*80 = 336 B: shaders.js:130-133; packed by
 * fluid-gpu.js:337-413 (active walls packed first, count in count_pad[0]). */
typedef struct mpm_wall_params {
    float count_pad[4];
    mpm_wall walls[MPM_MAX_WALLS];
} mpm_wall_params;

/* HandParams uniform, 80 B: shaders.js:395-402; packed by fluid-gpu.js:479-527. */
typedef struct mpm_hand_params {
    float px, py, pz, radius;
    float vx, vy, vz;
    uint32_t is_on;
    float strength, ex, ey, ez;
    int32_t bbox_min_x, bbox_min_y, bbox_min_z;
    int32_t bbox_max_x, bbox_max_y, bbox_max_z;
    int32_t _pad0, _pad1;
} mpm_hand_params;

/* GenParams uniform, 32 B: shaders.js:734-743; packed by diffuse-gpu.js:84-94. */
typedef struct mpm_gen_params {
    float ke_threshold, spawn_rate_k, density_spray_max, density_bubble_min;
    float lifetime_foam, pressure_threshold, crest_dot_threshold;
    uint32_t seed;
} mpm_gen_params;

/* AdvectParams uniform, 16 B: shaders.js:872-877; packed by diffuse-gpu.js:70-76. */
typedef struct mpm_advect_params {
    uint32_t diffuse_max;
    float buoyancy, drag, _pad;
} mpm_advect_params;

/* DiffuseParticle storage element, 48 B: shaders.js:725-732, diffuse-gpu.js:5. */
typedef struct mpm_diffuse_particle {
    float pos[4];
    float vel[4];
    uint32_t ptype;   /* 0 spray, 1 foam, 2 bubble (shaders.js:859-861) */
    uint32_t alive;
    float lifetime;
    float _pad;
} mpm_diffuse_particle;

/* RayParams uniform, 32 B: shaders.js:78 (delete cylinder / raycast). */
typedef struct mpm_ray_params {
    float ox, oy, oz, radius;
    float dx, dy, dz, _pad;
} mpm_ray_params;

#define MPM_DIFFUSE_SPRAY  0u
#define MPM_DIFFUSE_FOAM   1u
#define MPM_DIFFUSE_BUBBLE 2u

#ifdef __cplusplus
}
#endif

#endif /* MPM_TYPES_H */
