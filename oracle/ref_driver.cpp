/*
 * ref_driver.cpp — dispatch driver for the reference pin (oracle/_ref).
 *
 * TEST INFRASTRUCTURE ONLY.  Binds plain host arrays to the translated WGSL
 * shaders (oracle/_ref/ref_shaders.gen.hpp, generated from the reference's
 * shaders.js by wgsl2cpp.py) and runs their invocations in the order
 * FluidGPU.simFrame records them (fluid-gpu.js:648-684) and DiffuseGPU.step
 * (diffuse-gpu.js:148-166): one loop over global_invocation_id per
 * dispatchWorkgroups call, with the reference's workgroup counts
 * (wgP = ceil(active/64), wgG = ceil(grid/64), wgAdv = ceil(max/64), the
 * APPLY_HAND box in 4x4x4 groups).  With threads == 1 invocations run one at a
 * time in ascending id order; with threads > 1 a dispatch's invocations are
 * spread over OpenMP threads with hardware atomics (used only for timing the
 * reference on host cores; diffuse slot order is then unordered, as on a GPU).
 */
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "_ref/ref_shaders.gen.hpp"
#include "../include/mpm_types.h"

namespace wgsl_rt { bool g_parallel = false; }

using namespace wgsl_rt;

namespace {

const uint32_t WG = 64;  // config.js:2 WG_SIZE (desktop)

template <class F> void dispatch1d(uint32_t groups, int threads, F&& fn) {
    const int64_t n = (int64_t)groups * WG;
    if (threads > 1) {
        g_parallel = true;
#pragma omp parallel for schedule(static) num_threads(threads)
        for (int64_t g = 0; g < n; ++g) fn(vec3<u32>((u32)g, 0u, 0u));
        g_parallel = false;
    } else {
        for (int64_t g = 0; g < n; ++g) fn(vec3<u32>((u32)g, 0u, 0u));
    }
}

uint32_t ceil_div(uint64_t a, uint32_t b) { return (uint32_t)((a + b - 1) / b); }

template <class Dst> void set_uniform(Dst& dst, const void* src) {
    static_assert(sizeof(Dst) > 0, "");
    std::memcpy(&dst, src, sizeof(Dst));
}

}  // namespace

extern "C" {

int ref_abi_version(void) { return 1; }

/* One simFrame substep through the translated reference shaders. */
void ref_substep_f32(const mpm_params* P, const mpm_wall_params* W, const mpm_hand_params* hand,
                     const int32_t* hand_dims, float* pos, float* vel, float* aff, float* mass, float* dens,
                     int32_t* mv, int32_t* cm, float* mvf, float* cmf, const mpm_gen_params* gen,
                     const mpm_advect_params* adv, float* diffuse, uint32_t* free_list, int32_t* top,
                     int threads) {
    static_assert(sizeof(WGSL_CLEAR::Params) == sizeof(mpm_params), "Params");
    static_assert(sizeof(WGSL_G2P::WallParams) == sizeof(mpm_wall_params), "WallParams");
    static_assert(sizeof(WGSL_APPLY_HAND::HandParams) == sizeof(mpm_hand_params), "HandParams");
    static_assert(sizeof(WGSL_DIFFUSE_GENERATE::GenParams) == sizeof(mpm_gen_params), "GenParams");
    static_assert(sizeof(WGSL_DIFFUSE_ADVECT::AdvectParams) == sizeof(mpm_advect_params), "AdvectParams");
    static_assert(sizeof(WGSL_DIFFUSE_ADVECT::DiffuseParticle) == sizeof(mpm_diffuse_particle), "Diffuse");
    static_assert(sizeof(WGSL_COMPUTE_WEIGHTS::BaseWeights) == 60, "BaseWeights");

    const uint64_t G = (uint64_t)P->grid_X * P->grid_Y * P->grid_Z;
    const uint32_t wgP = ceil_div(P->particle_num, WG);
    const uint32_t wgG = ceil_div(G, WG);
    mpm_wall_params wz;
    if (!W) { std::memset(&wz, 0, sizeof wz); W = &wz; }
    std::vector<WGSL_COMPUTE_WEIGHTS::BaseWeights> weights(P->particle_num ? P->particle_num : 1);

    auto* pos4 = reinterpret_cast<vec4<f32>*>(pos);
    auto* vel4 = reinterpret_cast<vec4<f32>*>(vel);

    {   using namespace WGSL_CLEAR;
        set_uniform(params, P);
        cell_mv = reinterpret_cast<atomic<i32>*>(mv);
        cell_mass = reinterpret_cast<atomic<i32>*>(cm);
        dispatch1d(wgG, threads, [](vec3<u32> g) { main(g); });
    }
    {   using namespace WGSL_COMPUTE_WEIGHTS;
        set_uniform(params, P);
        particle_pos = pos4;
        out_weights = weights.data();
        dispatch1d(wgP, threads, [](vec3<u32> g) { main(g); });
    }
    {   using namespace WGSL_P2G_MASS;
        set_uniform(params, P);
        particle_mass = mass;
        cell_mass = reinterpret_cast<atomic<i32>*>(cm);
        WGSL_P2G_MASS::weights = reinterpret_cast<BaseWeights*>(weights.data());
        dispatch1d(wgP, threads, [](vec3<u32> g) { main(g); });
    }
    {   using namespace WGSL_DECODE_MASS;
        set_uniform(params, P);
        cell_mass = reinterpret_cast<atomic<i32>*>(cm);
        cell_mass_f32 = cmf;
        dispatch1d(wgG, threads, [](vec3<u32> g) { main(g); });
    }
    {   using namespace WGSL_P2G_MOM;
        set_uniform(params, P);
        particle_vel = vel4;
        particle_affine = aff;
        particle_mass = mass;
        cell_mass_f32 = cmf;
        cell_mv = reinterpret_cast<atomic<i32>*>(mv);
        particle_density = dens;
        WGSL_P2G_MOM::weights = reinterpret_cast<BaseWeights*>(weights.data());
        dispatch1d(wgP, threads, [](vec3<u32> g) { main(g); });
    }
    {   using namespace WGSL_UPDATE_GRID;
        set_uniform(params, P);
        set_uniform(wallp, W);
        cell_mv = reinterpret_cast<atomic<i32>*>(mv);
        cell_mass = reinterpret_cast<atomic<i32>*>(cm);
        cell_mv_f32 = mvf;
        dispatch1d(wgG, threads, [](vec3<u32> g) { main(g); });
    }
    if (hand && hand_dims) {   // fluid-gpu.js:670-679
        using namespace WGSL_APPLY_HAND;
        const uint32_t gx = ceil_div(hand_dims[0] > 0 ? hand_dims[0] : 0, 4);
        const uint32_t gy = ceil_div(hand_dims[1] > 0 ? hand_dims[1] : 0, 4);
        const uint32_t gz = ceil_div(hand_dims[2] > 0 ? hand_dims[2] : 0, 4);
        if (gx > 0 && gy > 0 && gz > 0) {
            set_uniform(params, P);
            set_uniform(WGSL_APPLY_HAND::hand, hand);
            cell_mv_f32 = mvf;
            for (uint32_t z = 0; z < gz * 4; ++z)
                for (uint32_t y = 0; y < gy * 4; ++y)
                    for (uint32_t x = 0; x < gx * 4; ++x) main(vec3<u32>(x, y, z));
        }
    }
    {   using namespace WGSL_G2P;
        set_uniform(params, P);
        set_uniform(wallp, W);
        particle_pos = pos4;
        particle_vel = vel4;
        particle_affine = aff;
        cell_mv_f32 = mvf;
        WGSL_G2P::weights = reinterpret_cast<BaseWeights*>(weights.data());
        dispatch1d(wgP, threads, [](vec3<u32> g) { main(g); });
    }
    if (gen && adv && diffuse && free_list && top) {   // diffuse-gpu.js:148-166
        {   using namespace WGSL_DIFFUSE_GENERATE;
            set_uniform(params, P);
            set_uniform(WGSL_DIFFUSE_GENERATE::gen, gen);
            particle_pos = pos4;
            particle_vel = vel4;
            particle_mass = mass;
            particle_density = dens;
            cell_mass_f32 = cmf;
            diffuse_particles = reinterpret_cast<DiffuseParticle*>(diffuse);
            WGSL_DIFFUSE_GENERATE::free_list = free_list;
            free_list_top.v = *top;
            dispatch1d(wgP, threads, [](vec3<u32> g) { main(g); });
            *top = free_list_top.v;
        }
        {   using namespace WGSL_DIFFUSE_ADVECT;
            set_uniform(params, P);
            set_uniform(WGSL_DIFFUSE_ADVECT::adv, adv);
            set_uniform(wallp, W);
            diffuse_particles = reinterpret_cast<DiffuseParticle*>(diffuse);
            cell_mv_f32 = mvf;
            WGSL_DIFFUSE_ADVECT::free_list = free_list;
            free_list_top.v = *top;
            dispatch1d(ceil_div(adv->diffuse_max, WG), threads, [](vec3<u32> g) { main(g); });
            *top = free_list_top.v;
        }
    }
}

/* COMPACT (fluid-gpu.js:549-573): survivors in dispatch order; returns count. */
uint32_t ref_compact_f32(const mpm_params* P, const mpm_ray_params* del, const float* pos_in,
                         const float* vel_in, const float* mass_in, float* pos_out, float* vel_out,
                         float* mass_out) {
    using namespace WGSL_COMPACT;
    set_uniform(params, P);
    set_uniform(WGSL_COMPACT::del, del);
    WGSL_COMPACT::pos_in = reinterpret_cast<vec4<f32>*>(const_cast<float*>(pos_in));
    WGSL_COMPACT::vel_in = reinterpret_cast<vec4<f32>*>(const_cast<float*>(vel_in));
    WGSL_COMPACT::mass_in = const_cast<float*>(mass_in);
    WGSL_COMPACT::pos_out = reinterpret_cast<vec4<f32>*>(pos_out);
    WGSL_COMPACT::vel_out = reinterpret_cast<vec4<f32>*>(vel_out);
    WGSL_COMPACT::mass_out = mass_out;
    counter.v = 0;
    dispatch1d(ceil_div(P->particle_num, WG), 1, [](vec3<u32> g) { main(g); });
    return counter.v;
}

/* RAYCAST (fluid-gpu.js:594-616): hit_t starts at 0xFFFFFFFF. */
uint32_t ref_raycast_f32(const mpm_params* P, const mpm_ray_params* ray, const float* pos_in) {
    using namespace WGSL_RAYCAST;
    set_uniform(params, P);
    set_uniform(WGSL_RAYCAST::ray, ray);
    WGSL_RAYCAST::pos_in = reinterpret_cast<vec4<f32>*>(const_cast<float*>(pos_in));
    hit_t.v = 0xFFFFFFFFu;
    dispatch1d(ceil_div(P->particle_num, WG), 1, [](vec3<u32> g) { main(g); });
    return hit_t.v;
}

}  // extern "C"
