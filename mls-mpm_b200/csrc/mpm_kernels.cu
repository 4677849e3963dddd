// mpm_kernels.cu — per-pass CUDA kernels of the MLS-MPM substep and the
// diffuse spray/foam update, one kernel per reference compute shader.
//
// Compiled with --fmad=false; see mpm_device.cuh for the numerics contract.
// Each kernel restates the WGSL shader named in its comment with the same
// loop order and operation order, so per-particle f32 results and i32 grid
// contributions are bit-identical to the reference's.  Grid accumulation uses
// 32-bit integer atomics, whose sum does not depend on the order of arrival.
//
// Memory safety: the reference leaves P2G_MOM's and G2P's stencil indices
// unchecked (shaders.js:303-304, 598-599) and relies on particles staying in
// [2, dim-2].  Here a linear stencil index outside the grid buffer is skipped
// (reads give 0, writes are dropped), which changes nothing for particles that
// keep the reference's invariant and never touches memory outside the buffer.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "mpm_device.cuh"
#include "mpm_kernels.h"

namespace mpm {

constexpr int kThreads = 256;

static inline uint32_t blocks_for(uint64_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

// ---------------------------------------------------------------------------
// P2G_MASS (shaders.js:242-274), weights of COMPUTE_WEIGHTS (shaders.js:216-240)
// recomputed in registers.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_p2g_mass(const float4* __restrict__ pos, const float* __restrict__ mass,
                                                        int32_t* __restrict__ cm, uint32_t n, int32_t X, int32_t Y,
                                                        int32_t Z) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const float4 q = pos[p];
    const float pm = mass[p];
    int32_t cx, cy, cz;
    float fx, fy, fz;
    cell_frac(q.x, cx, fx);
    cell_frac(q.y, cy, fy);
    cell_frac(q.z, cz, fz);
    float wx[3], wy[3], wz[3];
    qweights(fx, wx[0], wx[1], wx[2]);
    qweights(fy, wy[0], wy[1], wy[2]);
    qweights(fz, wz[0], wz[1], wz[2]);
    const int32_t bx = cx - 1, by = cy - 1, bz = cz - 1;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int32_t zz = bz + k;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int32_t yy = by + j;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int32_t xx = bx + i;
                if (xx < 0 || xx >= X || yy < 0 || yy >= Y || zz < 0 || zz >= Z) continue;
                const int32_t idx = (zz * Y + yy) * X + xx;
                const float w = wx[i] * wy[j] * wz[k];
                atomicAdd(&cm[idx], encode(w * pm));
            }
        }
    }
}

// DECODE_MASS (shaders.js:373-384)
__global__ void __launch_bounds__(kThreads) k_decode_mass(const int32_t* __restrict__ cm, float* __restrict__ cmf,
                                                           uint64_t G) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < G) cmf[i] = decode(cm[i]);
}

// ---------------------------------------------------------------------------
// P2G_MOM (shaders.js:276-371)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_p2g_mom(const float4* __restrict__ pos, const float4* __restrict__ vel,
                                                       const float* __restrict__ aff, const float* __restrict__ mass,
                                                       const float* __restrict__ cmf, int32_t* __restrict__ mv,
                                                       float* __restrict__ dens, const mpm_params P, uint32_t G) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P.particle_num) return;
    const float4 q = pos[p];
    const float4 v = vel[p];
    const float m = mass[p];
    const float* a = aff + 9ull * p;
    const float a00 = a[0], a01 = a[1], a02 = a[2], a10 = a[3], a11 = a[4], a12 = a[5], a20 = a[6], a21 = a[7],
                a22 = a[8];
    int32_t cx, cy, cz;
    float fx, fy, fz;
    cell_frac(q.x, cx, fx);
    cell_frac(q.y, cy, fy);
    cell_frac(q.z, cz, fz);
    float wx[3], wy[3], wz[3];
    qweights(fx, wx[0], wx[1], wx[2]);
    qweights(fy, wy[0], wy[1], wy[2]);
    qweights(fz, wz[0], wz[1], wz[2]);
    const uint32_t X = P.grid_X, Y = P.grid_Y;
    const uint32_t SLICE = X * Y;
    const uint32_t baseIdx = (uint32_t)(((cz - 1) * (int32_t)Y + (cy - 1)) * (int32_t)X + (cx - 1));

    float density = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)j * X + (uint32_t)i;
                const float cmass = cidx < G ? cmf[cidx] : 0.0f;
                density += wx[i] * wy[j] * wz[k] * cmass;
            }
    dens[p] = density;
    if (density <= 1e-8f) return;

    const float rest = P.rest_density;
    const float vol = __fdiv_rn(m, fmaxf(density, rest * 0.15f));
    float pressure = P.stiffness * (eos_pow(__fdiv_rn(density, rest), P.eos_power) - 1.0f);
    const float pFloor = density > rest * kCohesionGate ? kCohesionPressure : 0.0f;
    pressure = fmaxf(pressure, pFloor);
    const float visc = P.viscosity;
    const float s00 = -pressure + visc * (a00 + a00);
    const float s11 = -pressure + visc * (a11 + a11);
    const float s22 = -pressure + visc * (a22 + a22);
    const float s01 = visc * (a01 + a10);
    const float s02 = visc * (a02 + a20);
    const float s12 = visc * (a12 + a21);
    const float coef = -vol * 4.0f * P.dt;
    const float dxs[3] = {-fx - 1.0f, -fx, 1.0f - fx};
    const float dys[3] = {-fy - 1.0f, -fy, 1.0f - fy};
    const float dzs[3] = {-fz - 1.0f, -fz, 1.0f - fz};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float wzk = wz[k], dzk = dzs[k];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float wyzk = wy[j] * wzk, dyj = dys[j];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const float w = wx[i] * wyzk;
                const float dxi = dxs[i];
                const uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)j * X + (uint32_t)i;
                const float Qx = a00 * dxi + a01 * dyj + a02 * dzk;
                const float Qy = a10 * dxi + a11 * dyj + a12 * dzk;
                const float Qz = a20 * dxi + a21 * dyj + a22 * dzk;
                const float fxf = coef * (s00 * dxi + s01 * dyj + s02 * dzk);
                const float fyf = coef * (s01 * dxi + s11 * dyj + s12 * dzk);
                const float fzf = coef * (s02 * dxi + s12 * dyj + s22 * dzk);
                if (cidx < G) {
                    int32_t* c = mv + 3ull * cidx;
                    atomicAdd(c + 0, encode(w * (m * (v.x + Qx) + fxf)));
                    atomicAdd(c + 1, encode(w * (m * (v.y + Qy) + fyf)));
                    atomicAdd(c + 2, encode(w * (m * (v.z + Qz) + fzf)));
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// UPDATE_GRID (shaders.js:435-513)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_update_grid(const int32_t* __restrict__ mv,
                                                           const int32_t* __restrict__ cm, float* __restrict__ mvf,
                                                           const mpm_params P, const mpm_wall_params W) {
    const uint32_t X = P.grid_X, Y = P.grid_Y, Z = P.grid_Z;
    const uint64_t G = (uint64_t)X * Y * Z;
    const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= G) return;
    const float c = decode(cm[idx]);
    float* out = mvf + 3 * idx;
    if (c <= 0.0f) { out[0] = 0.0f; out[1] = 0.0f; out[2] = 0.0f; return; }
    float vx = __fdiv_rn(decode(mv[3 * idx + 0]), c);
    float vy = __fdiv_rn(decode(mv[3 * idx + 1]), c);
    float vz = __fdiv_rn(decode(mv[3 * idx + 2]), c);
    vy += P.gravity * P.dt;
    const int32_t cx = (int32_t)(idx % X);
    const int32_t cy = (int32_t)((idx / X) % Y);
    const int32_t cz = (int32_t)(idx / ((uint64_t)X * Y));
    if (cx < 2 || cx > (int32_t)X - 3) vx = 0.0f;
    if (cy < 2 && vy < 0.0f) vy = 0.0f;
    if (cy > (int32_t)Y - 3 && vy > 0.0f) vy = 0.0f;
    if (cz < 2 || cz > (int32_t)Z - 3) vz = 0.0f;
    if (cy < 2) { vx *= 0.85f; vz *= 0.9f; }
    const uint32_t nw = wall_count_of(W.count_pad[0]);
    if (nw > 0) {
        const f3 cellPos = mk(__int2float_rn(cx) + 0.5f, __int2float_rn(cy) + 0.5f, __int2float_rn(cz) + 0.5f);
        f3 wv = mk(vx, vy, vz);
        for (uint32_t wi = 0; wi < nw; ++wi) {
            const WallD w = load_wall(W.walls[wi]);
            const f3 lp = wall_to_local(cellPos, w);
            if (lp.x < w.mn.x - 1.0f || lp.y < w.mn.y - 1.0f || lp.z < w.mn.z - 1.0f || lp.x > w.mx.x + 1.0f ||
                lp.y > w.mx.y + 1.0f || lp.z > w.mx.z + 1.0f)
                continue;
            const f3 wvel = wall_vel_at(cellPos, w);
            f3 n;
            const float sw = wall_sdf_normal(lp, w.mn, w.mx, n);
            if (sw < 0.0f) {
                wv = wvel;
            } else if (sw < 1.0f) {
                const f3 nn = wall_to_world_dir(n, w);
                const f3 vrel = sub(wv, wvel);
                const float vn = dot3(vrel, nn);
                if (vn < 0.0f) wv = mk(wv.x - vn * nn.x, wv.y - vn * nn.y, wv.z - vn * nn.z);
            }
        }
        vx = wv.x; vy = wv.y; vz = wv.z;
    }
    out[0] = vx; out[1] = vy; out[2] = vz;
}

// ---------------------------------------------------------------------------
// APPLY_HAND (shaders.js:394-433): 4x4x4 groups over the CPU-computed box.
// ---------------------------------------------------------------------------
__global__ void k_apply_hand(float* __restrict__ mvf, const mpm_params P, const mpm_hand_params H) {
    if (H.is_on == 0u) return;
    const int32_t cx = H.bbox_min_x + (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
    const int32_t cy = H.bbox_min_y + (int32_t)(blockIdx.y * blockDim.y + threadIdx.y);
    const int32_t cz = H.bbox_min_z + (int32_t)(blockIdx.z * blockDim.z + threadIdx.z);
    if (cx > H.bbox_max_x || cy > H.bbox_max_y || cz > H.bbox_max_z) return;
    if (cx < 0 || cy < 0 || cz < 0 || cx >= (int32_t)P.grid_X || cy >= (int32_t)P.grid_Y || cz >= (int32_t)P.grid_Z)
        return;
    const uint32_t idx = (uint32_t)((cz * (int32_t)P.grid_Y + cy) * (int32_t)P.grid_X + cx);
    const f3 cell = mk(__int2float_rn(cx) + 0.5f, __int2float_rn(cy) + 0.5f, __int2float_rn(cz) + 0.5f);
    const f3 hp = mk(H.px, H.py, H.pz);
    const f3 dv = sub(hp, mk(H.ex, H.ey, H.ez));
    const float dl = len3(dv);
    const f3 dir = mk(__fdiv_rn(dv.x, dl), __fdiv_rn(dv.y, dl), __fdiv_rn(dv.z, dl));
    const f3 to_cell = sub(cell, hp);
    const float t0 = dot3(to_cell, dir);
    const f3 perp = mk(to_cell.x - t0 * dir.x, to_cell.y - t0 * dir.y, to_cell.z - t0 * dir.z);
    const float d = len3(perp);
    if (d >= H.radius) return;
    const float t = 1.0f - __fdiv_rn(d, H.radius);
    const float w = t * t * H.strength;
    mvf[idx * 3u + 0u] += H.vx * w;
    mvf[idx * 3u + 1u] += H.vy * w;
    mvf[idx * 3u + 2u] += H.vz * w;
}

// ---------------------------------------------------------------------------
// G2P (shaders.js:579-705)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_g2p(float4* __restrict__ pos, float4* __restrict__ vel,
                                                   float* __restrict__ aff, const float* __restrict__ mvf,
                                                   const mpm_params P, const mpm_wall_params W, uint32_t G) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P.particle_num) return;
    const float4 q = pos[p];
    int32_t cx, cy, cz;
    float fx, fy, fz;
    cell_frac(q.x, cx, fx);
    cell_frac(q.y, cy, fy);
    cell_frac(q.z, cz, fz);
    float wx[3], wy[3], wz[3];
    qweights(fx, wx[0], wx[1], wx[2]);
    qweights(fy, wy[0], wy[1], wy[2]);
    qweights(fz, wz[0], wz[1], wz[2]);
    const int32_t bx = cx - 1, by = cy - 1, bz = cz - 1;
    const uint32_t X = P.grid_X, Y = P.grid_Y;
    const uint32_t SLICE = X * Y;
    const uint32_t baseIdx = (uint32_t)((bz * (int32_t)Y + by) * (int32_t)X + bx);
    float gvx = 0.0f, gvy = 0.0f, gvz = 0.0f;
    float B00 = 0.0f, B01 = 0.0f, B02 = 0.0f, B10 = 0.0f, B11 = 0.0f, B12 = 0.0f, B20 = 0.0f, B21 = 0.0f, B22 = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float wzk = wz[k];
        const float dzk = __int2float_rn(bz + k) - q.z + 0.5f;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float wyzk = wy[j] * wzk;
            const float dyj = __int2float_rn(by + j) - q.y + 0.5f;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const float w = wx[i] * wyzk;
                const float dxi = __int2float_rn(bx + i) - q.x + 0.5f;
                const uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)j * X + (uint32_t)i;
                float cvx = 0.0f, cvy = 0.0f, cvz = 0.0f;
                if (cidx < G) {
                    const float* c = mvf + 3ull * cidx;
                    cvx = c[0]; cvy = c[1]; cvz = c[2];
                }
                const float wvx = w * cvx, wvy = w * cvy, wvz = w * cvz;
                gvx += wvx; gvy += wvy; gvz += wvz;
                B00 += wvx * dxi; B01 += wvx * dyj; B02 += wvx * dzk;
                B10 += wvy * dxi; B11 += wvy * dyj; B12 += wvy * dzk;
                B20 += wvz * dxi; B21 += wvz * dyj; B22 += wvz * dzk;
            }
        }
    }
    float* a = aff + 9ull * p;
    a[0] = B00 * 4.0f; a[1] = B01 * 4.0f; a[2] = B02 * 4.0f;
    a[3] = B10 * 4.0f; a[4] = B11 * 4.0f; a[5] = B12 * 4.0f;
    a[6] = B20 * 4.0f; a[7] = B21 * 4.0f; a[8] = B22 * 4.0f;

    const float dt = P.dt, lk = P.lookahead_k, ws = P.wall_stiffness;
    f3 np = mk(q.x + dt * gvx, q.y + dt * gvy, q.z + dt * gvz);
    f3 nv = mk(gvx, gvy, gvz);
    const float floorZoneY = P.hard_min + kFloorBand;
    const float xny = np.y + nv.y * dt * lk;
    if (xny < floorZoneY) {
        const float distBelowFloor = floorZoneY - xny;
        const float blend = wclamp(__fdiv_rn(distBelowFloor, kFloorBand), 0.0f, 1.0f);
        nv.y += ws * blend * distBelowFloor;
    }
    const uint32_t nw = wall_count_of(W.count_pad[0]);
    for (uint32_t wi = 0; wi < nw; ++wi) {
        const WallD w = load_wall(W.walls[wi]);
        const f3 xnw = mk(np.x + nv.x * dt * lk, np.y + nv.y * dt * lk, np.z + nv.z * dt * lk);
        const f3 lxn = wall_to_local(xnw, w);
        if (inside_open(lxn, w.mn, w.mx)) {
            f3 nl;
            const float sw = wall_sdf_normal(lxn, w.mn, w.mx, nl);
            const float dist = -sw;
            const float blend = wclamp(__fdiv_rn(dist, P.wall_min), 0.0f, 1.0f);
            const f3 nwd = wall_to_world_dir(nl, w);
            const float sc = ws * blend * dist;
            nv = mk(nv.x + nwd.x * sc, nv.y + nwd.y * sc, nv.z + nwd.z * sc);
        }
        const f3 lnp = wall_to_local(np, w);
        if (inside_open(lnp, w.mn, w.mx)) {
            f3 nl;
            const float sw = wall_sdf_normal(lnp, w.mn, w.mx, nl);
            const f3 nn = wall_to_world_dir(nl, w);
            const float mm = fmaxf(sw, -0.5f);
            np = mk(np.x - nn.x * mm, np.y - nn.y * mm, np.z - nn.z * mm);
            const float vn = dot3(sub(nv, wall_vel_at(np, w)), nn);
            if (vn < 0.0f) nv = mk(nv.x - vn * nn.x, nv.y - vn * nn.y, nv.z - vn * nn.z);
        }
    }
    const float hmin = P.hard_min;
    if (np.x < hmin) { np.x = hmin; nv.x = 0.0f; }
    if (np.x > P.hard_max_x) { np.x = P.hard_max_x; nv.x = 0.0f; }
    if (np.y < hmin) { np.y = hmin; nv.y = 0.0f; }
    if (np.y > P.hard_max_y) { np.y = P.hard_max_y; nv.y = 0.0f; }
    if (np.z < hmin) { np.z = hmin; nv.z = 0.0f; }
    if (np.z > P.hard_max_z) { np.z = P.hard_max_z; nv.z = 0.0f; }
    pos[p] = make_float4(np.x, np.y, np.z, 0.0f);
    vel[p] = make_float4(nv.x, nv.y, nv.z, 0.0f);
}

// ---------------------------------------------------------------------------
// Diffuse GENERATE (shaders.js:721-856), split in three so that slot
// assignment is deterministic: (1) every particle decides whether it spawns
// and stages its record at staging[id], setting bit id; (2) popcounts + one
// scan give each spawner its rank among spawners in ascending id; (3) the
// spawner of rank r takes free_list[top-1-r] if r < top — exactly the slots a
// one-at-a-time try_spawn (shaders.js:791-798) hands out in ascending id.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool estimate_normal(const float* __restrict__ cmf, const mpm_params& P, float px,
                                                float py, float pz, f3& n) {
    const int32_t X = P.grid_X, Y = P.grid_Y, Z = P.grid_Z;
    const int32_t gx = __float2int_rz(floorf(px)), gy = __float2int_rz(floorf(py)), gz = __float2int_rz(floorf(pz));
    if (gx < 1 || gx >= X - 1 || gy < 1 || gy >= Y - 1 || gz < 1 || gz >= Z - 1) return false;
    const uint32_t idxL = (uint32_t)((gz * Y + gy) * X + (gx - 1));
    const uint32_t idxR = (uint32_t)((gz * Y + gy) * X + (gx + 1));
    const uint32_t idxD = (uint32_t)((gz * Y + (gy - 1)) * X + gx);
    const uint32_t idxU = (uint32_t)((gz * Y + (gy + 1)) * X + gx);
    const uint32_t idxB = (uint32_t)(((gz - 1) * Y + gy) * X + gx);
    const uint32_t idxF = (uint32_t)(((gz + 1) * Y + gy) * X + gx);
    const f3 v = mk(cmf[idxL] - cmf[idxR], cmf[idxD] - cmf[idxU], cmf[idxB] - cmf[idxF]);
    const float len = len3(v);
    if (len < 1e-6f) return false;
    n = mk(__fdiv_rn(v.x, len), __fdiv_rn(v.y, len), __fdiv_rn(v.z, len));
    return true;
}

// Spawn decision + record for fluid particle `id` with post-G2P pos/vel.
__device__ __forceinline__ bool diffuse_spawn_record(uint32_t id, float4 q, float4 v, float m, float density,
                                                     const float* __restrict__ cmf, const mpm_params& P,
                                                     const mpm_gen_params& gen, mpm_diffuse_particle& r) {
    if (density <= 0.0f || density > gen.density_bubble_min) return false;
    const f3 vel = mk(v.x, v.y, v.z);
    const float speed2 = dot3(vel, vel);
    const float speed = __fsqrt_rn(speed2);
    const float ke = 0.5f * m * speed2;
    const float rest = P.rest_density;
    float pressure = P.stiffness * (eos_pow(__fdiv_rn(density, rest), P.eos_power) - 1.0f);
    const float pFloor = density > rest * kCohesionGate ? kCohesionPressure : 0.0f;
    pressure = fmaxf(pressure, pFloor);
    const float trappedAir = fmaxf(0.0f, pressure - gen.pressure_threshold);
    f3 nrm;
    const bool ok = estimate_normal(cmf, P, q.x, q.y, q.z, nrm);
    float waveCrest = 0.0f;
    if (speed > 1e-4f && ok) {
        const f3 vs = mk(__fdiv_rn(vel.x, speed), __fdiv_rn(vel.y, speed), __fdiv_rn(vel.z, speed));
        const float dotVal = dot3(vs, nrm);
        if (dotVal > gen.crest_dot_threshold) waveCrest = dotVal * speed;
    }
    const float score = ke + trappedAir * 2.0f + waveCrest * 1.5f;
    if (score < gen.ke_threshold) return false;
    const uint32_t randSeed = id * 9781u + gen.seed;
    const float spawnChance = fminf(1.0f, (score - gen.ke_threshold) * gen.spawn_rate_k * P.dt);
    if (diffuse_rand(randSeed) > spawnChance) return false;
    const float jitter = 0.3f;
    const float jx = (diffuse_rand(randSeed + 1u) - 0.5f) * jitter * speed;
    const float jy = (diffuse_rand(randSeed + 2u) - 0.5f) * jitter * speed;
    const float jz = (diffuse_rand(randSeed + 3u) - 0.5f) * jitter * speed;
    uint32_t ptype = MPM_DIFFUSE_FOAM;
    if (density < gen.density_spray_max) ptype = MPM_DIFFUSE_SPRAY;
    const float lifetime =
        ptype == MPM_DIFFUSE_FOAM ? gen.lifetime_foam * fminf(1.0f, __fdiv_rn(score, gen.ke_threshold)) : 999.0f;
    r.pos[0] = q.x; r.pos[1] = q.y; r.pos[2] = q.z; r.pos[3] = 0.0f;
    r.vel[0] = vel.x + jx; r.vel[1] = vel.y + jy; r.vel[2] = vel.z + jz; r.vel[3] = 0.0f;
    r.ptype = ptype; r.alive = 1u; r.lifetime = lifetime; r._pad = 0.0f;
    return true;
}

// Plain engine: spawn decision per particle; one 256-thread block covers one
// rank group, so the group's spawn count is written here too.
__global__ void __launch_bounds__(kThreads) k_diffuse_gen_eval(const float4* __restrict__ pos,
                                                                const float4* __restrict__ vel,
                                                                const float* __restrict__ mass,
                                                                const float* __restrict__ dens,
                                                                const float* __restrict__ cmf, const mpm_params P,
                                                                const mpm_gen_params gen,
                                                                mpm_diffuse_particle* __restrict__ staging,
                                                                uint32_t* __restrict__ bits,
                                                                uint32_t* __restrict__ counts) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    bool s = false;
    if (p < P.particle_num) {
        mpm_diffuse_particle r;
        s = diffuse_spawn_record(p, pos[p], vel[p], mass[p], dens[p], cmf, P, gen, r);
        if (s) staging[p] = r;
    }
    const unsigned b = __ballot_sync(0xffffffffu, s);
    __shared__ uint32_t wc[kThreads / 32];
    if ((threadIdx.x & 31) == 0) {
        if ((p >> 5) < (P.particle_num + 31u) / 32u) bits[p >> 5] = b;
        wc[threadIdx.x >> 5] = __popc(b);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int i = 0; i < kThreads / 32; ++i) t += wc[i];
        counts[blockIdx.x] = t;
    }
}

// ---------------------------------------------------------------------------
// Diffuse ADVECT (shaders.js:858-997).  Kills set alive = 0 and a bit per
// slot; k_freelist_pass (mode 1) then pushes killed slots in ascending slot
// order (the order a one-at-a-time kill_particle, shaders.js:914-918, produces).
// ---------------------------------------------------------------------------
// vel4 (binned engine): the same velocities as float4, one 16-byte load per cell.
__device__ __forceinline__ f3 sample_grid_velocity(const float* __restrict__ mvf, const float4* __restrict__ vel4,
                                                   const mpm_params& P, f3 pos) {
    const int32_t X = P.grid_X, Y = P.grid_Y, Z = P.grid_Z;
    int32_t cx, cy, cz;
    float fx, fy, fz;
    cell_frac(pos.x, cx, fx);
    cell_frac(pos.y, cy, fy);
    cell_frac(pos.z, cz, fz);
    float wx[3], wy[3], wz[3];
    qweights(fx, wx[0], wx[1], wx[2]);
    qweights(fy, wy[0], wy[1], wy[2]);
    qweights(fz, wz[0], wz[1], wz[2]);
    f3 v = mk(0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int32_t zz = cz - 1 + k;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int32_t yy = cy - 1 + j;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int32_t xx = cx - 1 + i;
                if (xx < 0 || xx >= X || yy < 0 || yy >= Y || zz < 0 || zz >= Z) continue;
                const uint32_t idx = (uint32_t)((zz * Y + yy) * X + xx);
                const float w = wx[i] * wy[j] * wz[k];
                float cx, cy, cz;
                if (vel4) {
                    const float4 c = vel4[idx];
                    cx = c.x; cy = c.y; cz = c.z;
                } else {
                    cx = mvf[idx * 3u + 0u]; cy = mvf[idx * 3u + 1u]; cz = mvf[idx * 3u + 2u];
                }
                v.x += w * cx;
                v.y += w * cy;
                v.z += w * cz;
            }
        }
    }
    return v;
}

__device__ __forceinline__ void reflect_axis(float& p, float& v, float lo, float hi) {
    float np = p, nv = v;
    if (np < lo) { np = lo + (lo - np); nv = -nv * kRestitution; }
    else if (np > hi) { np = hi - (np - hi); nv = -nv * kRestitution; }
    p = wclamp(np, lo, hi);
    v = nv;
}

__device__ __forceinline__ void diffuse_advect(mpm_diffuse_particle* __restrict__ pool, const float* __restrict__ mvf,
                                               const float4* __restrict__ vel4, const mpm_params& P,
                                               const mpm_advect_params& adv, const mpm_wall_params& W,
                                               uint32_t* __restrict__ kill_bits, uint32_t* __restrict__ counts,
                                               uint32_t* __restrict__ alive_mask) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t M = adv.diffuse_max;
    const uint32_t nwords = (M + 31u) / 32u;
    // the warp's 32 slots are one mask word: a dead slot's record is never read
    // (the reference tests pool[i].alive; the mask holds exactly those flags)
    const uint32_t word = (i >> 5) < nwords ? alive_mask[i >> 5] : 0u;
    bool kill = false;
    if (i < M && ((word >> (i & 31u)) & 1u)) {
        mpm_diffuse_particle p = pool[i];
        const f3 pos3 = mk(p.pos[0], p.pos[1], p.pos[2]);
        const float dt = P.dt, g = P.gravity;
        bool dead = false;
        if (p.ptype == MPM_DIFFUSE_SPRAY) {
            p.vel[1] += g * dt;
            p.pos[0] = pos3.x + dt * p.vel[0]; p.pos[1] = pos3.y + dt * p.vel[1]; p.pos[2] = pos3.z + dt * p.vel[2];
            p.pos[3] = 0.0f;
        } else if (p.ptype == MPM_DIFFUSE_FOAM) {
            const f3 gv = sample_grid_velocity(mvf, vel4, P, pos3);
            p.pos[0] = pos3.x + dt * gv.x; p.pos[1] = pos3.y + dt * gv.y; p.pos[2] = pos3.z + dt * gv.z;
            p.pos[3] = 0.0f;
            p.lifetime -= dt;
            if (p.lifetime <= 0.0f) dead = true;
        } else if (p.ptype == MPM_DIFFUSE_BUBBLE) {
            const f3 gv = sample_grid_velocity(mvf, vel4, P, pos3);
            p.vel[0] += dt * adv.drag * (gv.x - p.vel[0]);
            p.vel[1] += dt * (adv.buoyancy * -g + adv.drag * (gv.y - p.vel[1]));
            p.vel[2] += dt * adv.drag * (gv.z - p.vel[2]);
            p.pos[0] = pos3.x + dt * p.vel[0]; p.pos[1] = pos3.y + dt * p.vel[1]; p.pos[2] = pos3.z + dt * p.vel[2];
            p.pos[3] = 0.0f;
        }
        if (!dead) {
            const uint32_t nw = wall_count_of(W.count_pad[0]);
            for (uint32_t wi = 0; wi < nw; ++wi) {
                const WallD w = load_wall(W.walls[wi]);
                const f3 lp = wall_to_local(mk(p.pos[0], p.pos[1], p.pos[2]), w);
                if (!inside_open(lp, w.mn, w.mx)) continue;
                f3 nl;
                const float sw = wall_sdf_normal(lp, w.mn, w.mx, nl);
                const f3 nn = wall_to_world_dir(nl, w);
                p.pos[0] = p.pos[0] - nn.x * sw; p.pos[1] = p.pos[1] - nn.y * sw; p.pos[2] = p.pos[2] - nn.z * sw;
                p.pos[3] = 0.0f;
                const f3 wvel = wall_vel_at(mk(p.pos[0], p.pos[1], p.pos[2]), w);
                const f3 vrel = sub(mk(p.vel[0], p.vel[1], p.vel[2]), wvel);
                const float vn = dot3(vrel, nn);
                if (vn < 0.0f) {
                    const float kk = (1.0f + kRestitution) * vn;
                    const f3 nvr = mk(vrel.x - kk * nn.x, vrel.y - kk * nn.y, vrel.z - kk * nn.z);
                    p.vel[0] = wvel.x + nvr.x; p.vel[1] = wvel.y + nvr.y; p.vel[2] = wvel.z + nvr.z;
                    p.vel[3] = 0.0f;
                }
            }
            if (p.pos[1] < P.hard_min) dead = true;
        }
        if (dead) {
            pool[i].alive = 0u;
            kill = true;
        } else {
            reflect_axis(p.pos[0], p.vel[0], P.hard_min, P.hard_max_x);
            reflect_axis(p.pos[1], p.vel[1], P.hard_min, P.hard_max_y);
            reflect_axis(p.pos[2], p.vel[2], P.hard_min, P.hard_max_z);
            p.pos[3] = 0.0f;
            p.vel[3] = 0.0f;
            pool[i] = p;
        }
    }
    const unsigned b = __ballot_sync(0xffffffffu, kill);
    __shared__ uint32_t wc[kThreads / 32];
    if ((threadIdx.x & 31) == 0) {
        if ((i >> 5) < nwords) {
            kill_bits[i >> 5] = b;
            if (b) alive_mask[i >> 5] = word & ~b;   // this warp owns the word
        }
        wc[threadIdx.x >> 5] = __popc(b);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int k = 0; k < kThreads / 32; ++k) t += wc[k];
        counts[blockIdx.x] = t;
    }
}

// ADVECT with the uniforms as kernel parameters (plain engine).
__global__ void __launch_bounds__(kThreads) k_diffuse_advect(mpm_diffuse_particle* __restrict__ pool,
                                                              const float* __restrict__ mvf,
                                                              const float4* __restrict__ vel4, const mpm_params P,
                                                              const mpm_advect_params adv, const mpm_wall_params W,
                                                              uint32_t* __restrict__ kill_bits,
                                                              uint32_t* __restrict__ counts,
                                                              uint32_t* __restrict__ alive_mask) {
    diffuse_advect(pool, mvf, vel4, P, adv, W, kill_bits, counts, alive_mask);
}

// ADVECT with the uniforms read from device memory (binned engine; graph-capturable).
__global__ void __launch_bounds__(kThreads) k_diffuse_advect_dev(mpm_diffuse_particle* __restrict__ pool,
                                                                  const float4* __restrict__ vel4,
                                                                  const mpm_params* __restrict__ P,
                                                                  const mpm_advect_params* __restrict__ adv,
                                                                  const mpm_wall_params* __restrict__ W,
                                                                  uint32_t* __restrict__ kill_bits,
                                                                  uint32_t* __restrict__ counts,
                                                                  uint32_t* __restrict__ alive_mask) {
    diffuse_advect(pool, nullptr, vel4, *P, *adv, *W, kill_bits, counts, alive_mask);
}

// Rebuilds the alive mask from the pool's alive flags (after the pool was
// written from outside the diffuse passes).
__global__ void __launch_bounds__(kThreads) k_alive_mask_build(const mpm_diffuse_particle* __restrict__ pool,
                                                              uint32_t M, uint32_t* __restrict__ alive_mask) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned b = __ballot_sync(0xffffffffu, i < M && pool[i].alive != 0u);
    if ((threadIdx.x & 31u) == 0 && (i >> 5) < (M + 31u) / 32u) alive_mask[i >> 5] = b;
}

// One free-list pass in a single launch: the exclusive scan of the group
// counts and the ordered pops or pushes of the free-list stack
// (shaders.js:789-798 try_spawn, shaders.js:914-918 kill_particle), taken one
// at a time in ascending id order.  Mode 0 (spawn): the spawner of rank r
// takes free_list[top-1-r] while r < min(total, top).  Mode 1 (kill): the
// killed slot of rank r goes to free_list[top+r].  Block b owns the
// contiguous groups [b*R, (b+1)*R); every block reads all counts (a few KB)
// for its prefix and the total, so no block waits on another.  One warp per
// group: the group's 8 bitmap words are taken in ascending order, lane l
// holding bit l of the word.  state = {top before, total, applied, ticket}:
// the last block to finish (ticket) writes the new top and resets the ticket;
// a kill pass also appends the new top to top_hist (state[4] counts them) and
// clears the spawn bits and counts (clear_bits, clear_counts) that the spawn
// pass before it read, ready for the next substep's G2P.
constexpr int kPassThreads = 512;
constexpr uint32_t kNoSlot = 0xFFFFFFFFu;
__global__ void __launch_bounds__(kPassThreads, 2) k_freelist_pass(const uint32_t* __restrict__ bits, uint32_t nbits,
                                                                const uint32_t* __restrict__ counts, uint32_t ng,
                                                                uint32_t R, int32_t* __restrict__ top,
                                                                int32_t* __restrict__ state,
                                                                uint32_t* __restrict__ free_list,
                                                                const mpm_diffuse_particle* __restrict__ staging,
                                                                mpm_diffuse_particle* __restrict__ pool, uint32_t M,
                                                                int mode, int32_t* __restrict__ top_hist,
                                                                uint32_t* __restrict__ clear_bits, uint32_t nclear_bits,
                                                                uint32_t* __restrict__ clear_counts,
                                                                uint32_t nclear_counts,
                                                                uint32_t* __restrict__ alive_mask) {
    constexpr int kWarps = kPassThreads / 32;
    __shared__ uint32_t red[2][kWarps];
    __shared__ uint32_t excl[kPassThreads];
    __shared__ int32_t s_t0;
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    const uint32_t g0 = blockIdx.x * R, g1 = min(ng, g0 + R);
    if (threadIdx.x == 0) s_t0 = *top;
    // the total and the count before this block's first group
    uint32_t all = 0, before = 0;
    {
        const uint32_t n4 = ng / 4;   // counts is 16-byte aligned (a device allocation)
        const uint4* c4 = reinterpret_cast<const uint4*>(counts);
        for (uint32_t i = threadIdx.x; i < n4; i += kPassThreads) {
            const uint4 c = c4[i];
            const uint32_t g = 4 * i;
            all += c.x + c.y + c.z + c.w;
            before += (g < g0 ? c.x : 0u) + (g + 1 < g0 ? c.y : 0u) + (g + 2 < g0 ? c.z : 0u) + (g + 3 < g0 ? c.w : 0u);
        }
        for (uint32_t g = 4 * n4 + threadIdx.x; g < ng; g += kPassThreads) {
            const uint32_t c = counts[g];
            all += c;
            if (g < g0) before += c;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        all += __shfl_xor_sync(0xffffffffu, all, o);
        before += __shfl_xor_sync(0xffffffffu, before, o);
    }
    if (lane == 0) { red[0][wid] = all; red[1][wid] = before; }
    __syncthreads();
    all = 0;
    before = 0;
    for (int k = 0; k < kWarps; ++k) { all += red[0][k]; before += red[1][k]; }
    const int32_t t0 = s_t0, total = (int32_t)all;
    const int32_t applied = mode == 0 ? (t0 > 0 ? (total < t0 ? total : t0) : 0) : total;
    const uint32_t nwords = (nbits + 31u) / 32u;
    uint32_t carry = before;
    for (uint32_t base = g0; base < g1; base += kPassThreads) {
        // exclusive scan of this tile's group counts
        const uint32_t g = base + threadIdx.x;
        const uint32_t c = g < g1 ? counts[g] : 0u;
        uint32_t x = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        __syncthreads();   // red is free again
        if (lane == 31) red[0][wid] = x;
        __syncthreads();
        uint32_t wpre = 0;
        for (uint32_t k = 0; k < wid; ++k) wpre += red[0][k];
        excl[threadIdx.x] = carry + wpre + x - c;
        uint32_t tile_total = 0;
        for (int k = 0; k < kWarps; ++k) tile_total += red[0][k];
        __syncthreads();
        // one warp per group with members
        const uint32_t tn = min(g1 - base, (uint32_t)kPassThreads);
        for (uint32_t t = wid; t < tn; t += kWarps) {
            const uint32_t gg = base + t;
            const uint32_t r0 = excl[t];
            const uint32_t cnt = (t + 1 < tn ? excl[t + 1] : carry + tile_total) - r0;
            if (cnt == 0) continue;                                    // warp-uniform
            if (mode == 0 && (int32_t)r0 >= applied) continue;         // no slot left for this group
            const uint32_t wi = gg * (kGroupIds / 32) + (lane & 7u);
            const uint32_t myword = lane < 8u && wi < nwords ? bits[wi] : 0u;
            // lane l takes bit l of each of the 8 words; every load and store of
            // the group is independent of the others, so all are in flight at once
            uint32_t r = r0;
            uint32_t slot[kGroupIds / 32];
#pragma unroll
            for (uint32_t j = 0; j < kGroupIds / 32; ++j) {
                const uint32_t word = __shfl_sync(0xffffffffu, myword, j);
                const bool bit = (word >> lane) & 1u;
                const uint32_t rr = r + __popc(word & ((1u << lane) - 1u));
                const uint32_t id = gg * kGroupIds + j * 32u + lane;
                slot[j] = kNoSlot;
                if (bit && id < nbits) {
                    if (mode == 0) {
                        const int32_t fi = t0 - 1 - (int32_t)rr;
                        // free-list state uploaded by a caller may be inconsistent: never index outside the pool
                        if ((int32_t)rr < applied && fi >= 0 && (uint32_t)fi < M) slot[j] = free_list[fi];
                    } else {
                        const int32_t fi = t0 + (int32_t)rr;
                        if (fi >= 0 && (uint32_t)fi < M) free_list[fi] = id;
                    }
                }
                r += __popc(word);
            }
            if (mode == 0) {
                // 48-byte records as three 16-byte words (device allocations and
                // 48-byte strides keep every record 16-byte aligned); kBatch records'
                // loads are issued before their stores
                constexpr uint32_t kBatch = 2;
                static_assert(sizeof(mpm_diffuse_particle) == 48, "three 16-byte words per record");
#pragma unroll
                for (uint32_t jb = 0; jb < kGroupIds / 32; jb += kBatch) {
                    uint4 rec[kBatch][3];
#pragma unroll
                    for (uint32_t q = 0; q < kBatch; ++q) {
                        if (slot[jb + q] < M) {
                            const uint4* src =
                                reinterpret_cast<const uint4*>(staging + gg * kGroupIds + (jb + q) * 32u + lane);
                            rec[q][0] = src[0];
                            rec[q][1] = src[1];
                            rec[q][2] = src[2];
                        }
                    }
#pragma unroll
                    for (uint32_t q = 0; q < kBatch; ++q) {
                        if (slot[jb + q] < M) {
                            const uint32_t sl = slot[jb + q];
                            uint4* dst = reinterpret_cast<uint4*>(pool + sl);
                            dst[0] = rec[q][0];
                            dst[1] = rec[q][1];
                            dst[2] = rec[q][2];
                            atomicOr(&alive_mask[sl >> 5], 1u << (sl & 31u));   // staged records are alive
                        }
                    }
                }
            }
        }
        carry += tile_total;
        __syncthreads();   // excl is rewritten by the next tile
    }
    // (kill pass) the spawn bits and counts were last read by the spawn pass:
    // clear them for the next substep's G2P
    for (uint32_t i = blockIdx.x * kPassThreads + threadIdx.x; i < nclear_bits; i += gridDim.x * kPassThreads)
        clear_bits[i] = 0u;
    for (uint32_t i = blockIdx.x * kPassThreads + threadIdx.x; i < nclear_counts; i += gridDim.x * kPassThreads)
        clear_counts[i] = 0u;
    // the last block to finish publishes the new top
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t done = atomicAdd(reinterpret_cast<uint32_t*>(&state[3]), 1u);
        if (done == gridDim.x - 1) {
            const int32_t nt = mode == 0 ? t0 - applied : t0 + total;
            *top = nt;
            state[0] = t0;
            state[1] = total;
            state[2] = applied;
            state[3] = 0;
            if (mode == 1) {   // kill pass k leaves the substep's final top in top_hist[k % kTopHist]
                const uint32_t k = (uint32_t)state[4];
                top_hist[k % DiffuseState::kTopHist] = nt;
                state[4] = (int32_t)(k + 1u);
            }
        }
    }
}

// Blocks of one free-list pass over ng groups: about one group per warp, at
// most two blocks per SM's worth.
static inline void freelist_grid(uint32_t ng, uint32_t& B, uint32_t& R) {
    constexpr uint32_t kWarps = kPassThreads / 32, kMaxBlocks = 2 * 148;
    B = std::max(1u, std::min(blocks_for(ng, kWarps), kMaxBlocks));
    R = std::max(1u, blocks_for(ng, B));
    B = std::max(1u, blocks_for(ng, R));
}

cudaError_t launch_alive_mask_build(Scene& s) {
    const DiffuseState& d = s.diffuse;
    k_alive_mask_build<<<blocks_for(d.max_count, kThreads), kThreads, 0, s.stream>>>(d.pool, d.max_count, d.alive_mask);
    s.launches++;
    return cudaGetLastError();
}

cudaError_t launch_apply_hand(Scene& s) {
    dim3 grid(blocks_for(s.hand_dims[0], 4), blocks_for(s.hand_dims[1], 4), blocks_for(s.hand_dims[2], 4));
    k_apply_hand<<<grid, dim3(4, 4, 4), 0, s.stream>>>(s.mvf, s.params, s.hand);
    return cudaGetLastError();
}

// DiffuseGPU.step (diffuse-gpu.js:148-166) after G2P.  With eval the spawn
// decision pass runs here (plain engine); the binned engine makes that
// decision in its G2P epilogue and has already bumped the seed.
cudaError_t launch_diffuse(Scene& s, bool eval, const mpm_params* P_dev, const mpm_wall_params* W_dev,
                           cudaStream_t stream) {
    static_assert(kThreads == (int)kGroupIds, "one rank group per 256-thread block");
    cudaStream_t st = stream ? stream : s.stream;
    const mpm_params& P = s.params;
    DiffuseState& d = s.diffuse;
    const uint32_t n = P.particle_num;
    const uint32_t ng = blocks_for(n, kGroupIds);
    if (n > 0) {
        Phase ph(s, MPM_PHASE_DIFFUSE_GEN);
        if (eval) {
            d.seed = d.seed + 1u;                 // diffuse-gpu.js:149
            mpm_gen_params gen = d.gen;
            gen.seed = d.seed;
            k_diffuse_gen_eval<<<ng, kThreads, 0, st>>>(s.pos, s.vel, s.mass, s.dens, s.cmf, P, gen, d.staging,
                                                        d.spawn_bits, d.block_counts);
            s.launches++;
        }
        // (the binned engine's G2P has already counted the spawners per group)
        uint32_t B, R;
        freelist_grid(ng, B, R);
        k_freelist_pass<<<B, kPassThreads, 0, st>>>(d.spawn_bits, n, d.block_counts, ng, R, d.top, d.rank_state,
                                                    d.free_list, d.staging, d.pool, d.max_count, 0, nullptr, nullptr, 0,
                                                    nullptr, 0, d.alive_mask);
        s.launches += 1;
    } else if (eval) {
        d.seed = d.seed + 1u;
    }
    const uint32_t M = d.max_count;
    const uint32_t mg = blocks_for(M, kGroupIds);
    mpm_advect_params adv = d.adv;
    adv.diffuse_max = M;
    {
        Phase ph(s, MPM_PHASE_DIFFUSE_ADV);
        if (P_dev && W_dev && s.vel4)
            k_diffuse_advect_dev<<<mg, kThreads, 0, st>>>(d.pool, s.vel4, P_dev, d.adv_dev, W_dev, d.kill_bits,
                                                          d.kill_counts, d.alive_mask);
        else
            k_diffuse_advect<<<mg, kThreads, 0, st>>>(d.pool, s.mvf, s.vel4, P, adv, s.walls, d.kill_bits,
                                                      d.kill_counts, d.alive_mask);
        uint32_t B, R;
        freelist_grid(mg, B, R);
        k_freelist_pass<<<B, kPassThreads, 0, st>>>(d.kill_bits, M, d.kill_counts, mg, R, d.top, d.rank_state,
                                                    d.free_list, nullptr, d.pool, M, 1, d.top_hist, d.spawn_bits,
                                                    (n + 31u) / 32u, d.block_counts, ng, nullptr);
        s.launches += 2;
        d.passes++;
        d.top_written = false;
    }
    return cudaGetLastError();
}

// One substep of the plain engine: one kernel per reference pass, in the
// reference's order (fluid-gpu.js:663-682), on reference-layout buffers.
cudaError_t launch_substep_plain(Scene& s) {
    cudaStream_t st = s.stream;
    const mpm_params& P = s.params;
    const uint32_t n = P.particle_num;
    const uint64_t G = s.G;
    {
        Phase ph(s, MPM_PHASE_CLEAR);
        cudaError_t e = cudaMemsetAsync(s.grid_i32, 0, 16 * G, st);   // CLEAR
        if (e != cudaSuccess) return e;
    }
    if (n > 0) {
        Phase ph(s, MPM_PHASE_P2G_MASS);
        k_p2g_mass<<<blocks_for(n, kThreads), kThreads, 0, st>>>(s.pos, s.mass, s.cm, n, (int32_t)s.X,
                                                                 (int32_t)s.Y, (int32_t)s.Z);
        s.launches++;
    }
    {
        Phase ph(s, MPM_PHASE_DECODE_MASS);
        k_decode_mass<<<blocks_for(G, kThreads), kThreads, 0, st>>>(s.cm, s.cmf, G);
        s.launches++;
    }
    if (n > 0) {
        Phase ph(s, MPM_PHASE_P2G_MOM);
        k_p2g_mom<<<blocks_for(n, kThreads), kThreads, 0, st>>>(s.pos, s.vel, s.aff, s.mass, s.cmf, s.mv, s.dens, P,
                                                                (uint32_t)G);
        s.launches++;
    }
    {
        Phase ph(s, MPM_PHASE_UPDATE_GRID);
        k_update_grid<<<blocks_for(G, kThreads), kThreads, 0, st>>>(s.mv, s.cm, s.mvf, P, s.walls);
        s.launches++;
    }
    if (s.hand_active && s.hand_dims[0] > 0 && s.hand_dims[1] > 0 && s.hand_dims[2] > 0) {
        Phase ph(s, MPM_PHASE_APPLY_HAND);
        cudaError_t e = launch_apply_hand(s);
        if (e != cudaSuccess) return e;
        s.launches++;
    }
    if (n > 0) {
        Phase ph(s, MPM_PHASE_G2P);
        k_g2p<<<blocks_for(n, kThreads), kThreads, 0, st>>>(s.pos, s.vel, s.aff, s.mvf, P, s.walls, (uint32_t)G);
        s.launches++;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (s.diffuse.enabled) e = launch_diffuse(s, /*eval=*/true);
    return e;
}

}  // namespace mpm
