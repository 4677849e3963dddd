// mpm_fast.cu — the binned, item-major MLS-MPM substep.
//
// Same arithmetic as mpm_kernels.cu (and so the same bits), organised for
// the B200:
//   * Particles live in cell-sorted order (double-buffered, SoA-ish):
//       posm  float4 (x, y, z, mass)    velid float4 (vx, vy, vz, id bits)
//       aff   9 floats                  dens  float
//     G2P writes the next state in the current sorted order and counts each
//     particle into its new cell; the next substep's binning turns the counts
//     into cell ranges and a permutation (sorted slot -> previous slot).
//   * Work item = up to `chunk` particles of one cell.  One thread owns an
//     item: the 27 neighbour masses (P2G_MOM) or velocities (G2P) are loaded
//     once per item, and P2G contributions are summed in registers as i32
//     (the same wrapping sums the reference's atomics produce) and flushed
//     with one atomic per (cell, component) per item.
//   * The grid is processed per tile (16x8x8 cells) and only for tiles a
//     particle stencil touches now or touched last substep (cells elsewhere
//     are zero, as the reference's CLEAR/DECODE/UPDATE would leave them).
//     The i32 grid is double-buffered: UPDATE_GRID of substep s reads
//     buffer s%2 and zeroes buffer (s+1)%2, which is the CLEAR of s+1.
//   * The diffuse spawn decision runs in the G2P epilogue (post-G2P pos/vel,
//     this substep's density), staging records by particle id.
// Reference-layout buffers (pos4/vel4/affine9/mass/density) are produced on
// demand by an export kernel that scatters by particle id.
#include <cuda_runtime.h>

#include <cstdint>

#include "mpm_device.cuh"
#include "mpm_fast.h"
#include "mpm_kernels.h"
#include "mpm_scene.h"

namespace mpm {

namespace {

constexpr int kItemThreads = 128;

__device__ __forceinline__ uint32_t cell_of(int32_t x, int32_t y, int32_t z, uint32_t X, uint32_t Y) {
    return ((uint32_t)z * Y + (uint32_t)y) * X + (uint32_t)x;
}

__device__ __forceinline__ int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---------------------------------------------------------------------------
// Binning
// ---------------------------------------------------------------------------

// Count particle `j` of state buffer `cur` into its cell; mark the tiles its
// 3x3x3 stencil touches.  Cells are clamped into the grid for binning only.
__device__ __forceinline__ void bin_particle(const FastView& v, uint32_t j, float px, float py, float pz) {
    int32_t cx, cy, cz;
    float fx, fy, fz;
    cell_frac(px, cx, fx);
    cell_frac(py, cy, fy);
    cell_frac(pz, cz, fz);
    cx = clampi(cx, 0, (int32_t)v.X - 1);
    cy = clampi(cy, 0, (int32_t)v.Y - 1);
    cz = clampi(cz, 0, (int32_t)v.Z - 1);
    const uint32_t c = cell_of(cx, cy, cz, v.X, v.Y);
    const uint32_t r = atomicAdd(&v.cell_count[c], 1u);
    v.key[j] = c;
    v.rank[j] = r;
    const int32_t tx0 = max(cx - 1, 0) / kTileX, tx1 = min(cx + 1, (int32_t)v.X - 1) / kTileX;
    const int32_t ty0 = max(cy - 1, 0) / kTileY, ty1 = min(cy + 1, (int32_t)v.Y - 1) / kTileY;
    const int32_t tz0 = max(cz - 1, 0) / kTileZ, tz1 = min(cz + 1, (int32_t)v.Z - 1) / kTileZ;
    const uint32_t own = ((uint32_t)(cz / kTileZ) * v.nty + (uint32_t)(cy / kTileY)) * v.ntx + (uint32_t)(cx / kTileX);
    if ((v.tile_flags[own] & 3u) != 3u) atomicOr(&v.tile_flags[own], 3u);   // occupied (bit0) + stencil (bit1)
    if (tx0 != tx1 || ty0 != ty1 || tz0 != tz1) {
        for (int32_t tz = tz0; tz <= tz1; ++tz)
            for (int32_t ty = ty0; ty <= ty1; ++ty)
                for (int32_t tx = tx0; tx <= tx1; ++tx) {
                    const uint32_t t = ((uint32_t)tz * v.nty + (uint32_t)ty) * v.ntx + (uint32_t)tx;
                    if (t != own) atomicOr(&v.tile_flags[t], 2u);
                }
    }
}

// Identity-order import: keys for the state just copied in.
__global__ void k_import_keys(FastView v, const float4* __restrict__ posm, uint32_t n) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const float4 q = posm[j];
    bin_particle(v, j, q.x, q.y, q.z);
}

// Per substep: build the occupied-tile list (for binning) and the grid-tile
// list (stencil tiles of this substep or the last one, plus the hand box);
// shift the flags.  tile_flags bits: 0 occupied, 1 stencil (this substep),
// 2 stencil (last substep), 3 hand box (this substep).
__global__ void k_tiles(FastView v, int32_t hx0, int32_t hy0, int32_t hz0, int32_t hx1, int32_t hy1, int32_t hz1) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= v.ntiles) return;
    uint32_t f = v.tile_flags[t];
    const uint32_t tx = t % v.ntx, ty = (t / v.ntx) % v.nty, tz = t / (v.ntx * v.nty);
    if (hx0 <= hx1) {
        const int32_t x0 = (int32_t)tx * kTileX, y0 = (int32_t)ty * kTileY, z0 = (int32_t)tz * kTileZ;
        if (x0 <= hx1 && x0 + kTileX - 1 >= hx0 && y0 <= hy1 && y0 + kTileY - 1 >= hy0 && z0 <= hz1 &&
            z0 + kTileZ - 1 >= hz0)
            f |= 8u;
    }
    const bool occ = f & 1u;
    const bool now = (f & (2u | 8u)) != 0;
    const bool prev = (f & 4u) != 0;
    if (occ) v.tile_occ_list[atomicAdd(&v.counters[kCntOcc], 1u)] = t;
    if (now || prev) v.tile_grid_list[atomicAdd(&v.counters[kCntGrid], 1u)] = t;
    v.tile_flags[t] = now ? 4u : 0u;
}

// Block-wide exclusive scan of one value per thread (blockDim.x == 1024).
__device__ __forceinline__ uint32_t block_scan_1024(uint32_t x, uint32_t* total, uint32_t* ws) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t s = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
    }
    if (lane == 31) ws[wid] = s;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = ws[lane];
        uint32_t ww = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, ww, o);
            if (lane >= o) ww += y;
        }
        ws[lane] = ww - w;   // exclusive warp offsets
        if (lane == 31) ws[32] = ww;
    }
    __syncthreads();
    const uint32_t r = ws[wid] + s - x;
    *total = ws[32];
    __syncthreads();
    return r;
}

// One block per occupied tile (grid-stride over the list): cell counts ->
// cell ranges in sorted order and work items (cell, begin, len <= chunk).
__global__ void __launch_bounds__(kTileCells) k_bin_tiles(FastView v, uint32_t chunk) {
    __shared__ uint32_t ws[33];
    __shared__ uint32_t base_s[2];
    const uint32_t nocc = v.counters[kCntOcc];
    for (uint32_t ti = blockIdx.x; ti < nocc; ti += gridDim.x) {
        const uint32_t t = v.tile_occ_list[ti];
        const uint32_t tx = t % v.ntx, ty = (t / v.ntx) % v.nty, tz = t / (v.ntx * v.nty);
        const uint32_t lx = threadIdx.x % kTileX, ly = (threadIdx.x / kTileX) % kTileY, lz = threadIdx.x / (kTileX * kTileY);
        const uint32_t x = tx * kTileX + lx, y = ty * kTileY + ly, z = tz * kTileZ + lz;
        const bool inside = x < v.X && y < v.Y && z < v.Z;
        const uint32_t c = inside ? cell_of(x, y, z, v.X, v.Y) : 0u;
        uint32_t cnt = 0;
        if (inside) {
            cnt = v.cell_count[c];
            if (cnt) v.cell_count[c] = 0u;
        }
        const uint32_t nit = (cnt + chunk - 1) / chunk;
        uint32_t tot, itot;
        const uint32_t off = block_scan_1024(cnt, &tot, ws);
        const uint32_t ioff = block_scan_1024(nit, &itot, ws);
        if (threadIdx.x == 0) {
            base_s[0] = tot ? atomicAdd(&v.counters[kCntSorted], tot) : 0u;
            base_s[1] = itot ? atomicAdd(&v.counters[kCntItems], itot) : 0u;
        }
        __syncthreads();
        if (cnt) {
            const uint32_t b = base_s[0] + off;
            v.cell_start[c] = b;
            for (uint32_t k = 0; k < nit; ++k) {
                const uint32_t beg = b + k * chunk;
                const uint32_t len = min(chunk, cnt - k * chunk);
                v.items[base_s[1] + ioff + k] = make_uint4(c, beg, len, 0u);
            }
        }
        __syncthreads();
    }
}

// perm[sorted position] = previous slot
__global__ void k_scatter(FastView v, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t j = v.cell_start[v.key[i]] + v.rank[i];
    if (j < n) v.perm[j] = i;
}

// ---------------------------------------------------------------------------
// Per-particle helpers
// ---------------------------------------------------------------------------
struct PW {
    int32_t cx, cy, cz;
    float fx, fy, fz;
    float wx[3], wy[3], wz[3];
};

__device__ __forceinline__ PW particle_weights(float px, float py, float pz) {
    PW w;
    cell_frac(px, w.cx, w.fx);
    cell_frac(py, w.cy, w.fy);
    cell_frac(pz, w.cz, w.fz);
    qweights(w.fx, w.wx[0], w.wx[1], w.wx[2]);
    qweights(w.fy, w.wy[0], w.wy[1], w.wy[2]);
    qweights(w.fz, w.wz[0], w.wz[1], w.wz[2]);
    return w;
}

__device__ __forceinline__ void item_cell(const FastView& v, uint32_t c, int32_t& x, int32_t& y, int32_t& z) {
    x = (int32_t)(c % v.X);
    y = (int32_t)((c / v.X) % v.Y);
    z = (int32_t)(c / (v.X * v.Y));
}

// ---------------------------------------------------------------------------
// P2G_MASS (shaders.js:242-274), item-major
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kItemThreads) k_p2g_mass_items(FastView v, const float4* __restrict__ posm,
                                                                 int32_t* __restrict__ cm) {
    const uint32_t nitems = v.counters[kCntItems];
    const int32_t X = v.X, Y = v.Y, Z = v.Z;
    for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < nitems; it += gridDim.x * blockDim.x) {
        const uint4 item = v.items[it];
        int32_t ix, iy, iz;
        item_cell(v, item.x, ix, iy, iz);
        int32_t acc[27];
#pragma unroll
        for (int q = 0; q < 27; ++q) acc[q] = 0;
        for (uint32_t k = 0; k < item.z; ++k) {
            const float4 p = posm[v.perm[item.y + k]];
            const PW w = particle_weights(p.x, p.y, p.z);
            if (w.cx == ix && w.cy == iy && w.cz == iz) {
                float wxy[9];
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int i = 0; i < 3; ++i) wxy[j * 3 + i] = w.wx[i] * w.wy[j];
#pragma unroll
                for (int kk = 0; kk < 3; ++kk)
#pragma unroll
                    for (int j = 0; j < 3; ++j)
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            const float ww = wxy[j * 3 + i] * w.wz[kk];
                            acc[kk * 9 + j * 3 + i] += encode(ww * p.w);
                        }
            } else {
                // particle outside its binning cell (positions outside the grid): per-particle path
                for (int kk = 0; kk < 3; ++kk)
                    for (int j = 0; j < 3; ++j)
                        for (int i = 0; i < 3; ++i) {
                            const int32_t xx = w.cx - 1 + i, yy = w.cy - 1 + j, zz = w.cz - 1 + kk;
                            if (xx < 0 || xx >= X || yy < 0 || yy >= Y || zz < 0 || zz >= Z) continue;
                            const float ww = w.wx[i] * w.wy[j] * w.wz[kk];
                            atomicAdd(&cm[(zz * Y + yy) * X + xx], encode(ww * p.w));
                        }
            }
        }
#pragma unroll
        for (int kk = 0; kk < 3; ++kk)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const int32_t xx = ix - 1 + i, yy = iy - 1 + j, zz = iz - 1 + kk;
                    const int32_t a = acc[kk * 9 + j * 3 + i];
                    if (a != 0 && xx >= 0 && xx < X && yy >= 0 && yy < Y && zz >= 0 && zz < Z)
                        atomicAdd(&cm[(zz * Y + yy) * X + xx], a);
                }
    }
}

// ---------------------------------------------------------------------------
// Grid passes over the grid-tile list: DECODE_MASS and UPDATE_GRID (+ clear
// of the other i32 buffer).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool tile_cell(const FastView& v, uint32_t t, uint32_t lid, uint32_t& c, int32_t& x,
                                          int32_t& y, int32_t& z) {
    const uint32_t tx = t % v.ntx, ty = (t / v.ntx) % v.nty, tz = t / (v.ntx * v.nty);
    x = (int32_t)(tx * kTileX + lid % kTileX);
    y = (int32_t)(ty * kTileY + (lid / kTileX) % kTileY);
    z = (int32_t)(tz * kTileZ + lid / (kTileX * kTileY));
    if ((uint32_t)x >= v.X || (uint32_t)y >= v.Y || (uint32_t)z >= v.Z) return false;
    c = cell_of(x, y, z, v.X, v.Y);
    return true;
}

__global__ void __launch_bounds__(256) k_decode_tiles(FastView v, const int32_t* __restrict__ cm,
                                                      float* __restrict__ cmf) {
    const uint32_t ng = v.counters[kCntGrid];
    const uint32_t total = ng * kTileCells;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        uint32_t c;
        int32_t x, y, z;
        if (tile_cell(v, v.tile_grid_list[g / kTileCells], g % kTileCells, c, x, y, z)) cmf[c] = decode(cm[c]);
    }
}

__global__ void __launch_bounds__(256) k_update_tiles(FastView v, const int32_t* __restrict__ cm,
                                                      const int32_t* __restrict__ mv, float* __restrict__ mvf,
                                                      int32_t* __restrict__ cm_next, int32_t* __restrict__ mv_next,
                                                      const mpm_params P, const mpm_wall_params W) {
    const uint32_t ng = v.counters[kCntGrid];
    const uint32_t total = ng * kTileCells;
    const uint32_t nw = wall_count_of(W.count_pad[0]);
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        uint32_t idx;
        int32_t cx, cy, cz;
        if (!tile_cell(v, v.tile_grid_list[g / kTileCells], g % kTileCells, idx, cx, cy, cz)) continue;
        cm_next[idx] = 0;
        mv_next[3 * idx + 0] = 0; mv_next[3 * idx + 1] = 0; mv_next[3 * idx + 2] = 0;
        const float c = decode(cm[idx]);
        float* out = mvf + 3 * (size_t)idx;
        if (c <= 0.0f) { out[0] = 0.0f; out[1] = 0.0f; out[2] = 0.0f; continue; }
        float vx = __fdiv_rn(decode(mv[3 * idx + 0]), c);
        float vy = __fdiv_rn(decode(mv[3 * idx + 1]), c);
        float vz = __fdiv_rn(decode(mv[3 * idx + 2]), c);
        vy += P.gravity * P.dt;
        const int32_t X = P.grid_X, Y = P.grid_Y, Z = P.grid_Z;
        if (cx < 2 || cx > X - 3) vx = 0.0f;
        if (cy < 2 && vy < 0.0f) vy = 0.0f;
        if (cy > Y - 3 && vy > 0.0f) vy = 0.0f;
        if (cz < 2 || cz > Z - 3) vz = 0.0f;
        if (cy < 2) { vx *= 0.85f; vz *= 0.9f; }
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
}

// ---------------------------------------------------------------------------
// P2G_MOM (shaders.js:276-371), item-major
// ---------------------------------------------------------------------------
struct MomIn {
    float vx, vy, vz, m;
    float a00, a01, a02, a10, a11, a12, a20, a21, a22;
};

// The scatter part of P2G_MOM for one particle whose density is known.
// Adds the 81 encoded contributions into acc (or, with direct != nullptr,
// atomically into the grid at the particle's own stencil).
template <bool kDirect>
__device__ __forceinline__ void mom_scatter(const PW& w, const MomIn& in, float density, const mpm_params& P,
                                            int32_t* acc, int32_t* mv, uint32_t baseIdx, uint32_t G) {
    const float rest = P.rest_density;
    const float vol = __fdiv_rn(in.m, fmaxf(density, rest * 0.15f));
    float pressure = P.stiffness * (eos_pow(__fdiv_rn(density, rest), P.eos_power) - 1.0f);
    const float pFloor = density > rest * kCohesionGate ? kCohesionPressure : 0.0f;
    pressure = fmaxf(pressure, pFloor);
    const float visc = P.viscosity;
    const float s00 = -pressure + visc * (in.a00 + in.a00);
    const float s11 = -pressure + visc * (in.a11 + in.a11);
    const float s22 = -pressure + visc * (in.a22 + in.a22);
    const float s01 = visc * (in.a01 + in.a10);
    const float s02 = visc * (in.a02 + in.a20);
    const float s12 = visc * (in.a12 + in.a21);
    const float coef = -vol * 4.0f * P.dt;
    const float dxs[3] = {-w.fx - 1.0f, -w.fx, 1.0f - w.fx};
    const float dys[3] = {-w.fy - 1.0f, -w.fy, 1.0f - w.fy};
    const float dzs[3] = {-w.fz - 1.0f, -w.fz, 1.0f - w.fz};
    const uint32_t X = P.grid_X, SLICE = P.grid_X * P.grid_Y;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float wzk = w.wz[k], dzk = dzs[k];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float wyzk = w.wy[j] * wzk, dyj = dys[j];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const float ww = w.wx[i] * wyzk;
                const float dxi = dxs[i];
                const float Qx = in.a00 * dxi + in.a01 * dyj + in.a02 * dzk;
                const float Qy = in.a10 * dxi + in.a11 * dyj + in.a12 * dzk;
                const float Qz = in.a20 * dxi + in.a21 * dyj + in.a22 * dzk;
                const float fxf = coef * (s00 * dxi + s01 * dyj + s02 * dzk);
                const float fyf = coef * (s01 * dxi + s11 * dyj + s12 * dzk);
                const float fzf = coef * (s02 * dxi + s12 * dyj + s22 * dzk);
                const int32_t ex = encode(ww * (in.m * (in.vx + Qx) + fxf));
                const int32_t ey = encode(ww * (in.m * (in.vy + Qy) + fyf));
                const int32_t ez = encode(ww * (in.m * (in.vz + Qz) + fzf));
                if (kDirect) {
                    const uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)j * X + (uint32_t)i;
                    if (cidx < G) {
                        atomicAdd(mv + 3ull * cidx + 0, ex);
                        atomicAdd(mv + 3ull * cidx + 1, ey);
                        atomicAdd(mv + 3ull * cidx + 2, ez);
                    }
                } else {
                    const int q = (k * 9 + j * 3 + i) * 3;
                    acc[q + 0] += ex;
                    acc[q + 1] += ey;
                    acc[q + 2] += ez;
                }
            }
        }
    }
}

__global__ void __launch_bounds__(kItemThreads) k_p2g_mom_items(FastView v, const float4* __restrict__ posm,
                                                                const float4* __restrict__ velid,
                                                                const float* __restrict__ aff,
                                                                const float* __restrict__ cmf,
                                                                int32_t* __restrict__ mv, float* __restrict__ dens,
                                                                const mpm_params P) {
    const uint32_t nitems = v.counters[kCntItems];
    const uint32_t X = P.grid_X, SLICE = P.grid_X * P.grid_Y;
    const uint32_t G = (uint32_t)v.G;
    for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < nitems; it += gridDim.x * blockDim.x) {
        const uint4 item = v.items[it];
        int32_t ix, iy, iz;
        item_cell(v, item.x, ix, iy, iz);
        const uint32_t ibase = (uint32_t)(((iz - 1) * (int32_t)v.Y + (iy - 1)) * (int32_t)X + (ix - 1));
        float m27[27];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const uint32_t cidx = ibase + (uint32_t)k * SLICE + (uint32_t)j * X + (uint32_t)i;
                    m27[k * 9 + j * 3 + i] = cidx < G ? cmf[cidx] : 0.0f;
                }
        int32_t acc[81];
#pragma unroll
        for (int q = 0; q < 81; ++q) acc[q] = 0;
        for (uint32_t kk = 0; kk < item.z; ++kk) {
            const uint32_t j = item.y + kk;
            const uint32_t slot = v.perm[j];
            const float4 p = posm[slot];
            const float4 vv = velid[slot];
            const float* a = aff + 9ull * slot;
            MomIn in{vv.x, vv.y, vv.z, p.w, a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8]};
            const PW w = particle_weights(p.x, p.y, p.z);
            const bool same = (w.cx == ix && w.cy == iy && w.cz == iz);
            const uint32_t baseIdx = (uint32_t)(((w.cz - 1) * (int32_t)v.Y + (w.cy - 1)) * (int32_t)X + (w.cx - 1));
            float density = 0.0f;
            if (same) {
#pragma unroll
                for (int k = 0; k < 3; ++k)
#pragma unroll
                    for (int jj = 0; jj < 3; ++jj)
#pragma unroll
                        for (int i = 0; i < 3; ++i) density += w.wx[i] * w.wy[jj] * w.wz[k] * m27[k * 9 + jj * 3 + i];
            } else {
                for (int k = 0; k < 3; ++k)
                    for (int jj = 0; jj < 3; ++jj)
                        for (int i = 0; i < 3; ++i) {
                            const uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)jj * X + (uint32_t)i;
                            const float cmass = cidx < G ? cmf[cidx] : 0.0f;
                            density += w.wx[i] * w.wy[jj] * w.wz[k] * cmass;
                        }
            }
            dens[j] = density;
            if (density <= 1e-8f) continue;
            if (same) mom_scatter<false>(w, in, density, P, acc, mv, baseIdx, G);
            else mom_scatter<true>(w, in, density, P, acc, mv, baseIdx, G);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int jj = 0; jj < 3; ++jj)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const uint32_t cidx = ibase + (uint32_t)k * SLICE + (uint32_t)jj * X + (uint32_t)i;
                    const int q = (k * 9 + jj * 3 + i) * 3;
                    if (cidx < G) {
                        if (acc[q + 0]) atomicAdd(mv + 3ull * cidx + 0, acc[q + 0]);
                        if (acc[q + 1]) atomicAdd(mv + 3ull * cidx + 1, acc[q + 1]);
                        if (acc[q + 2]) atomicAdd(mv + 3ull * cidx + 2, acc[q + 2]);
                    }
                }
    }
}

// ---------------------------------------------------------------------------
// G2P (shaders.js:579-705), item-major, + binning of the new positions and
// the diffuse spawn decision (shaders.js:800-855).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool estimate_normal_f(const float* __restrict__ cmf, const mpm_params& P, float px,
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
    const f3 vv = mk(cmf[idxL] - cmf[idxR], cmf[idxD] - cmf[idxU], cmf[idxB] - cmf[idxF]);
    const float len = len3(vv);
    if (len < 1e-6f) return false;
    n = mk(__fdiv_rn(vv.x, len), __fdiv_rn(vv.y, len), __fdiv_rn(vv.z, len));
    return true;
}

__device__ __forceinline__ bool spawn_record(uint32_t id, float4 q, float4 v, float m, float density,
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
    const bool ok = estimate_normal_f(cmf, P, q.x, q.y, q.z, nrm);
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

// G2P for one particle given its gathered grid velocity / B matrix.
__device__ __forceinline__ void g2p_finish(const float4 q, float gvx, float gvy, float gvz, const float* B,
                                           const mpm_params& P, const mpm_wall_params& W, f3& np, f3& nv) {
    const float dt = P.dt, lk = P.lookahead_k, ws = P.wall_stiffness;
    np = mk(q.x + dt * gvx, q.y + dt * gvy, q.z + dt * gvz);
    nv = mk(gvx, gvy, gvz);
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
}

__global__ void __launch_bounds__(kItemThreads) k_g2p_items(FastView v, const float4* __restrict__ posm,
                                                            const float4* __restrict__ velid,
                                                            const float* __restrict__ mvf,
                                                            float4* __restrict__ posm_out,
                                                            float4* __restrict__ velid_out,
                                                            float* __restrict__ aff_out, const mpm_params P,
                                                            const mpm_wall_params W, DiffuseView dv) {
    const uint32_t nitems = v.counters[kCntItems];
    const uint32_t X = P.grid_X, SLICE = P.grid_X * P.grid_Y;
    const uint32_t G = (uint32_t)v.G;
    for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < nitems; it += gridDim.x * blockDim.x) {
        const uint4 item = v.items[it];
        int32_t ix, iy, iz;
        item_cell(v, item.x, ix, iy, iz);
        const uint32_t ibase = (uint32_t)(((iz - 1) * (int32_t)v.Y + (iy - 1)) * (int32_t)X + (ix - 1));
        float cv[81];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const uint32_t cidx = ibase + (uint32_t)k * SLICE + (uint32_t)j * X + (uint32_t)i;
                    const int q = (k * 9 + j * 3 + i) * 3;
                    if (cidx < G) {
                        const float* c = mvf + 3ull * cidx;
                        cv[q + 0] = c[0]; cv[q + 1] = c[1]; cv[q + 2] = c[2];
                    } else {
                        cv[q + 0] = 0.0f; cv[q + 1] = 0.0f; cv[q + 2] = 0.0f;
                    }
                }
        for (uint32_t kk = 0; kk < item.z; ++kk) {
            const uint32_t j = item.y + kk;
            const uint32_t slot = v.perm[j];
            const float4 q = posm[slot];
            const float4 vi = velid[slot];
            const PW w = particle_weights(q.x, q.y, q.z);
            const bool same = (w.cx == ix && w.cy == iy && w.cz == iz);
            const int32_t bx = w.cx - 1, by = w.cy - 1, bz = w.cz - 1;
            const uint32_t baseIdx = (uint32_t)((bz * (int32_t)v.Y + by) * (int32_t)X + bx);
            float gvx = 0.0f, gvy = 0.0f, gvz = 0.0f;
            float B[9] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float wzk = w.wz[k];
                const float dzk = __int2float_rn(bz + k) - q.z + 0.5f;
#pragma unroll
                for (int jj = 0; jj < 3; ++jj) {
                    const float wyzk = w.wy[jj] * wzk;
                    const float dyj = __int2float_rn(by + jj) - q.y + 0.5f;
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const float ww = w.wx[i] * wyzk;
                        const float dxi = __int2float_rn(bx + i) - q.x + 0.5f;
                        float cvx, cvy, cvz;
                        if (same) {
                            const int qq = (k * 9 + jj * 3 + i) * 3;
                            cvx = cv[qq + 0]; cvy = cv[qq + 1]; cvz = cv[qq + 2];
                        } else {
                            const uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)jj * X + (uint32_t)i;
                            cvx = cvy = cvz = 0.0f;
                            if (cidx < G) {
                                const float* c = mvf + 3ull * cidx;
                                cvx = c[0]; cvy = c[1]; cvz = c[2];
                            }
                        }
                        const float wvx = ww * cvx, wvy = ww * cvy, wvz = ww * cvz;
                        gvx += wvx; gvy += wvy; gvz += wvz;
                        B[0] += wvx * dxi; B[1] += wvx * dyj; B[2] += wvx * dzk;
                        B[3] += wvy * dxi; B[4] += wvy * dyj; B[5] += wvy * dzk;
                        B[6] += wvz * dxi; B[7] += wvz * dyj; B[8] += wvz * dzk;
                    }
                }
            }
            float* a = aff_out + 9ull * j;
#pragma unroll
            for (int e = 0; e < 9; ++e) a[e] = B[e] * 4.0f;
            f3 np, nv;
            g2p_finish(q, gvx, gvy, gvz, B, P, W, np, nv);
            posm_out[j] = make_float4(np.x, np.y, np.z, q.w);
            velid_out[j] = make_float4(nv.x, nv.y, nv.z, vi.w);
            bin_particle(v, j, np.x, np.y, np.z);
            if (dv.enabled && __float_as_uint(vi.w) < v.n) {
                const uint32_t id = __float_as_uint(vi.w);
                mpm_diffuse_particle r;
                if (spawn_record(id, make_float4(np.x, np.y, np.z, 0.0f), make_float4(nv.x, nv.y, nv.z, 0.0f), q.w,
                                 v.dens[j], dv.cmf, P, dv.gen, r)) {
                    dv.staging[id] = r;
                    atomicOr(&dv.spawn_bits[id >> 5], 1u << (id & 31u));
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Import / export between the internal sorted state and reference layouts.
// ---------------------------------------------------------------------------
__global__ void k_import(const float4* __restrict__ pos, const float4* __restrict__ vel,
                         const float* __restrict__ aff, const float* __restrict__ mass, float4* __restrict__ posm,
                         float4* __restrict__ velid, float* __restrict__ aff_out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i], v = vel[i];
    posm[i] = make_float4(p.x, p.y, p.z, mass[i]);
    velid[i] = make_float4(v.x, v.y, v.z, __uint_as_float(i));
#pragma unroll
    for (int e = 0; e < 9; ++e) aff_out[9ull * i + e] = aff[9ull * i + e];
}

__global__ void k_export(const float4* __restrict__ posm, const float4* __restrict__ velid,
                         const float* __restrict__ aff, const float* __restrict__ dens, float4* __restrict__ pos,
                         float4* __restrict__ vel, float* __restrict__ aff_out, float* __restrict__ mass,
                         float* __restrict__ dens_out, uint32_t n) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const float4 p = posm[j], v = velid[j];
    const uint32_t id = __float_as_uint(v.w);
    if (id >= n) return;
    pos[id] = make_float4(p.x, p.y, p.z, 0.0f);
    vel[id] = make_float4(v.x, v.y, v.z, 0.0f);
    mass[id] = p.w;
    if (dens_out) dens_out[id] = dens[j];
#pragma unroll
    for (int e = 0; e < 9; ++e) aff_out[9ull * id + e] = aff[9ull * j + e];
}

inline uint32_t cdiv(uint64_t a, uint32_t b) { return (uint32_t)((a + b - 1) / b); }

}  // namespace

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
cudaError_t fast_alloc(FastEngine& f, uint32_t X, uint32_t Y, uint32_t Z, uint32_t capacity, int device) {
    f.X = X; f.Y = Y; f.Z = Z;
    f.G = (uint64_t)X * Y * Z;
    f.ntx = cdiv(X, kTileX); f.nty = cdiv(Y, kTileY); f.ntz = cdiv(Z, kTileZ);
    f.ntiles = f.ntx * f.nty * f.ntz;
    f.capacity = capacity;
    const size_t N = capacity ? capacity : 1;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    f.item_blocks = (uint32_t)sms * 8;
    f.grid_blocks = (uint32_t)sms * 8;
    f.bin_blocks = (uint32_t)sms * 2;
    cudaError_t e = cudaSuccess;
    auto A = [&](auto** p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc((void**)p, bytes ? bytes : 16);
    };
    for (int b = 0; b < 2; ++b) {
        A(&f.posm[b], N * 16);
        A(&f.velid[b], N * 16);
        A(&f.aff[b], N * 36);
        A(&f.grid_i32[b], f.G * 16);
    }
    A(&f.dens, N * 4);
    A(&f.cell_count, (f.G + 1) * 4);
    A(&f.cell_start, f.G * 4);
    A(&f.key, N * 4);
    A(&f.rank, N * 4);
    A(&f.perm, N * 4);
    A(&f.items, N * 16);
    A(&f.tile_flags, f.ntiles * 4);
    A(&f.tile_occ_list, f.ntiles * 4);
    A(&f.tile_grid_list, f.ntiles * 4);
    A(&f.counters, 64);
    if (e != cudaSuccess) return e;
    f.cm_current = f.grid_i32[0];
    return cudaSuccess;
}

void fast_free(FastEngine& f) {
    void* ptrs[] = {f.posm[0], f.posm[1], f.velid[0], f.velid[1], f.aff[0], f.aff[1], f.grid_i32[0], f.grid_i32[1],
                    f.dens, f.cell_count, f.cell_start, f.key, f.rank, f.perm, f.items, f.tile_flags,
                    f.tile_occ_list, f.tile_grid_list, f.counters};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    f = FastEngine();
}

cudaError_t fast_import(FastEngine& f, const float4* pos, const float4* vel, const float* aff, const float* mass,
                        uint32_t n, cudaStream_t st) {
    FastView v = f.view();
    cudaError_t e = cudaMemsetAsync(f.cell_count, 0, (f.G + 1) * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(f.tile_flags, 0, f.ntiles * 4, st);
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) e = cudaMemsetAsync(f.grid_i32[b], 0, 16 * f.G, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(f.dens, 0, (size_t)(f.capacity ? f.capacity : 1) * 4, st);
    if (e != cudaSuccess) return e;
    f.cur = 0;
    f.gbuf = 0;
    f.n = n;
    f.cm_current = f.grid_i32[0];
    if (n) {
        k_import<<<cdiv(n, 256), 256, 0, st>>>(pos, vel, aff, mass, f.posm[0], f.velid[0], f.aff[0], n);
        k_import_keys<<<cdiv(n, 256), 256, 0, st>>>(v, f.posm[0], n);
        f.launches += 2;
    }
    f.dens_valid = false;
    return cudaGetLastError();
}

cudaError_t fast_export(FastEngine& f, float4* pos, float4* vel, float* aff, float* mass, float* dens,
                        cudaStream_t st) {
    if (f.n == 0) return cudaSuccess;
    k_export<<<cdiv(f.n, 256), 256, 0, st>>>(f.posm[f.cur], f.velid[f.cur], f.aff[f.cur], f.dens, pos, vel, aff,
                                            mass, dens, f.n);
    f.launches++;
    return cudaGetLastError();
}

cudaError_t fast_substep(Scene& s) {
    FastEngine& f = s.fast;
    cudaStream_t st = s.stream;
    const mpm_params& P = s.params;
    const mpm_wall_params& W = s.walls;
    FastView v = f.view();
    const uint32_t n = f.n;
    const int cur = f.cur, nxt = cur ^ 1;
    int32_t* cm = f.grid_i32[f.gbuf];
    int32_t* mv = cm + f.G;
    int32_t* cm_n = f.grid_i32[f.gbuf ^ 1];
    int32_t* mv_n = cm_n + f.G;
    const uint32_t gridItems = f.item_blocks;
    const bool hand = s.hand_active && s.hand_dims[0] > 0 && s.hand_dims[1] > 0 && s.hand_dims[2] > 0 &&
                      s.hand.is_on != 0u;
    int32_t hx0 = 1, hy0 = 1, hz0 = 1, hx1 = 0, hy1 = 0, hz1 = 0;
    if (hand) {   // cells APPLY_HAND may write (its dispatch box clipped to the grid)
        hx0 = s.hand.bbox_min_x; hy0 = s.hand.bbox_min_y; hz0 = s.hand.bbox_min_z;
        hx1 = s.hand.bbox_min_x + (s.hand_dims[0] + 3) / 4 * 4 - 1;
        hy1 = s.hand.bbox_min_y + (s.hand_dims[1] + 3) / 4 * 4 - 1;
        hz1 = s.hand.bbox_min_z + (s.hand_dims[2] + 3) / 4 * 4 - 1;
        hx1 = min(hx1, s.hand.bbox_max_x); hy1 = min(hy1, s.hand.bbox_max_y); hz1 = min(hz1, s.hand.bbox_max_z);
    }
    cudaError_t e;
    {
        Phase ph(s, MPM_PHASE_SORT);
        e = cudaMemsetAsync(f.counters, 0, 64, st);
        if (e != cudaSuccess) return e;
        k_tiles<<<cdiv(f.ntiles, 256), 256, 0, st>>>(v, hx0, hy0, hz0, hx1, hy1, hz1);
        k_bin_tiles<<<f.bin_blocks, kTileCells, 0, st>>>(v, f.chunk);
        if (n) k_scatter<<<cdiv(n, 256), 256, 0, st>>>(v, n);
        f.launches += n ? 3 : 2;
    }
    if (n) {
        Phase ph(s, MPM_PHASE_P2G_MASS);
        k_p2g_mass_items<<<gridItems, kItemThreads, 0, st>>>(v, f.posm[cur], cm);
        f.launches++;
    }
    {
        Phase ph(s, MPM_PHASE_DECODE_MASS);
        k_decode_tiles<<<f.grid_blocks, 256, 0, st>>>(v, cm, s.cmf);
        f.launches++;
    }
    if (n) {
        Phase ph(s, MPM_PHASE_P2G_MOM);
        k_p2g_mom_items<<<gridItems, kItemThreads, 0, st>>>(v, f.posm[cur], f.velid[cur], f.aff[cur], s.cmf, mv,
                                                            f.dens, P);
        f.launches++;
    }
    {
        Phase ph(s, MPM_PHASE_UPDATE_GRID);
        k_update_tiles<<<f.grid_blocks, 256, 0, st>>>(v, cm, mv, s.mvf, cm_n, mv_n, P, W);
        f.launches++;
    }
    if (hand) {
        Phase ph(s, MPM_PHASE_APPLY_HAND);
        e = launch_apply_hand(s);
        if (e != cudaSuccess) return e;
        f.launches++;
    }
    DiffuseState& d = s.diffuse;
    DiffuseView dv{};
    dv.enabled = d.enabled ? 1 : 0;
    if (d.enabled) {
        d.seed = d.seed + 1u;                 // diffuse-gpu.js:149
        dv.gen = d.gen;
        dv.gen.seed = d.seed;
        dv.staging = d.staging;
        dv.spawn_bits = d.spawn_bits;
        dv.cmf = s.cmf;
        e = cudaMemsetAsync(d.spawn_bits, 0, ((size_t)(n + 31) / 32) * 4, st);
        if (e != cudaSuccess) return e;
    }
    if (n) {
        Phase ph(s, MPM_PHASE_G2P);
        k_g2p_items<<<gridItems, kItemThreads, 0, st>>>(v, f.posm[cur], f.velid[cur], s.mvf, f.posm[nxt],
                                                        f.velid[nxt], f.aff[nxt], P, W, dv);
        f.launches++;
    }
    f.cur = nxt;
    f.gbuf ^= 1;
    f.cm_current = cm;
    f.dens_valid = true;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (d.enabled) e = launch_diffuse(s, /*eval=*/false);
    return e;
}

}  // namespace mpm
