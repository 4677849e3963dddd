// mpm_fast.cu — the binned, item-major MLS-MPM substep.
//
// Same arithmetic as mpm_kernels.cu (and so the same bits), organised for
// the B200:
//   * Work item = up to kMaxL particles of one cell.  One thread owns an
//     item: the 27 neighbour masses (P2G_MOM) or velocities (G2P) are loaded
//     once per item, and P2G contributions are summed in registers as i32
//     (the same wrapping sums the reference's atomics produce), flushed with
//     one atomic per (cell, component) per item.
//   * Items are bucketed by length, and particles are stored warp-interleaved:
//     the k-th particle of the item held by lane l of warp w of bucket b sits
//     at position pos_off[b] + w*32*b + k*32 + l.  All 32 lanes of a warp run
//     the same trip count and every per-particle load/store is coalesced.
//   * Within a bucket, items are ordered by (tile, cell) — a deterministic
//     layout that changes little from one substep to the next, so reading a
//     particle through the permutation (new position -> previous position)
//     stays nearly coalesced.  Cells holding more than kMaxL particles are
//     split into several items placed after the ordered ones.
//   * State (double-buffered, indexed by position):
//       posm  float4 (x, y, z, mass)    velid float4 (vx, vy, vz, id bits)
//       aff   9 planes                  dens  float
//     G2P writes the next state in the current layout and the binning cell
//     of every particle; the next substep counts particles per cell, turns
//     the counts into items and a permutation.
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

// Register-pressure strategies of the item kernels (compile-time; defaults
// are the measured best).
#ifndef MPM_MOM_LB
#define MPM_MOM_LB 1
#endif
#ifndef MPM_MOM_M27_SMEM
#define MPM_MOM_M27_SMEM 0
#endif
#ifndef MPM_MOM_ACC_SMEM
#define MPM_MOM_ACC_SMEM 1
#endif
#ifndef MPM_MOM_KLOOP
#define MPM_MOM_KLOOP 1
#endif
#ifndef MPM_G2P_LB
#define MPM_G2P_LB 3
#endif
#ifndef MPM_G2P_CV_SMEM
#define MPM_G2P_CV_SMEM 0
#endif

__device__ __forceinline__ uint32_t cell_of(int32_t x, int32_t y, int32_t z, uint32_t X, uint32_t Y) {
    return ((uint32_t)z * Y + (uint32_t)y) * X + (uint32_t)x;
}

__device__ __forceinline__ int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---------------------------------------------------------------------------
// Binning
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t tile_of(const FastView& v, int32_t cx, int32_t cy, int32_t cz) {
    return ((uint32_t)(cz / kTileZ) * v.nty + (uint32_t)(cy / kTileY)) * v.ntx + (uint32_t)(cx / kTileX);
}

// Mark a tile as holding particles for the next substep (bit 0).
__device__ __forceinline__ void mark_occupied(const FastView& v, uint32_t t) {
    if ((v.tile_flags[t] & 1u) == 0u) atomicOr(&v.tile_flags[t], 1u);
}

// Binning cell of a position (clamped into the grid; binning only).
__device__ __forceinline__ void bin_cell(const FastView& v, float px, float py, float pz, int32_t& cx, int32_t& cy,
                                         int32_t& cz) {
    cx = clampi(__float2int_rz(floorf(px)), 0, (int32_t)v.X - 1);
    cy = clampi(__float2int_rz(floorf(py)), 0, (int32_t)v.Y - 1);
    cz = clampi(__float2int_rz(floorf(pz)), 0, (int32_t)v.Z - 1);
}

// Identity-layout import: binning cells for the state just copied in.
__global__ void k_import_keys(FastView v, const float4* __restrict__ posm, uint32_t n) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j == 0) {
        v.ctrl->total_pos = n;
        v.ctrl->prev_total_pos = n;
    }
    if (j >= n) return;
    const float4 q = posm[j];
    int32_t cx, cy, cz;
    bin_cell(v, q.x, q.y, q.z, cx, cy, cz);
    v.key[j] = cell_of(cx, cy, cz, v.X, v.Y);
    mark_occupied(v, tile_of(v, cx, cy, cz));
}

// Rank of every particle of the current state within its binning cell.
__global__ void k_count(FastView v) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= v.ctrl->total_pos) return;
    const uint32_t c = v.key[i];
    if (c != kHole) v.rank[i] = atomicAdd(&v.cell_count[c], 1u);
}

// Occupied-tile list for the binning and the occupancy used by the scans.
// tile_flags bits: 0 occupied (set by G2P), 1 stencil now (set by the
// binning), 2 stencil last substep.
__global__ void k_tiles_occ(FastView v) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= v.ntiles) return;
    const uint32_t occ = v.tile_flags[t] & 1u;
    v.tile_occ[t] = occ;
    if (occ) v.tile_occ_list[atomicAdd(&v.ctrl->n_occ, 1u)] = t;
}

// One block per occupied tile, one thread per cell.  A cell with 1..kMaxL
// particles becomes one item in bucket `count`, ranked within the tile by
// cell index (match + warp prefix); the tile's per-bucket totals go to
// tile_hist.  Larger cells are split into items that take unordered slots
// after the ordered ones.  Also marks every tile the particles' 3x3x3
// stencils touch (bit 1) and clears the counts.
__global__ void __launch_bounds__(kTileCells) k_bin_cells(FastView v) {
    __shared__ uint32_t wcnt[kTileCells / 32][kMaxL + 1];
    __shared__ uint32_t dirs;
    const uint32_t nocc = v.ctrl->n_occ;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (uint32_t ti = blockIdx.x; ti < nocc; ti += gridDim.x) {
        const uint32_t t = v.tile_occ_list[ti];
        const uint32_t tx = t % v.ntx, ty = (t / v.ntx) % v.nty, tz = t / (v.ntx * v.nty);
        const uint32_t lx = threadIdx.x % kTileX, ly = (threadIdx.x / kTileX) % kTileY,
                       lz = threadIdx.x / (kTileX * kTileY);
        const uint32_t x = tx * kTileX + lx, y = ty * kTileY + ly, z = tz * kTileZ + lz;
        const bool inside = x < v.X && y < v.Y && z < v.Z;
        const uint32_t c = inside ? cell_of(x, y, z, v.X, v.Y) : 0u;
        uint32_t cnt = 0;
        if (inside) {
            cnt = v.cell_count[c];
            if (cnt) v.cell_count[c] = 0u;
        }
        if (threadIdx.x == 0) dirs = 0u;
        for (int b = lane; b <= kMaxL; b += 32) wcnt[wid][b] = 0u;
        __syncthreads();
        // neighbour tiles this cell's stencil reaches (3x3x3 direction bits)
        uint32_t m = 0;
        if (cnt) {
            const int dx = lx == 0 ? -1 : (lx == kTileX - 1 ? 1 : 0);
            const int dy = ly == 0 ? -1 : (ly == kTileY - 1 ? 1 : 0);
            const int dz = lz == 0 ? -1 : (lz == kTileZ - 1 ? 1 : 0);
            for (int kz = 0; kz <= (dz != 0); ++kz)
                for (int ky = 0; ky <= (dy != 0); ++ky)
                    for (int kx = 0; kx <= (dx != 0); ++kx)
                        m |= 1u << ((kz * dz + 1) * 9 + (ky * dy + 1) * 3 + (kx * dx + 1));
        }
        const uint32_t wm = __reduce_or_sync(0xffffffffu, m);
        if (lane == 0 && wm) atomicOr(&dirs, wm);
        const uint32_t b = (cnt >= 1 && cnt <= (uint32_t)kMaxL) ? cnt : 0u;
        const uint32_t grp = __match_any_sync(0xffffffffu, b);
        const uint32_t lrank = __popc(grp & ((1u << lane) - 1u));
        if (b && lrank == 0) wcnt[wid][b] = __popc(grp);
        __syncthreads();
        // exclusive prefix over the 32 warps for each length; tile totals
        if (threadIdx.x >= 1 && threadIdx.x <= kMaxL) {
            uint32_t acc = 0;
            for (int w = 0; w < kTileCells / 32; ++w) {
                const uint32_t k = wcnt[w][threadIdx.x];
                wcnt[w][threadIdx.x] = acc;
                acc += k;
            }
            v.tile_hist[(threadIdx.x - 1) * v.ntiles + t] = acc;
        }
        if (threadIdx.x < 27 && ((dirs >> threadIdx.x) & 1u)) {
            const int ox = (int)(threadIdx.x % 3) - 1, oy = (int)((threadIdx.x / 3) % 3) - 1,
                      oz = (int)(threadIdx.x / 9) - 1;
            const int nx = (int)tx + ox, ny = (int)ty + oy, nz = (int)tz + oz;
            if (nx >= 0 && ny >= 0 && nz >= 0 && nx < (int)v.ntx && ny < (int)v.nty && nz < (int)v.ntz) {
                const uint32_t nt = ((uint32_t)nz * v.nty + (uint32_t)ny) * v.ntx + (uint32_t)nx;
                if ((v.tile_flags[nt] & 2u) == 0u) atomicOr(&v.tile_flags[nt], 2u);
            }
        }
        __syncthreads();
        if (b) {
            v.cell_info[c] = make_uint4(b | (b << 8) | (1u << 16), wcnt[wid][b] + lrank, 0u, 0u);
        } else if (cnt) {
            // overpacked cell: q items of length L (the last of Llast), unordered tail slots
            const uint32_t q = (cnt + kMaxL - 1) / kMaxL;
            const uint32_t L = (cnt + q - 1) / q;
            const uint32_t Llast = cnt - (q - 1) * L;
            const uint32_t nL = (Llast == L) ? q : q - 1;
            const uint32_t idxL = atomicAdd(&v.ctrl->tail_cnt[L], nL);
            const uint32_t idxLast = (Llast != L) ? atomicAdd(&v.ctrl->tail_cnt[Llast], 1u) : idxL + q - 1;
            v.cell_info[c] = make_uint4(L | (Llast << 8) | (q << 16) | 0x80000000u, idxL, idxLast, 0u);
        }
        __syncthreads();
    }
}

// Grid-tile list (stencil tiles of this substep or the last one, plus the
// hand box); shifts the flags for the next substep.
__global__ void k_tiles_grid(FastView v, int32_t hx0, int32_t hy0, int32_t hz0, int32_t hx1, int32_t hy1,
                             int32_t hz1) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= v.ntiles) return;
    const uint32_t f = v.tile_flags[t];
    const uint32_t tx = t % v.ntx, ty = (t / v.ntx) % v.nty, tz = t / (v.ntx * v.nty);
    bool hand = false;
    if (hx0 <= hx1) {
        const int32_t x0 = (int32_t)tx * kTileX, y0 = (int32_t)ty * kTileY, z0 = (int32_t)tz * kTileZ;
        hand = x0 <= hx1 && x0 + kTileX - 1 >= hx0 && y0 <= hy1 && y0 + kTileY - 1 >= hy0 && z0 <= hz1 &&
               z0 + kTileZ - 1 >= hz0;
    }
    const bool now = (f & 2u) != 0 || hand || (v.tile_occ[t] != 0u);
    const bool prev = (f & 4u) != 0;
    if (now || prev) v.tile_grid_list[atomicAdd(&v.ctrl->n_grid, 1u)] = t;
    if (f != (now ? 4u : 0u)) v.tile_flags[t] = now ? 4u : 0u;
}

// Per length bucket (one block each): exclusive scan of the ordered item
// counts over all tiles in index order -> tile_base; total -> bucket_reg.
__global__ void __launch_bounds__(1024) k_tile_scan(FastView v) {
    __shared__ uint32_t ws[33];
    const uint32_t b = blockIdx.x + 1;
    const uint32_t* hist = v.tile_hist + (size_t)blockIdx.x * v.ntiles;
    uint32_t* base = v.tile_base + (size_t)blockIdx.x * v.ntiles;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t carry = 0;
    for (uint32_t t0 = 0; t0 < v.ntiles; t0 += 1024) {
        const uint32_t t = t0 + threadIdx.x;
        const uint32_t x = (t < v.ntiles && v.tile_occ[t]) ? hist[t] : 0u;
        uint32_t sc = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, sc, o);
            if (lane >= o) sc += y;
        }
        if (lane == 31) ws[wid] = sc;
        __syncthreads();
        if (wid == 0) {
            const uint32_t w = ws[lane];
            uint32_t ww = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, ww, o);
                if (lane >= o) ww += y;
            }
            ws[lane] = ww - w;
            if (lane == 31) ws[32] = ww;
        }
        __syncthreads();
        if (t < v.ntiles) base[t] = carry + ws[wid] + sc - x;
        carry += ws[32];
        __syncthreads();
    }
    if (threadIdx.x == 0) v.ctrl->bucket_reg[b] = carry;
}

// Bucket offsets (one warp): ordered + tail items, padded to whole warps.
__global__ void k_bucket_scan(Ctrl* ctrl) {
    const int lane = threadIdx.x;
    const uint32_t b = (uint32_t)lane;
    const uint32_t cnt = (b >= 1 && b <= (uint32_t)kMaxL) ? ctrl->bucket_reg[b] + ctrl->tail_cnt[b] : 0u;
    const uint32_t pad = (cnt + 31u) & ~31u;
    uint32_t si = pad, sp = pad * b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t yi = __shfl_up_sync(0xffffffffu, si, o);
        const uint32_t yp = __shfl_up_sync(0xffffffffu, sp, o);
        if (lane >= o) { si += yi; sp += yp; }
    }
    if (b <= (uint32_t)kMaxL + 1) {
        ctrl->item_off[b] = si - pad;
        ctrl->pos_off[b] = sp - pad * b;
        ctrl->bucket_cnt[b] = cnt;
    }
    const uint32_t ti = __shfl_sync(0xffffffffu, si, kMaxL);
    const uint32_t tp = __shfl_sync(0xffffffffu, sp, kMaxL);
    if (lane == 0) {
        ctrl->total_items = ti;
        ctrl->prev_total_pos = ctrl->total_pos;
        ctrl->total_pos = tp;
    }
}

__device__ __forceinline__ uint32_t item_position(const uint32_t* pos_off, uint32_t b, uint32_t idx) {
    return pos_off[b] + (idx >> 5) * 32u * b + (idx & 31u);
}

// perm[new position] = previous position for every particle; the first
// particle of each item also records the item's cell.
__global__ void k_scatter(FastView v) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    __shared__ uint32_t pos_off[kMaxL + 2];
    __shared__ uint32_t reg[kMaxL + 2];
    if (threadIdx.x < kMaxL + 2) {
        pos_off[threadIdx.x] = v.ctrl->pos_off[threadIdx.x];
        reg[threadIdx.x] = v.ctrl->bucket_reg[threadIdx.x];
    }
    __syncthreads();
    if (i >= v.ctrl->prev_total_pos) return;
    const uint32_t c = v.key[i];
    if (c == kHole) return;
    const uint32_t r = v.rank[i];
    const uint4 info = v.cell_info[c];
    uint32_t b, idx, kk;
    if (!(info.x & 0x80000000u)) {
        b = info.x & 0xFFu;
        const int32_t cx = (int32_t)(c % v.X), cy = (int32_t)((c / v.X) % v.Y), cz = (int32_t)(c / (v.X * v.Y));
        idx = v.tile_base[(b - 1) * v.ntiles + tile_of(v, cx, cy, cz)] + info.y;
        kk = r;
    } else {
        const uint32_t L = info.x & 0xFFu, Llast = (info.x >> 8) & 0xFFu, q = (info.x >> 16) & 0x7FFFu;
        const uint32_t it = r / L;
        kk = r - it * L;
        if (it + 1 < q || Llast == L) { b = L; idx = reg[L] + info.y + it; }
        else { b = Llast; idx = reg[Llast] + info.z; }
    }
    if (b < 1 || b > (uint32_t)kMaxL) return;
    const uint32_t pos = item_position(pos_off, b, idx) + kk * 32u;
    if (pos >= v.npos) return;
    v.perm[pos] = i;
    if (kk == 0 && v.cap_off[b] + idx < v.cap_off[b + 1]) v.bucket_items[v.cap_off[b] + idx] = c;
}

// Shared copy of the bucket tables for the item kernels.
struct ItemTables {
    uint32_t item_off[kMaxL + 2];
    uint32_t pos_off[kMaxL + 2];
    uint32_t cnt[kMaxL + 2];
};

__device__ __forceinline__ void load_tables(const FastView& v, ItemTables& t) {
    if (threadIdx.x < kMaxL + 2) {
        t.item_off[threadIdx.x] = v.ctrl->item_off[threadIdx.x];
        t.pos_off[threadIdx.x] = v.ctrl->pos_off[threadIdx.x];
        t.cnt[threadIdx.x] = (threadIdx.x >= 1 && threadIdx.x <= kMaxL) ? v.ctrl->bucket_cnt[threadIdx.x] : 0u;
    }
    __syncthreads();
}

struct ItemRef {
    uint32_t b, idx, cell, pbase;
    bool valid;
};

__device__ __forceinline__ ItemRef item_ref(const FastView& v, const ItemTables& t, uint32_t g) {
    ItemRef r;
    uint32_t b = 1;
    while (b < (uint32_t)kMaxL && g >= t.item_off[b + 1]) ++b;
    r.b = b;
    r.idx = g - t.item_off[b];
    r.valid = r.idx < t.cnt[b];
    r.cell = r.valid ? v.bucket_items[v.cap_off[b] + r.idx] : 0u;
    r.pbase = item_position(t.pos_off, b, r.idx);
    return r;
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

__device__ __forceinline__ void cell_xyz(const FastView& v, uint32_t c, int32_t& x, int32_t& y, int32_t& z) {
    x = (int32_t)(c % v.X);
    y = (int32_t)((c / v.X) % v.Y);
    z = (int32_t)(c / (v.X * v.Y));
}

// encode() without the clamp, for values already known to lie in +-20000.
__device__ __forceinline__ int32_t encode_unclamped(float v) { return __float2int_rz(v * kFixed); }

// ---------------------------------------------------------------------------
// P2G_MASS (shaders.js:242-274), item-major
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kItemThreads) k_p2g_mass_items(FastView v, const float4* __restrict__ posm,
                                                                 int32_t* __restrict__ cm) {
    __shared__ ItemTables tabs;
    load_tables(v, tabs);
    const uint32_t nitems = v.ctrl->total_items;
    const int32_t X = v.X, Y = v.Y, Z = v.Z;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < nitems; g += gridDim.x * blockDim.x) {
        const ItemRef it = item_ref(v, tabs, g);
        if (!it.valid) continue;
        int32_t ix, iy, iz;
        cell_xyz(v, it.cell, ix, iy, iz);
        int32_t acc[27];
#pragma unroll
        for (int q = 0; q < 27; ++q) acc[q] = 0;
        for (uint32_t k = 0; k < it.b; ++k) {
            const float4 p = posm[v.perm[it.pbase + k * 32u]];
            const PW w = particle_weights(p.x, p.y, p.z);
            // weight <= 0.4219: for |mass| < 47000 encode's clamp is the identity
            const bool safe = fabsf(p.w) < 47000.0f;
            if (w.cx == ix && w.cy == iy && w.cz == iz) {
                float wxy[9];
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int i = 0; i < 3; ++i) wxy[j * 3 + i] = w.wx[i] * w.wy[j];
                if (safe) {
#pragma unroll
                    for (int kk = 0; kk < 3; ++kk)
#pragma unroll
                        for (int q = 0; q < 9; ++q) acc[kk * 9 + q] += encode_unclamped(wxy[q] * w.wz[kk] * p.w);
                } else {
#pragma unroll
                    for (int kk = 0; kk < 3; ++kk)
#pragma unroll
                        for (int q = 0; q < 9; ++q) acc[kk * 9 + q] += encode(wxy[q] * w.wz[kk] * p.w);
                }
            } else {
                // particle outside its item's cell (positions outside the grid): per-particle path
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
    const uint32_t total = v.ctrl->n_grid * kTileCells;
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
    const uint32_t total = v.ctrl->n_grid * kTileCells;
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

#if MPM_MOM_ACC_SMEM
__shared__ int32_t g_sacc[81][kItemThreads];   // per-thread accumulator slots (experiment)
#endif

// The scatter part of P2G_MOM for one particle whose density is known.
// kDirect: atomics straight into the grid at the particle's own stencil;
// otherwise the 81 encoded contributions are added into acc.
// kClamp: full encode; without it the caller has bounded every value inside
// +-20000, where encode's clamp is the identity.
template <bool kDirect, bool kClamp>
__device__ __forceinline__ void mom_scatter(const PW& w, const MomIn& in, const float* s, float coef,
                                            const mpm_params& P, int32_t* acc, int32_t* mv, uint32_t baseIdx,
                                            uint32_t G) {
    const float s00 = s[0], s11 = s[1], s22 = s[2], s01 = s[3], s02 = s[4], s12 = s[5];
    const float dxs[3] = {-w.fx - 1.0f, -w.fx, 1.0f - w.fx};
    const float dys[3] = {-w.fy - 1.0f, -w.fy, 1.0f - w.fy};
    const float dzs[3] = {-w.fz - 1.0f, -w.fz, 1.0f - w.fz};
    const uint32_t X = P.grid_X, SLICE = P.grid_X * P.grid_Y;
#if MPM_MOM_KLOOP && MPM_MOM_ACC_SMEM
#pragma unroll 1
#else
#pragma unroll
#endif
    for (int k = 0; k < 3; ++k) {
        const float wzk = k == 0 ? w.wz[0] : (k == 1 ? w.wz[1] : w.wz[2]);
        const float dzk = k == 0 ? dzs[0] : (k == 1 ? dzs[1] : dzs[2]);
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
                const float vx = ww * (in.m * (in.vx + Qx) + fxf);
                const float vy = ww * (in.m * (in.vy + Qy) + fyf);
                const float vz = ww * (in.m * (in.vz + Qz) + fzf);
                const int32_t ex = kClamp ? encode(vx) : encode_unclamped(vx);
                const int32_t ey = kClamp ? encode(vy) : encode_unclamped(vy);
                const int32_t ez = kClamp ? encode(vz) : encode_unclamped(vz);
                if (kDirect) {
                    const uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)j * X + (uint32_t)i;
                    if (cidx < G) {
                        atomicAdd(mv + 3ull * cidx + 0, ex);
                        atomicAdd(mv + 3ull * cidx + 1, ey);
                        atomicAdd(mv + 3ull * cidx + 2, ez);
                    }
                } else {
                    const int q = (k * 9 + j * 3 + i) * 3;
#if MPM_MOM_ACC_SMEM
                    (void)acc;
                    atomicAdd(&g_sacc[q + 0][threadIdx.x], ex);
                    atomicAdd(&g_sacc[q + 1][threadIdx.x], ey);
                    atomicAdd(&g_sacc[q + 2][threadIdx.x], ez);
#else
                    acc[q + 0] += ex;
                    acc[q + 1] += ey;
                    acc[q + 2] += ez;
#endif
                }
            }
        }
    }
}

__global__ void __launch_bounds__(kItemThreads, MPM_MOM_LB) k_p2g_mom_items(FastView v, const float4* __restrict__ posm,
                                                                const float4* __restrict__ velid,
                                                                const float* __restrict__ aff,
                                                                const float* __restrict__ cmf,
                                                                int32_t* __restrict__ mv, float* __restrict__ dens,
                                                                const mpm_params P) {
    __shared__ ItemTables tabs;
    load_tables(v, tabs);
    const uint32_t nitems = v.ctrl->total_items;
    const uint32_t X = P.grid_X, SLICE = P.grid_X * P.grid_Y;
    const uint32_t G = (uint32_t)v.G;
    const size_t plane = v.npos;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < nitems; g += gridDim.x * blockDim.x) {
        const ItemRef it = item_ref(v, tabs, g);
        if (!it.valid) continue;
        int32_t ix, iy, iz;
        cell_xyz(v, it.cell, ix, iy, iz);
        const uint32_t ibase = (uint32_t)(((iz - 1) * (int32_t)v.Y + (iy - 1)) * (int32_t)X + (ix - 1));
#if MPM_MOM_M27_SMEM
        __shared__ float sm27[27][kItemThreads];
#define M27(q) sm27[q][threadIdx.x]
#else
        float m27[27];
#define M27(q) m27[q]
#endif
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const uint32_t cidx = ibase + (uint32_t)k * SLICE + (uint32_t)j * X + (uint32_t)i;
                    M27(k * 9 + j * 3 + i) = cidx < G ? cmf[cidx] : 0.0f;
                }
#if MPM_MOM_ACC_SMEM
#pragma unroll
        for (int q = 0; q < 81; ++q) g_sacc[q][threadIdx.x] = 0;
        int32_t* acc = nullptr;
#else
        int32_t acc[81];
#pragma unroll
        for (int q = 0; q < 81; ++q) acc[q] = 0;
#endif
        // software pipeline: the next particle's permutation entry and record are
        // loaded while the current one is processed
        uint32_t slot_n = it.b > 1 ? v.perm[it.pbase + 32u] : 0u;
        float4 p_c, v_c;
        float a_c[9];
        {
            const uint32_t slot = v.perm[it.pbase];
            p_c = posm[slot];
            v_c = velid[slot];
#pragma unroll
            for (int e = 0; e < 9; ++e) a_c[e] = aff[e * plane + slot];
        }
        for (uint32_t kk = 0; kk < it.b; ++kk) {
            const uint32_t pos = it.pbase + kk * 32u;
            float4 p_n = p_c, v_n = v_c;
            float a_n[9];
#pragma unroll
            for (int e = 0; e < 9; ++e) a_n[e] = a_c[e];
            uint32_t slot_nn = slot_n;
            if (kk + 1 < it.b) {
                p_n = posm[slot_n];
                v_n = velid[slot_n];
#pragma unroll
                for (int e = 0; e < 9; ++e) a_n[e] = aff[e * plane + slot_n];
                if (kk + 2 < it.b) slot_nn = v.perm[pos + 64u];
            }
            const float4 p = p_c;
            const MomIn in{v_c.x, v_c.y, v_c.z, p.w, a_c[0], a_c[1], a_c[2], a_c[3], a_c[4], a_c[5],
                           a_c[6], a_c[7], a_c[8]};
            p_c = p_n;
            v_c = v_n;
#pragma unroll
            for (int e = 0; e < 9; ++e) a_c[e] = a_n[e];
            slot_n = slot_nn;
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
                        for (int i = 0; i < 3; ++i) density += w.wx[i] * w.wy[jj] * w.wz[k] * M27(k * 9 + jj * 3 + i);
            } else {
                for (int k = 0; k < 3; ++k)
                    for (int jj = 0; jj < 3; ++jj)
                        for (int i = 0; i < 3; ++i) {
                            const uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)jj * X + (uint32_t)i;
                            const float cmass = cidx < G ? cmf[cidx] : 0.0f;
                            density += w.wx[i] * w.wy[jj] * w.wz[k] * cmass;
                        }
            }
            dens[pos] = density;
            if (density <= 1e-8f) continue;
            // stress (shaders.js:325-338)
            const float rest = P.rest_density;
            const float vol = __fdiv_rn(in.m, fmaxf(density, rest * 0.15f));
            float pressure = P.stiffness * (eos_pow(__fdiv_rn(density, rest), P.eos_power) - 1.0f);
            const float pFloor = density > rest * kCohesionGate ? kCohesionPressure : 0.0f;
            pressure = fmaxf(pressure, pFloor);
            const float visc = P.viscosity;
            float s[6];
            s[0] = -pressure + visc * (in.a00 + in.a00);
            s[1] = -pressure + visc * (in.a11 + in.a11);
            s[2] = -pressure + visc * (in.a22 + in.a22);
            s[3] = visc * (in.a01 + in.a10);
            s[4] = visc * (in.a02 + in.a20);
            s[5] = visc * (in.a12 + in.a21);
            const float coef = -vol * 4.0f * P.dt;
            // |value| <= 0.4219 * (|m| (|v| + 1.5 |A row|_1) + |coef| 1.5 |S row|_1): when that bound
            // is well inside +-20000 encode's clamp cannot change any value (NaN/Inf fail the test).
            const float am = fabsf(in.m), ac = fabsf(coef);
            const float bx = am * (fabsf(in.vx) + 1.5f * (fabsf(in.a00) + fabsf(in.a01) + fabsf(in.a02))) +
                             ac * 1.5f * (fabsf(s[0]) + fabsf(s[3]) + fabsf(s[4]));
            const float by = am * (fabsf(in.vy) + 1.5f * (fabsf(in.a10) + fabsf(in.a11) + fabsf(in.a12))) +
                             ac * 1.5f * (fabsf(s[3]) + fabsf(s[1]) + fabsf(s[5]));
            const float bz = am * (fabsf(in.vz) + 1.5f * (fabsf(in.a20) + fabsf(in.a21) + fabsf(in.a22))) +
                             ac * 1.5f * (fabsf(s[4]) + fabsf(s[5]) + fabsf(s[2]));
            const bool safe = fmaxf(bx, fmaxf(by, bz)) * 0.4222f < 19000.0f;
            if (same) {
                if (safe) mom_scatter<false, false>(w, in, s, coef, P, acc, mv, baseIdx, G);
                else mom_scatter<false, true>(w, in, s, coef, P, acc, mv, baseIdx, G);
            } else {
                mom_scatter<true, true>(w, in, s, coef, P, acc, mv, baseIdx, G);
            }
        }
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int jj = 0; jj < 3; ++jj)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const uint32_t cidx = ibase + (uint32_t)k * SLICE + (uint32_t)jj * X + (uint32_t)i;
                    const int q = (k * 9 + jj * 3 + i) * 3;
#if MPM_MOM_ACC_SMEM
                    const int32_t a0 = g_sacc[q + 0][threadIdx.x], a1 = g_sacc[q + 1][threadIdx.x],
                                  a2 = g_sacc[q + 2][threadIdx.x];
#else
                    const int32_t a0 = acc[q + 0], a1 = acc[q + 1], a2 = acc[q + 2];
#endif
                    if (cidx < G) {
                        if (a0) atomicAdd(mv + 3ull * cidx + 0, a0);
                        if (a1) atomicAdd(mv + 3ull * cidx + 1, a1);
                        if (a2) atomicAdd(mv + 3ull * cidx + 2, a2);
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

// G2P for one particle given its gathered grid velocity (shaders.js:636-700).
__device__ __forceinline__ void g2p_finish(const float4 q, float gvx, float gvy, float gvz, const mpm_params& P,
                                           const mpm_wall_params& W, f3& np, f3& nv) {
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

// G2P gather for a particle outside its item's cell (positions outside the
// grid): the reference's linear stencil index with a bounds guard.
__device__ __noinline__ void g2p_gather_direct(const PW& w, const float4 q, const float* __restrict__ mvf,
                                               const mpm_params& P, uint32_t G, float& gvx, float& gvy, float& gvz,
                                               float* B) {
    const uint32_t X = P.grid_X, SLICE = P.grid_X * P.grid_Y;
    const int32_t bx = w.cx - 1, by = w.cy - 1, bz = w.cz - 1;
    const uint32_t baseIdx = (uint32_t)((bz * (int32_t)P.grid_Y + by) * (int32_t)X + bx);
    for (int k = 0; k < 3; ++k) {
        const float wzk = w.wz[k];
        const float dzk = __int2float_rn(bz + k) - q.z + 0.5f;
        for (int jj = 0; jj < 3; ++jj) {
            const float wyzk = w.wy[jj] * wzk;
            const float dyj = __int2float_rn(by + jj) - q.y + 0.5f;
            for (int i = 0; i < 3; ++i) {
                const float ww = w.wx[i] * wyzk;
                const float dxi = __int2float_rn(bx + i) - q.x + 0.5f;
                const uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)jj * X + (uint32_t)i;
                float cvx = 0.0f, cvy = 0.0f, cvz = 0.0f;
                if (cidx < G) {
                    const float* c = mvf + 3ull * cidx;
                    cvx = c[0]; cvy = c[1]; cvz = c[2];
                }
                const float wvx = ww * cvx, wvy = ww * cvy, wvz = ww * cvz;
                gvx += wvx; gvy += wvy; gvz += wvz;
                B[0] += wvx * dxi; B[1] += wvx * dyj; B[2] += wvx * dzk;
                B[3] += wvy * dxi; B[4] += wvy * dyj; B[5] += wvy * dzk;
                B[6] += wvz * dxi; B[7] += wvz * dyj; B[8] += wvz * dzk;
            }
        }
    }
}

// Spawn decision + staging, out of line (most particles fail the density test first).
__device__ __noinline__ void spawn_eval(uint32_t id, f3 np, f3 nv, float m, float density,
                                        const mpm_params& P, const DiffuseView& dv) {
    mpm_diffuse_particle r;
    if (spawn_record(id, make_float4(np.x, np.y, np.z, 0.0f), make_float4(nv.x, nv.y, nv.z, 0.0f), m, density, dv.cmf,
                     P, dv.gen, r)) {
        dv.staging[id] = r;
        atomicOr(&dv.spawn_bits[id >> 5], 1u << (id & 31u));
    }
}

__global__ void __launch_bounds__(kItemThreads, MPM_G2P_LB) k_g2p_items(FastView v, const float4* __restrict__ posm,
                                                            const float4* __restrict__ velid,
                                                            const float* __restrict__ mvf,
                                                            float4* __restrict__ posm_out,
                                                            float4* __restrict__ velid_out,
                                                            float* __restrict__ aff_out, const mpm_params P,
                                                            const mpm_wall_params W, DiffuseView dv) {
    __shared__ ItemTables tabs;
    load_tables(v, tabs);
    const uint32_t nitems = v.ctrl->total_items;
    const uint32_t X = P.grid_X, SLICE = P.grid_X * P.grid_Y;
    const uint32_t G = (uint32_t)v.G;
    const size_t plane = v.npos;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < nitems; g += gridDim.x * blockDim.x) {
        const ItemRef it = item_ref(v, tabs, g);
        if (!it.valid) {
            // padding lane: mark its positions as holes for the next binning and the export
            for (uint32_t kk = 0; kk < it.b; ++kk) {
                const uint32_t pos = it.pbase + kk * 32u;
                if (pos < v.npos) {
                    v.key[pos] = kHole;
                    velid_out[pos] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(kHole));
                }
            }
            continue;
        }
        int32_t ix, iy, iz;
        cell_xyz(v, it.cell, ix, iy, iz);
        const uint32_t item_tile = tile_of(v, ix, iy, iz);
        mark_occupied(v, item_tile);
        const uint32_t ibase = (uint32_t)(((iz - 1) * (int32_t)v.Y + (iy - 1)) * (int32_t)X + (ix - 1));
#if MPM_G2P_CV_SMEM
        __shared__ float scv[81][kItemThreads];
#define CV(q) scv[q][threadIdx.x]
#else
        float cv[81];
#define CV(q) cv[q]
#endif
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
                        CV(q + 0) = c[0]; CV(q + 1) = c[1]; CV(q + 2) = c[2];
                    } else {
                        CV(q + 0) = 0.0f; CV(q + 1) = 0.0f; CV(q + 2) = 0.0f;
                    }
                }
        uint32_t slot_n = it.b > 1 ? v.perm[it.pbase + 32u] : 0u;
        float4 q_c, vi_c;
        {
            const uint32_t slot = v.perm[it.pbase];
            q_c = posm[slot];
            vi_c = velid[slot];
        }
        for (uint32_t kk = 0; kk < it.b; ++kk) {
            const uint32_t pos = it.pbase + kk * 32u;
            float4 q_n = q_c, vi_n = vi_c;
            uint32_t slot_nn = slot_n;
            if (kk + 1 < it.b) {
                q_n = posm[slot_n];
                vi_n = velid[slot_n];
                if (kk + 2 < it.b) slot_nn = v.perm[pos + 64u];
            }
            const float4 q = q_c;
            const float4 vi = vi_c;
            q_c = q_n;
            vi_c = vi_n;
            slot_n = slot_nn;
            const PW w = particle_weights(q.x, q.y, q.z);
            const bool same = (w.cx == ix && w.cy == iy && w.cz == iz);
            float gvx = 0.0f, gvy = 0.0f, gvz = 0.0f;
            float B[9] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
            if (same) {
                const int32_t bx = w.cx - 1, by = w.cy - 1, bz = w.cz - 1;
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
                            const int qq = (k * 9 + jj * 3 + i) * 3;
                            const float wvx = ww * CV(qq + 0), wvy = ww * CV(qq + 1), wvz = ww * CV(qq + 2);
                            gvx += wvx; gvy += wvy; gvz += wvz;
                            B[0] += wvx * dxi; B[1] += wvx * dyj; B[2] += wvx * dzk;
                            B[3] += wvy * dxi; B[4] += wvy * dyj; B[5] += wvy * dzk;
                            B[6] += wvz * dxi; B[7] += wvz * dyj; B[8] += wvz * dzk;
                        }
                    }
                }
            } else {
                g2p_gather_direct(w, q, mvf, P, G, gvx, gvy, gvz, B);
            }
#pragma unroll
            for (int e = 0; e < 9; ++e) aff_out[e * plane + pos] = B[e] * 4.0f;
            f3 np, nv;
            g2p_finish(q, gvx, gvy, gvz, P, W, np, nv);
            posm_out[pos] = make_float4(np.x, np.y, np.z, q.w);
            velid_out[pos] = make_float4(nv.x, nv.y, nv.z, vi.w);
            // binning of the new position
            int32_t cx, cy, cz;
            bin_cell(v, np.x, np.y, np.z, cx, cy, cz);
            const uint32_t c = cell_of(cx, cy, cz, v.X, v.Y);
            v.key[pos] = c;
            if (c != it.cell) {
                const uint32_t t = tile_of(v, cx, cy, cz);
                if (t != item_tile) mark_occupied(v, t);
            }
            if (dv.enabled && __float_as_uint(vi.w) < v.n) {
                const float density = v.dens[pos];
                // spawn_record's first test (shaders.js:806), checked inline
                if (density > 0.0f && density <= dv.gen.density_bubble_min)
                    spawn_eval(__float_as_uint(vi.w), np, nv, q.w, density, P, dv);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Import / export between the internal state and reference layouts.
// ---------------------------------------------------------------------------
__global__ void k_import(const float4* __restrict__ pos, const float4* __restrict__ vel,
                         const float* __restrict__ aff, const float* __restrict__ mass, float4* __restrict__ posm,
                         float4* __restrict__ velid, float* __restrict__ aff_out, uint32_t n, size_t plane) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i], v = vel[i];
    posm[i] = make_float4(p.x, p.y, p.z, mass[i]);
    velid[i] = make_float4(v.x, v.y, v.z, __uint_as_float(i));
#pragma unroll
    for (int e = 0; e < 9; ++e) aff_out[e * plane + i] = aff[9ull * i + e];
}

__global__ void k_export(const Ctrl* __restrict__ ctrl, const float4* __restrict__ posm,
                         const float4* __restrict__ velid, const float* __restrict__ aff,
                         const float* __restrict__ dens, float4* __restrict__ pos, float4* __restrict__ vel,
                         float* __restrict__ aff_out, float* __restrict__ mass, float* __restrict__ dens_out,
                         uint32_t n, size_t plane) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ctrl->total_pos || j >= plane) return;
    const float4 p = posm[j], v = velid[j];
    const uint32_t id = __float_as_uint(v.w);
    if (id >= n) return;   // padding position
    pos[id] = make_float4(p.x, p.y, p.z, 0.0f);
    vel[id] = make_float4(v.x, v.y, v.z, 0.0f);
    mass[id] = p.w;
    if (dens_out) dens_out[id] = dens[j];
#pragma unroll
    for (int e = 0; e < 9; ++e) aff_out[9ull * id + e] = aff[e * plane + j];
}

inline uint32_t cdiv(uint64_t a, uint32_t b) { return (uint32_t)((a + b - 1) / b); }

}  // namespace

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
cudaError_t fast_alloc(FastEngine& f, uint32_t X, uint32_t Y, uint32_t Z, uint32_t capacity, int device) {
    f.X = X; f.Y = Y; f.Z = Z;
    f.G = (uint64_t)X * Y * Z;
    f.ntx = cdiv(X, kTileX); f.nty = cdiv(Y, kTileY); f.ntz = cdiv(Z, kTileZ);
    f.ntiles = f.ntx * f.nty * f.ntz;
    f.capacity = capacity;
    f.npos = capacity + kPosSlack;
    uint32_t off = 0;
    f.cap_off[0] = 0;
    for (int b = 1; b <= kMaxL; ++b) {
        f.cap_off[b] = off;
        off += capacity / b + 1;
    }
    f.cap_off[kMaxL + 1] = off;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    f.item_blocks = (uint32_t)sms * 8;
    f.grid_blocks = (uint32_t)sms * 8;
    f.bin_blocks = (uint32_t)sms * 2;
    const size_t P = f.npos;
    cudaError_t e = cudaSuccess;
    auto A = [&](auto** p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc((void**)p, bytes ? bytes : 16);
    };
    for (int b = 0; b < 2; ++b) {
        A(&f.posm[b], P * 16);
        A(&f.velid[b], P * 16);
        A(&f.aff[b], P * 36);
        A(&f.grid_i32[b], f.G * 16);
    }
    A(&f.dens, P * 4);
    A(&f.cell_count, (f.G + 1) * 4);
    A(&f.cell_info, f.G * 16);
    A(&f.bucket_items, (size_t)off * 4);
    A(&f.key, P * 4);
    A(&f.rank, P * 4);
    A(&f.perm, P * 4);
    A(&f.tile_flags, f.ntiles * 4);
    A(&f.tile_occ, f.ntiles * 4);
    A(&f.tile_hist, (size_t)kMaxL * f.ntiles * 4);
    A(&f.tile_base, (size_t)kMaxL * f.ntiles * 4);
    A(&f.tile_occ_list, f.ntiles * 4);
    A(&f.tile_grid_list, f.ntiles * 4);
    A(&f.ctrl, sizeof(Ctrl));
    if (e != cudaSuccess) return e;
    f.cm_current = f.grid_i32[0];
    return cudaSuccess;
}

void fast_free(FastEngine& f) {
    void* ptrs[] = {f.posm[0], f.posm[1], f.velid[0], f.velid[1], f.aff[0], f.aff[1], f.grid_i32[0], f.grid_i32[1],
                    f.dens, f.cell_count, f.cell_info, f.bucket_items, f.key, f.rank, f.perm, f.tile_flags, f.tile_occ, f.tile_hist, f.tile_base,
                    f.tile_occ_list, f.tile_grid_list, f.ctrl};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    f = FastEngine();
}

cudaError_t fast_import(FastEngine& f, const float4* pos, const float4* vel, const float* aff, const float* mass,
                        uint32_t n, cudaStream_t st) {
    f.n = n;
    FastView v = f.view();
    cudaError_t e = cudaMemsetAsync(f.cell_count, 0, (f.G + 1) * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(f.tile_flags, 0, f.ntiles * 4, st);
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) e = cudaMemsetAsync(f.grid_i32[b], 0, 16 * f.G, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(f.dens, 0, (size_t)f.npos * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(f.ctrl, 0, sizeof(Ctrl), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(f.key, 0xFF, (size_t)f.npos * 4, st);
    // every permutation entry always names a valid position, even if a bug left one unwritten
    if (e == cudaSuccess) e = cudaMemsetAsync(f.perm, 0, (size_t)f.npos * 4, st);
    if (e != cudaSuccess) return e;
    f.gbuf = 0;
    f.cur = 0;
    f.cm_current = f.grid_i32[0];
    if (n) k_import<<<cdiv(n, 256), 256, 0, st>>>(pos, vel, aff, mass, f.posm[0], f.velid[0], f.aff[0], n, f.npos);
    k_import_keys<<<cdiv(n ? n : 1, 256), 256, 0, st>>>(v, f.posm[0], n);   // also sets the layout size
    f.launches += n ? 2 : 1;
    f.dens_valid = false;
    return cudaGetLastError();
}

cudaError_t fast_export(FastEngine& f, float4* pos, float4* vel, float* aff, float* mass, float* dens,
                        cudaStream_t st) {
    if (f.n == 0) return cudaSuccess;
    k_export<<<cdiv(f.npos, 256), 256, 0, st>>>(f.ctrl, f.posm[f.cur], f.velid[f.cur], f.aff[f.cur], f.dens, pos, vel,
                                                aff, mass, dens, f.n, f.npos);
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
    if (hand) {   // cells APPLY_HAND may write (its dispatch box clipped to bbox_max)
        hx0 = s.hand.bbox_min_x; hy0 = s.hand.bbox_min_y; hz0 = s.hand.bbox_min_z;
        hx1 = min(s.hand.bbox_min_x + (s.hand_dims[0] + 3) / 4 * 4 - 1, s.hand.bbox_max_x);
        hy1 = min(s.hand.bbox_min_y + (s.hand_dims[1] + 3) / 4 * 4 - 1, s.hand.bbox_max_y);
        hz1 = min(s.hand.bbox_min_z + (s.hand_dims[2] + 3) / 4 * 4 - 1, s.hand.bbox_max_z);
    }
    cudaError_t e;
    {
        Phase ph(s, MPM_PHASE_SORT);
        e = cudaMemsetAsync(f.ctrl, 0, kCtrlZeroBytes, st);
        if (e != cudaSuccess) return e;
        k_count<<<cdiv(f.npos, 256), 256, 0, st>>>(v);
        k_tiles_occ<<<cdiv(f.ntiles, 256), 256, 0, st>>>(v);
        k_bin_cells<<<f.bin_blocks, kTileCells, 0, st>>>(v);
        k_tiles_grid<<<cdiv(f.ntiles, 256), 256, 0, st>>>(v, hx0, hy0, hz0, hx1, hy1, hz1);
        k_tile_scan<<<kMaxL, 1024, 0, st>>>(v);
        k_bucket_scan<<<1, 32, 0, st>>>(f.ctrl);
        k_scatter<<<cdiv(f.npos, 256), 256, 0, st>>>(v);
        f.launches += 7;
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
        if (n) {
            e = cudaMemsetAsync(d.spawn_bits, 0, ((size_t)(n + 31) / 32) * 4, st);
            if (e != cudaSuccess) return e;
        }
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
