/*
 * mpm_oracle.cpp — CPU restatement of the reference's MLS-MPM compute passes.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * path; it is imported by tests/, by __graft_entry__.smoke() and by bench.py's
 * CPU-baseline leg, and by nothing else.  The product never calls it.
 *
 * Each function restates one WGSL compute shader of shaders.js (line ranges in
 * the comments) operation for operation: same evaluation order, same
 * association, IEEE-754 binary32 arithmetic with no FMA contraction (build
 * with -ffp-contract=off), IEEE division and sqrt.  One thread of the
 * reference's dispatch becomes one iteration of a loop in ascending
 * global_invocation_id order, which is a legal execution of the WGSL (the only
 * cross-thread interaction is atomics; integer adds commute, and the diffuse
 * free-list pops/pushes then happen in ascending particle/slot order — the
 * "canonical" slot order the CUDA path reproduces with prefix sums).
 *
 * The template parameter T is float for the parity oracle and double for the
 * f64 drift reference (the reference's JS numbers are IEEE doubles).
 *
 * Pinning: the same passes compiled straight from the reference's shader
 * source (oracle/wgsl2cpp.py -> oracle/_ref) are compared with this file
 * bit-for-bit in tests/test_oracle_pin.py, and golden digests produced from
 * that build live in tests/golden/.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/mpm_types.h"

namespace {

/* ---- WGSL scalar semantics ------------------------------------------------ */

// max/min: if one operand is NaN the other is returned (WGSL builtin spec).
template <class T> inline T wmax(T a, T b) { return std::fmax(a, b); }
template <class T> inline T wmin(T a, T b) { return std::fmin(a, b); }
// clamp(e, lo, hi) = min(max(e, lo), hi)
template <class T> inline T wclamp(T e, T lo, T hi) { return wmin(wmax(e, lo), hi); }

// i32(f): round toward zero, saturate, NaN -> 0 (what cvt.rzi.s32.f32 does).
template <class T> inline int32_t to_i32(T x) {
    if (x != x) return 0;
    if (x >= T(2147483647.0)) return INT32_MAX;
    if (x <= T(-2147483648.0)) return INT32_MIN;
    return (int32_t)x;
}

// shaders.js:15-25 encode/decode (FIXED = 1e5, clamp +-20000).
template <class T> inline int32_t encode(T v) {
    T c = wclamp(v, T(-20000.0), T(20000.0));
    return to_i32(c * T(100000.0));
}
template <class T> inline T decode(int32_t v) { return T(v) / T(100000.0); }

// Wrapping i32 add (WGSL atomicAdd on i32 wraps).
inline int32_t wrap_add(int32_t a, int32_t b) {
    return (int32_t)((uint32_t)a + (uint32_t)b);
}

// pow(x, eos_power): the reference's default EOS_POWER is 1 (fluid-gpu.js:27);
// x^1 is x exactly, so that case never calls a libm pow.
template <class T> inline T eos_pow(T x, T e) {
    if (e == T(1)) return x;
    return std::pow(x, e);
}

template <class T> struct V3 { T x, y, z; };
template <class T> inline V3<T> v3(T x, T y, T z) { return V3<T>{x, y, z}; }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> mul(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> mul(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline T length(V3<T> a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

/* ---- quadratic B-spline weights: shaders.js:53-59 and 222-238 ------------- */

template <class T> struct BaseW {
    int32_t bx, by, bz;
    T fx, fy, fz;
    T wx[3], wy[3], wz[3];
};

template <class T> inline void qw(T f, T* w) {
    w[0] = T(0.5) * (T(0.5) - f) * (T(0.5) - f);
    w[1] = T(0.75) - f * f;
    w[2] = T(0.5) * (T(0.5) + f) * (T(0.5) + f);
}

template <class T> inline BaseW<T> compute_weights(T px, T py, T pz) {
    BaseW<T> o;
    int32_t cx = to_i32(std::floor(px)), cy = to_i32(std::floor(py)), cz = to_i32(std::floor(pz));
    o.bx = cx - 1; o.by = cy - 1; o.bz = cz - 1;
    o.fx = px - T(cx) - T(0.5);
    o.fy = py - T(cy) - T(0.5);
    o.fz = pz - T(cz) - T(0.5);
    qw(o.fx, o.wx); qw(o.fy, o.wy); qw(o.fz, o.wz);
    return o;
}

/* ---- moving-wall helpers: shaders.js:135-193 ------------------------------ */

template <class T> struct WallT {
    V3<T> c; T cy, sy, cp, sp;
    V3<T> mn, mx, vel, om;
};

template <class T> inline WallT<T> load_wall(const mpm_wall& w) {
    WallT<T> o;
    o.c = v3<T>(w.center_cy[0], w.center_cy[1], w.center_cy[2]);
    o.cy = w.center_cy[3]; o.sy = w.lmin_sy[3]; o.cp = w.lmax_cp[3]; o.sp = w.vel_sp[3];
    o.mn = v3<T>(w.lmin_sy[0], w.lmin_sy[1], w.lmin_sy[2]);
    o.mx = v3<T>(w.lmax_cp[0], w.lmax_cp[1], w.lmax_cp[2]);
    o.vel = v3<T>(w.vel_sp[0], w.vel_sp[1], w.vel_sp[2]);
    o.om = v3<T>(w.omega_pad[0], w.omega_pad[1], w.omega_pad[2]);
    return o;
}

template <class T> inline V3<T> wall_to_local(V3<T> p, const WallT<T>& w) {
    V3<T> d = p - w.c;
    T x1 = w.cy * d.x - w.sy * d.z;
    T z1 = w.sy * d.x + w.cy * d.z;
    return {x1, w.cp * d.y + w.sp * z1, -w.sp * d.y + w.cp * z1};
}

template <class T> inline V3<T> wall_to_world_dir(V3<T> v, const WallT<T>& w) {
    T y1 = w.cp * v.y - w.sp * v.z;
    T z1 = w.sp * v.y + w.cp * v.z;
    return {w.cy * v.x + w.sy * z1, y1, -w.sy * v.x + w.cy * z1};
}

template <class T> inline V3<T> wall_vel_at(V3<T> p, const WallT<T>& w) {
    V3<T> r = p - w.c;
    return w.vel + cross(w.om, r);
}

// returns normal in n, signed distance as result
template <class T> inline T wall_sdf_normal(V3<T> lp, V3<T> mn, V3<T> mx, V3<T>& n) {
    V3<T> dmin = mn - lp;
    V3<T> dmax = lp - mx;
    V3<T> q = {wmax(dmin.x, dmax.x), wmax(dmin.y, dmax.y), wmax(dmin.z, dmax.z)};
    T qmax = wmax(q.x, wmax(q.y, q.z));
    if (qmax > T(0)) {
        V3<T> nearest = {wclamp(lp.x, mn.x, mx.x), wclamp(lp.y, mn.y, mx.y), wclamp(lp.z, mn.z, mx.z)};
        V3<T> diff = lp - nearest;
        T len = length(diff);
        if (len > T(1e-6)) n = {diff.x / len, diff.y / len, diff.z / len};
        else n = {T(0), T(1), T(0)};
        return len;
    }
    n = {T(0), T(1), T(0)};
    if (qmax == q.x)      n = {dmax.x > dmin.x ? T(1) : T(-1), T(0), T(0)};
    else if (qmax == q.y) n = {T(0), dmax.y > dmin.y ? T(1) : T(-1), T(0)};
    else                  n = {T(0), T(0), dmax.z > dmin.z ? T(1) : T(-1)};
    return qmax;
}

inline uint32_t wall_count(const mpm_wall_params* wp) {
    if (!wp) return 0;
    float c = wp->count_pad[0];
    if (!(c > 0.0f)) return 0;           // u32(f32): negative/NaN -> 0
    uint32_t n = (uint32_t)c;
    return n > MPM_MAX_WALLS ? MPM_MAX_WALLS : n;
}

template <class T> struct Scene {
    const mpm_params* P;
    const mpm_wall_params* W;
    T* pos; T* vel; T* aff; const T* mass; T* dens;
    int32_t* mv; int32_t* cm; T* mvf; T* cmf;
    int threads;
};

/* ---- CLEAR: shaders.js:196-210 -------------------------------------------- */
template <class T> void pass_clear(Scene<T>& s) {
    const size_t G = (size_t)s.P->grid_X * s.P->grid_Y * s.P->grid_Z;
    std::memset(s.cm, 0, G * sizeof(int32_t));
    std::memset(s.mv, 0, 3 * G * sizeof(int32_t));
}

/* ---- P2G_MASS: shaders.js:242-274 ----------------------------------------- */
template <class T> void pass_p2g_mass(Scene<T>& s) {
    const mpm_params& P = *s.P;
    const int32_t X = P.grid_X, Y = P.grid_Y, Z = P.grid_Z;
    const int64_t n = P.particle_num;
#pragma omp parallel for schedule(static) num_threads(s.threads) if (s.threads > 1)
    for (int64_t p = 0; p < n; ++p) {
        T pm = s.mass[p];
        BaseW<T> bw = compute_weights(s.pos[4 * p], s.pos[4 * p + 1], s.pos[4 * p + 2]);
        for (int k = 0; k < 3; ++k) {
            int32_t cz = bw.bz + k;
            for (int j = 0; j < 3; ++j) {
                int32_t cy = bw.by + j;
                for (int i = 0; i < 3; ++i) {
                    int32_t cx = bw.bx + i;
                    if (cx < 0 || cx >= X || cy < 0 || cy >= Y || cz < 0 || cz >= Z) continue;
                    int32_t idx = (cz * Y + cy) * X + cx;
                    T w = bw.wx[i] * bw.wy[j] * bw.wz[k];
                    int32_t e = encode(w * pm);
                    if (s.threads > 1) __atomic_fetch_add(&s.cm[idx], e, __ATOMIC_RELAXED);
                    else s.cm[idx] = wrap_add(s.cm[idx], e);
                }
            }
        }
    }
}

/* ---- DECODE_MASS: shaders.js:373-384 -------------------------------------- */
template <class T> void pass_decode_mass(Scene<T>& s) {
    const int64_t G = (int64_t)s.P->grid_X * s.P->grid_Y * s.P->grid_Z;
#pragma omp parallel for schedule(static) num_threads(s.threads) if (s.threads > 1)
    for (int64_t i = 0; i < G; ++i) s.cmf[i] = decode<T>(s.cm[i]);
}

/* ---- P2G_MOM: shaders.js:276-371 ------------------------------------------ */
template <class T> void pass_p2g_mom(Scene<T>& s) {
    const mpm_params& P = *s.P;
    const uint32_t X = P.grid_X, Y = P.grid_Y;
    const int64_t n = P.particle_num;
    const T rest = P.rest_density, stiff = P.stiffness, eos = P.eos_power, visc = P.viscosity, dt = P.dt;
#pragma omp parallel for schedule(static) num_threads(s.threads) if (s.threads > 1)
    for (int64_t p = 0; p < n; ++p) {
        const T vx = s.vel[4 * p], vy = s.vel[4 * p + 1], vz = s.vel[4 * p + 2];
        const T mass = s.mass[p];
        const T* a = s.aff + 9 * p;
        const T a00 = a[0], a01 = a[1], a02 = a[2], a10 = a[3], a11 = a[4], a12 = a[5], a20 = a[6], a21 = a[7], a22 = a[8];
        BaseW<T> bw = compute_weights(s.pos[4 * p], s.pos[4 * p + 1], s.pos[4 * p + 2]);
        const uint32_t SLICE = X * Y;
        const uint32_t baseIdx = (uint32_t)((bw.bz * (int32_t)Y + bw.by) * (int32_t)X + bw.bx);

        T density = T(0);
        for (int k = 0; k < 3; ++k)
            for (int j = 0; j < 3; ++j)
                for (int i = 0; i < 3; ++i) {
                    uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)j * X + (uint32_t)i;
                    density += bw.wx[i] * bw.wy[j] * bw.wz[k] * s.cmf[cidx];
                }
        s.dens[p] = density;
        if (density <= T(1e-8)) continue;

        T vol = mass / wmax(density, rest * T(0.15));
        T pressure = stiff * (eos_pow(density / rest, eos) - T(1.0));
        T pFloor = (density > rest * T(0.7)) ? T(-0.1) : T(0.0);
        pressure = wmax(pressure, pFloor);

        T s00 = -pressure + visc * (a00 + a00);
        T s11 = -pressure + visc * (a11 + a11);
        T s22 = -pressure + visc * (a22 + a22);
        T s01 = visc * (a01 + a10);
        T s02 = visc * (a02 + a20);
        T s12 = visc * (a12 + a21);
        T coef = -vol * T(4.0) * dt;

        T dxs[3] = {-bw.fx - T(1.0), -bw.fx, T(1.0) - bw.fx};
        T dys[3] = {-bw.fy - T(1.0), -bw.fy, T(1.0) - bw.fy};
        T dzs[3] = {-bw.fz - T(1.0), -bw.fz, T(1.0) - bw.fz};

        for (int k = 0; k < 3; ++k) {
            T wzk = bw.wz[k], dzk = dzs[k];
            for (int j = 0; j < 3; ++j) {
                T wyzk = bw.wy[j] * wzk, dyj = dys[j];
                for (int i = 0; i < 3; ++i) {
                    T w = bw.wx[i] * wyzk;
                    T dxi = dxs[i];
                    uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)j * X + (uint32_t)i;
                    T Qx = a00 * dxi + a01 * dyj + a02 * dzk;
                    T Qy = a10 * dxi + a11 * dyj + a12 * dzk;
                    T Qz = a20 * dxi + a21 * dyj + a22 * dzk;
                    T fxf = coef * (s00 * dxi + s01 * dyj + s02 * dzk);
                    T fyf = coef * (s01 * dxi + s11 * dyj + s12 * dzk);
                    T fzf = coef * (s02 * dxi + s12 * dyj + s22 * dzk);
                    int32_t ex = encode(w * (mass * (vx + Qx) + fxf));
                    int32_t ey = encode(w * (mass * (vy + Qy) + fyf));
                    int32_t ez = encode(w * (mass * (vz + Qz) + fzf));
                    int32_t* m = s.mv + 3 * (size_t)cidx;
                    if (s.threads > 1) {
                        __atomic_fetch_add(&m[0], ex, __ATOMIC_RELAXED);
                        __atomic_fetch_add(&m[1], ey, __ATOMIC_RELAXED);
                        __atomic_fetch_add(&m[2], ez, __ATOMIC_RELAXED);
                    } else {
                        m[0] = wrap_add(m[0], ex); m[1] = wrap_add(m[1], ey); m[2] = wrap_add(m[2], ez);
                    }
                }
            }
        }
    }
}

/* ---- UPDATE_GRID: shaders.js:435-513 -------------------------------------- */
template <class T> void pass_update_grid(Scene<T>& s) {
    const mpm_params& P = *s.P;
    const uint32_t X = P.grid_X, Y = P.grid_Y, Z = P.grid_Z;
    const int64_t G = (int64_t)X * Y * Z;
    const uint32_t nw = wall_count(s.W);
    WallT<T> walls[MPM_MAX_WALLS];
    for (uint32_t i = 0; i < nw; ++i) walls[i] = load_wall<T>(s.W->walls[i]);
    const T gdt = T(P.gravity) * T(P.dt);
#pragma omp parallel for schedule(static) num_threads(s.threads) if (s.threads > 1)
    for (int64_t idx = 0; idx < G; ++idx) {
        T cmv = decode<T>(s.cm[idx]);
        T* out = s.mvf + 3 * idx;
        if (cmv <= T(0)) { out[0] = T(0); out[1] = T(0); out[2] = T(0); continue; }
        T vx = decode<T>(s.mv[3 * idx + 0]) / cmv;
        T vy = decode<T>(s.mv[3 * idx + 1]) / cmv;
        T vz = decode<T>(s.mv[3 * idx + 2]) / cmv;
        vy += gdt;
        const int32_t cx = (int32_t)(idx % X);
        const int32_t cy = (int32_t)((idx / X) % Y);
        const int32_t cz = (int32_t)(idx / ((int64_t)X * Y));
        if (cx < 2 || cx > (int32_t)X - 3) vx = T(0);
        if (cy < 2 && vy < T(0)) vy = T(0);
        if (cy > (int32_t)Y - 3 && vy > T(0)) vy = T(0);
        if (cz < 2 || cz > (int32_t)Z - 3) vz = T(0);
        if (cy < 2) { vx *= T(0.85); vz *= T(0.9); }

        V3<T> cellPos = {T(cx) + T(0.5), T(cy) + T(0.5), T(cz) + T(0.5)};
        V3<T> wv = {vx, vy, vz};
        for (uint32_t wi = 0; wi < nw; ++wi) {
            const WallT<T>& w = walls[wi];
            V3<T> lp = wall_to_local(cellPos, w);
            V3<T> mn = w.mn, mx = w.mx;
            if (lp.x < mn.x - T(1) || lp.y < mn.y - T(1) || lp.z < mn.z - T(1) ||
                lp.x > mx.x + T(1) || lp.y > mx.y + T(1) || lp.z > mx.z + T(1)) continue;
            V3<T> wvel = wall_vel_at(cellPos, w);
            V3<T> n;
            T sw = wall_sdf_normal(lp, mn, mx, n);
            if (sw < T(0)) {
                wv = wvel;
            } else if (sw < T(1)) {
                V3<T> nn = wall_to_world_dir(n, w);
                V3<T> vrel = wv - wvel;
                T vn = dot(vrel, nn);
                if (vn < T(0)) wv = wv - mul(vn, nn);
            }
        }
        out[0] = wv.x; out[1] = wv.y; out[2] = wv.z;
    }
}

/* ---- APPLY_HAND: shaders.js:394-433 (dispatch: fluid-gpu.js:670-678) ------ */
template <class T> void pass_apply_hand(Scene<T>& s, const mpm_hand_params* h, const int32_t dims[3]) {
    if (!h || dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0) return;
    if (h->is_on == 0u) return;
    const mpm_params& P = *s.P;
    const int32_t X = P.grid_X, Y = P.grid_Y, Z = P.grid_Z;
    // dispatch extent: ceil(dim/4) workgroups of 4 per axis
    const int32_t ex = (dims[0] + 3) / 4 * 4, ey = (dims[1] + 3) / 4 * 4, ez = (dims[2] + 3) / 4 * 4;
    V3<T> hand_pos = {T(h->px), T(h->py), T(h->pz)};
    V3<T> dv = hand_pos - v3<T>(h->ex, h->ey, h->ez);
    T dl = length(dv);
    V3<T> ray_dir = {dv.x / dl, dv.y / dl, dv.z / dl};
    for (int32_t gz = 0; gz < ez; ++gz)
        for (int32_t gy = 0; gy < ey; ++gy)
            for (int32_t gx = 0; gx < ex; ++gx) {
                int32_t cx = h->bbox_min_x + gx, cy = h->bbox_min_y + gy, cz = h->bbox_min_z + gz;
                if (cx > h->bbox_max_x || cy > h->bbox_max_y || cz > h->bbox_max_z) continue;
                if (cx < 0 || cy < 0 || cz < 0 || cx >= X || cy >= Y || cz >= Z) continue;
                uint32_t idx = (uint32_t)((cz * Y + cy) * X + cx);
                V3<T> cell = {T(cx) + T(0.5), T(cy) + T(0.5), T(cz) + T(0.5)};
                V3<T> to_cell = cell - hand_pos;
                V3<T> perp = to_cell - mul(dot(to_cell, ray_dir), ray_dir);
                T d = length(perp);
                if (d >= T(h->radius)) continue;
                T t = T(1.0) - d / T(h->radius);
                T w = t * t * T(h->strength);
                s.mvf[3 * idx + 0] += T(h->vx) * w;
                s.mvf[3 * idx + 1] += T(h->vy) * w;
                s.mvf[3 * idx + 2] += T(h->vz) * w;
            }
}

/* ---- G2P: shaders.js:579-705 ---------------------------------------------- */
template <class T> void pass_g2p(Scene<T>& s) {
    const mpm_params& P = *s.P;
    const uint32_t X = P.grid_X, Y = P.grid_Y;
    const int64_t n = P.particle_num;
    const uint32_t nw = wall_count(s.W);
    WallT<T> walls[MPM_MAX_WALLS];
    for (uint32_t i = 0; i < nw; ++i) walls[i] = load_wall<T>(s.W->walls[i]);
    const T dt = P.dt, lk = P.lookahead_k, ws = P.wall_stiffness, wmin_ = P.wall_min;
    const T hmin = P.hard_min;
    const T hmax[3] = {T(P.hard_max_x), T(P.hard_max_y), T(P.hard_max_z)};
#pragma omp parallel for schedule(static) num_threads(s.threads) if (s.threads > 1)
    for (int64_t p = 0; p < n; ++p) {
        V3<T> pos = {s.pos[4 * p], s.pos[4 * p + 1], s.pos[4 * p + 2]};
        BaseW<T> bw = compute_weights(pos.x, pos.y, pos.z);
        const uint32_t SLICE = X * Y;
        const uint32_t baseIdx = (uint32_t)((bw.bz * (int32_t)Y + bw.by) * (int32_t)X + bw.bx);
        T gvx = 0, gvy = 0, gvz = 0;
        T B00 = 0, B01 = 0, B02 = 0, B10 = 0, B11 = 0, B12 = 0, B20 = 0, B21 = 0, B22 = 0;
        for (int k = 0; k < 3; ++k) {
            T wzk = bw.wz[k];
            T dzk = T(bw.bz + k) - pos.z + T(0.5);
            for (int j = 0; j < 3; ++j) {
                T wyzk = bw.wy[j] * wzk;
                T dyj = T(bw.by + j) - pos.y + T(0.5);
                for (int i = 0; i < 3; ++i) {
                    T w = bw.wx[i] * wyzk;
                    T dxi = T(bw.bx + i) - pos.x + T(0.5);
                    uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)j * X + (uint32_t)i;
                    T cvx = s.mvf[3 * (size_t)cidx], cvy = s.mvf[3 * (size_t)cidx + 1], cvz = s.mvf[3 * (size_t)cidx + 2];
                    T wvx = w * cvx, wvy = w * cvy, wvz = w * cvz;
                    gvx += wvx; gvy += wvy; gvz += wvz;
                    B00 += wvx * dxi; B01 += wvx * dyj; B02 += wvx * dzk;
                    B10 += wvy * dxi; B11 += wvy * dyj; B12 += wvy * dzk;
                    B20 += wvz * dxi; B21 += wvz * dyj; B22 += wvz * dzk;
                }
            }
        }
        T* a = s.aff + 9 * p;
        a[0] = B00 * T(4.0); a[1] = B01 * T(4.0); a[2] = B02 * T(4.0);
        a[3] = B10 * T(4.0); a[4] = B11 * T(4.0); a[5] = B12 * T(4.0);
        a[6] = B20 * T(4.0); a[7] = B21 * T(4.0); a[8] = B22 * T(4.0);

        V3<T> np = {pos.x + dt * gvx, pos.y + dt * gvy, pos.z + dt * gvz};
        V3<T> nv = {gvx, gvy, gvz};

        const T floorZoneY = hmin + T(3.0);
        V3<T> xn = {np.x + nv.x * dt * lk, np.y + nv.y * dt * lk, np.z + nv.z * dt * lk};
        if (xn.y < floorZoneY) {
            T distBelowFloor = floorZoneY - xn.y;
            T blend = wclamp(distBelowFloor / T(3.0), T(0.0), T(1.0));
            nv.y += ws * blend * distBelowFloor;
        }

        for (uint32_t wi = 0; wi < nw; ++wi) {
            const WallT<T>& w = walls[wi];
            V3<T> wmn = w.mn, wmx = w.mx;
            V3<T> xnw = {np.x + nv.x * dt * lk, np.y + nv.y * dt * lk, np.z + nv.z * dt * lk};
            V3<T> lxn = wall_to_local(xnw, w);
            if (lxn.x > wmn.x && lxn.y > wmn.y && lxn.z > wmn.z && lxn.x < wmx.x && lxn.y < wmx.y && lxn.z < wmx.z) {
                V3<T> nl;
                T sw = wall_sdf_normal(lxn, wmn, wmx, nl);
                T dist = -sw;
                T blend = wclamp(dist / wmin_, T(0.0), T(1.0));
                V3<T> nwd = wall_to_world_dir(nl, w);
                T sc = ws * blend * dist;
                nv = {nv.x + nwd.x * sc, nv.y + nwd.y * sc, nv.z + nwd.z * sc};
            }
            V3<T> lnp = wall_to_local(np, w);
            if (lnp.x > wmn.x && lnp.y > wmn.y && lnp.z > wmn.z && lnp.x < wmx.x && lnp.y < wmx.y && lnp.z < wmx.z) {
                V3<T> nl;
                T sw = wall_sdf_normal(lnp, wmn, wmx, nl);
                V3<T> nn = wall_to_world_dir(nl, w);
                T m = wmax(sw, T(-0.5));
                np = {np.x - nn.x * m, np.y - nn.y * m, np.z - nn.z * m};
                T vn = dot(nv - wall_vel_at(np, w), nn);
                if (vn < T(0)) nv = {nv.x - vn * nn.x, nv.y - vn * nn.y, nv.z - vn * nn.z};
            }
        }

        T* npp[3] = {&np.x, &np.y, &np.z};
        T* nvp[3] = {&nv.x, &nv.y, &nv.z};
        for (int ax = 0; ax < 3; ++ax) {
            T q = *npp[ax], v = *nvp[ax];
            if (q < hmin) { q = hmin; v = T(0); }
            if (q > hmax[ax]) { q = hmax[ax]; v = T(0); }
            *npp[ax] = q; *nvp[ax] = v;
        }
        s.pos[4 * p] = np.x; s.pos[4 * p + 1] = np.y; s.pos[4 * p + 2] = np.z; s.pos[4 * p + 3] = T(0);
        s.vel[4 * p] = nv.x; s.vel[4 * p + 1] = nv.y; s.vel[4 * p + 2] = nv.z; s.vel[4 * p + 3] = T(0);
    }
}

/* ---- diffuse: shaders.js:721-997 ------------------------------------------ */

template <class T> struct DiffT { T pos[4], vel[4]; uint32_t ptype, alive; T lifetime, pad; };

inline float diffuse_rand(uint32_t seed) {          // shaders.js:756-762
    uint32_t x = seed;
    x = x ^ (x << 13u);
    x = x ^ (x >> 17u);
    x = x ^ (x << 5u);
    return (float)x / 4294967295.0f;
}
inline double diffuse_rand_d(uint32_t seed) {
    uint32_t x = seed;
    x = x ^ (x << 13u);
    x = x ^ (x >> 17u);
    x = x ^ (x << 5u);
    return (double)x / 4294967295.0;
}
template <class T> inline T drand(uint32_t s);
template <> inline float drand<float>(uint32_t s) { return diffuse_rand(s); }
template <> inline double drand<double>(uint32_t s) { return diffuse_rand_d(s); }

// shaders.js:766-787 estimate_normal; returns false for the reference's w=0.
template <class T> inline bool estimate_normal(const Scene<T>& s, V3<T> pos, V3<T>& n) {
    const int32_t X = s.P->grid_X, Y = s.P->grid_Y, Z = s.P->grid_Z;
    int32_t gx = to_i32(std::floor(pos.x)), gy = to_i32(std::floor(pos.y)), gz = to_i32(std::floor(pos.z));
    if (gx < 1 || gx >= X - 1 || gy < 1 || gy >= Y - 1 || gz < 1 || gz >= Z - 1) return false;
    uint32_t idxL = (uint32_t)((gz * Y + gy) * X + (gx - 1));
    uint32_t idxR = (uint32_t)((gz * Y + gy) * X + (gx + 1));
    uint32_t idxD = (uint32_t)((gz * Y + (gy - 1)) * X + gx);
    uint32_t idxU = (uint32_t)((gz * Y + (gy + 1)) * X + gx);
    uint32_t idxB = (uint32_t)(((gz - 1) * Y + gy) * X + gx);
    uint32_t idxF = (uint32_t)(((gz + 1) * Y + gy) * X + gx);
    V3<T> v = {s.cmf[idxL] - s.cmf[idxR], s.cmf[idxD] - s.cmf[idxU], s.cmf[idxB] - s.cmf[idxF]};
    T len = length(v);
    if (len < T(1e-6)) return false;
    n = {v.x / len, v.y / len, v.z / len};
    return true;
}

// GENERATE (shaders.js:800-855).  Phase 1 (parallel) decides which particles
// spawn; phase 2 pops slots in ascending particle order (the canonical order
// of a serial try_spawn, shaders.js:791-798).
template <class T> void pass_diffuse_generate(Scene<T>& s, const mpm_gen_params* gen, DiffT<T>* dp,
                                              uint32_t* free_list, int32_t* top) {
    const mpm_params& P = *s.P;
    const int64_t n = P.particle_num;
    const T rest = P.rest_density, stiff = P.stiffness, eos = P.eos_power, dt = P.dt;
    const T keth = gen->ke_threshold;
    std::vector<uint8_t> spawn((size_t)n, 0);
    std::vector<DiffT<T>> rec((size_t)n);
#pragma omp parallel for schedule(static) num_threads(s.threads) if (s.threads > 1)
    for (int64_t p = 0; p < n; ++p) {
        T density = s.dens[p];
        if (density <= T(0) || density > T(gen->density_bubble_min)) continue;
        V3<T> vel = {s.vel[4 * p], s.vel[4 * p + 1], s.vel[4 * p + 2]};
        T speed2 = dot(vel, vel);
        T speed = std::sqrt(speed2);
        T ke = T(0.5) * s.mass[p] * speed2;
        T pressure = stiff * (eos_pow(density / rest, eos) - T(1.0));
        T pFloor = (density > rest * T(0.7)) ? T(-0.1) : T(0.0);
        pressure = wmax(pressure, pFloor);
        T trappedAir = wmax(T(0.0), pressure - T(gen->pressure_threshold));
        V3<T> pos = {s.pos[4 * p], s.pos[4 * p + 1], s.pos[4 * p + 2]};
        V3<T> nrm;
        bool ok = estimate_normal(s, pos, nrm);
        T waveCrest = T(0);
        if (speed > T(1e-4) && ok) {
            V3<T> vs = {vel.x / speed, vel.y / speed, vel.z / speed};
            T dotVal = dot(vs, nrm);
            if (dotVal > T(gen->crest_dot_threshold)) waveCrest = dotVal * speed;
        }
        T score = ke + trappedAir * T(2.0) + waveCrest * T(1.5);
        if (score < keth) continue;
        uint32_t randSeed = (uint32_t)p * 9781u + gen->seed;
        T spawnChance = wmin(T(1.0), (score - keth) * T(gen->spawn_rate_k) * dt);
        if (drand<T>(randSeed) > spawnChance) continue;
        T jitter = T(0.3);
        T jx = (drand<T>(randSeed + 1u) - T(0.5)) * jitter * speed;
        T jy = (drand<T>(randSeed + 2u) - T(0.5)) * jitter * speed;
        T jz = (drand<T>(randSeed + 3u) - T(0.5)) * jitter * speed;
        uint32_t ptype = MPM_DIFFUSE_FOAM;
        if (density < T(gen->density_spray_max)) ptype = MPM_DIFFUSE_SPRAY;
        T lifetime = (ptype == MPM_DIFFUSE_FOAM) ? T(gen->lifetime_foam) * wmin(T(1.0), score / keth) : T(999.0);
        DiffT<T> r;
        r.pos[0] = pos.x; r.pos[1] = pos.y; r.pos[2] = pos.z; r.pos[3] = T(0);
        r.vel[0] = vel.x + jx; r.vel[1] = vel.y + jy; r.vel[2] = vel.z + jz; r.vel[3] = T(0);
        r.ptype = ptype; r.alive = 1u; r.lifetime = lifetime; r.pad = T(0);
        rec[(size_t)p] = r;
        spawn[(size_t)p] = 1;
    }
    for (int64_t p = 0; p < n; ++p) {
        if (!spawn[(size_t)p]) continue;
        int32_t prevTop = *top;
        *top = prevTop - 1;
        if (prevTop <= 0) { *top = *top + 1; continue; }
        uint32_t slot = free_list[(uint32_t)(prevTop - 1)];
        dp[slot] = rec[(size_t)p];
    }
}

// shaders.js:889-912
template <class T> inline V3<T> sample_grid_velocity(const Scene<T>& s, V3<T> pos) {
    const int32_t X = s.P->grid_X, Y = s.P->grid_Y, Z = s.P->grid_Z;
    BaseW<T> bw = compute_weights(pos.x, pos.y, pos.z);
    V3<T> v = {T(0), T(0), T(0)};
    for (int k = 0; k < 3; ++k) {
        int32_t cz = bw.bz + k;
        for (int j = 0; j < 3; ++j) {
            int32_t cy = bw.by + j;
            for (int i = 0; i < 3; ++i) {
                int32_t cx = bw.bx + i;
                if (cx < 0 || cx >= X || cy < 0 || cy >= Y || cz < 0 || cz >= Z) continue;
                int32_t idx = (cz * Y + cy) * X + cx;
                T w = bw.wx[i] * bw.wy[j] * bw.wz[k];
                v.x += w * s.mvf[(uint32_t)idx * 3u + 0u];
                v.y += w * s.mvf[(uint32_t)idx * 3u + 1u];
                v.z += w * s.mvf[(uint32_t)idx * 3u + 2u];
            }
        }
    }
    return v;
}

// shaders.js:922-927
template <class T> inline void reflect_axis(T& p, T& v, T lo, T hi) {
    const T R = T(0.3);
    T np = p, nv = v;
    if (np < lo) { np = lo + (lo - np); nv = -nv * R; }
    else if (np > hi) { np = hi - (np - hi); nv = -nv * R; }
    p = wclamp(np, lo, hi); v = nv;
}

// ADVECT (shaders.js:929-996).  Kills push in ascending slot order (the
// canonical order of a serial kill_particle, shaders.js:914-918).
template <class T> void pass_diffuse_advect(Scene<T>& s, const mpm_advect_params* adv, DiffT<T>* dp,
                                            uint32_t* free_list, int32_t* top) {
    const mpm_params& P = *s.P;
    const int64_t M = adv->diffuse_max;
    const T dt = P.dt, g = P.gravity, hmin = P.hard_min;
    const T hmax[3] = {T(P.hard_max_x), T(P.hard_max_y), T(P.hard_max_z)};
    const uint32_t nw = wall_count(s.W);
    WallT<T> walls[MPM_MAX_WALLS];
    for (uint32_t i = 0; i < nw; ++i) walls[i] = load_wall<T>(s.W->walls[i]);
    std::vector<uint8_t> kill((size_t)M, 0);
#pragma omp parallel for schedule(static) num_threads(s.threads) if (s.threads > 1)
    for (int64_t i = 0; i < M; ++i) {
        if (dp[i].alive == 0u) continue;
        DiffT<T> p = dp[i];
        V3<T> pos3 = {p.pos[0], p.pos[1], p.pos[2]};
        if (p.ptype == MPM_DIFFUSE_SPRAY) {
            p.vel[1] += g * dt;
            p.pos[0] = pos3.x + dt * p.vel[0]; p.pos[1] = pos3.y + dt * p.vel[1]; p.pos[2] = pos3.z + dt * p.vel[2]; p.pos[3] = T(0);
        } else if (p.ptype == MPM_DIFFUSE_FOAM) {
            V3<T> gv = sample_grid_velocity(s, pos3);
            p.pos[0] = pos3.x + dt * gv.x; p.pos[1] = pos3.y + dt * gv.y; p.pos[2] = pos3.z + dt * gv.z; p.pos[3] = T(0);
            p.lifetime -= dt;
            if (p.lifetime <= T(0)) { kill[(size_t)i] = 1; continue; }
        } else if (p.ptype == MPM_DIFFUSE_BUBBLE) {
            V3<T> gv = sample_grid_velocity(s, pos3);
            const T drag = adv->drag, buoy = adv->buoyancy;
            p.vel[0] += dt * drag * (gv.x - p.vel[0]);
            p.vel[1] += dt * (buoy * -g + drag * (gv.y - p.vel[1]));
            p.vel[2] += dt * drag * (gv.z - p.vel[2]);
            p.pos[0] = pos3.x + dt * p.vel[0]; p.pos[1] = pos3.y + dt * p.vel[1]; p.pos[2] = pos3.z + dt * p.vel[2]; p.pos[3] = T(0);
        }
        for (uint32_t wi = 0; wi < nw; ++wi) {
            const WallT<T>& w = walls[wi];
            V3<T> lp = wall_to_local(v3<T>(p.pos[0], p.pos[1], p.pos[2]), w);
            if (!(lp.x > w.mn.x && lp.y > w.mn.y && lp.z > w.mn.z && lp.x < w.mx.x && lp.y < w.mx.y && lp.z < w.mx.z)) continue;
            V3<T> nl;
            T sw = wall_sdf_normal(lp, w.mn, w.mx, nl);
            V3<T> nn = wall_to_world_dir(nl, w);
            p.pos[0] = p.pos[0] - nn.x * sw; p.pos[1] = p.pos[1] - nn.y * sw; p.pos[2] = p.pos[2] - nn.z * sw; p.pos[3] = T(0);
            V3<T> wvel = wall_vel_at(v3<T>(p.pos[0], p.pos[1], p.pos[2]), w);
            V3<T> vrel = v3<T>(p.vel[0], p.vel[1], p.vel[2]) - wvel;
            T vn = dot(vrel, nn);
            if (vn < T(0)) {
                T k = (T(1.0) + T(0.3)) * vn;
                V3<T> newvrel = {vrel.x - k * nn.x, vrel.y - k * nn.y, vrel.z - k * nn.z};
                p.vel[0] = wvel.x + newvrel.x; p.vel[1] = wvel.y + newvrel.y; p.vel[2] = wvel.z + newvrel.z; p.vel[3] = T(0);
            }
        }
        if (p.pos[1] < hmin) { kill[(size_t)i] = 1; continue; }
        reflect_axis(p.pos[0], p.vel[0], hmin, hmax[0]);
        reflect_axis(p.pos[1], p.vel[1], hmin, hmax[1]);
        reflect_axis(p.pos[2], p.vel[2], hmin, hmax[2]);
        p.pos[3] = T(0); p.vel[3] = T(0);
        dp[i] = p;
    }
    for (int64_t i = 0; i < M; ++i) {
        if (!kill[(size_t)i]) continue;
        dp[i].alive = 0u;
        int32_t slot = *top;
        *top = slot + 1;
        free_list[(uint32_t)slot] = (uint32_t)i;
    }
}

/* ---- COMPACT (shaders.js:532-546) and RAYCAST (shaders.js:563-576) -------- */
template <class T> inline T ray_perp_dist(V3<T> pos, V3<T> origin, V3<T> dir) {
    V3<T> to_p = pos - origin;
    V3<T> perp = to_p - mul(dot(to_p, dir), dir);
    return length(perp);
}

}  // namespace

/* ---- C entry points (ctypes) ---------------------------------------------- */

template <class T>
static void substep_impl(const mpm_params* P, const mpm_wall_params* W, const mpm_hand_params* hand,
                         const int32_t* hand_dims, T* pos, T* vel, T* aff, const T* mass, T* dens,
                         int32_t* mv, int32_t* cm, T* mvf, T* cmf, const mpm_gen_params* gen,
                         const mpm_advect_params* adv, T* diffuse, uint32_t* free_list, int32_t* top,
                         int threads) {
    Scene<T> s{P, W, pos, vel, aff, mass, dens, mv, cm, mvf, cmf, threads < 1 ? 1 : threads};
    // fluid-gpu.js:663-682 pass order
    pass_clear(s);
    pass_p2g_mass(s);
    pass_decode_mass(s);
    pass_p2g_mom(s);
    pass_update_grid(s);
    if (hand && hand_dims) pass_apply_hand(s, hand, hand_dims);
    pass_g2p(s);
    if (gen && adv && diffuse && free_list && top) {
        pass_diffuse_generate(s, gen, reinterpret_cast<DiffT<T>*>(diffuse), free_list, top);
        pass_diffuse_advect(s, adv, reinterpret_cast<DiffT<T>*>(diffuse), free_list, top);
    }
}

extern "C" {

int oracle_abi_version(void) { return 1; }

/* One simFrame substep (fluid-gpu.js:663-682 + diffuse-gpu.js:148-166) on f32
 * state.  hand/hand_dims may be NULL (hand inactive); gen/adv/diffuse/... may
 * be NULL (no diffuse).  gen->seed must already hold the bumped seed. */
void oracle_substep_f32(const mpm_params* P, const mpm_wall_params* W, const mpm_hand_params* hand,
                        const int32_t* hand_dims, float* pos, float* vel, float* aff, const float* mass,
                        float* dens, int32_t* mv, int32_t* cm, float* mvf, float* cmf,
                        const mpm_gen_params* gen, const mpm_advect_params* adv, float* diffuse,
                        uint32_t* free_list, int32_t* top, int threads) {
    substep_impl<float>(P, W, hand, hand_dims, pos, vel, aff, mass, dens, mv, cm, mvf, cmf, gen, adv,
                        diffuse, free_list, top, threads);
}

/* Same pass sequence evaluated in binary64 (the f64 drift reference). */
void oracle_substep_f64(const mpm_params* P, const mpm_wall_params* W, const mpm_hand_params* hand,
                        const int32_t* hand_dims, double* pos, double* vel, double* aff, const double* mass,
                        double* dens, int32_t* mv, int32_t* cm, double* mvf, double* cmf,
                        const mpm_gen_params* gen, const mpm_advect_params* adv, double* diffuse,
                        uint32_t* free_list, int32_t* top, int threads) {
    substep_impl<double>(P, W, hand, hand_dims, pos, vel, aff, mass, dens, mv, cm, mvf, cmf, gen, adv,
                         diffuse, free_list, top, threads);
}

/* Single passes (f32), for per-pass parity tests. */
void oracle_p2g_f32(const mpm_params* P, const float* pos, const float* vel, const float* aff,
                    const float* mass, float* dens, int32_t* mv, int32_t* cm, float* cmf, int threads) {
    Scene<float> s{P, nullptr, const_cast<float*>(pos), const_cast<float*>(vel), const_cast<float*>(aff),
                   mass, dens, mv, cm, nullptr, cmf, threads < 1 ? 1 : threads};
    pass_clear(s);
    pass_p2g_mass(s);
    pass_decode_mass(s);
    pass_p2g_mom(s);
}

void oracle_update_grid_f32(const mpm_params* P, const mpm_wall_params* W, const int32_t* mv,
                            const int32_t* cm, float* mvf, int threads) {
    Scene<float> s{P, W, nullptr, nullptr, nullptr, nullptr, nullptr, const_cast<int32_t*>(mv),
                   const_cast<int32_t*>(cm), mvf, nullptr, threads < 1 ? 1 : threads};
    pass_update_grid(s);
}

void oracle_apply_hand_f32(const mpm_params* P, const mpm_hand_params* hand, const int32_t* dims, float* mvf) {
    Scene<float> s{P, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, mvf, nullptr, 1};
    pass_apply_hand(s, hand, dims);
}

void oracle_g2p_f32(const mpm_params* P, const mpm_wall_params* W, float* pos, float* vel, float* aff,
                    const float* mvf, int threads) {
    Scene<float> s{P, W, pos, vel, aff, nullptr, nullptr, nullptr, nullptr, const_cast<float*>(mvf), nullptr,
                   threads < 1 ? 1 : threads};
    pass_g2p(s);
}

/* COMPACT with the canonical (stable, ascending p) survivor order.
 * Returns the survivor count (the reference's counter). */
uint32_t oracle_compact_f32(const mpm_params* P, const mpm_ray_params* del, const float* pos_in,
                            const float* vel_in, const float* mass_in, float* pos_out, float* vel_out,
                            float* mass_out) {
    uint32_t counter = 0;
    V3<float> origin = {del->ox, del->oy, del->oz}, dir = {del->dx, del->dy, del->dz};
    for (uint32_t p = 0; p < P->particle_num; ++p) {
        V3<float> pos = {pos_in[4 * p], pos_in[4 * p + 1], pos_in[4 * p + 2]};
        if (ray_perp_dist(pos, origin, dir) < del->radius) continue;
        uint32_t idx = counter++;
        std::memcpy(pos_out + 4 * (size_t)idx, pos_in + 4 * (size_t)p, 16);
        std::memcpy(vel_out + 4 * (size_t)idx, vel_in + 4 * (size_t)p, 16);
        mass_out[idx] = mass_in[p];
    }
    return counter;
}

/* RAYCAST: returns the atomicMin'd u32 bit pattern (0xFFFFFFFF = no hit). */
uint32_t oracle_raycast_f32(const mpm_params* P, const mpm_ray_params* ray, const float* pos_in) {
    uint32_t hit = 0xFFFFFFFFu;
    V3<float> origin = {ray->ox, ray->oy, ray->oz}, dir = {ray->dx, ray->dy, ray->dz};
    for (uint32_t p = 0; p < P->particle_num; ++p) {
        V3<float> pos = {pos_in[4 * p], pos_in[4 * p + 1], pos_in[4 * p + 2]};
        float t = dot(pos - origin, dir);
        if (t <= 0.0f) continue;
        if (ray_perp_dist(pos, origin, dir) >= ray->radius) continue;
        uint32_t b;
        std::memcpy(&b, &t, 4);
        hit = std::min(hit, b);
    }
    return hit;
}

}  // extern "C"
