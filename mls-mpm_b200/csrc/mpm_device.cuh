// mpm_device.cuh — device helpers shared by the MLS-MPM kernels.
//
// Numerics contract: every translation unit that includes this header is
// compiled with --fmad=false (no multiply-add contraction) and IEEE division
// and square root (-prec-div=true -prec-sqrt=true, nvcc's defaults without
// --use_fast_math).  Expressions are written in the reference's evaluation
// order (shaders.js), so each f32 result is the correctly rounded result of
// the same operation sequence the reference specifies, and each i32 grid
// contribution is bit-identical to the reference's.
#pragma once

#include <cstdint>

#include "../../include/mpm_types.h"

namespace mpm {

constexpr float kFixed = 100000.0f;        // shaders.js:15 FIXED
constexpr float kEncodeClamp = 20000.0f;   // shaders.js:22
constexpr float kCohesionPressure = -0.1f; // shaders.js:12
constexpr float kCohesionGate = 0.7f;      // shaders.js:13
constexpr float kFloorBand = 3.0f;         // shaders.js:5 FLOOR_SPRING_BAND
constexpr float kRestitution = 0.3f;       // shaders.js:921

// shaders.js:21-24.  fminf/fmaxf return the non-NaN operand (WGSL min/max);
// the float->int conversion truncates toward zero (cvt.rzi saturates).
__device__ __forceinline__ int32_t encode(float v) {
    float c = fminf(fmaxf(v, -kEncodeClamp), kEncodeClamp);
    return __float2int_rz(c * kFixed);
}
// 1 when an encoded value sits at encode's clamp (|value| >= 20000 before
// scaling): the health flag MPM_HEALTH_SATURATED.
constexpr int32_t kEncodedMax = 2000000000;   // kEncodeClamp * kFixed, exact in f32
__device__ __forceinline__ uint32_t at_clamp(int32_t e) { return (e == kEncodedMax || e == -kEncodedMax) ? 1u : 0u; }

// shaders.js:25 (IEEE division)
__device__ __forceinline__ float decode(int32_t v) { return __fdiv_rn(__int2float_rn(v), kFixed); }

__device__ __forceinline__ float wclamp(float e, float lo, float hi) { return fminf(fmaxf(e, lo), hi); }

// pow(x, eos_power) (shaders.js:326): x^1 == x exactly; other exponents use
// CUDA powf (documented tolerance, not bit-exact against libm).
__device__ __forceinline__ float eos_pow(float x, float e) { return e == 1.0f ? x : powf(x, e); }

// shaders.js:53-59 quadratic_weights for one axis.
__device__ __forceinline__ void qweights(float f, float& w0, float& w1, float& w2) {
    float a = 0.5f - f, b = 0.5f + f;
    w0 = 0.5f * a * a;
    w1 = 0.75f - f * f;
    w2 = 0.5f * b * b;
}

// shaders.js:226-230: cellI = i32(floor(pos)), f = pos - f32(cellI) - 0.5
__device__ __forceinline__ void cell_frac(float p, int32_t& cell, float& f) {
    cell = __float2int_rz(floorf(p));
    f = (p - __int2float_rn(cell)) - 0.5f;
}

struct f3 { float x, y, z; };
__device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 sub(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 add(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len3(f3 a) { return __fsqrt_rn(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ f3 cross3(f3 a, f3 b) {
    return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// ---- moving walls: shaders.js:135-193 --------------------------------------
struct WallD {
    f3 c; float cy, sy, cp, sp;
    f3 mn, mx, vel, om;
};

__device__ __forceinline__ WallD load_wall(const mpm_wall& w) {
    WallD o;
    o.c = mk(w.center_cy[0], w.center_cy[1], w.center_cy[2]);
    o.cy = w.center_cy[3]; o.sy = w.lmin_sy[3]; o.cp = w.lmax_cp[3]; o.sp = w.vel_sp[3];
    o.mn = mk(w.lmin_sy[0], w.lmin_sy[1], w.lmin_sy[2]);
    o.mx = mk(w.lmax_cp[0], w.lmax_cp[1], w.lmax_cp[2]);
    o.vel = mk(w.vel_sp[0], w.vel_sp[1], w.vel_sp[2]);
    o.om = mk(w.omega_pad[0], w.omega_pad[1], w.omega_pad[2]);
    return o;
}

__device__ __forceinline__ f3 wall_to_local(f3 p, const WallD& w) {
    f3 d = sub(p, w.c);
    float x1 = w.cy * d.x - w.sy * d.z;
    float z1 = w.sy * d.x + w.cy * d.z;
    return f3{x1, w.cp * d.y + w.sp * z1, -w.sp * d.y + w.cp * z1};
}

__device__ __forceinline__ f3 wall_to_world_dir(f3 v, const WallD& w) {
    float y1 = w.cp * v.y - w.sp * v.z;
    float z1 = w.sp * v.y + w.cp * v.z;
    return f3{w.cy * v.x + w.sy * z1, y1, -w.sy * v.x + w.cy * z1};
}

__device__ __forceinline__ f3 wall_vel_at(f3 p, const WallD& w) {
    f3 r = sub(p, w.c);
    return add(w.vel, cross3(w.om, r));
}

// Signed distance (returned) and local normal n.
__device__ __forceinline__ float wall_sdf_normal(f3 lp, f3 mn, f3 mx, f3& n) {
    f3 dmin = sub(mn, lp);
    f3 dmax = sub(lp, mx);
    f3 q = mk(fmaxf(dmin.x, dmax.x), fmaxf(dmin.y, dmax.y), fmaxf(dmin.z, dmax.z));
    float qmax = fmaxf(q.x, fmaxf(q.y, q.z));
    if (qmax > 0.0f) {
        f3 nearest = mk(wclamp(lp.x, mn.x, mx.x), wclamp(lp.y, mn.y, mx.y), wclamp(lp.z, mn.z, mx.z));
        f3 diff = sub(lp, nearest);
        float len = len3(diff);
        if (len > 1e-6f) n = mk(__fdiv_rn(diff.x, len), __fdiv_rn(diff.y, len), __fdiv_rn(diff.z, len));
        else n = mk(0.0f, 1.0f, 0.0f);
        return len;
    }
    n = mk(0.0f, 1.0f, 0.0f);
    if (qmax == q.x)      n = mk(dmax.x > dmin.x ? 1.0f : -1.0f, 0.0f, 0.0f);
    else if (qmax == q.y) n = mk(0.0f, dmax.y > dmin.y ? 1.0f : -1.0f, 0.0f);
    else                  n = mk(0.0f, 0.0f, dmax.z > dmin.z ? 1.0f : -1.0f);
    return qmax;
}

__device__ __forceinline__ bool inside_open(f3 l, f3 mn, f3 mx) {
    return l.x > mn.x && l.y > mn.y && l.z > mn.z && l.x < mx.x && l.y < mx.y && l.z < mx.z;
}

// u32(count_pad.x), bounded by the uniform's capacity.
__host__ __device__ __forceinline__ uint32_t wall_count_of(float c) {
    if (!(c > 0.0f)) return 0u;
    uint32_t n = (uint32_t)c;
    return n > MPM_MAX_WALLS ? MPM_MAX_WALLS : n;
}

// shaders.js:756-762
__device__ __forceinline__ float diffuse_rand(uint32_t seed) {
    uint32_t x = seed;
    x = x ^ (x << 13u);
    x = x ^ (x >> 17u);
    x = x ^ (x << 5u);
    return __fdiv_rn(__uint2float_rn(x), 4294967295.0f);
}

}  // namespace mpm
