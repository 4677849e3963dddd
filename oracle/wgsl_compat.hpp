/*
 * wgsl_compat.hpp — a tiny C++ runtime for WGSL compute-shader source.
 *
 * TEST INFRASTRUCTURE ONLY (builds oracle/_ref, the reference pin).
 *
 * wgsl2cpp.py rewrites the reference's WGSL text into C++ syntax (declarations,
 * function signatures, struct bodies, literals) without changing a single
 * expression; this header supplies what WGSL provides as builtins: the
 * vector types, component-wise operators, the numeric builtins and the
 * atomics.  Semantics follow the WGSL spec with IEEE-754 binary32 rounding on
 * every operation (compile with -ffp-contract=off -fwrapv):
 *   max/min return the non-NaN operand; clamp(e,lo,hi) = min(max(e,lo),hi);
 *   i32(f32)/u32(f32) truncate toward zero and saturate (NaN -> 0);
 *   length(v) = sqrt(dot(v,v)) summed left to right; normalize(v) = v/length(v);
 *   atomics are sequential when the driver runs one invocation at a time and
 *   relaxed hardware atomics when it runs invocations on several threads.
 */
#pragma once
#include <cstdint>
#include <cstring>

namespace wgsl_rt {

typedef float f32;
typedef int32_t i32;
typedef uint32_t u32;

extern bool g_parallel;  // set by the driver around multi-threaded dispatches

/* ---- scalar conversions (WGSL value constructors) ---- */
inline i32 to_i32(f32 x) {
    if (x != x) return 0;
    if (x >= 2147483647.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return (i32)x;
}
inline i32 to_i32(i32 x) { return x; }
inline i32 to_i32(u32 x) { return (i32)x; }
inline u32 to_u32(f32 x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967295.0f) return UINT32_MAX;
    return (u32)x;
}
inline u32 to_u32(i32 x) { return (u32)x; }
inline u32 to_u32(u32 x) { return x; }
inline f32 to_f32(i32 x) { return (f32)x; }
inline f32 to_f32(u32 x) { return (f32)x; }
inline f32 to_f32(f32 x) { return x; }

template <class To> inline To conv(f32 x);
template <> inline f32 conv<f32>(f32 x) { return x; }
template <> inline i32 conv<i32>(f32 x) { return to_i32(x); }
template <> inline u32 conv<u32>(f32 x) { return to_u32(x); }
template <class To> inline To conv(i32 x) { return (To)x; }
template <class To> inline To conv(u32 x) { return (To)x; }
template <class To> inline To conv(bool x) { return (To)x; }

template <class U, class T> inline U bitcast(T x) {
    static_assert(sizeof(U) == sizeof(T), "bitcast size");
    U u;
    std::memcpy(&u, &x, sizeof(U));
    return u;
}

/* ---- vectors ---- */
template <class T> struct vec3;

template <class T> struct vec2 {
    T x, y;
    vec2() : x(T(0)), y(T(0)) {}
    explicit vec2(T s) : x(s), y(s) {}
    vec2(T a, T b) : x(a), y(b) {}
};

template <class T> struct vec3 {
    T x, y, z;
    vec3() : x(T(0)), y(T(0)), z(T(0)) {}
    explicit vec3(T s) : x(s), y(s), z(s) {}
    vec3(T a, T b, T c) : x(a), y(b), z(c) {}
    template <class U> explicit vec3(const vec3<U>& o) : x(conv<T>(o.x)), y(conv<T>(o.y)), z(conv<T>(o.z)) {}
    T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    const T& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    vec3& operator+=(const vec3& o) { x = x + o.x; y = y + o.y; z = z + o.z; return *this; }
    vec3& operator-=(const vec3& o) { x = x - o.x; y = y - o.y; z = z - o.z; return *this; }
    vec3& operator*=(T s) { x = x * s; y = y * s; z = z * s; return *this; }
};

template <class T> struct vec4 {
    T x, y, z, w;
    vec4() : x(T(0)), y(T(0)), z(T(0)), w(T(0)) {}
    explicit vec4(T s) : x(s), y(s), z(s), w(s) {}
    vec4(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
    vec4(const vec3<T>& v, T d) : x(v.x), y(v.y), z(v.z), w(d) {}
    vec3<T> xyz() const { return vec3<T>(x, y, z); }
};
template <class T> inline vec3<T> swz_xyz(const vec4<T>& v) { return v.xyz(); }

#define WGSL_V3_BINOP(OP)                                                                          \
    template <class T> inline vec3<T> operator OP(const vec3<T>& a, const vec3<T>& b) {            \
        return vec3<T>(a.x OP b.x, a.y OP b.y, a.z OP b.z);                                        \
    }                                                                                              \
    template <class T> inline vec3<T> operator OP(const vec3<T>& a, T s) {                         \
        return vec3<T>(a.x OP s, a.y OP s, a.z OP s);                                              \
    }                                                                                              \
    template <class T> inline vec3<T> operator OP(T s, const vec3<T>& a) {                         \
        return vec3<T>(s OP a.x, s OP a.y, s OP a.z);                                              \
    }
WGSL_V3_BINOP(+)
WGSL_V3_BINOP(-)
WGSL_V3_BINOP(*)
WGSL_V3_BINOP(/)
#undef WGSL_V3_BINOP
template <class T> inline vec3<T> operator-(const vec3<T>& a) { return vec3<T>(-a.x, -a.y, -a.z); }

#define WGSL_V3_CMP(OP)                                                                            \
    template <class T> inline vec3<bool> operator OP(const vec3<T>& a, const vec3<T>& b) {         \
        vec3<bool> r;                                                                              \
        r.x = a.x OP b.x; r.y = a.y OP b.y; r.z = a.z OP b.z;                                      \
        return r;                                                                                  \
    }
WGSL_V3_CMP(<)
WGSL_V3_CMP(>)
WGSL_V3_CMP(<=)
WGSL_V3_CMP(>=)
#undef WGSL_V3_CMP

inline bool all(const vec3<bool>& b) { return b.x && b.y && b.z; }
inline bool any(const vec3<bool>& b) { return b.x || b.y || b.z; }

template <class T, int N> struct array {
    T v[N];
    T& operator[](int i) { return v[i]; }
    const T& operator[](int i) const { return v[i]; }
    T& operator[](u32 i) { return v[i]; }
    const T& operator[](u32 i) const { return v[i]; }
};

/* ---- numeric builtins ---- */
inline f32 max(f32 a, f32 b) { return __builtin_fmaxf(a, b); }
inline f32 min(f32 a, f32 b) { return __builtin_fminf(a, b); }
inline i32 max(i32 a, i32 b) { return a > b ? a : b; }
inline i32 min(i32 a, i32 b) { return a < b ? a : b; }
inline u32 max(u32 a, u32 b) { return a > b ? a : b; }
inline u32 min(u32 a, u32 b) { return a < b ? a : b; }
inline vec3<f32> max(const vec3<f32>& a, const vec3<f32>& b) { return vec3<f32>(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline vec3<f32> min(const vec3<f32>& a, const vec3<f32>& b) { return vec3<f32>(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline f32 clamp(f32 e, f32 lo, f32 hi) { return min(max(e, lo), hi); }
inline vec3<f32> clamp(const vec3<f32>& e, const vec3<f32>& lo, const vec3<f32>& hi) { return min(max(e, lo), hi); }
inline f32 floor(f32 x) { return __builtin_floorf(x); }
inline vec3<f32> floor(const vec3<f32>& v) { return vec3<f32>(floor(v.x), floor(v.y), floor(v.z)); }
inline f32 sqrt(f32 x) { return __builtin_sqrtf(x); }
inline f32 pow(f32 x, f32 y) { return __builtin_powf(x, y); }
inline f32 dot(const vec3<f32>& a, const vec3<f32>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline f32 length(const vec3<f32>& v) { return sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
inline vec3<f32> normalize(const vec3<f32>& v) { f32 l = length(v); return vec3<f32>(v.x / l, v.y / l, v.z / l); }
inline vec3<f32> cross(const vec3<f32>& a, const vec3<f32>& b) {
    return vec3<f32>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class T> inline T select(T f, T t, bool c) { return c ? t : f; }

/* ---- atomics ---- */
template <class T> struct atomic { T v; };
template <class T> inline void atomicStore(atomic<T>* a, T x) { a->v = x; }
inline void atomicStore(atomic<i32>* a, int x) { a->v = x; }
template <class T> inline T atomicLoad(atomic<T>* a) { return a->v; }
inline i32 atomicAdd(atomic<i32>* a, i32 x) {
    if (g_parallel) return __atomic_fetch_add(&a->v, x, __ATOMIC_RELAXED);
    i32 o = a->v; a->v = (i32)((u32)o + (u32)x); return o;
}
inline u32 atomicAdd(atomic<u32>* a, u32 x) {
    if (g_parallel) return __atomic_fetch_add(&a->v, x, __ATOMIC_RELAXED);
    u32 o = a->v; a->v = o + x; return o;
}
inline i32 atomicSub(atomic<i32>* a, i32 x) {
    if (g_parallel) return __atomic_fetch_sub(&a->v, x, __ATOMIC_RELAXED);
    i32 o = a->v; a->v = (i32)((u32)o - (u32)x); return o;
}
inline u32 atomicMin(atomic<u32>* a, u32 x) {
    if (g_parallel) {
        u32 o = __atomic_load_n(&a->v, __ATOMIC_RELAXED);
        while (x < o && !__atomic_compare_exchange_n(&a->v, &o, x, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {}
        return o;
    }
    u32 o = a->v; if (x < o) a->v = x; return o;
}

}  // namespace wgsl_rt
