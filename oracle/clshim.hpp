// clshim.hpp -- just enough OpenCL C for g++ to compile the reference's
// tracking kernels on the CPU (test infrastructure only).
//
// oracle/build_ref.py captures the OpenCL source the reference assembles for
// a (domain, field, algorithm) combination, rewrites its vector literals
// ((float4)(...) and (T){...}) into make_T(...) calls, and compiles it after
// this header.  Built-ins map to the C library in binary32 (sqrtf, expf,
// logf, cosf, sincosf, acosf, atan2f ...), OpenCL's max/min/clamp semantics
// are kept (max(x, y) = x < y ? y : x; clamp = fmin(fmax(x, lo), hi)).
#pragma once

#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>

#define __kernel
#define kernel
#define __global
#define global
#define __constant const
#define constant const
#define __local
#define __private

typedef unsigned int uint;
typedef unsigned char uchar;
typedef unsigned short ushort;
typedef unsigned long ulong;

extern thread_local size_t tgref_global_id;
static inline size_t get_global_id(int) { return tgref_global_id; }

// ------------------------------------------------------------------ vectors

template <typename T>
struct vec2 {
    T x, y;
    T& operator[](size_t i) { return (&x)[i]; }
    T operator[](size_t i) const { return (&x)[i]; }
};

template <typename T>
struct vec3 {
    T x, y, z;
    T& operator[](size_t i) { return (&x)[i]; }
    T operator[](size_t i) const { return (&x)[i]; }
};

template <typename T>
struct vec4 {
    union {
        struct {
            T x, y, z, w;
        };
        vec3<T> xyz;
        T s[4];
    };
    T& operator[](size_t i) { return s[i]; }
    T operator[](size_t i) const { return s[i]; }
};

typedef vec2<float> float2;
typedef vec3<float> float3;
typedef vec4<float> float4;
typedef vec2<uint> uint2;
typedef vec3<uint> uint3;
typedef vec4<uint> uint4;
typedef vec2<int> int2;
typedef vec3<int> int3;
typedef vec4<int> int4;

#define TGREF_MAKE(T, S)                                                                                 \
    static inline T##2 make_##T##2(S a) { return T##2{a, a}; }                                           \
    static inline T##2 make_##T##2(S a, S b) { return T##2{a, b}; }                                      \
    static inline T##3 make_##T##3(S a) { return T##3{a, a, a}; }                                        \
    static inline T##3 make_##T##3(S a, S b, S c) { return T##3{a, b, c}; }                             \
    static inline T##4 make_##T##4(S a)                                                                  \
    {                                                                                                    \
        T##4 r;                                                                                          \
        r.x = r.y = r.z = r.w = a;                                                                       \
        return r;                                                                                        \
    }                                                                                                    \
    static inline T##4 make_##T##4(S a, S b, S c, S d)                                                   \
    {                                                                                                    \
        T##4 r;                                                                                          \
        r.x = a; r.y = b; r.z = c; r.w = d;                                                              \
        return r;                                                                                        \
    }                                                                                                    \
    static inline T##4 make_##T##4(T##3 v, S d) { return make_##T##4(v.x, v.y, v.z, d); }

TGREF_MAKE(float, float)
TGREF_MAKE(uint, uint)
TGREF_MAKE(int, int)

#define TGREF_OPS(V, N)                                                                                  \
    template <typename T> static inline V<T> operator+(V<T> a, V<T> b) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] + b[i]; return r; } \
    template <typename T> static inline V<T> operator-(V<T> a, V<T> b) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] - b[i]; return r; } \
    template <typename T> static inline V<T> operator*(V<T> a, V<T> b) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] * b[i]; return r; } \
    template <typename T> static inline V<T> operator/(V<T> a, V<T> b) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] / b[i]; return r; } \
    template <typename T> static inline V<T> operator*(V<T> a, T s) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] * s; return r; } \
    template <typename T> static inline V<T> operator*(T s, V<T> a) { V<T> r; for (int i = 0; i < N; ++i) r[i] = s * a[i]; return r; } \
    template <typename T> static inline V<T> operator/(V<T> a, T s) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] / s; return r; } \
    template <typename T> static inline V<T> operator+(V<T> a, T s) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] + s; return r; } \
    template <typename T> static inline V<T> operator-(V<T> a, T s) { V<T> r; for (int i = 0; i < N; ++i) r[i] = a[i] - s; return r; } \
    template <typename T> static inline V<T> operator-(V<T> a) { V<T> r; for (int i = 0; i < N; ++i) r[i] = -a[i]; return r; } \
    template <typename T> static inline V<T>& operator+=(V<T>& a, V<T> b) { for (int i = 0; i < N; ++i) a[i] += b[i]; return a; } \
    template <typename T> static inline V<T>& operator-=(V<T>& a, V<T> b) { for (int i = 0; i < N; ++i) a[i] -= b[i]; return a; }

TGREF_OPS(vec2, 2)
TGREF_OPS(vec3, 3)
TGREF_OPS(vec4, 4)

// Mixed float-literal / double forms the sources use (e.g. 1e-4f * v).
static inline float3 operator*(double s, float3 a) { return (float)s * a; }

// ---------------------------------------------------------------- built-ins

static inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float dot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
static inline float length(float3 a) { return sqrtf(dot(a, a)); }
static inline float length(float4 a) { return sqrtf(dot(a, a)); }
static inline float3 normalize(float3 a) { return a / length(a); }
static inline float3 cross(float3 a, float3 b)
{
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

static inline float max(float x, float y) { return x < y ? y : x; }
static inline float min(float x, float y) { return y < x ? y : x; }
static inline uint max(uint x, uint y) { return x < y ? y : x; }
static inline uint min(uint x, uint y) { return y < x ? y : x; }
static inline int max(int x, int y) { return x < y ? y : x; }
static inline int min(int x, int y) { return y < x ? y : x; }
static inline float clamp(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

static inline float sincos(float x, float* c)
{
    float s;
    sincosf(x, &s, c);
    return s;
}
static inline float native_sqrt(float x) { return sqrtf(x); }
static inline float sqrt(float x) { return sqrtf(x); }
static inline float log(float x) { return logf(x); }
static inline float exp(float x) { return expf(x); }
static inline float cos(float x) { return cosf(x); }
static inline float sin(float x) { return sinf(x); }
static inline float acos(float x) { return acosf(x); }
static inline float atan2(float y, float x) { return atan2f(y, x); }
static inline float fabs(float x) { return fabsf(x); }
static inline float floor(float x) { return floorf(x); }
static inline float rint(float x) { return rintf(x); }
static inline float round(float x) { return roundf(x); }

static inline float3 floor(float3 v) { return make_float3(floorf(v.x), floorf(v.y), floorf(v.z)); }
static inline float3 rint(float3 v) { return make_float3(rintf(v.x), rintf(v.y), rintf(v.z)); }
static inline int3 convert_int3(float3 v) { return make_int3((int)v.x, (int)v.y, (int)v.z); }

static inline uint mul_hi(uint a, uint b) { return (uint)(((unsigned long long)a * b) >> 32); }

// Relational built-ins on vectors: -1 (all bits) for true, 0 for false;
// all() tests the sign bit of every component.
static inline bool isfinite(float x) { return std::isfinite(x); }
static inline int3 isfinite(float3 v)
{
    return make_int3(std::isfinite(v.x) ? -1 : 0, std::isfinite(v.y) ? -1 : 0, std::isfinite(v.z) ? -1 : 0);
}
static inline int4 isfinite(float4 v)
{
    return make_int4(std::isfinite(v.x) ? -1 : 0, std::isfinite(v.y) ? -1 : 0, std::isfinite(v.z) ? -1 : 0,
                     std::isfinite(v.w) ? -1 : 0);
}
static inline int all(int3 v) { return v.x < 0 && v.y < 0 && v.z < 0; }
static inline int all(int4 v) { return v.x < 0 && v.y < 0 && v.z < 0 && v.w < 0; }

static inline uint atomic_cmpxchg(volatile uint* p, uint cmp, uint val)
{
    __atomic_compare_exchange_n(const_cast<uint*>(p), &cmp, val, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
    return cmp;
}
