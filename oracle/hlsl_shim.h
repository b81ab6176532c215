// ORACLE -- test infrastructure only.  A small host C++ stand-in for the HLSL/Slang vector types and
// intrinsics that the reference's shader math uses (src/Shaders/common/rng.hlsli, common.hlsli,
// microfacet.hlsli and D3DX_DXGIFormatConvert.inl of Stratum2), so that those files compile as host
// C++ and the oracle can be checked against the reference's own code.  Component-wise semantics as
// in HLSL: vector-vector and vector-scalar arithmetic, comparisons giving bool vectors, scalar
// broadcast on construction.  Swizzles are member functions (xy(), yx(), set_xy()); the build
// recipe (oracle/build_oracle.py) rewrites the few swizzles the shaders use into those calls.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>

namespace hlsl {

typedef uint32_t uint;

template <class T, int N> struct vec;

template <class T> struct vec<T, 2> {
    T x, y;
    vec() : x(0), y(0) {}
    vec(T s) : x(s), y(s) {}
    vec(T a, T b) : x(a), y(b) {}
    template <class U> explicit vec(const vec<U, 2>& o) : x((T)o.x), y((T)o.y) {}
    T& operator[](int i) { return i == 0 ? x : y; }
    T operator[](int i) const { return i == 0 ? x : y; }
    vec<T, 2> yx() const { return vec<T, 2>(y, x); }
};
template <class T> struct vec<T, 3> {
    T x, y, z;
    vec() : x(0), y(0), z(0) {}
    vec(T s) : x(s), y(s), z(s) {}
    vec(T a, T b, T c) : x(a), y(b), z(c) {}
    vec(const vec<T, 2>& v, T c) : x(v.x), y(v.y), z(c) {}
    template <class U> explicit vec(const vec<U, 3>& o) : x((T)o.x), y((T)o.y), z((T)o.z) {}
    T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    vec<T, 2> xy() const { return vec<T, 2>(x, y); }
    vec<T, 2> yx() const { return vec<T, 2>(y, x); }
    void set_xy(const vec<T, 2>& v) { x = v.x; y = v.y; }
};
template <class T> struct vec<T, 4> {
    T x, y, z, w;
    vec() : x(0), y(0), z(0), w(0) {}
    vec(T s) : x(s), y(s), z(s), w(s) {}
    vec(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
    vec(const vec<T, 2>& v, T c, T d) : x(v.x), y(v.y), z(c), w(d) {}
    vec(const vec<T, 3>& v, T d) : x(v.x), y(v.y), z(v.z), w(d) {}
    template <class U> explicit vec(const vec<U, 4>& o) : x((T)o.x), y((T)o.y), z((T)o.z), w((T)o.w) {}
    T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    vec<T, 2> xy() const { return vec<T, 2>(x, y); }
};

typedef vec<float, 2> float2;
typedef vec<float, 3> float3;
typedef vec<float, 4> float4;
typedef vec<int, 2> int2;
typedef vec<int, 4> int4;
typedef vec<uint, 2> uint2;
typedef vec<uint, 4> uint4;
typedef vec<bool, 2> bool2;
typedef vec<bool, 3> bool3;

struct float3x3 {
    float3 r[3];
    float3& operator[](int i) { return r[i]; }
    const float3& operator[](int i) const { return r[i]; }
};

// ---- component-wise operators (vector op vector, vector op scalar, scalar op vector)
#define HLSL_BINOP(OP)                                                                             \
    template <class T, int N> vec<T, N> operator OP(const vec<T, N>& a, const vec<T, N>& b) {     \
        vec<T, N> r;                                                                               \
        for (int i = 0; i < N; ++i) r[i] = a[i] OP b[i];                                           \
        return r;                                                                                  \
    }                                                                                              \
    template <class T, int N, class S, class = std::enable_if_t<std::is_arithmetic<S>::value>>     \
    vec<T, N> operator OP(const vec<T, N>& a, S s) {                                               \
        vec<T, N> r;                                                                               \
        for (int i = 0; i < N; ++i) r[i] = a[i] OP (T)s;                                           \
        return r;                                                                                  \
    }                                                                                              \
    template <class T, int N, class S, class = std::enable_if_t<std::is_arithmetic<S>::value>>     \
    vec<T, N> operator OP(S s, const vec<T, N>& a) {                                               \
        vec<T, N> r;                                                                               \
        for (int i = 0; i < N; ++i) r[i] = (T)s OP a[i];                                           \
        return r;                                                                                  \
    }
HLSL_BINOP(+)
HLSL_BINOP(-)
HLSL_BINOP(*)
HLSL_BINOP(/)
HLSL_BINOP(^)
HLSL_BINOP(|)
HLSL_BINOP(&)
HLSL_BINOP(>>)
HLSL_BINOP(<<)
#undef HLSL_BINOP

#define HLSL_CMP(OP)                                                                               \
    template <class T, int N, class S, class = std::enable_if_t<std::is_arithmetic<S>::value>>     \
    vec<bool, N> operator OP(const vec<T, N>& a, S s) {                                            \
        vec<bool, N> r;                                                                            \
        for (int i = 0; i < N; ++i) r[i] = a[i] OP (T)s;                                           \
        return r;                                                                                  \
    }
HLSL_CMP(>=)
HLSL_CMP(<=)
HLSL_CMP(>)
HLSL_CMP(<)
#undef HLSL_CMP

template <class T, int N> vec<T, N> operator-(const vec<T, N>& a) {
    vec<T, N> r;
    for (int i = 0; i < N; ++i) r[i] = -a[i];
    return r;
}
template <class T, int N> vec<T, N>& operator+=(vec<T, N>& a, const vec<T, N>& b) { return a = a + b; }
template <class T, int N> vec<T, N>& operator*=(vec<T, N>& a, const vec<T, N>& b) { return a = a * b; }

// ---- scalar intrinsics (float overloads: HLSL float arithmetic, not double)
inline float sqrt(float x) { return std::sqrt(x); }
inline float pow(float x, float y) { return std::pow(x, y); }
inline float log(float x) { return std::log(x); }
inline float cos(float x) { return std::cos(x); }
inline float sin(float x) { return std::sin(x); }
inline float floor(float x) { return std::floor(x); }
inline float trunc(float x) { return std::trunc(x); }
inline float abs(float x) { return std::fabs(x); }
inline int abs(int x) { return x < 0 ? -x : x; }
inline bool isnan(float x) { return std::isnan(x); }
inline float saturate(float x) { return x < 0.f ? 0.f : (x > 1.f ? 1.f : x); }
template <class A, class B, class = std::enable_if_t<std::is_arithmetic<A>::value && std::is_arithmetic<B>::value>>
inline std::common_type_t<A, B> max(A a, B b) {
    typedef std::common_type_t<A, B> T;
    return (T)a > (T)b ? (T)a : (T)b;
}
template <class A, class B, class = std::enable_if_t<std::is_arithmetic<A>::value && std::is_arithmetic<B>::value>>
inline std::common_type_t<A, B> min(A a, B b) {
    typedef std::common_type_t<A, B> T;
    return (T)a < (T)b ? (T)a : (T)b;
}
inline float asfloat(uint u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint asuint(float f) { uint u; std::memcpy(&u, &f, 4); return u; }
inline float4 asfloat(const uint4& u) { return float4(asfloat(u.x), asfloat(u.y), asfloat(u.z), asfloat(u.w)); }
// half conversions (f32tof16 / f16tof32): IEEE binary16 in the low 16 bits, round to nearest even
inline uint f32tof16(float f) { _Float16 h = (_Float16)f; uint16_t b; std::memcpy(&b, &h, 2); return b; }
inline float f16tof32(uint u) { const uint16_t b = (uint16_t)(u & 0xffffu); _Float16 h; std::memcpy(&h, &b, 2); return (float)h; }

// ---- vector intrinsics
template <int N> vec<float, N> abs(const vec<float, N>& a) {
    vec<float, N> r;
    for (int i = 0; i < N; ++i) r[i] = std::fabs(a[i]);
    return r;
}
template <class T, int N> T dot(const vec<T, N>& a, const vec<T, N>& b) {
    T s = 0;
    for (int i = 0; i < N; ++i) s += a[i] * b[i];
    return s;
}
template <class T, int N, class S, class = std::enable_if_t<std::is_arithmetic<S>::value>>
T dot(S s, const vec<T, N>& b) { return dot(vec<T, N>((T)s), b); }
inline float3 cross(const float3& a, const float3& b) {
    return float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <int N> vec<float, N> normalize(const vec<float, N>& a) { return a / sqrt(dot(a, a)); }
template <int N> vec<float, N> saturate(const vec<float, N>& a) {
    vec<float, N> r;
    for (int i = 0; i < N; ++i) r[i] = saturate(a[i]);
    return r;
}
// lerp(a, b, t) = a + (b - a) t, with scalar ends and a vector t as the shaders call it
template <int N> vec<float, N> lerp(float a, float b, const vec<float, N>& t) { return a + (b - a) * t; }

}  // namespace hlsl
