// glsl_emu.hpp -- TEST INFRASTRUCTURE: a minimal GLSL-subset runtime in C++,
// enough to compile and run the shader text that the reference's shader
// generator (hpmc/src/shadergen.cpp) emits for texture fields, so that the
// oracle can be checked against the reference's own arithmetic without a GL
// driver (none exists on this machine).
//
// Covered: float/int/bool vectors of 2-4 components with .x .y .z .w members
// and .xy()/.xyz() swizzles (also as assignable views), component-wise
// arithmetic, floor/fract/dot/mix/equal, and samplers with NEAREST filtering
// and GL_CLAMP wrapping (the reference's texture setup,
// apps/texture3d/texture3d.cpp:135-139, texfbosetup.cpp).  Literals are
// rewritten to float by the translator, so arithmetic is FP32 as in GLSL.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

namespace glsl {

struct vec2;
struct vec3;
struct vec4;

struct ivec2 {
    int x, y;
    ivec2() : x(0), y(0) {}
    ivec2(int a, int b) : x(a), y(b) {}
    explicit ivec2(const vec2& v);
    ivec2& operator+=(const ivec2& o) { x += o.x; y += o.y; return *this; }
};
inline ivec2 operator*(int s, const ivec2& v) { return ivec2(s * v.x, s * v.y); }
inline ivec2 operator+(const ivec2& a, const ivec2& b) { return ivec2(a.x + b.x, a.y + b.y); }

struct bvec2 {
    bool x, y;
    bvec2(bool a, bool b) : x(a), y(b) {}
};
struct bvec3 {
    bool x, y, z;
    bvec3(bool a, bool b, bool c) : x(a), y(b), z(c) {}
};

// assignable two-component view (p.xy -= ...)
struct swz2 {
    float& a;
    float& b;
    inline swz2& operator-=(const vec2& o);
    inline swz2& operator+=(const vec2& o);
    inline swz2& operator*=(const vec2& o);
    inline operator vec2() const;
};

struct vec2 {
    float x, y;
    vec2() : x(0), y(0) {}
    explicit vec2(float s) : x(s), y(s) {}
    vec2(float a, float b) : x(a), y(b) {}
    explicit vec2(const ivec2& v) : x((float)v.x), y((float)v.y) {}
    vec2(const swz2& s) : x(s.a), y(s.b) {}
    swz2 xy() { return swz2{x, y}; }
};
inline ivec2::ivec2(const vec2& v) : x((int)v.x), y((int)v.y) {}
inline swz2& swz2::operator-=(const vec2& o) { a -= o.x; b -= o.y; return *this; }
inline swz2& swz2::operator+=(const vec2& o) { a += o.x; b += o.y; return *this; }
inline swz2& swz2::operator*=(const vec2& o) { a *= o.x; b *= o.y; return *this; }
inline swz2::operator vec2() const { return vec2(a, b); }

struct vec3 {
    float x, y, z;
    vec3() : x(0), y(0), z(0) {}
    explicit vec3(float s) : x(s), y(s), z(s) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    vec3(const vec2& v, float c) : x(v.x), y(v.y), z(c) {}
    explicit vec3(const bvec3& b) : x(b.x ? 1.f : 0.f), y(b.y ? 1.f : 0.f), z(b.z ? 1.f : 0.f) {}
    swz2 xy() { return swz2{x, y}; }
    vec2 xy() const { return vec2(x, y); }
    vec3& operator+=(const vec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
    vec3& operator*=(const vec3& o) { x *= o.x; y *= o.y; z *= o.z; return *this; }
    vec3& operator*=(float s) { x *= s; y *= s; z *= s; return *this; }
    vec3& operator-=(float s) { x -= s; y -= s; z -= s; return *this; }
    vec3& operator+=(float s) { x += s; y += s; z += s; return *this; }
};

struct vec4 {
    float x, y, z, w;
    vec4() : x(0), y(0), z(0), w(0) {}
    explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
    vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    vec2 xy() const { return vec2(x, y); }
    vec3 xyz() const { return vec3(x, y, z); }
    float a() const { return w; }
};

#define GLSL_V2(op) \
    inline vec2 operator op(const vec2& a, const vec2& b) { return vec2(a.x op b.x, a.y op b.y); } \
    inline vec2 operator op(float s, const vec2& b) { return vec2(s op b.x, s op b.y); } \
    inline vec2 operator op(const vec2& a, float s) { return vec2(a.x op s, a.y op s); }
#define GLSL_V3(op) \
    inline vec3 operator op(const vec3& a, const vec3& b) { return vec3(a.x op b.x, a.y op b.y, a.z op b.z); } \
    inline vec3 operator op(float s, const vec3& b) { return vec3(s op b.x, s op b.y, s op b.z); } \
    inline vec3 operator op(const vec3& a, float s) { return vec3(a.x op s, a.y op s, a.z op s); }
#define GLSL_V4(op) \
    inline vec4 operator op(const vec4& a, const vec4& b) { \
        return vec4(a.x op b.x, a.y op b.y, a.z op b.z, a.w op b.w); } \
    inline vec4 operator op(float s, const vec4& b) { return vec4(s op b.x, s op b.y, s op b.z, s op b.w); }
GLSL_V2(+) GLSL_V2(-) GLSL_V2(*) GLSL_V2(/)
GLSL_V3(+) GLSL_V3(-) GLSL_V3(*) GLSL_V3(/)
GLSL_V4(+) GLSL_V4(-) GLSL_V4(*)
#undef GLSL_V2
#undef GLSL_V3
#undef GLSL_V4

inline float floor(float v) { return std::floor(v); }
inline vec2 floor(const vec2& v) { return vec2(std::floor(v.x), std::floor(v.y)); }
inline vec3 floor(const vec3& v) { return vec3(std::floor(v.x), std::floor(v.y), std::floor(v.z)); }
inline vec4 floor(const vec4& v) { return vec4(std::floor(v.x), std::floor(v.y), std::floor(v.z), std::floor(v.w)); }
inline float fract(float v) { return v - std::floor(v); }
inline vec2 fract(const vec2& v) { return vec2(fract(v.x), fract(v.y)); }
inline vec3 fract(const vec3& v) { return vec3(fract(v.x), fract(v.y), fract(v.z)); }
inline float dot(const vec2& a, const vec2& b) { return a.x * b.x + a.y * b.y; }
inline float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(const vec4& a, const vec4& b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
// GLSL mix(x, y, a) = x * (1 - a) + y * a
inline vec3 mix(const vec3& x, const vec3& y, float a) { return x * (1.0f - a) + y * a; }
inline bvec3 equal(const vec3& a, const vec3& b) { return bvec3(a.x == b.x, a.y == b.y, a.z == b.z); }

// --- textures: NEAREST + GL_CLAMP; texel (i) of coordinate u over n texels
inline int nearest(float u, int n) {
    u = u < 0.f ? 0.f : (u > 1.f ? 1.f : u);
    int i = (int)std::floor(u * (float)n);
    return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

struct sampler1D {
    const float* rgba = nullptr;  // n texels x 4
    int n = 0;
};
struct sampler2D {
    // level l: w_l x h_l texels x 4, row-major
    std::vector<const float*> levels;
    std::vector<int> w, h;
};
struct sampler3D {
    const float* alpha = nullptr;  // x fastest, one channel (.a)
    const float* rgba = nullptr;   // or x fastest, four channels (an RGBA float texture)
    int nx = 0, ny = 0, nz = 0;
};

inline vec4 texture1D(const sampler1D& s, float u) {
    const float* t = s.rgba + 4 * nearest(u, s.n);
    return vec4(t[0], t[1], t[2], t[3]);
}
inline vec4 texture2D(const sampler2D& s, const vec2& uv) {
    const int i = nearest(uv.x, s.w[0]), j = nearest(uv.y, s.h[0]);
    const float* t = s.levels[0] + 4 * ((size_t)j * s.w[0] + i);
    return vec4(t[0], t[1], t[2], t[3]);
}
inline vec4 texelFetch(const sampler2D& s, const ivec2& p, int level) {
    const float* t = s.levels[level] + 4 * ((size_t)p.y * s.w[level] + p.x);
    return vec4(t[0], t[1], t[2], t[3]);
}
inline vec4 texture3D(const sampler3D& s, const vec3& p) {
    const int i = nearest(p.x, s.nx), j = nearest(p.y, s.ny), k = nearest(p.z, s.nz);
    const size_t o = ((size_t)k * s.ny + j) * s.nx + i;
    if (s.rgba) return vec4(s.rgba[4 * o], s.rgba[4 * o + 1], s.rgba[4 * o + 2], s.rgba[4 * o + 3]);
    return vec4(0.f, 0.f, 0.f, s.alpha[o]);  // a GL_ALPHA texture reads rgb = 0
}

}  // namespace glsl
