// hpmc_fetch.cuh -- scalar-field access: device arrays and registered functors.
//
// Array fields follow the reference's Texture3D fetch (shadergen.cpp:245-268
// with apps/texture3d/texture3d.cpp:135-139): NEAREST sampling at texel
// centres with GL_CLAMP, i.e. clamp-to-edge integer indexing.  uint8 arrays
// read either as float(b) (kFieldU8) or as GL's normalised b/255
// (kFieldUNorm8, a GL_ALPHA/GL_UNSIGNED_BYTE texture).  float4 arrays
// (kFieldF32X4) hold a GL RGBA float texture: the field is the alpha (value)
// channel, and the gradient-mode traversal reads .xyz as the gradient
// (shadergen.cpp:260-266).
//
// Functor fields replace the reference's custom GLSL fetch snippet
// (HPMCsetFieldCustom, hpiface.cpp:187-200; shadergen.cpp:270-286): the
// snippet's HPMC_fetch(p) receives normalised texel centres
// p = ((x+0.5)/FX, (y+0.5)/FY, (z+0.5)/FZ) without clamping (hpmc.h:409-444);
// here a registered device functor receives the same p.
#pragma once
#include "hpmc_device.cuh"

namespace hpmc {

enum FunctorId : int {
    kFunctorCayley = 1,         // apps/cayley/cayley.cpp:75-94 (with gradient)
    kFunctorMetaballs = 2,      // sum_i r_i^2 / |p - c_i|^2; p = {n, (cx,cy,cz,r) x n}
    kFunctorTwistMetaballs = 3, // apps/metaballs/metaballs.cpp:72-94; p = {twist, (cx,cy,cz) x 8}
    kFunctorSpheres = 4,        // signed distance of a union of spheres; p = {n, (cx,cy,cz,r) x n}
};

// Functor arithmetic is written with round-to-nearest intrinsics in a fixed
// order (no FMA contraction), so a host restatement in plain FP32 C with
// contraction off gives bit-identical values -- and the same topology.
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }

__device__ __forceinline__ float functor_value(const FunctorParams& F, float px, float py, float pz) {
    switch (F.id) {
        case kFunctorCayley: {
            const float x = fs(fm(2.0f, px), 1.0f), y = fs(fm(2.0f, py), 1.0f), z = fs(fm(2.0f, pz), 1.0f);
            // 1 - 16xyz - 4x^2 - 4y^2 - 4z^2, left to right
            float v = fs(1.0f, fm(fm(fm(16.0f, x), y), z));
            v = fs(v, fm(fm(4.0f, x), x));
            v = fs(v, fm(fm(4.0f, y), y));
            return fs(v, fm(fm(4.0f, z), z));
        }
        case kFunctorMetaballs: {
            const int n = (int)F.p[0];
            float s = 0.0f;
            for (int i = 0; i < n; i++) {
                const float dx = fs(px, F.p[1 + 4 * i]), dy = fs(py, F.p[2 + 4 * i]), dz = fs(pz, F.p[3 + 4 * i]);
                const float r = F.p[4 + 4 * i];
                s = fa(s, __fdiv_rn(fm(r, r), fa(fa(fm(dx, dx), fm(dy, dy)), fm(dz, dz))));
            }
            return s;
        }
        case kFunctorTwistMetaballs: {
            // sin/cos: device and host libraries round differently, so this
            // functor agrees with a host restatement only to a few ulps
            float x = 2.0f * px - 1.0f, y = 2.0f * py - 1.0f, z = 2.0f * pz - 1.0f;
            float twist = F.p[0];
            float rot1 = twist * z, rot2 = 0.7f * twist * y;
            float c1 = cosf(rot1), s1 = sinf(rot1), c2 = cosf(rot2), s2 = sinf(rot2);
            // GLSL mat3 constructors are column-major: p' = M p
            float x1 = c1 * x + s1 * y, y1 = -s1 * x + c1 * y, z1 = z;
            float x2 = c2 * x1 + s2 * z1, y2 = y1, z2 = -s2 * x1 + c2 * z1;
            x = 0.5f * x2 + 0.5f;
            y = 0.5f * y2 + 0.5f;
            z = 0.5f * z2 + 0.5f;
            float s = 0.0f;
            for (int i = 0; i < 8; i++) {
                float dx = x - F.p[1 + 3 * i], dy = y - F.p[2 + 3 * i], dz = z - F.p[3 + 3 * i];
                s += 0.05f / (dx * dx + dy * dy + dz * dz);
            }
            return s;
        }
        case kFunctorSpheres: {
            const int n = (int)F.p[0];
            float d = 3.0e38f;
            for (int i = 0; i < n; i++) {
                const float dx = fs(px, F.p[1 + 4 * i]), dy = fs(py, F.p[2 + 4 * i]), dz = fs(pz, F.p[3 + 4 * i]);
                d = fminf(d, fs(__fsqrt_rn(fa(fa(fm(dx, dx), fm(dy, dy)), fm(dz, dz))), F.p[4 + 4 * i]));
            }
            return d;
        }
        default:
            return 0.0f;
    }
}

// Functors with an analytic gradient (HPMC_fetchGrad of the reference's
// custom snippet, e.g. apps/cayley/cayley.cpp:85-93).
__host__ __device__ __forceinline__ bool functor_has_gradient(int id) { return id == kFunctorCayley; }

// The gradient in the snippet's own coordinates (cayley: with respect to
// x = 2p - 1, as apps/cayley/cayley.cpp:90-92 returns it).
__device__ __forceinline__ void functor_gradient(const FunctorParams& F, float px, float py, float pz,
                                                 float& gx, float& gy, float& gz) {
    if (F.id == kFunctorCayley) {
        const float x = fs(fm(2.0f, px), 1.0f), y = fs(fm(2.0f, py), 1.0f), z = fs(fm(2.0f, pz), 1.0f);
        gx = fs(fm(fm(-16.0f, y), z), fm(8.0f, x));
        gy = fs(fm(fm(-16.0f, x), z), fm(8.0f, y));
        gz = fs(fm(fm(-16.0f, x), y), fm(8.0f, z));
    } else {
        gx = gy = gz = 0.0f;
    }
}

// Texel centre of lattice index i along an axis of `n` samples (the
// reference's normalised coordinate, shadergen.cpp:257).
__device__ __forceinline__ float texel_centre(int i, int n) {
    return __fdiv_rn(fa((float)i, 0.5f), (float)n);
}

// uint8 -> float without the conversion pipe: exact for b < 2^23.
__device__ __forceinline__ float u8_to_float(uint32_t b) {
    return __int_as_float(0x4B000000u | b) - 8388608.0f;
}

// b/255 correctly rounded (GL's UNORM8 -> float) with two FMAs; equal to the
// IEEE quotient for every b in 0..255 (checked exhaustively).
__device__ __forceinline__ float unorm8_to_float(uint32_t b) {
    const float fb = u8_to_float(b);
    const float r255 = 1.0f / 255.0f;
    const float q = fb * r255;
    return fmaf(fmaf(-q, 255.0f, fb), r255, q);
}

template <int FT>
__device__ __forceinline__ float fetch_raw(const Volume& V, long long off) {
    if constexpr (FT == kFieldF32) {
        return __ldg(static_cast<const float*>(V.field) + off);
    } else if constexpr (FT == kFieldF32X4) {
        return __ldg(static_cast<const float*>(V.field) + 4 * off + 3);
    } else if constexpr (FT == kFieldU8) {
        return u8_to_float(__ldg(static_cast<const unsigned char*>(V.field) + off));
    } else {
        return unorm8_to_float(__ldg(static_cast<const unsigned char*>(V.field) + off));
    }
}

// f(x,y,z) with the reference's addressing; x,y,z may lie outside the lattice.
// UF: the caller's functor type when FT == kFieldUser (include/hpmc_functor.cuh).
template <int FT, class UF = NoUserField>
__device__ __forceinline__ float fetch(const Volume& V, int x, int y, int z) {
    if constexpr (FT == kFieldFunctor) {
        return functor_value(V.functor, texel_centre(x, V.lattice[0]), texel_centre(y, V.lattice[1]),
                             texel_centre(z, V.lattice[2]));
    } else if constexpr (FT == kFieldUser) {
        return UF::value(V.functor.p, V.functor.count, texel_centre(x, V.lattice[0]),
                         texel_centre(y, V.lattice[1]), texel_centre(z, V.lattice[2]));
    } else {
        x = min(max(x, 0), V.lattice[0] - 1);
        y = min(max(y, 0), V.lattice[1] - 1);
        z = min(max(z, 0), V.lattice[2] - 1);
        return fetch_raw<FT>(V, (long long)z * V.slice_pitch + (long long)y * V.row_pitch + x);
    }
}

// The whole RGBA sample (gradient x, y, z, value) of a float4 field, with the
// reference's clamp-to-edge addressing.
__device__ __forceinline__ float4 fetch_rgba(const Volume& V, int x, int y, int z) {
    x = min(max(x, 0), V.lattice[0] - 1);
    y = min(max(y, 0), V.lattice[1] - 1);
    z = min(max(z, 0), V.lattice[2] - 1);
    return __ldg(static_cast<const float4*>(V.field) + ((long long)z * V.slice_pitch + (long long)y * V.row_pitch + x));
}

}  // namespace hpmc
