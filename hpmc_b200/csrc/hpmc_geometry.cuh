// hpmc_geometry.cuh -- vertex geometry of one MC edge crossing
// (shadergen.cpp:512-563): crossing parameter t, position and normal.
//
// FP32 samples and FP32 outputs.  The crossing parameter and the normal lerp
// are evaluated in "float-float" arithmetic (error-free TwoSum / FMA
// transformations, ~44 significant bits) on the FP32 pipes: a normal that
// nearly cancels, (1-t) A + t B with A ~ -B, keeps its direction to the
// rounding of the FP32 result, and no float<->double conversions are issued.
#pragma once
#include "hpmc_fetch.cuh"

namespace hpmc {

struct FF {
    float hi, lo;
};

// a + b = s + e exactly (Knuth)
__device__ __forceinline__ FF two_sum(float a, float b) {
    const float s = a + b;
    const float bb = s - a;
    const float e = (a - (s - bb)) + (b - bb);
    return {s, e};
}

__device__ __forceinline__ FF ff_sub(FF a, FF b) {
    FF s = two_sum(a.hi, -b.hi);
    s.lo += a.lo - b.lo;
    return two_sum(s.hi, s.lo);
}

__device__ __forceinline__ FF ff_add(FF a, FF b) {
    FF s = two_sum(a.hi, b.hi);
    s.lo += a.lo + b.lo;
    return two_sum(s.hi, s.lo);
}

__device__ __forceinline__ FF ff_mul(FF a, FF b) {
    const float p = a.hi * b.hi;
    const float e = fmaf(a.hi, b.hi, -p) + (a.hi * b.lo + a.lo * b.hi);
    return two_sum(p, e);
}

// (a - b) / (c - d) for floats, as float-float
__device__ __forceinline__ FF ff_ratio_of_diffs(float a, float b, float c, float d) {
    const FF num = two_sum(a, -b);
    const FF den = two_sum(c, -d);
    const float q = num.hi / den.hi;
    float r = fmaf(-q, den.hi, num.hi);  // exact residual of the leading terms
    r += num.lo;
    r = fmaf(-q, den.lo, r);
    return two_sum(q, r / den.hi);
}

// lerp(A, B, t) = A + t (B - A), all float-float
__device__ __forceinline__ float ff_lerp(FF A, FF B, FF t) {
    const FF r = ff_add(A, ff_mul(t, ff_sub(B, A)));
    return r.hi + r.lo;
}

// Integer lattice index -> float without the conversion pipe (0 <= v < 2^23).
__device__ __forceinline__ float index_to_float(int v) { return __int_as_float(0x4B000000 | v) - 8388608.0f; }

// The field samples one vertex reads around its edge a -> b = a + e_axis:
// f(a), f(b), f(a +- e_i), f(b +- e_i).  All loads of a vertex are issued in
// one branch-free block: interior cells (every sample inside the lattice)
// through precomputed element offsets, boundary cells with each coordinate
// clamped (GL_CLAMP + NEAREST), functor fields by evaluating the functor.
struct EdgeField {
    float va, vb;
    float ap[3], bp[3];  // f(a + e_i), f(b + e_i)
    float am[3], bm[3];  // f(a - e_i), f(b - e_i)   (central differences only)
};

template <int FT, bool CENTRAL, class UF = NoUserField>
__device__ __forceinline__ void gather_edge(const Volume& V, const int* a, int axis, int cx, int cy, int cz,
                                            EdgeField& F) {
    const int ex = axis == 0, ey = axis == 1, ez = axis == 2;
    constexpr bool kArray = FT != kFieldFunctor && FT != kFieldUser;
    // samples span cell-1 .. cell+3 on each axis
    const bool interior = kArray && cx >= 1 && cx <= V.lattice[0] - 4 && cy >= 1 && cy <= V.lattice[1] - 4 &&
                          cz >= 1 && cz <= V.lattice[2] - 4;
    if (kArray && interior && V.idx32) {
        // 32-bit element offsets from the sample at a (one wide address each)
        using T = typename std::conditional<
            FT == kFieldF32, float, typename std::conditional<FT == kFieldF32X4, float4, unsigned char>::type>::type;
        const int o[3] = {1, (int)V.row_pitch, (int)V.slice_pitch};
        const T* pa = static_cast<const T*>(V.field) + (a[2] * o[2] + a[1] * o[1] + a[0]);
        const T* pb = pa + (axis == 0 ? o[0] : axis == 1 ? o[1] : o[2]);
        auto ld = [](const T* p) -> float {
            if constexpr (FT == kFieldF32) return __ldg(p);
            else if constexpr (FT == kFieldF32X4) return __ldg(&p->w);
            else if constexpr (FT == kFieldU8) return u8_to_float(__ldg(p));
            else return unorm8_to_float(__ldg(p));
        };
        F.va = ld(pa);
        F.vb = ld(pb);
#pragma unroll
        for (int i = 0; i < 3; i++) {
            F.ap[i] = ld(pa + o[i]);
            F.bp[i] = ld(pb + o[i]);
            if (CENTRAL) {
                F.am[i] = ld(pa - o[i]);
                F.bm[i] = ld(pb - o[i]);
            }
        }
    } else if (kArray && interior) {
        const long long o[3] = {1ll, V.row_pitch, V.slice_pitch};
        const long long pa = (long long)a[2] * V.slice_pitch + (long long)a[1] * V.row_pitch + a[0];
        const long long pb = pa + (axis == 0 ? o[0] : axis == 1 ? o[1] : o[2]);
        F.va = fetch_raw<FT>(V, pa);
        F.vb = fetch_raw<FT>(V, pb);
#pragma unroll
        for (int i = 0; i < 3; i++) {
            F.ap[i] = fetch_raw<FT>(V, pa + o[i]);
            F.bp[i] = fetch_raw<FT>(V, pb + o[i]);
            if (CENTRAL) {
                F.am[i] = fetch_raw<FT>(V, pa - o[i]);
                F.bm[i] = fetch_raw<FT>(V, pb - o[i]);
            }
        }
    } else {
        F.va = fetch<FT, UF>(V, a[0], a[1], a[2]);
        F.vb = fetch<FT, UF>(V, a[0] + ex, a[1] + ey, a[2] + ez);
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const int dx = i == 0, dy = i == 1, dz = i == 2;
            F.ap[i] = fetch<FT, UF>(V, a[0] + dx, a[1] + dy, a[2] + dz);
            F.bp[i] = fetch<FT, UF>(V, a[0] + ex + dx, a[1] + ey + dy, a[2] + ez + dz);
            if (CENTRAL) {
                F.am[i] = fetch<FT, UF>(V, a[0] - dx, a[1] - dy, a[2] - dz);
                F.bm[i] = fetch<FT, UF>(V, a[0] + ex - dx, a[1] + ey - dy, a[2] + ez - dz);
            }
        }
    }
}

enum { kGeomForward = 0, kGeomCentral = 1, kGeomBinary = 2 };

// Position (lattice index * extent / cells) and normal (scaled by extent /
// cells like the reference, shadergen.cpp:556-563) of the vertex on the edge
// from a (cell + shift) along `axis`.  Forward: n_i = iso - lerp(f(a+e_i),
// f(b+e_i), t); central: n_i = -lerp(g_i(a), g_i(b), t), g_i = half the
// central difference.
//
// The normal is first evaluated in plain FP32 (n_i = A_i + t (B_i - A_i) with
// A_i, B_i the end-point differences).  Its rounding error is bounded by
// 7u sqrt(sum_i (|A_i|+|B_i|)^2), u = 2^-24; when that bound exceeds 2e-6 of
// |n| (a normal that nearly cancels) the vertex is recomputed in float-float.
template <int FT, int MODE, class UF = NoUserField>
__device__ __forceinline__ void edge_vertex(const Volume& V, const int* a, int axis, int cx, int cy, int cz,
                                            const float* binary_normal, float p[3], float n[3], float& t_out) {
    float t;
    if (MODE == kGeomBinary) {
        t = 0.5f;
        n[0] = binary_normal[0];
        n[1] = binary_normal[1];
        n[2] = binary_normal[2];
    } else if (V.gradient) {
        // gradient mode (shadergen.cpp:539-551): t from the values at a and b,
        // the gradients from HPMC_fetchGrad -- a functor's analytic gradient or
        // the .xyz of an RGBA field (single-channel fields read zero there, as
        // GL's alpha textures do); forward mode keeps the reference's
        // n = iso - lerp(grad a, grad b, t), central mode gives -lerp(grad a, grad b, t)
        const int b[3] = {a[0] + (axis == 0), a[1] + (axis == 1), a[2] + (axis == 2)};
        float va, vb, ga[3] = {0.f, 0.f, 0.f}, gb[3] = {0.f, 0.f, 0.f};
        if constexpr (FT == kFieldFunctor) {
            const float pa[3] = {texel_centre(a[0], V.lattice[0]), texel_centre(a[1], V.lattice[1]),
                                 texel_centre(a[2], V.lattice[2])};
            const float pb[3] = {texel_centre(b[0], V.lattice[0]), texel_centre(b[1], V.lattice[1]),
                                 texel_centre(b[2], V.lattice[2])};
            va = functor_value(V.functor, pa[0], pa[1], pa[2]);
            vb = functor_value(V.functor, pb[0], pb[1], pb[2]);
            functor_gradient(V.functor, pa[0], pa[1], pa[2], ga[0], ga[1], ga[2]);
            functor_gradient(V.functor, pb[0], pb[1], pb[2], gb[0], gb[1], gb[2]);
        } else if constexpr (FT == kFieldUser) {
            const float pa[3] = {texel_centre(a[0], V.lattice[0]), texel_centre(a[1], V.lattice[1]),
                                 texel_centre(a[2], V.lattice[2])};
            const float pb[3] = {texel_centre(b[0], V.lattice[0]), texel_centre(b[1], V.lattice[1]),
                                 texel_centre(b[2], V.lattice[2])};
            va = UF::value(V.functor.p, V.functor.count, pa[0], pa[1], pa[2]);
            vb = UF::value(V.functor.p, V.functor.count, pb[0], pb[1], pb[2]);
            if constexpr (UF::kHasGradient) {
                UF::gradient(V.functor.p, V.functor.count, pa[0], pa[1], pa[2], ga);
                UF::gradient(V.functor.p, V.functor.count, pb[0], pb[1], pb[2], gb);
            }
        } else if constexpr (FT == kFieldF32X4) {
            const float4 sa = fetch_rgba(V, a[0], a[1], a[2]), sb = fetch_rgba(V, b[0], b[1], b[2]);
            va = sa.w;
            vb = sb.w;
            ga[0] = sa.x; ga[1] = sa.y; ga[2] = sa.z;
            gb[0] = sb.x; gb[1] = sb.y; gb[2] = sb.z;
        } else {
            va = fetch<FT, UF>(V, a[0], a[1], a[2]);
            vb = fetch<FT, UF>(V, b[0], b[1], b[2]);
        }
        const float iso = V.iso;
        const FF tf = ff_ratio_of_diffs(va, iso, va, vb);
        t = tf.hi + tf.lo;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const float g = ff_lerp(FF{ga[i], 0.0f}, FF{gb[i], 0.0f}, tf);
            n[i] = (MODE == kGeomCentral) ? -g : iso - g;
        }
    } else {
        EdgeField F;
        gather_edge<FT, MODE == kGeomCentral, UF>(V, a, axis, cx, cy, cz, F);
        const float iso = V.iso;
        t = (F.va - iso) / (F.va - F.vb);  // (f(a) - iso) / (f(a) - f(b)), relative error <= 3u
        float s2 = 0.0f, n2 = 0.0f;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            float A, B;
            if (MODE == kGeomForward) {
                A = iso - F.ap[i];
                B = iso - F.bp[i];
            } else {
                A = F.ap[i] - F.am[i];
                B = F.bp[i] - F.bm[i];
            }
            n[i] = fmaf(t, B - A, A);
            const float s = fabsf(A) + fabsf(B);
            s2 = fmaf(s, s, s2);
            n2 = fmaf(n[i], n[i], n2);
        }
        if (s2 > 23.0f * n2) {
            // ill-conditioned: float-float crossing parameter and lerps
            const FF tf = ff_ratio_of_diffs(F.va, iso, F.va, F.vb);
#pragma unroll
            for (int i = 0; i < 3; i++) {
                if (MODE == kGeomForward)
                    n[i] = ff_lerp(two_sum(iso, -F.ap[i]), two_sum(iso, -F.bp[i]), tf);
                else
                    n[i] = ff_lerp(two_sum(F.ap[i], -F.am[i]), two_sum(F.bp[i], -F.bm[i]), tf);
            }
            t = tf.hi + tf.lo;
        }
        if (MODE == kGeomCentral) {
#pragma unroll
            for (int i = 0; i < 3; i++) n[i] *= -0.5f;
        }
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
        float q = index_to_float(a[i]);
        if (i == axis) q += t;
        p[i] = q * V.scale[i];
        n[i] *= V.scale[i];
    }
    t_out = t;
}

}  // namespace hpmc
