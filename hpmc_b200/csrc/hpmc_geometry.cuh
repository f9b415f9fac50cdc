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

// Samples around edge end point a: interior cells (all samples inside the
// lattice) read through precomputed element offsets, others clamp each
// coordinate (GL_CLAMP + NEAREST).  Functor fields evaluate the functor.
template <int FT>
struct EdgeSamples {
    const Volume& V;
    int a[3];
    int ex, ey, ez;            // a -> b
    long long base, ob;        // element index of a; offset a -> b
    long long o[3];            // offsets of +x, +y, +z
    bool interior;
    __device__ __forceinline__ EdgeSamples(const Volume& Vv, const int* aa, int axis, int cx, int cy, int cz)
        : V(Vv) {
        a[0] = aa[0];
        a[1] = aa[1];
        a[2] = aa[2];
        ex = axis == 0;
        ey = axis == 1;
        ez = axis == 2;
        // samples span cell-1 .. cell+3 on each axis
        interior = FT != kFieldFunctor && cx >= 1 && cx <= V.lattice[0] - 4 && cy >= 1 &&
                   cy <= V.lattice[1] - 4 && cz >= 1 && cz <= V.lattice[2] - 4;
        o[0] = 1;
        o[1] = V.row_pitch;
        o[2] = V.slice_pitch;
        base = (long long)a[2] * V.slice_pitch + (long long)a[1] * V.row_pitch + a[0];
        ob = axis == 0 ? o[0] : axis == 1 ? o[1] : o[2];
    }
    // f(a + (dx,dy,dz)) given the matching element offset
    __device__ __forceinline__ float at(int dx, int dy, int dz, long long off) const {
        if (FT != kFieldFunctor && interior) return fetch_raw<FT>(V, base + off);
        return fetch<FT>(V, a[0] + dx, a[1] + dy, a[2] + dz);
    }
    __device__ __forceinline__ float fa() const { return at(0, 0, 0, 0); }
    __device__ __forceinline__ float fb() const { return at(ex, ey, ez, ob); }
    __device__ __forceinline__ float fa_plus(int i) const { return at(i == 0, i == 1, i == 2, o[i]); }
    __device__ __forceinline__ float fa_minus(int i) const { return at(-(i == 0), -(i == 1), -(i == 2), -o[i]); }
    __device__ __forceinline__ float fb_plus(int i) const {
        return at(ex + (i == 0), ey + (i == 1), ez + (i == 2), ob + o[i]);
    }
    __device__ __forceinline__ float fb_minus(int i) const {
        return at(ex - (i == 0), ey - (i == 1), ez - (i == 2), ob - o[i]);
    }
};

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
template <int FT, int MODE>
__device__ __forceinline__ void edge_vertex(const Volume& V, const int* a, int axis, int cx, int cy, int cz,
                                            const float* binary_normal, float p[3], float n[3], float& t_out) {
    float t;
    if (MODE == kGeomBinary) {
        t = 0.5f;
        n[0] = binary_normal[0];
        n[1] = binary_normal[1];
        n[2] = binary_normal[2];
    } else {
        const EdgeSamples<FT> f(V, a, axis, cx, cy, cz);
        const float iso = V.iso;
        const float va = f.fa(), vb = f.fb();
        t = (va - iso) / (va - vb);  // (f(a) - iso) / (f(a) - f(b)), relative error <= 3u
        float s2 = 0.0f, n2 = 0.0f;
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const float fap = (i == axis) ? vb : f.fa_plus(i);
            const float fbp = f.fb_plus(i);
            float A, B;
            if (MODE == kGeomForward) {
                A = iso - fap;
                B = iso - fbp;
            } else {
                A = fap - f.fa_minus(i);
                B = fbp - ((i == axis) ? va : f.fb_minus(i));
            }
            n[i] = fmaf(t, B - A, A);
            const float s = fabsf(A) + fabsf(B);
            s2 = fmaf(s, s, s2);
            n2 = fmaf(n[i], n[i], n2);
        }
        if (s2 > 23.0f * n2) {
            // ill-conditioned: float-float crossing parameter and lerps
            const FF tf = ff_ratio_of_diffs(va, iso, va, vb);
#pragma unroll
            for (int i = 0; i < 3; i++) {
                const float fap = (i == axis) ? vb : f.fa_plus(i);
                const float fbp = f.fb_plus(i);
                if (MODE == kGeomForward) {
                    n[i] = ff_lerp(two_sum(iso, -fap), two_sum(iso, -fbp), tf);
                } else {
                    const float fam = f.fa_minus(i);
                    const float fbm = (i == axis) ? va : f.fb_minus(i);
                    n[i] = ff_lerp(two_sum(fap, -fam), two_sum(fbp, -fbm), tf);
                }
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
