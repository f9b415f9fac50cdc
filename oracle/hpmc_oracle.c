/*
 * hpmc_oracle.c -- CPU restatement of HPMC's HistoPyramid marching cubes.
 *
 * TEST INFRASTRUCTURE ONLY (see hpmc_oracle.h).  Links the reference's own
 * tables (hpmc/src/tables.cpp, compiled from the HPMC tree by
 * oracle/Makefile); every other line is a restatement with a citation.
 * Built with -ffp-contract=off so float table derivations round exactly as
 * the reference's host code does.
 */
#include "hpmc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* The reference's tables, linked from hpmc/src/tables.cpp (global C++
 * arrays have unmangled symbol names). */
extern int HPMC_triangle_table[256][16];  /* tables.cpp:38-296, Bourke case order */
extern float HPMC_edge_table[12][4];      /* tables.cpp:299-307, shift xyz + axis  */
extern float HPMC_midpoint_table[12][3];  /* tables.cpp:314-323                    */

/* The reference's edge table (tables.cpp:299-307): per edge the shift of its
 * first corner and its axis. */
void oracle_edge_table(float out[48])
{
    memcpy(out, HPMC_edge_table, sizeof(float) * 48);
}

int oracle_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------- */
/* init.cpp:72-149 */
static int tile_exponent(int cells)
{
    /* init.cpp:106-111: 1u << (GLsizei)ceilf(log2f(cells/2.0f)).  For
     * cells == 1 the exponent is -1 and the reference's shift is undefined;
     * the restatement clamps the exponent at 0 (one texel per tile). */
    int e = (int)ceilf(log2f((float)cells / 2.0f));
    return e < 0 ? 0 : e;
}

int oracle_layout(const int lattice[3], const int cells[3], oracle_layout_t* L)
{
    for (int i = 0; i < 3; i++) {
        if (lattice[i] < 2 || lattice[i] > 16384) return 0;      /* init.cpp:82-90 */
        if (lattice[i] <= cells[i]) return 0;                    /* init.cpp:98-103 */
        if (cells[i] < 1) return 0;  /* the reference takes log2f(0) here: undefined */
    }
    int tile_x = 1 << tile_exponent(cells[0]);
    int tile_y = 1 << tile_exponent(cells[1]);
    float aspect = (float)tile_x / (float)tile_y;                /* init.cpp:112-114 */
    float lx = ceilf(log2f(sqrtf((float)cells[2] / aspect)));    /* init.cpp:116-119 */
    if (lx < 0.0f) lx = 0.0f;
    int layout_x = 1 << (int)lx;
    int layout_y = (cells[2] + layout_x - 1) / layout_x;         /* init.cpp:120-121 */
    int wx = tile_x * layout_x, wy = tile_y * layout_y;
    int size_l2 = (int)ceilf(log2f((float)(wx > wy ? wx : wy))); /* init.cpp:123-127 */
    int size = 1 << size_l2;                                     /* init.cpp:128 */
    for (int i = 0; i < 3; i++) {
        L->lattice[i] = lattice[i];
        L->cells[i] = cells[i];
    }
    L->tile[0] = tile_x;
    L->tile[1] = tile_y;
    L->layout[0] = size / tile_x;                                /* init.cpp:129-130 */
    L->layout[1] = size / tile_y;
    L->size_l2 = size_l2;
    L->size = size;
    return 1;
}

/* ------------------------------------------------------------------------- */
/* constants.cpp:42-50: Bourke corner order -> HPMC bit (dx + 2dy + 4dz). */
int oracle_remap_code(int c)
{
    return (((c >> 0) & 1) << 0) | (((c >> 1) & 1) << 1) | (((c >> 4) & 1) << 2) |
           (((c >> 5) & 1) << 3) | (((c >> 3) & 1) << 4) | (((c >> 2) & 1) << 5) |
           (((c >> 7) & 1) << 6) | (((c >> 6) & 1) << 7);
}

void oracle_tables(uint8_t* count, uint8_t* edge_index, float* edge_decode,
                   float* edge_decode_normal)
{
    /* constants.cpp:217-252: binary-field normals per (code, triangle). The
     * scale multiplies by 0.5*|n| (a quirk of the reference, kept). */
    float edge_normals[256 * 6 * 4];
    memset(edge_normals, 0, sizeof edge_normals);
    for (int j = 0; j < 256; j++) {
        for (int i = 0; i < 6; i++) {
            const float* vp[3];
            for (int k = 0; k < 3; k++) {
                int idx = 3 * i + k;
                if (idx > 15) idx = 15;
                int ix = HPMC_triangle_table[j][idx];
                if (ix < 0) ix = 0;
                vp[k] = HPMC_midpoint_table[ix];
            }
            float u[3], v[3], n[3];
            for (int k = 0; k < 3; k++) {
                u[k] = vp[2][k] - vp[0][k];
                v[k] = vp[1][k] - vp[0][k];
            }
            n[0] = u[1] * v[2] - u[2] * v[1];
            n[1] = u[2] * v[0] - u[0] * v[2];
            n[2] = u[0] * v[1] - u[1] * v[0];
            float s = 0.5f * sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            int r = oracle_remap_code(j);
            for (int k = 0; k < 3; k++) {
                float tmp = s * n[k] + 0.5f;
                if (tmp < 0.f) tmp = 0.000001f;
                if (tmp >= 1.f) tmp = 0.999999f;
                edge_normals[4 * (6 * r + i) + k] = tmp;
            }
            edge_normals[4 * (6 * r + i) + 3] = 0.f;
        }
    }
    /* constants.cpp:255-264: edge decode, HPMC code order; -1 entries -> edge 0 */
    static float ed[256 * 16 * 4];
    uint8_t ei[256 * 16];
    for (int j = 0; j < 256; j++) {
        int r = oracle_remap_code(j);
        for (int i = 0; i < 16; i++) {
            int e = HPMC_triangle_table[j][i];
            if (e < 0) e = 0;
            ei[16 * r + i] = (uint8_t)e;
            for (int k = 0; k < 4; k++) ed[4 * 16 * r + 4 * i + k] = HPMC_edge_table[e][k];
        }
    }
    if (edge_index) memcpy(edge_index, ei, sizeof ei);
    if (edge_decode) memcpy(edge_decode, ed, sizeof ed);
    /* constants.cpp:266-273: entries 0..14 get the triangle normal added */
    if (edge_decode_normal) {
        memset(edge_decode_normal, 0, sizeof(float) * 256 * 16 * 4);
        for (int j = 0; j < 256; j++)
            for (int i = 0; i < 15; i++)
                for (int k = 0; k < 4; k++)
                    edge_decode_normal[4 * (16 * j + i) + k] =
                        ed[4 * (16 * j + i) + k] + edge_normals[4 * (6 * j + i / 3) + k];
    }
    /* constants.cpp:304-314: vertex count = entries before the first -1 */
    if (count) {
        for (int j = 0; j < 256; j++) {
            int c = 0;
            while (c < 16 && HPMC_triangle_table[j][c] != -1) c++;
            count[oracle_remap_code(j)] = (uint8_t)c;
        }
    }
}

/* ------------------------------------------------------------------------- */
static inline long clampl(long v, long lo, long hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* Functor fields in plain FP32 (this file is compiled with contraction off),
 * the operations in the same order as the device's, so that values agree bit
 * for bit (sin/cos of the twisted metaballs excepted). */
static float functor_value(const oracle_functor_t* F, float px, float py, float pz)
{
    switch (F->id) {
    case 1: {
        const float x = 2.0f * px - 1.0f, y = 2.0f * py - 1.0f, z = 2.0f * pz - 1.0f;
        return 1.0f - 16.0f * x * y * z - 4.0f * x * x - 4.0f * y * y - 4.0f * z * z;
    }
    case 2: {
        const int n = (int)F->p[0];
        float s = 0.0f;
        for (int i = 0; i < n; i++) {
            const float dx = px - F->p[1 + 4 * i], dy = py - F->p[2 + 4 * i], dz = pz - F->p[3 + 4 * i];
            const float r = F->p[4 + 4 * i];
            s = s + (r * r) / (dx * dx + dy * dy + dz * dz);
        }
        return s;
    }
    case 3: {
        float x = 2.0f * px - 1.0f, y = 2.0f * py - 1.0f, z = 2.0f * pz - 1.0f;
        const float twist = F->p[0];
        const float rot1 = twist * z, rot2 = 0.7f * twist * y;
        const float c1 = cosf(rot1), s1 = sinf(rot1), c2 = cosf(rot2), s2 = sinf(rot2);
        const float x1 = c1 * x + s1 * y, y1 = -s1 * x + c1 * y, z1 = z;
        const float x2 = c2 * x1 + s2 * z1, y2 = y1, z2 = -s2 * x1 + c2 * z1;
        x = 0.5f * x2 + 0.5f;
        y = 0.5f * y2 + 0.5f;
        z = 0.5f * z2 + 0.5f;
        float s = 0.0f;
        for (int i = 0; i < 8; i++) {
            const float dx = x - F->p[1 + 3 * i], dy = y - F->p[2 + 3 * i], dz = z - F->p[3 + 3 * i];
            s += 0.05f / (dx * dx + dy * dy + dz * dz);
        }
        return s;
    }
    case 4: {
        const int n = (int)F->p[0];
        float d = 3.0e38f;
        for (int i = 0; i < n; i++) {
            const float dx = px - F->p[1 + 4 * i], dy = py - F->p[2 + 4 * i], dz = pz - F->p[3 + 4 * i];
            d = fminf(d, sqrtf(dx * dx + dy * dy + dz * dz) - F->p[4 + 4 * i]);
        }
        return d;
    }
    case 5: {
        /* a caller-registered functor (hpmc_b200/apps/custom_functor.cu): the
         * torus (sqrt(x^2 + y^2) - R)^2 + z^2 - r^2 on [-1,1]^3, p = {R, r} */
        const float x = 2.0f * px - 1.0f, y = 2.0f * py - 1.0f, z = 2.0f * pz - 1.0f;
        const float d = sqrtf(x * x + y * y) - F->p[0];
        return d * d + z * z - F->p[1] * F->p[1];
    }
    default:
        return 0.0f;
    }
}

/* HPMC_fetchGrad of the cayley snippet (apps/cayley/cayley.cpp:85-93). */
static void functor_gradient(const oracle_functor_t* F, float px, float py, float pz, float g[3])
{
    if (F->id == 1) {
        const float x = 2.0f * px - 1.0f, y = 2.0f * py - 1.0f, z = 2.0f * pz - 1.0f;
        g[0] = -16.0f * y * z - 8.0f * x;
        g[1] = -16.0f * x * z - 8.0f * y;
        g[2] = -16.0f * x * y - 8.0f * z;
    } else if (F->id == 5) {
        const float x = 2.0f * px - 1.0f, y = 2.0f * py - 1.0f, z = 2.0f * pz - 1.0f;
        const float q = sqrtf(x * x + y * y);
        const float d = q - F->p[0];
        g[0] = 2.0f * d * x / q;
        g[1] = 2.0f * d * y / q;
        g[2] = 2.0f * z;
    } else {
        g[0] = g[1] = g[2] = 0.0f;
    }
}

static inline float texel_centre(long i, int n) { return ((float)i + 0.5f) / (float)n; }

/* GL_CLAMP + NEAREST (apps/texture3d/texture3d.cpp:135-139): clamp to edge.
 * uint8 fetch: U8 is float(b); UNORM8 is b/255 as a GL_ALPHA texture reads.
 * Functors are evaluated at the texel centre, unclamped (shadergen.cpp:270-279). */
static inline float sample_f(const void* field, int type, const oracle_layout_t* L,
                             size_t rp, size_t sp, long x, long y, long z)
{
    if (type == ORACLE_FUNCTOR)
        return functor_value((const oracle_functor_t*)field, texel_centre(x, L->lattice[0]),
                             texel_centre(y, L->lattice[1]), texel_centre(z, L->lattice[2]));
    x = clampl(x, 0, L->lattice[0] - 1);
    y = clampl(y, 0, L->lattice[1] - 1);
    z = clampl(z, 0, L->lattice[2] - 1);
    size_t off = (size_t)z * sp + (size_t)y * rp + (size_t)x;
    if (type == ORACLE_F32) return ((const float*)field)[off];
    if (type == ORACLE_F32X4) return ((const float*)field)[4 * off + 3]; /* texture3D(...).a */
    uint8_t b = ((const uint8_t*)field)[off];
    if (type == ORACLE_U8) return (float)b;
    return (float)b / 255.0f;
}

double oracle_sample(const void* field, int type, const oracle_layout_t* L, size_t rp,
                     size_t sp, long x, long y, long z)
{
    if (type == ORACLE_F64) {
        x = clampl(x, 0, L->lattice[0] - 1);
        y = clampl(y, 0, L->lattice[1] - 1);
        z = clampl(z, 0, L->lattice[2] - 1);
        return ((const double*)field)[(size_t)z * sp + (size_t)y * rp + (size_t)x];
    }
    return (double)sample_f(field, type, L, rp, sp, x, y, z);
}

/* shadergen.cpp:132-153: 3x3x2 fetch per base texel; per cell the bit
 * (dx + 2dy + 4dz) is set iff f < threshold (strict: f == iso -> 0, NaN -> 0). */
void oracle_codes(const void* field, int type, const oracle_layout_t* L, size_t rp, size_t sp,
                  float iso, int binary, uint8_t* codes)
{
    const float thr = binary ? 0.5f : iso; /* shadergen.cpp:99-101 */
    const int cx = L->cells[0], cy = L->cells[1], cz = L->cells[2];
#pragma omp parallel for schedule(static)
    for (int z = 0; z < cz; z++) {
        for (int y = 0; y < cy; y++) {
            for (int x = 0; x < cx; x++) {
                int code = 0;
                for (int b = 0; b < 8; b++) {
                    int dx = b & 1, dy = (b >> 1) & 1, dz = (b >> 2) & 1;
                    if (sample_f(field, type, L, rp, sp, x + dx, y + dy, z + dz) < thr)
                        code |= 1 << b;
                }
                codes[((size_t)z * cy + y) * cx + x] = (uint8_t)code;
            }
        }
    }
}

/* ------------------------------------------------------------------------- */
static inline uint64_t spread(uint64_t v)
{
    v &= 0xffffffffull;
    v = (v | (v << 16)) & 0x0000ffff0000ffffull;
    v = (v | (v << 8)) & 0x00ff00ff00ff00ffull;
    v = (v | (v << 4)) & 0x0f0f0f0f0f0f0f0full;
    v = (v | (v << 2)) & 0x3333333333333333ull;
    v = (v | (v << 1)) & 0x5555555555555555ull;
    return v;
}
static inline uint32_t compact(uint64_t v)
{
    v &= 0x5555555555555555ull;
    v = (v | (v >> 1)) & 0x3333333333333333ull;
    v = (v | (v >> 2)) & 0x0f0f0f0f0f0f0f0full;
    v = (v | (v >> 4)) & 0x00ff00ff00ff00ffull;
    v = (v | (v >> 8)) & 0x0000ffff0000ffffull;
    v = (v | (v >> 16)) & 0x00000000ffffffffull;
    return (uint32_t)v;
}

/* shadergen.cpp:103-104 (slice -> tile) and 148-153 (channel order r,g,b,a =
 * (0,0),(1,0),(0,1),(1,1)), recursively through the reduction's child order
 * (shadergen.cpp:215-218): key = Morton(X, Y) with X on the even bits. */
uint64_t oracle_cell_key(const oracle_layout_t* L, int x, int y, int z)
{
    uint64_t X = (uint64_t)2 * L->tile[0] * (uint64_t)(z % L->layout[0]) + (uint64_t)x;
    uint64_t Y = (uint64_t)2 * L->tile[1] * (uint64_t)(z / L->layout[0]) + (uint64_t)y;
    return spread(X) | (spread(Y) << 1);
}

int oracle_key_cell(const oracle_layout_t* L, uint64_t key, int* x, int* y, int* z)
{
    uint64_t X = compact(key), Y = compact(key >> 1);
    uint64_t wx = 2 * (uint64_t)L->tile[0], wy = 2 * (uint64_t)L->tile[1];
    uint64_t tu = X / wx, tv = Y / wy;
    if (tu >= (uint64_t)L->layout[0] || tv >= (uint64_t)L->layout[1]) return 0;
    long xx = (long)(X % wx), yy = (long)(Y % wy), zz = (long)(tv * L->layout[0] + tu);
    if (xx >= L->cells[0] || yy >= L->cells[1] || zz >= L->cells[2]) return 0;
    *x = (int)xx;
    *y = (int)yy;
    *z = (int)zz;
    return 1;
}

uint64_t oracle_level_entries(const oracle_layout_t* L, int j)
{
    int e = L->size_l2 + 1 - j;
    return e <= 0 ? 1 : (uint64_t)1 << (2 * e);
}

/* buildpass.cpp:62-159 with shadergen.cpp:163 (base: count per cell, masked),
 * shadergen.cpp:174-225 (each level sums the four child channels). */
uint64_t oracle_pyramid(const oracle_layout_t* L, const uint8_t* codes,
                        const uint8_t* count_table, uint32_t** levels)
{
    const int cx = L->cells[0], cy = L->cells[1], cz = L->cells[2];
    uint64_t n0 = oracle_level_entries(L, 0);
    memset(levels[0], 0, sizeof(uint32_t) * n0);
#pragma omp parallel for schedule(static)
    for (int z = 0; z < cz; z++)
        for (int y = 0; y < cy; y++)
            for (int x = 0; x < cx; x++)
                levels[0][oracle_cell_key(L, x, y, z)] =
                    count_table[codes[((size_t)z * cy + y) * cx + x]];
    for (int j = 1; j <= L->size_l2 + 1; j++) {
        uint64_t n = oracle_level_entries(L, j);
        const uint32_t* src = levels[j - 1];
        uint32_t* dst = levels[j];
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < (long long)n; e++)
            dst[e] = src[4 * e] + src[4 * e + 1] + src[4 * e + 2] + src[4 * e + 3];
    }
    return levels[L->size_l2 + 1][0];
}

/* shadergen.cpp:103-167: base texel (i,j) channel c holds cell
 * X = 2i + (c&1), Y = 2j + (c>>1); value mask*(count + (code+0.5)/256);
 * texels of slices >= cells_z hold (0, 0, 0.4, 0). */
void oracle_level0_texture(const oracle_layout_t* L, const uint8_t* codes,
                           const uint8_t* count_table, float* tex)
{
    const int size = L->size, cx = L->cells[0], cy = L->cells[1], cz = L->cells[2];
    for (int j = 0; j < size; j++) {
        for (int i = 0; i < size; i++) {
            float* t = tex + 4 * ((size_t)j * size + i);
            int tu = i / L->tile[0], tv = j / L->tile[1];
            int slice = tu + L->layout[0] * tv;
            if (slice >= cz) {
                t[0] = 0.f; t[1] = 0.f; t[2] = 0.4f; t[3] = 0.f;
                continue;
            }
            for (int c = 0; c < 4; c++) {
                int x = 2 * (i % L->tile[0]) + (c & 1);
                int y = 2 * (j % L->tile[1]) + (c >> 1);
                if (x < cx && y < cy) {
                    int code = codes[((size_t)slice * cy + y) * cx + x];
                    float frac = ((float)code + 0.5f) * (1.0f / 256.0f);
                    t[c] = (float)count_table[code] + frac;
                } else {
                    t[c] = 0.f;
                }
            }
        }
    }
}

/* shadergen.cpp:445-495 (GL3+ path): descend from the top texel; at each
 * level take the first child whose running sum exceeds the key, subtracting
 * the skipped children. */
void oracle_traverse(const oracle_layout_t* L, const uint8_t* codes, uint32_t* const* levels,
                     const uint8_t* edge_index, uint64_t v0, uint64_t v1, int32_t* cell_xyz,
                     uint8_t* code_out, uint8_t* k_out, uint8_t* edge_out)
{
    const int l2 = L->size_l2;
#pragma omp parallel for schedule(static)
    for (long long vv = (long long)v0; vv < (long long)v1; vv++) {
        uint64_t key = (uint64_t)vv;
        uint64_t node = 0;
        for (int i = l2; i >= 0; i--) {
            const uint32_t* s = levels[i] + 4 * node;
            int c;
            if (s[0] <= key) {
                key -= s[0];
                if (s[1] <= key) {
                    key -= s[1];
                    if (s[2] <= key) {
                        key -= s[2];
                        c = 3;
                    } else {
                        c = 2;
                    }
                } else {
                    c = 1;
                }
            } else {
                c = 0;
            }
            node = 4 * node + (uint64_t)c;
        }
        int x = 0, y = 0, z = 0;
        oracle_key_cell(L, node, &x, &y, &z);
        int code = codes[((size_t)z * L->cells[1] + y) * L->cells[0] + x];
        size_t o = (size_t)(vv - (long long)v0);
        cell_xyz[3 * o + 0] = x;
        cell_xyz[3 * o + 1] = y;
        cell_xyz[3 * o + 2] = z;
        if (code_out) code_out[o] = (uint8_t)code;
        if (k_out) k_out[o] = (uint8_t)key;
        if (edge_out) edge_out[o] = edge_index[16 * code + key];
    }
}

/* shadergen.cpp:512-563.  Edge e: a = cell + shift, b = a + e_axis.
 *  forward:  t = (f(a)-iso)/(f(a)-f(b)); n_i = iso - lerp(f(a+e_i), f(b+e_i), t)
 *  central:  n_i = -lerp(g_i(a), g_i(b), t), g_i(q) = (f(q+e_i) - f(q-e_i))/2
 *  binary:   p = midpoint, n = 2*fract(edge_decode_normal.xyz) - 1
 *  p = (a + t e_axis) * extent / cells;  n *= extent / cells (reference scaling). */
void oracle_geometry(const void* field, int type, const oracle_layout_t* L, size_t rp, size_t sp,
                     float iso, int binary, int normal_mode, const float extent[3],
                     const float* edge_decode_normal, uint64_t n, const int32_t* cell_xyz,
                     const uint8_t* code, const uint8_t* k, const uint8_t* edge, double* t_out,
                     double* pos, double* nrm)
{
    const double thr = binary ? 0.5 : (double)iso;
    double scale[3];
    for (int i = 0; i < 3; i++) scale[i] = (double)extent[i] / (double)L->cells[i];
#pragma omp parallel for schedule(static)
    for (long long v = 0; v < (long long)n; v++) {
        const float* et = HPMC_edge_table[edge[v]];
        long a[3], b[3];
        int axis = (int)et[3];
        for (int i = 0; i < 3; i++) {
            a[i] = cell_xyz[3 * v + i] + (long)et[i];
            b[i] = a[i] + (i == axis ? 1 : 0);
        }
        double t, nn[3];
        if (binary) {
            t = 0.5;
            const float* en = edge_decode_normal + 4 * (16 * code[v] + k[v]);
            for (int i = 0; i < 3; i++) {
                float fr = en[i] - floorf(en[i]);
                nn[i] = 2.0 * (double)fr - 1.0;
            }
        } else if (normal_mode >= ORACLE_NORMALS_GRADIENT && type != ORACLE_FUNCTOR) {
            /* HPMC_sampleGrad of a texture (shadergen.cpp:260-266): the RGBA
             * sample at each edge end, value in .a, gradient in .rgb (zero for
             * a single-channel field) */
            double va = oracle_sample(field, type, L, rp, sp, a[0], a[1], a[2]);
            double vb = oracle_sample(field, type, L, rp, sp, b[0], b[1], b[2]);
            double ga[3] = {0.0, 0.0, 0.0}, gb[3] = {0.0, 0.0, 0.0};
            if (type == ORACLE_F32X4) {
                const float* f4 = (const float*)field;
                const size_t oa = 4 * ((size_t)clampl(a[2], 0, L->lattice[2] - 1) * sp +
                                       (size_t)clampl(a[1], 0, L->lattice[1] - 1) * rp +
                                       (size_t)clampl(a[0], 0, L->lattice[0] - 1));
                const size_t ob = 4 * ((size_t)clampl(b[2], 0, L->lattice[2] - 1) * sp +
                                       (size_t)clampl(b[1], 0, L->lattice[1] - 1) * rp +
                                       (size_t)clampl(b[0], 0, L->lattice[0] - 1));
                for (int i = 0; i < 3; i++) {
                    ga[i] = f4[oa + i];
                    gb[i] = f4[ob + i];
                }
            }
            t = (va - thr) / (va - vb);
            for (int i = 0; i < 3; i++) {
                const double g = (1.0 - t) * ga[i] + t * gb[i];
                nn[i] = normal_mode == ORACLE_NORMALS_GRADIENT ? thr - g : -g;
            }
        } else if (normal_mode >= ORACLE_NORMALS_GRADIENT && type == ORACLE_FUNCTOR) {
            const oracle_functor_t* F = (const oracle_functor_t*)field;
            const float pa[3] = {texel_centre(a[0], L->lattice[0]), texel_centre(a[1], L->lattice[1]),
                                 texel_centre(a[2], L->lattice[2])};
            const float pb[3] = {texel_centre(b[0], L->lattice[0]), texel_centre(b[1], L->lattice[1]),
                                 texel_centre(b[2], L->lattice[2])};
            const double va = functor_value(F, pa[0], pa[1], pa[2]);
            const double vb = functor_value(F, pb[0], pb[1], pb[2]);
            float ga[3], gb[3];
            functor_gradient(F, pa[0], pa[1], pa[2], ga);
            functor_gradient(F, pb[0], pb[1], pb[2], gb);
            t = (va - thr) / (va - vb);
            for (int i = 0; i < 3; i++) {
                const double g = (1.0 - t) * ga[i] + t * gb[i];
                nn[i] = normal_mode == ORACLE_NORMALS_GRADIENT ? thr - g : -g;
            }
        } else {
            double va = oracle_sample(field, type, L, rp, sp, a[0], a[1], a[2]);
            double vb = oracle_sample(field, type, L, rp, sp, b[0], b[1], b[2]);
            t = (va - thr) / (va - vb);
            for (int i = 0; i < 3; i++) {
                long da[3] = {a[0], a[1], a[2]}, db[3] = {b[0], b[1], b[2]};
                da[i] += 1;
                db[i] += 1;
                double fa = oracle_sample(field, type, L, rp, sp, da[0], da[1], da[2]);
                double fb = oracle_sample(field, type, L, rp, sp, db[0], db[1], db[2]);
                if (normal_mode == ORACLE_NORMALS_FORWARD) {
                    nn[i] = (1.0 - t) * (thr - fa) + t * (thr - fb);
                } else {
                    long ma[3] = {a[0], a[1], a[2]}, mb[3] = {b[0], b[1], b[2]};
                    ma[i] -= 1;
                    mb[i] -= 1;
                    double ga = 0.5 * (fa - oracle_sample(field, type, L, rp, sp, ma[0], ma[1], ma[2]));
                    double gb = 0.5 * (fb - oracle_sample(field, type, L, rp, sp, mb[0], mb[1], mb[2]));
                    nn[i] = -((1.0 - t) * ga + t * gb);
                }
            }
        }
        if (t_out) t_out[v] = t;
        for (int i = 0; i < 3; i++) {
            double pl = (double)a[i] + (i == axis ? t : 0.0);
            pos[3 * v + i] = pl * scale[i];
            nrm[3 * v + i] = nn[i] * scale[i];
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Adjoint of the geometry above (no reference counterpart: the reference has
 * no gradients).  With c = iso, t = (f_a - c)/(f_a - f_b):
 *   dt/df_a = (c - f_b)/(f_a - f_b)^2,  dt/df_b = (f_a - c)/(f_a - f_b)^2,
 *   p_axis = (a_axis + t) s_axis,
 *   forward: n_i = s_i((1-t)(c - f(a+e_i)) + t(c - f(b+e_i))),
 *   central: n_i = -s_i((1-t) g_i(a) + t g_i(b)), g_i(q) = (f(q+e_i) - f(q-e_i))/2. */
static double* g_adj_abs; /* optional sum of |terms| per sample (error scale for FP32 checks) */

static inline void scatter_add(double* g, const oracle_layout_t* L, long x, long y, long z, double v)
{
    x = clampl(x, 0, L->lattice[0] - 1);
    y = clampl(y, 0, L->lattice[1] - 1);
    z = clampl(z, 0, L->lattice[2] - 1);
    const size_t o = ((size_t)z * (size_t)L->lattice[1] + (size_t)y) * (size_t)L->lattice[0] + (size_t)x;
    g[o] += v;
    if (g_adj_abs) g_adj_abs[o] += fabs(v);
}

void oracle_adjoint(const void* field, int type, const oracle_layout_t* L, size_t rp, size_t sp,
                    float iso, int normal_mode, const float extent[3], uint64_t n,
                    const int32_t* cell_xyz, const uint8_t* edge, const double* dpos,
                    const double* dnrm, double* dfield, double* dfield_abs)
{
    g_adj_abs = dfield_abs;
    const double c = (double)iso;
    double scale[3];
    for (int i = 0; i < 3; i++) scale[i] = (double)extent[i] / (double)L->cells[i];
    for (uint64_t v = 0; v < n; v++) {
        const float* et = HPMC_edge_table[edge[v]];
        long a[3], b[3];
        const int axis = (int)et[3];
        for (int i = 0; i < 3; i++) {
            a[i] = cell_xyz[3 * v + i] + (long)et[i];
            b[i] = a[i] + (i == axis ? 1 : 0);
        }
        const double va = oracle_sample(field, type, L, rp, sp, a[0], a[1], a[2]);
        const double vb = oracle_sample(field, type, L, rp, sp, b[0], b[1], b[2]);
        const double den = va - vb;
        const double t = (va - c) / den;
        double dLdt = dpos[3 * v + axis] * scale[axis];
        for (int i = 0; i < 3; i++) {
            const double dn = dnrm[3 * v + i] * scale[i];
            const long e[3] = {i == 0, i == 1, i == 2};
            const double fa = oracle_sample(field, type, L, rp, sp, a[0] + e[0], a[1] + e[1], a[2] + e[2]);
            const double fb = oracle_sample(field, type, L, rp, sp, b[0] + e[0], b[1] + e[1], b[2] + e[2]);
            if (normal_mode == ORACLE_NORMALS_FORWARD) {
                dLdt += dn * (fa - fb);
                scatter_add(dfield, L, a[0] + e[0], a[1] + e[1], a[2] + e[2], -(1.0 - t) * dn);
                scatter_add(dfield, L, b[0] + e[0], b[1] + e[1], b[2] + e[2], -t * dn);
            } else {
                const double fam = oracle_sample(field, type, L, rp, sp, a[0] - e[0], a[1] - e[1], a[2] - e[2]);
                const double fbm = oracle_sample(field, type, L, rp, sp, b[0] - e[0], b[1] - e[1], b[2] - e[2]);
                dLdt += dn * (0.5 * (fa - fam) - 0.5 * (fb - fbm));
                scatter_add(dfield, L, a[0] + e[0], a[1] + e[1], a[2] + e[2], -0.5 * (1.0 - t) * dn);
                scatter_add(dfield, L, a[0] - e[0], a[1] - e[1], a[2] - e[2], 0.5 * (1.0 - t) * dn);
                scatter_add(dfield, L, b[0] + e[0], b[1] + e[1], b[2] + e[2], -0.5 * t * dn);
                scatter_add(dfield, L, b[0] - e[0], b[1] - e[1], b[2] - e[2], 0.5 * t * dn);
            }
        }
        scatter_add(dfield, L, a[0], a[1], a[2], dLdt * (c - vb) / (den * den));
        scatter_add(dfield, L, b[0], b[1], b[2], dLdt * (va - c) / (den * den));
    }
    g_adj_abs = NULL;
}

/* ------------------------------------------------------------------------- */
uint64_t oracle_extract(const void* field, int type, const int lattice[3], const int cells[3],
                        float iso, int binary, int normal_mode, const float extent[3], float* pos,
                        float* nrm, uint64_t capacity, int threads)
{
#ifdef _OPENMP
    int saved = omp_get_max_threads();
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    oracle_layout_t L;
    uint64_t total = 0;
    if (!oracle_layout(lattice, cells, &L)) goto done;
    {
        uint8_t count[256], eidx[256 * 16];
        static float edn[256 * 16 * 4];
        oracle_tables(count, eidx, NULL, edn);
        size_t ncell = (size_t)cells[0] * cells[1] * cells[2];
        size_t rp = (size_t)lattice[0], sp = (size_t)lattice[0] * lattice[1];
        uint8_t* codes = (uint8_t*)malloc(ncell);
        oracle_codes(field, type, &L, rp, sp, iso, binary, codes);
        uint32_t* levels[40];
        for (int j = 0; j <= L.size_l2 + 1; j++)
            levels[j] = (uint32_t*)malloc(sizeof(uint32_t) * oracle_level_entries(&L, j));
        total = oracle_pyramid(&L, codes, count, levels);
        if (pos && nrm && total <= capacity && total > 0) {
            int32_t* cxyz = (int32_t*)malloc(sizeof(int32_t) * 3 * total);
            uint8_t* cc = (uint8_t*)malloc(total);
            uint8_t* kk = (uint8_t*)malloc(total);
            uint8_t* ee = (uint8_t*)malloc(total);
            double* p64 = (double*)malloc(sizeof(double) * 3 * total);
            double* n64 = (double*)malloc(sizeof(double) * 3 * total);
            oracle_traverse(&L, codes, levels, eidx, 0, total, cxyz, cc, kk, ee);
            oracle_geometry(field, type, &L, rp, sp, iso, binary, normal_mode, extent, edn, total,
                            cxyz, cc, kk, ee, NULL, p64, n64);
#pragma omp parallel for schedule(static)
            for (long long i = 0; i < (long long)(3 * total); i++) {
                pos[i] = (float)p64[i];
                nrm[i] = (float)n64[i];
            }
            free(cxyz); free(cc); free(kk); free(ee); free(p64); free(n64);
        }
        for (int j = 0; j <= L.size_l2 + 1; j++) free(levels[j]);
        free(codes);
    }
done:
#ifdef _OPENMP
    omp_set_num_threads(saved);
#endif
    return total;
}
