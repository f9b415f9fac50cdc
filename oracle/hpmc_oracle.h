/*
 * hpmc_oracle.h -- CPU restatement of HPMC's HistoPyramid marching cubes.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA product
 * (hpmc_b200/), never part of it: only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline / reference legs load it.  Each function cites the
 * reference file:line it restates (paths relative to the HPMC source tree).
 *
 * Parity pin: the layout is checked against the reference's own
 * HPMCdetermineLayout and the tables are the reference's own tables.cpp
 * arrays (both compiled from the HPMC sources into oracle/_ref/); the
 * classification / reduction / traversal / geometry arithmetic is checked
 * against the reference's generated GLSL compiled as C++
 * (oracle/glsl_emu.hpp, tests/test_glsl_pin.py).
 *
 * Integer topology (codes, counts, every pyramid level, vertex order) is
 * exact (uint32/uint64; the reference's RGBA32F pyramid is exact only below
 * 2^24).  Geometry is FP64.
 */
#ifndef HPMC_ORACLE_H
#define HPMC_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_F32 = 0, ORACLE_U8 = 1, ORACLE_UNORM8 = 2, ORACLE_F64 = 3 /* geometry and adjoint only */,
       ORACLE_FUNCTOR = 4 /* `field` points to an oracle_functor_t */,
       ORACLE_F32X4 = 5 /* float4 samples (gradient x, y, z, value): a GL RGBA float texture whose
                           alpha is the field (shadergen.cpp:260-266); pitches in float4s */ };

/* A field functor: the custom fetch snippet of HPMCsetFieldCustom
 * (hpiface.cpp:187-200, shadergen.cpp:270-286) evaluated at normalised texel
 * centres ((i + 0.5) / n per axis, no clamping).  Ids: 1 cayley
 * (apps/cayley/cayley.cpp:75-94), 2 metaballs {n, (cx,cy,cz,r) x n},
 * 3 twisted metaballs {twist, (cx,cy,cz) x 8} (apps/metaballs/metaballs.cpp:
 * 72-94), 4 union of spheres (signed distance) {n, (cx,cy,cz,r) x n},
 * 5 torus {R, r}, with gradient (the caller-registered functor of the
 * custom-functor example app). */
typedef struct oracle_functor_t {
    int id;
    int count;
    float p[136];
} oracle_functor_t;
/* Normals.  The GRADIENT modes use HPMC_fetchGrad (shadergen.cpp:260-266,
 * 539-551): a functor's analytic gradient, the .xyz of an ORACLE_F32X4
 * field, or zero for a single-channel field (a GL alpha texture reads
 * rgb = 0); t from the values at the edge ends; n = iso - lerp(grad a,
 * grad b, t) (the reference) or -lerp(grad a, grad b, t). */
enum { ORACLE_NORMALS_FORWARD = 0, ORACLE_NORMALS_CENTRAL = 1, ORACLE_NORMALS_GRADIENT = 2,
       ORACLE_NORMALS_GRADIENT_CENTRAL = 3 };

typedef struct {
    int lattice[3];   /* samples per axis (m_field.m_size) */
    int cells[3];     /* MC cells per axis (m_field.m_cells) */
    int tile[2];      /* base-level texels per tile (m_tiling.m_tile_size) */
    int layout[2];    /* tiles per axis (m_tiling.m_layout) */
    int size_l2;      /* log2 of the pyramid base size */
    int size;         /* pyramid base size in texels (2x2 cells each) */
} oracle_layout_t;

/* init.cpp:72-149.  Returns 1 and fills *L, or 0 if the sizes are rejected. */
int oracle_layout(const int lattice[3], const int cells[3], oracle_layout_t* L);

/* constants.cpp:42-50 */
int oracle_remap_code(int bourke_index);

/* constants.cpp:217-314 over the tables of tables.cpp:38-323.
 *   count[256]                 vertices per HPMC code
 *   edge_index[256*16]         MC edge (0..11) of vertex k of code c (0 past count)
 *   edge_decode[256*16*4]      (shift x,y,z, axis) as float, HPMC layout
 *   edge_decode_normal[256*16*4]  edge_decode + binary-mode normal in the fraction
 * Any output pointer may be NULL. */
void oracle_tables(uint8_t* count, uint8_t* edge_index, float* edge_decode,
                   float* edge_decode_normal);

/* Scalar sample f(x,y,z) with clamp-to-edge addressing (GL_CLAMP + NEAREST,
 * apps/texture3d/texture3d.cpp:135-139). */
double oracle_sample(const void* field, int type, const oracle_layout_t* L,
                     size_t row_pitch, size_t slice_pitch, long x, long y, long z);

/* shadergen.cpp:86-171: MC code of every cell, bit (dx + 2dy + 4dz) set iff
 * f < iso (strict).  codes is [cells_z][cells_y][cells_x].  Pitches are in
 * elements.  binary != 0 forces iso = 0.5 (shadergen.cpp:99-101). */
void oracle_codes(const void* field, int type, const oracle_layout_t* L,
                  size_t row_pitch, size_t slice_pitch, float iso, int binary,
                  uint8_t* codes);

/* Virtual 2-D cell coordinates of cell (x,y,z) (shadergen.cpp:103-104,
 * 497-503) and its Morton key (X in even bits, shadergen.cpp:148-153). */
uint64_t oracle_cell_key(const oracle_layout_t* L, int x, int y, int z);
/* Inverse: returns 1 and the cell for a key that maps to a real cell, else 0. */
int oracle_key_cell(const oracle_layout_t* L, uint64_t key, int* x, int* y, int* z);

/* Number of entries of compact level j (= 4^(size_l2+1-j), at least 1). */
uint64_t oracle_level_entries(const oracle_layout_t* L, int j);

/* Compact pyramid: level j entry e = number of vertices in the Morton key
 * range [e*4^j, (e+1)*4^j).  Level j of this array equals channel-flattened
 * level j of the reference's HistoPyramid texture (buildpass.cpp:42-178,
 * shadergen.cpp:174-225).  levels[j] must hold oracle_level_entries(L,j)
 * uint32 for j = 0..size_l2+1.  Returns the total vertex count
 * (hpiface.cpp:323-327, integer). */
uint64_t oracle_pyramid(const oracle_layout_t* L, const uint8_t* codes, const uint8_t* count_table,
                        uint32_t** levels);

/* Reference base-level texel value (shadergen.cpp:163-167) for every texel:
 * tex is size*size*4 floats, row-major over (j, i), channel fastest. */
void oracle_level0_texture(const oracle_layout_t* L, const uint8_t* codes,
                           const uint8_t* count_table, float* tex);

/* Traversal descent (shadergen.cpp:445-495) for vertices [v0, v1): writes the
 * cell (x,y,z), its code, the vertex index within the cell k, and the MC edge.
 * levels as filled by oracle_pyramid. */
void oracle_traverse(const oracle_layout_t* L, const uint8_t* codes,
                     uint32_t* const* levels, const uint8_t* edge_index,
                     uint64_t v0, uint64_t v1, int32_t* cell_xyz, uint8_t* code_out,
                     uint8_t* k_out, uint8_t* edge_out);

/* FP64 geometry of vertices given their cell and edge (shadergen.cpp:497-563):
 * t, position (lattice index * extent / cells) and normal.
 * normal_mode: forward differences (reference default, shadergen.cpp:528-537,
 * 550-551) or central differences.  binary != 0: midpoint position and
 * table normal (shadergen.cpp:507-510, 521-522, edge_decode_normal). */
void oracle_geometry(const void* field, int type, const oracle_layout_t* L,
                     size_t row_pitch, size_t slice_pitch, float iso, int binary,
                     int normal_mode, const float extent[3], const float* edge_decode_normal,
                     uint64_t n, const int32_t* cell_xyz, const uint8_t* code,
                     const uint8_t* k, const uint8_t* edge, double* t_out, double* pos,
                     double* nrm);

/* Whole extraction (classify + pyramid + count + traversal + geometry), the
 * CPU baseline.  Allocates internally; returns the vertex count and, if
 * pos/nrm are non-NULL and capacity suffices, FP32 positions/normals (xyz,
 * 3 floats per vertex).  threads <= 0 uses all OpenMP threads. */
/* Adjoint of oracle_geometry for continuous fields, in FP64: accumulates
 * dL/df = sum_v dL/dp_v . dp_v/df + dL/dn_v . dn_v/df into dfield (dense,
 * lattice shape, x fastest).  dpos/dnrm: 3 doubles per vertex.  A clamped
 * fetch passes its gradient to the sample it read.  dfield_abs (may be NULL)
 * accumulates the absolute values of the same terms. */
void oracle_adjoint(const void* field, int type, const oracle_layout_t* L, size_t rp, size_t sp,
                    float iso, int normal_mode, const float extent[3], uint64_t n,
                    const int32_t* cell_xyz, const uint8_t* edge, const double* dpos,
                    const double* dnrm, double* dfield, double* dfield_abs);

uint64_t oracle_extract(const void* field, int type, const int lattice[3], const int cells[3],
                        float iso, int binary, int normal_mode, const float extent[3],
                        float* pos, float* nrm, uint64_t capacity, int threads);

void oracle_edge_table(float out[48]);
int oracle_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
