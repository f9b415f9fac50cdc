/*
 * ref_glue.cpp -- C entry points into the REFERENCE's own code, for tests.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle).  oracle/Makefile compiles this file
 * together with three unmodified reference sources, read in place from the
 * HPMC source tree:
 *   hpmc/src/init.cpp       HPMCdetermineLayout  (layout / tiling, init.cpp:72-149)
 *   hpmc/src/tables.cpp     HPMC_triangle_table, HPMC_edge_table,
 *                           HPMC_midpoint_table  (tables.cpp:38-323)
 *   hpmc/src/shadergen.cpp  HPMCgenerate*        (GLSL text, shadergen.cpp:45-574)
 * against oracle/shim/GL/glew.h (GL scalar typedefs only).  None of these
 * three files calls into GL; the only link dependencies they have are the
 * three HPMC-internal set-up functions that HPMCsetup (init.cpp:48-69)
 * names, stubbed below because HPMCsetup is never called here.
 *
 * The result, oracle/_ref/libhpmc_ref.so, lets the tests:
 *   - check the oracle's layout restatement against the real HPMCdetermineLayout,
 *   - read the real case tables,
 *   - obtain the exact GLSL text the reference generates for a configuration,
 *     which tests/glsl_exec compiles as C++ (oracle/glsl_emu.hpp) and runs on
 *     the CPU as a second, reference-derived oracle.
 */
#include <cstring>
#include <cstdlib>
#include <string>
#include <hpmc.h>
#include <hpmc_internal.h>

// --- link stubs for HPMC-internal GL set-up (never reached: HPMCsetup is not called) ---
bool HPMCsetupTexAndFBOs(struct HPMCHistoPyramid*) { return true; }
bool HPMCfreeHPBuildShaders(struct HPMCHistoPyramid*) { return true; }
bool HPMCbuildHPBuildShaders(struct HPMCHistoPyramid*) { return true; }

namespace {

struct RefState {
    HPMCConstants c;
    HPMCHistoPyramid h;
};

// Fill the handle the way HPMCcreateHistoPyramid + HPMCsetLatticeSize +
// HPMCsetGridSize + HPMCsetGridExtent leave it (hpiface.cpp:45-161); the GL
// object names stay zero.
void init_state(RefState& s, const int lattice[3], const int cells[3],
                const float extent[3], int binary, int gradient, int gl_target)
{
    s.c.m_vertex_count_tex = 0;
    s.c.m_edge_decode_tex = 0;
    s.c.m_edge_decode_normal_tex = 0;
    s.c.m_enumerate_vbo = 0;
    s.c.m_enumerate_vbo_n = 3 * 1000;
    s.c.m_gpgpu_quad_vbo = 0;
    s.c.m_target = static_cast<HPMCTarget>(gl_target);

    HPMCHistoPyramid& h = s.h;
    h.m_tainted = true;
    h.m_broken = false;
    h.m_constants = &s.c;
    h.m_threshold = 0.f;
    h.m_tiling.m_tile_size[0] = h.m_tiling.m_tile_size[1] = 0;
    h.m_tiling.m_layout[0] = h.m_tiling.m_layout[1] = 0;
    h.m_histopyramid.m_size = 0;
    h.m_histopyramid.m_size_l2 = 0;
    h.m_histopyramid.m_tex = 0;
    h.m_histopyramid.m_top_pbo = 0;
    h.m_histopyramid.m_top_count = 0;
    h.m_histopyramid.m_top_count_updated = 0;
    for (int i = 0; i < 3; i++) {
        h.m_field.m_size[i] = lattice[i];
        h.m_field.m_cells[i] = cells[i];
        h.m_field.m_extent[i] = extent[i];
    }
    h.m_field.m_binary = binary != 0;
    h.m_fetch.m_mode = HPMC_VOLUME_LAYOUT_TEXTURE_3D;
    h.m_fetch.m_shader_source = "";
    h.m_fetch.m_tex = 0;
    h.m_fetch.m_gradient = gradient != 0;
}

}  // namespace

extern "C" {

/* Runs the reference's HPMCdetermineLayout.  out = {tile_x, tile_y,
 * layout_x, layout_y, size_l2, size}.  Returns 1 when the reference accepts
 * the sizes, 0 when it rejects them. */
int hpmc_ref_layout(int fx, int fy, int fz, int cx, int cy, int cz, int out[6])
{
    RefState s;
    const int lat[3] = {fx, fy, fz};
    const int cel[3] = {cx, cy, cz};
    const float ext[3] = {1.f, 1.f, 1.f};
    init_state(s, lat, cel, ext, 0, 0, HPMC_TARGET_GL43_GLSL430);
    if (!HPMCdetermineLayout(&s.h)) return 0;
    out[0] = s.h.m_tiling.m_tile_size[0];
    out[1] = s.h.m_tiling.m_tile_size[1];
    out[2] = s.h.m_tiling.m_layout[0];
    out[3] = s.h.m_tiling.m_layout[1];
    out[4] = s.h.m_histopyramid.m_size_l2;
    out[5] = s.h.m_histopyramid.m_size;
    return 1;
}

const int* hpmc_ref_triangle_table(void) { return &HPMC_triangle_table[0][0]; }
const float* hpmc_ref_edge_table(void) { return &HPMC_edge_table[0][0]; }
const float* hpmc_ref_midpoint_table(void) { return &HPMC_midpoint_table[0][0]; }

/* The GLSL text the reference generates for one configuration.
 * which: 0 defines, 1 scalar-field fetch (Texture3D mode), 2 base-level
 * shader, 3 first reduction (filter "floor"), 4 upper reduction, 5 extract
 * vertex function.  Returns a malloc'd string (free with hpmc_ref_free), or
 * NULL if the layout is rejected. */
char* hpmc_ref_glsl(int which, const int lattice[3], const int cells[3],
                    const float extent[3], int binary, int gradient, int gl_target)
{
    RefState s;
    init_state(s, lattice, cells, extent, binary, gradient, gl_target);
    if (!HPMCdetermineLayout(&s.h)) return nullptr;
    std::string src;
    switch (which) {
        case 0: src = HPMCgenerateDefines(&s.h); break;
        case 1: src = HPMCgenerateScalarFieldFetch(&s.h); break;
        case 2: src = HPMCgenerateBaselevelShader(&s.h); break;
        case 3: src = HPMCgenerateReductionShader(&s.h, "floor"); break;
        case 4: src = HPMCgenerateReductionShader(&s.h, ""); break;
        case 5: src = HPMCgenerateExtractVertexFunction(&s.h); break;
        default: return nullptr;
    }
    return strdup(src.c_str());
}

/* The same for the custom-fetch mode (HPMCsetFieldCustom, hpiface.cpp:187-200):
 * `source` is the application's GLSL snippet defining HPMC_fetch (and, with
 * gradient, HPMC_fetchGrad), spliced in by HPMCgenerateScalarFieldFetch
 * (shadergen.cpp:270-286). */
char* hpmc_ref_glsl_custom(int which, const int lattice[3], const int cells[3], const float extent[3],
                           int binary, int gradient, int gl_target, const char* source)
{
    RefState s;
    init_state(s, lattice, cells, extent, binary, gradient, gl_target);
    s.h.m_fetch.m_mode = HPMC_VOLUME_LAYOUT_CUSTOM;
    s.h.m_fetch.m_shader_source = source ? source : "";
    if (!HPMCdetermineLayout(&s.h)) return nullptr;
    std::string src;
    switch (which) {
        case 0: src = HPMCgenerateDefines(&s.h); break;
        case 1: src = HPMCgenerateScalarFieldFetch(&s.h); break;
        case 2: src = HPMCgenerateBaselevelShader(&s.h); break;
        case 3: src = HPMCgenerateReductionShader(&s.h, "floor"); break;
        case 4: src = HPMCgenerateReductionShader(&s.h, ""); break;
        case 5: src = HPMCgenerateExtractVertexFunction(&s.h); break;
        default: return nullptr;
    }
    return strdup(src.c_str());
}

void hpmc_ref_free(char* p) { free(p); }

}  // extern "C"
