// hpmc_api.cu -- host runtime and C ABI (include/hpmc.h).
//
// Mirrors the reference's handle model (hpmc/include/hpmc_internal.h:67-211):
// constants, a HistoPyramid per volume configuration with lazy set-up on a
// "tainted" flag and a sticky "broken" flag, and traversal handles.  GL
// objects become device allocations; the pass driver of buildpass.cpp:42-178
// becomes two kernel launches (classify, reduce) on the handle's stream and
// the draw loop of triface.cpp:423-428 becomes one persistent traversal launch.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>

#include "hpmc.h"
#include "hpmc_device.cuh"
#include "hpmc_fetch.cuh"
#include "hpmc_geometry.cuh"
#include "hpmc_host.h"
#include "hpmc_kernels.h"

using hpmc::Ctrl;
using hpmc::Volume;

namespace {

using hpmc::host::kMagicConstants;
constexpr uint32_t kMagicPyramid = 0x48505931u;
constexpr uint32_t kMagicTraversal = 0x48505431u;

struct FieldDesc {
    const void* ptr = nullptr;
    int type = HPMC_SCALAR_F32;
    int size[3] = {0, 0, 0};
    size_t row_pitch = 0;    // bytes, 0 = dense
    size_t slice_pitch = 0;  // bytes, 0 = dense
};

std::mutex g_fields_mu;
std::map<GLuint, FieldDesc> g_fields;
GLuint g_next_field = 1;

// Caller-registered field functors (HPMCregisterFieldFunctor), by name.
std::mutex g_functors_mu;
std::map<std::string, HPMCFieldFunctorOps> g_functors;

using hpmc::host::determine_layout;  // init.cpp:72-149
using hpmc::host::elem_size;

}  // namespace

struct HPMCHistoPyramid {
    uint32_t magic = kMagicPyramid;
    HPMCConstants* constants = nullptr;
    bool tainted = true;
    bool broken = true;  // hpiface.cpp:57
    int status = HPMC_OK;
    int lattice[3] = {0, 0, 0};
    int cells[3] = {0, 0, 0};
    float extent[3] = {1.f, 1.f, 1.f};
    bool binary = false;
    // field source
    enum { kNone, kArray, kFunctor } fmode = kNone;
    FieldDesc field;
    hpmc::FunctorParams functor{};
    bool user_functor = false;          // functor.id == 0: the caller's registered functor below
    HPMCFieldFunctorOps user_ops{};
    bool gradient = false;
    int normal_mode = HPMC_NORMALS_FORWARD;
    cudaStream_t stream = nullptr;
    // layout
    int layout[6] = {0, 0, 0, 0, 0, 0};
    // device state
    Volume V{};
    // Column layouts keep two sets of levels and arena, and builds alternate
    // between them: a build may then overlap the previous extraction, which
    // reads the other set (Volume::overlap).  One control block.
    uint32_t* d_levels = nullptr;  // nsets x levels_cap entries
    size_t levels_cap = 0;         // entries per set
    uint32_t* d_arena = nullptr;   // nsets x arena_cap slots
    size_t arena_cap = 0;          // slots per set
    int nsets = 0;
    int set = 0;                   // the set of the last build
    Ctrl* d_ctrl = nullptr;
    // the last extraction's outputs (byte ranges), stream and set: the next
    // build overlaps it only on the same stream, into the other set, and with
    // a field that is none of those outputs
    struct Range {
        const void* p;
        size_t n;
    };
    Range last_out[5] = {};
    cudaStream_t last_out_stream = nullptr;
    int last_out_set = 0;
    bool have_last_out = false;
    uint8_t* codes_capture = nullptr;
    CUtensorMap tmap;
    bool have_tmap = false;
    bool built = false;
    float threshold = 0.f;
    unsigned long long count_cached = 0;
    bool count_valid = false;
    // test hook (HPMCsetTestStall): a classifier box that never arrives
    int test_stall_box = -1;
    unsigned long long test_wait_ns = hpmc::kWaitLimitNs;
};

struct HPMCTraversalHandle {
    uint32_t magic = kMagicTraversal;
    HPMCHistoPyramid* h = nullptr;
    float* pos = nullptr;
    float* nrm = nullptr;
    size_t cap = 0;
    float* feedback = nullptr;
    size_t feedback_cap = 0;
    int32_t* dbg_cell = nullptr;
    float* dbg_t = nullptr;
    // indexed-mesh scratch (grown on demand, one allocation)
    unsigned char* mesh_mem = nullptr;
    size_t mesh_cap = 0;  // soup vertices it was sized for
};

namespace {

bool valid(const HPMCHistoPyramid* h) { return h && h->magic == kMagicPyramid; }
bool valid(const HPMCTraversalHandle* th) { return th && th->magic == kMagicTraversal && valid(th->h); }

void set_error(HPMCHistoPyramid* h, int status, bool brk) {
    h->status = status;
    if (brk) h->broken = true;
}

void release_device(HPMCHistoPyramid* h) {
    cudaFree(h->d_levels);
    cudaFree(h->d_arena);
    cudaFree(h->d_ctrl);
    h->d_levels = nullptr;
    h->d_arena = nullptr;
    h->d_ctrl = nullptr;
    h->levels_cap = h->arena_cap = 0;
    h->nsets = 0;
}

// Resolve the field source into the Volume's field members.
int bind_field(HPMCHistoPyramid* h) {
    Volume& V = h->V;
    if (h->fmode == HPMCHistoPyramid::kFunctor) {
        V.ftype = h->user_functor ? hpmc::kFieldUser : hpmc::kFieldFunctor;
        V.field = nullptr;
        V.row_pitch = V.slice_pitch = 0;
        V.functor = h->functor;
        const bool has_grad = h->user_functor ? h->user_ops.has_gradient != 0
                                              : hpmc::functor_has_gradient(h->functor.id);
        V.gradient = (h->gradient && has_grad) ? 1 : 0;
        h->have_tmap = false;
        return HPMC_OK;
    }
    if (h->fmode != HPMCHistoPyramid::kArray || !h->field.ptr) return HPMC_ERR_NO_FIELD;
    V.gradient = h->gradient ? 1 : 0;
    const FieldDesc& f = h->field;
    const size_t es = elem_size(f.type);
    const size_t rp = f.row_pitch ? f.row_pitch : (size_t)h->lattice[0] * es;
    const size_t sp = f.slice_pitch ? f.slice_pitch : rp * (size_t)h->lattice[1];
    if (rp % es || sp % es || rp < (size_t)h->lattice[0] * es || sp < rp * (size_t)h->lattice[1])
        return HPMC_ERR_INVALID_VALUE;
    V.field = f.ptr;
    V.ftype = hpmc::host::field_type(f.type);
    V.row_pitch = (long long)(rp / es);
    V.slice_pitch = (long long)(sp / es);
    V.idx32 = (V.slice_pitch * ((long long)h->lattice[2] + 1) < (1ll << 31)) ? 1 : 0;
    // TMA column path: column layout, 16-byte aligned base and pitches
    // (scalar fields only: a float4 field takes the generic classifier)
    h->have_tmap = V.column_layout && f.type != HPMC_SCALAR_F32X4 && ((uintptr_t)f.ptr % 16 == 0) &&
                   rp % 16 == 0 && sp % 16 == 0 &&
                   hpmc::host::encode_column_map(&h->tmap, f.ptr, f.type, h->lattice, rp, sp);
    return HPMC_OK;
}

// HPMCsetup (init.cpp:48-69): layout + device memory for it.
//
// Everything the device sees is ordered on the handle's stream: buffers are
// cleared with stream-ordered memsets (work still in flight on the stream --
// an extraction reading the levels and the work queue -- finishes first), and
// buffers that must grow are freed only after the stream has drained.
bool setup(HPMCHistoPyramid* h) {
    if (!h->tainted) return true;
    int L[6];
    if (!determine_layout(h->lattice, h->cells, L)) {
        h->status = HPMC_ERR_LAYOUT;
        return false;
    }
    std::memcpy(h->layout, L, sizeof L);
    Volume& V = h->V;
    V = Volume{};
    long long levels_total = 0, slots = 0;
    hpmc::host::volume_layout(V, h->lattice, h->cells, h->extent, L, &levels_total, &slots);
    V.column_slices = hpmc::host::default_column_slices(V, h->constants->num_sms);
    const int nsets = V.column_layout ? 2 : 1;
    // (re)allocate
    if ((size_t)levels_total > h->levels_cap || (size_t)slots > h->arena_cap || nsets > h->nsets || !h->d_ctrl) {
        if (h->d_ctrl && cudaStreamSynchronize(h->stream) != cudaSuccess) {
            cudaGetLastError();
            h->status = HPMC_ERR_CUDA;
            return false;
        }
        release_device(h);
        if (cudaMalloc(&h->d_levels, sizeof(uint32_t) * levels_total * nsets) != cudaSuccess ||
            cudaMalloc(&h->d_arena, hpmc::kSlotBytes * (size_t)slots * nsets) != cudaSuccess ||
            cudaMalloc(&h->d_ctrl, sizeof(Ctrl)) != cudaSuccess) {
            cudaGetLastError();
            release_device(h);
            h->status = HPMC_ERR_OUT_OF_MEMORY;
            return false;
        }
        h->levels_cap = (size_t)levels_total;
        h->arena_cap = (size_t)slots;
        h->nsets = nsets;
    }
    // every set's levels start at zero (padding blocks' level-5 entries stay zero)
    if (cudaMemsetAsync(h->d_ctrl, 0, sizeof(Ctrl), h->stream) != cudaSuccess ||
        cudaMemsetAsync(h->d_levels, 0, sizeof(uint32_t) * h->levels_cap * h->nsets, h->stream) != cudaSuccess) {
        cudaGetLastError();
        h->status = HPMC_ERR_CUDA;
        return false;
    }
    V.levels = h->d_levels;
    V.arena = h->d_arena;
    V.arena_slots = slots;
    V.ctrl = h->d_ctrl;
    h->set = 0;
    h->tainted = false;
    h->built = false;
    h->count_valid = false;
    return true;
}

int traverse_grid(const HPMCHistoPyramid* h) {
    const HPMCConstants* c = h->constants;
    int grid = c->num_sms * c->traverse_ctas_per_sm;
    if (h->count_valid) {
        const unsigned long long per_cta = 32ull * hpmc::kTraverseRounds * hpmc::kWarps;
        const unsigned long long need = (h->count_cached + per_cta - 1) / per_cta;
        grid = (int)std::max<unsigned long long>(1, std::min<unsigned long long>((unsigned long long)grid, need));
    }
    return grid;
}

int launch_extract(HPMCTraversalHandle* th, float* pos, float* nrm, float* feedback, size_t cap) {
    HPMCHistoPyramid* h = th->h;
    if (h->broken) return HPMC_ERR_BROKEN;
    if (!h->built) return HPMC_ERR_NOT_BUILT;
    hpmc::TraverseOut O{};
    O.pos = reinterpret_cast<float4*>(pos);
    O.nrm = reinterpret_cast<float4*>(nrm);
    O.feedback = feedback;
    O.capacity = cap;
    O.dbg_cell = reinterpret_cast<int4*>(th->dbg_cell);
    O.dbg_t = th->dbg_t;
    if (h->count_valid && h->count_cached > cap) h->status = HPMC_ERR_CAPACITY;
    cudaError_t e;
    if (h->V.ftype == hpmc::kFieldUser) {
        // the caller's instantiation of the traversal (include/hpmc_functor.cuh)
        const int mode = h->binary ? hpmc::kGeomBinary
                                   : (h->normal_mode == HPMC_NORMALS_CENTRAL ? hpmc::kGeomCentral : hpmc::kGeomForward);
        e = h->user_ops.traverse(&h->V, &O, mode, traverse_grid(h), h->stream) == HPMC_OK ? cudaSuccess
                                                                                       : cudaErrorLaunchFailure;
    } else {
        e = hpmc::launch_traverse(h->V, O, h->normal_mode, traverse_grid(h), h->stream);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(h, HPMC_ERR_CUDA, true);
        return HPMC_ERR_CUDA;
    }
    h->last_out[0] = {O.pos, O.pos ? cap * sizeof(float4) : 0};
    h->last_out[1] = {O.nrm, O.nrm ? cap * sizeof(float4) : 0};
    h->last_out[2] = {O.feedback, O.feedback ? cap * 6 * sizeof(float) : 0};
    h->last_out[3] = {O.dbg_cell, O.dbg_cell ? cap * sizeof(int4) : 0};
    h->last_out[4] = {O.dbg_t, O.dbg_t ? cap * sizeof(float) : 0};
    h->last_out_stream = h->stream;
    h->last_out_set = h->set;
    h->have_last_out = true;
    return (h->count_valid && h->count_cached > cap) ? HPMC_ERR_CAPACITY : HPMC_OK;
}

// A build may overlap the previous extraction (Volume::overlap) when it
// runs the column classifier on the extraction's stream, writes the set that
// extraction does not read (h->set is the build's), captures no codes, and
// its field bytes are none of the extraction's outputs.
bool may_overlap_extraction(const HPMCHistoPyramid* h) {
    if (!h->V.column_layout || !h->have_tmap || h->nsets < 2 || h->codes_capture || !h->have_last_out ||
        h->last_out_stream != h->stream || h->last_out_set == h->set || h->fmode != HPMCHistoPyramid::kArray)
        return false;
    const FieldDesc& f = h->field;
    const size_t es = elem_size(f.type);
    const size_t rp = f.row_pitch ? f.row_pitch : (size_t)h->lattice[0] * es;
    const size_t sp = f.slice_pitch ? f.slice_pitch : rp * (size_t)h->lattice[1];
    const uintptr_t a = (uintptr_t)f.ptr, an = sp * (size_t)h->lattice[2];
    for (const auto& r : h->last_out) {
        const uintptr_t b = (uintptr_t)r.p;
        if (r.n && a < b + r.n && b < a + an) return false;
    }
    return true;
}

}  // namespace

// ============================== C ABI ======================================
extern "C" {

HPMCConstants* HPMCcreateConstants(GLint max_gl_major, GLint max_gl_minor) {
    (void)max_gl_minor;
    if (max_gl_major < 2) return nullptr;  // constants.cpp:115-123
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    auto* c = new (std::nothrow) HPMCConstants;
    if (!c) return nullptr;
    c->magic = kMagicConstants;
    c->device = dev;
    c->num_sms = prop.multiProcessorCount;
    c->traverse_ctas_per_sm = hpmc::traverse_blocks_per_sm();
    hpmc::column_smem_ok();
    return c;
}

void HPMCdestroyConstants(HPMCConstants* c) {
    if (!c || c->magic != kMagicConstants) return;
    c->magic = 0;
    delete c;
}

HPMCHistoPyramid* HPMCcreateHistoPyramid(HPMCConstants* s) {
    if (!s || s->magic != kMagicConstants) return nullptr;
    auto* h = new (std::nothrow) HPMCHistoPyramid;
    if (!h) return nullptr;
    h->constants = s;
    return h;
}

void HPMCsetLatticeSize(HPMCHistoPyramid* h, GLsizei x, GLsizei y, GLsizei z) {
    if (!valid(h)) return;
    h->lattice[0] = x;
    h->lattice[1] = y;
    h->lattice[2] = z;
    h->cells[0] = std::max(1, x) - 1;
    h->cells[1] = std::max(1, y) - 1;
    h->cells[2] = std::max(1, z) - 1;
    h->tainted = true;
    h->broken = false;
    h->status = HPMC_OK;
}

void HPMCsetFieldAsBinary(HPMCHistoPyramid* h) {
    if (valid(h)) h->binary = true;
}

void HPMCsetFieldAsContinuous(HPMCHistoPyramid* h) {
    if (valid(h)) h->binary = false;
}

void HPMCsetGridSize(HPMCHistoPyramid* h, GLsizei x, GLsizei y, GLsizei z) {
    if (!valid(h)) return;
    h->cells[0] = x;
    h->cells[1] = y;
    h->cells[2] = z;
    h->tainted = true;
    h->broken = false;
    h->status = HPMC_OK;
}

void HPMCsetGridExtent(HPMCHistoPyramid* h, GLfloat x, GLfloat y, GLfloat z) {
    if (!valid(h)) return;
    h->extent[0] = x;
    h->extent[1] = y;
    h->extent[2] = z;
    h->tainted = true;
    h->broken = false;
    h->status = HPMC_OK;
}

void HPMCsetFieldTexture3D(HPMCHistoPyramid* h, GLuint texture, GLboolean gradient) {
    if (!valid(h)) return;
    FieldDesc f;
    {
        std::lock_guard<std::mutex> lk(g_fields_mu);
        auto it = g_fields.find(texture);
        if (it == g_fields.end()) {
            set_error(h, HPMC_ERR_INVALID_VALUE, true);
            return;
        }
        f = it->second;
    }
    // The layout and the device buffers do not depend on the field (it is
    // bound at every build), so a new field does not taint the handle -- as
    // in the reference, where only a change of fetch mode does
    // (hpiface.cpp:164-184).
    h->fmode = HPMCHistoPyramid::kArray;
    h->field = f;
    h->gradient = gradient != 0;
    h->broken = false;
    h->status = HPMC_OK;
}

void HPMCsetFieldCustom(HPMCHistoPyramid* h, const char* src, GLuint builder_texunit, GLboolean gradient) {
    (void)builder_texunit;
    if (!valid(h)) return;
    int id = 0;
    bool user = false;
    HPMCFieldFunctorOps ops{};
    if (src) {
        const std::string s(src);
        if (s == "hpmc:cayley") id = 1;
        else if (s == "hpmc:metaballs") id = 2;
        else if (s == "hpmc:twist_metaballs") id = 3;
        else if (s == "hpmc:spheres") id = 4;
        else {
            std::lock_guard<std::mutex> lk(g_functors_mu);
            auto it = g_functors.find(s);
            if (it != g_functors.end()) {
                user = true;
                ops = it->second;
            }
        }
    }
    if (!id && !user) {
        set_error(h, HPMC_ERR_UNSUPPORTED, true);
        return;
    }
    h->fmode = HPMCHistoPyramid::kFunctor;
    h->functor = hpmc::FunctorParams{};
    h->functor.id = id;
    h->user_functor = user;
    h->user_ops = ops;
    h->gradient = gradient != 0;
    h->broken = false;  // the field is bound at every build: no taint
    h->status = HPMC_OK;
}

GLuint HPMCgetBuilderProgram(HPMCHistoPyramid* h) {
    if (!valid(h) || h->broken) return 0;
    if (h->tainted && !setup(h)) return 0;
    if (h->fmode != HPMCHistoPyramid::kFunctor) return 0u;
    return h->user_functor ? 0x200u : 0x100u + (GLuint)h->functor.id;
}

void HPMCdestroyHandle(HPMCHistoPyramid* h) {
    if (!valid(h)) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    else cudaDeviceSynchronize();
    release_device(h);
    h->magic = 0;
    delete h;
}

void HPMCbuildHistopyramid(HPMCHistoPyramid* h, GLfloat threshold) {
    if (!valid(h) || h->broken) return;  // hpiface.cpp:229-231
    if (h->tainted && !setup(h)) return;  // hpiface.cpp:253-260: stays tainted, nothing built
    int st = bind_field(h);
    if (st != HPMC_OK) {
        set_error(h, st, true);
        return;
    }
    Volume& V = h->V;
    V.iso = threshold;
    V.binary = h->binary ? 1 : 0;
    // uint8 fields: f(b) is monotonic in b, so f(b) < iso  <=>  b < u8_thr
    V.u8_thr = hpmc::host::u8_threshold(V.ftype, h->binary ? 0.5f : threshold);
    V.codes_out = h->codes_capture;
    V.stall_box = h->test_stall_box;
    V.wait_limit_ns = h->test_wait_ns;
    // alternate the sets: the previous extraction (if still running) reads the other one
    if (V.column_layout && h->nsets == 2) {
        h->set ^= 1;
        V.levels = h->d_levels + (size_t)h->set * h->levels_cap;
        V.arena = h->d_arena + (size_t)h->set * h->arena_cap * hpmc::kSlotWords;
    }
    V.overlap = may_overlap_extraction(h) ? 1 : 0;
    h->threshold = threshold;
    const int max_ctas = h->constants->num_sms * 16;
    cudaError_t e;
    if (V.ftype == hpmc::kFieldUser) {
        // the caller's instantiation of the generic classifier (include/hpmc_functor.cuh)
        const int grid = (int)std::min<long long>(V.nblocks, (long long)max_ctas);
        e = h->user_ops.classify(&V, grid, h->stream) == HPMC_OK ? cudaSuccess : cudaErrorLaunchFailure;
    } else {
        e = hpmc::launch_classify(V, h->have_tmap ? &h->tmap : nullptr, max_ctas, h->stream);
    }
    if (e == cudaSuccess) e = hpmc::launch_reduce(V, h->stream);
    if (e != cudaSuccess) {
        set_error(h, HPMC_ERR_CUDA, true);  // hpiface.cpp:263-266
        return;
    }
    h->built = true;
    h->count_valid = false;
}

GLuint HPMCacquireNumberOfVertices(HPMCHistoPyramid* h) {
    if (!valid(h) || h->broken) return 0;  // hpiface.cpp:296-298
    if (!h->built) return 0;               // init.cpp:146-147: count starts at zero
    if (!h->count_valid) {
        Ctrl c;
        if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
            cudaMemcpy(&c, h->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost) != cudaSuccess) {
            set_error(h, HPMC_ERR_CUDA, true);
            return 0;
        }
        if (c.status & (hpmc::kStatusTimeout | hpmc::kStatusOverflow)) {
            // reported once: the next build starts from a clean status word
            // (the handle may be un-broken by a setter that does not taint)
            cudaMemsetAsync(&h->d_ctrl->status, 0, sizeof(unsigned int), h->stream);
        }
        if (c.status & hpmc::kStatusTimeout) {
            set_error(h, HPMC_ERR_TIMEOUT, true);
            return 0;
        }
        if ((c.status & hpmc::kStatusOverflow) || c.total > 0xffffffffull) {
            h->status = HPMC_ERR_OVERFLOW;
            return 0;
        }
        h->count_cached = c.total;
        h->count_valid = true;
    }
    return (GLuint)h->count_cached;
}

HPMCTraversalHandle* HPMCcreateTraversalHandle(HPMCHistoPyramid* h) {
    if (!valid(h)) return nullptr;
    if (!setup(h)) return nullptr;  // triface.cpp:79-84
    auto* th = new (std::nothrow) HPMCTraversalHandle;
    if (!th) return nullptr;
    th->h = h;
    return th;
}

void HPMCdestroyTraversalHandle(HPMCTraversalHandle* th) {
    if (!th || th->magic != kMagicTraversal) return;
    if (th->mesh_mem) {
        cudaDeviceSynchronize();
        cudaFree(th->mesh_mem);
    }
    th->magic = 0;
    delete th;
}

char* HPMCgetTraversalShaderFunctions(HPMCTraversalHandle* th) {
    if (valid(th)) th->h->status = HPMC_ERR_UNSUPPORTED;
    return nullptr;
}

bool HPMCsetTraversalHandleProgram(HPMCTraversalHandle* th, GLuint, GLuint, GLuint, GLuint) {
    if (valid(th)) th->h->status = HPMC_ERR_UNSUPPORTED;
    return false;
}

bool HPMCextractVertices(HPMCTraversalHandle* th) {
    if (!valid(th)) return false;
    if (!th->pos && !th->nrm) return false;  // triface.cpp:350-355: no program bound
    const int st = launch_extract(th, th->pos, th->nrm, nullptr, th->cap);
    if (st != HPMC_OK) th->h->status = st;
    return st == HPMC_OK;
}

static bool extract_feedback(HPMCTraversalHandle* th) {
    if (!valid(th) || !th->feedback) return false;
    const int st = launch_extract(th, nullptr, nullptr, th->feedback, th->feedback_cap);
    if (st != HPMC_OK) th->h->status = st;
    return st == HPMC_OK;
}

bool HPMCextractVerticesTransformFeedback(HPMCTraversalHandle* th) { return extract_feedback(th); }
bool HPMCextractVerticesTransformFeedbackNV(HPMCTraversalHandle* th) { return extract_feedback(th); }
bool HPMCextractVerticesTransformFeedbackEXT(HPMCTraversalHandle* th) { return extract_feedback(th); }

// ------------------------------------------------------------------------
int HPMCgetLastError(HPMCHistoPyramid* h) { return valid(h) ? h->status : HPMC_ERR_INVALID_HANDLE; }

GLuint HPMCregisterDeviceField(const void* ptr, int type, GLsizei x, GLsizei y, GLsizei z, size_t row_pitch,
                               size_t slice_pitch) {
    if (!ptr || x < 1 || y < 1 || z < 1 || type < HPMC_SCALAR_F32 || type > HPMC_SCALAR_F32X4) return 0;
    if (type == HPMC_SCALAR_F32X4 && (uintptr_t)ptr % 16) return 0;
    FieldDesc f;
    f.ptr = ptr;
    f.type = type;
    f.size[0] = x;
    f.size[1] = y;
    f.size[2] = z;
    f.row_pitch = row_pitch;
    f.slice_pitch = slice_pitch;
    std::lock_guard<std::mutex> lk(g_fields_mu);
    const GLuint name = g_next_field++;
    g_fields[name] = f;
    return name;
}

void HPMCunregisterDeviceField(GLuint name) {
    std::lock_guard<std::mutex> lk(g_fields_mu);
    g_fields.erase(name);
}

int HPMCsetFieldDevice(HPMCHistoPyramid* h, const void* ptr, int type, size_t row_pitch, size_t slice_pitch) {
    if (!valid(h)) return HPMC_ERR_INVALID_HANDLE;
    if (!ptr || type < HPMC_SCALAR_F32 || type > HPMC_SCALAR_F32X4 ||
        (type == HPMC_SCALAR_F32X4 && (uintptr_t)ptr % 16)) {
        h->status = HPMC_ERR_INVALID_VALUE;
        return h->status;
    }
    h->fmode = HPMCHistoPyramid::kArray;
    h->field = FieldDesc{};
    h->field.ptr = ptr;
    h->field.type = type;
    h->field.row_pitch = row_pitch;
    h->field.slice_pitch = slice_pitch;
    h->gradient = false;
    h->broken = false;  // the field is bound at every build: no taint
    h->status = HPMC_OK;
    return HPMC_OK;
}

int HPMCsetBuilderUniforms(HPMCHistoPyramid* h, const float* values, int count) {
    if (!valid(h)) return HPMC_ERR_INVALID_HANDLE;
    if (h->fmode != HPMCHistoPyramid::kFunctor || count < 0 || count > hpmc::kFunctorMaxParams ||
        (count && !values)) {
        h->status = HPMC_ERR_INVALID_VALUE;
        return h->status;
    }
    h->functor.count = count;
    for (int i = 0; i < count; i++) h->functor.p[i] = values[i];
    h->V.functor = h->functor;
    return HPMC_OK;
}

int HPMCsetStream(HPMCHistoPyramid* h, void* stream) {
    if (!valid(h)) return HPMC_ERR_INVALID_HANDLE;
    h->stream = static_cast<cudaStream_t>(stream);
    return HPMC_OK;
}

int HPMCsetNormalMode(HPMCHistoPyramid* h, int mode) {
    if (!valid(h)) return HPMC_ERR_INVALID_HANDLE;
    if (mode != HPMC_NORMALS_FORWARD && mode != HPMC_NORMALS_CENTRAL) return HPMC_ERR_INVALID_VALUE;
    h->normal_mode = mode;
    return HPMC_OK;
}

int HPMCgetDeviceVertexCount(HPMCHistoPyramid* h, const unsigned long long** device_count) {
    if (!valid(h)) return HPMC_ERR_INVALID_HANDLE;
    if (!device_count) return HPMC_ERR_INVALID_VALUE;
    if (h->tainted && !setup(h)) return h->status;
    *device_count = &h->d_ctrl->total;
    return HPMC_OK;
}

int HPMCsetTraversalHandleBuffers(HPMCTraversalHandle* th, float* pos, float* nrm, size_t cap) {
    if (!valid(th)) return HPMC_ERR_INVALID_HANDLE;
    if ((pos && (uintptr_t)pos % 16) || (nrm && (uintptr_t)nrm % 16)) return HPMC_ERR_INVALID_VALUE;
    th->pos = pos;
    th->nrm = nrm;
    th->cap = cap;
    return HPMC_OK;
}

int HPMCsetTraversalHandleFeedbackBuffer(HPMCTraversalHandle* th, float* buf, size_t cap) {
    if (!valid(th)) return HPMC_ERR_INVALID_HANDLE;
    if (buf && (uintptr_t)buf % 8) return HPMC_ERR_INVALID_VALUE;
    th->feedback = buf;
    th->feedback_cap = cap;
    return HPMC_OK;
}

int HPMCextractVerticesToBuffers(HPMCTraversalHandle* th, float* pos, float* nrm, size_t cap, uint64_t* n_written) {
    if (!valid(th)) return HPMC_ERR_INVALID_HANDLE;
    if ((pos && (uintptr_t)pos % 16) || (nrm && (uintptr_t)nrm % 16)) return HPMC_ERR_INVALID_VALUE;
    int st = launch_extract(th, pos, nrm, nullptr, cap);
    if (st != HPMC_OK && st != HPMC_ERR_CAPACITY) return st;
    if (n_written) {
        Ctrl c;
        if (cudaStreamSynchronize(th->h->stream) != cudaSuccess ||
            cudaMemcpy(&c, th->h->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost) != cudaSuccess) {
            set_error(th->h, HPMC_ERR_CUDA, true);
            return HPMC_ERR_CUDA;
        }
        *n_written = c.written;
        if (c.total > cap) st = HPMC_ERR_CAPACITY;
    }
    return st;
}

int HPMCextractVerticesAdjoint(HPMCTraversalHandle* th, const float* dpos, const float* dnrm, uint64_t count,
                               float* dfield) {
    if (!valid(th)) return HPMC_ERR_INVALID_HANDLE;
    HPMCHistoPyramid* h = th->h;
    if (h->broken) return HPMC_ERR_BROKEN;
    if (!h->built) return HPMC_ERR_NOT_BUILT;
    if (!dfield || (dpos && (uintptr_t)dpos % 16) || (dnrm && (uintptr_t)dnrm % 16)) return HPMC_ERR_INVALID_VALUE;
    if (h->V.ftype == hpmc::kFieldFunctor || h->V.ftype == hpmc::kFieldUser || h->V.ftype == hpmc::kFieldF32X4 ||
        h->V.gradient)
        return HPMC_ERR_UNSUPPORTED;
    if (h->binary) return HPMC_OK;  // midpoints and table normals: no dependence on f
    hpmc::AdjointIO A{};
    A.dpos = reinterpret_cast<const float4*>(dpos);
    A.dnrm = reinterpret_cast<const float4*>(dnrm);
    A.dfield = dfield;
    A.count = count;
    cudaError_t e = hpmc::launch_adjoint(h->V, A, h->normal_mode, traverse_grid(h), h->stream);
    if (e != cudaSuccess) {
        set_error(h, HPMC_ERR_CUDA, true);
        return HPMC_ERR_CUDA;
    }
    return HPMC_OK;
}

int HPMCextractVerticesIndexed(HPMCTraversalHandle* th, float* positions, float* normals, size_t vertex_capacity,
                               uint32_t* indices, size_t index_capacity, uint64_t* n_vertices, uint64_t* n_indices) {
    if (!valid(th)) return HPMC_ERR_INVALID_HANDLE;
    HPMCHistoPyramid* h = th->h;
    if (h->broken) return HPMC_ERR_BROKEN;
    if (!h->built) return HPMC_ERR_NOT_BUILT;
    if ((positions && (uintptr_t)positions % 16) || (normals && (uintptr_t)normals % 16) ||
        (indices && (uintptr_t)indices % 4))
        return HPMC_ERR_INVALID_VALUE;
    if (h->V.ftype == hpmc::kFieldUser) return HPMC_ERR_UNSUPPORTED;  // its kernels live in the caller's code
    const GLuint n = HPMCacquireNumberOfVertices(h);  // sizes the scratch (host sync)
    if (n == 0 && h->status != HPMC_OK) return h->status;
    // scratch: keys | table keys | first | scan | table vals | tile sums | meta | unique count
    size_t tsize = 1;
    while (tsize < 2 * (size_t)n + 2) tsize <<= 1;
    const size_t tiles = (size_t)n / 2048 + 2;
    auto up = [](size_t v) { return (v + 255) & ~size_t(255); };
    const size_t o_keys = 0, o_tkeys = up(o_keys + 8 * (size_t)n), o_first = up(o_tkeys + 8 * tsize),
                 o_scan = up(o_first + 4 * (size_t)n), o_tvals = up(o_scan + 4 * (size_t)n),
                 o_tiles = up(o_tvals + 4 * tsize), o_meta = up(o_tiles + 4 * tiles),
                 o_unique = up(o_meta + 2 * (size_t)n), bytes = o_unique + 256;
    if (!th->mesh_mem || th->mesh_cap < bytes) {
        if (th->mesh_mem) {
            cudaStreamSynchronize(h->stream);
            cudaFree(th->mesh_mem);
        }
        th->mesh_mem = nullptr;
        th->mesh_cap = 0;
        if (cudaMalloc(&th->mesh_mem, bytes) != cudaSuccess) {
            cudaGetLastError();
            return HPMC_ERR_OUT_OF_MEMORY;
        }
        th->mesh_cap = bytes;
    }
    unsigned char* m = th->mesh_mem;
    hpmc::MeshIO M{};
    M.count = n;
    M.keys = reinterpret_cast<unsigned long long*>(m + o_keys);
    M.table_keys = reinterpret_cast<unsigned long long*>(m + o_tkeys);
    M.first = reinterpret_cast<uint32_t*>(m + o_first);
    M.scan = reinterpret_cast<uint32_t*>(m + o_scan);
    M.table_vals = reinterpret_cast<uint32_t*>(m + o_tvals);
    M.tile_sums = reinterpret_cast<uint32_t*>(m + o_tiles);
    M.meta = reinterpret_cast<uint16_t*>(m + o_meta);
    M.unique = reinterpret_cast<unsigned long long*>(m + o_unique);
    M.table_mask = (uint32_t)(tsize - 1);
    M.pos = reinterpret_cast<float4*>(positions);
    M.nrm = reinterpret_cast<float4*>(normals);
    M.vcap = vertex_capacity;
    M.indices = indices;
    M.icap = index_capacity;
    const int grid = h->constants->num_sms * 8;
    cudaError_t e = hpmc::launch_mesh(h->V, M, h->normal_mode, traverse_grid(h), grid, h->stream);
    unsigned long long unique = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&unique, M.unique, sizeof unique, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(h, HPMC_ERR_CUDA, true);
        return HPMC_ERR_CUDA;
    }
    if (n == 0) unique = 0;
    if (n_vertices) *n_vertices = unique;
    if (n_indices) *n_indices = n;
    return (unique > vertex_capacity || (size_t)n > index_capacity) ? HPMC_ERR_CAPACITY : HPMC_OK;
}

int HPMCregisterFieldFunctor(const char* name, const HPMCFieldFunctorOps* ops) {
    if (!name || !*name || std::strncmp(name, "hpmc:", 5) == 0 || !ops || ops->abi != HPMC_FIELD_FUNCTOR_ABI ||
        ops->volume_bytes != (int)sizeof(Volume) || ops->outputs_bytes != (int)sizeof(hpmc::TraverseOut) ||
        !ops->classify || !ops->traverse)
        return HPMC_ERR_INVALID_VALUE;
    std::lock_guard<std::mutex> lk(g_functors_mu);
    g_functors[name] = *ops;
    return HPMC_OK;
}

int HPMCunregisterFieldFunctor(const char* name) {
    if (!name) return HPMC_ERR_INVALID_VALUE;
    std::lock_guard<std::mutex> lk(g_functors_mu);
    return g_functors.erase(name) ? HPMC_OK : HPMC_ERR_INVALID_VALUE;
}

int HPMCsetCodeCapture(HPMCHistoPyramid* h, uint8_t* device_codes) {
    if (!valid(h)) return HPMC_ERR_INVALID_HANDLE;
    h->codes_capture = device_codes;
    return HPMC_OK;
}

int HPMCgetLayout(HPMCHistoPyramid* h, int out[6]) {
    if (!valid(h)) return HPMC_ERR_INVALID_HANDLE;
    if (!out) return HPMC_ERR_INVALID_VALUE;
    if (h->tainted && !setup(h)) return h->status;
    std::memcpy(out, h->layout, sizeof h->layout);
    return HPMC_OK;
}

int HPMCreadLevel(HPMCHistoPyramid* h, int level, uint32_t* host_out, size_t entries) {
    if (!valid(h)) return HPMC_ERR_INVALID_HANDLE;
    if (!h->built) return HPMC_ERR_NOT_BUILT;
    const Volume& V = h->V;
    if (level < hpmc::kBlockLevel || level > V.jtop || !host_out) return HPMC_ERR_INVALID_VALUE;
    const long long n = hpmc::level_entries(V.size_l2, level);
    if ((size_t)n > entries) return HPMC_ERR_INVALID_VALUE;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
        cudaMemcpy(host_out, V.levels + V.level_off[level], sizeof(uint32_t) * n, cudaMemcpyDeviceToHost) !=
            cudaSuccess)
        return HPMC_ERR_CUDA;
    if (level == hpmc::kBlockLevel && V.column_layout) {
        // entries of padding blocks are never written by the column kernel
        for (long long b = 0; b < n; b++) {
            int z, fx, fy;
            if (!hpmc::column_block(V, (uint64_t)b, z, fx, fy)) host_out[b] = 0;
        }
    }
    return HPMC_OK;
}

int HPMCsetTraversalDebugBuffers(HPMCTraversalHandle* th, int32_t* cell_info, float* t) {
    if (!valid(th)) return HPMC_ERR_INVALID_HANDLE;
    if (cell_info && (uintptr_t)cell_info % 16) return HPMC_ERR_INVALID_VALUE;
    th->dbg_cell = cell_info;
    th->dbg_t = t;
    return HPMC_OK;
}

int HPMCsetTestStall(HPMCHistoPyramid* h, int box, unsigned int wait_limit_us) {
    if (!valid(h)) return HPMC_ERR_INVALID_HANDLE;
    h->test_stall_box = box < 0 ? -1 : box;
    h->test_wait_ns = wait_limit_us ? 1000ull * wait_limit_us : hpmc::kWaitLimitNs;
    return HPMC_OK;
}

int HPMCgetClassifyPath(HPMCHistoPyramid* h, int* path) {
    if (!valid(h)) return HPMC_ERR_INVALID_HANDLE;
    if (!path) return HPMC_ERR_INVALID_VALUE;
    if (!h->built) return HPMC_ERR_NOT_BUILT;
    *path = (h->V.column_layout && h->have_tmap) ? 1 : 0;
    return HPMC_OK;
}

int HPMCgetDeviceStatus(HPMCHistoPyramid* h, unsigned int* status) {
    if (!valid(h)) return HPMC_ERR_INVALID_HANDLE;
    if (!status) return HPMC_ERR_INVALID_VALUE;
    if (!h->d_ctrl) {
        *status = 0;
        return HPMC_OK;
    }
    Ctrl c;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
        cudaMemcpy(&c, h->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost) != cudaSuccess)
        return HPMC_ERR_CUDA;
    *status = c.status;
    const unsigned int zero = 0;
    cudaMemcpy(&h->d_ctrl->status, &zero, sizeof zero, cudaMemcpyHostToDevice);
    return HPMC_OK;
}

}  // extern "C"

// ============================================================================
// HPMCextractStatic: build + count + extract with every scratch buffer in one
// fixed device array (no device allocation).  See include/hpmc.h.
// ============================================================================
namespace {

// The scratch of HPMCextractStatic.  In host code `g_static_scratch` names a
// host-side stand-in, not device memory: kernels are given the address that
// cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) unsigned char g_static_scratch[HPMC_STATIC_SCRATCH_BYTES];

constexpr int kStaticMaxDevices = 64;

struct StaticDeviceState {
    unsigned char* scratch = nullptr;  // device address of g_static_scratch on this device
    int num_sms = 0;
    int traverse_ctas_per_sm = 0;
    bool ready = false;
};

std::mutex g_static_mu;
StaticDeviceState g_static_dev[kStaticMaxDevices];

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Once per device, with that device current: look up the scratch array's
// device address and configure the kernels.
int static_device_setup(StaticDeviceState** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return HPMC_ERR_CUDA;
    }
    if (dev < 0 || dev >= kStaticMaxDevices) return HPMC_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_static_mu);
    StaticDeviceState& s = g_static_dev[dev];
    if (!s.ready) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return HPMC_ERR_CUDA;
        }
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
            cudaGetLastError();
            return HPMC_ERR_CUDA;
        }
        s.scratch = static_cast<unsigned char*>(p);
        s.num_sms = prop.multiProcessorCount;
        s.traverse_ctas_per_sm = hpmc::traverse_blocks_per_sm();
        hpmc::column_smem_ok();
        s.ready = true;
    }
    *out = &s;
    return HPMC_OK;
}

}  // namespace

extern "C" int HPMCextractStatic(const void* field, int scalar_type, GLsizei x_size, GLsizei y_size,
                                 GLsizei z_size, size_t row_pitch_bytes, size_t slice_pitch_bytes, GLfloat iso,
                                 int normal_mode, const GLfloat* extent, float* positions, float* normals,
                                 size_t capacity_vertices, unsigned int* device_vertex_count,
                                 unsigned int* device_status, void* cuda_stream) {
    if (!field || !device_vertex_count || scalar_type < HPMC_SCALAR_F32 || scalar_type > HPMC_SCALAR_UNORM8 ||
        (normal_mode != HPMC_NORMALS_FORWARD && normal_mode != HPMC_NORMALS_CENTRAL) ||
        (positions && (uintptr_t)positions % 16) || (normals && (uintptr_t)normals % 16) ||
        ((uintptr_t)device_vertex_count % 4) || (device_status && (uintptr_t)device_status % 4))
        return HPMC_ERR_INVALID_VALUE;
    const int lattice[3] = {x_size, y_size, z_size};
    const int cells[3] = {x_size - 1, y_size - 1, z_size - 1};
    int L[6];
    if (!determine_layout(lattice, cells, L)) return HPMC_ERR_LAYOUT;  // init.cpp:82-103
    StaticDeviceState* dev = nullptr;
    int st = static_device_setup(&dev);
    if (st != HPMC_OK) return st;
    cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);

    Volume V{};
    const float ext[3] = {extent ? extent[0] : 1.0f, extent ? extent[1] : 1.0f, extent ? extent[2] : 1.0f};
    long long level_entries_total = 0, slots = 0;
    hpmc::host::volume_layout(V, lattice, cells, ext, L, &level_entries_total, &slots);
    V.column_slices = hpmc::host::default_column_slices(V, dev->num_sms);

    // carve the scratch: control block | dense levels | block codes
    const size_t ctrl_bytes = align256(sizeof(Ctrl));
    const size_t levels_bytes = align256(sizeof(uint32_t) * (size_t)level_entries_total);
    const size_t arena_bytes = hpmc::kSlotBytes * (size_t)slots;
    if (ctrl_bytes + levels_bytes + arena_bytes > (size_t)HPMC_STATIC_SCRATCH_BYTES) return HPMC_ERR_TOO_LARGE;
    unsigned char* base = dev->scratch;
    V.ctrl = reinterpret_cast<Ctrl*>(base);
    V.levels = reinterpret_cast<uint32_t*>(base + ctrl_bytes);
    V.arena = reinterpret_cast<uint32_t*>(base + ctrl_bytes + levels_bytes);
    V.arena_slots = slots;

    // field
    const size_t es = elem_size(scalar_type);
    const size_t rp = row_pitch_bytes ? row_pitch_bytes : (size_t)lattice[0] * es;
    const size_t sp = slice_pitch_bytes ? slice_pitch_bytes : rp * (size_t)lattice[1];
    if (rp % es || sp % es || rp < (size_t)lattice[0] * es || sp < rp * (size_t)lattice[1])
        return HPMC_ERR_INVALID_VALUE;
    V.field = field;
    V.ftype = hpmc::host::field_type(scalar_type);
    V.row_pitch = (long long)(rp / es);
    V.slice_pitch = (long long)(sp / es);
    V.idx32 = (V.slice_pitch * ((long long)lattice[2] + 1) < (1ll << 31)) ? 1 : 0;
    V.iso = iso;
    V.binary = 0;
    V.u8_thr = hpmc::host::u8_threshold(V.ftype, iso);
    CUtensorMap tmap;
    const bool have_tmap = V.column_layout && ((uintptr_t)field % 16 == 0) && rp % 16 == 0 && sp % 16 == 0 &&
                           hpmc::host::encode_column_map(&tmap, field, scalar_type, lattice, rp, sp);

    // the array keeps the previous call's contents: clear the control block
    // (counters, status) and the dense levels (padding entries read as zero)
    cudaError_t e = cudaMemsetAsync(base, 0, ctrl_bytes + levels_bytes, stream);
    if (e == cudaSuccess) e = hpmc::launch_classify(V, have_tmap ? &tmap : nullptr, dev->num_sms * 16, stream);
    if (e == cudaSuccess) e = hpmc::launch_reduce(V, stream);
    if (e == cudaSuccess) {
        hpmc::TraverseOut O{};
        O.pos = reinterpret_cast<float4*>(positions);
        O.nrm = reinterpret_cast<float4*>(normals);
        O.capacity = capacity_vertices;
        e = hpmc::launch_traverse(V, O, normal_mode, dev->num_sms * dev->traverse_ctas_per_sm, stream);
    }
    // full vertex count (little-endian low word of the 64-bit total) and the
    // device status bits of this call (the next call clears them)
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(device_vertex_count, &V.ctrl->total, sizeof(unsigned int), cudaMemcpyDeviceToDevice,
                            stream);
    if (e == cudaSuccess && device_status)
        e = cudaMemcpyAsync(device_status, &V.ctrl->status, sizeof(unsigned int), cudaMemcpyDeviceToDevice, stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return HPMC_ERR_CUDA;
    }
    return HPMC_OK;
}
