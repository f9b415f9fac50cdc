/*
 * hpmc.h -- C ABI of the B200-native HistoPyramid marching-cubes extractor.
 *
 * Drop-in for HPMC's public interface (hpmc/include/hpmc.h:291-549 of the
 * reference, "extern C", opaque handles): every reference entry point keeps
 * its name, argument list and error convention (NULL / false / 0 returns and a
 * sticky "broken" flag on the pyramid handle).  The GL context leaves the hot
 * path: fields are device arrays or registered device functors, the pyramid
 * lives in device memory, and traversal writes vertices into caller-owned
 * device buffers instead of a GL draw or transform feedback.  The extra entry
 * points below the reference block are CUDA-native; each returns an
 * HPMCStatus.  Handles are not thread-safe; distinct handles are independent.
 *
 * Scalar types come from hpmc_types.h (GL's widths, no GL header needed).
 */
#ifndef HPMC_B200_H
#define HPMC_B200_H

#include <stddef.h>
#include <stdint.h>

#include "hpmc_types.h"

#ifdef __cplusplus
extern "C" {
#else
#include <stdbool.h>
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

struct HPMCConstants;
struct HPMCHistoPyramid;
struct HPMCTraversalHandle;

/* ---- status codes (HPMCgetLastError and the CUDA-native entry points) ---- */
typedef enum HPMCStatus {
    HPMC_OK = 0,
    HPMC_ERR_INVALID_HANDLE = 1,  /* NULL or destroyed handle */
    HPMC_ERR_INVALID_VALUE = 2,   /* bad argument */
    HPMC_ERR_LAYOUT = 3,          /* lattice/grid sizes rejected (init.cpp:82-103) */
    HPMC_ERR_UNSUPPORTED = 4,     /* GL/GLSL-only feature with no device equivalent */
    HPMC_ERR_CUDA = 5,            /* a CUDA call failed */
    HPMC_ERR_OUT_OF_MEMORY = 6,
    HPMC_ERR_CAPACITY = 7,        /* output buffer smaller than the vertex count */
    HPMC_ERR_NOT_BUILT = 8,       /* extraction before HPMCbuildHistopyramid */
    HPMC_ERR_BROKEN = 9,          /* handle is broken until reconfigured */
    HPMC_ERR_NO_FIELD = 10,       /* no field source set */
    HPMC_ERR_OVERFLOW = 11,       /* vertex count does not fit 32 bits */
    HPMC_ERR_TIMEOUT = 12,        /* a bounded device wait gave up */
    HPMC_ERR_TOO_LARGE = 13       /* lattice too large for HPMCextractStatic's fixed scratch or for a batch */
} HPMCStatus;

/* ---- field element types of device arrays ---- */
typedef enum HPMCScalarType {
    HPMC_SCALAR_F32 = 0,     /* float */
    HPMC_SCALAR_U8 = 1,      /* uint8 read as float(b) */
    HPMC_SCALAR_UNORM8 = 2,  /* uint8 read as b/255, like a GL_ALPHA / GL_UNSIGNED_BYTE texture */
    HPMC_SCALAR_F32X4 = 3    /* float4 per sample: gradient x, y, z and the value, like a GL RGBA
                                float texture (value in alpha); the field is the value, and
                                HPMCsetFieldTexture3D(..., GL_TRUE) uses the stored gradient */
} HPMCScalarType;

/* ---- normal estimation ---- */
typedef enum HPMCNormalMode {
    HPMC_NORMALS_FORWARD = 0,  /* reference: iso - lerp(f(a+e_i), f(b+e_i), t) (shadergen.cpp:528-551) */
    HPMC_NORMALS_CENTRAL = 1   /* -lerp(central difference at a, at b, t) / 2 steps, same scaling */
} HPMCNormalMode;

/* ======================= reference entry points ========================= */

/* hpmc.h:310-311 / constants.cpp:54-347.  Device-side constant tables for
 * the current CUDA device.  NULL if no CUDA device is usable or if
 * max_gl_major < 2 (the reference's "GL 2.0 required" rejection). */
struct HPMCConstants* HPMCcreateConstants(GLint max_gl_major, GLint max_gl_minor);

/* hpmc.h:319-320 / constants.cpp:350-392.  NULL-safe. */
void HPMCdestroyConstants(struct HPMCConstants* c);

/* hpmc.h:330-331 / hpiface.cpp:45-97.  NULL if constants is NULL.  Starts
 * broken until a lattice/grid/field setter is called (hpiface.cpp:57). */
struct HPMCHistoPyramid* HPMCcreateHistoPyramid(struct HPMCConstants* s);

/* hpmc.h:345-349 / hpiface.cpp:100-114.  cells := size - 1; taints. */
void HPMCsetLatticeSize(struct HPMCHistoPyramid* h, GLsizei x_size, GLsizei y_size, GLsizei z_size);

/* hpmc.h:351-352 / hpiface.cpp:131-135.  Threshold 0.5, edge midpoints and
 * table normals.  Does not taint (as in the reference). */
void HPMCsetFieldAsBinary(struct HPMCHistoPyramid* h);

/* hpmc.h:354-355 / hpiface.cpp:138-142. */
void HPMCsetFieldAsContinuous(struct HPMCHistoPyramid* h);

/* hpmc.h:374-378 / hpiface.cpp:117-128.  Checked lazily (init.cpp:98-103). */
void HPMCsetGridSize(struct HPMCHistoPyramid* h, GLsizei x_size, GLsizei y_size, GLsizei z_size);

/* hpmc.h:391-395 / hpiface.cpp:145-161.  Default (1,1,1). */
void HPMCsetGridExtent(struct HPMCHistoPyramid* h, GLfloat x_extent, GLfloat y_extent, GLfloat z_extent);

/* hpmc.h:404-407 / hpiface.cpp:164-184.  `texture` is a field name returned
 * by HPMCregisterDeviceField (the stand-in for a GL 3-D texture name).  The
 * field is the value (alpha) channel.  gradient = GL_TRUE uses the stored
 * gradient of an HPMC_SCALAR_F32X4 field (shadergen.cpp:260-266): t from the
 * values at the edge ends and, as the reference computes it
 * (shadergen.cpp:539-551), n = iso - lerp(grad a, grad b, t); with
 * HPMC_NORMALS_CENTRAL, n = -lerp(grad a, grad b, t).  Single-channel fields
 * read a zero gradient there, as GL's alpha textures return rgb = 0. */
void HPMCsetFieldTexture3D(struct HPMCHistoPyramid* h, GLuint texture, GLboolean gradient);

/* hpmc.h:440-444 / hpiface.cpp:187-200.  shader_source names a device
 * functor instead of carrying GLSL: a built-in one ("hpmc:cayley",
 * "hpmc:metaballs", "hpmc:twist_metaballs", "hpmc:spheres") or one the
 * caller registered with HPMCregisterFieldFunctor.  Any other text sets
 * HPMC_ERR_UNSUPPORTED and breaks the handle.  builder_texunit is ignored.
 * gradient = GL_TRUE uses the functor's analytic gradient where it has one
 * (cayley; a registered functor with has_gradient): t from the functor
 * values at the edge ends and, as the reference computes it
 * (shadergen.cpp:539-551), n = iso - lerp(grad a, grad b, t); with
 * HPMC_NORMALS_CENTRAL, n = -lerp(grad a, grad b, t). */
void HPMCsetFieldCustom(struct HPMCHistoPyramid* h, const char* shader_source, GLuint builder_texunit,
                        GLboolean gradient);

/* hpmc.h:446-447 / hpiface.cpp:202-222.  Returns a non-zero parameter-block
 * name for the functor's uniforms (set them with HPMCsetBuilderUniforms), 0
 * if the handle is broken. */
GLuint HPMCgetBuilderProgram(struct HPMCHistoPyramid* h);

/* hpmc.h:451-452 (declared, never defined by the reference).  Destroys the
 * pyramid and its device memory; NULL-safe. */
void HPMCdestroyHandle(struct HPMCHistoPyramid* handle);

/* hpmc.h:460-462 / hpiface.cpp:225-290.  Classifies the field at `threshold`
 * and builds the pyramid on the handle's stream (asynchronous).  Errors set
 * the broken flag.
 *
 * On the TMA column path a build may start while the handle's previous
 * extraction on the same stream is still writing its vertices.  Builds on
 * column layouts alternate between two sets of pyramid levels and block
 * codes (twice the memory), so the running extraction keeps its own.  The
 * early start never happens when the field's bytes overlap that
 * extraction's outputs, or when any other work (a kernel, copy or event
 * wait) comes between the two calls on the stream; the build is then fully
 * ordered.  A kernel launched by the
 * caller with programmatic stream serialization between an extraction and a
 * build must call cudaGridDependencySynchronize() before it writes the field,
 * which is the rule for such launches in any case. */
void HPMCbuildHistopyramid(struct HPMCHistoPyramid* h, GLfloat threshold);

/* hpmc.h:468-469 / hpiface.cpp:293-345.  Vertex count of the last build;
 * waits for it (host sync).  0 on error or if the count exceeds 32 bits. */
GLuint HPMCacquireNumberOfVertices(struct HPMCHistoPyramid* handle);

/* hpmc.h:478-479 / triface.cpp:43-109.  NULL if the pyramid cannot be set up. */
struct HPMCTraversalHandle* HPMCcreateTraversalHandle(struct HPMCHistoPyramid* handle);

/* hpmc.h:485-486 / triface.cpp:112-122. */
void HPMCdestroyTraversalHandle(struct HPMCTraversalHandle* th);

/* hpmc.h:495-496 / triface.cpp:125-192.  There is no GLSL to hand out:
 * returns NULL and sets HPMC_ERR_UNSUPPORTED. */
char* HPMCgetTraversalShaderFunctions(struct HPMCTraversalHandle* th);

/* hpmc.h:516-521 / triface.cpp:195-327.  No GL program exists: returns false
 * and sets HPMC_ERR_UNSUPPORTED.  Bind output buffers with
 * HPMCsetTraversalHandleBuffers instead. */
bool HPMCsetTraversalHandleProgram(struct HPMCTraversalHandle* th, GLuint program, GLuint tex_unit_work1,
                                   GLuint tex_unit_work2, GLuint tex_unit_work3);

/* hpmc.h:534-535 / triface.cpp:460-464.  Writes every vertex of the last
 * build into the buffers bound by HPMCsetTraversalHandleBuffers (float4
 * positions and normals).  false if no buffers are bound, the pyramid is
 * broken or the buffers are too small (the first `capacity` vertices are
 * written and HPMC_ERR_CAPACITY is set). */
bool HPMCextractVertices(struct HPMCTraversalHandle* th);

/* hpmc.h:537-544 / triface.cpp:468-500.  Transform-feedback capture: writes
 * interleaved N3F_V3F (normal xyz, position xyz) into the buffer bound by
 * HPMCsetTraversalHandleFeedbackBuffer.  The NV and EXT variants are the same
 * call. */
bool HPMCextractVerticesTransformFeedback(struct HPMCTraversalHandle* th);
bool HPMCextractVerticesTransformFeedbackNV(struct HPMCTraversalHandle* th);
bool HPMCextractVerticesTransformFeedbackEXT(struct HPMCTraversalHandle* th);

/* ===================== CUDA-native entry points ========================= */

/* Last status of a pyramid handle (cleared by a successful reconfiguration). */
int HPMCgetLastError(struct HPMCHistoPyramid* h);

/* Stand-in for glTexImage3D + a texture name: registers a device array as a
 * field and returns its non-zero name for HPMCsetFieldTexture3D (0 on bad
 * arguments).  Pitches in bytes; 0 means dense.  The array is not copied. */
GLuint HPMCregisterDeviceField(const void* device_ptr, int scalar_type, GLsizei x_size, GLsizei y_size,
                               GLsizei z_size, size_t row_pitch_bytes, size_t slice_pitch_bytes);
void HPMCunregisterDeviceField(GLuint name);

/* Sets a device array as the field directly (lattice size from
 * HPMCsetLatticeSize).  Pitches in bytes, 0 = dense.  Does not taint the
 * handle: the field is bound at the next build (a new field therefore never
 * disturbs work still in flight on the handle's stream). */
int HPMCsetFieldDevice(struct HPMCHistoPyramid* h, const void* device_ptr, int scalar_type,
                       size_t row_pitch_bytes, size_t slice_pitch_bytes);

/* Uniform values of a functor field (glUniform on the builder program in
 * the reference's custom-fetch use, apps/metaballs/metaballs.cpp:277-281). */
int HPMCsetBuilderUniforms(struct HPMCHistoPyramid* h, const float* values, int count);

/* CUDA stream all work of this handle is issued on (default: stream 0). */
int HPMCsetStream(struct HPMCHistoPyramid* h, void* cuda_stream);

/* Normal estimation (default HPMC_NORMALS_FORWARD, the reference's). */
int HPMCsetNormalMode(struct HPMCHistoPyramid* h, int mode);

/* Device-side vertex count of the last build (uint64, device pointer) for
 * stream-ordered consumers; valid after the build completes on the stream. */
int HPMCgetDeviceVertexCount(struct HPMCHistoPyramid* h, const unsigned long long** device_count);

/* Output buffers used by HPMCextractVertices (device pointers; float4 x,y,z,1
 * and nx,ny,nz,0 per vertex; either may be NULL) and their capacity. */
int HPMCsetTraversalHandleBuffers(struct HPMCTraversalHandle* th, float* positions, float* normals,
                                  size_t capacity_vertices);

/* Output buffer of HPMCextractVerticesTransformFeedback*: 6 floats per vertex. */
int HPMCsetTraversalHandleFeedbackBuffer(struct HPMCTraversalHandle* th, float* n3f_v3f,
                                         size_t capacity_vertices);

/* One-call extraction into device buffers without a host sync: the kernel
 * reads the vertex count on the device.  If n_written is non-NULL the call
 * waits and stores the number of vertices written. */
int HPMCextractVerticesToBuffers(struct HPMCTraversalHandle* th, float* positions, float* normals,
                                 size_t capacity_vertices, uint64_t* n_written);

/* Adjoint of the extraction: given dL/dp and dL/dn per vertex (float4, w
 * ignored; either may be NULL) for the first `count` vertices of the last
 * build, ACCUMULATES dL/df into d_field, a float array with the field's
 * lattice shape and element pitches (dense when the field is dense).
 * Recomputes the traversal; topology is piecewise constant.  F32/U8/UNORM8
 * array fields, forward or central normals; binary fields have zero
 * gradient. */
int HPMCextractVerticesAdjoint(struct HPMCTraversalHandle* th, const float* dL_dpositions,
                               const float* dL_dnormals, uint64_t count, float* d_field);

/* ---- inspection (tests, tools) ---- */

/* Capture every cell's MC code during the next builds into a device buffer
 * of cells_x*cells_y*cells_z bytes ([z][y][x]); NULL stops capturing. */
int HPMCsetCodeCapture(struct HPMCHistoPyramid* h, uint8_t* device_codes);

/* Layout of the pyramid: out[0..5] = tile_x, tile_y, layout_x, layout_y,
 * size_l2, size (init.cpp:105-130). */
int HPMCgetLayout(struct HPMCHistoPyramid* h, int out[6]);

/* Copies dense pyramid level j (5 <= j <= size_l2 + 1, the reference's mip
 * level j flattened channel-wise in Morton order; entries = 4^(size_l2+1-j))
 * into host memory. */
int HPMCreadLevel(struct HPMCHistoPyramid* h, int level, uint32_t* host_out, size_t entries);

/* Per-vertex debug outputs of the next extractions (device pointers, may be
 * NULL): int4 (x, y, z, code | k << 8 | edge << 16) and float t. */
int HPMCsetTraversalDebugBuffers(struct HPMCTraversalHandle* th, int32_t* cell_info, float* t);

/* Device status word of the pyramid (bits: 1 overflow, 2 capacity,
 * 8 timeout); waits for the handle's stream. */
int HPMCgetDeviceStatus(struct HPMCHistoPyramid* h, unsigned int* status);

/* Test hook for failure detection (no counterpart in the reference; it
 * makes a bounded device wait run out without any fault).  From the next
 * build on, the producer of every persistent TMA column classifier CTA never
 * issues box `box` (0-based) of the CTA's stream of boxes -- neither the
 * expected-byte count nor the copy -- so the consumers' waits on that box
 * give up after wait_limit_us
 * microseconds (0: the default limit of 2 s), the CTAs drain their copies
 * in flight and exit, and the build reports HPMC_ERR_TIMEOUT
 * (HPMCacquireNumberOfVertices returns 0 and breaks the handle).  box < 0
 * turns the hook off.  Builds on the generic classifier are not affected. */
int HPMCsetTestStall(struct HPMCHistoPyramid* h, int box, unsigned int wait_limit_us);

/* Classification path of the last build: 1 = TMA column kernel (every 32x32
 * cell block inside one slice tile, 16-byte aligned array field), 0 = generic
 * per-block kernel (narrow tiles, unaligned pitches, functor fields). */
int HPMCgetClassifyPath(struct HPMCHistoPyramid* h, int* path);

/* ---- caller-defined field functors ----
 *
 * The reference compiles whatever HPMC_fetch GLSL the application hands to
 * HPMCsetFieldCustom into its shaders (hpmc.h:409-444).  Here the
 * application compiles its field as a CUDA functor type in its own .cu file
 * with include/hpmc_functor.cuh, whose HPMC_FIELD_FUNCTOR macro instantiates
 * the classification and traversal kernels for that type in the
 * application's device code and fills this launch table; registering the
 * table under a name makes that name valid for HPMCsetFieldCustom.  The
 * table is copied; the functions it points to must stay loaded while handles
 * use the name.  Names starting with "hpmc:" are reserved. */
#define HPMC_FIELD_FUNCTOR_ABI 1u
typedef struct HPMCFieldFunctorOps {
    unsigned int abi;   /* HPMC_FIELD_FUNCTOR_ABI */
    int volume_bytes;   /* size of the volume descriptor the functor was compiled against */
    int outputs_bytes;  /* size of the output descriptor */
    int has_gradient;   /* the functor has an analytic gradient (HPMC_fetchGrad) */
    /* launches the classification of the volume descriptor on a grid of `grid` CTAs */
    int (*classify)(const void* volume, int grid, void* cuda_stream);
    /* launches the extraction: normal_mode 0 forward, 1 central, 2 binary field */
    int (*traverse)(const void* volume, const void* outputs, int normal_mode, int grid, void* cuda_stream);
} HPMCFieldFunctorOps;

/* No counterpart in the reference (its custom fetch is GLSL text).
 * HPMC_ERR_INVALID_VALUE for a reserved or empty name, a NULL or mismatched
 * table (ABI, descriptor sizes); registering a name again replaces it. */
int HPMCregisterFieldFunctor(const char* name, const HPMCFieldFunctorOps* ops);
int HPMCunregisterFieldFunctor(const char* name);

/* ---- indexed (welded) output ----
 *
 * No counterpart in the reference, which emits triangle soup only.  One
 * vertex per crossed lattice edge, numbered in order of first occurrence in
 * the soup of HPMCextractVertices, written as float4 positions / normals
 * (either may be NULL), and one uint32 index per soup vertex -- three per
 * triangle, in the soup's triangle order.  A unique vertex's values equal
 * those of its soup vertices (binary fields: the normal of its first
 * occurrence, as table normals depend on the cell's case).  Waits for the
 * result; n_vertices / n_indices receive the full counts (HPMC_ERR_CAPACITY
 * if an output was too small: what fits is written).  Device scratch of
 * about 40 bytes per soup vertex is kept with the traversal handle. */
int HPMCextractVerticesIndexed(struct HPMCTraversalHandle* th, float* positions, float* normals,
                               size_t vertex_capacity, uint32_t* indices, size_t index_capacity,
                               uint64_t* n_vertices, uint64_t* n_indices);

/* ---- batched extraction ----
 *
 * No counterpart in the reference, which builds one volume per HistoPyramid
 * handle.  A batch holds many volumes of uneven lattices and iso-values (one
 * scalar type per batch) and extracts all of them with three launches --
 * classify over every volume's bricks, reduce over every volume's pyramid,
 * one persistent traversal -- captured once in a CUDA graph and replayed.
 * Per volume the vertices, their order and their values equal those of
 * HPMCbuildHistopyramid + HPMCextractVerticesToBuffers on that volume.
 * Vertices of volume v are written at [offsets[v], offsets[v+1]) of the
 * float4 position/normal outputs (either may be NULL).  Batches are not
 * thread-safe; calls on different streams must be ordered by the caller. */
typedef struct HPMCBatchVolume {
    const void* field;        /* device array, x fastest */
    int scalar_type;          /* HPMCScalarType, the same for every volume */
    GLsizei size[3];          /* lattice size (HPMCsetLatticeSize); grid = size - 1 */
    size_t row_pitch_bytes;   /* 0 = dense */
    size_t slice_pitch_bytes; /* 0 = dense */
    GLfloat iso;              /* threshold of this volume */
    GLfloat extent[3];        /* HPMCsetGridExtent; all zero means (1,1,1) */
} HPMCBatchVolume;

struct HPMCBatch;

/* Lays out every volume (reference layout per volume) and allocates the
 * batch.  HPMC_ERR_LAYOUT for a lattice the reference rejects,
 * HPMC_ERR_TOO_LARGE for a volume whose base level exceeds 2^15 x 2^15
 * texels, HPMC_ERR_INVALID_VALUE for mixed scalar types or bad pitches. */
int HPMCcreateBatch(struct HPMCConstants* c, const HPMCBatchVolume* volumes, int count, struct HPMCBatch** out);
void HPMCdestroyBatch(struct HPMCBatch* b);
/* New iso-values (count entries); the fields themselves may change in place. */
int HPMCbatchSetIsoValues(struct HPMCBatch* b, const GLfloat* iso);
int HPMCbatchSetNormalMode(struct HPMCBatch* b, int mode);
/* Asynchronous build + count + extraction of every volume on `cuda_stream`
 * (a graph replay; the graph is captured again only when the outputs,
 * capacity, normal mode or tuning change). */
int HPMCbatchExtract(struct HPMCBatch* b, float* positions, float* normals, size_t capacity_vertices,
                     void* cuda_stream);
/* count + 1 output offsets of the last extraction (the last entry is the
 * total, which may exceed the capacity); waits for it.  Returns
 * HPMC_ERR_CAPACITY if the outputs were too small (the vertices that fit
 * are written). */
int HPMCbatchGetOffsets(struct HPMCBatch* b, unsigned long long* host_offsets);
/* Device array of the count + 1 offsets, for stream-ordered consumers. */
int HPMCbatchGetDeviceOffsets(struct HPMCBatch* b, const unsigned long long** device_offsets);
/* Brick depth (slices per column CTA: 7, 15, 31, 63; 0 = automatic),
 * traversal CTAs per SM (0 = maximum) and rounds of 32 vertices per
 * traversal work item (1..64; 0 = default). */
int HPMCbatchSetTuning(struct HPMCBatch* b, int column_slices, int traverse_ctas_per_sm, int rounds);
int HPMCbatchGetTuning(struct HPMCBatch* b, int out[3]);
/* Test hook (see HPMCsetTestStall): the column classifier never receives box
 * `box` of volume `volume`'s first column; HPMCbatchGetOffsets then returns
 * HPMC_ERR_TIMEOUT.  box < 0 turns it off (the volume index is still
 * checked). */
int HPMCbatchSetTestStall(struct HPMCBatch* b, int volume, int box, unsigned int wait_limit_us);
/* Times every tuning choice on these outputs (graph replays, CUDA events)
 * and keeps the fastest; `chosen` (may be NULL) receives it.  The choice is
 * remembered for the rest of the process per batch signature (scalar type,
 * normal mode, SM count, every volume's lattice size): autotuning a batch of
 * the same signature again takes it without timing. */
int HPMCbatchAutotune(struct HPMCBatch* b, float* positions, float* normals, size_t capacity_vertices,
                      void* cuda_stream, int chosen[3]);

/* ---- extraction without device allocation ----
 *
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory at extraction time: hosts that reserve the whole GPU memory budget
 * up front (render engines and plugins handed fixed buffers) and real-time
 * loops where cudaMalloc/cudaFree -- which synchronise the device -- are not
 * allowed.  One call builds, counts and extracts like HPMCbuildHistopyramid +
 * HPMCextractVerticesToBuffers, but every scratch buffer (pyramid levels,
 * code arena, control block) lives in one fixed device array of
 * HPMC_STATIC_SCRATCH_BYTES that the library holds on every GPU that loads
 * it until the process exits; it calls no cudaMalloc, cudaFree or other
 * allocating routine.
 *
 * The caller passes the field (device pointer, pitches in bytes, 0 = dense),
 * the outputs (float4 positions and normals, either may be NULL; capacity
 * in vertices) and a device uint32 that receives the full vertex count (so
 * that count > capacity shows truncation).  device_status (a device uint32,
 * may be NULL) receives the call's device status bits, as
 * HPMCgetDeviceStatus reports them for a handle: 1 the count does not fit
 * 32 bits, 2 the outputs were too small (the first `capacity` vertices are
 * written), 8 a bounded wait in the classifier gave up (HPMC_ERR_TIMEOUT:
 * the count and the outputs of that call are invalid).  Both are written on
 * the stream after the extraction, so no host sync is needed to read them in
 * stream order.  extent may be NULL (1,1,1).  Work is issued on
 * `cuda_stream`.  Lattices whose pyramid and block codes do not fit
 * the scratch (e.g. larger than about 225^3) are rejected with
 * HPMC_ERR_TOO_LARGE.  The first call on a device looks up the scratch
 * array's device address and configures the kernels, so make it before any
 * stream capture.  All calls share the one scratch array, which keeps the
 * last call's contents (the call clears what must start at zero): calls that
 * overlap on the GPU -- different streams, or concurrent host threads -- race
 * and must be serialised by the caller. */
#define HPMC_STATIC_SCRATCH_BYTES (16u << 20)
int HPMCextractStatic(const void* field, int scalar_type, GLsizei x_size, GLsizei y_size, GLsizei z_size,
                      size_t row_pitch_bytes, size_t slice_pitch_bytes, GLfloat iso, int normal_mode,
                      const GLfloat* extent, float* positions, float* normals, size_t capacity_vertices,
                      unsigned int* device_vertex_count, unsigned int* device_status, void* cuda_stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif
