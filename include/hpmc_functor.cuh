/*
 * hpmc_functor.cuh -- caller-defined field functors (CUDA C++, header-only).
 *
 * The reference's custom fetch (HPMCsetFieldCustom, hpmc/include/hpmc.h:409-444
 * of the reference; hpiface.cpp:187-200, shadergen.cpp:270-286) takes any
 * GLSL function HPMC_fetch(vec3 p) -- and HPMC_fetchGrad(vec3 p) for gradient
 * normals -- that the application writes, and compiles it into the
 * HistoPyramid's shaders.  Here the application writes the same function as a
 * CUDA functor type and compiles it in its own .cu file with this header:
 * HPMC_FIELD_FUNCTOR instantiates the library's generic classifier and its
 * traversal for that type in the application's own device code and defines
 * the launch table that HPMCregisterFieldFunctor takes.  After registration,
 * HPMCsetFieldCustom(h, name, unit, gradient) selects the functor by name, and
 * HPMCgetBuilderProgram / HPMCsetBuilderUniforms set its parameters as for
 * the built-in functors.
 *
 * A functor type F:
 *
 *   namespace {                       // internal linkage for its kernels
 *   struct F {
 *       static constexpr bool kHasGradient = true;   // HPMC_fetchGrad exists
 *       // the field at p = normalised texel centres ((i + 0.5) / n per axis,
 *       // not clamped: p may lie one texel outside [0, 1]), params = the
 *       // values of HPMCsetBuilderUniforms (count of them)
 *       __device__ static float value(const float* params, int count, float x, float y, float z);
 *       // its gradient (only called if kHasGradient), in the functor's own
 *       // coordinates, as HPMC_fetchGrad returns it
 *       __device__ static void gradient(const float* params, int count, float x, float y, float z,
 *                                       float g[3]);
 *   };
 *   }
 *   HPMC_FIELD_FUNCTOR(my_ops, F)      // at namespace scope
 *   ...
 *   HPMCregisterFieldFunctor("app:my-field", &my_ops);
 *
 * Classification (f < iso, strict) uses value(); gradient mode takes t from
 * the values at the edge ends and n = iso - lerp(grad a, grad b, t), as the
 * reference does (shadergen.cpp:539-551), or -lerp(...) with
 * HPMC_NORMALS_CENTRAL; without gradient mode the normals are differences of
 * value() like the reference's.  Functor fields take the generic (per-block)
 * classifier.  Adjoint and indexed extraction are not available for them.
 *
 * Build the .cu with nvcc -gencode arch=compute_100a,code=sm_100a -std=c++17
 * and the include paths of include/ and hpmc_b200/csrc/ (the kernel bodies and
 * the build-time case tables), and link libhpmc_b200.so.
 */
#ifndef HPMC_B200_FUNCTOR_CUH
#define HPMC_B200_FUNCTOR_CUH

#include <cuda_runtime.h>

#include "hpmc.h"
#include "hpmc_classify_core.cuh"
#include "hpmc_traverse_core.cuh"

namespace hpmc {

// Launch wrappers of a caller's functor type (instantiated in the caller's
// translation unit; the library calls them through the registered table).
template <class F>
int user_classify(const void* volume, int grid, void* stream) {
    const Volume& V = *static_cast<const Volume*>(volume);
    classify_blocks<kFieldUser, F><<<grid, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(V);
    return cudaGetLastError() == cudaSuccess ? HPMC_OK : HPMC_ERR_CUDA;
}

template <class F>
int user_traverse(const void* volume, const void* outputs, int mode, int grid, void* stream) {
    const Volume& V = *static_cast<const Volume*>(volume);
    const TraverseOut& O = *static_cast<const TraverseOut*>(outputs);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    if (mode == kModeBinary)
        e = launch_dependent(traverse_kernel<kFieldUser, kModeBinary, F>, grid, kThreads, kTraverseSmem, st, V, O);
    else if (mode == kModeCentral)
        e = launch_dependent(traverse_kernel<kFieldUser, kModeCentral, F>, grid, kThreads, kTraverseSmem, st, V, O);
    else
        e = launch_dependent(traverse_kernel<kFieldUser, kModeForward, F>, grid, kThreads, kTraverseSmem, st, V, O);
    return e == cudaSuccess ? HPMC_OK : HPMC_ERR_CUDA;
}

}  // namespace hpmc

/* Defines `static const HPMCFieldFunctorOps ops` for functor type F. */
#define HPMC_FIELD_FUNCTOR(ops, F)                                                             \
    static const HPMCFieldFunctorOps ops = {HPMC_FIELD_FUNCTOR_ABI, (int)sizeof(hpmc::Volume), \
                                            (int)sizeof(hpmc::TraverseOut), (F::kHasGradient) ? 1 : 0, \
                                            &hpmc::user_classify<F>, &hpmc::user_traverse<F>}

#endif
