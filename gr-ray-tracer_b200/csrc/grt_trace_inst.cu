// Persistent trace kernels of one precision form and one leg.  The Makefile
// compiles this file eight times, with GRT_MIXED in {0, 1} and GRT_LEG in
// {0, 1, 2, 3}, all with -fmad=false so that every product and sum rounds
// separately, as in the reference's host build:
//   trace_fp64<I,B,SHARE,LEG>   FP64 parity form (integrate_cart_ks.hpp:230-419)
//   trace_mixed<I,B,SHARE,LEG>  mixed FP32/FP64 form (grt_rhs_mixed.cuh)
// I = integrator (0 RK4, 1 RK45); B = resident 128-thread blocks per SM, which
// caps the registers per thread at 65536 / (128 * B): 255, 170, 128 for
// B = 2, 3, 4; SHARE = frequency channels share one geodesic; LEG = whole
// rays (0), the backward leg (1) or the rest (2) of image-mode rays, or
// whole disk-mode rays without the image-mode code (3).
#include "grt_launch.h"
#include "grt_trace.cuh"

// The image-mode legs take the branch-free reciprocal and square root in the
// FP64 right-hand side (dev::Fp64RhsT<true>); the disk-mode kernel measured
// slower with them and keeps CUDA's.
#define GRT_RHS_BF (GRT_LEG != 3)
// The 2-blocks/SM kernels (255 registers; the workloads with about one warp
// per scheduler) are latency-bound: their policies take LAT (grt_trace.cuh).
#if GRT_MIXED
#include "grt_rhs_mixed.cuh"
#define GRT_TRACE_KERNEL trace_mixed
#define GRT_TRACE_RHS(MINB) dev::MixedRhsT<GRT_RHS_BF, (MINB) == 2>
#else
#define GRT_TRACE_KERNEL trace_fp64
#define GRT_TRACE_RHS(MINB) dev::Fp64RhsT<GRT_RHS_BF, (MINB) == 2>
#endif
#define GRT_CAT2(a, b) a##b
#define GRT_CAT(a, b) GRT_CAT2(a, b)
#define GRT_LAUNCHER GRT_CAT(GRT_CAT(launch_, GRT_TRACE_KERNEL), GRT_CAT(_leg, GRT_LEG))

namespace grt {

template <int INTEGRATOR, int MINB, bool SHARE, int LEG>
__global__ void __launch_bounds__(128, MINB) GRT_TRACE_KERNEL(const __grid_constant__ KParams kp) {
    extern __shared__ double smem[];
    dev::Axes ax;
    dev::KStore kk;
    dev::stage_grid(kp, smem, INTEGRATOR, ax, kk);
    dev::trace_body<INTEGRATOR, GRT_TRACE_RHS(MINB), false, SHARE, LEG>(kp, ax, kk);
}

namespace {

template <int I, int B>
cudaError_t launch_v(const KParams& kp, int blocks, size_t smem, cudaStream_t stream) {
    if constexpr (GRT_LEG == 3) {
        // disk mode never shares channels
        if (kp.ngroups > 0) return cudaErrorInvalidValue;
    } else if (kp.ngroups > 0) {
        cudaFuncSetAttribute(GRT_TRACE_KERNEL<I, B, true, GRT_LEG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
        GRT_TRACE_KERNEL<I, B, true, GRT_LEG><<<blocks, 128, smem, stream>>>(kp);
        return cudaGetLastError();
    }
    {
        cudaFuncSetAttribute(GRT_TRACE_KERNEL<I, B, false, GRT_LEG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
        GRT_TRACE_KERNEL<I, B, false, GRT_LEG><<<blocks, 128, smem, stream>>>(kp);
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t GRT_LAUNCHER(const KParams& kp, int integrator, int blocks_per_sm, int blocks, size_t smem,
                         cudaStream_t stream) {
    if (integrator == 0) {
        switch (blocks_per_sm) {
            case 2: return launch_v<0, 2>(kp, blocks, smem, stream);
            case 3: return launch_v<0, 3>(kp, blocks, smem, stream);
            case 4: return launch_v<0, 4>(kp, blocks, smem, stream);
            default: return cudaErrorInvalidConfiguration;
        }
    }
    switch (blocks_per_sm) {
        case 2: return launch_v<1, 2>(kp, blocks, smem, stream);
        case 3: return launch_v<1, 3>(kp, blocks, smem, stream);
        case 4: return launch_v<1, 4>(kp, blocks, smem, stream);
        default: return cudaErrorInvalidConfiguration;
    }
}

#if GRT_LEG == 2 && !GRT_MIXED
// Packet generation between the two legs (dev::generate_body): one thread per
// queue index, the separable axes staged in shared memory for the lookup.
template <bool SHARE>
__global__ void __launch_bounds__(128) generate_pending(const __grid_constant__ KParams kp) {
    extern __shared__ double smem[];
    dev::Axes ax;
    dev::KStore kk;
    dev::stage_grid(kp, smem, 0, ax, kk);
    dev::generate_body<SHARE>(kp, ax);
}

cudaError_t launch_generate_pending(const KParams& kp, int sm_count, size_t smem, cudaStream_t stream) {
    if (kp.n == 0) return cudaSuccess;
    const unsigned long long want = (kp.n + 127) / 128;
    const unsigned long long cap = static_cast<unsigned long long>(sm_count) * 16;
    const unsigned blocks = static_cast<unsigned>(want < cap ? want : cap);
    if (kp.ngroups > 0) {
        cudaFuncSetAttribute(generate_pending<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        generate_pending<true><<<blocks, 128, smem, stream>>>(kp);
    } else {
        cudaFuncSetAttribute(generate_pending<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
        generate_pending<false><<<blocks, 128, smem, stream>>>(kp);
    }
    return cudaGetLastError();
}
#endif

}  // namespace grt
