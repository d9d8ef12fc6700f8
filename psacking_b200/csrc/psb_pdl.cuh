// psb_pdl.cuh — programmatic dependent launch (sm_90 and later) for the
// chains of dependent kernels the packing loop queues on one stream.
//
// A kernel launched through pdl(...) may be scheduled while the kernel
// before it on the stream is still draining its last CTAs, so its launch and
// CTA rasterisation overlap that tail instead of following the previous
// grid's completion.  Every kernel of the engine opens with pdl_enter():
//
//   griddepcontrol.wait              blocks until the previous grid of the
//                                    stream has completed and its memory
//                                    operations are visible -- before this
//                                    kernel reads or writes any global memory,
//                                    so neither read-after-write nor
//                                    write-after-read hazards change;
//   griddepcontrol.launch_dependents lets the next kernel be scheduled once
//                                    every CTA of this grid has passed here
//                                    (all of them resident or done).
//
// Launched the ordinary way (no attribute), the wait returns at once.  The
// wait is hardware-managed and ends when the previous grid ends: it adds no
// spin of its own.  Ordering across kernels is transitive: kernel C waits
// for B, which could not end before A had ended and published its writes.
#pragma once
#include <cuda_runtime.h>

#include <utility>

__device__ __forceinline__ void pdl_enter() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}

// set from PSB_PDL (0 = ordinary stream order for every launch)
inline bool g_pdl = true;

template <typename... KArgs>
struct PdlLaunch {
    void (*k)(KArgs...);
    dim3 grid, block;
    size_t smem;
    cudaStream_t st;
    // errors are left in the runtime's last-error slot, as a <<<>>> launch
    // leaves them, for the CKL() that follows every launch
    template <typename... Args>
    void operator()(Args&&... args) const {
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grid;
        cfg.blockDim = block;
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cfg.attrs = attr;
        cfg.numAttrs = g_pdl ? 1 : 0;
        (void)cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
    }
};

template <typename... KArgs>
PdlLaunch<KArgs...> pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st) {
    return PdlLaunch<KArgs...>{k, grid, block, smem, st};
}
