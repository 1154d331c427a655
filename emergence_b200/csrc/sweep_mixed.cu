// Mixed-precision form of the fused sweep: midpoint reconstruction and HLLC
// in FP32; primitives, limiter, divergence and RK accumulation in FP64.
#include "sweep_launch.h"

namespace emg {

template <int P, int D>
__global__ void __launch_bounds__(SWEEP_THREADS, 2) sweep_mixed_kernel(const SweepParams p) {
    Sweep<float, P, D>::run(p);
}

template <int P, int D> static cudaError_t launch(const SweepParams& p, dim3 grid, cudaStream_t s) {
    sweep_mixed_kernel<P, D><<<grid, SWEEP_THREADS, SweepSmem<float, P>::bytes(), s>>>(p);
    return cudaGetLastError();
}

cudaError_t sweep_launch_mixed(int P, const SweepParams& p, dim3 grid, cudaStream_t s) {
    const int D = p.d;
#define EMG_CASE(PP) \
    case PP: return D == 0 ? launch<PP, 0>(p, grid, s) : (D == 1 ? launch<PP, 1>(p, grid, s) : launch<PP, 2>(p, grid, s));
    switch (P) {
        EMG_CASE(8)
        EMG_CASE(16)
        EMG_CASE(32)
        default: return cudaErrorInvalidValue;
    }
#undef EMG_CASE
}

cudaError_t sweep_prepare_mixed() {
    cudaError_t e = cudaSuccess;
#define EMG_ATTR(PP, DD)                                                                              \
    if (e == cudaSuccess)                                                                             \
        e = cudaFuncSetAttribute(sweep_mixed_kernel<PP, DD>, cudaFuncAttributeMaxDynamicSharedMemorySize,          \
                                 (int)SweepSmem<float, PP>::bytes());
    EMG_ATTR(8, 0) EMG_ATTR(8, 1) EMG_ATTR(8, 2)
    EMG_ATTR(16, 0) EMG_ATTR(16, 1) EMG_ATTR(16, 2)
    EMG_ATTR(32, 0) EMG_ATTR(32, 1) EMG_ATTR(32, 2)
#undef EMG_ATTR
    return e;
}

}  // namespace emg
