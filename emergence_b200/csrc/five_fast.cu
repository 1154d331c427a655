// Fast FP64 form of the five-equation fused sweep: every value and operation
// in FP64, built with FMA contraction, with the WENO5-Z weights, the
// characteristic projection's coefficients, the mixture closure (1/(γ − 1) of
// each phase precomputed), the Kapila coefficient, the primitive recovery and
// the HLLC star states from the one-ulp reciprocals of physics.cuh's fast
// section. Held to a tolerance of the plain form (which stays bit-exact with
// the reference CPU solver) instead of bit equality.
#include "five_launch.h"

namespace emg {

template <int P, int D, int MODE, bool AMR>
__global__ void __launch_bounds__(SWEEP_THREADS, 2) five_fast_sweep_kernel(const FiveSweepParams p) {
    FiveSweep<P, D, MODE, AMR, true>::run(p);
}

template <int P, int MODE, bool AMR> static cudaError_t launch_d(const FiveSweepParams& p, dim3 grid, cudaStream_t s) {
    const size_t b = FiveSmem<P, MODE>::bytes();
    if (p.d == 0)
        five_fast_sweep_kernel<P, 0, MODE, AMR><<<grid, SWEEP_THREADS, b, s>>>(p);
    else if (p.d == 1)
        five_fast_sweep_kernel<P, 1, MODE, AMR><<<grid, SWEEP_THREADS, b, s>>>(p);
    else
        five_fast_sweep_kernel<P, 2, MODE, AMR><<<grid, SWEEP_THREADS, b, s>>>(p);
    return cudaGetLastError();
}
template <int MODE, bool AMR> static cudaError_t launch_p(int P, const FiveSweepParams& p, dim3 grid, cudaStream_t s) {
    switch (P) {
        case 8: return AMR ? cudaErrorInvalidValue : launch_d<8, MODE, false>(p, grid, s);
        case 16: return launch_d<16, MODE, AMR>(p, grid, s);
        case 32: return launch_d<32, MODE, AMR>(p, grid, s);
        default: return cudaErrorInvalidValue;
    }
}
template <bool AMR> static cudaError_t launch(int P, int mode, const FiveSweepParams& p, dim3 grid, cudaStream_t s) {
    switch (mode) {
        case MODE_WENO: return launch_p<MODE_WENO, AMR>(P, p, grid, s);
        case MODE_HYBRID: return launch_p<MODE_HYBRID, AMR>(P, p, grid, s);
        case MODE_CENTRAL: return launch_p<MODE_CENTRAL, AMR>(P, p, grid, s);
        default: return cudaErrorInvalidValue;
    }
}
cudaError_t five_sweep_launch_fast(int P, int mode, const FiveSweepParams& p, dim3 grid, cudaStream_t s) {
    return launch<false>(P, mode, p, grid, s);
}
cudaError_t five_sweep_launch_amr_fast(int P, int mode, const FiveSweepParams& p, dim3 grid, cudaStream_t s) {
    return launch<true>(P, mode, p, grid, s);
}

template <int P, int MODE, bool AMR> static cudaError_t attr_d() {
    const int b = (int)FiveSmem<P, MODE>::bytes();
    cudaError_t e = cudaFuncSetAttribute(five_fast_sweep_kernel<P, 0, MODE, AMR>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(five_fast_sweep_kernel<P, 1, MODE, AMR>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(five_fast_sweep_kernel<P, 2, MODE, AMR>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    return e;
}
template <int MODE> static cudaError_t attr_p() {
    cudaError_t e = attr_d<8, MODE, false>();
    if (e == cudaSuccess) e = attr_d<16, MODE, false>();
    if (e == cudaSuccess) e = attr_d<32, MODE, false>();
    if (e == cudaSuccess) e = attr_d<16, MODE, true>();
    if (e == cudaSuccess) e = attr_d<32, MODE, true>();
    return e;
}
cudaError_t five_sweep_prepare_fast() {
    cudaError_t e = attr_p<MODE_WENO>();
    if (e == cudaSuccess) e = attr_p<MODE_HYBRID>();
    if (e == cudaSuccess) e = attr_p<MODE_CENTRAL>();
    return e;
}

}  // namespace emg
