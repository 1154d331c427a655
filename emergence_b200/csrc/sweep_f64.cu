// Plain FP64 form of the fused sweep. Built with -fmad=false: every f64
// multiply and add is rounded separately, as in the reference CPU solver.
#include "sweep_launch.h"

namespace emg {

template <int P, int D, int MODE, int KIND = KIND_GRID>
__global__ void __launch_bounds__(SWEEP_THREADS, 4) sweep_f64_kernel(const SweepParams p) {
    Sweep<double, P, D, MODE, KIND>::run(p);
}

// batched block-AMR leaves: P = 16 or 32 pencils, one block per lane set
template <int P, int D, int MODE> static cudaError_t launch_amr(const SweepParams& p, dim3 grid, cudaStream_t s) {
    sweep_f64_kernel<P, D, MODE, KIND_AMR><<<grid, SWEEP_THREADS, SweepSmem<double, P, MODE>::bytes(), s>>>(p);
    return cudaGetLastError();
}
template <int P, int MODE> static cudaError_t launch_amr_d(const SweepParams& p, dim3 grid, cudaStream_t s) {
    return p.d == 0 ? launch_amr<P, 0, MODE>(p, grid, s) : (p.d == 1 ? launch_amr<P, 1, MODE>(p, grid, s) : launch_amr<P, 2, MODE>(p, grid, s));
}
template <int MODE> static cudaError_t launch_amr_p(int P, const SweepParams& p, dim3 grid, cudaStream_t s) {
    return P == 16 ? launch_amr_d<16, MODE>(p, grid, s) : (P == 32 ? launch_amr_d<32, MODE>(p, grid, s) : cudaErrorInvalidValue);
}
cudaError_t sweep_launch_amr_f64(int P, int mode, const SweepParams& p, dim3 grid, cudaStream_t s) {
    switch (mode) {
        case MODE_WENO: return launch_amr_p<MODE_WENO>(P, p, grid, s);
        case MODE_HYBRID: return launch_amr_p<MODE_HYBRID>(P, p, grid, s);
        case MODE_CENTRAL: return launch_amr_p<MODE_CENTRAL>(P, p, grid, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int P, int D, int MODE> static cudaError_t launch(const SweepParams& p, dim3 grid, cudaStream_t s) {
    sweep_f64_kernel<P, D, MODE><<<grid, SWEEP_THREADS, SweepSmem<double, P, MODE>::bytes(), s>>>(p);
    return cudaGetLastError();
}

template <int P, int MODE> static cudaError_t launch_d(const SweepParams& p, dim3 grid, cudaStream_t s) {
    return p.d == 0 ? launch<P, 0, MODE>(p, grid, s) : (p.d == 1 ? launch<P, 1, MODE>(p, grid, s) : launch<P, 2, MODE>(p, grid, s));
}

template <int MODE> static cudaError_t launch_p(int P, const SweepParams& p, dim3 grid, cudaStream_t s) {
    switch (P) {
        case 8: return launch_d<8, MODE>(p, grid, s);
        case 16: return launch_d<16, MODE>(p, grid, s);
        case 32: return launch_d<32, MODE>(p, grid, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t sweep_launch_f64(int P, int mode, const SweepParams& p, dim3 grid, cudaStream_t s) {
    switch (mode) {
        case MODE_WENO: return launch_p<MODE_WENO>(P, p, grid, s);
        case MODE_HYBRID: return launch_p<MODE_HYBRID>(P, p, grid, s);
        case MODE_CENTRAL: return launch_p<MODE_CENTRAL>(P, p, grid, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int P, int MODE> static cudaError_t attr_d() {
    cudaError_t e = cudaSuccess;
    const int b = (int)SweepSmem<double, P, MODE>::bytes();
    if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_f64_kernel<P, 0, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_f64_kernel<P, 1, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_f64_kernel<P, 2, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if constexpr (P >= 16) {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_f64_kernel<P, 0, MODE, KIND_AMR>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_f64_kernel<P, 1, MODE, KIND_AMR>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_f64_kernel<P, 2, MODE, KIND_AMR>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    }
    return e;
}

template <int MODE> static cudaError_t attr_p() {
    cudaError_t e = attr_d<8, MODE>();
    if (e == cudaSuccess) e = attr_d<16, MODE>();
    if (e == cudaSuccess) e = attr_d<32, MODE>();
    return e;
}

// batched independent 1-D lines along axis 0, P = 32 segments per CTA
template <int MODE> static cudaError_t launch_batch(const SweepParams& p, dim3 grid, cudaStream_t s) {
    sweep_f64_kernel<32, 0, MODE, KIND_BATCH><<<grid, SWEEP_THREADS, SweepSmem<double, 32, MODE>::bytes(), s>>>(p);
    return cudaGetLastError();
}
cudaError_t sweep_launch_batch_f64(int mode, const SweepParams& p, dim3 grid, cudaStream_t s) {
    switch (mode) {
        case MODE_WENO: return launch_batch<MODE_WENO>(p, grid, s);
        case MODE_HYBRID: return launch_batch<MODE_HYBRID>(p, grid, s);
        case MODE_CENTRAL: return launch_batch<MODE_CENTRAL>(p, grid, s);
        default: return cudaErrorInvalidValue;
    }
}

static cudaError_t tma_attr_f64();

cudaError_t sweep_prepare_f64() {
    cudaError_t e = attr_p<MODE_WENO>();
    if (e == cudaSuccess) e = attr_p<MODE_HYBRID>();
    if (e == cudaSuccess) e = attr_p<MODE_CENTRAL>();
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(sweep_f64_kernel<32, 0, MODE_WENO, KIND_BATCH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SweepSmem<double, 32, MODE_WENO>::bytes());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(sweep_f64_kernel<32, 0, MODE_HYBRID, KIND_BATCH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SweepSmem<double, 32, MODE_HYBRID>::bytes());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(sweep_f64_kernel<32, 0, MODE_CENTRAL, KIND_BATCH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SweepSmem<double, 32, MODE_CENTRAL>::bytes());
    if (e == cudaSuccess) e = tma_attr_f64();
    return e;
}

// 3-D uniform grids, WENO mode, 32 pencils per CTA: phase-A rows by TMA
template <int D>
__global__ void __launch_bounds__(SWEEP_THREADS, 3) sweep_f64_tma_kernel(const SweepParams p,
                                                                          const __grid_constant__ CUtensorMap tm) {
    Sweep<double, 32, D, MODE_WENO, KIND_GRID_TMA>::run(p, &tm);
}
static size_t tma_smem_f64() { return SweepSmem<double, 32, MODE_WENO>::bytes() + tma_stage_bytes<32>(); }
cudaError_t sweep_launch_tma_f64(const SweepParams& p, const CUtensorMap& tm, dim3 grid, cudaStream_t s) {
    const size_t b = tma_smem_f64();
    switch (p.d) {
        case 0: sweep_f64_tma_kernel<0><<<grid, SWEEP_THREADS, b, s>>>(p, tm); break;
        case 1: sweep_f64_tma_kernel<1><<<grid, SWEEP_THREADS, b, s>>>(p, tm); break;
        case 2: sweep_f64_tma_kernel<2><<<grid, SWEEP_THREADS, b, s>>>(p, tm); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}
static cudaError_t tma_attr_f64() {
    const int b = (int)tma_smem_f64();
    cudaError_t e = cudaFuncSetAttribute(sweep_f64_tma_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_f64_tma_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(sweep_f64_tma_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    return e;
}
int sweep_tma_ctas_per_sm_f64() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_f64_tma_kernel<2>, SWEEP_THREADS, tma_smem_f64()) !=
        cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// resident CTAs per SM of the uniform-grid sweep (the three axes share registers and shared memory)
template <int P, int MODE> static int occupancy() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_f64_kernel<P, 0, MODE>, SWEEP_THREADS,
                                                      SweepSmem<double, P, MODE>::bytes()) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return n > 0 ? n : 1;
}
template <int MODE> static int occupancy_p(int P) {
    return P == 8 ? occupancy<8, MODE>() : (P == 16 ? occupancy<16, MODE>() : occupancy<32, MODE>());
}
int sweep_ctas_per_sm_f64(int P, int mode) {
    return mode == MODE_HYBRID ? occupancy_p<MODE_HYBRID>(P)
                               : (mode == MODE_CENTRAL ? occupancy_p<MODE_CENTRAL>(P) : occupancy_p<MODE_WENO>(P));
}

}  // namespace emg
