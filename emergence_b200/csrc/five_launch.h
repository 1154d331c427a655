// Launchers of the five-equation fused sweep for other translation units
// (the block-AMR solver), instantiated in five.cu (compiled without FMA
// contraction), and of its fast FP64 form, instantiated in five_fast.cu.
#pragma once
#include "five_sweep.cuh"

namespace emg {
// Batched block-AMR leaves (FiveSweepParams AMR fields set), P = 16 or 32;
// mode = SweepMode. Returns the launch error.
cudaError_t five_sweep_launch_amr(int P, int mode, const FiveSweepParams& p, dim3 grid, cudaStream_t s);
// Fast FP64 form: uniform grids (P = 8, 16 or 32) and block-AMR leaves (P = 16 or 32).
cudaError_t five_sweep_launch_fast(int P, int mode, const FiveSweepParams& p, dim3 grid, cudaStream_t s);
cudaError_t five_sweep_launch_amr_fast(int P, int mode, const FiveSweepParams& p, dim3 grid, cudaStream_t s);
cudaError_t five_sweep_prepare_fast();
// The sweeps' dynamic shared-memory opt-in for the current device (once per device).
cudaError_t five_sweep_prepare_device();
}  // namespace emg
