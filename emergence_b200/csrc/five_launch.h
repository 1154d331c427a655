// Launchers of the five-equation fused sweep for other translation units
// (the block-AMR solver), instantiated in five.cu (compiled without FMA
// contraction).
#pragma once
#include "five_sweep.cuh"

namespace emg {
// Batched block-AMR leaves (FiveSweepParams AMR fields set), P = 16 or 32;
// mode = SweepMode. Returns the launch error.
cudaError_t five_sweep_launch_amr(int P, int mode, const FiveSweepParams& p, dim3 grid, cudaStream_t s);
// The sweeps' dynamic shared-memory opt-in for the current device (once per device).
cudaError_t five_sweep_prepare_device();
}  // namespace emg
