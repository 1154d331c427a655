// Launchers of the fused sweep kernels (instantiated in sweep_f64.cu, which is
// compiled without FMA contraction so its f64 arithmetic rounds like the
// reference CPU solver, in sweep_mixed.cu, FP32 flux arithmetic, and in
// sweep_fast.cu, the fast FP64 form).
#pragma once
#include "sweep.cuh"

namespace emg {
// P = pencils per CTA (8, 16 or 32); mode = SweepMode. Returns the launch error.
cudaError_t sweep_launch_f64(int P, int mode, const SweepParams& p, dim3 grid, cudaStream_t s);
cudaError_t sweep_launch_mixed(int P, int mode, const SweepParams& p, dim3 grid, cudaStream_t s);
cudaError_t sweep_launch_fast(int P, int mode, const SweepParams& p, dim3 grid, cudaStream_t s);
// Batched block-AMR leaves (SweepParams::amr set), P = 16 or 32.
cudaError_t sweep_launch_amr_f64(int P, int mode, const SweepParams& p, dim3 grid, cudaStream_t s);
cudaError_t sweep_launch_amr_mixed(int P, int mode, const SweepParams& p, dim3 grid, cudaStream_t s);
cudaError_t sweep_launch_amr_fast(int P, int mode, const SweepParams& p, dim3 grid, cudaStream_t s);
// Batched independent 1-D lines (SweepParams::segs), 32 segments per CTA.
cudaError_t sweep_launch_batch_f64(int mode, const SweepParams& p, dim3 grid, cudaStream_t s);
cudaError_t sweep_launch_batch_mixed(int mode, const SweepParams& p, dim3 grid, cudaStream_t s);
cudaError_t sweep_launch_batch_fast(int mode, const SweepParams& p, dim3 grid, cudaStream_t s);
// 3-D uniform grids, WENO mode, P = 32: phase-A rows staged by TMA from the
// stage input described by `tm` (a 4-D map: k, j, i, field; box RM rows ×
// 32 lanes × 1 × 5 fields, the row axis being p.d). Resident CTAs per SM of
// that kernel (after the prepare call).
cudaError_t sweep_launch_tma_f64(const SweepParams& p, const CUtensorMap& tm, dim3 grid, cudaStream_t s);
cudaError_t sweep_launch_tma_mixed(const SweepParams& p, const CUtensorMap& tm, dim3 grid, cudaStream_t s);
int sweep_tma_ctas_per_sm_f64();
int sweep_tma_ctas_per_sm_mixed();
// Resident CTAs per SM of the uniform-grid sweep kernel (after the prepare call).
int sweep_ctas_per_sm_f64(int P, int mode);
int sweep_ctas_per_sm_mixed(int P, int mode);
int sweep_ctas_per_sm_fast(int P, int mode);
// Opt the kernels into their dynamic shared memory size (once per device).
cudaError_t sweep_prepare_f64();
cudaError_t sweep_prepare_mixed();
cudaError_t sweep_prepare_fast();
// Both forms' opt-ins for the current device, done once per device; safe to
// call from several host threads.
cudaError_t sweep_prepare_device();
}  // namespace emg
