// Launch interface of the adjoint sweep (adjoint.cu), shared by the uniform
// solver's adjoint and the batched-lines adjoint (batch1d.cu).
#pragma once
#include "physics.cuh"
#include <cuda_runtime.h>
#include <stdint.h>

namespace emg {

constexpr int ADJ_T = 256;                 // threads per CTA
constexpr int ADJ_P = 4;                   // pencils per CTA
constexpr int ADJ_L = ADJ_T / ADJ_P - 5;   // owned rows per pencil (one midpoint per thread: L + 5 = 64)
constexpr int ADJ_ROWS = ADJ_L + 10;       // staged rows per pencil
constexpr int ADJ_FACES = ADJ_L + 9;       // faces whose cotangents a CTA forms
// 2 CTAs per SM (128 registers, some spills) measured 10 % faster than 1 CTA
// per SM without spills on the 2-D explosion 512^2
constexpr int ADJ_MINB = 2;

struct AdjSweepParams {
    const double* __restrict__ u;      // stage input X_s, ghost-filled, SoA with field stride ncell
    const double* __restrict__ theta;  // recorded limiter blend weights of this stage and axis (null: none)
    const double* __restrict__ ybar;   // cotangent of the stage output (interior cells)
    double coef;                       // β_s·dt: ∂(stage output)/∂(residual)
    double* xbar;                      // cotangent of X_s, accumulated (ghost cells included)
    double* gpart;                     // per-CTA partial sums of the γ cotangent
    int64_t ncell;
    int64_t sd, sl, so;                // strides of the sweep, lane and other axes
    int nd, nl, no;                    // interior extents
    int gl, go;                        // ghost offsets of the lane and other axes
    int ng;
    double inv;                        // 1/dx along the sweep axis (the forward multiplies by it)
    EosD eos;
    // ---- batched independent lines (KIND 1): lane z of the launch is line
    // segment lanes[z]; each instance has its own cell size and time step
    const struct AdjLane* lanes;
    int nlanes;
    const double* inst_dx;
    const double* inst_dt;  // 0: the instance took no step here (its lanes are skipped)
    double beta;            // coef = beta·dt of the lane's instance
};

// A segment of a batched line: `base` is the flat index of the instance's
// padded row 0, `n` its interior cells, rows [c0, c0 + ADJ_L) are owned.
struct AdjLane {
    int64_t base;
    int n;
    int c0;
    int inst;
    int pad;
};

// One reverse sweep along axis d of a uniform grid (grid: lane tiles, row
// segments, other-axis rows).
cudaError_t adj_sweep_launch(int d, const AdjSweepParams& p, dim3 grid, cudaStream_t s);
// Batched independent 1-D lines: one launch over every lane of `p.lanes`.
cudaError_t adj_sweep_launch_batch(const AdjSweepParams& p, cudaStream_t s);

}  // namespace emg
