// Internal interface of the uniform-grid solver (uniform.cu), shared with the
// discrete adjoint (adjoint.cu), which drives the same forward stages with
// the limiter's blend weights recorded.
#pragma once
#include "../../include/emergence_b200.h"
#include "sweep_launch.h"

#include <cuda.h>

#include <string>
#include <vector>

namespace emg {

int set_error(int code, const std::string& msg);

#define EMG_CUDA(call)                                                                                 \
    do {                                                                                               \
        cudaError_t _e = (call);                                                                       \
        if (_e != cudaSuccess)                                                                         \
            return set_error(EMG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e));      \
    } while (0)

struct CellRange {
    int64_t n[3], g[3], stride[3];
    int64_t cells;
    __device__ int64_t index(int64_t t) const {
        const int64_t k = t % n[2];
        const int64_t j = (t / n[2]) % n[1];
        const int64_t i = t / (n[1] * n[2]);
        return (i + g[0]) * stride[0] + (j + g[1]) * stride[1] + (k + g[2]) * stride[2];
    }
};

__global__ void ctl_begin_host(StepCtl* ctl, double dt);
__global__ void ctl_begin_device(StepCtl* ctl, double cfl);
__global__ void ctl_end(StepCtl* ctl);

}  // namespace emg

struct emg_uniform {
    int device = 0;
    cudaStream_t stream = nullptr;
    emg_mesh mesh{};
    emg_eos eos{};
    emg_bc bc[6]{};
    emg_opts opts{};
    int64_t m[3]{}, stride[3]{}, ncell = 0, cells = 0;
    int active[3]{};
    int ndim = 0;
    bool deep = false;
    double* u = nullptr;
    double* sa = nullptr;
    double* sb = nullptr;
    double* rhs = nullptr;
    double* staging = nullptr;
    double* partial = nullptr;
    emg::StepCtl* ctl = nullptr;
    emg::StepCtl* ctl_host = nullptr;  // pinned mirror
    bool rate_valid = false;
    double t_host = 0.0;          // mirror of ctl->t when the device is idle
    uint64_t faces = 0, weno_faces = 0;  // host-side face counts
    uint64_t launches = 0;
    // profiling
    bool profiling = false;
    struct Rec {
        int kind;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
    double prof_ms[EMG_K_COUNT]{};
    uint64_t prof_n[EMG_K_COUNT]{};
    // sweep shapes per axis
    int sweepP[3]{}, sweepSeg[3]{};
    dim3 sweepGrid[3];
    int lane_axis[3]{}, other_axis[3]{};
    // when set (by the discrete adjoint), the sweeps of stage s along axis d
    // record the positivity limiter's blend weights into theta_rec[s-1][d]
    double* theta_rec[3][3]{};
    // TMA staging of the sweeps' row loads (3-D grids, WENO mode): a tensor
    // map of each stage input (u, sa, sb) per sweep axis; tma = 0 when the
    // grid does not qualify (see setup_tma)
    CUtensorMap tmap[3][3];
    int tma = 0;
};


namespace emg {
// ghost fill of `arr` (padded SoA) along every active axis, in axis order
int launch_ghosts(emg_uniform* h, double* arr);
// three SSP-RK3 stages and the time advance of one step (dt read from the control block)
int launch_step_body(emg_uniform* h);
// CFL rate of the current state into the control block, if not already there
int ensure_rate(emg_uniform* h);
// control block → host mirror (synchronizes the stream)
int sync_ctl(emg_uniform* h);
// null check and cudaSetDevice
int check_handle(emg_uniform* h);
// EMG_OK, or the error the device raised (status of the control block mirror)
int check_status(emg_uniform* h);
}  // namespace emg
