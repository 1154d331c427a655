/*
 * emergence_b200 — B200-native (sm_100a) compressible-Euler step: C ABI.
 *
 * This is the drop-in boundary for the explicit finite-volume step of the
 * emergence workspace's `compressible` crate (characteristic WENO5-Z / WCNS
 * reconstruction, HLLC flux, Hu–Adams–Shu positivity limiter, SSP-RK3
 * stages, ghost fill and the CFL max-wavespeed reduction). Each entry point
 * names the reference interface it replaces (paths relative to the
 * reference repository; `G/` = fluid/crates/compressible-cuda/src,
 * `C/` = fluid/crates/compressible/src).
 *
 * Conventions
 *  - Plain C types only: pointers, sizes, doubles, fixed-width integers.
 *  - Every function returns an `int` status: EMG_OK (0) or an EMG_ERR_* code.
 *    `emg_last_error()` returns a thread-local message for the last failure.
 *    Nothing aborts or traps.
 *  - Host state layout (what `create` takes and `download` returns) is the
 *    reference CPU layout: array-of-structures `double[len][5]` of conserved
 *    variables (ρ, ρu, ρv, ρw, E), ghost-padded with `ng` layers on active
 *    axes only, last axis contiguous: cell (i,j,k) (padded indices) sits at
 *    `(i*m1 + j)*m2 + k` with `m_d = n_d + 2 ng` on active axes, 1 otherwise
 *    (C/solver.rs:22-86).
 *  - A handle owns its device memory and one CUDA stream; caller buffers are
 *    only borrowed for the duration of a call. Handles are not thread-safe;
 *    distinct handles may be used concurrently from different threads.
 */
#ifndef EMERGENCE_B200_H
#define EMERGENCE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
enum emg_status {
    EMG_OK = 0,
    EMG_ERR_INVALID = 1,      /* invalid argument (null pointer, size mismatch, unsupported option) */
    EMG_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    EMG_ERR_DT_COLLAPSED = 3, /* time step not finite or ≤ 1e-12·|t_end| (C/solver.rs:763, G/lib.rs:447) */
    EMG_ERR_INADMISSIBLE = 4, /* non-finite or inadmissible state met by the CFL reduction */
    EMG_ERR_UNFILLABLE = 5,   /* AMR ghost cell with no source (G/kernels.cu:845-848) */
    EMG_ERR_BOUNDS = 6,       /* device-side bounds check failed */
    EMG_ERR_NO_DEVICE = 7,    /* no CUDA device of compute capability 10.x visible */
    EMG_ERR_TIMEOUT = 8       /* a bounded device-side wait ran out */
};

/* ------------------------------------------------------------------ types */
/* Noble–Abel stiffened-gas EOS (C/eos.rs:12-25). Ideal gas: p_inf = b = q = 0. */
typedef struct emg_eos {
    double gamma;
    double p_inf;
    double b;
    double q;
    double cv;
} emg_eos;

/* Uniform mesh (C/solver.rs:22-28): n cells per axis (1 = inactive axis),
 * lower corner, cell size, ghost layers (≥ 5 for the WCNS path). */
typedef struct emg_mesh {
    int64_t n[3];
    double lo[3];
    double dx[3];
    int64_t ng;
} emg_mesh;

/* Boundary conditions (C/solver.rs:8-20). `state` is the conserved
 * Dirichlet / far-field state (ignored by the other kinds). */
enum emg_bc_kind {
    EMG_BC_PERIODIC = 0,
    EMG_BC_OUTFLOW = 1, /* zero-gradient extrapolation (transmissive) */
    EMG_BC_REFLECT = 2,
    EMG_BC_DIRICHLET = 3,
    EMG_BC_CHARACTERISTIC = 4
};
typedef struct emg_bc {
    int32_t kind;
    int32_t reserved;
    double state[5];
} emg_bc;

/* Flux modes (C/scheme.rs:39-47). */
enum emg_flux_mode { EMG_MODE_HYBRID = 0, EMG_MODE_WENO = 1, EMG_MODE_CENTRAL = 2 };

/* Arithmetic of the flux evaluation. The conserved state, the RK stage
 * accumulation and the conservation sums are always f64. */
enum emg_precision {
    EMG_PRECISION_F64 = 0,  /* plain FP64 form: all scheme arithmetic in f64 */
    EMG_PRECISION_MIXED = 1, /* FP32 WENO-Z interpolation and HLLC wave-speed bounds; FP64 state, primitive
                                recovery, projections, HLLC and central fluxes (reciprocals to ~1e-12), limiter */
    EMG_PRECISION_F64_FAST = 2 /* fast FP64 form (every solver but the adjoint): all arithmetic in f64 with FMA
                                  contraction and Newton-refined reciprocals and square roots (about one ulp)
                                  in place of correctly rounded divisions; within 1e-12 relative L1 of the
                                  plain form instead of bitwise */
};

/* Scheme knobs mirroring the public fields of `Solver` (C/solver.rs:139-160). */
typedef struct emg_opts {
    double cfl;         /* CFL number (0.5 in the reference) */
    double tol;         /* hybrid sensor tolerance (1e-3) */
    int32_t mode;       /* emg_flux_mode */
    int32_t positivity; /* Hu–Adams–Shu limiter on/off (1) */
    int32_t precision;  /* emg_precision */
    int32_t flags;      /* EMG_OPT_* bits (0: none) */
} emg_opts;

/* emg_opts.flags: time the fused-sweep launch shapes (pencils per CTA, segment
 * length) of each axis on the initial state at creation and keep the fastest
 * (uniform grids; cached per mesh extents, flux mode and precision). Results
 * are the same for every shape. */
#define EMG_OPT_AUTOTUNE 1
/* emg_opts.flags, block AMR only: subcycling (Amr::subcycle, C/amr.rs:233-
 * 236). emg_amr_run_to then advances with emg_amr_dt_cfl_subcycled steps of
 * emg_amr_step_subcycled; emg_amr_step / emg_amr_dt_cfl keep the global
 * time step, as the reference's step / dt_cfl do. */
#define EMG_OPT_SUBCYCLE 2

/* ------------------------------------------------------------------ misc */

/* Message of the last failed call on this thread ("" if none). */
const char* emg_last_error(void);

/* Library version as "major.minor.patch". */
const char* emg_version(void);

/* Number of visible sm_100 devices. */
int emg_device_count(int* count);

/* Fingerprint of a ghost-padded AoS conserved state (host memory, host code:
 * no device needed): over the interior cells in (i, j, k) order and their 5
 * fields in order, h ← (h XOR bits(v))·0x100000001b3 from h = 0xcbf29ce484222325,
 * each value's IEEE-754 bits folded in whole. Equal states give equal
 * hashes; ghost layers do not enter. Replaces the `hash` of
 * fluid/crates/compressible/examples/cpu_validate.rs:7-22, which the
 * reference's CPU benchmark script uses to show that two builds agree bit for
 * bit. `len` counts cells and must equal the padded mesh. */
int emg_state_hash(const emg_mesh* mesh, const double* u_aos, size_t len, uint64_t* out);

/* ------------------------------------------------------------------ uniform grids */
typedef struct emg_uniform emg_uniform;

/* Upload a ghost-padded AoS conserved state and build a device solver on the
 * current CUDA device. Replaces `GpuSolver::<f64|f32>::from_cpu(&Solver,
 * GpuSystem::Euler(eos))` (G/lib.rs:184-282). `bc` is [axis][side] flattened
 * (6 entries); `len` counts cells (not doubles) and must equal the padded
 * cell count of `mesh`. Time starts at 0. */
int emg_uniform_create(const emg_mesh* mesh, const emg_eos* eos, const emg_bc bc[6], const emg_opts* opts,
                       const double* u_aos, size_t len, emg_uniform** out);

/* Free the handle and its device memory (Drop of GpuSolver). The five
 * state-sized arrays return to a library-owned stream-ordered pool per
 * device, which keeps up to 32 GB of freed memory so that the next
 * emg_uniform_create reuses it instead of calling the driver. */
int emg_uniform_destroy(emg_uniform* h);

/* Return the memory kept by the library's pools to the device (no Rust
 * counterpart: the reference frees through cudarc on drop). */
int emg_release_memory(void);

/* One SSP-RK3 step of size dt (G/lib.rs:402-412; C/solver.rs:659-738). */
int emg_uniform_step(emg_uniform* h, double dt);

/* CFL time step cfl / max_cells Σ_d (|u_d|+c)/dx_d (G/lib.rs:415-441; C/solver.rs:478-523). */
int emg_uniform_dt_cfl(emg_uniform* h, double* dt);

/* Advance to t_end with CFL steps (G/lib.rs:443-455; C/solver.rs:758-768).
 * The step count is written to *steps. Stops within 1e-10·|t_end| of t_end. */
int emg_uniform_run_to(emg_uniform* h, double t_end, uint64_t* steps);

/* Take `nsteps` CFL steps, each with dt = min(dt_cfl, t_end − t) computed on
 * the device (no host round trip per step), stopping early at t_end. Pass
 * t_end = +inf for a fixed number of steps. The number of steps actually
 * taken is written to *taken (may be NULL). New in this library: the
 * reference's `run_to` reads dt back to the host every step (G/lib.rs:430). */
int emg_uniform_advance(emg_uniform* h, uint64_t nsteps, double t_end, uint64_t* taken);

/* Download the full padded AoS state, ghosts included (G/lib.rs:457-461). */
int emg_uniform_download(emg_uniform* h, double* u_aos, size_t len);

/* Replace the device state by a padded AoS host state (time unchanged). */
int emg_uniform_upload(emg_uniform* h, const double* u_aos, size_t len);

/* Conserved totals Σ u·vol over interior cells (C/solver.rs:784-794), in f64. */
int emg_uniform_totals(emg_uniform* h, double out[5]);

/* Face statistics since creation: [faces, shock-path faces, first-order
 * fallbacks, positivity-limited faces] (C/scheme.rs:101-117; G/lib.rs:464-467
 * reports the last three). */
int emg_uniform_counters(emg_uniform* h, uint64_t out[4]);

/* Simulation time t (Solver::t). */
int emg_uniform_get_time(emg_uniform* h, double* t);
int emg_uniform_set_time(emg_uniform* h, double t);

/* Block until the handle's stream is idle (G/lib.rs:469-472). */
int emg_uniform_synchronize(emg_uniform* h);

/* The handle's CUDA stream (cudaStream_t) as an opaque pointer. */
int emg_uniform_stream(emg_uniform* h, void** stream);

/* Per-kernel CUDA-event timing of subsequent launches: on = 1 enables. Times
 * accumulate per kernel kind until read with emg_uniform_kernel_times. */
int emg_uniform_set_profiling(emg_uniform* h, int on);

/* Kernel kinds reported by emg_uniform_kernel_times. */
enum emg_kernel_kind {
    EMG_K_GHOST = 0,   /* ghost-layer fill, one launch per active axis per stage */
    EMG_K_AXIS_0 = 1,  /* fused WCNS/HLLC/limiter/divergence sweep along axis 0 */
    EMG_K_AXIS_1 = 2,
    EMG_K_AXIS_2 = 3,
    EMG_K_CFL = 4,     /* CFL reduction and device dt */
    EMG_K_COUNT = 5
};

/* Accumulated device milliseconds and launch counts per kernel kind since the
 * last call (synchronizes the stream; resets the accumulators).
 * `ms` and `launches` hold EMG_K_COUNT entries each. */
int emg_uniform_kernel_times(emg_uniform* h, double* ms, uint64_t* launches);

/* Number of kernel launches issued by the handle since creation. */
int emg_uniform_launch_count(emg_uniform* h, uint64_t* launches);

/* Device paths the handle uses, as EMG_FEATURE_* bits (no counterpart in the
 * reference). EMG_FEATURE_TMA: the fused sweeps receive each round's rows of
 * the stage input as a TMA bulk tensor copy (cp.async.bulk.tensor into shared
 * memory, issued a round ahead) instead of per-thread loads; used on 3-D grids
 * in WENO mode with ng and n2 even when EMG_TMA=1 is set in the environment
 * at creation (off by default: measured no faster on the B200). */
#define EMG_FEATURE_TMA 1u
int emg_uniform_features(emg_uniform* h, uint32_t* flags);

/* Largest padded cell count (m0·m1·m2) accepted by emg_uniform_step_noalloc. */
#define EMG_NOALLOC_MAX_CELLS 131072

/* One SSP-RK3 step of size dt on a uniform grid that allocates no memory:
 * no counterpart in the reference (its GpuSolver always owns device buffers).
 * For callers that cannot call cudaMalloc — code running where a framework or
 * an allocator owns all device memory, or between allocator-free phases — the
 * caller passes device pointers to the input and output states (SoA
 * u[q·ncell + cell], q = 0..4, the ghost-padded layout of emg_uniform_create)
 * and the library uses a fixed scratch area in its own static device memory
 * (3·5·EMG_NOALLOC_MAX_CELLS doubles plus a control block, ≈15.7 MB, held by
 * every GPU that loads the library until the process exits). u_in is read
 * only; u_out receives the new state with the ghost layers of the stage-1 fill.
 * The argument checks of emg_uniform_create apply; in addition grids above
 * EMG_NOALLOC_MAX_CELLS padded cells, u_in and u_out ranges that share any
 * byte, and a dt that is not finite and > 0 return EMG_ERR_INVALID before any
 * device work. The first call on a device sets kernel attributes (make it
 * before any stream capture); the scratch address is looked up again on every
 * call, so a device reset in between is harmless. All calls share the one
 * scratch area, so calls that overlap on the GPU (other streams, other host
 * threads) race; serialize them. Work is queued on `stream` (a cudaStream_t,
 * NULL for the legacy default stream) and the call does not synchronize. */
int emg_uniform_step_noalloc(const emg_mesh* mesh, const emg_eos* eos, const emg_bc bc[6], const emg_opts* opts,
                             const double* u_in, double* u_out, double dt, void* stream);

/* ------------------------------------------------------------------ five-equation system */
/* Two-phase flow with Kapila's five-equation model (C/multiphase.rs:1-392):
 * conserved variables (α1ρ1, α2ρ2, ρu, ρv, ρw, E, α1), primitive (α1ρ1, α2ρ2,
 * u, v, w, p, α1), one NASG equation of state per phase (`cv` unused).
 * `kapila` = 1 keeps the K∇·u term of the α1 equation (Wood's mixture sound
 * speed), 0 drops it (FiveEq::kapila, C/multiphase.rs:27-31). */
typedef struct emg_five_system {
    emg_eos eos[2];
    int32_t kapila;
    int32_t reserved;
} emg_five_system;

/* Boundary condition of a 7-variable system: as emg_bc with a conserved
 * Dirichlet / far-field state of 7 values. */
typedef struct emg_bc7 {
    int32_t kind;
    int32_t reserved;
    double state[7];
} emg_bc7;

typedef struct emg_five emg_five;

/* Upload a ghost-padded AoS state double[len][7] (the padded layout of
 * emg_uniform_create) and build a device solver of the five-equation system
 * on the current device: GpuSolver::from_cpu(&Solver<7, FiveEq>,
 * GpuSystem::FiveEq{..}) (G/lib.rs:184-282). Plain FP64 form (opts->precision
 * must be EMG_PRECISION_F64); every flux mode; boundaries periodic, outflow,
 * reflect (axes with n >= ng), Dirichlet and characteristic. */
int emg_five_create(const emg_mesh* mesh, const emg_five_system* sys, const emg_bc7 bc[6], const emg_opts* opts,
                    const double* u_aos, size_t len, emg_five** out);
int emg_five_destroy(emg_five* h);

/* One SSP-RK3 step of size dt (C/solver.rs:659-738; G/lib.rs:391-401). */
int emg_five_step(emg_five* h, double dt);

/* CFL step: min(cfl / max Σ_d (|u_d|+c)/dx_d, 0.5 / max dilatation rate)
 * over interior cells (C/solver.rs:478-523, C/multiphase.rs:363-377). */
int emg_five_dt_cfl(emg_five* h, double* dt);

/* Advance to t_end with CFL steps (C/solver.rs:758-768). */
int emg_five_run_to(emg_five* h, double t_end, uint64_t* steps);

/* The padded AoS state double[len][7], ghosts included (G/lib.rs:450-455). */
int emg_five_download(emg_five* h, double* u_aos, size_t len);

/* [faces, shock-path faces, first-order fallbacks, positivity-limited faces]. */
int emg_five_counters(emg_five* h, uint64_t out[4]);

/* Σ u·vol over interior cells (C/solver.rs:784-794), 7 values. */
int emg_five_totals(emg_five* h, double out[7]);

int emg_five_get_time(emg_five* h, double* t);

/* Kernel launches issued by the handle since creation. */
int emg_five_launch_count(emg_five* h, uint64_t* launches);

/* The handle's CUDA stream (cudaStream_t) as an opaque pointer. */
int emg_five_stream(emg_five* h, void** stream);

/* ------------------------------------------------------------------ batched 1-D lines */
/* Many independent 1-D problems advanced together: every RK stage is one
 * fused-sweep launch over all instances, each instance with its own cell size
 * and its own CFL time step. No counterpart in the reference, which solves one
 * Solver at a time (each instance here follows Solver::run_to,
 * C/solver.rs:758-768, on a 1-D mesh). */
typedef struct emg_batch1d emg_batch1d;

/* ninst instances; instance i has n[i] cells of size dx[i] and interior
 * conserved data u[(off_i + c)*5 + q] with off_i = Σ_{j<i} n[j]. The two
 * boundary conditions (low, high) are shared by all instances (periodic,
 * outflow, reflect or Dirichlet). ng = 6 ghost layers are added internally. */
int emg_batch1d_create(const emg_eos* eos, const emg_opts* opts, const emg_bc bc[2], size_t ninst, const int64_t* n,
                       const double* dx, const double* u, emg_batch1d** out);
int emg_batch1d_destroy(emg_batch1d* h);

/* Advance every instance to t_end with its own CFL steps (stopping rule and
 * collapse check of Solver::run_to). Steps run without host round trips;
 * *launched receives the number of batch steps issued (the step count of the
 * slowest instance). */
int emg_batch1d_run_to(emg_batch1d* h, double t_end, uint64_t* launched);

/* Interior conserved data of all instances (same layout as create). */
int emg_batch1d_download(emg_batch1d* h, double* u);

/* Per-instance time and step count. */
int emg_batch1d_status(emg_batch1d* h, double* t, uint64_t* steps);

/* The handle's CUDA stream (cudaStream_t) as an opaque pointer. */
int emg_batch1d_stream(emg_batch1d* h, void** stream);

/* Discrete adjoint of a batched run (no counterpart in the reference, which
 * has no adjoint; each instance is the 1-D Solver::step map, C/solver.rs:659-738).
 * Records a run of every instance to t_end from the initial state given at
 * creation (WENO mode), keeping the batch state every `checkpoint_every` batch
 * steps (0: 64); *batch_steps receives the number of batch steps. Time steps
 * and limiter blend weights are held fixed. An FP64 batch is differentiated
 * exactly; a mixed (FP32-flux) batch records its own run, and the backward
 * pass applies the transposed Jacobian of the FP64 step at the recorded
 * mixed stage states (the FP32 rounding is not differentiated). */
int emg_batch1d_record(emg_batch1d* h, double t_end, uint64_t checkpoint_every, uint64_t* batch_steps);

/* Per-instance box objective J_i on the recorded final state over cells with
 * centre (c+½)·dx_i in [x_lo, x_hi] (EMG_OBJ_PRESSURE: Σ p·dx, EMG_OBJ_ENERGY:
 * Σ E·dx); J receives ninst values. Seeds the backward pass. */
int emg_batch1d_objective(emg_batch1d* h, int kind, double x_lo, double x_hi, double* J);

/* Backward pass: grad6[6·i..] = ∂J_i/∂(ρ, u, p) of the initial primitive
 * state summed over the cells left of x_split, then right of it (for Riemann
 * problems, the gradient with respect to the six initial values); wbar, if
 * not NULL, receives ∂J/∂W⁰ per cell in the layout of create's u. */
int emg_batch1d_backward(emg_batch1d* h, double x_split, double* grad6, double* wbar);

/* Device milliseconds of the last recorded run, and of the last backward pass
 * split into checkpoint recompute and reverse sweeps. */
int emg_batch1d_adjoint_times(emg_batch1d* h, double ms[3]);

/* ------------------------------------------------------------------ block AMR */

/* Block-AMR configuration (C/amr.rs:49-63). Blocks are b cells per active
 * side; base_blocks[d] = 0 marks an inactive axis; ghosts ≥ 5 is enforced. */
typedef struct emg_amr_config {
    int64_t b;
    int64_t levels;
    double eps;
    int64_t regrid_every;
    int64_t base_blocks[3];
    int64_t ghosts;
} emg_amr_config;

/* Primitive initial condition: fills w[i*5 + 0..4] = (ρ,u,v,w,p) at the n cell
 * centres x[i*3 + 0..2]; called once per new block (the closure of
 * Amr::new, C/amr.rs:289). */
typedef void (*emg_init_fn)(void* ctx, const double* x, int64_t n, double* w);

typedef struct emg_amr emg_amr;

/* Build the hierarchy on the device like Amr::new (base blocks, then refine
 * on the initial data until the details are resolved, C/amr.rs:289-344) and
 * keep it there (GpuAmr::new, G/amr.rs:95-212). opts->cfl is the AMR CFL
 * number (0.4 in the reference). */
int emg_amr_create(const emg_amr_config* cfg, const emg_eos* eos, const double lo[3], const double hi[3],
                   const emg_bc bc[6], const emg_opts* opts, emg_init_fn init, void* ctx, emg_amr** out);

/* Adopt an existing hierarchy (what GpuAmr::new receives from a CPU Amr):
 * nblocks blocks with (level, i, j, k, leaf) in `desc[5*id..]` and conserved
 * block data `u[id][cell][5]` (b^D cells per block, no ghosts). */
int emg_amr_create_from_blocks(const emg_amr_config* cfg, const emg_eos* eos, const double lo[3], const double hi[3],
                               const emg_bc bc[6], const emg_opts* opts, const int64_t* desc, size_t nblocks,
                               const double* u, emg_amr** out);

/* The five-equation two-phase system (Kapila's model, 7 conserved variables)
 * on the block hierarchy: GpuAmr::new with GpuSystem::FiveEq
 * (G/amr.rs:132-212) on an Amr<7, FiveEq> (C/amr.rs:289-344). `init` fills
 * 7 primitives (α1ρ1, α2ρ2, u, v, w, p, α1) per cell; Dirichlet states hold 7
 * conserved values; characteristic boundaries are not available; plain FP64
 * form only. Every other emg_amr_* call works on the handle, with 7 values
 * per cell in block data and totals. The block residual carries the α
 * equation's non-conservative term and the CFL step the dilatation limit
 * (C/amr.rs:1276-1279, 1426-1461). */
int emg_amr_create_five(const emg_amr_config* cfg, const emg_five_system* sys, const double lo[3], const double hi[3],
                        const emg_bc7 bc[6], const emg_opts* opts, emg_init_fn init, void* ctx, emg_amr** out);

/* Adopt an existing five-equation hierarchy: as emg_amr_create_from_blocks
 * with block data u[id][cell][7]. */
int emg_amr_create_five_from_blocks(const emg_amr_config* cfg, const emg_five_system* sys, const double lo[3],
                                    const double hi[3], const emg_bc7 bc[6], const emg_opts* opts,
                                    const int64_t* desc, size_t nblocks, const double* u, emg_amr** out);

/* Conserved variables per cell of the handle's system: 5 (Euler) or 7. */
int emg_amr_nv(emg_amr* h, int32_t* nv);

int emg_amr_destroy(emg_amr* h);

/* One global SSP-RK3 step of size dt, regridding when due (Amr::step,
 * C/amr.rs:1470-1512; GpuAmr::step, G/amr.rs:683-700). */
int emg_amr_step(emg_amr* h, double dt);

/* Global CFL step over the leaves (C/amr.rs:1409-1467; G/amr.rs:769-805). */
int emg_amr_dt_cfl(emg_amr* h, double* dt);

/* Advance to t_end (C/amr.rs:1639-1652): stops at t ≥ t_end(1 − 1e-14);
 * subcycled steps when the handle was created with EMG_OPT_SUBCYCLE. */
int emg_amr_run_to(emg_amr* h, double t_end, uint64_t* steps);

/* One subcycled step (Amr::step_subcycled, C/amr.rs:1912-1952): the coarsest
 * level holding leaves advances by dt, each finer level l by dt/2^(l-lmin)
 * with its ancestors, coarse ghost data interpolated linearly in time and
 * coarse–fine faces corrected from flux registers; then every ancestor is
 * restricted and the regrid schedule of subcycling applies. Coarse–fine
 * corrections of one cell are applied in the order direction, side (the
 * reference applies them in hash-map order). No counterpart on the
 * reference's GPU (G/amr.rs:140-142 refuses subcycling). */
int emg_amr_step_subcycled(emg_amr* h, double dt);

/* Level step of subcycling (Amr::dt_cfl_subcycled, C/amr.rs:1681-1692):
 * every level's CFL limit over its leaves and ancestors, scaled by 2^(l-lmin),
 * and the global limit at the finest leaf level. */
int emg_amr_dt_cfl_subcycled(emg_amr* h, double* dt);

/* Regrid now (C/amr.rs:1039-1046). */
int emg_amr_regrid(emg_amr* h);

/* Number of blocks (leaves and ancestors) and of leaves. */
int emg_amr_block_count(emg_amr* h, uint64_t* blocks, uint64_t* leaves);

/* Hierarchy: (level, i, j, k, leaf) per block in id order (Amr::structure,
 * C/amr.rs:1539-1541); `cap` blocks of room. */
int emg_amr_structure(emg_amr* h, int64_t* desc, size_t cap);

/* Block data u[id][cell][nv] of all blocks (GpuAmr::download, G/amr.rs:821-843). */
int emg_amr_download(emg_amr* h, double* u, size_t nblocks);

/* Σ u·vol over leaves (C/amr.rs:1991-2005), nv values. */
int emg_amr_totals(emg_amr* h, double* out);

/* [faces, shock-path faces, fallbacks, limited faces] since creation. */
int emg_amr_counters(emg_amr* h, uint64_t out[4]);

int emg_amr_get_time(emg_amr* h, double* t);

/* Steps taken so far (Amr::steps). */
int emg_amr_steps(emg_amr* h, uint64_t* steps);

int emg_amr_synchronize(emg_amr* h);

/* The handle's CUDA stream (cudaStream_t) as an opaque pointer. */
int emg_amr_stream(emg_amr* h, void** stream);

/* Per-phase device milliseconds since the last call:
 * [restrict, ghosts, fluxes, reflux+update, regrid] (GpuAmr::prof, G/amr.rs:111-116). */
int emg_amr_phase_times(emg_amr* h, double out[5]);

/* Kernel launches issued by the handle since creation. */
int emg_amr_launch_count(emg_amr* h, uint64_t* launches);

/* ------------------------------------------------------------------ discrete adjoint
 * Reverse-mode derivative of the uniform-grid FP64 step (WENO flux mode):
 * SSP-RK3, the WCNS/HLLC/positivity-limited flux divergence and the ghost
 * fill, with √N checkpointing of the forward run. No counterpart in the
 * reference, which only runs forward (its Solver::step, C/solver.rs:659-738,
 * is the map differentiated here). The recorded run's time steps, the
 * positivity limiter's blend weights and the admissibility fallbacks are held
 * fixed: the result is the gradient of the discrete map the forward run
 * applied. Host arrays use the AoS padded layout of emg_uniform_create. */
typedef struct emg_adjoint emg_adjoint;

/* Box objectives over interior cells whose centre lo + (i+½)dx lies in
 * [box_lo, box_hi] on every active axis. */
enum emg_objective {
    EMG_OBJ_PRESSURE = 0, /* J = Σ p·vol */
    EMG_OBJ_ENERGY = 1    /* J = Σ E·vol */
};

/* Differentiable solver from an initial conserved state (opts: FP64, WENO
 * mode; boundaries periodic, outflow, reflect or Dirichlet; n ≥ ng on every
 * active axis). */
int emg_adjoint_create(const emg_mesh* mesh, const emg_eos* eos, const emg_bc bc[6], const emg_opts* opts,
                       const double* u_aos, size_t len, emg_adjoint** out);
int emg_adjoint_destroy(emg_adjoint* h);

/* Replace the initial state (drops a recorded run). */
int emg_adjoint_set_initial(emg_adjoint* h, const double* u_aos, size_t len);

/* Record a forward run from the initial state: up to nsteps steps with the
 * CFL time step (as Solver::run_to, stopping at t_end; +inf for a fixed step
 * count), keeping the state every `checkpoint_every` steps (0: ⌈√nsteps⌉).
 * *taken receives the steps run. */
int emg_adjoint_forward(emg_adjoint* h, uint64_t nsteps, double t_end, uint64_t checkpoint_every, uint64_t* taken);

/* Record a forward run with the given time steps (frozen-dt runs, e.g. for
 * finite-difference checks). */
int emg_adjoint_forward_dts(emg_adjoint* h, const double* dts, uint64_t nsteps, uint64_t checkpoint_every);

/* Time steps of the recorded run (`cap` entries of room; out may be NULL to
 * query the count). */
int emg_adjoint_dts(emg_adjoint* h, double* out, size_t cap, uint64_t* nsteps);

/* Final state of the recorded run (the initial state if none). */
int emg_adjoint_download(emg_adjoint* h, double* u_aos, size_t len);

/* J of the recorded run's final state; seeds the backward pass with ∂J/∂U
 * and the direct ∂J/∂γ. */
int emg_adjoint_objective(emg_adjoint* h, int kind, const double box_lo[3], const double box_hi[3], double* J);

/* Seed the backward pass with a caller cotangent of the final conserved state. */
int emg_adjoint_seed(emg_adjoint* h, const double* ubar_aos, size_t len);

/* Backward pass (recomputing each checkpoint segment). Outputs, each optional:
 * ubar0 = ∂J/∂U⁰ (conserved initial state), wbar0 = ∂J/∂W⁰ (primitive initial
 * state, through U⁰ = to_cons(W⁰)), gamma_bar = [∂J/∂γ with U⁰ fixed, with W⁰
 * fixed]. Ghost entries of the arrays are zero. */
int emg_adjoint_backward(emg_adjoint* h, double* ubar0_aos, double* wbar0_aos, double gamma_bar[2]);

/* One step's vector–Jacobian product: for U' = step(U, dt), ubar = (∂U'/∂U)ᵀ·ubar_next
 * and *gamma_bar = (∂U'/∂γ)ᵀ·ubar_next. The differentiable-step primitive. */
int emg_adjoint_step_vjp(emg_adjoint* h, const double* u_aos, size_t len, double dt, const double* ubar_next_aos,
                         double* ubar_aos, double* gamma_bar);

/* Device milliseconds of the last forward run, and of the last backward pass
 * split into checkpoint recompute and reverse sweeps. */
int emg_adjoint_times(emg_adjoint* h, double ms[3]);

/* The handle's CUDA stream (cudaStream_t) as an opaque pointer. */
int emg_adjoint_stream(emg_adjoint* h, void** stream);

#ifdef __cplusplus
}
#endif

#endif /* EMERGENCE_B200_H */
