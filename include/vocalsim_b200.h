/*
 * vocalsim_b200.h -- C ABI of the B200 2.5D FDTD vocal-tract solver.
 *
 * The reference project (Debasishray19/VocalSim-2p5D-FDTD) exposes its time
 * stepping path as C++ classes: SimulationParams -> FDTDSolver::setupWaveSolver
 * -> FDTDEngineCPU / FDTDEngineEigen::startSolverEngine.  This header is the
 * plain-C boundary that replaces that path.  Every entry point below names the
 * reference interface it stands in for (file:line inside the reference tree).
 *
 * Conventions
 *   - Every function returns a vs_status (0 = ok).  vs_last_error() gives text.
 *   - The caller owns every host buffer passed in; a solver/batch handle owns
 *     its device memory.  One handle must not be used from two host threads at
 *     once; distinct handles are independent.
 *   - Frame arrays are row-major frameH x frameW (row 0 = top, as in the
 *     reference's PV_N[row * frameW + col]).
 *   - Nothing here falls back to the CPU: when no CUDA device is present the
 *     device entry points return VS_ERR_CUDA.  vs_build_maps() is host-only.
 */
#ifndef VOCALSIM_B200_H_
#define VOCALSIM_B200_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VS_ABI_VERSION 1

typedef enum vs_status {
    VS_OK               = 0,
    VS_ERR_INVALID_ARG  = 1,  /* bad pointer, size or enum value                 */
    VS_ERR_GEOMETRY     = 2,  /* area function unusable (empty, area <= 0, ...)  */
    VS_ERR_CUDA         = 3,  /* CUDA runtime / launch error, or no device       */
    VS_ERR_TIMEOUT      = 4,  /* a bounded device wait gave up                   */
    VS_ERR_NONFINITE    = 5,  /* NaN/Inf detected in the listener trace          */
    VS_ERR_ALLOC        = 6,  /* host or device allocation failed                */
    VS_ERR_UNSUPPORTED  = 7,  /* option outside the implemented scope            */
    VS_ERR_NEGATIVE_SQRT= 8   /* depth formula met a negative radicand; the
                                 reference traps here (TubeDepth.cu:273-288)     */
} vs_status;

/* Cell type codes, identical to the reference enum CellTypes
 * (include/SolverParams.h:21-35). */
enum {
    VS_CELL_WALL = 0, VS_CELL_AIR = 1, VS_CELL_EXCITATION = 2,
    VS_CELL_PML0 = 3, VS_CELL_PML1 = 4, VS_CELL_PML2 = 5, VS_CELL_PML3 = 6,
    VS_CELL_PML4 = 7, VS_CELL_PML5 = 8, VS_CELL_DYNAMIC = 9, VS_CELL_DEAD = 10,
    VS_CELL_NOPRESSURE = 11, VS_CELL_HEAD = 12
};

/* Source types, as FDTDSolver::source_type (FDTDSolver.cu:80,
 * GlottalExcitations.cu:17-44).  VS_SRC_GAUSS_STD is an addition: the same
 * Gaussian written with a standard deviation, exp(-(t-tp)^2 / (2 s^2)). */
enum { VS_SRC_SINE = 0, VS_SRC_GAUSS = 1, VS_SRC_TMM = 2, VS_SRC_GAUSS_STD = 3 };

/* Engine arithmetic.  Both reference engines run the same update; they round
 * the pressure denominator differently: FDTDEngineCPU.cpp:330 uses
 * (1 + sigma) * dP, FDTDEngineEigen.cpp:251 uses sigma * dP + dP. */
enum { VS_ENGINE_CPU = 1, VS_ENGINE_EIGEN = 2 };

/* Listener placement. */
enum { VS_LISTENER_REFERENCE = 0, VS_LISTENER_EXPLICIT = 1 };

/* Run parameters.  Replaces SimulationParams(10 args) (SimulationParams.cu:36-57)
 * plus the constants the reference hard-codes (SimulationParams.cu:7-34,
 * GlottalExcitations.cu:19-32, TwoMassModel.cpp:52, FDTDSolver.cu:614).
 * vs_params_init() fills every field with the reference's value. */
typedef struct vs_params {
    int32_t fdtd_solver_type;      /* 0 = 2D, 1 = 2.5D                                   */
    int32_t simulation_type;       /* 0 = open space (43 x 341 domain), 1 = tube         */
    int32_t cross_sectional_shape; /* 1 = circular, 2 = elliptical 3:1, 3 = single-plane   */
                                   /* symmetric (ShapeGenerator.cpp:35-197; host build)  */
    int32_t mouth_radiation_cond;  /* 0 = open end, 1 = Dirichlet p = 0 column           */
    int32_t srate_mul;             /* fs = 44100 * srate_mul                             */
    int32_t source_type;           /* VS_SRC_*                                           */
    int32_t pml_flag;              /* 0 = off, 1 = six graded PML layers                 */
    int32_t engine;                /* VS_ENGINE_*                                        */
    float   audio_dur;             /* seconds; sets num_steps when num_steps <= 0        */
    int32_t pad0;
    int64_t num_steps;             /* > 0: explicit step count (overrides audio_dur)     */
    /* sources */
    float   gauss_peak_s;          /* reference: 0.646f / 10 kHz                          */
    float   gauss_width_s;         /* reference form: width w in exp(-((t-tp)/w)^2)       */
    float   gauss_amp;             /* reference: 0.025                                    */
    float   sine_freq_hz;          /* reference: 440                                      */
    float   sine_amp;              /* reference: 25                                       */
    float   tmm_ps_pa;             /* two-mass subglottal pressure; reference 686.46      */
    /* walls */
    float   mu3d;                  /* wall reflection parameter; <= 0 -> reference value
                                      (0.025 in 2.5D, 0.005 in 2D; FDTDSolver.cu:614)   */
    float   wall_coupling;         /* wall_pressure_coupling_coeff; reference 0          */
    /* depth */
    float   uniform_depth_m;       /* > 0: tube air cells get this depth before the
                                      reference smoothing / clamp                        */
    int32_t depth_fma;             /* 1: circular depth radicand r^2 - d^2 as one fused
                                      multiply-add, as nvcc contracts the reference
                                      kernel (TubeDepth.cu:355-370); 0: two roundings    */
    /* listener */
    int32_t listener_mode;         /* VS_LISTENER_*                                      */
    int32_t listener_x, listener_y;/* used when listener_mode == VS_LISTENER_EXPLICIT    */
    /* two-mass precision (no counterpart in the reference) */
    int32_t tmm_f64;               /* 0: the reference's float model (TwoMassModel.h:18-
                                      60 members), bit-exact with it; 1: the same
                                      equations in double, fields stay FP32.  The float
                                      model's displacement update loses digits at
                                      fs = 661.5 kHz and drifts from its double
                                      restatement (0.2% rel-L2 of the flow by 2000
                                      steps); the double model tracks it to ~1e-8.    */
    /* arithmetic (no counterpart in the reference) */
    int32_t fast_math;             /* 0: the reference's expressions and rounding (traces
                                      equal the FP32 engine's); 1: reciprocal form --
                                      (P - K1 S / dP) / (1 + sigma) with a 1-ulp
                                      reciprocal, and the velocity denominators as
                                      correctly rounded table reciprocals -- for the
                                      quad-strip kernels (no coupled wall).  Every tube
                                      of a batch must use the same value.            */
    int32_t reserved[6];
} vs_params;

/* Area function: n sections of (length cm, area cm^2), the pairs the reference
 * reads from the data/tube-geometry text files (TubeGeometry.cu:83-88). */
typedef struct vs_geometry {
    int32_t      n_sections;
    int32_t      pad0;
    const float* section_length_cm;
    const float* section_area_cm2;
} vs_geometry;

/* Everything about a built grid that a caller needs to size buffers. */
typedef struct vs_dims {
    int32_t frame_h, frame_w;        /* FDTDSolver::frameH / frameW                     */
    int32_t listener_x, listener_y;  /* FDTDSolver::listenerX / listenerY               */
    int32_t excitation_x, excitation_y;
    int32_t tube_length_cells;       /* TubeGeometry::tube_length_incells (0 open space)*/
    int32_t tube_start_x, tube_end_x, tube_mid_y;
    int64_t num_steps;               /* FDTDSolver::num_steps                           */
    int64_t interior_cells;          /* (frameH-2) * (frameW-2)                         */
    float   dt, ds;                  /* SimulationParams::dt / ds                       */
    float   z_inv_val;               /* FDTDSolver.cu:617                               */
    int32_t pad0;
} vs_dims;

typedef struct vs_solver vs_solver;
typedef struct vs_batch  vs_batch;

/* Library version (VS_ABI_VERSION). */
int vs_version(void);

/* Fill *p with the reference's defaults: 2.5D, tube, circular, open mouth,
 * srate_mul 15, Gaussian source, PML on, FDTDEngineCPU arithmetic, 100 ms
 * (main.cu:160-187 uses 100 ms; reference source constants from
 * GlottalExcitations.cu:19-32 and TwoMassModel.cpp:52). */
int vs_params_init(vs_params* p);

/* Host-only: build the grid maps that FDTDSolver::setupWaveSolver produces
 * (FDTDSolver.cu:289-476: TubeGeometry.cu:53-612, TubeDepth.cu:95-762,
 * FDTDSolver.cu:553-649,816-857,1058-1070).  Any output pointer may be NULL.
 * cell_type, depth_* and z_inv are frameH*frameW arrays; call once with all
 * NULL to learn the dims.  cell_type matches the reference's GridCellComponents
 * ::cell_type values; depths match depthP/X/Y; z_inv matches the z_inv map. */
int vs_build_maps(const vs_params* p, const vs_geometry* g, vs_dims* dims,
                  int32_t* cell_type, float* depth_p, float* depth_x,
                  float* depth_y, float* z_inv);

/* Host-only: the tube rasterisation behind the maps, for tube simulations.
 * upper_wall / lower_wall / column_segment have tube_length_cells entries
 * (TubeGeometry::upper_wall_pos / lower_wall_pos, TubeGeometry.cu:197-199,
 * and the segment id the depth kernel uses per column, TubeDepth.cu:417);
 * major_axis_m / minor_axis_m have n_sections entries (the section widths and
 * the elliptical minor axes, TubeGeometry.cu:316-364; minor 0 for circles).
 * Any pointer may be NULL. */
int vs_tube_layout(const vs_params* p, const vs_geometry* g, vs_dims* dims, int32_t* upper_wall,
                   int32_t* lower_wall, int32_t* column_segment, float* major_axis_m, float* minor_axis_m);

/* Host-only: the per-step excitation table of GlottalExcitations::
 * setExcitationVelocity (GlottalExcitations.cu:9-52); zeros for the two-mass
 * source, whose velocity is computed on the device each step. */
int vs_source_table(const vs_params* p, int64_t num_steps, float* out);

/* Build the grid and place it on the current CUDA device.  Replaces
 * FDTDSolver(SimulationParams) + setupWaveSolver() + the engine constructor
 * (FDTDSolver.cu:71-83,289-476; FDTDEngineCPU.cpp:4-103).  State starts at
 * zero, as GridCellComponents initValue (FDTDSolver.cu:569). */
int vs_create(const vs_params* p, const vs_geometry* g, vs_solver** out);

/* Dims of a created solver. */
int vs_get_dims(const vs_solver* s, vs_dims* dims);

/* Advance `steps` time steps from the current state and write the listener
 * pressure of each step to `trace` (a device pointer when trace_on_device is
 * nonzero, else host memory).  Replaces FDTDEngineCPU::startSolverEngine
 * (FDTDEngineCPU.cpp:222-304) and FDTDEngineEigen::startSolverEngine
 * (FDTDEngineEigen.cpp:121-189); record_pressure[t] == trace[t]. */
int vs_run(vs_solver* s, int64_t steps, float* trace, int trace_on_device);

/* Zero the fields and the two-mass state and restart at step 0. */
int vs_reset(vs_solver* s);

/* Copy the current P, Vx, Vy frames (frameH*frameW floats each) to host
 * buffers; NULL skips a field.  Stands in for the PV_N readback the reference
 * uses for validation (FDTDEngineCPU.cpp:500-531). */
int vs_get_fields(const vs_solver* s, float* p, float* vx, float* vy);

/* Use this CUDA stream (a cudaStream_t) for every later call on s; NULL means
 * the handle's own stream. */
int vs_set_stream(vs_solver* s, void* cuda_stream);

/* Release device memory and the handle.  Replaces FDTDEngineCPU::freeCUDAMemory
 * (FDTDEngineCPU.cpp:199-219). */
void vs_destroy(vs_solver* s);

/* ---- batches: many independent tubes in one launch sequence ------------- */

/* Build n tubes (params[i], geoms[i]) and pack them into one device arena.
 * No reference counterpart: the reference runs one tube per process
 * (main.cu:203-232). */
int vs_batch_create(int32_t n, const vs_params* params, const vs_geometry* geoms,
                    vs_batch** out);

/* Dims of tube i of a batch. */
int vs_batch_get_dims(const vs_batch* b, int32_t i, vs_dims* dims);

/* Advance every tube `steps` time steps; traces is n x steps, row i = tube i.
 * Each row equals what vs_run gives for that tube alone. */
int vs_batch_run(vs_batch* b, int64_t steps, float* traces, int traces_on_device);

/* Zero all fields and restart every tube at step 0. */
int vs_batch_reset(vs_batch* b);

/* Use this CUDA stream (a cudaStream_t) for every later call on b; NULL means
 * the handle's own stream. */
int vs_batch_set_stream(vs_batch* b, void* cuda_stream);

/* Select the tile shape used by the step kernel (index into the compiled
 * shape table, see vs_tile_shape) or -1 for the default choice.  The last
 * shape of the table is the cluster kernel: each tube of a batch without the
 * coupled wall oscillator (up to 64 tubes, each with at least one interior
 * row per CTA) keeps its state on its own thread-block cluster (up to 16
 * CTAs, one band of rows each, halo rows exchanged through distributed shared
 * memory; the configuration sized for the largest frame) and runs every step
 * of a vs_batch_run / vs_run call in one launch.  It is the default for a
 * single tube, and for a batch whose clusters are all resident at once. */
int vs_batch_set_tile(vs_batch* b, int32_t tile_index);

/* Device time of the last vs_batch_adjoint call, split into the segments'
 * recomputation (history-capturing forward steps) and the reverse steps
 * (ms, CUDA events).  No counterpart in the reference. */
int vs_batch_adjoint_times(const vs_batch* b, float* recompute_ms, float* reverse_ms);

/* Kernel form of the reverse steps of vs_batch_adjoint, no counterpart in the
 * reference: 0 = automatic (the default): form 2 for a batch of table-source
 * tubes large enough to give every SM four strips, else form 1;
 * 1 = 32 x 8 tiles with mu in shared memory, one reverse step per launch;
 * 2 = row-marching warp strips (two columns per lane) running two reverse
 * steps per launch, which reads and writes the adjoint planes and the
 * gradient accumulators once per two steps; a batch with a two-mass tube
 * runs it as form 3 (the two-mass reverse step runs beside every step);
 * 3 = the same strips, one reverse step per launch.  All forms compute the
 * same transposed step; they differ only in float rounding. */
int vs_batch_set_adjoint_form(vs_batch* b, int32_t form);

/* Rows per warp strip of the strip forms: 4, 8 or 16, or 0 (the default: 8
 * for form 2, 4 for form 3).  No counterpart in the reference. */
int vs_batch_set_adjoint_rows(vs_batch* b, int32_t rows);

/* Failure-path hook, no counterpart in the reference: the number of polls a
 * kernel's wait for its bulk row copies (band and staged quad-strip shapes)
 * makes before it gives up, and the run returns VS_ERR_TIMEOUT with the
 * state not valid; 0 restores the default (2^22).  A kernel that gives up
 * still waits, with the default limit, for its own copies in flight before it
 * exits.  Tests lower it to drive the timeout path without a fault. */
int vs_batch_set_wait_limit(vs_batch* b, uint32_t polls);

/* Time every compiled tile shape on `steps` steps and keep the fastest.  The
 * state is reset afterwards.  best_index / best_ms may be NULL. */
int vs_batch_autotune(vs_batch* b, int64_t steps, int32_t* best_index, float* best_ms);

/* Number of compiled tile shapes, and the rows x cols of shape i (0 x 0 for
 * the cluster shape, the last one). */
int vs_tile_shape_count(void);
int vs_tile_shape(int32_t i, int32_t* rows, int32_t* cols);

/* Time steps one kernel launch of shape i advances: 1, or 2 for the two-step
 * shapes (fast_math batches without the coupled wall; they keep a third set
 * of state planes and a third two-mass state slot beside the two parity sets),
 * or 0 for the cluster shape (all the steps of a run in one launch). */
int vs_tile_shape_steps(int32_t i, int32_t* steps_per_launch);

void vs_batch_destroy(vs_batch* b);

/* Formants of listener traces on the device: for each of n_traces traces of
 * n samples (device, row-major) at sampling rate fs, the first num_formants
 * spectral peaks as the reference's get_formants_bw computes them
 * (results/formants_bandwidths.py:5-80: level = 10 log10 |FFT|^2, df =
 * fs / (n - 1), -3 dB crossings by numpy.interp).  out (device, doubles) =
 * n_traces x [bandwidth Hz, centre Hz, peak dB] x num_formants, zeros where
 * fewer peaks exist.  Uses cuFFT (double); allocates its work buffers and
 * returns after the work on cuda_stream (a cudaStream_t; NULL = default) is
 * done. */
int vs_formants(const float* traces, int32_t n_traces, int64_t n, double fs, int32_t num_formants, double* out,
                void* cuda_stream);

/* WAV samples of listener traces on the device, as results/generate_audio.py
 * (lines 14-42) makes them from recorded-pressure.txt: each trace divided by
 * its largest |P| and clipped to [-1, 1]; for srate_mul > 1 low-passed by the
 * 2nd-order Butterworth filter at 5050 Hz (vs_audio_filter) with
 * scipy.signal.lfilter's direct form II transposed recursion in double, and
 * every srate_mul-th sample kept.  traces: device, n_traces x n floats; out:
 * device, n_traces x ceil(n / srate_mul) floats (the 44100 Hz WAV samples).
 * Returns after the work on cuda_stream (a cudaStream_t; NULL = default). */
int vs_audio(const float* traces, int32_t n_traces, int64_t n, int32_t srate_mul, float* out, void* cuda_stream);

/* The filter vs_audio applies for srate_mul (scipy.signal.butter(2, 5050 /
 * (44100 srate_mul / 2)) coefficients, a[0] = 1); host only. */
int vs_audio_filter(int32_t srate_mul, double* b3, double* a3);

/* ---- gradients: checkpointed forward + reverse-time discrete adjoint -----
 * No counterpart in the reference (it has no differentiation).  The adjoint
 * covers table sources (Gaussian, sine) and the two-mass source (whose flow
 * depends on the pressure at the excitation point) without wall coupling;
 * the coupled wall oscillator returns VS_ERR_UNSUPPORTED. */

/* Replace tube i's depth maps (frameH*frameW each, NULL keeps one) and its
 * z_inv value; cell types stay.  Invalidates stored checkpoints. */
int vs_batch_set_maps(vs_batch* b, int32_t tube, const float* depth_p, const float* depth_x,
                      const float* depth_y, float z_inv);

/* The maps tube i steps with, read back from the device (frameH*frameW each,
 * host buffers, NULL skips one), in the layout of vs_build_maps: cell types,
 * depth_p / depth_x / depth_y and the z_inv map.  Circular and elliptical
 * tube sections are painted on the device at vs_batch_create (the batched map
 * builder, FDTDSolver::setupWaveSolver's setup kernels restated); the
 * open-space domain and single-plane-symmetric sections are built on the
 * host.  Either way the values are vs_build_maps's bit for bit. */
int vs_batch_get_maps(const vs_batch* b, int32_t tube, int32_t* cell_type, float* depth_p, float* depth_x,
                      float* depth_y, float* z_inv);

/* vs_get_fields for tube i of a batch: its current P, Vx, Vy frames
 * (frameH*frameW floats each, host buffers, NULL skips one). */
int vs_batch_get_fields(const vs_batch* b, int32_t tube, float* p, float* vx, float* vy);

/* Forward `steps` steps from rest, keeping a state checkpoint every
 * ckpt_every steps for vs_batch_adjoint; traces (host, n x steps) may be NULL. */
int vs_batch_forward_ckpt(vs_batch* b, int64_t steps, int32_t ckpt_every, float* traces);

/* Gradients of a loss L(traces) given dL/dtrace (host, n x steps of the last
 * vs_batch_forward_ckpt): per-cell dL/d depth_p, depth_x, depth_y (host, the
 * tubes' frames concatenated) and dL/d z_inv per tube (n).  Each segment of
 * ckpt_every steps is recomputed from its checkpoint, then stepped backwards.
 * Any output pointer may be NULL. */
int vs_batch_adjoint(vs_batch* b, const float* dL_dtrace, float* grad_depth_p, float* grad_depth_x,
                     float* grad_depth_y, float* grad_z_inv);

/* The same two calls with the traces and dL/dtrace in device memory (n x
 * steps floats), so a loss computed on the GPU (the spectral loss of the
 * inversion) feeds the adjoint without a host round trip; the per-cell
 * gradient outputs stay host buffers.  The work runs on the batch's stream
 * (vs_batch_set_stream): put the caller's loss kernels on the same stream. */
int vs_batch_forward_ckpt_device(vs_batch* b, int64_t steps, int32_t ckpt_every, float* traces);
int vs_batch_adjoint_device(vs_batch* b, const float* dL_dtrace, float* grad_depth_p, float* grad_depth_x,
                            float* grad_depth_y, float* grad_z_inv);

/* Depth maps of every tube from section parameters, computed on the device:
 * the reference's elliptical depth kernel and post-processing
 * (TubeDepth.cu:392-490, 642-762) on each tube's nominal rasterisation (the
 * wall rows stay where the nominal widths put them; a section's width
 * scales the semi-major axis of its cells, its depth the minor axis).
 * width_m, depth_m: the tubes' sections concatenated in tube order (m);
 * z_inv: one value per tube (NULL keeps them).  2.5D 3:1 elliptical tubes
 * only.  Invalidates stored checkpoints. */
int vs_batch_set_sections(vs_batch* b, const double* width_m, const double* depth_m, const double* z_inv);

/* dL/d width and dL/d depth of every section (host, concatenated like
 * vs_batch_set_sections), from the map gradients of the last
 * vs_batch_adjoint run on maps set by vs_batch_set_sections. */
int vs_batch_section_gradients(vs_batch* b, double* grad_width, double* grad_depth);

/* ---- running without allocating ------------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * when they step a tube: a real-time audio host calling from its processing
 * thread, where an allocation may block for an unbounded time, or an
 * application whose device memory is reserved by another allocator, so a
 * direct cudaMalloc can fail.  The caller passes device buffers it already
 * owns: the H x W maps of vs_build_maps (cell_type, depth_p/x/y, z_inv), the
 * excitation table of vs_source_table (>= steps entries; NULL for the
 * two-mass source), the dims vs_build_maps returned, and a device trace of
 * `steps` floats.  The listener trace equals what vs_run gives for the same
 * tube.  Everything else lives in a 16 MiB static device array that every
 * GPU loading the library holds until exit; a frame larger than it (about
 * 37 bytes x H x roundup(W, 32)) is rejected with VS_ERR_INVALID_ARG, and so
 * are listener or excitation cells outside the frame's interior
 * (1..W-2 x 1..H-2).  The maps stay on the device, so they are checked there:
 * a cell_type outside 0..12 is run as a dead cell and the whole trace is
 * returned as NaN.  The call allocates nothing and returns once the work is
 * queued on cuda_stream (a cudaStream_t; NULL = default stream); synchronise
 * the stream before reading the trace.  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress) and keeps it for the
 * life of the process, so make that call before any stream capture, and do
 * not use this entry point across a cudaDeviceReset of that device.  Calls
 * share the array: it is re-initialised on every call, and calls whose work
 * overlaps on the GPU race on it. */
int vs_run_noalloc(const vs_params* p, const vs_dims* dims, const int32_t* cell_type,
                   const float* depth_p, const float* depth_x, const float* depth_y,
                   const float* z_inv, const float* source, int64_t steps, float* trace,
                   void* cuda_stream);

/* Last error text of this host thread (never NULL). */
const char* vs_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* VOCALSIM_B200_H_ */
