/*
 * virs.h -- C ABI of the B200 implementation of the VIRS FDTD simulation path.
 *
 * One opaque handle (virs_sim) owns every device buffer of one simulation on
 * one GPU.  All entry points return a virs_status; none of them exits the
 * process or prints.  virs_last_error() gives the message of the last
 * failure on the calling thread.  Plain pointers and sizes only: host
 * buffers are read or written synchronously unless a call says otherwise.
 *
 * Layout of every voxel array exchanged through this ABI is the reference's:
 *   idx = (z * ny + y) * nx + x            (src/simulator/vectorspace.h:200-203)
 *
 * Each declaration names the reference interface it replaces, as
 * path:line in the Snipet/VIRS tree.
 */
#ifndef VIRS_H
#define VIRS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VIRS_ABI_VERSION 1

typedef enum virs_status {
    VIRS_OK = 0,
    VIRS_E_ARG = 1,      /* invalid argument: sizes, indices, ranges, order   */
    VIRS_E_OOM = 2,      /* device or host allocation failed                  */
    VIRS_E_CUDA = 3,     /* CUDA runtime error (message has the CUDA string)  */
    VIRS_E_UNSTABLE = 4, /* non-finite receiver sample or energy blow-up      */
    VIRS_E_TIMEOUT = 5,  /* a bounded device wait gave up                     */
    VIRS_E_STATE = 6,    /* call out of order (e.g. run before classify)      */
    VIRS_E_IO = 7        /* a file could not be read or parsed                */
} virs_status;

typedef struct virs_sim virs_sim;

/* pressure storage precision (updates are always FP32) */
enum { VIRS_STORAGE_F32 = 0, VIRS_STORAGE_F16 = 1, VIRS_STORAGE_BF16 = 2 };

/* boundary correction of flag-2 voxels.  REFERENCE is simulator_gpu.cu:148:
 * p+ -= K*g*w*(mix_filtered*y + mix_direct*(p - p-)), explicit.  CENTERED
 * takes the direct damping term at the centre of the step, (p+ - p-)/2,
 * which dissipates every mode; the explicit form can diverge in a boundary
 * layer several voxels thick at the 3D Courant limit. */
enum { VIRS_BOUNDARY_REFERENCE = 0, VIRS_BOUNDARY_CENTERED = 1 };

/* roles of OBJ material ids (virs_set_material_roles) */
#define VIRS_ROLE_IGNORE 0xFF /* triangles are not voxelised                     */
#define VIRS_ROLE_SOURCE 0xFE /* "speaker": flag 3, hard source (simulator.cpp:445-449) */
/* values 0..63: wall (flag 1) with that absorber material index (simulator.cpp:439-444) */

typedef struct virs_params {
    uint32_t struct_size;    /* sizeof(virs_params)                                   */
    int32_t device;          /* CUDA device ordinal                                   */
    float sound_speed;       /* c = 343 m/s            (simulator_gpu.cu:195)          */
    float courant;           /* dt = courant*h/(c*sqrt 3); 0.5 (simulator_gpu.cu:196)  */
    float cell_size;         /* h; 0 = 343/(22050*2*2) (simulator.cpp:17-18, 321)      */
    float bbox_nudge;        /* 0.1 m                  (simulator.cpp:304)             */
    int32_t sponge_width;    /* W = 1                  (sponge_kernel.cu:5)            */
    int32_t storage;         /* VIRS_STORAGE_*                                         */
    int32_t boundary_form;   /* VIRS_BOUNDARY_REFERENCE or VIRS_BOUNDARY_CENTERED        */
    float storage_scale;     /* stored = p*scale for 16-bit storage; 0 = automatic     */
    float boundary_gain;     /* 0.4f                   (simulator_gpu.cu:148)          */
    float boundary_k;        /* 0 = (c*dt)/h*0.95 on the host (simulator_gpu.cu:147)  */
    double mix_filtered;     /* 0.1                    (simulator_gpu.cu:148)          */
    double mix_direct;       /* 0.9                    (simulator_gpu.cu:148)          */
    int32_t rigid_walls;     /* 1: boundary voxels take the rigid-wall update from their
                              * air neighbours (fdtd_kernel_rigid_walls,
                              * simulator_gpu.cu:152-180, whose launch the reference
                              * keeps commented at :280) before the filter correction;
                              * 0 = the interior update with the wall mirror          */
} virs_params;

typedef struct virs_grid_info {
    uint64_t nx, ny, nz;     /* grid dimensions                                       */
    float cell_size;         /* h                                                     */
    float bbox_min[3];       /* world position of voxel corner (0,0,0)                */
    float dt;                /* time step (float, as the step kernel uses it)         */
    double sample_rate;      /* 1/dt in double, as the filter design gets it          */
    uint64_t boundary_count; /* flag-2 voxels after virs_classify                     */
    uint64_t steps_done;     /* steps run since virs_start_simulation                 */
} virs_grid_info;

typedef struct virs_timing {
    double step_kernel_ms;   /* summed CUDA-event time of the stencil kernel         */
    double boundary_kernel_ms; /* summed CUDA-event time of the boundary-list kernel */
    uint64_t step_launches;  /* stencil launches timed                                */
    uint64_t kernel_launches;/* all kernels this library launched while timing        */
} virs_timing;

/* ---- lifetime -------------------------------------------------------------- */

/* Reference defaults for every field. */
virs_status virs_params_default(virs_params *p);

/* Replaces fdtd_setup / fdtd_gpu_setup (simulator_dispatch.cpp:12-19,
 * simulator_gpu.cpp:7-235).  Device memory is allocated when a grid is set. */
virs_status virs_create(const virs_params *p, virs_sim **out);

/* Replaces fdtd_cleanup / fdtd_gpu_cleanup (simulator_dispatch.cpp:51-58,
 * simulator_gpu.cpp:237-305).  NULL is accepted. */
virs_status virs_destroy(virs_sim *sim);

/* Message of the last failed call on this thread ("" if none). */
const char *virs_last_error(void);

/* ---- geometry -------------------------------------------------------------- */

/* Material id -> role table used by the voxeliser.  Default {0: wall absorber
 * 0, 1: source}, the reference's mapping (simulator.cpp:439-449). */
virs_status virs_set_material_roles(virs_sim *sim, const uint8_t *roles, size_t n);

/* Replaces the geometry half of Simulator::loadObj (simulator.cpp:262-452):
 * parse an OBJ (+ its mtllib), bounding box with nudge, grid sizing,
 * allocation, triangle/box voxelisation into flags 1 (wall) and 3 (source). */
virs_status virs_load_obj(virs_sim *sim, const char *path);

/* The same from an in-memory mesh: verts [nverts][3] (world metres),
 * tris [ntris][3] vertex indices, tri_material [ntris] OBJ material ids. */
virs_status virs_set_mesh(virs_sim *sim, const float *verts, size_t nverts, const uint32_t *tris,
                          const int32_t *tri_material, size_t ntris);

/* Replaces updateGPUFromGrid for the flags (simulator_dispatch.cpp:70-81):
 * set the grid directly.  flags [nx*ny*nz] with values 0..3 (reference
 * layout); wall_material [nx*ny*nz] or NULL (all absorber 0). */
virs_status virs_set_grid(virs_sim *sim, uint64_t nx, uint64_t ny, uint64_t nz, float cell_size,
                          const uint8_t *flags, const uint8_t *wall_material);

/* z-slabs: one grid over several GPUs (no reference counterpart, which runs
 * one grid on one GPU; the step is a nearest-neighbour stencil, so a split
 * along z needs one plane of p^n from each neighbour per step).  The interior
 * planes 1..nz-2 of an nx*ny*nz grid are split into contiguous ranges, one
 * per handle.  A slab handle owns the planes [z_lo, z_hi)
 * (1 <= z_lo < z_hi <= nz-1) and keeps one ghost plane on each side: its
 * own grid is nx*ny*(z_hi - z_lo + 2), local plane k = global plane
 * z_lo - 1 + k, and voxel indices given to it (sources, receivers) are
 * local.  At a global border the ghost is the border plane itself (never
 * written, 0).  flags / wall_material (NULL: absorber 0) hold the global
 * planes [z_first, z_first + nz_ext), which must include the planes
 * max(0, z_lo - W - 2) .. min(nz, z_hi + W + 2) - 1 for sponge width W:
 * virs_classify classifies them all and keeps the slab's planes, so the
 * sponge layer, normals, cell codes and boundary list of the owned planes
 * are the whole grid's.  Before every step the caller copies the
 * neighbours' first / last owned planes of p^n into the ghost planes
 * (virs_slab_planes); the slabs then advance exactly as the whole grid.
 * 16-bit storage needs an explicit storage_scale (every slab stores
 * alike). */
virs_status virs_set_grid_slab(virs_sim *sim, uint64_t nx, uint64_t ny, uint64_t nz, float cell_size, uint64_t z_lo,
                               uint64_t z_hi, const uint8_t *flags, const uint8_t *wall_material, uint64_t z_first,
                               uint64_t nz_ext);

/* The same from a mesh, for slab `part` of `parts` (0 <= part < parts): the
 * whole grid is sized from the mesh as virs_set_mesh / virs_load_obj size
 * it, its interior planes are split into `parts` ranges whose sizes differ
 * by at most one (lower ranges first), and only this slab's uploaded planes
 * are voxelised, with the whole grid's origin, so every flag equals the
 * whole grid's.  No handle ever holds the whole grid.  bbox_min in
 * virs_get_grid_info is the whole grid's origin. */
virs_status virs_set_mesh_slab(virs_sim *sim, const float *verts, size_t nverts, const uint32_t *tris,
                               const int32_t *tri_material, size_t ntris, uint32_t part, uint32_t parts);
virs_status virs_load_obj_slab(virs_sim *sim, const char *path, uint32_t part, uint32_t parts);

/* Owned planes [*z_lo, *z_hi) of a slab and the planes *nz of its whole
 * grid; VIRS_E_STATE for a handle that is not a slab. */
virs_status virs_get_slab_info(const virs_sim *sim, uint64_t *z_lo, uint64_t *z_hi, uint64_t *nz);

/* Device addresses of the planes of p^n (the state the next step reads)
 * that a slab exchanges before that step, each plane_bytes long (rows of nx
 * rounded up to 32 voxels, in the storage type): first / last = its first
 * and last owned planes (sent to the slab below / above), ghost_lo /
 * ghost_hi = its ghost planes (received from the slab below / above).
 * They alternate between two buffers from step to step: ask before each
 * step, after queueing the previous one. */
virs_status virs_slab_planes(const virs_sim *sim, void **first, void **last, void **ghost_lo, void **ghost_hi,
                             size_t *plane_bytes);

/* The exchange in the library (no reference counterpart): lo and hi are
 * adjacent slabs of one grid (lo's owned planes end where hi's begin) at the
 * same step, on one GPU or two GPUs of this process.  Each handle pulls its
 * ghost plane of p^n from the other -- lo's ghost_hi from hi's first owned
 * plane, hi's ghost_lo from lo's last -- with a device (or peer) copy on its
 * own stream, after the other handle's last queued work; the kernels only
 * ever read their own GPU's memory.  Returns when the copies are queued; the
 * handles' next runs follow them.  Call it for every adjacent pair before
 * every step (a slab's step writes the buffer its neighbour pulled from one
 * step later). */
virs_status virs_slab_exchange(virs_sim *lo, virs_sim *hi);

/* `steps` steps of a grid split into the n slabs slabs[0..n-1] (in order,
 * covering planes 1..nz-2).  Per step and slab: the stencil over the slab's
 * interior planes (which read no ghost plane) on its own stream, while a
 * second stream of the handle pulls its two ghost planes from the
 * neighbours (after their previous step); then the two edge planes, the
 * boundary pass and the sources and receivers.  The copies overlap the
 * interior work; slabs on different GPUs of this process run concurrently.
 * Returns when the work is queued (virs_synchronize each handle to wait).
 * Single steps (no two-step passes).  When every slab is on one GPU, runs of
 * 16 steps or more replay a CUDA graph of 16 steps of all slabs (captured
 * at the first such call and kept by slabs[0] while the same unchanged
 * slabs run) and take the remaining steps as direct launches; slabs on
 * several GPUs always take direct launches.  The device stop rule is
 * refused. */
virs_status virs_slab_run(virs_sim *const *slabs, uint32_t n, uint64_t steps);

/* One step of a slab in two parts, for hosts that exchange the ghost planes
 * themselves (no reference counterpart; one process per GPU, the planes
 * sent with NCCL or MPI between the parts):
 *   virs_slab_step_begin  the stencil over the slab's interior planes 2 ..
 *                         nz-3, which read no ghost plane, on `stream`
 *                         (NULL: the handle's stream) after the handle's
 *                         last queued work;
 *   virs_slab_step_end    the edge planes 1 and nz-2, the boundary pass and
 *                         the sources and receivers, then the step count
 *                         and buffer parity advance.
 * Between the two the host sends the slab's first and last owned planes of
 * p^n (virs_slab_planes, before this step) and receives its ghost planes:
 * the interior launch reads neither and writes only p^{n+1}, so the
 * exchange can run beside it.  virs_slab_step_end must follow, in stream
 * order, both virs_slab_step_begin and the receives.  A second begin
 * before the end, or virs_run / virs_slab_run in between, is refused
 * (VIRS_E_STATE).  The device stop rule is refused. */
virs_status virs_slab_step_begin(virs_sim *sim, void *stream);
virs_status virs_slab_step_end(virs_sim *sim, void *stream);

virs_status virs_get_grid_info(const virs_sim *sim, virs_grid_info *out);

/* Replaces buildSpongeLayer / buildSpongeLayerGPU (simulator_dispatch.cpp:83-91,
 * sponge_kernel.cu:65-99) plus the normals, boundary-list and filter-state
 * steps of loadObj (simulator.cpp:472-610, uploadNormalsToGPU :102-109,
 * uploadBoundaryIndicesToGPU :120-130, allocFilterStates :132-160).
 * All on the GPU. */
virs_status virs_classify(virs_sim *sim);

/* Parity exports (reference layout).  Flags are the voxeliser's (0..3)
 * before virs_classify and the classified ones after; wall materials are
 * the absorber index of each wall voxel as voxelised or set. */
virs_status virs_get_flags(const virs_sim *sim, uint8_t *out, size_t n);
virs_status virs_get_wall_materials(const virs_sim *sim, uint8_t *out, size_t n);
virs_status virs_get_normals(const virs_sim *sim, uint8_t *out, size_t n);
virs_status virs_get_boundary_indices(const virs_sim *sim, uint32_t *out, size_t n);
/* per boundary voxel (list order): material index and sponge weight */
virs_status virs_get_boundary_materials(const virs_sim *sim, uint8_t *material, float *weight, size_t n);

/* ---- filters, sources, receivers ----------------------------------------- */

/* Replaces allocFilterCoeffs + uploadFilterCoeffsToGPU
 * (simulator_dispatch.cpp:162-280): coeffs [n_materials][n_sections][5] as
 * {b0, b1, b2, a1, a2}; sections run in series.  Resets filter states. */
virs_status virs_set_filters(virs_sim *sim, uint32_t n_materials, uint32_t n_sections, const float *coeffs);

/* computeHighpassBiquad / computeLowpassBiquad (biquad.cpp:3-43), with the
 * reference's float/double promotions; out5 = {b0, b1, b2, a1, a2}. */
virs_status virs_design_highpass(float sample_rate, float cutoff, float q, float gain, float *out5);
virs_status virs_design_lowpass(float sample_rate, float cutoff, float q, float gain, float *out5);

/* FP64 designs of absorbing-boundary filters (no reference counterpart; the
 * reference designs one RBJ high-pass, simulator.cpp:955-967).
 * First order: bilinear transform, prewarped at fc, of G*wc/(s + wc) with
 * G = (1 - R)/(1 + R) for the reflection coefficient R; out5 as above.
 * Octave cascade: low shelf / peak / high shelf at freqs (NULL = 250, 1000,
 * 4000 Hz) with band gains G_b from absorption alpha[b]; out15 = 3 x out5. */
virs_status virs_design_first_order(double sample_rate, double reflection, double fc, double *out5);
virs_status virs_design_octave_cascade(double sample_rate, const double *alpha, const double *freqs, double *out15);

/* Values given to flag-3 voxels at step n (n < len; 0 after).  Default: 10
 * for steps 0..9 (simulator_gpu.cu:214-218). */
virs_status virs_set_hard_source(virs_sim *sim, const float *values, size_t len);

/* Additive point sources (no reference counterpart; the reference's
 * commented audio-file source, simulator_gpu.cu:220-245).  idx [n] voxel
 * indices, distinct, interior; signal [n][len]; p(idx) += signal[s][step]. */
virs_status virs_set_sources(virs_sim *sim, uint32_t n, const uint64_t *idx, const float *signal, size_t len);

/* Receivers (the reference reads the single voxel (334,225,270) after every
 * step, simulator_gpu.cu:295-300).  idx [n] voxel indices. */
virs_status virs_set_receivers(virs_sim *sim, uint32_t n, const uint64_t *idx);

/* Audio-driven sources (the design written out, commented, at
 * simulator_gpu.cu:219-231, and TODO.md "Audio file implementation"): a
 * signal sampled at sample_rate is read at the simulation times step * dt
 * by linear interpolation (float time and sample index; 0 once index + 1
 * reaches the end) for `steps` steps.  The hard-source form drives the
 * flag-3 voxels, as the reference's design does; the soft-source form
 * gives one channel per source, samples [n][len].  Need a grid (dt). */
virs_status virs_set_hard_source_audio(virs_sim *sim, const float *samples, size_t len, float sample_rate,
                                       uint64_t steps);
virs_status virs_set_sources_audio(virs_sim *sim, uint32_t n, const uint64_t *idx, const float *samples, size_t len,
                                   float sample_rate, uint64_t steps);

/* ---- running ---------------------------------------------------------------- */

/* Replaces fdtd_start_simulation (simulator_dispatch.cpp:93-100): reserve
 * receiver storage for `steps` steps and start from rest (fields, filter
 * states and the step counter set to zero). */
virs_status virs_start_simulation(virs_sim *sim, uint64_t steps);

/* Replaces fdtd_step / fdtd_gpu_step (simulator_dispatch.cpp:21-29,
 * simulator_gpu.cu:184-332): one step numbered `step`, then the first
 * receiver's new sample is read back into *sample (may be NULL) and the
 * reference's RMS stop rule (simulator_gpu.cu:303-330, on receiver 0) sets
 * *keep_going (may be NULL). */
virs_status virs_step(virs_sim *sim, uint32_t step, int *keep_going, float *sample);

/* The reference's stop rule (simulator_gpu.cu:303-330, applied on the host
 * after every step; virs_step keeps that form) evaluated on the device, so
 * that graph-launched runs can stop too: with enable = 1, after every step
 * of virs_run / virs_run_host past step 3000 the post kernel takes the RMS
 * of receiver 0's last 100 samples through the reference's slow filter, and
 * once it is below 0.0009 every later kernel of the run returns at once.
 * The run then ends after the step that fired the rule: virs_run /
 * virs_run_host synchronise when the rule is on, steps_done
 * (virs_get_grid_info) is that step + 1, the fields and samples are those
 * of that step (virs_run_host still copies the samples it was asked for:
 * those of steps that did not run are 0), and further runs do nothing
 * until virs_start_simulation.
 * Off by default (benchmarks run every step).  virs_step, the adjoint and
 * batches refuse or ignore it: they run every step. */
virs_status virs_set_stop_rule(virs_sim *sim, int enable);
/* whether the rule fired, and at which step */
virs_status virs_get_stop(const virs_sim *sim, int *stopped, uint64_t *stop_step);

/* Run `steps` steps on `stream` (a cudaStream_t, NULL = the handle's own
 * stream) with no host traffic; the step loop is a CUDA graph.  Returns
 * when the work is queued.  The handle's own stream is a non-blocking
 * stream: work on CUDA's legacy default stream is not ordered with it, so a
 * caller that wants the legacy stream passes cudaStreamLegacy. */
virs_status virs_run(virs_sim *sim, uint64_t steps, void *stream);

/* End-to-end form for host callers: copies `signal` [n_src][steps] (or NULL
 * to keep the signals set before) for the next `steps` steps from host
 * memory, runs, and copies the new receiver samples [n_rcv][steps] to
 * `ir_out`; synchronous. */
virs_status virs_run_host(virs_sim *sim, uint64_t steps, const float *signal, float *ir_out, void *stream);

/* Wait for the handle's queued work. */
virs_status virs_synchronize(virs_sim *sim);

/* Receiver samples [n_rcv][steps] of steps first .. first+steps-1. */
virs_status virs_get_ir(const virs_sim *sim, uint64_t first, uint64_t steps, float *out);

/* Replaces updateCurrentGridFromGPU (simulator_dispatch.cpp:42-49): p^n
 * (and p^{n-1} if prev != NULL) in the reference layout, unscaled. */
virs_status virs_get_pressure(const virs_sim *sim, float *cur, float *prev, size_t n);
virs_status virs_set_pressure(virs_sim *sim, const float *cur, const float *prev, size_t n);

/* Replaces initPressureSphereGPU (init_sphere.cu:27-55). */
virs_status virs_init_pressure_sphere(virs_sim *sim, uint64_t x, uint64_t y, uint64_t z, uint64_t radius,
                                      float pressure, int init);

/* FP64 discrete energy of the current state (the physics health monitor). */
virs_status virs_energy(virs_sim *sim, double *out);

/* The same energy for callers that cannot allocate device memory (no
 * counterpart in the reference): real-time threads, where cudaMalloc and
 * cudaFree may synchronise the device and block, or hosts that own all
 * device memory through their own pool.  virs_energy allocates its
 * reduction buffer on first use; this variant keeps one partial sum per z
 * plane in a static device array of VIRS_ENERGY_MAX_PLANES doubles (64 KiB,
 * held by every GPU that loads the library until exit) and calls no
 * allocator.  Grids with more planes get VIRS_E_ARG.  The result is written
 * to the caller's device double `d_out`, in order on `stream` (NULL = the
 * handle's stream); nothing waits for it.  The first call on a device looks
 * up the array's address (cudaGetSymbolAddress): make it before any stream
 * capture.  All calls share the array, so calls whose work overlaps on the
 * GPU race: callers serialise them.  The call records the handle's
 * completion event on the stream it used, so virs_synchronize and
 * virs_destroy wait for its reads of the fields. */
#define VIRS_ENERGY_MAX_PLANES 8192
virs_status virs_energy_noalloc(virs_sim *sim, double *d_out, void *stream);

/* ---- measurement ------------------------------------------------------------- */

/* While enabled, virs_run launches without a graph and brackets every
 * stencil launch and every boundary-list launch with CUDA events;
 * virs_get_timing sums them. */
virs_status virs_set_timing(virs_sim *sim, int enable);
virs_status virs_get_timing(virs_sim *sim, virs_timing *out);

/* Kernel variant: tile height (4, 8 or 16 rows; 0 = 8), planes per block
 * (0 = the library's choice) and pipeline depth: 0 = the register-streaming
 * kernel, 1..3 = the TMA kernel with that many planes in flight, -1 = the
 * default (TMA, 2).  All variants give bit-identical results. */
virs_status virs_set_tiling(virs_sim *sim, int tile_rows, int planes_per_block, int pipeline_depth);

/* Time blocking (no reference counterpart): with steps_per_pass = 2, virs_run
 * and virs_run_host advance whole groups of four steps two at a time: one
 * kernel reads p^n and p^{n-1} once and writes p^{n+1} and p^{n+2}, over two
 * more field buffers allocated on first use (a grid for which they do not fit
 * runs single steps).  The voxels next to boundary voxels and sources are
 * recomputed after the first step is complete, so the results are
 * bit-identical to single steps.  tile_rows 12, 14, 16 or 32 (0 = 14; with
 * 12, 14 and 16 rows 4, 3 and 2 planes are in flight), planes per block
 * 0 = all.  Off (1) by default; not used with the register-streaming
 * kernel (pipeline depth 0).  With the device stop rule, a run that stops
 * inside a group of four steps leaves the stop step's fields in the usual
 * buffers, as single steps do.  *active tells whether the current settings
 * run two steps per pass. */
virs_status virs_set_time_blocking(virs_sim *sim, int steps_per_pass, int tile_rows, int planes_per_block);
virs_status virs_get_time_blocking(const virs_sim *sim, int *steps_per_pass, int *tile_rows, int *planes_per_block,
                                   int *active);

/* Rounding of the values stored in 16-bit fields (no reference counterpart;
 * the reference stores FP32).  VIRS_ROUND_NEAREST (default): to nearest,
 * ties to even.  VIRS_ROUND_STOCHASTIC: a value is rounded up in magnitude
 * with the probability of its distance from the value below, from 16 bits of
 * a counter-based hash of (voxel, step), so a run is reproducible and equal
 * for every kernel variant, in batches and in z-slabs; FP16 values below
 * 2^-14 or of 65504 and more in magnitude still round to nearest.  It
 * applies to the step's stores (stencil, boundary pass, sources); values set
 * with virs_set_pressure or virs_init_pressure_sphere round to nearest.  No
 * effect on FP32 storage.  Two steps per pass do not apply it: with it on,
 * virs_run takes single steps and the autotuner tries no two-step variant. */
enum { VIRS_ROUND_NEAREST = 0, VIRS_ROUND_STOCHASTIC = 1 };
virs_status virs_set_rounding(virs_sim *sim, int mode);

typedef struct virs_tiling {
    int32_t tile_rows;        /* 4, 8 or 16                                        */
    int32_t planes_per_block; /* z planes streamed by one block                    */
    int32_t pipeline_depth;   /* 0 = register kernel, 1..3 = TMA planes in flight  */
    float ms_per_step;        /* measured by virs_autotune (0 otherwise)           */
} virs_tiling;

/* Autotuner (no reference counterpart): right after virs_start_simulation,
 * times `trial_steps` steps of each TMA variant (tile rows 4/8/16, depth
 * 1..3, 8..64 planes per block) and then of the two-step variants (time
 * blocking: tile rows 14/16/12, 32..102 planes per block, trial_steps
 * rounded up to a multiple of four, at least eight) on this handle's own
 * grid and keeps the fastest: the tiling it returns, and the steps per pass
 * that virs_get_time_blocking reports.  Every candidate is timed twice, in
 * forward and then reverse order, because a sustained load reaches the
 * GPU's power cap within about a second and would favour the candidates
 * timed first.  The simulation is then back at rest.  Results are cached
 * per device, storage and grid shape for the life of the process.
 * virs_batch_autotune does the same for a batch's tilings (one tile per
 * block or persistent). */
virs_status virs_autotune(virs_sim *sim, uint32_t trial_steps, virs_tiling *best);
virs_status virs_get_tiling(const virs_sim *sim, virs_tiling *out);

/* ---- adjoint ----------------------------------------------------------------- */

/* Gradients of a receiver loss (no reference counterpart; used for inverse
 * design of boundary materials).  virs_forward_checkpointed starts from rest
 * and runs `steps` FP32 steps, keeping the state every `every` steps.
 * virs_adjoint then takes dL/dIR (dl_dir [n_rcv][steps], host) and returns
 * dL/dcoeff (grad_coef [n_materials][n_sections][5] = {b0 b1 b2 a1 a2},
 * FP64) and dL/dsignal (grad_signal [n_src][steps]); either output may be
 * NULL.  Each checkpoint segment is recomputed once; the reverse pass runs
 * the step backwards in time (the interior update is self-adjoint, the
 * filters run transposed).  The receiver samples of the forward run stay
 * readable; the fields do not, so start again before running. */
virs_status virs_forward_checkpointed(virs_sim *sim, uint64_t steps, uint32_t every, void *stream);
virs_status virs_adjoint(virs_sim *sim, const float *dl_dir, double *grad_coef, float *grad_signal);

/* ---- batched runs ------------------------------------------------------------ */

/* Many simulations advanced together (no reference counterpart: the
 * reference runs one room with one source at a time).  Members are handles
 * that are classified, configured and started, on one device, with one
 * storage type, at the same step; they keep their buffers and results (read
 * them with virs_get_ir on each member).  Every step is three launches for
 * the whole batch -- one persistent TMA stencil kernel over the tiles of all
 * members, one boundary-list kernel, one source/receiver kernel -- and
 * virs_batch_run replays them as CUDA graphs.  Changing a member after
 * virs_batch_create makes virs_batch_run fail with VIRS_E_STATE. */
typedef struct virs_batch virs_batch;
virs_status virs_batch_create(virs_sim *const *members, uint32_t n, virs_batch **out);
virs_status virs_batch_run(virs_batch *batch, uint64_t steps, void *stream);
virs_status virs_batch_synchronize(virs_batch *batch);
virs_status virs_batch_set_tiling(virs_batch *batch, int tile_rows, int planes_per_block, int pipeline_depth);
virs_status virs_batch_autotune(virs_batch *batch, uint32_t trial_steps, virs_tiling *best);
virs_status virs_batch_destroy(virs_batch *batch);

/* ---- IR post-processing ----------------------------------------------------- */

/* Replaces designChebyshevI_LP with distributeDCGain
 * (src/util/downsampling_filter_iir.cpp:11-193): a Chebyshev-I low-pass for
 * anti-aliasing before resampling, as second-order sections
 * sos [n][6] = {b0, b1, b2, a0, a1, a2} (a0 = 1), DC gain 1.  fstop <= 0
 * means min(0.499 fs, 1.15 fc).  The sections equal the reference's bit for
 * bit.  VIRS_E_ARG for invalid specs or when more than max_sections are
 * needed (*n_sections is not written then). */
virs_status virs_design_chebyshev_lowpass(double fs, double fc, double fstop, double ripple_db, double atten_db,
                                          double *sos, uint32_t max_sections, uint32_t *n_sections);

/* Replaces the IR post-processing of Simulator::simulate
 * (simulator.cpp:1029-1080), which resamples the receiver trace from the
 * simulation rate to 48 kHz with a library resampler (kfr) and divides it
 * by its peak.  Here, on the GPU, for every receiver over the steps run so
 * far: the cascade `sos` (n_sections <= 32, 0 = none) in FP64 transposed
 * direct form II at the simulation rate, linear interpolation at k / rate
 * (the interpolation written at simulator.cpp:1046-1057; the last sample
 * is held past the end), and, if normalize, division by that receiver's
 * peak magnitude (a silent receiver stays zero).  The output length is
 * (uint64_t)(rate * steps * dt) as at simulator.cpp:1037-1038.
 * out [n_receivers][*out_len]; out == NULL only reports *out_len;
 * VIRS_E_ARG when capacity < *out_len. */
virs_status virs_postprocess_ir(virs_sim *sim, double rate, const double *sos, uint32_t n_sections, int normalize,
                                float *out, uint64_t capacity, uint64_t *out_len);

/* The same resampling with a band-limited interpolator instead of the
 * Chebyshev cascade and linear interpolation, in the manner of the
 * reference's kfr resampler (resample_quality::high, simulator.cpp:1056-1063;
 * kfr is absent and its design unknown, so the output is not bit-equal to
 * the reference's): output sample k sits at input position
 * t = k * fs / rate (fs = 1/dt) and takes sum_n x[n] h(t - n) over the
 * |t - n| < half_taps input samples around it, with the Kaiser-windowed sinc
 * h(tau) = 2 fc sinc(2 fc tau) I0(beta sqrt(1 - (tau/half_taps)^2)) / I0(beta),
 * fc = cutoff * min(fs, rate) / 2 / fs cycles per input sample, in FP64.
 * Peak normalisation and the output length as virs_postprocess_ir.  For the
 * reference's default cell (fs = 305.5 kHz) to 48 kHz, half_taps 245,
 * beta 10.06 and cutoff 0.9167 give a 20-24 kHz transition band and about
 * 100 dB of stop-band attenuation (the Kaiser design rules).
 * half_taps 1..4096, beta 0..50, cutoff in (0, 1]. */
virs_status virs_postprocess_ir_sinc(virs_sim *sim, double rate, uint32_t half_taps, double beta, double cutoff,
                                     int normalize, float *out, uint64_t capacity, uint64_t *out_len);

/* Failure-path self test (no reference counterpart): launches a kernel that
 * waits `limit` microseconds (1..2^20) on an mbarrier that nothing completes,
 * with the bounded wait of the step kernels; returns VIRS_E_TIMEOUT when the
 * timeout was reported, and the handle stays usable. */
virs_status virs_check_bounded_wait(virs_sim *sim, uint32_t limit);

#ifdef __cplusplus
}
#endif

#endif /* VIRS_H */
