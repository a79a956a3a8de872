/* plume_b200.h -- C ABI of libplume_b200.so: the sm_100a fluid step and volume render of chadmv/plume.
 *
 * The drop-in boundary is the reference's Python API (src/plume/sim/*, src/plume/render/*); the Python
 * package plume_b200 keeps those names and binds this ABI with ctypes. Each entry point below replaces the
 * Warp kernel launch(es) cited beside it (paths relative to the reference project).
 *
 * Conventions
 *   - Every array is a caller-owned, C-contiguous float32 device array, shape (n0, n1, n2), n2 contiguous.
 *     Cell arrays are (nx, ny, nz); face arrays (nx+1, ny, nz), (nx, ny+1, nz), (nx, ny, nz+1).
 *     The library never allocates or frees caller memory; scratch is passed in by the caller.
 *   - `stream` is a cudaStream_t (0 = the legacy default stream). Calls only enqueue work unless noted.
 *   - Every call returns PLUME_OK (0) or a negative status; plume_last_error() returns a thread-local message
 *     for the last failure. Calls come from one host thread per stream.
 */
#ifndef PLUME_B200_H
#define PLUME_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PLUME_OK 0
#define PLUME_ERR_INVALID (-1) /* bad argument (null pointer, size, count) */
#define PLUME_ERR_LAUNCH (-2)  /* a kernel launch or CUDA runtime call failed */
#define PLUME_ERR_DEVICE (-3)  /* a device-side check failed (reported through a status word) */

/* Storage of velocity, smoke and temperature arrays (plume_step, the render calls, plume_grid_speed); kernels
 * always compute in float. Pressure, divergence and scratch arrays are float in every mode. */
#define PLUME_STORAGE_F32 0
#define PLUME_STORAGE_BF16 1 /* bfloat16, rounded to nearest even on store */
#define PLUME_STORAGE_F16 2  /* IEEE half, rounded to nearest even on store */

#define PLUME_MAX_EMITTERS 16 /* emitters applied per launch; longer lists are applied in order, in chunks */
#define PLUME_STEP_PHASES 6   /* forces, velocity advection, divergence, pressure solve, gradient, scalars */

/* GridInfo (sim/grid.py:21-33). fill_hi and ghost_gap describe multigrid coarse levels (multigrid.py:84-94);
 * the simulation grid has fill_hi = (1,1,1), ghost_gap = 0.5. open_lo/open_hi: 1 = open face, 0 = wall. */
typedef struct PlumeGridInfo {
  int32_t dims[3];
  float cell_m;
  float origin_m[3];
  int32_t open_lo[3];
  int32_t open_hi[3];
  float fill_hi[3];
  float ghost_gap;
} PlumeGridInfo;

/* EmitterParams (sim/emitters.py:23-38). shape: 0 sphere, 1 box. */
typedef struct PlumeEmitter {
  int32_t shape;
  float center_m[3];
  float radius_m;
  float half_size_m[3];
  float edge_softness;
  float start_s;
  float end_s;
  float smoke_per_s;
  float temperature_k;
  float velocity_mps[3];
  int32_t outward;
  float noise_scale_m;
  float noise_strength;
  int32_t stream;
} PlumeEmitter;

/* ViewParams and LookParams (render/raymarch.py:30-52). */
typedef struct PlumeViewParams {
  float right[3];
  float up[3];
  float toward[3];
  float left_m;
  float top_m;
  float pixel_m;
  int32_t perspective;
  float eye[3];
} PlumeViewParams;

typedef struct PlumeLookParams {
  float opacity_per_density;
  float glow_start_k;
  float smoke_hides_heat;
  float normal_fade_thickness;
  int32_t shade_layout;
  float shade_fill;
} PlumeLookParams;

/* One advected quantity's buffers (AdvectedField, sim/grid.py:36-51), elements of the step's storage type.
 * `back` is not needed: the MacCormack correction recomputes the backward pass on the fly. */
typedef struct PlumeField {
  void* data;
  void* hat;
  void* next;
} PlumeField;

/* One multigrid level (multigrid.py:71-77): its geometry and pressure, right-hand side, residual arrays. */
typedef struct PlumeLevel {
  PlumeGridInfo info;
  float* q;
  float* rhs;
  float* residual;
} PlumeLevel;

/* Everything one substep reads and writes (Stepper.step, sim/stepper.py:28-44). */
typedef struct PlumeStepState {
  PlumeGridInfo info;
  PlumeField u, v, w, smoke, temperature;
  float* pressure;
  float* divergence;
  /* scratch: confinement curl and push, 3 arrays of nx*ny*nz floats each (x, y, z components) */
  float* curl[3];
  float* push[3];
  /* scratch: the smoke budget's partial sums (plume_smoke_scratch_doubles() doubles) and its factor (1 float) */
  double* sums;
  float* factor;
  /* scratch (optional, may be null): plume_advect_scratch_floats() floats; with it the MacCormack forward
   * pass stores each element's clamp range (two values of the storage type) and the correction does not
   * trace forward a second time */
  float* advect_scratch;
  /* pressure-solve levels: levels[0] aliases pressure/divergence and its residual array is the sweeps' second
   * pressure array (Gauss-Seidel uses levels[0] only); coarser multigrid levels are caller-allocated */
  const PlumeLevel* levels;
  int32_t level_count;
  int32_t storage;          /* PLUME_STORAGE_*: the type of the u, v, w, smoke and temperature arrays */
} PlumeStepState;

typedef struct PlumeStepParams {
  float time_s;
  float dt;
  float dt_over_cell;       /* dt / info.cell_m, computed in double and rounded (advect.py:61) */
  int32_t seed;
  const PlumeEmitter* emitters; /* host array */
  int32_t emitter_count;
  float gravity, heat_buoyancy, smoke_weight, ambient_k;
  float confinement;        /* 0: no confinement pass */
  float turbulence_scale_m, turbulence_strength, turbulence_pattern_time;  /* strength 0: no pass */
  int32_t apply_drag;       /* 0: no drag pass */
  float wind[3];
  float drag_keep;          /* exp(-drag_per_s * dt) in double, rounded */
  int32_t solver;           /* 0 multigrid, 1 Gauss-Seidel */
  int32_t solver_iterations;/* multigrid cycles or Gauss-Seidel sweeps */
  int32_t multigrid_sweeps;
  int32_t apply_dissipation;/* 0: no dissipation pass */
  float smoke_keep, heat_keep;
  void* const* phase_events;/* null, or PLUME_STEP_PHASES + 1 cudaEvent_t recorded at the phase boundaries */
} PlumeStepParams;

const char* plume_last_error(void);
int plume_abi_version(void);
/* Kernels this library has enqueued in this process (all streams); for launch accounting in benchmarks. */
unsigned long long plume_launch_count(void);

/* ---- per-operator entry points (used by the Python mirror of each reference function) ---------------- */

/* advect.py:53-56,71-76 semi_lagrangian_kernel: dst = sample(src, trace(p, dt_over_cell)). */
int plume_advect_semi_lagrangian(const PlumeGridInfo* info, const int32_t shape[3], const float* src, float* dst,
                                 const float* u, const float* v, const float* w, float dt_over_cell,
                                 const float offset[3], float outside, int32_t uses_outside, void* stream);

/* advect.py:59-68 advect_maccormack (semi_lagrangian_kernel twice + maccormack_correct_kernel): writes the
 * forward pass into `hat` and the clamped correction into `next`. */
int plume_advect_maccormack(const PlumeGridInfo* info, const int32_t shape[3], const float* data, float* hat,
                            float* next, const float* u, const float* v, const float* w, float dt_over_cell,
                            const float offset[3], float outside, int32_t uses_outside, void* stream);

/* emitters.py:147-153 emit (emit_scalars_kernel + 3 x emit_velocity_kernel); `emitters` is a host array. */
int plume_emit(const PlumeGridInfo* info, float* smoke, float* temperature, float* u, float* v, float* w,
               const PlumeEmitter* emitters, int32_t count, int32_t seed, float time_s, float dt, void* stream);

/* forces.py:26-31 apply_buoyancy (buoyancy_kernel). */
int plume_buoyancy(const PlumeGridInfo* info, float* v, const float* smoke, const float* temperature,
                   float gravity, float heat_buoyancy, float smoke_weight, float ambient_k, float dt, void* stream);

/* forces.py:40-48 apply_drag (drag_kernel x 3): f = wind + (f - wind) * keep. */
int plume_drag(const PlumeGridInfo* info, float* u, float* v, float* w, const float wind[3], float keep,
               void* stream);

/* vorticity.py:95-111 VorticityConfinement.apply / measure_curl: writes curl[3] (and push[3] and adds
 * push*dt to the faces when `apply` is 1). */
int plume_confinement(const PlumeGridInfo* info, float* u, float* v, float* w, float* curl_xyz[3],
                      float* push_xyz[3], float strength, float dt, int32_t apply, void* stream);

/* turbulence.py:59-67 apply_turbulence (turbulence_kernel x 3). */
int plume_turbulence(const PlumeGridInfo* info, float* u, float* v, float* w, int32_t seed, float scale_m,
                     float strength, float pattern_time, float dt, void* stream);

/* pressure.py:144-154 project: zero_closed_faces_kernel x 3 + divergence_kernel (this call), then the solve,
 * then subtract_gradient_kernel x 3 (plume_subtract_gradient). */
int plume_project_begin(const PlumeGridInfo* info, float* u, float* v, float* w, float* divergence,
                        void* stream);
int plume_divergence(const PlumeGridInfo* info, const float* u, const float* v, const float* w,
                     float* divergence, void* stream);
int plume_subtract_gradient(const PlumeGridInfo* info, float* u, float* v, float* w, const float* q,
                            void* stream);

/* pressure.py:124-141 GaussSeidel / red_black_sweeps (red_black_sweep_kernel, colour 0 then 1 per sweep).
 * Each sweep is one launch that reads one pressure array and writes the other: `scratch` (same size as q,
 * contents ignored) is the second array; the result is always left in q. */
int plume_red_black_sweeps(const PlumeGridInfo* info, float* q, float* scratch, const float* rhs, int32_t sweeps,
                           float relaxation, void* stream);

/* multigrid.py:124-147 Multigrid.__call__: `cycles` V-cycles over caller-allocated levels. Every level's
 * `residual` array serves as its second pressure array (the residual is restricted without being stored). */
int plume_multigrid(const PlumeLevel* levels, int32_t level_count, int32_t cycles, int32_t sweeps, void* stream);

/* Pressure-solve strategy (no reference counterpart; results do not depend on it): levels with at least
 * `tiled_min_cells` cells sweep in shared-memory tiles (one launch per sweep), smaller levels one colour per
 * launch; the first level with at most `bottom_max_cells` cells and all coarser ones run in one launch:
 * bottom_kind 1 an 8-CTA thread-block cluster (levels split in x-slabs over the CTAs' shared memory), 0 one
 * 1024-thread block; at most 200 KiB of shared memory per CTA. Process-wide; defaults 2^40, 2048, 0. */
int plume_tune_solver(long long tiled_min_cells, long long bottom_max_cells, int32_t bottom_kind);
/* The current pressure-solve strategy (the three values plume_tune_solver sets). */
int plume_solver_tuning(long long* tiled_min_cells, long long* bottom_max_cells, int32_t* bottom_kind);

/* Pressure solves replay a CUDA graph of their launches, captured once per levels/cycles/strategy (default
 * on). 0 turns that off (every kernel launched one by one); results are the same either way. When the
 * caller's stream is itself being captured, launches are always made one by one into that capture. */
int plume_use_graphs(int32_t enable);

/* No counterpart in the reference (the same solve, another storage). plume_multigrid with caller scratch of
 * plume_split_scratch_floats(&levels[0].info) floats: when the top level has at least the plume_tune_split
 * threshold of cells, it is swept in colour-split storage (red and black cells in separate arrays, converted in
 * and out around the cycles), so that a colour pass moves only the sectors of the cells it needs. Every value
 * equals plume_multigrid's. plume_step does the same with its advect_scratch. The threshold is 1 << 23 cells
 * by default (levels whose q and rhs exceed L2, where the split passes measured faster on B200); the scratch
 * must be 16-byte aligned, or the natural layout runs. */
long long plume_split_scratch_floats(const PlumeGridInfo* info);
int plume_tune_split(long long min_cells);
long long plume_split_min_cells(void); /* the current threshold */
int plume_multigrid_split(const PlumeLevel* levels, int32_t level_count, int32_t cycles, int32_t sweeps,
                          float* scratch, void* stream);

/* multigrid.py:36-43 residual_kernel. */
int plume_residual(const PlumeGridInfo* info, const float* q, const float* rhs, float* residual, void* stream);

/* ---- solving to a residual (no reference counterpart: the reference runs a fixed number of cycles) --------
 * Defect correction: the residual r = rhs - A q of the float pressure is evaluated in double, the correction
 * e solves A e = r by one float V-cycle from e = 0 whose coarsest level is swept in double, and q += e.
 *
 * The pressure may be carried as the unevaluated sum of two floats, q + q_lo (q_lo null for q alone), so that
 * the iterate can go below the float rounding of q: the correction is added as a two-sum and renormalised.
 *
 * plume_residual_f64 stores r (as float) in `residual` and writes norms[0] = sum r^2, norms[1] = sum rhs^2
 * (device doubles, summed in a fixed order); `scratch` holds plume_norm_scratch_doubles(info) doubles.
 * plume_multigrid_correct runs one correction: levels[0] is {info, q = e, rhs = r, residual = a scratch
 * array}, the coarser levels as for plume_multigrid; `pressure` (+ `pressure_lo`) gets e added. */
long long plume_norm_scratch_doubles(const PlumeGridInfo* info);
int plume_residual_f64(const PlumeGridInfo* info, const float* q, const float* q_lo, const float* rhs,
                       float* residual, double* scratch, double* norms, void* stream);
int plume_multigrid_correct(const PlumeLevel* levels, int32_t level_count, int32_t sweeps, float* pressure,
                            float* pressure_lo, void* stream);

/* conserve.py:45-52 SmokeBudget.hold + reduce.py:28-38 TripleSum, on the device: totals of data, hat and next
 * (each line summed along x in float, the lines added in double in a fixed order), the held factor
 * max(sl, min(mc, before)) / mc (1 when mc <= 0) stored as float in *factor, and next *= factor.
 * `sums` needs plume_smoke_scratch_doubles(info) doubles. If `totals_out` is not null the three totals are
 * also copied to it (device memory, 3 doubles). */
int plume_smoke_scratch_doubles(const PlumeGridInfo* info);
long long plume_advect_scratch_floats(const PlumeGridInfo* info);
int plume_smoke_budget(const PlumeGridInfo* info, const float* data, const float* hat, float* next,
                       double* sums, float* factor, double* totals_out, void* stream);

/* No counterpart in the reference. The smoke budget for callers that cannot allocate device memory: a host
 * engine that passes in only the field arrays it owns while its allocator is locked or budgeted, or code that
 * runs where a cudaMalloc would synchronise the device or is not allowed. Same result as plume_smoke_budget
 * (next *= factor, optional device totals_out of 3 doubles), but the partial sums and the factor live in a
 * fixed 96 KiB array inside the library, reserved on every device that loads it until the process exits; no
 * memory is allocated or freed by the call. Limit: ny * nz <= 1048576 (1 << 20) lines, else PLUME_ERR_INVALID.
 * The first call on a device looks up the array's device address on that device (make it before any stream
 * capture). That address is kept for the life of the process: after cudaDeviceReset, or a release and
 * re-creation of the device's primary context, the library's module reloads and the kept address is stale, so
 * a process that resets a device must not call this entry point again on it. All calls share the one array:
 * calls that overlap on the GPU (other streams, other threads) race and must be ordered by the caller. */
int plume_smoke_budget_static(const PlumeGridInfo* info, const float* data, const float* hat, float* next,
                              double* totals_out, void* stream);

/* No counterpart in the reference. Which of plume_step's advections use the fused passes below: bit 0 the
 * velocity (plume_maccormack_velocity), bit 1 smoke and temperature (plume_maccormack_scalars); the others use
 * the two-pass kernels of plume_advect_maccormack, whose blends keep the reference's a*(1-t) + b*t. Default 1
 * (fused velocity, two-pass scalars: the fastest measured on B200). A process-wide switch. */
int plume_use_fused_advection(int32_t mask);

/* advect.py:59-68 advect_maccormack of u, v and w by themselves (the step's velocity advection,
 * stepper.py:46-52), in one fused pass: the forward semi-Lagrangian value is kept in on-chip memory and never
 * stored, and the limiter's range comes from the same samples. Trilinear blends are fused multiply-adds, so
 * values agree with the three-pass form to about an ulp. next arrays must not alias the data arrays. */
int plume_maccormack_velocity(const PlumeGridInfo* info, const float* u, const float* v, const float* w,
                              float* u_next, float* v_next, float* w_next, float dt_over_cell, void* stream);

/* advect.py:59-68 advect_maccormack of smoke and temperature by (u, v, w) in one fused pass (they share every
 * trace), with the smoke budget's line sums (reduce.py:12-25) of data, hat and next taken on the way:
 * `scratch` needs plume_maccormack_scratch_floats(info) floats and `sums` plume_smoke_scratch_doubles(info)
 * doubles; if `totals_out` is not null, the three totals (before, semi-Lagrangian, MacCormack; 3 doubles on the
 * device) are written there. Values beyond open faces are smoke_outside and heat_outside when uses_outside is
 * 1 (sample.py:64-71). next is not rescaled: plume_step applies the held factor afterwards. */
long long plume_maccormack_scratch_floats(const PlumeGridInfo* info);
int plume_maccormack_scalars(const PlumeGridInfo* info, const float* u, const float* v, const float* w,
                             const float* smoke, const float* temperature, float* smoke_next, float* temperature_next,
                             float dt_over_cell, float smoke_outside, float heat_outside, int32_t uses_outside,
                             float* scratch, double* sums, double* totals_out, void* stream);

/* reduce.py:28-38 TripleSum: the three totals (device, 3 doubles) without scaling. */
int plume_triple_sum(const int32_t shape[3], const float* a, const float* b, const float* c, double* sums,
                     double* totals_out, void* stream);

/* dissipate.py:18-24 dissipate (dissipate_kernel). */
int plume_dissipate(const PlumeGridInfo* info, float* smoke, float* temperature, float smoke_keep,
                    float heat_keep, float ambient_k, void* stream);

/* step_cap.py:50-55 StepCap.grid_speed: largest |u|, |v|, |w| (stored as `storage`) into *speed (device float). */
int plume_grid_speed(const PlumeGridInfo* info, const void* u, const void* v, const void* w, int32_t storage,
                     float* speed, void* stream);

/* stepper.py:28-44 Stepper.step: one whole substep. On return the caller swaps data/next of u, v, w, smoke and
 * temperature, as the reference's AdvectedField.swap does. */
int plume_step(const PlumeStepState* state, const PlumeStepParams* params, void* stream);

/* ---- render ------------------------------------------------------------------------------------------ */

/* light_volume.py:18-51 light_volume_kernel. `bricks` (optional, plume_brick_floats() floats) is scratch for a
 * map of each 4x4x4 brick's largest smoke value; with it, runs of samples whose eight corners are all <= 0 are
 * stepped over, which leaves every result bit unchanged (they add exactly 0). */
long long plume_brick_floats(const int32_t shape[3]);
int plume_light_volume(const int32_t shape[3], const void* smoke, int32_t storage, const float toward_light[3],
                       float cell_m, float opacity_per_density, float* light, float* bricks, void* stream);

/* plume_light_volume for a camera march of the same smoke (frame_renderer.py:53-63 prepare then march): only
 * the cells such a march reads get their light_volume_kernel value, bit for bit; every other cell gets 1.
 * A march reads the light at the corners of samples with smoke > 0, so a cell is read only when one of the 27
 * cells around it (itself included) holds smoke > 0. `bricks` is required and is left holding the smoke's brick
 * map. */
int plume_march_light_volume(const int32_t shape[3], const void* smoke, int32_t storage, const float toward_light[3],
                             float cell_m, float opacity_per_density, float* light, float* bricks, void* stream);

/* normal_field.py:52-61 NormalField.compute (blur_axis_kernel x 3 + gradient_kernel); gradient is
 * (n0, n1, n2, 3). */
int plume_normal_field(const int32_t shape[3], const void* smoke, int32_t storage, float* blurred, float* scratch,
                       float* gradient, const float* weights_host, int32_t radius, void* stream);

/* The brick map of a field (largest value of each 4x4x4 brick and the next cell past it on each axis). */
int plume_brick_max(const int32_t shape[3], const void* field, int32_t storage, float* bricks, void* stream);

/* raymarch.py:86-140 raymarch_kernel; image is (height, width, 5). gradient/light are the unused pass's
 * 1-cell stand-in when not read (frame_renderer.py:29-35). `bricks` (optional, plume_brick_floats() floats)
 * is scratch for the march's brick map of the smoke and temperature, built by this call; with it, samples with
 * no smoke skip their smoke sample and runs of samples with neither smoke nor glow are stepped over. Terms
 * that are exactly 0 are never evaluated, so the image is the same with or without it. */
int plume_raymarch(const PlumeGridInfo* info, const void* smoke, const void* temperature, int32_t storage,
                   const float* gradient, const int32_t gradient_shape[3], const float* light,
                   const int32_t light_shape[3], const PlumeViewParams* view, const PlumeLookParams* look, float* image,
                   int32_t height, int32_t width, float* bricks, void* stream);

/* ---- sheet assembly and the numbers file (sheet/assemble.py:39-77, report/numbers.py:42-100) ------------- */
/* Raw frames are one (frames, height, width, 5) float32 device array; finished frames (frames, size, size, 5)
 * double; quantised frames (frames, size, size, 4) bytes. Scratch and outputs are caller-owned device memory. */

/* crop.py:29-43 content_box: *heat_key = the order key of the largest heat; box = (left, top, right, bottom),
 * right and bottom exclusive (right <= left when no frame shows anything). */
int plume_sheet_content_box(const float* raw, int32_t frames, int32_t height, int32_t width, uint32_t* heat_key,
                            int32_t* box, void* stream);

/* resample.py:16-41 resample_frame: the crop square of every frame, padded by `pad` empty pixels, resampled to
 * out x out with the bicubic two-pass filter of the per-pass tap tables (first source index, window length,
 * ksize normalised double weights per output index; source indices are padded-image indices); the horizontal
 * pass covers padded rows [row_first, row_first + rows). temp: frames * 5 * rows * out floats. */
int plume_sheet_resample(const float* raw, int32_t frames, int32_t height, int32_t width, int32_t pad,
                         const float empty[5], const int32_t* h_first, const int32_t* h_count, const double* h_weights,
                         int32_t h_ksize, const int32_t* v_first, const int32_t* v_count, const double* v_weights,
                         int32_t v_ksize, int32_t row_first, int32_t rows, int32_t out, int32_t shade_layout,
                         float* temp, double* frame, void* stream);

/* soften.py:21-49 blur: `channels` planes starting at `offset` of `stride` interleaved doubles per pixel,
 * blurred along rows then columns (edges extended) with 2 * radius + 1 device weights; dst may equal src. */
int plume_sheet_blur(const double* src, double* dst, double* scratch, int32_t frames, int32_t size, int32_t channels,
                     int32_t stride, int32_t offset, const double* weights, int32_t radius, void* stream);

/* soften.py:52-60 _renormalize (normal layout). */
int plume_sheet_renormalize(double* frame, int32_t frames, int32_t size, void* stream);

/* shade.py:22-42 ease_thin_pixels, given `blurred`: a frame-shaped array whose thickness and shade-times-
 * thickness channels hold those planes blurred by the neighbourhood Gaussian; sums: 2 doubles per frame. */
int plume_sheet_ease(double* frame, const double* blurred, double* sums, int32_t frames, int32_t size,
                     double fade_thickness, void* stream);

/* The largest value of `channel` over every pixel of every frame whose thickness is >= floor:
 * out[0] = that value (0 when none), out[1] = 1 if any pixel qualified. key, any: scratch. */
int plume_sheet_channel_max(const double* frame, int32_t frames, int32_t size, int32_t channel, double floor,
                            unsigned long long* key, int32_t* any, double* out, void* stream);

/* quantize.py:20-39 quantize, then assemble.py:70-73: *touched = 1 when a frame has a non-zero R or G byte
 * within `gutter` pixels of its edge. */
int plume_sheet_quantize(const double* frame, int32_t frames, int32_t size, double heat_divisor,
                         double shade_divisor, int32_t shade_layout, int32_t gutter, uint8_t* rgba, int32_t* touched,
                         void* stream);

/* pack.py:13-20 pack: frames in rows of `columns`, unused slots zero; sheet is (rows * size, columns * size, 4). */
int plume_sheet_pack(const uint8_t* rgba, int32_t frames, int32_t size, int32_t columns, uint8_t* sheet, void* stream);

/* numbers.py:80-100 per frame (9 int64s): covered count (G >= covered_level), covered box left, top, right,
 * bottom (right/bottom exclusive), R and G byte sums over covered pixels, G byte sum, largest R byte. */
int plume_sheet_measure(const uint8_t* rgba, int32_t frames, int32_t size, int32_t covered_level, long long* stats,
                        void* stream);

/* ---- live viewer compute (view/viewport.py, view/slice_plane.py, view/live_run.py, view/frame_cache.py) ---- */

/* LookInputs (viewport.py:50-59): view 0 look, 1 heat, 2 thickness, 3 shade (the normal in the normal layout);
 * toward_light in the drawn camera's space; background linear RGB. */
typedef struct PlumeLookInputs {
  int32_t view;
  int32_t shade_layout;
  float heat_divisor;
  float shade_divisor;
  float shade_depth;
  float ambient;
  float toward_light[3];
  float background[3];
} PlumeLookInputs;

/* viewport.py:78-113 look_kernel: a raw march image (height, width, 5) to display bytes (height, width, 4);
 * smoke_ramp/emission_ramp: ramp_n linear RGB float triples; srgb: srgb_n bytes of the sRGB curve. */
int plume_view_look(const float* raw, int32_t height, int32_t width, const float* smoke_ramp,
                    const float* emission_ramp, int32_t ramp_n, const uint8_t* srgb, int32_t srgb_n,
                    const PlumeLookInputs* inputs, uint8_t* out, void* stream);

/* viewport.py:116-140 center_depth_kernel: *result (device) = distance along the ray where the march's
 * thickness first reaches threshold, -1 if never. */
int plume_view_center_depth(const float* smoke, const PlumeGridInfo* info, const float origin[3],
                            const float direction[3], float opacity_per_density, float threshold, float* result,
                            void* stream);

/* vorticity.py:17-22 center_velocity_kernel: centers is (nx, ny, nz, 3). */
int plume_view_center_velocity(const PlumeGridInfo* info, const float* u, const float* v, const float* w,
                               float* centers, void* stream);

/* vorticity.py:25-45 curl_kernel on a cell-centred (nx, ny, nz, 3) field (the slice plane's swirl). */
int plume_view_curl(const PlumeGridInfo* info, const float* centers, float* curl, void* stream);

/* slice_plane.py:104-107 speed_kernel: out[c] = |vectors[c]|. */
int plume_view_speed(const float* vectors, long long cells, float* out, void* stream);

/* slice_plane.py:110-137 slice_kernel over the display bytes `image` (height, width, 4), in place. */
int plume_view_slice(const PlumeViewParams* view, const PlumeGridInfo* info, int32_t axis, float coordinate_m,
                     const float* values, float low, float high, const float* ramp, int32_t ramp_n, uint8_t* image,
                     int32_t height, int32_t width, void* stream);

/* live_run.py:42-57 boundary_layer_kernel: layers is (6, S, S) with S the largest dimension. */
int plume_view_boundary_layers(const float* smoke, const int32_t shape[3], float* layers, void* stream);

/* frame_cache.py:26-50 narrow/widen kernels: float32 <-> IEEE half (round to nearest even). */
int plume_view_narrow(const float* src, void* dst, long long count, void* stream);
int plume_view_widen(const void* src, float* dst, long long count, void* stream);

/* ---- the smoke path's adjoint (no counterpart in the reference, which has no derivatives) ------------------ */
/* For fitting a smoke source field to a target thickness image: the derivative of a thickness loss through the
 * smoke path of the step (source add, MacCormack advection by a given velocity, smoke budget, dissipation) and
 * the thickness march. Exact when the velocity does not depend on the smoke (forces.smoke_weight = 0). */

/* smoke[corner + idx] += scale * source[idx] over the source box's cells inside the grid (a source field). */
int plume_add_source(float* smoke, const int32_t shape[3], const float* source, const int32_t source_shape[3],
                     const int32_t corner[3], float scale, void* stream);

/* grad[idx] += scale * a_smoke[corner + idx]: the source field's share of a smoke derivative. */
int plume_source_grad(const float* a_smoke, const int32_t shape[3], float* grad, const int32_t source_shape[3],
                      const int32_t corner[3], float scale, void* stream);

/* One substep of the smoke path backwards. Inputs: the velocity the smoke was advected by, the advected smoke
 * `data`, its forward pass `hat` and correction `next_pre` (before the budget's scale), the budget's totals
 * (before, semi-Lagrangian, MacCormack; 3 device doubles), dissipation's keep factor, and a_out = the derivative
 * with respect to the substep's output smoke. Writes a_data = the derivative with respect to `data`; a_next,
 * a_hat are scratch of the field's size, partial >= 1024 doubles, coeffs 4 doubles. */
int plume_smoke_adjoint(const PlumeGridInfo* info, const float* u, const float* v, const float* w, const float* data,
                        const float* hat, const float* next_pre, const double* totals, float dt_over_cell, float keep,
                        const float* a_out, float* a_next, float* a_hat, float* a_data, double* partial,
                        double* coeffs, void* stream);

/* The orthographic march's thickness (raymarch.py:86-140) of `smoke` for `view`, written to thickness
 * (height, width); *loss += sum (thickness - target)^2; a_smoke += d loss / d smoke. */
int plume_thickness_adjoint(const PlumeGridInfo* info, const PlumeViewParams* view, float opacity, const float* smoke,
                            const float* target, int32_t height, int32_t width, float* thickness, double* loss,
                            float* a_smoke, void* stream);

/* ---- the velocity path of the adjoint (no counterpart in the reference, which has no derivatives) ----------
 * plume_maccormack_adjoint: for next = MacCormack(data) advected by (u, v, w) (advect.py:59-68) with `hat` the
 * forward semi-Lagrangian values, adds d loss / d data to a_data given a_next; a_hat is the derivative of hat
 * (it must hold any derivative known for hat already, e.g. the smoke budget's term). With a_u, a_v, a_w (all or
 * none) it also adds the derivatives with respect to the advecting velocity, through both traces' endpoints
 * and midpoints. Any field shape and offset (cells or faces). Atomic adds: last bits vary between runs.
 * plume_buoyancy_adjoint (forces.py:13-23): a_temperature (and a_smoke with a smoke weight) receive a_v's share;
 * *grad_heat_buoyancy (device double) += d loss / d heat_buoyancy.
 * plume_drag_adjoint (forces.py:34-48): *grad_drag += d loss / d drag_per_s (u, v, w: the velocity before drag,
 * keep = exp(-drag dt)), then a_u, a_v, a_w *= keep.
 * plume_emit_adjoint (emitters.py:90-121): the temperature and velocity blends scale their derivatives by 1 - b. */
/* plume_budget_adjoint (conserve.py:45-52 then dissipate.py:10-15 for the smoke): given a_out, the derivative
 * of the smoke after the budget's rescale and dissipation by `keep`, writes a_next (of next before the rescale)
 * and starts a_data and a_hat with the rescale factor's uniform terms (from the three totals). `partial` needs
 * 1024 doubles, `coeffs` 4. */
int plume_budget_adjoint(const PlumeGridInfo* info, const float* next_pre, const double* totals, float keep,
                         const float* a_out, float* a_next, float* a_data, float* a_hat, double* partial,
                         double* coeffs, void* stream);
int plume_maccormack_adjoint(const PlumeGridInfo* info, const int32_t shape[3], const float offset[3], const float* data,
                             const float* hat, const float* u, const float* v, const float* w, const float* a_next,
                             float* a_data, float* a_hat, float* a_u, float* a_v, float* a_w, float dt_over_cell,
                             float outside, int32_t uses_outside, void* stream);
int plume_buoyancy_adjoint(const PlumeGridInfo* info, const float* a_v, const float* smoke, const float* temperature,
                           float* a_smoke, float* a_temperature, float gravity, float heat_buoyancy,
                           float smoke_weight, float ambient_k, float dt, double* grad_heat_buoyancy, void* stream);
int plume_drag_adjoint(const PlumeGridInfo* info, float* a_u, float* a_v, float* a_w, const float* u, const float* v,
                       const float* w, const float wind[3], float keep, float dt, double* grad_drag, void* stream);
/* plume_confinement_adjoint (vorticity.py:17-84, VorticityConfinement.apply): given a_u, a_v, a_w, the derivative
 * of the velocity after confinement, adds the confinement's transposed Jacobian so that they become the
 * derivative of the velocity before it (u, v, w: that velocity, recorded by the caller), and adds
 * d loss / d strength to *grad_strength (device double). `scratch` holds
 * plume_confinement_adjoint_scratch_floats(info) floats (10 per cell). No atomics on the face arrays. */
int plume_confinement_adjoint(const PlumeGridInfo* info, const float* u, const float* v, const float* w, float* a_u,
                              float* a_v, float* a_w, float strength, float dt, float* scratch, double* grad_strength,
                              void* stream);
long plume_confinement_adjoint_scratch_floats(const PlumeGridInfo* info);
int plume_emit_adjoint(const PlumeGridInfo* info, float* a_temperature, float* a_u, float* a_v, float* a_w,
                       const PlumeEmitter* emitters, int32_t count, int32_t seed, float time_s, float dt, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PLUME_B200_H */
