/* oceanlib-b200 - C ABI of the B200 (sm_100a) ocean library.
 *
 * Part 1 re-declares the reference oceanlib C ABI (include/ocean/ocean.h of
 * DarshanVShah/oceanlib) with identical names, struct layouts, status codes
 * and NULL-handle behaviour, so a binding written against the reference binds
 * this library unchanged. Each declaration cites the reference line it
 * replaces. Part 2 adds entry points that only a GPU library needs: device
 * buffer access, asynchronous updates on a caller's stream, batched updates
 * of many oceans in one launch, batched world queries, and persistent foam.
 *
 * All compute runs on the GPU; there is no CPU fallback. A handle is created
 * on the CUDA device that is current on the calling thread.
 */
#ifndef OCEAN_B200_H
#define OCEAN_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__cplusplus)
extern "C" {
#endif

#if defined(_WIN32)
#define OCEAN_API __declspec(dllexport)
#else
#define OCEAN_API __attribute__((visibility("default")))
#endif

/* =========================================================================
 * Part 1: the reference C ABI (drop-in)
 * ========================================================================= */

/* Opaque handle. include/ocean/ocean.h:35 */
typedef struct ocean_sim ocean_sim;

/* include/ocean/ocean.h:37-42. Values are part of the ABI; new codes are only
 * ever appended. */
typedef enum ocean_status {
    OCEAN_OK                  = 0,
    OCEAN_ERROR_INVALID_ARG   = 1,
    OCEAN_ERROR_OUT_OF_MEMORY = 2,
    OCEAN_ERROR_UNKNOWN       = 3,
    OCEAN_ERROR_DEVICE        = 4, /* a CUDA call failed (appended)          */
    OCEAN_ERROR_TIMEOUT       = 5  /* a bounded device wait gave up          */
} ocean_status;

/* include/ocean/ocean.h:46 */
OCEAN_API const char* ocean_status_string(ocean_status status);

/* include/ocean/ocean.h:53-63. The hook is called exactly four times per
 * ocean_update, each with count == 1, and every call launches and completes
 * one device stage (row pass, column pass, displacement copy-back, normal
 * copy-back). */
typedef void (*ocean_task_fn)(void* ctx, uint32_t index);
typedef void (*ocean_parallel_for_fn)(void* user, ocean_task_fn task, void* ctx,
                                      uint32_t count);

/* include/ocean/ocean.h:75-83. Never grows (embedded by value below). */
typedef struct ocean_spectrum_desc {
    float wind_speed;
    float fetch;
    float wind_direction;
    float peak_enhancement;
    float swell;
    float small_wave_cutoff;
    float gravity;
} ocean_spectrum_desc;

/* include/ocean/ocean.h:85-134. 96 bytes on LP64; struct_size prefix
 * versioning: a smaller struct_size takes defaults for the missing tail, zero
 * or a larger one is OCEAN_ERROR_INVALID_ARG. thread_count is accepted and
 * ignored (the GPU does the work). */
typedef struct ocean_desc {
    size_t struct_size;
    uint32_t size;
    float    patch_length;
    ocean_spectrum_desc spectrum;
    float    choppiness;
    float    foam_threshold;
    uint64_t seed;
    ocean_parallel_for_fn parallel_for;
    void*                 parallel_for_user;
    uint32_t              thread_count;
    float    water_depth;
    int32_t  compute_velocity;
} ocean_desc;

/* include/ocean/ocean.h:139 */
OCEAN_API void ocean_desc_init(ocean_desc* desc);

/* include/ocean/ocean.h:155-160. Host pointers into a pinned mirror that
 * ocean_update refreshes before it returns. */
typedef struct ocean_buffers {
    const float* displacement;
    const float* normal;
    uint32_t     size;
    float        patch_length;
} ocean_buffers;

/* include/ocean/ocean.h:162-170 */
typedef struct ocean_surface {
    float height;
    float offset_x;
    float offset_z;
    float normal_x;
    float normal_y;
    float normal_z;
    float foam;
} ocean_surface;

/* include/ocean/ocean.h:181. Allocates device memory, builds h0(k) on the
 * device and evaluates t = 0. NULL + status on failure. */
OCEAN_API ocean_sim* ocean_create(const ocean_desc* desc, ocean_status* out_status);

/* include/ocean/ocean.h:184. NULL tolerated. */
OCEAN_API void ocean_destroy(ocean_sim* sim);

/* include/ocean/ocean.h:193. Absolute time; a pure function of
 * (seed, desc, time). Runs the device frame and refreshes the host mirror
 * synchronously. No allocation. */
OCEAN_API void ocean_update(ocean_sim* sim, double time);

/* include/ocean/ocean.h:195 */
OCEAN_API ocean_buffers ocean_get_buffers(const ocean_sim* sim);

/* include/ocean/ocean.h:197 */
OCEAN_API double ocean_get_time(const ocean_sim* sim);

/* include/ocean/ocean.h:205. The reference's 4-step fixed-point inversion,
 * run by the GPU query kernel on the device outputs (one query is a launch
 * plus a copy; use ocean_sample_many for many). */
OCEAN_API float ocean_height_at(const ocean_sim* sim, float world_x, float world_z);

/* include/ocean/ocean.h:215 (frozen: returned by value). */
OCEAN_API ocean_surface ocean_sample_at(const ocean_sim* sim, float world_x, float world_z);

/* include/ocean/ocean.h:223-234 */
typedef struct ocean_surface_ex {
    float height;
    float offset_x;
    float offset_z;
    float normal_x;
    float normal_y;
    float normal_z;
    float foam;
    float velocity_x;
    float velocity_y;
    float velocity_z;
} ocean_surface_ex;

/* include/ocean/ocean.h:234 */
OCEAN_API void ocean_sample_ex(const ocean_sim* sim, float world_x, float world_z,
                               ocean_surface_ex* out);

/* include/ocean/ocean.h:240 */
OCEAN_API const float* ocean_get_velocity(const ocean_sim* sim);

/* include/ocean/ocean.h:249. Reports "sm_100a" by default, or the level name
 * last forced with ocean_force_simd_level. */
OCEAN_API const char* ocean_simd_level(void);

/* include/ocean/ocean.h:262. "scalar" (and "sse2", "avx2", "neon", "exact")
 * select the exact FFT form, whose results are bit-identical to the
 * reference's scalar kernels; "fast" selects the FMA form and "precise" the
 * FP64-block form (OCEAN_FFT_PRECISE). Affects handles
 * created after the call. Returns the reference's spelling of the level for
 * the reference names, so "scalar" returns "scalar". */
OCEAN_API const char* ocean_force_simd_level(const char* name);

/* include/ocean/ocean.h:265. Reports 1.0.0, the reference ABI version this
 * library implements. */
OCEAN_API void ocean_version(uint32_t* major, uint32_t* minor, uint32_t* patch);

/* -------------------------------------------------------------------------
 * Local interaction (iWave), include/ocean/ocean.h:267-415. The field lives
 * on the GPU; ocean_interaction_get_buffers returns a pinned host mirror that
 * ocean_interaction_update / _recenter refresh before returning.
 * ------------------------------------------------------------------------- */

/* include/ocean/ocean.h:285 */
typedef struct ocean_interaction ocean_interaction;

/* include/ocean/ocean.h:290-293 */
typedef enum ocean_obstruction {
    OCEAN_OBSTRUCTION_NEUMANN   = 0,
    OCEAN_OBSTRUCTION_DIRICHLET = 1
} ocean_obstruction;

/* include/ocean/ocean.h:295-298 */
typedef enum ocean_source_kind {
    OCEAN_SOURCE_IMPULSE    = 0,
    OCEAN_SOURCE_CONTINUOUS = 1
} ocean_source_kind;

/* include/ocean/ocean.h:300-318; same struct_size rules as ocean_desc.
 * thread_count and the parallel_for hook are accepted and ignored. */
typedef struct ocean_interaction_desc {
    size_t struct_size;
    uint32_t size;
    float    extent;
    uint32_t kernel_radius;
    float    damping;
    uint32_t absorb_cells;
    float    fixed_dt;
    uint32_t max_substeps;
    uint32_t max_sources;
    float    gravity;
    float    water_depth;
    int32_t  obstruction;
    ocean_parallel_for_fn parallel_for;
    void*                 parallel_for_user;
    uint32_t              thread_count;
} ocean_interaction_desc;

/* include/ocean/ocean.h:320 */
OCEAN_API void ocean_interaction_desc_init(ocean_interaction_desc* desc);
/* include/ocean/ocean.h:322 */
OCEAN_API ocean_interaction* ocean_interaction_create(const ocean_interaction_desc* desc,
                                                      ocean_status* out_status);
/* include/ocean/ocean.h:324 */
OCEAN_API void ocean_interaction_destroy(ocean_interaction* field);

/* include/ocean/ocean.h:335-345 */
typedef struct ocean_disturbance {
    float world_x;
    float world_z;
    float radius;
    float strength;
    float velocity_y;
    float velocity_x;
    float velocity_z;
    int32_t kind;
} ocean_disturbance;

/* include/ocean/ocean.h:349 */
OCEAN_API void ocean_interaction_add(ocean_interaction* field, const ocean_disturbance* d);
/* include/ocean/ocean.h:351 */
OCEAN_API uint64_t ocean_interaction_dropped(const ocean_interaction* field);
/* include/ocean/ocean.h:356. Substeps, sources and the stencil all run on the
 * device; the host mirror is refreshed before returning. */
OCEAN_API void ocean_interaction_update(ocean_interaction* field, float dt);
/* include/ocean/ocean.h:362 */
OCEAN_API int32_t ocean_interaction_recenter(ocean_interaction* field, float world_x,
                                             float world_z);
/* include/ocean/ocean.h:367 */
OCEAN_API void ocean_interaction_set_obstruction(ocean_interaction* field, const uint8_t* mask);

/* include/ocean/ocean.h:369-381 */
typedef struct ocean_interaction_buffers {
    const float* field;
    uint32_t     size;
    float        extent;
    float        origin_x;
    float        origin_z;
} ocean_interaction_buffers;

/* include/ocean/ocean.h:383 */
OCEAN_API ocean_interaction_buffers ocean_interaction_get_buffers(const ocean_interaction* field);

/* include/ocean/ocean.h:386-391 */
typedef struct ocean_interaction_sample {
    float height;
    float slope_x;
    float slope_z;
    float velocity_y;
} ocean_interaction_sample;

/* include/ocean/ocean.h:393, :396 (GPU query kernel) */
OCEAN_API void ocean_interaction_sample_at(const ocean_interaction* field, float world_x,
                                           float world_z, ocean_interaction_sample* out);
OCEAN_API float ocean_interaction_height_at(const ocean_interaction* field, float world_x,
                                            float world_z);
/* include/ocean/ocean.h:403, :404, :408 */
OCEAN_API float ocean_interaction_fixed_dt(const ocean_interaction* field);
OCEAN_API float ocean_interaction_dt_limit(const ocean_interaction* field);
OCEAN_API float ocean_interaction_dispersion_error(const ocean_interaction* field);
/* include/ocean/ocean.h:413 */
OCEAN_API void ocean_sample_combined(const ocean_sim* sim, const ocean_interaction* field,
                                     float world_x, float world_z, ocean_surface_ex* out);

/* =========================================================================
 * Part 2: GPU entry points (no reference counterpart; new symbols only)
 * ========================================================================= */

/* Device pointers (valid until destroy). RGBA32F layouts as in ocean_buffers;
 * foam is N*N floats. Members are NULL when the feature is off. */
typedef struct ocean_device_buffers {
    float*   displacement;
    float*   normal;
    float*   velocity;
    float*   foam;
    uint32_t size;
    float    patch_length;
} ocean_device_buffers;

/* FFT arithmetic forms. */
typedef enum ocean_fft_form {
    OCEAN_FFT_EXACT = 0, /* radix-2 Stockham in the reference's operation order,
                            no FMA: bit-identical to the reference           */
    OCEAN_FFT_FAST  = 1, /* same dataflow with fused multiply-adds           */
    OCEAN_FFT_TENSOR = 2, /* four-step DFT on the tensor cores (tcgen05):
                            operands cut into four signed 8-bit digits held
                            as FP16, exact digit products, levels combined
                            in FP32; N = 64, 128, 256 and 512 */
    OCEAN_FFT_PRECISE = 3 /* the radix-2 dataflow with each register block of
                            stages computed in FP64 and stored in FP32 once:
                            within 2e-6 of FP64, every size */
} ocean_fft_form;

/* `count` unnormalised inverse DFTs (sign +, as src/core/fft.cpp) of
 * complex sequences of length `size` (a power of two in [16, 1024]; 64 to
 * 512 for the tensor form), in the given form. `input` and
 * `output` are DEVICE arrays of count * size interleaved (re, im) floats;
 * the call waits for the result. For accuracy checks of the forms. */
OCEAN_API ocean_status ocean_dft_batch(uint32_t size, uint32_t count, int32_t form, const float* input,
                                       float* output, void* stream);

/* Device pointers of a single ocean. */
OCEAN_API ocean_status ocean_get_device_buffers(const ocean_sim* sim, ocean_device_buffers* out);

/* Run the frame on `stream` (a cudaStream_t; NULL = the handle's own stream)
 * and return without waiting or refreshing the host mirror. */
OCEAN_API ocean_status ocean_update_async(ocean_sim* sim, double time, void* stream);

/* Copy the current device outputs into the host mirror (synchronous). */
OCEAN_API ocean_status ocean_refresh_host(ocean_sim* sim);

/* Batched world queries on the device: `xz` holds count (x, z) pairs and
 * `out` count ocean_surface_ex records. Both are HOST arrays here; the call
 * copies them across and waits. Results are bit-identical to ocean_sample_ex
 * point by point. */
OCEAN_API ocean_status ocean_sample_many(const ocean_sim* sim, const float* xz, uint64_t count,
                                         ocean_surface_ex* out);

/* --- Persistent advected foam (reference: include/ocean/foam.hpp:38-142) - */

/* Mirrors ocean::FoamDesc (include/ocean/foam.hpp:38-74). */
typedef struct ocean_foam_desc {
    size_t   struct_size;
    float    decay;
    float    source_gain;
    float    advect_scale;
    float    wind_drift_x;
    float    wind_drift_z;
    float    fixed_dt;
    uint32_t max_substeps;
} ocean_foam_desc;

OCEAN_API void ocean_foam_desc_init(ocean_foam_desc* desc);

/* --- Batches: many independent oceans advanced by one launch per pass ---- */

typedef struct ocean_batch ocean_batch;

/* How a batch frame is scheduled on the device. */
typedef enum ocean_schedule {
    OCEAN_SCHEDULE_PERSISTENT = 0, /* one persistent launch per frame: CTAs pull
                                      row and column tasks from an ordered queue */
    OCEAN_SCHEDULE_CHUNKED    = 1  /* a row launch and a column launch per chunk */
} ocean_schedule;

typedef struct ocean_batch_desc {
    size_t            struct_size;
    const ocean_desc* oceans;          /* `count` descriptors, all the same size N */
    uint32_t          count;
    int32_t           fft_form;        /* ocean_fft_form                          */
    int32_t           persistent_foam; /* non-zero: a FoamField per ocean (needs
                                          compute_velocity on every ocean)        */
    ocean_foam_desc   foam;
    uint32_t          chunk;           /* oceans per row/column pass pair; 0 = auto
                                          (sized so the intermediate stays in L2) */
    int32_t           schedule;        /* ocean_schedule                            */
} ocean_batch_desc;

OCEAN_API void ocean_batch_desc_init(ocean_batch_desc* desc);
OCEAN_API ocean_batch* ocean_batch_create(const ocean_batch_desc* desc, ocean_status* out_status);
OCEAN_API void ocean_batch_destroy(ocean_batch* batch);
OCEAN_API uint32_t ocean_batch_count(const ocean_batch* batch);

/* Advance every ocean to its absolute time (times[i], or times[0] for all
 * when `per_ocean_times` is zero) and, when persistent foam is on, run the
 * foam accumulator by foam_dt. Asynchronous on `stream` (NULL = the batch's
 * own stream). No allocation. */
OCEAN_API ocean_status ocean_batch_update(ocean_batch* batch, const double* times,
                                          int32_t per_ocean_times, float foam_dt, void* stream);

/* The same frame, end to end for host callers: times come from host memory
 * and every ocean's outputs are copied into the caller's host arrays
 * (displacement, normal, and velocity / foam when present; each array holds
 * count * N*N*4 floats, foam count * N*N). Pinned host memory gives full
 * copy bandwidth. Returns when the copies are complete. */
OCEAN_API ocean_status ocean_batch_update_host(ocean_batch* batch, const double* times,
                                               int32_t per_ocean_times, float foam_dt,
                                               float* displacement, float* normal,
                                               float* velocity, float* foam);

/* As ocean_batch_update_host, with every output narrowed to RGBA16F on the
 * device (IEEE round-to-nearest-even, overflow to infinity) before the copy -
 * half the bytes. With persistent foam the displacement's alpha is the
 * persistent foam rather than the frame's Jacobian foam, as the reference
 * viewer's upload substitutes it (examples/viewer/ocean_view.cpp:830-862).
 * Arrays of count * N * N * 4 uint16 (binary16 bit patterns); any may be NULL. */
OCEAN_API ocean_status ocean_batch_update_host_rgba16(ocean_batch* batch, const double* times,
                                                      int32_t per_ocean_times, float foam_dt,
                                                      uint16_t* displacement, uint16_t* normal,
                                                      uint16_t* velocity);

/* The reference viewer's pack_rgba16 (examples/viewer/half.hpp:99-112) on the
 * device: `texels` RGBA32F texels of `src` to RGBA16F in `dst`, the alpha taken
 * from `alpha` (one float per texel) when it is not NULL. Device pointers;
 * queued on `stream` (a cudaStream_t). Bit-identical to the reference's
 * float_to_half, NaNs included. */
OCEAN_API ocean_status ocean_pack_rgba16(const float* src, const float* alpha, uint64_t texels,
                                         uint16_t* dst, void* stream);

OCEAN_API ocean_status ocean_batch_get_device_buffers(const ocean_batch* batch, uint32_t index,
                                                      ocean_device_buffers* out);

/* Number of foam substeps the last update ran (0..max_substeps). */
OCEAN_API uint32_t ocean_batch_last_foam_substeps(const ocean_batch* batch);

/* The rest of ocean::FoamField (include/ocean/foam.hpp:88-142) for a batch
 * with persistent foam; OCEAN_ERROR_INVALID_ARG without it. These are ordered
 * after the work queued on the batch's own stream; updates queued on another
 * stream must be complete first. */
/* FoamField::clear (src/foam.cpp:254-260): every ocean's foam to zero and the
 * substep accumulator reset (after a seek). Returns when done. */
OCEAN_API ocean_status ocean_batch_foam_clear(ocean_batch* batch);
/* FoamField::set_desc (src/foam.cpp:266-283): decay, source_gain,
 * advect_scale and the wind drift apply from the next update on; fixed_dt
 * and max_substeps keep the values the batch was created with. The stored
 * foam is untouched. */
OCEAN_API ocean_status ocean_batch_foam_set_desc(ocean_batch* batch, const ocean_foam_desc* desc);
/* FoamField::desc(): the descriptor in effect. */
OCEAN_API ocean_status ocean_batch_foam_get_desc(const ocean_batch* batch, ocean_foam_desc* out);
/* FoamField::foam_at (src/foam.cpp:291-305) at `count` world points of ocean
 * `index`: the same displacement inversion as ocean_sample_at, then the
 * periodic bilinear foam fetch. xz (count (x, z) pairs) and out (count
 * floats) are HOST arrays; returns when out is written. Bit-identical to the
 * reference point by point. */
OCEAN_API ocean_status ocean_batch_foam_at_many(const ocean_batch* batch, uint32_t index, const float* xz,
                                                uint64_t count, float* out);
/* FoamField::coverage (src/foam.cpp:307-313): mean foam of ocean `index`,
 * summed in double on the device in a fixed order (the reference sums in
 * index order; the two differ by double rounding only). */
OCEAN_API ocean_status ocean_batch_foam_coverage(const ocean_batch* batch, uint32_t index, double* out);

/* Waits for all work queued on the batch's own stream. Returns
 * OCEAN_ERROR_TIMEOUT (once) if a bounded device wait of the persistent
 * frame kernel gave up since the last check. */
OCEAN_API ocean_status ocean_batch_synchronize(ocean_batch* batch);

/* Device spectrum tables of ocean `index`, written to HOST memory as
 * n*n float2 h0(k) (re, im) followed by n*n float2 (omega, 1/|k|). For
 * parity checks of the device h0 generation. */
OCEAN_API ocean_status ocean_batch_read_spectrum(const ocean_batch* batch, uint32_t index,
                                                 float* h0, float* omega_kinv);

/* --- Ensembles: independent sea states of uneven size (no reference
 *     counterpart; the reference updates oceans one at a time) ------------ */

typedef struct ocean_ensemble ocean_ensemble;

/* Groups the oceans by size. Schedules of a frame: the sizes in sequence,
 * each size's persistent kernel on its own stream concurrently with SM shares
 * (by estimated or by measured cost; the three-pass schedule at N = 2048 and
 * 4096), or - when every size is 32..1024, all with the same velocity flag,
 * in an FP32 form - one persistent launch whose work queue holds every
 * size's tasks. With autotune != 0 the schedule is chosen by timing each
 * candidate on this GPU at creation (the one launch unless another schedule
 * is more than 3 % faster: concurrent launches vary from run to run);
 * otherwise it is the concurrent one. */
OCEAN_API ocean_ensemble* ocean_ensemble_create(const ocean_desc* oceans, uint32_t count,
                                                int32_t autotune, ocean_status* out_status);
/* As ocean_ensemble_create, in a given ocean_fft_form instead of the
 * process-wide one. With OCEAN_FFT_TENSOR the sizes the tensor-core form
 * covers (64 to 512) run on it and the others (16, 32, 1024) in the exact
 * FP32 form; ocean_ensemble_describe names them. The tensor-core form runs
 * the sequential or concurrent schedules (the one-launch schedule is FP32). */
OCEAN_API ocean_ensemble* ocean_ensemble_create_form(const ocean_desc* oceans, uint32_t count,
                                                     int32_t autotune, int32_t fft_form,
                                                     ocean_status* out_status);
OCEAN_API void ocean_ensemble_destroy(ocean_ensemble* ensemble);
OCEAN_API uint32_t ocean_ensemble_count(const ocean_ensemble* ensemble);
/* All oceans to absolute time `time`, asynchronously on `stream` (NULL = the
 * ensemble's stream). */
OCEAN_API ocean_status ocean_ensemble_update(ocean_ensemble* ensemble, double time, void* stream);
/* Waits for the ensemble's stream; OCEAN_ERROR_TIMEOUT (once) if a bounded
 * device wait of the one-launch schedule gave up. */
OCEAN_API ocean_status ocean_ensemble_synchronize(ocean_ensemble* ensemble);
/* Forces a schedule: 0 sizes in sequence, 1 concurrent with SM shares by the
 * work estimate, 2 one launch for every size (OCEAN_ERROR_INVALID_ARG where
 * the sizes do not qualify). */
OCEAN_API ocean_status ocean_ensemble_set_schedule(ocean_ensemble* ensemble, int32_t schedule);
/* The schedule in use: 0, 1 or 2 as above (-1 for NULL). */
OCEAN_API int32_t ocean_ensemble_schedule(const ocean_ensemble* ensemble);
/* With enable != 0 (the default) each update replays one CUDA graph of the
 * whole frame - the time upload, the fork onto one stream per size, every
 * size's persistent launch and the join - captured at the first update under
 * the schedule the autotuner chose; with 0, each update issues the calls. */
OCEAN_API ocean_status ocean_ensemble_set_graph(ocean_ensemble* ensemble, int32_t enable);
OCEAN_API ocean_status ocean_ensemble_device_buffers(const ocean_ensemble* ensemble, uint32_t index,
                                                     ocean_device_buffers* out);
/* The chosen schedule in words (with the timings that chose it); returns the
 * full length, writes at most capacity - 1 characters and a terminator. */
OCEAN_API uint64_t ocean_ensemble_describe(const ocean_ensemble* ensemble, char* buf,
                                           uint64_t capacity);

/* --- Cascades (reference: CascadeStack, include/ocean/cascade.hpp:45-92,
 *     C++ only there; a C API is the reference's planned v1.1 item) -------- */

typedef struct ocean_cascade ocean_cascade;

/* `count` levels (at most 8), each an ordinary ocean descriptor; levels of
 * equal size advance together in one launch. Evaluates t = 0. */
OCEAN_API ocean_cascade* ocean_cascade_create(const ocean_desc* levels, uint32_t count,
                                              ocean_status* out_status);
/* As ocean_cascade_create, in a given ocean_fft_form instead of the
 * process-wide one (OCEAN_FFT_TENSOR: every level of N = 64 to 512;
 * other sizes give OCEAN_ERROR_INVALID_ARG). Queries are unchanged. */
OCEAN_API ocean_cascade* ocean_cascade_create_form(const ocean_desc* levels, uint32_t count,
                                                   int32_t fft_form, ocean_status* out_status);
OCEAN_API void ocean_cascade_destroy(ocean_cascade* cascade);

/* Advances every level to absolute time `time` (CascadeStack::update,
 * src/cascade.cpp:42-55). Asynchronous on `stream` (a cudaStream_t; NULL =
 * the cascade's own stream); later work on the cascade's stream waits for it. */
OCEAN_API ocean_status ocean_cascade_update(ocean_cascade* cascade, double time, void* stream);
OCEAN_API uint32_t ocean_cascade_level_count(const ocean_cascade* cascade);
OCEAN_API double ocean_cascade_get_time(const ocean_cascade* cascade);
OCEAN_API ocean_status ocean_cascade_level_device_buffers(const ocean_cascade* cascade,
                                                          uint32_t level,
                                                          ocean_device_buffers* out);
OCEAN_API ocean_status ocean_cascade_synchronize(ocean_cascade* cascade);

/* Summed surface of all levels at `count` world points (CascadeStack::sample_at,
 * src/cascade.cpp:82-153): per level `iterations` fixed-point steps (4 is the
 * reference's), stopping early once a step moves both parameter coordinates
 * by <= `tolerance` metres (0 = always run all of them). With
 * device_pointers == 0, xz/out are host arrays and the call waits; otherwise
 * they are device arrays and the work is queued on `stream` (a cudaStream_t,
 * NULL = the cascade's stream). With iterations = 4 and tolerance = 0 each
 * record is bit-identical to the reference's. */
OCEAN_API ocean_status ocean_cascade_sample_many(ocean_cascade* cascade, const float* xz,
                                                 uint64_t count, ocean_surface_ex* out,
                                                 int32_t iterations, float tolerance,
                                                 int32_t device_pointers, void* stream);

/* --- Interaction field extensions ---------------------------------------- */

/* Device pointer of the N*N float4 (eta, dEta/dx, dEta/dz, dEta/dt) output. */
OCEAN_API const float* ocean_interaction_device_field(const ocean_interaction* field);

/* Substeps the last update ran, and whether it hit max_substeps
 * (InteractionField::last_substeps / last_update_clamped). */
OCEAN_API uint32_t ocean_interaction_last_substeps(const ocean_interaction* field);
OCEAN_API int32_t ocean_interaction_last_clamped(const ocean_interaction* field);

/* The whole-cell shift the last ocean_interaction_recenter applied (both 0
 * when it did not move): InteractionField::last_shift_x / last_shift_z,
 * include/ocean/interaction.hpp:300-301. */
OCEAN_API void ocean_interaction_last_shift(const ocean_interaction* field, int32_t* dx, int32_t* dz);

/* The obstruction tables the last ocean_interaction_set_obstruction (or
 * recentre) built on the device: the solid cells in index order
 * (*solid_count of them; `solid` holds up to N*N entries) and, per cell, the
 * index of the fluid cell a solid cell copies under the Neumann condition
 * (itself for fluid cells, 0xFFFFFFFF where no fluid is reachable), as the
 * reference's multi-source BFS assigns them (src/interaction.cpp:255-292).
 * Either array may be NULL; *solid_count is 0 without an obstruction. */
OCEAN_API ocean_status ocean_interaction_obstruction_tables(const ocean_interaction* field, uint32_t* solid,
                                                            uint32_t* nearest, uint32_t* solid_count);

/* Discrete energy the undamped leapfrog conserves (InteractionField::energy,
 * src/interaction.cpp:803-846), evaluated on the device. */
OCEAN_API double ocean_interaction_energy(const ocean_interaction* field);

/* Snapshot / restore of the two time levels (host arrays of N*N floats each,
 * row-major): a session checkpoint, and a way to replay a known state. */
OCEAN_API ocean_status ocean_interaction_get_state(const ocean_interaction* field, float* cur,
                                                   float* old);
OCEAN_API ocean_status ocean_interaction_set_state(ocean_interaction* field, const float* cur,
                                                   const float* old);

/* The (2P+1)^2 stencil taps in use (host array, row-major over (j, i)). */
OCEAN_API ocean_status ocean_interaction_kernel_taps(const ocean_interaction* field, float* taps);

/* Batched queries of the interaction field alone (`out` = count records of
 * ocean_interaction_sample) and of the combined surface (FFT ocean plus
 * field, as ocean_sample_combined). Host arrays; the calls wait. */
OCEAN_API ocean_status ocean_interaction_sample_many(const ocean_interaction* field,
                                                     const float* xz, uint64_t count,
                                                     ocean_interaction_sample* out);
OCEAN_API ocean_status ocean_sample_combined_many(const ocean_sim* sim,
                                                  const ocean_interaction* field,
                                                  const float* xz, uint64_t count,
                                                  ocean_surface_ex* out);

/* --- Serving loop (no reference counterpart; the reference serves one
 *     caller per object, on the calling thread) -------------------------- */

typedef struct ocean_server ocean_server;

typedef struct ocean_server_desc {
    size_t   struct_size;        /* sizeof(ocean_server_desc) */
    uint64_t hbm_budget;         /* device bytes sessions may hold (default 120e9) */
    uint32_t max_inflight;       /* batches queued on the GPU at once (default 2) */
    uint32_t max_batch_requests; /* requests one batch takes at most (default 4096) */
    uint32_t max_batch_points;   /* query points one batch takes at most (default 1 << 20) */
    uint32_t max_query_points;   /* points one query request may carry (default 65536) */
    int32_t  fft_form;           /* ocean_fft_form of every session's ocean (default exact;
                                    the tensor form admits N = 64 to 512) */
    uint32_t reserved;
} ocean_server_desc;

typedef enum ocean_session_state {
    OCEAN_SESSION_WAITING = 0, /* queued for admission: the budget is full */
    OCEAN_SESSION_ACTIVE  = 1, /* admitted: its state lives on the device */
    OCEAN_SESSION_CLOSED  = 2  /* closed, or an unknown id */
} ocean_session_state;

typedef struct ocean_server_stats {
    uint64_t sessions_active;
    uint64_t sessions_waiting;
    uint64_t sessions_closed;
    uint64_t bytes_in_use;        /* admitted sessions plus shared tables and staging */
    uint64_t hbm_budget;
    uint64_t requests_submitted;
    uint64_t requests_completed;
    uint64_t requests_failed;
    uint64_t updates_completed;
    uint64_t queries_completed;
    uint64_t query_points_completed;
    uint64_t batches;             /* batches launched */
    uint64_t kernel_launches;     /* kernels those batches launched */
    uint64_t bytes_staging;       /* per-batch device staging (outside the budget) */
    double   mean_batch_requests;
    double   latency_p50_ms;      /* submit -> result ready (host clock), all requests */
    double   latency_p99_ms;
    double   latency_max_ms;
    double   update_p50_ms;
    double   update_p99_ms;
    double   query_p50_ms;
    double   query_p99_ms;
    double   gpu_busy_ms;         /* summed device time of the batches (CUDA events) */
    double   wall_ms;             /* since creation or the last reset */
    double   dispatch_max_ms;     /* longest single host step of the dispatcher */
    uint64_t staging_growths;     /* staging buffers grown past their reserve */
} ocean_server_stats;

OCEAN_API void ocean_server_desc_init(ocean_server_desc* desc);
/* Starts the server's dispatcher thread, stream and memory pool on the
 * current device. */
OCEAN_API ocean_server* ocean_server_create(const ocean_server_desc* desc, ocean_status* out_status);
/* Finishes every request of admitted sessions, fails those of sessions still
 * waiting for admission, then frees everything. */
OCEAN_API void ocean_server_destroy(ocean_server* server);

/* Device bytes one session with these descriptors holds (field may be NULL). */
OCEAN_API uint64_t ocean_server_session_bytes(const ocean_desc* ocean,
                                              const ocean_interaction_desc* field);

/* Opens a session: an ocean (ocean_create) and, when `field` is not NULL, an
 * interaction field over it (ocean_interaction_create; origin fixed at 0, no
 * obstruction). Ids start at 1. The session is admitted as soon as its
 * device state fits in the budget, in the order sessions were opened;
 * until then it waits, and requests submitted to it queue behind its
 * admission. A session larger than the whole budget is refused with
 * OCEAN_ERROR_OUT_OF_MEMORY. Invalid descriptors: OCEAN_ERROR_INVALID_ARG. */
OCEAN_API ocean_status ocean_server_open_session(ocean_server* server, const ocean_desc* ocean,
                                                 const ocean_interaction_desc* field,
                                                 uint64_t* out_session);
/* Closes a session after every request submitted to it before; its memory
 * returns to the budget and waiting sessions are admitted. */
OCEAN_API ocean_status ocean_server_close_session(ocean_server* server, uint64_t session);
OCEAN_API ocean_session_state ocean_server_session_state(ocean_server* server, uint64_t session);

/* Queues one frame of a session: the ocean to absolute `time` (ocean_update)
 * and, with a field, the `count` disturbances added in order
 * (ocean_interaction_add) and the field advanced by `dt`
 * (ocean_interaction_update). `sources` is copied before the call returns. */
OCEAN_API ocean_status ocean_server_submit_update(ocean_server* server, uint64_t session,
                                                  double time, float dt,
                                                  const ocean_disturbance* sources,
                                                  uint32_t count, uint64_t* out_ticket);
/* Queues `count` surface heights at world points xz[2*count] (copied before
 * the call returns): ocean_height_at plus, with a field,
 * ocean_interaction_height_at, as WaterSurface::height_at. A query sees every
 * update submitted to its session before it and none after. `heights` (count
 * floats of host memory) is written when the ticket completes and must stay
 * valid until then. */
OCEAN_API ocean_status ocean_server_submit_query(ocean_server* server, uint64_t session,
                                                 const float* xz, uint32_t count,
                                                 float* heights, uint64_t* out_ticket);

/* Waits up to timeout_ms for a ticket: OCEAN_OK once its result is written,
 * OCEAN_ERROR_TIMEOUT while it is still pending, OCEAN_ERROR_DEVICE if its
 * batch failed, OCEAN_ERROR_INVALID_ARG for a ticket never issued. */
OCEAN_API ocean_status ocean_server_wait(ocean_server* server, uint64_t ticket, uint32_t timeout_ms);
/* Waits up to timeout_ms for every request submitted so far. */
OCEAN_API ocean_status ocean_server_drain(ocean_server* server, uint32_t timeout_ms);

/* Copies a session's current state to host memory after waiting for every
 * request submitted to it: ocean displacement and normal (N*N*4 floats
 * each) and the field output (M*M*4 floats); any pointer may be NULL. */
OCEAN_API ocean_status ocean_server_read_session(ocean_server* server, uint64_t session,
                                                 float* displacement, float* normal,
                                                 float* field);

OCEAN_API ocean_status ocean_server_get_stats(ocean_server* server, ocean_server_stats* out);
/* Per-request samples since the last reset, in completion order: for each,
 * submit time (ms since the reset), latency (ms) and kind (0 update, 1
 * query). Writes at most `capacity` of each; returns how many exist. */
OCEAN_API uint64_t ocean_server_latency_samples(ocean_server* server, double* submit_ms,
                                                double* latency_ms, int32_t* kind,
                                                uint64_t capacity);
/* Clears latencies and counters (not the session counts or bytes). */
OCEAN_API ocean_status ocean_server_reset_stats(ocean_server* server);

/* Per-kernel device time of the frame passes, from CUDA events recorded on
 * the launching stream around every launch while profiling is on. */
typedef struct ocean_pass_profile {
    uint64_t row_launches;
    uint64_t col_launches;
    uint64_t foam_launches;
    double   row_ms;   /* summed launch durations */
    double   col_ms;
    double   foam_ms;
    uint64_t frame_launches; /* persistent frame kernel */
    double   frame_ms;
} ocean_pass_profile;

/* Turn per-launch event timing on or off (allocates its event pool when
 * turned on, so do it outside any timed region). */
OCEAN_API ocean_status ocean_batch_set_profiling(ocean_batch* batch, int32_t enable);

/* Waits for the batch's work, returns the accumulated profile and resets it. */
OCEAN_API ocean_status ocean_batch_read_profile(ocean_batch* batch, ocean_pass_profile* out);

/* Task plans of the batch's persistent kernel (no reference counterpart):
 * plan 0 is the default; N = 256 and 512 also have single-row tasks (plan
 * 1), N = 1024 sequences over 64 lanes with single-row tasks (plan 1). Every
 * plan gives the same bits. plan_count is 1 or 2; set_plan returns
 * OCEAN_ERROR_INVALID_ARG for a plan the batch does not have. The ring
 * slots are how many oceans' row-pass results may be in flight: 2 or 3 (1
 * for a batch of one ocean; at most the ocean count); fewer keep a large
 * size's ring in L2, more overlap an ocean's rows with the previous ones'
 * columns; same bits. Other values return OCEAN_ERROR_INVALID_ARG.
 * The deferred publish (1) lets a CTA of the persistent kernel announce a
 * finished row task only once its next task has staged its inputs, so the
 * release does not stall it; 0 announces it before the next task. Same
 * bits; the default is 1 with velocity, 0 without.
 * ocean_batch_autotune_plan times a few frames of every (plan, ring slots,
 * publish) combination on the batch's stream (advancing any persistent
 * foam), keeps the fastest and writes each plan's best milliseconds per frame
 * to `ms` (plan_count entries; may be NULL). */
OCEAN_API ocean_status ocean_batch_set_plan(ocean_batch* batch, int32_t plan);
OCEAN_API int32_t ocean_batch_plan(const ocean_batch* batch);
OCEAN_API int32_t ocean_batch_plan_count(const ocean_batch* batch);
OCEAN_API ocean_status ocean_batch_set_ring_slots(ocean_batch* batch, int32_t slots);
OCEAN_API int32_t ocean_batch_ring_slots(const ocean_batch* batch);
OCEAN_API ocean_status ocean_batch_set_deferred_publish(ocean_batch* batch, int32_t defer);
OCEAN_API int32_t ocean_batch_deferred_publish(const ocean_batch* batch);
OCEAN_API ocean_status ocean_batch_autotune_plan(ocean_batch* batch, double* ms);

/* Kernels this batch has launched (all kinds) since it was created. */
OCEAN_API uint64_t ocean_batch_launch_count(const ocean_batch* batch);

/* One frame of one ocean (exact form) that allocates no device memory. No
 * counterpart in the reference, which never touches a GPU: this is for
 * callers that are not allowed to call cudaMalloc - an engine or renderer
 * whose GPU memory is owned by its own allocator and budget, or a real-time
 * thread that cannot take cudaMalloc's implicit synchronisation. The caller
 * passes every input and output as its own device buffer (16-byte aligned):
 *   h0          N*N float2 (re, im)      \  as ocean_batch_read_spectrum
 *   omega_kinv  N*N float2 (omega, 1/|k|) /  returns them
 *   displacement, normal (and velocity, or NULL)  N*N float4 each.
 * The row-pass intermediate lives in a fixed device array inside this
 * library (about 12 MiB, held on every GPU that loads it until exit), so N
 * is limited to 16..512; larger N returns OCEAN_ERROR_INVALID_ARG. All calls
 * on a device share that array: calls whose GPU work overlaps (e.g. on two
 * streams) race and corrupt each other. The first call on a device looks up
 * the array's device address (a CUDA runtime query), so make that first call
 * before any stream capture begins. Work is queued on `stream` (a
 * cudaStream_t, NULL = legacy default stream). A buffer that is NULL (other
 * than velocity) or not 16-byte aligned returns OCEAN_ERROR_INVALID_ARG
 * before anything is queued. The call returns once the work is queued; a
 * bounded device wait that gave up during the frame is reported by
 * ocean_frame_static_scratch_status. */
OCEAN_API ocean_status ocean_frame_static_scratch(uint32_t size, float patch_length, double time,
                                                  float choppiness, float foam_threshold,
                                                  const float* h0, const float* omega_kinv,
                                                  float* displacement, float* normal,
                                                  float* velocity, void* stream);

/* Status of the last ocean_frame_static_scratch call on the current device:
 * waits for `stream` (the stream that call used), then returns OCEAN_OK, or
 * OCEAN_ERROR_TIMEOUT if a bounded wait of that frame gave up (its outputs
 * are then not valid). The word lives in the same static array and each
 * frame call clears it, so read it before the next call. Allocates nothing.
 * No counterpart in the reference. */
OCEAN_API ocean_status ocean_frame_static_scratch_status(void* stream);

/* Self-test of that status word: runs the frame's bounded mbarrier wait
 * (the h0 copy's wait) on a barrier nothing arrives at, with the static
 * array's status word as its error word, for `timeout_ms`, then returns what
 * ocean_frame_static_scratch_status reads: OCEAN_ERROR_TIMEOUT is the
 * expected outcome. Leaves the device usable; the next frame call clears
 * the word. */
OCEAN_API ocean_status ocean_check_static_scratch_status(uint32_t timeout_ms);

/* Runs the frame kernels' bounded waits with the given limit on things that
 * never complete - the work queue's wait on a counter nothing increments and
 * the h0 copy's wait on an mbarrier nothing arrives at - and reports
 * OCEAN_ERROR_TIMEOUT when both gave up and returned (the expected outcome):
 * a self-test of the timeout paths that leaves the device usable. */
OCEAN_API ocean_status ocean_check_bounded_wait(uint32_t timeout_ms);

/* Synchronous copy of `bytes` from a device pointer this library handed out
 * (e.g. an ocean_device_buffers member) into host memory, for callers that
 * have no CUDA binding of their own. */
OCEAN_API ocean_status ocean_copy_to_host(void* host_dst, const void* device_src, uint64_t bytes);

/* Name of the device the library was built for ("sm_100a"). */
OCEAN_API const char* ocean_device_arch(void);

#if defined(__cplusplus)
} /* extern "C" */
#endif

#endif /* OCEAN_B200_H */
