// oceanlib-b200: host-side interface of the device kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ocean_b200 {

// Inputs of the init-time spectrum build (the fields of ocean::OceanDesc the
// reference's build_spectrum reads, src/core/spectrum.cpp:264-339).
struct SpectrumParams {
    uint32_t n;
    float patch_length;
    float wind_speed, fetch, wind_direction, peak_enhancement, swell;
    float small_wave_cutoff, gravity, depth;
    uint64_t seed;
};

cudaError_t launch_h0(const SpectrumParams& p, float2* h0, cudaStream_t stream);
cudaError_t launch_geometry(const SpectrumParams& p, float2* omega_kinv, float* kvec,
                            cudaStream_t stream);

// Per-ocean constants of the finalize stage (src/core/evolve.cpp:238-327).
struct OceanConsts {
    float lambda;         // choppiness
    float foam_threshold;
    float inv_threshold;  // 1/threshold, or 0 for a degenerate threshold
    int32_t geom;         // index of the ocean's (omega, 1/|k|) table
};

// One ocean's own buffers, for frames over oceans that do not live in one
// batch array (the serving loop's sessions, each allocated on admission).
struct OceanSlot {
    const float2* h0;          // [N*N]
    const float2* omega_kinv;  // [N*N]
    const float* kvec;         // [N]
    float4* disp;              // [N*N]
    float4* normal;            // [N*N]
    float4* velocity;          // [N*N] or null
    OceanConsts cst;           // geom unused
};

// One frame's worth of device pointers for a batch of same-N oceans.
struct FrameArgs {
    const float2* h0;          // [count][N*N]
    const float2* omega_kinv;  // [geoms][N*N]
    const float* kvec;         // [geoms][N]
    const float2* twiddles;    // [N-1] per-stage inverse twiddles
    const OceanConsts* consts; // [count]
    const double* t_over_2pi;  // [count]
    float2* inter;             // [chunk][N][N][NF] row-pass output
    float4* disp;              // [count][N*N]
    float4* normal;            // [count][N*N]
    float4* velocity;          // [count][N*N] or null
    // persistent foam (only read when a foam substep is fused)
    const float* foam_cur;     // [count][N*N]
    float* foam_next;          // [count][N*N]
    float foam_dt, foam_decay, foam_gain, foam_scale, foam_drift_x, foam_drift_z;
    float foam_inv_cell;       // 1 / (patch_length / N); per batch (same L)
    int32_t ocean_base;        // first ocean of this chunk
    int32_t chunk;             // oceans in this chunk
    // When set, ocean i of the frame is table[i] (h0, geometry, outputs and
    // constants) and the batch arrays above are unused, except t_over_2pi
    // (indexed by i) and the intermediate. No persistent foam in this form.
    const OceanSlot* table;
    // Sticky error word of the row / column passes (a bounded wait that gave
    // up sets it); may be null. The persistent kernel uses QueueArgs::error.
    unsigned* error;
};

// Work queue of the persistent frame kernel. `ticket`, `rows_done[count]` and
// `cols_done[count]` must be zero at launch (one contiguous block).
struct QueueArgs {
    unsigned* ticket;
    unsigned* rows_done;
    unsigned* cols_done;
    unsigned* error;      // sticky: set to 1 when a bounded wait gives up
    int32_t count;        // oceans in the frame (inter holds `slots` of them)
    int32_t slots;        // intermediate ring slots
    unsigned long long wait_ns;
    // 1: a row task's counter add waits until the CTA's next task has staged
    // its inputs (when that task waits on nothing), so its release does not
    // stall the CTA; 0: the add comes before the next task. Either way a
    // column task adds its own counter once it has staged its slot.
    int32_t defer;
};

// The transforms' arithmetic of an ocean_fft_form, for the `ar` arguments
// below: 0 the reference's FP32 operations, 1 fused multiply-adds, 2 FP64
// within each register stage block (the precise form). The tensor-core form
// (2) has its own engine and passes through launch_frame's `form`.
inline int arith_of_form(int form) { return form == 1 ? 1 : (form == 3 ? 2 : 0); }

// One persistent launch for the whole frame of `q.count` oceans (foam fused
// when fuse_foam). `form` is an ocean_fft_form (the tensor form: N = 64 to 512).
// `grid` = CTAs to launch (0 = one wave of resident CTAs).
// `plan` picks the task plan (0: the default; 1: the alternative of N = 256,
// 512 and 1024, see frame_plan_count).
cudaError_t launch_frame(int log_n, int nf, int form, bool fuse_foam, const FrameArgs& args,
                         const QueueArgs& q, int grid, cudaStream_t stream, int plan = 0);
// Resident CTAs per SM of the persistent frame kernel (0: no such variant).
int frame_blocks_per_sm(int log_n, int nf, int form, bool fuse_foam, int plan = 0);
// Task plans the persistent kernel has for a size and form (1 or 2).
int frame_plan_count(int log_n, int form);
constexpr int kMaxFramePlans = 2;  // frame_plan_count never exceeds it
// Bounded waits that nothing completes (tests the timeout paths): on
// `counter`, which nothing increments, setting *error, and on an mbarrier
// nothing arrives at, setting *bar_error.
cudaError_t launch_wait_probe(const unsigned* counter, unsigned target, unsigned* error, unsigned* bar_error,
                              unsigned long long limit_ns, cudaStream_t stream);

// Mixed-size frames: the frames of several same-size groups of oceans (each
// a batch with its own arrays, counters and intermediate ring) as one
// persistent launch whose ticket queue holds group after group. Sizes N = 32
// .. 1024 (log_n 5..10), one field count for all groups, FP32 forms, no
// persistent foam. Group g's tickets are [first, first + tasks), tasks =
// mixed_tasks(log_n, count); its rows_done / cols_done (count each) and the
// ticket must be zero at launch.
constexpr int kMaxMixedGroups = 6;
struct MixedGroup {
    FrameArgs a;          // the group's arrays, or its pointer table (ocean_base 0)
    unsigned* rows_done;  // [count]
    unsigned* cols_done;  // [count]
    uint32_t first;       // first ticket of the group
    int32_t count;        // oceans
    int32_t slots;        // intermediate ring slots (a.inter holds them)
    int32_t log_n;
};
struct MixedArgs {
    MixedGroup g[kMaxMixedGroups];
    int32_t groups;
    uint32_t total;       // tickets of all groups
    unsigned* ticket;
    unsigned* error;      // sticky: set when a bounded wait gives up
    unsigned long long wait_ns;
    int32_t defer;        // as QueueArgs::defer, for every group
};
bool mixed_size_ok(int log_n);
uint32_t mixed_tasks(int log_n, int count);
int mixed_blocks_per_sm(int nf, int ar);
cudaError_t launch_mixed_frame(int nf, int ar, const MixedArgs& m, int grid, cudaStream_t stream);

// Row pass (evolve + row FFTs) and column pass (column FFTs + finalize, with
// an optional fused foam substep) for `args.chunk` oceans starting at
// args.ocean_base. log_n in [4, 10]; nf is 4 or 6 complex fields.
cudaError_t launch_row_pass(int log_n, int nf, int ar, const FrameArgs& args,
                            cudaStream_t stream);
cudaError_t launch_col_pass(int log_n, int nf, int ar, bool fuse_foam,
                            const FrameArgs& args, cudaStream_t stream);

// The frame at N = 2048 and 4096 (log_n 11, 12; frame_large.cu), for
// `args.chunk` oceans from args.ocean_base, in three launches: rows (evolve +
// row FFTs), column FFTs in place, finalize (+ the first foam substep when
// fuse_foam; nf = 6). The intermediate is field-major: field f of chunk ocean
// o at args.inter + (o * nf + f) * N * N. args.table must be null.
cudaError_t launch_large_rows(int log_n, int nf, int ar, const FrameArgs& args, cudaStream_t stream);
cudaError_t launch_large_cols(int log_n, int nf, int ar, const FrameArgs& args, cudaStream_t stream);
cudaError_t launch_large_finalize(int log_n, int nf, bool fuse_foam, const FrameArgs& args,
                                  cudaStream_t stream);

// Stand-alone foam substep for oceans [0, count) (used for substeps after the
// first in one update).
cudaError_t launch_foam_step(int n, int count, const float4* disp, const float4* velocity,
                             const float* cur, float* next, float dt, float decay, float gain,
                             float scale, float drift_x, float drift_z, float inv_cell,
                             cudaStream_t stream);

// FoamField::foam_at (src/foam.cpp:291-305) at `count` world points of one
// ocean: the displacement inversion, then the periodic bilinear foam fetch.
// inv_cell = N / patch_length (the inversion's), cell = patch_length / N.
cudaError_t launch_foam_at(int n, float inv_cell, float cell, const float4* disp, const float4* normal,
                           const float* foam, const float2* xz, uint64_t count, float* out,
                           cudaStream_t stream);
// FoamField::coverage (src/foam.cpp:307-313): mean of `cells` floats, in
// double, deterministic (fixed partial sums and tree).
cudaError_t launch_foam_coverage(const float* foam, uint64_t cells, double* out, cudaStream_t stream);

// Batched world queries (src/ocean.cpp:375-452), one thread per point.
struct SurfaceEx {
    float height, offset_x, offset_z, normal_x, normal_y, normal_z, foam;
    float velocity_x, velocity_y, velocity_z;
};
cudaError_t launch_sample(int n, float inv_cell, const float4* disp, const float4* normal,
                          const float4* velocity, const float2* xz, uint64_t count,
                          SurfaceEx* out, cudaStream_t stream);

// Cascade levels for the summed query (at most kMaxCascadeLevels).
constexpr int kMaxCascadeLevels = 8;
struct LevelView {
    const float4* disp;
    const float4* normal;
    const float4* velocity;  // may be null
    int32_t n;
    float inv_cell;          // N / patch_length
};
struct CascadeLevels {
    LevelView level[kMaxCascadeLevels];
    int32_t count;
};
cudaError_t launch_cascade_sample(const CascadeLevels& levels, const float2* xz, uint64_t count,
                                  SurfaceEx* out, int iters, float tol, cudaStream_t stream);

// RGBA32F -> RGBA16F, alpha optionally from a separate plane (pack.cu).
cudaError_t launch_pack_rgba16(const float4* src, const float* alpha, uint64_t cells, ushort4* dst,
                               cudaStream_t st);

// Shared-memory bytes each pass needs at a given size (for checks).
size_t row_pass_smem(int log_n, int nf);
size_t col_pass_smem(int log_n, int nf);

}  // namespace ocean_b200
