/* Test infrastructure: a plain-C restatement of oceanlib's per-frame path.
 *
 * This is the CHECKER for the CUDA library, never part of it. Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it. Each
 * function names the reference file:line whose arithmetic it restates; every
 * float operation is written in the same order as the reference and the file
 * is compiled with -ffp-contract=off, so results are bit-identical to the
 * reference's scalar kernels (pinned by tests/test_oracle_pins.py against the
 * reference compiled from its own sources, and against its known answers).
 */
#ifndef OCEAN_ORACLE_H
#define OCEAN_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Flat descriptor (the fields of ocean::OceanDesc that the path reads). */
typedef struct or_desc {
    uint32_t n;
    float patch_length;
    float wind_speed, fetch, wind_direction, peak_enhancement, swell;
    float small_wave_cutoff, gravity, depth;
    float choppiness, foam_threshold;
    uint64_t seed;
    int32_t velocity;
} or_desc;

typedef struct or_pcg32 {
    uint64_t state, inc;
} or_pcg32;

or_pcg32 or_pcg32_seed(uint64_t seed, uint64_t stream);
uint32_t or_pcg32_next(or_pcg32* r);
void or_pcg32_fill(uint64_t seed, uint64_t stream, uint32_t count, uint32_t* out);
uint64_t or_mix64(uint64_t x);
void or_row_gaussians(uint64_t seed, uint32_t row, uint32_t pairs, float* out);

/* Spectrum tables: 8 planes of n*n floats, in the order
 * h0_re, h0_im, h0c_re, h0c_im, omega, kx, kz, k_inv. */
void or_build_spectrum(const or_desc* d, float* tables);

/* Per-frame evolve into 8 (or 12 with velocity) planes re0, im0, re1, im1, ... */
void or_evolve(const or_desc* d, const float* tables, double t, float* fields);

/* Unnormalised radix-2 Stockham FFT; sign +1 = inverse, -1 = forward. */
void or_fft_1d(uint32_t n, float* re, float* im, int sign);
void or_fft_2d(uint32_t n, float* re, float* im, int sign);

/* Finalize: displacement and normal RGBA32F (n*n*4 each), velocity if non-NULL. */
void or_finalize(const or_desc* d, const float* fields, float* disp, float* normal,
                 float* velocity);

/* Whole update: evolve -> 2-D inverse FFTs -> finalize. `fields` is scratch of
 * 8 (12) * n*n floats. */
void or_update(const or_desc* d, const float* tables, double t, float* fields,
               float* disp, float* normal, float* velocity);

/* World query (Ocean::sample_at). out[10] = height, offset_x, offset_z,
 * normal xyz, foam, velocity xyz. velocity may be NULL. */
void or_sample_at(uint32_t n, float patch_length, const float* disp, const float* normal,
                  const float* velocity, float x, float z, float* out);
void or_sample_many(uint32_t n, float patch_length, const float* disp, const float* normal,
                    const float* velocity, const float* xz, uint64_t count, float* out);

/* Ocean::sample_at with `iters` fixed-point steps (4 = the reference) that
 * stop early once both parameter coordinates move by <= tol (0 = never). */
void or_sample_at_iter(uint32_t n, float patch_length, const float* disp, const float* normal,
                       const float* velocity, float x, float z, int iters, float tol, float* out);

/* CascadeStack::sample_at over `levels` oceans at `count` points, each level
 * inverted with (iters, tol); out is count x 10 as or_sample_at. */
void or_cascade_sample_many(uint32_t levels, const uint32_t* n, const float* patch_length,
                            const float* const* disp, const float* const* normal,
                            const float* const* velocity, const float* xz, uint64_t count, int iters,
                            float tol, float* out);

/* FoamField::foam_at at `count` world points: out[i] for (xz[2i], xz[2i+1]). */
void or_foam_at_many(uint32_t n, float patch_length, const float* disp, const float* normal,
                     const float* foam, const float* xz, uint64_t count, float* out);

/* One persistent-foam substep (FoamField step_rows). `decay` is the already
 * evaluated expf(-decay_rate * dt), as the reference computes it on the host. */
void or_foam_step(uint32_t n, float cell, float dt, float decay, float gain, float scale,
                  float drift_x, float drift_z, const float* disp, const float* velocity,
                  const float* cur, float* next);

/* FP64 oracle: the direct 2-D inverse DFT of a complex n*n field evaluated in
 * double at `count` output points (x[i], y[i]); O(n^2) per point, sharing no
 * structure with the FFT. */
void or_dft2d_points(uint32_t n, const float* re, const float* im, uint32_t count,
                     const uint32_t* xs, const uint32_t* ys, double* out_re, double* out_im);
/* Full O(n^4) direct 2-D inverse DFT (small n only). */
void or_dft2d_full(uint32_t n, const float* re, const float* im, double* out_re,
                   double* out_im);

/* iWave interaction field (src/core/iwave_step.cpp, src/interaction.cpp).
 * Planes are interior pointers into arrays with a p-cell halo and row stride
 * `stride`; `d` is (world_x, world_z, radius, strength, velocity_y,
 * velocity_x, velocity_z). */
void or_iwave_damping(uint32_t n, float damping, uint32_t absorb, float dt, float* c1, float* c2);
void or_iwave_step(uint32_t n, uint32_t p, size_t stride, const float* taps, const float* c1,
                   const float* c2, float gdt2, const float* cur, float* old);
void or_iwave_finalize(uint32_t n, size_t stride, const float* cur, const float* old,
                       float inv_two_cell, float inv_dt, float* out);
void or_iwave_inject(uint32_t n, size_t stride, float cell, int32_t origin_x, int32_t origin_z,
                     float dt, const float* d, float sub_time, float scale, float* cur, float* old);
uint32_t or_iwave_nearest(uint32_t n, const uint8_t* mask, uint32_t* nearest, uint32_t* solid);
void or_iwave_obstruction(uint32_t n, size_t stride, const uint32_t* solid, uint32_t count,
                          const uint32_t* nearest, int dirichlet, float* cur);

#ifdef __cplusplus
}
#endif

#endif
