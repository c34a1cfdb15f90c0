// oceanlib-b200: iWave interaction field kernels.
//
// Per substep (reference: src/interaction.cpp:531-587):
//   sources  - Ricker stamps, 4-sigma clipped, mean-removed, added to both
//              time levels (src/interaction.cpp:322-391); one kernel computes
//              each source's stamp mean, a second adds every source to every
//              cell in submission order (so overlapping sources add in the
//              reference's order);
//   obstruction - Dirichlet zero or Neumann copy-from-nearest-fluid
//              (src/interaction.cpp:295-318);
//   step     - h_new = c1 * (2h - c2 h_old - g dt^2 (G * h)), the (2P+1)^2
//              convolution accumulated j-outer / i-inner in one float, no FMA,
//              flushed below 1e-30 (src/core/iwave_step.cpp:7-54). Shared-memory
//              tile with a P-cell halo; each thread keeps R vertically
//              adjacent outputs (R = 4 for batches of fields, 2 when one
//              launch has too few tiles to fill the SMs), so every loaded
//              value feeds up to R accumulators while each accumulator still
//              sees its taps in the reference order. The taps travel as
//              kernel parameters (constant bank), so each multiply takes its
//              tap as an operand, no load.
// After the substeps, finalize writes (eta, d/dx, d/dz, d/dt)
// (src/core/iwave_step.cpp:93-124). Compiled with -fmad=false.
#include "iwave.h"
#include "query_device.cuh"

namespace ocean_b200 {
namespace {

constexpr float kFlush = 1.0e-30f;
constexpr int kTileX = 32;
constexpr int kTileY = 32;

// kRowsPerThread outputs per thread down a column of the 32 x 32 tile.
template <int P, int kRowsPerThread>
__global__ void __launch_bounds__(kTileX * (kTileY / kRowsPerThread))
iwave_step_kernel(const IWaveField* __restrict__ fields, IWaveTaps taps)
{
    constexpr int W = 2 * P + 1;
    constexpr int SX = kTileX + 2 * P;
    constexpr int SY = kTileY + 2 * P;
    __shared__ float tile[SY][SX + 1];

    const IWaveField f = fields[blockIdx.z];
    const int x0 = blockIdx.x * kTileX;
    const int y0 = blockIdx.y * kTileY;
    if (x0 >= f.n || y0 >= f.n) return;  // fields of a smaller size in the batch
    const int tx = threadIdx.x;
    const int ty = threadIdx.y;
    const int tid = ty * kTileX + tx;
    constexpr int NT = kTileX * (kTileY / kRowsPerThread);

    // The halo reads land in the plane's P-cell zero border.
    for (int i = tid; i < SY * SX; i += NT) {
        const int r = i / SX, c = i % SX;
        tile[r][c] = f.cur[static_cast<ptrdiff_t>(y0 + r - P) * f.stride + (x0 + c - P)];
    }
    __syncthreads();

    float acc[kRowsPerThread];
#pragma unroll
    for (int q = 0; q < kRowsPerThread; ++q) acc[q] = 0.0f;
    const int ry = ty * kRowsPerThread;  // first output row of this thread in the tile
#pragma unroll
    for (int r = 0; r < kRowsPerThread + 2 * P; ++r) {
#pragma unroll
        for (int i = 0; i < W; ++i) {
            const float v = tile[ry + r][tx + i];
#pragma unroll
            for (int q = 0; q < kRowsPerThread; ++q) {
                const int j = r - q;  // tap row (0 .. 2P) for output q
                if (j >= 0 && j < W) acc[q] += taps.t[j * W + i] * v;
            }
        }
    }

#pragma unroll
    for (int q = 0; q < kRowsPerThread; ++q) {
        const int y = y0 + ry + q;
        const int x = x0 + tx;
        const ptrdiff_t pi = static_cast<ptrdiff_t>(y) * f.stride + x;
        const size_t ci = static_cast<size_t>(y) * f.n + x;
        const float hc = tile[ry + q + P][tx + P];
        const float hp = f.old[pi];
        const float v = f.c1[ci] * (2.0f * hc - f.c2[ci] * hp - f.gdt2 * acc[q]);
        f.old[pi] = (v > -kFlush && v < kFlush) ? 0.0f : v;
    }
}

__global__ void iwave_finalize_kernel(const IWaveField* __restrict__ fields)
{
    const IWaveField f = fields[blockIdx.z];
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= f.n || y >= f.n) return;
    const float* c = f.cur + static_cast<ptrdiff_t>(y) * f.stride + x;
    const float gx = (c[1] - c[-1]) * f.inv_two_cell;
    const float gz = (c[f.stride] - c[-static_cast<ptrdiff_t>(f.stride)]) * f.inv_two_cell;
    const float vy = (*c - f.old[static_cast<ptrdiff_t>(y) * f.stride + x]) * f.inv_dt;
    f.out[static_cast<size_t>(y) * f.n + x] = make_float4(*c, gx, gz, vy);
}

// The 2-D Ricker profile (1 - u) e^-u, u = r^2 / (2 sigma^2).
//
// The reference evaluates e^-u with the host's single-precision expf
// (glibc), which rounds to nearest except on a small fraction of arguments
// (about 0.07% of them by a uniform sample; none of the stamps of the
// scripted interaction test). e^-u is taken here in double precision and
// rounded once to float, which is the correctly rounded value wherever the
// double result is not within its own error of a float rounding boundary: so
// the stamps equal the reference's wherever glibc rounds to nearest, instead
// of wherever two different single-precision approximations happen to agree.
__device__ __forceinline__ float ricker(float r2, float inv_two_sigma2)
{
    const float u = r2 * inv_two_sigma2;
    return (1.0f - u) * static_cast<float>(exp(-static_cast<double>(u)));
}

__device__ __forceinline__ float stamp_r2(const IWaveSource& s, int x, int z)
{
    const float px = (static_cast<float>(x) + 0.5f) - s.gx;
    const float pz = (static_cast<float>(z) + 0.5f) - s.gz;
    return (px * px + pz * pz) * s.cell * s.cell;
}

// Mean of each source's clipped stamp, summed in double (deterministic tree
// order) and rounded to float. The reference sums the same float terms
// sequentially in double (src/interaction.cpp:357-366); the two orders' sums
// differ by roundings near 1e-16 relative, far below the float mean's
// 6e-8, so the float means agree (all 400 seeded random stamps of sizes up
// to 257 x 257 cells compared equal). One CTA per source.
__global__ void source_mean_kernel(IWaveSource* __restrict__ src, int count)
{
    const int k = blockIdx.x;
    if (k >= count) return;
    IWaveSource& s = src[k];
    const int wx = s.x1 - s.x0 + 1;
    const int wz = s.z1 - s.z0 + 1;
    const long long cells = static_cast<long long>(wx) * wz;
    double sum = 0.0;
    for (long long i = threadIdx.x; i < cells; i += blockDim.x) {
        const int x = s.x0 + static_cast<int>(i % wx);
        const int z = s.z0 + static_cast<int>(i / wx);
        sum += static_cast<double>(ricker(stamp_r2(s, x, z), s.inv_two_sigma2));
    }
    __shared__ double part[256];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        s.mean = static_cast<float>(part[0] / (static_cast<double>(wx) * static_cast<double>(wz)));
}

// Adds every source, in submission order, to cell (x, z) of one field.
// One source's contribution to both time levels of a cell it covers.
__device__ __forceinline__ void apply_source(const IWaveSource& s, int x, int z, float& cur, float& old,
                                             bool& touched)
{
    if (x < s.x0 || x > s.x1 || z < s.z0 || z > s.z1) return;
    const float sh = ricker(stamp_r2(s, x, z), s.inv_two_sigma2) - s.mean;
    const float dd = s.disp * sh;
    const float dv = s.vel * sh;
    cur += dd;
    old += dd - dv * s.dt;
    touched = true;
}

__device__ __forceinline__ void apply_sources_cell(const IWaveField& f, const IWaveSource* __restrict__ src,
                                                   int count, int x, int z)
{
    const ptrdiff_t ci = static_cast<ptrdiff_t>(z) * f.stride + x;
    float cur = f.cur[ci];
    float old = f.old[ci];
    bool touched = false;
    for (int k = 0; k < count; ++k) apply_source(src[k], x, z, cur, old, touched);
    if (touched) {
        f.cur[ci] = cur;
        f.old[ci] = old;
    }
}

__global__ void source_apply_kernel(IWaveField f, const IWaveSource* __restrict__ src, int count)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= f.n || z >= f.n) return;
    apply_sources_cell(f, src, count, x, z);
}

// Many fields at once (blockIdx.z = field; block 32 x 8 cells): field k
// takes sources [ranges[k].x, ranges[k].x + ranges[k].y). Warp 0 culls the
// sources against the block's tile 32 at a time, compacting the hits in
// submission order (ballot + prefix popcount), so each cell still adds its
// sources in the reference's order but visits only those near its tile.
__global__ void __launch_bounds__(256)
source_apply_batch_kernel(const IWaveField* __restrict__ fields, const int2* __restrict__ ranges,
                          const IWaveSource* __restrict__ src)
{
    const IWaveField f = fields[blockIdx.z];
    const int2 r = ranges[blockIdx.z];
    const int bx0 = blockIdx.x * 32, bz0 = blockIdx.y * 8;
    if (bx0 >= f.n || bz0 >= f.n || r.y == 0) return;  // uniform per block
    const int bx1 = min(bx0 + 32, f.n) - 1, bz1 = min(bz0 + 8, f.n) - 1;
    const IWaveSource* s0 = src + r.x;
    __shared__ int hit[32];
    __shared__ int nhit;
    const int x = bx0 + threadIdx.x, z = bz0 + threadIdx.y;
    const bool in = x < f.n && z < f.n;
    const ptrdiff_t ci = static_cast<ptrdiff_t>(z) * f.stride + x;
    float cur = 0.0f, old = 0.0f;
    if (in) {
        cur = f.cur[ci];
        old = f.old[ci];
    }
    bool touched = false;
    for (int c0 = 0; c0 < r.y; c0 += 32) {
        if (threadIdx.y == 0) {
            const int k = c0 + threadIdx.x;
            bool overlap = false;
            if (k < r.y) {
                const IWaveSource& s = s0[k];
                overlap = !(s.x1 < bx0 || s.x0 > bx1 || s.z1 < bz0 || s.z0 > bz1);
            }
            const unsigned m = __ballot_sync(0xffffffffu, overlap);
            if (overlap) hit[__popc(m & ((1u << threadIdx.x) - 1u))] = k;
            if (threadIdx.x == 0) nhit = __popc(m);
        }
        __syncthreads();
        const int nh = nhit;
        if (in)
            for (int j = 0; j < nh; ++j) apply_source(s0[hit[j]], x, z, cur, old, touched);
        __syncthreads();
    }
    if (touched) {
        f.cur[ci] = cur;
        f.old[ci] = old;
    }
}

// Boundary condition on h^n before the step (src/interaction.cpp:295-318).
__global__ void obstruction_kernel(IWaveField f, const uint32_t* __restrict__ solid,
                                   const uint32_t* __restrict__ nearest, uint32_t count,
                                   int dirichlet)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    const uint32_t i = solid[s];
    float* dst = f.cur + static_cast<ptrdiff_t>(i / f.n) * f.stride + (i % f.n);
    if (dirichlet) {
        *dst = 0.0f;
    } else {
        const uint32_t fl = nearest[i];
        if (fl == 0xFFFFFFFFu) return;
        *dst = f.cur[static_cast<ptrdiff_t>(fl / f.n) * f.stride + (fl % f.n)];
    }
}

// Integer recentre: dst(x, z) = src(x + dx, z + dz), zero where that falls
// outside the grid (src/interaction.cpp:601-705). Out of place.
__global__ void shift_kernel(const float* __restrict__ src, float* __restrict__ dst, int n,
                             int stride, int dx, int dz)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= n || z >= n) return;
    const int sx = x + dx, sz = z + dz;
    float v = 0.0f;
    if (sx >= 0 && sx < n && sz >= 0 && sz < n) v = src[static_cast<ptrdiff_t>(sz) * stride + sx];
    dst[static_cast<ptrdiff_t>(z) * stride + x] = v;
}

using qdev::interaction_tap;  // bilinear, zero outside the grid (query_device.cuh)

__global__ void interaction_sample_kernel(const float4* __restrict__ out, int n, float cell,
                                          float origin_x, float origin_z,
                                          const float2* __restrict__ xz, uint64_t count,
                                          float4* __restrict__ res)
{
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    bool inside;
    res[i] = interaction_tap(out, n, cell, origin_x, origin_z, xz[i].x, xz[i].y, inside);
}

// Energy terms (src/interaction.cpp:803-846) per row, in double; the host
// adds the rows in order.
__global__ void energy_rows_kernel(IWaveField f, const float* __restrict__ taps, int p,
                                   double* __restrict__ row_kin, double* __restrict__ row_pot)
{
    const int z = blockIdx.x;
    const int w = 2 * p + 1;
    double kin = 0.0, pot = 0.0;
    for (int x = threadIdx.x; x < f.n; x += blockDim.x) {
        const ptrdiff_t pi = static_cast<ptrdiff_t>(z) * f.stride + x;
        const double hc = f.cur[pi];
        const double hp = f.old[pi];
        const double v = (hc - hp) * f.inv_dt_d;
        kin += v * v;
        const float* centre = f.old + pi;
        double acc = 0.0;
        for (int j = -p; j <= p; ++j)
            for (int i = 0; i < w; ++i)
                acc += taps[(j + p) * w + i] * centre[static_cast<ptrdiff_t>(j) * f.stride - p + i];
        pot += hc * acc;
    }
    __shared__ double sk[256], sp[256];
    sk[threadIdx.x] = kin;
    sp[threadIdx.x] = pot;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            sk[threadIdx.x] += sk[threadIdx.x + s];
            sp[threadIdx.x] += sp[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        row_kin[z] = sk[0];
        row_pot[z] = sp[0];
    }
}

// FFT surface + interaction field (WaterSurface::sample_at,
// src/interaction.cpp:868-906): heights and vertical velocity add; normals
// compose through slopes when the FFT normal points up.
__global__ void combine_kernel(const SurfaceEx* __restrict__ ocean_s, const float4* __restrict__ e,
                               uint64_t count, SurfaceEx* __restrict__ out)
{
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    SurfaceEx s = ocean_s[i];
    const float4 f = e[i];
    s.height += f.x;
    s.velocity_y += f.w;
    if (s.normal_y > 1.0e-6f) {
        const float inv = 1.0f / s.normal_y;
        const float sx = -s.normal_x * inv + f.y;
        const float sz = -s.normal_z * inv + f.z;
        const float len = sqrtf(sx * sx + sz * sz + 1.0f);
        const float il = 1.0f / len;
        s.normal_x = -sx * il;
        s.normal_y = il;
        s.normal_z = -sz * il;
    }
    out[i] = s;
}

// Launches with fewer tiles than kFewTiles (a single field up to 512^2, or
// a few small ones) take two outputs per thread: 16 warps per tile instead
// of 8, so that the tile loads of twice as many warps are in flight on the
// SMs the launch reaches. Larger launches fill every SM several times over
// and keep four outputs per thread (fewer shared-memory loads per tap).
// Every cell sees the same taps in the same order either way.
constexpr long kFewTiles = 2 * 148;  // two tiles per SM on B200's 148 SMs

template <int P>
cudaError_t step_launch(const IWaveField* fields, int count, int max_n, const IWaveTaps& taps,
                        cudaStream_t st)
{
    dim3 grid((max_n + kTileX - 1) / kTileX, (max_n + kTileY - 1) / kTileY, count);
    const long tiles = static_cast<long>(grid.x) * grid.y * grid.z;
    if (tiles < kFewTiles) {
        iwave_step_kernel<P, 2><<<grid, dim3(kTileX, kTileY / 2), 0, st>>>(fields, taps);
    } else {
        iwave_step_kernel<P, 4><<<grid, dim3(kTileX, kTileY / 4), 0, st>>>(fields, taps);
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_iwave_step(int p, const IWaveField* fields, int count, int max_n,
                              const IWaveTaps& taps, cudaStream_t st)
{
    switch (p) {
        case 1: return step_launch<1>(fields, count, max_n, taps, st);
        case 2: return step_launch<2>(fields, count, max_n, taps, st);
        case 3: return step_launch<3>(fields, count, max_n, taps, st);
        case 4: return step_launch<4>(fields, count, max_n, taps, st);
        case 5: return step_launch<5>(fields, count, max_n, taps, st);
        case 6: return step_launch<6>(fields, count, max_n, taps, st);
        case 7: return step_launch<7>(fields, count, max_n, taps, st);
        case 8: return step_launch<8>(fields, count, max_n, taps, st);
        case 9: return step_launch<9>(fields, count, max_n, taps, st);
        case 10: return step_launch<10>(fields, count, max_n, taps, st);
        case 11: return step_launch<11>(fields, count, max_n, taps, st);
        case 12: return step_launch<12>(fields, count, max_n, taps, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_iwave_finalize(const IWaveField* fields, int count, int max_n, cudaStream_t st)
{
    dim3 block(32, 8);
    dim3 grid((max_n + 31) / 32, (max_n + 7) / 8, count);
    iwave_finalize_kernel<<<grid, block, 0, st>>>(fields);
    return cudaGetLastError();
}

cudaError_t launch_source_mean(IWaveSource* sources, int count, cudaStream_t st)
{
    if (count == 0) return cudaSuccess;
    source_mean_kernel<<<count, 256, 0, st>>>(sources, count);
    return cudaGetLastError();
}

cudaError_t launch_source_apply(const IWaveField& f, const IWaveSource* sources, int count,
                                cudaStream_t st)
{
    if (count == 0) return cudaSuccess;
    dim3 block(32, 8);
    dim3 grid((f.n + 31) / 32, (f.n + 7) / 8);
    source_apply_kernel<<<grid, block, 0, st>>>(f, sources, count);
    return cudaGetLastError();
}

cudaError_t launch_source_apply_batch(const IWaveField* fields, const int2* ranges,
                                      const IWaveSource* sources, int count, int max_n, cudaStream_t st)
{
    if (count == 0) return cudaSuccess;
    dim3 block(32, 8);
    dim3 grid((max_n + 31) / 32, (max_n + 7) / 8, count);
    source_apply_batch_kernel<<<grid, block, 0, st>>>(fields, ranges, sources);
    return cudaGetLastError();
}

cudaError_t launch_obstruction(const IWaveField& f, const uint32_t* solid, const uint32_t* nearest,
                               uint32_t count, bool dirichlet, cudaStream_t st)
{
    if (count == 0) return cudaSuccess;
    obstruction_kernel<<<(count + 255) / 256, 256, 0, st>>>(f, solid, nearest, count, dirichlet ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_shift(const float* src, float* dst, int n, int stride, int dx, int dz,
                         cudaStream_t st)
{
    dim3 block(32, 8);
    dim3 grid((n + 31) / 32, (n + 7) / 8);
    shift_kernel<<<grid, block, 0, st>>>(src, dst, n, stride, dx, dz);
    return cudaGetLastError();
}

cudaError_t launch_interaction_sample(const float4* out, int n, float cell, float origin_x,
                                      float origin_z, const float2* xz, uint64_t count,
                                      float4* res, cudaStream_t st)
{
    if (count == 0) return cudaSuccess;
    interaction_sample_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, st>>>(
        out, n, cell, origin_x, origin_z, xz, count, res);
    return cudaGetLastError();
}

cudaError_t launch_combine(const SurfaceEx* ocean_s, const float4* e, uint64_t count, SurfaceEx* out,
                           cudaStream_t st)
{
    if (count == 0) return cudaSuccess;
    combine_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, st>>>(ocean_s, e, count, out);
    return cudaGetLastError();
}

cudaError_t launch_energy_rows(const IWaveField& f, const float* taps, int p, double* row_kin,
                               double* row_pot, cudaStream_t st)
{
    energy_rows_kernel<<<f.n, 256, 0, st>>>(f, taps, p, row_kin, row_pot);
    return cudaGetLastError();
}

}  // namespace ocean_b200
