// oceanlib-b200: the obstruction tables of an interaction field, built on the
// device (InteractionField::rebuild_mask_tables, src/interaction.cpp:255-292).
//
// The reference runs a multi-source breadth-first search: every fluid cell,
// in index order, seeds a FIFO queue; a popped cell visits its neighbours in
// the order +x, -x, +z, -z and hands its nearest-fluid index to each solid
// neighbour not yet reached. Which fluid cell a solid cell inherits depends
// on that queue order, so the device reproduces it exactly, one BFS level per
// launch:
//
//   * a cell at level d (distance d from fluid) is reached by the level d-1
//     neighbour that comes first in the queue, through the direction e that
//     neighbour tries for it (0..3 in the order above);
//   * the queue order of level d is therefore the lexicographic order of
//     (queue order of that neighbour, e). Each cell carries an order key
//     with exactly that property: level 0 (fluid) cells their index; a level
//     d cell 4 * key(discoverer) + e. Keys grow by two bits per level; when a
//     level's largest key nears 2^62 the level's keys are replaced by their
//     ranks (a radix sort of that level), which keeps the order.
//
// A level touches every cell once and reads only level d-1 cells, whose
// state no thread of the launch writes, so the result does not depend on
// thread order. The solid list is the solid cells in index order (an ordered
// selection). The host reads back one count per level (and the last level's
// largest key) to know when the frontier is empty.
#include "iwave.h"

#include <cub/cub.cuh>

#include <cstdint>
#include <vector>

namespace ocean_b200 {
namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr int32_t kUnreached = -1;

struct LevelStats {
    unsigned long long count;
    unsigned long long max_key;
};

__global__ void bfs_seed_kernel(const uint8_t* __restrict__ mask, uint32_t cells, uint32_t* __restrict__ nearest,
                                int32_t* __restrict__ level, unsigned long long* __restrict__ key,
                                uint8_t* __restrict__ solid_flag)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cells) return;
    const bool solid = mask[i] != 0;
    nearest[i] = solid ? kNone : i;
    level[i] = solid ? kUnreached : 0;
    key[i] = solid ? 0ull : static_cast<unsigned long long>(i);
    solid_flag[i] = solid ? 1 : 0;
}

// Level d: every unreached cell with a level d-1 neighbour takes the first
// of them in queue order.
__global__ void bfs_level_kernel(int n, int d, uint32_t* __restrict__ nearest, int32_t* __restrict__ level,
                                 unsigned long long* __restrict__ key, LevelStats* __restrict__ stats)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t cells = static_cast<uint32_t>(n) * static_cast<uint32_t>(n);
    if (j >= cells || level[j] != kUnreached) return;
    const int x = static_cast<int>(j % static_cast<uint32_t>(n));
    const int z = static_cast<int>(j / static_cast<uint32_t>(n));
    // Direction e is the step from the discoverer to j: +x, -x, +z, -z, so
    // the discoverer sits at j - step.
    const int sx[4] = {-1, 1, 0, 0};
    const int sz[4] = {0, 0, -1, 1};
    unsigned long long best = ~0ull;
    uint32_t from = kNone;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int ix = x + sx[e], iz = z + sz[e];
        if (ix < 0 || iz < 0 || ix >= n || iz >= n) continue;
        const uint32_t i = static_cast<uint32_t>(iz) * static_cast<uint32_t>(n) + static_cast<uint32_t>(ix);
        if (level[i] != d - 1) continue;
        const unsigned long long c = key[i] * 4ull + static_cast<unsigned long long>(e);
        if (c < best) {
            best = c;
            from = i;
        }
    }
    if (from == kNone) return;
    nearest[j] = nearest[from];
    level[j] = d;
    key[j] = best;
    atomicAdd(&stats->count, 1ull);
    atomicMax(&stats->max_key, best);
}

__global__ void level_flags_kernel(const int32_t* __restrict__ level, uint32_t cells, int d,
                                   uint8_t* __restrict__ flag)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < cells) flag[i] = level[i] == d ? 1 : 0;
}

__global__ void gather_keys_kernel(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ count,
                                   const unsigned long long* __restrict__ key, unsigned long long* __restrict__ out)
{
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < *count) out[r] = key[idx[r]];
}

__global__ void scatter_ranks_kernel(const uint32_t* __restrict__ sorted_idx, const uint32_t* __restrict__ count,
                                     unsigned long long* __restrict__ key)
{
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < *count) key[sorted_idx[r]] = r;
}

inline cudaError_t ok_or(cudaError_t e) { return e != cudaSuccess ? e : cudaGetLastError(); }

}  // namespace

// Builds `solid` (solid cells in index order, *solid_count of them) and
// `nearest` (per cell: itself for fluid, the inherited fluid index for a
// reachable solid cell, 0xFFFFFFFF otherwise) from the device mask. Scratch
// is allocated here (once per set_obstruction, as the reference's tables
// are rebuilt) and released before returning. Waits for the stream.
cudaError_t build_obstruction_tables(const uint8_t* mask, int n, uint32_t* solid, uint32_t* nearest,
                                     uint32_t* solid_count, cudaStream_t st)
{
    const uint32_t cells = static_cast<uint32_t>(n) * static_cast<uint32_t>(n);
    const unsigned blocks = (cells + 255) / 256;
    int32_t* level = nullptr;
    unsigned long long* key = nullptr;
    unsigned long long* keys_in = nullptr;
    unsigned long long* keys_out = nullptr;
    uint32_t* idx_in = nullptr;
    uint32_t* idx_out = nullptr;
    uint8_t* flag = nullptr;
    uint32_t* dcount = nullptr;
    LevelStats* stats = nullptr;
    void* temp = nullptr;
    size_t temp_bytes = 0;
    cudaError_t e = cudaSuccess;
    auto run = [&]() -> cudaError_t {
        cudaError_t r;
        if ((r = cudaMallocAsync(&level, cells * sizeof(int32_t), st)) != cudaSuccess) return r;
        if ((r = cudaMallocAsync(&key, cells * sizeof(unsigned long long), st)) != cudaSuccess) return r;
        if ((r = cudaMallocAsync(&flag, cells, st)) != cudaSuccess) return r;
        if ((r = cudaMallocAsync(&dcount, sizeof(uint32_t), st)) != cudaSuccess) return r;
        if ((r = cudaMallocAsync(&stats, sizeof(LevelStats), st)) != cudaSuccess) return r;
        if ((r = cudaMallocAsync(&idx_in, cells * sizeof(uint32_t), st)) != cudaSuccess) return r;
        if ((r = cudaMallocAsync(&idx_out, cells * sizeof(uint32_t), st)) != cudaSuccess) return r;
        if ((r = cudaMallocAsync(&keys_in, cells * sizeof(unsigned long long), st)) != cudaSuccess) return r;
        if ((r = cudaMallocAsync(&keys_out, cells * sizeof(unsigned long long), st)) != cudaSuccess) return r;
        // One temporary block large enough for the selection and the sort.
        size_t sel_bytes = 0, sort_bytes = 0;
        cub::CountingInputIterator<uint32_t> iota(0);
        if ((r = cub::DeviceSelect::Flagged(nullptr, sel_bytes, iota, flag, solid, dcount, cells, st)) != cudaSuccess)
            return r;
        if ((r = cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, keys_in, keys_out, idx_in, idx_out,
                                                 static_cast<int>(cells), 0, 64, st)) != cudaSuccess)
            return r;
        temp_bytes = sel_bytes > sort_bytes ? sel_bytes : sort_bytes;
        if ((r = cudaMallocAsync(&temp, temp_bytes, st)) != cudaSuccess) return r;

        bfs_seed_kernel<<<blocks, 256, 0, st>>>(mask, cells, nearest, level, key, flag);
        if ((r = cudaGetLastError()) != cudaSuccess) return r;
        size_t tb = temp_bytes;
        if ((r = cub::DeviceSelect::Flagged(temp, tb, iota, flag, solid, dcount, cells, st)) != cudaSuccess) return r;
        if ((r = cudaMemcpyAsync(solid_count, dcount, sizeof(uint32_t), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return r;
        if ((r = cudaStreamSynchronize(st)) != cudaSuccess) return r;
        // Every level reaches at least one new cell until the frontier is
        // empty, so at most (solid count) levels run.
        for (int d = 1; d <= static_cast<int>(*solid_count); ++d) {
            if ((r = cudaMemsetAsync(stats, 0, sizeof(LevelStats), st)) != cudaSuccess) return r;
            bfs_level_kernel<<<blocks, 256, 0, st>>>(n, d, nearest, level, key, stats);
            if ((r = cudaGetLastError()) != cudaSuccess) return r;
            LevelStats h{};
            if ((r = cudaMemcpyAsync(&h, stats, sizeof(h), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return r;
            if ((r = cudaStreamSynchronize(st)) != cudaSuccess) return r;
            if (h.count == 0) break;
            if (h.max_key >= (1ull << 61)) {
                // Re-rank level d: its cells in index order, sorted by key,
                // then each cell's key becomes its rank.
                level_flags_kernel<<<blocks, 256, 0, st>>>(level, cells, d, flag);
                tb = temp_bytes;
                if ((r = ok_or(cub::DeviceSelect::Flagged(temp, tb, iota, flag, idx_in, dcount, cells, st))) !=
                    cudaSuccess)
                    return r;
                const uint32_t m = static_cast<uint32_t>(h.count);
                const unsigned mb = (m + 255) / 256;
                gather_keys_kernel<<<mb, 256, 0, st>>>(idx_in, dcount, key, keys_in);
                tb = temp_bytes;
                if ((r = ok_or(cub::DeviceRadixSort::SortPairs(temp, tb, keys_in, keys_out, idx_in, idx_out,
                                                               static_cast<int>(m), 0, 64, st))) != cudaSuccess)
                    return r;
                scatter_ranks_kernel<<<mb, 256, 0, st>>>(idx_out, dcount, key);
                if ((r = cudaGetLastError()) != cudaSuccess) return r;
            }
        }
        return cudaSuccess;
    };
    e = run();
    for (void* p : {static_cast<void*>(level), static_cast<void*>(key), static_cast<void*>(flag),
                    static_cast<void*>(dcount), static_cast<void*>(stats), static_cast<void*>(idx_in),
                    static_cast<void*>(idx_out), static_cast<void*>(keys_in), static_cast<void*>(keys_out), temp})
        if (p != nullptr) cudaFreeAsync(p, st);
    const cudaError_t s = cudaStreamSynchronize(st);
    return e != cudaSuccess ? e : s;
}

}  // namespace ocean_b200
