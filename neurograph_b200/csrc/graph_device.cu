// Device build of a single graph: the caller's CSR is uploaded once, and the GPU checks the arcs, drops zero weights,
// writes both arc-length arrays and builds the reverse CSR by a stable sort of the stored arcs by target. The arrays
// are bit-identical to the host build of graph.cu (same stored order, same lengths, within a target the in-arcs in
// ascending stored order), which replaces DistributedGraph's window construction (source/graph/DistributedGraph.cpp:
// 154-250: arcs uploaded per rank, zero weights skipped at :174-176 and :223-225).
//
// The host keeps two sequential pieces: the row checks (O(n)) and the mean arc lengths, summed in stored order as the
// host build does (so the default bucket widths have the same bits), on a thread of their own while the GPU works.
// The graph's locality order of sources is computed when a run first needs it (graph.cu, ensure_source_order).

#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cmath>
#include <cstring>
#include <string>
#include <thread>

#include "ngx_common.cuh"
#include "ngx_graph.h"

namespace ngx {
namespace {

constexpr int kBuildBlock = 256;

__device__ __forceinline__ unsigned lane_mask_below() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// One warp per caller row: checks every arc (target in range, finite weight; the smallest bad arc index wins) and
// counts the stored (non-zero) ones; the row's count goes to kept[u], the largest count and the extreme lengths to the
// reductions (non-negative doubles order like their bit patterns).
__global__ void count_rows_kernel(const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col, const double* __restrict__ w, int64_t n,
                                  int64_t* __restrict__ kept, unsigned long long* bad_arc, unsigned long long* max_degree,
                                  unsigned long long* min_len_bits, unsigned long long* max_len_bits) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    unsigned long long lo = ~0ull, hi = 0ull;
    for (int64_t u = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; u < n; u += warps) {
        const int64_t beg = row_ptr[u];
        const int64_t end = row_ptr[u + 1];
        int64_t count = 0;
        for (int64_t e = beg + lane; e < end; e += 32) {
            const int32_t v = col[e];
            const double x = w[e];
            if (v < 0 || v >= n || !isfinite(x)) {
                atomicMin(bad_arc, static_cast<unsigned long long>(e));
            }
            const double a = fabs(x);
            if (a != 0.0 && isfinite(a)) {
                ++count;
                const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(a));
                lo = bits < lo ? bits : lo;
                hi = bits > hi ? bits : hi;
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            count += __shfl_xor_sync(0xFFFFFFFFu, count, off);
        }
        if (lane == 0) {
            kept[u] = count;
            atomicMax(max_degree, static_cast<unsigned long long>(count));
        }
    }
    if (lo != ~0ull) {
        atomicMin(min_len_bits, lo);
    }
    if (hi != 0ull) {
        atomicMax(max_len_bits, hi);
    }
}

// One warp per caller row: the stored arcs in caller order (zero weights dropped), both lengths, the source of each
// stored arc, the stored index of each caller arc (-1 for zero weights), and the (target, stored index) pairs that the
// reverse CSR is sorted from.
__global__ void fill_rows_kernel(const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col, const double* __restrict__ w, int64_t n,
                                 const int64_t* __restrict__ stored_row, Arc* __restrict__ regular, Arc* __restrict__ inverse,
                                 int32_t* __restrict__ arc_src, int32_t* __restrict__ stored_of_user, uint32_t* __restrict__ target,
                                 int32_t* __restrict__ index) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    for (int64_t u = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; u < n; u += warps) {
        const int64_t end = row_ptr[u + 1];
        int64_t pos = stored_row[u];
        for (int64_t e0 = row_ptr[u]; e0 < end; e0 += 32) {
            const int64_t e = e0 + lane;
            const bool valid = e < end;
            const double a = valid ? fabs(w[e]) : 0.0;
            const bool keep = valid && a != 0.0;
            const unsigned mask = __ballot_sync(0xFFFFFFFFu, keep);
            if (keep) {
                const int64_t at = pos + __popc(mask & lane_mask_below());
                const int32_t v = col[e];
                regular[at] = Arc{ v, static_cast<int32_t>(e), a };
                inverse[at] = Arc{ v, static_cast<int32_t>(e), 1.0 / a };
                arc_src[at] = static_cast<int32_t>(u);
                stored_of_user[e] = static_cast<int32_t>(at);
                target[at] = static_cast<uint32_t>(v);
                index[at] = static_cast<int32_t>(at);
            } else if (valid) {
                stored_of_user[e] = -1;
            }
            pos += __popc(mask);
        }
    }
}

__global__ void in_degree_kernel(const uint32_t* __restrict__ target, int64_t m, int64_t* __restrict__ degree) {
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < m; e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        atomicAdd(reinterpret_cast<unsigned long long*>(&degree[target[e]]), 1ull);
    }
}

// The reverse records in sorted order: record i is stored arc sorted_index[i] seen from its target.
__global__ void reverse_records_kernel(const int32_t* __restrict__ sorted_index, int64_t m, const Arc* __restrict__ regular,
                                       const int32_t* __restrict__ arc_src, Arc* __restrict__ rarcs) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t e = sorted_index[i];
        rarcs[i] = Arc{ arc_src[e], e, regular[e].len };
    }
}

int grid_for(int64_t items, int per_block, int sm_count) {
    const int64_t want = (items + per_block - 1) / per_block;
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(want, static_cast<int64_t>(sm_count) * 16)));
}

int bits_for(int64_t n) {
    int b = 1;
    while (b < 31 && (int64_t(1) << b) <= n) {
        ++b;
    }
    return b;
}

// Temporary device buffers of the build, freed on every exit.
struct Scratch {
    void* p[12] = {};
    int used = 0;
    ~Scratch() {
        for (int i = 0; i < used; ++i) {
            cudaFree(p[i]);
        }
    }
    template <typename T>
    int take(T** out, size_t count) {
        void* ptr = nullptr;
        NGX_CUDA_TRY(cudaMalloc(&ptr, std::max<size_t>(1, count) * sizeof(T)));
        p[used++] = ptr;
        *out = static_cast<T*>(ptr);
        return NGX_OK;
    }
};

}  // namespace

int build_graph_on_device(const ngx_csr* csr, ngx_graph* g) {
    const int64_t n = csr->n;
    const int64_t m_user = csr->m;
    cudaStream_t s = g->stream;

    // the mean lengths in stored order, on the host beside the device work (the host build's sums, bit for bit)
    double sum_regular = 0.0, sum_inverse = 0.0;
    int64_t stored_count = 0;
    const auto mean_sums = [&] {
        for (int64_t e = 0; e < m_user; ++e) {
            const double a = std::fabs(csr->w[e]);
            if (a != 0.0 && std::isfinite(a)) {
                sum_regular += a;
                sum_inverse += 1.0 / a;
                ++stored_count;
            }
        }
    };
    std::thread sums_thread;
    try {
        sums_thread = std::thread(mean_sums);
    } catch (const std::system_error&) {
        mean_sums();  // no thread: summed here before the device work
    }
    struct Joiner {
        std::thread& t;
        ~Joiner() {
            if (t.joinable()) {
                t.join();
            }
        }
    } joiner{ sums_thread };

    Scratch tmp;
    int64_t* d_user_rows = nullptr;
    int32_t* d_col = nullptr;
    double* d_w = nullptr;
    int64_t* d_kept = nullptr;
    unsigned long long* d_red = nullptr;  // bad arc, max degree, min length bits, max length bits
    int rc = NGX_OK;
    if ((rc = tmp.take(&d_user_rows, static_cast<size_t>(n) + 1)) != NGX_OK) return rc;
    if ((rc = tmp.take(&d_col, static_cast<size_t>(m_user))) != NGX_OK) return rc;
    if ((rc = tmp.take(&d_w, static_cast<size_t>(m_user))) != NGX_OK) return rc;
    if ((rc = tmp.take(&d_kept, static_cast<size_t>(n) + 1)) != NGX_OK) return rc;
    if ((rc = tmp.take(&d_red, 4)) != NGX_OK) return rc;
    NGX_CUDA_TRY(cudaMemcpyAsync(d_user_rows, csr->row_ptr, (static_cast<size_t>(n) + 1) * 8, cudaMemcpyHostToDevice, s));
    if (m_user > 0) {
        NGX_CUDA_TRY(cudaMemcpyAsync(d_col, csr->col, static_cast<size_t>(m_user) * 4, cudaMemcpyHostToDevice, s));
        NGX_CUDA_TRY(cudaMemcpyAsync(d_w, csr->w, static_cast<size_t>(m_user) * 8, cudaMemcpyHostToDevice, s));
    }
    const unsigned long long red_init[4] = { ~0ull, 0ull, ~0ull, 0ull };
    NGX_CUDA_TRY(cudaMemcpyAsync(d_red, red_init, sizeof(red_init), cudaMemcpyHostToDevice, s));
    NGX_CUDA_TRY(cudaMemsetAsync(d_kept + n, 0, 8, s));
    const int row_grid = grid_for(n * 32, kBuildBlock, g->sm_count);
    count_rows_kernel<<<row_grid, kBuildBlock, 0, s>>>(d_user_rows, d_col, d_w, n, d_kept, d_red, d_red + 1, d_red + 2, d_red + 3);
    NGX_CUDA_TRY(cudaGetLastError());
    unsigned long long red[4];
    NGX_CUDA_TRY(cudaMemcpyAsync(red, d_red, sizeof(red), cudaMemcpyDeviceToHost, s));
    NGX_CUDA_TRY(cudaStreamSynchronize(s));
    if (red[0] != ~0ull) {
        const int64_t e = static_cast<int64_t>(red[0]);
        const bool bad_target = csr->col[e] < 0 || csr->col[e] >= n;
        return fail(NGX_INVALID_ARGUMENT, "ngx_graph_create: arc " + std::to_string(e) +
                                              (bad_target ? " has an out-of-range target" : " has a non-finite weight"));
    }

    // stored row offsets: exclusive sum of the kept counts (n + 1 entries, the last one m)
    NGX_CUDA_TRY(cudaMalloc(&g->d_row_ptr, (static_cast<size_t>(n) + 1) * 8));
    size_t scan_bytes = 0;
    NGX_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, d_kept, g->d_row_ptr, n + 1, s));
    char* d_scan = nullptr;
    if ((rc = tmp.take(&d_scan, scan_bytes)) != NGX_OK) return rc;
    NGX_CUDA_TRY(cub::DeviceScan::ExclusiveSum(d_scan, scan_bytes, d_kept, g->d_row_ptr, n + 1, s));
    int64_t m = 0;
    NGX_CUDA_TRY(cudaMemcpyAsync(&m, g->d_row_ptr + n, 8, cudaMemcpyDeviceToHost, s));
    NGX_CUDA_TRY(cudaStreamSynchronize(s));

    const size_t ms = static_cast<size_t>(m);
    NGX_CUDA_TRY(cudaMalloc(&g->d_arcs_regular, std::max<size_t>(1, ms) * sizeof(Arc)));
    NGX_CUDA_TRY(cudaMalloc(&g->d_arcs_inverse, std::max<size_t>(1, ms) * sizeof(Arc)));
    NGX_CUDA_TRY(cudaMalloc(&g->d_arc_src, std::max<size_t>(1, ms) * 4));
    NGX_CUDA_TRY(cudaMalloc(&g->d_stored_of_user, std::max<int64_t>(1, m_user) * 4));
    uint32_t *d_target = nullptr, *d_target_sorted = nullptr;  // unsigned keys: the sort looks at the low bits only
    int32_t *d_index = nullptr, *d_index_sorted = nullptr;
    if ((rc = tmp.take(&d_target, ms)) != NGX_OK) return rc;
    if ((rc = tmp.take(&d_index, ms)) != NGX_OK) return rc;
    if ((rc = tmp.take(&d_target_sorted, ms)) != NGX_OK) return rc;
    if ((rc = tmp.take(&d_index_sorted, ms)) != NGX_OK) return rc;
    fill_rows_kernel<<<row_grid, kBuildBlock, 0, s>>>(d_user_rows, d_col, d_w, n, g->d_row_ptr, g->d_arcs_regular, g->d_arcs_inverse, g->d_arc_src,
                                                      g->d_stored_of_user, d_target, d_index);
    NGX_CUDA_TRY(cudaGetLastError());

    // reverse CSR: in-degrees -> row offsets; a stable radix sort of (target, stored index) keeps each target's
    // in-arcs in ascending stored order, which is ascending source order
    NGX_CUDA_TRY(cudaMemsetAsync(d_kept, 0, (static_cast<size_t>(n) + 1) * 8, s));
    if (m > 0) {
        in_degree_kernel<<<grid_for(m, kBuildBlock, g->sm_count), kBuildBlock, 0, s>>>(d_target, m, d_kept);
        NGX_CUDA_TRY(cudaGetLastError());
    }
    NGX_CUDA_TRY(cudaMalloc(&g->d_rrow_ptr, (static_cast<size_t>(n) + 1) * 8));
    NGX_CUDA_TRY(cub::DeviceScan::ExclusiveSum(d_scan, scan_bytes, d_kept, g->d_rrow_ptr, n + 1, s));
    NGX_CUDA_TRY(cudaMalloc(&g->d_rarcs, std::max<size_t>(1, ms) * sizeof(Arc)));
    if (m > 0) {
        size_t sort_bytes = 0;
        NGX_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, d_target, d_target_sorted, d_index, d_index_sorted, m, 0, bits_for(n), s));
        char* d_sort = nullptr;
        if ((rc = tmp.take(&d_sort, sort_bytes)) != NGX_OK) return rc;
        NGX_CUDA_TRY(cub::DeviceRadixSort::SortPairs(d_sort, sort_bytes, d_target, d_target_sorted, d_index, d_index_sorted, m, 0, bits_for(n), s));
        reverse_records_kernel<<<grid_for(m, kBuildBlock, g->sm_count), kBuildBlock, 0, s>>>(d_index_sorted, m, g->d_arcs_regular, g->d_arc_src,
                                                                                            g->d_rarcs);
        NGX_CUDA_TRY(cudaGetLastError());
    }
    NGX_CUDA_TRY(cudaStreamSynchronize(s));
    if (sums_thread.joinable()) {
        sums_thread.join();
    }
    if (stored_count != m) {
        return fail(NGX_CUDA_ERROR, "ngx_graph_create: the device build stored " + std::to_string(m) + " arcs, the host counted " +
                                        std::to_string(stored_count));
    }

    GraphPart part;
    part.n = n;
    part.m_user = m_user;
    part.m_stored = m;
    if (m > 0) {
        part.mean_len_regular = sum_regular / static_cast<double>(m);
        part.mean_len_inverse = sum_inverse / static_cast<double>(m);
        g->mean_len_regular = part.mean_len_regular;
        g->mean_len_inverse = part.mean_len_inverse;
        double lo = 0.0, hi = 0.0;
        std::memcpy(&lo, &red[2], 8);
        std::memcpy(&hi, &red[3], 8);
        g->min_len_regular = lo;
        g->max_len_regular = hi;
    }
    g->parts.assign(1, part);
    g->n = n;
    g->n_total = n;
    g->m_user = m_user;
    g->m_stored = m;
    g->max_out_degree = static_cast<int64_t>(red[1]);
    return NGX_OK;
}

}  // namespace ngx
