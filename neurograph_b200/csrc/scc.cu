// Strongly connected components on the GPU: ngx_scc.
//
// Replaces StronglyConnectedComponents::compute_strongly_connected_components (source/metrics/connectivity/
// StronglyConnectedComponents.h:17-36): the number of components, the largest size and the size histogram, which
// every one of the reference's algorithms returns identically. Self arcs and weights are ignored; a vertex without
// arcs is a component of its own.
//
// Method (trimming + colouring, all passes over the device CSR and reverse CSR with one warp per vertex):
//   trim     an unassigned vertex without an unassigned in- or out-neighbour (other than itself) is a component;
//   colour   every unassigned vertex starts with its own id and takes the largest colour among its unassigned
//            in-neighbours until nothing changes: colour(v) = the largest id that reaches v;
//   peel     each vertex whose colour is its own id is a root (the largest vertex of its component, which names the
//            component); the vertices of its colour that reach it are its component, found backwards: a vertex joins
//            when one of its out-neighbours of the same colour has joined.
// Trim, colour and peel repeat until every vertex has a component. Every pass is a kernel launch followed by a host
// read of a change flag, so nothing waits on the device beyond one launch.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "ngx_common.cuh"
#include "ngx_graph.h"

namespace ngx {
namespace {

constexpr int kSccBlock = 256;

__device__ __forceinline__ int64_t global_warp() { return (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ int64_t warp_count() { return (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5; }

// Assigns every unassigned vertex that has no unassigned in- or out-neighbour besides itself.
__global__ void scc_trim_kernel(int64_t n, const int64_t* row_ptr, const Arc* arcs, const int64_t* rrow_ptr, const Arc* rarcs, int32_t* comp,
                                int* changed) {
    const int lane = threadIdx.x & 31;
    for (int64_t v = global_warp(); v < n; v += warp_count()) {
        if (comp[v] >= 0) {
            continue;  // warp-uniform
        }
        bool has_out = false, has_in = false;
        for (int64_t e = row_ptr[v] + lane; e < row_ptr[v + 1] && !has_out; e += 32) {
            const int32_t x = arcs[e].col;
            has_out = x != v && __ldcg(&comp[x]) < 0;
        }
        for (int64_t e = rrow_ptr[v] + lane; e < rrow_ptr[v + 1] && !has_in; e += 32) {
            const int32_t x = rarcs[e].col;
            has_in = x != v && __ldcg(&comp[x]) < 0;
        }
        const bool out_any = __any_sync(0xFFFFFFFFu, has_out);
        const bool in_any = __any_sync(0xFFFFFFFFu, has_in);
        if (lane == 0 && (!out_any || !in_any)) {
            comp[v] = static_cast<int32_t>(v);
            *changed = 1;
        }
    }
}

__global__ void scc_color_init_kernel(int64_t n, const int32_t* comp, int32_t* color, uint8_t* visited) {
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < n; v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        color[v] = comp[v] < 0 ? static_cast<int32_t>(v) : -1;
        visited[v] = 0;
    }
}

// colour(v) = max(colour(v), colour(u)) over unassigned in-neighbours u (pulled, so each vertex writes only itself).
__global__ void scc_color_kernel(int64_t n, const int64_t* rrow_ptr, const Arc* rarcs, const int32_t* comp, int32_t* color, int* changed) {
    const int lane = threadIdx.x & 31;
    for (int64_t v = global_warp(); v < n; v += warp_count()) {
        if (comp[v] >= 0) {
            continue;
        }
        int32_t best = -1;
        for (int64_t e = rrow_ptr[v] + lane; e < rrow_ptr[v + 1]; e += 32) {
            const int32_t u = rarcs[e].col;
            if (__ldcg(&comp[u]) < 0) {
                best = max(best, __ldcg(&color[u]));
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            best = max(best, __shfl_xor_sync(0xFFFFFFFFu, best, off));
        }
        if (lane == 0 && best > __ldcg(&color[v])) {
            atomicMax(&color[v], best);
            *changed = 1;
        }
    }
}

__global__ void scc_roots_kernel(int64_t n, const int32_t* comp, const int32_t* color, uint8_t* visited) {
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < n; v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (comp[v] < 0 && color[v] == static_cast<int32_t>(v)) {
            visited[v] = 1;
        }
    }
}

// A vertex joins its colour's root when one of its out-neighbours of the same colour already has.
__global__ void scc_backward_kernel(int64_t n, const int64_t* row_ptr, const Arc* arcs, const int32_t* comp, const int32_t* color, uint8_t* visited,
                                    int* changed) {
    const int lane = threadIdx.x & 31;
    for (int64_t v = global_warp(); v < n; v += warp_count()) {
        if (comp[v] >= 0 || __ldcg(&visited[v]) != 0) {
            continue;
        }
        const int32_t cv = color[v];
        bool hit = false;
        for (int64_t e = row_ptr[v] + lane; e < row_ptr[v + 1] && !hit; e += 32) {
            const int32_t x = arcs[e].col;
            hit = __ldcg(&visited[x]) != 0 && __ldcg(&color[x]) == cv && __ldcg(&comp[x]) < 0;
        }
        if (__any_sync(0xFFFFFFFFu, hit) && lane == 0) {
            visited[v] = 1;
            *changed = 1;
        }
    }
}

__global__ void scc_assign_kernel(int64_t n, int32_t* comp, const int32_t* color, const uint8_t* visited, int* remaining) {
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < n; v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (comp[v] < 0) {
            if (visited[v] != 0) {
                comp[v] = color[v];
            } else {
                atomicAdd(remaining, 1);
            }
        }
    }
}

__global__ void scc_count_kernel(int64_t n, const int32_t* comp, unsigned long long* sizes) {
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < n; v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        atomicAdd(&sizes[comp[v]], 1ull);
    }
}

// Runs `launch` (which may set *flag) until a pass leaves the flag clear. Every pass that sets it makes progress on a
// finite quantity (an assignment, a larger colour, a new member), so n + 1 passes always suffice.
template <typename Launch>
int until_stable(ngx_graph* g, int* d_flag, int* h_flag, int64_t max_passes, Launch launch) {
    for (int64_t pass = 0; pass <= max_passes; ++pass) {
        if (g->scc_pass_cap > 0 && ++g->scc_passes > g->scc_pass_cap) {
            return fail(NGX_TIMEOUT, "ngx_scc: more passes than the pre-pass allows");
        }
        NGX_CUDA_TRY(cudaMemsetAsync(d_flag, 0, sizeof(int), g->stream));
        launch();
        NGX_CUDA_TRY(cudaGetLastError());
        NGX_CUDA_TRY(cudaMemcpyAsync(h_flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, g->stream));
        NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
        if (*h_flag == 0) {
            return NGX_OK;
        }
    }
    return fail(NGX_TIMEOUT, "ngx_scc: a pass did not converge");
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace
}  // namespace ngx

using namespace ngx;

extern "C" {

int ngx_scc(ngx_graph* g, int32_t* component, uint64_t* number_components, uint64_t* largest_component, uint64_t* size_histogram) {
    return guard_host("ngx_scc", [&]() -> int {
        if (g == nullptr || number_components == nullptr || largest_component == nullptr) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_scc: graph or outputs are NULL");
        }
        if (g->parts.size() != 1) {
            return fail(NGX_INVALID_ARGUMENT, "ngx_scc: this handle holds a batch of graphs");
        }
        const int64_t n = g->n;
        *number_components = 0;
        *largest_component = 0;
        if (size_histogram != nullptr) {
            std::fill(size_histogram, size_histogram + n + 1, uint64_t(0));
        }
        if (n == 0) {
            return NGX_OK;
        }
        NGX_CUDA_TRY(cudaSetDevice(g->device));
        const size_t words = static_cast<size_t>(n);
        // device layout: comp i32[n] | color i32[n] | sizes u64[n] | visited u8[n] | flags i32[2], each 256-byte aligned
        const size_t off_color = align256(words * 4);
        const size_t off_sizes = off_color + align256(words * 4);
        const size_t off_visited = off_sizes + align256(words * 8);
        const size_t off_flags = off_visited + align256(words);
        const size_t bytes = off_flags + 256;
        if (const int rc = grow_buffer(g, &g->d_call_out, &g->call_out_bytes, bytes); rc != NGX_OK) {
            return rc;
        }
        char* base = static_cast<char*>(g->d_call_out);
        auto* comp = reinterpret_cast<int32_t*>(base);
        auto* color = reinterpret_cast<int32_t*>(base + off_color);
        auto* sizes = reinterpret_cast<unsigned long long*>(base + off_sizes);
        auto* visited = reinterpret_cast<uint8_t*>(base + off_visited);
        auto* flags = reinterpret_cast<int*>(base + off_flags);
        NGX_CUDA_TRY(cudaMemsetAsync(comp, 0xFF, words * 4, g->stream));  // -1: no component yet
        int h_flag = 0;
        const int vgrid = static_cast<int>(std::min<int64_t>((n + kSccBlock - 1) / kSccBlock, 8 * int64_t(g->sm_count)));
        const int wgrid = static_cast<int>(std::min<int64_t>((n * 32 + kSccBlock - 1) / kSccBlock, 32 * int64_t(g->sm_count)));
        const int64_t* row_ptr = g->d_row_ptr;
        const Arc* arcs = g->d_arcs_regular;
        const int64_t* rrow_ptr = g->d_rrow_ptr;
        const Arc* rarcs = g->d_rarcs;
        // every round assigns at least the largest unassigned vertex (its own colour's root)
        bool done = false;
        for (int64_t round = 0; round <= n && !done; ++round) {
            int rc = until_stable(g, flags, &h_flag, n, [&] {
                scc_trim_kernel<<<wgrid, kSccBlock, 0, g->stream>>>(n, row_ptr, arcs, rrow_ptr, rarcs, comp, flags);
            });
            if (rc != NGX_OK) {
                return rc;
            }
            scc_color_init_kernel<<<vgrid, kSccBlock, 0, g->stream>>>(n, comp, color, visited);
            NGX_CUDA_TRY(cudaGetLastError());
            rc = until_stable(g, flags, &h_flag, n, [&] { scc_color_kernel<<<wgrid, kSccBlock, 0, g->stream>>>(n, rrow_ptr, rarcs, comp, color, flags); });
            if (rc != NGX_OK) {
                return rc;
            }
            scc_roots_kernel<<<vgrid, kSccBlock, 0, g->stream>>>(n, comp, color, visited);
            NGX_CUDA_TRY(cudaGetLastError());
            rc = until_stable(g, flags, &h_flag, n,
                              [&] { scc_backward_kernel<<<wgrid, kSccBlock, 0, g->stream>>>(n, row_ptr, arcs, comp, color, visited, flags); });
            if (rc != NGX_OK) {
                return rc;
            }
            NGX_CUDA_TRY(cudaMemsetAsync(flags + 1, 0, sizeof(int), g->stream));
            scc_assign_kernel<<<vgrid, kSccBlock, 0, g->stream>>>(n, comp, color, visited, flags + 1);
            NGX_CUDA_TRY(cudaGetLastError());
            int remaining = 0;
            NGX_CUDA_TRY(cudaMemcpyAsync(&remaining, flags + 1, sizeof(int), cudaMemcpyDeviceToHost, g->stream));
            NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
            done = remaining == 0;
        }
        if (!done) {
            return fail(NGX_TIMEOUT, "ngx_scc: components did not converge");
        }
        // component sizes: a component is named by its largest vertex, so sizes[] is indexed by vertex
        NGX_CUDA_TRY(cudaMemsetAsync(sizes, 0, words * 8, g->stream));
        scc_count_kernel<<<vgrid, kSccBlock, 0, g->stream>>>(n, comp, sizes);
        NGX_CUDA_TRY(cudaGetLastError());
        std::vector<unsigned long long> host(words);
        NGX_CUDA_TRY(cudaMemcpyAsync(host.data(), sizes, words * 8, cudaMemcpyDeviceToHost, g->stream));
        if (component != nullptr) {
            NGX_CUDA_TRY(cudaMemcpyAsync(component, comp, words * 4, cudaMemcpyDeviceToHost, g->stream));
        }
        NGX_CUDA_TRY(cudaStreamSynchronize(g->stream));
        for (size_t v = 0; v < words; ++v) {
            if (host[v] != 0) {
                *number_components += 1;
                *largest_component = std::max<uint64_t>(*largest_component, host[v]);
                if (size_histogram != nullptr) {
                    size_histogram[host[v]] += 1;
                }
            }
        }
        return NGX_OK;
    });
}

}  // extern "C"
