// Shared device/host definitions of the neurograph-b200 library (sm_100a).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <exception>
#include <new>
#include <string>

#include "ngx_b200.h"

namespace ngx {

constexpr int kTile = NGX_TILE;     // sources per CTA in the batched form (one per lane)
constexpr int kAccDigits = 72;      // exact accumulator: 72 digits of 32 bits in 64-bit words
constexpr int kAccExp0 = -1088;     // digit 0, bit 0 weighs 2^-1088 (below the smallest subnormal, 2^-1074)
constexpr unsigned long long kInfBits = 0x7FF0000000000000ull;  // +inf; non-negative doubles order like their bits

// Device arc record: one 128-bit load brings target, original arc index and FP64 length.
struct __align__(16) Arc {
    int32_t col;  // target (forward CSR) or source (reverse CSR)
    int32_t id;   // index of the arc in the caller's CSR (for gradients)
    double len;   // |w| or 1/|w|; zero-weight arcs are not stored
};
static_assert(sizeof(Arc) == 16, "Arc must be 16 bytes");

// Arc records are read-only while a kernel runs: loaded through the read-only data path (L1 kept), one 128-bit load.
__device__ __forceinline__ Arc ldg_arc(const Arc* p) {
    const int4 v = __ldg(reinterpret_cast<const int4*>(p));
    Arc a;
    a.col = v.x;
    a.id = v.y;
    a.len = __hiloint2double(v.w, v.z);
    return a;
}

struct DeviceCsr {
    int64_t n;
    int64_t m;               // stored (non-zero-weight) arcs
    const int64_t* row_ptr;  // n + 1
    const Arc* arcs;         // m
};

// One graph of a batch: its slice of the concatenated CSR arrays, its sources and outputs. A single-graph run is a
// batch of one.
struct GraphDesc {
    int64_t n;            // vertices (local ids 0..n-1)
    int64_t m;            // stored arcs
    int64_t row_off;      // start of the graph's n + 1 row offsets (forward and reverse CSR); values are global arc indices
    int64_t src_off;      // start of the graph's sources in `sources` and in the per-source outputs
    int64_t num_sources;
    int64_t bc_off;       // start of the graph's vertices in the betweenness output
    double delta;         // bucket width
};

// A unit of work of the persistent kernel: one tile of up to 32 sources of one graph.
struct WorkItem {
    int32_t graph;
    int32_t tile;
};

// What a tile computes after its distances are final.
enum TileMode : int { kModeApsp = 0, kModeBrandes = 1, kModeGrad = 2 };

// Per-graph launch counters (unsigned 64-bit words, kCounterCount per graph).
enum Counter : int {
    kUnreachable = 0,
    kReachedPairs = 1,
    kTraversedArcs = 2,
    kHistOverflow = 3,
    kDiameterBits = 4,
    kIterations = 5,   // near iterations (phases) over all tiles
    kExpansions = 6,   // vertex expansions (one warp pass over a vertex's arcs)
    kLaneExpansions = 7,  // (vertex, source) expansions; kLaneExpansions / kExpansions = sources sharing one arc pass
    kCyclesSssp = 8,      // SM cycles spent per phase, summed over CTAs (thread 0 between barriers)
    kCyclesCount = 9,
    kCyclesSigma = 10,
    kCyclesDelta = 11,
    kCyclesEpilogue = 12,
    kDagLevels = 13,      // Kahn levels of the shortest-path DAG, summed over tiles (Brandes / adjoint)
    kDagEntries = 14,     // (vertex, level) entries of the Kahn level lists, summed over tiles
    kDagScanTiles = 15,   // tiles whose DAG overflowed the successor lists (arc-scanning passes used)
    kCounterCount = 16
};

// Error codes written by kernels into a device flag (first writer wins).
enum DeviceError : int { kDevOk = 0, kDevTimeout = 1, kDevAborted = 2 };

// Bits of the lanes below this one in the warp.
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned mask;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(mask));
    return mask;
}

// ------------------------------------------------------------------------------------------ exact accumulation
// A non-negative finite double x = mant * 2^e (53-bit integer mant) is added exactly into 32-bit digits held in
// 64-bit words: its bit 0 lands at absolute bit p = e - kAccExp0 >= 14 and the shifted mantissa touches at most three
// digits, each of which grows by less than 2^33 per add. Word-wise integer addition is associative, so the result is
// independent of the order of the adds; acc_round() then rounds the exact value once, to nearest even.

__device__ __forceinline__ void acc_add_shared(unsigned long long* acc, double x) {
    const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(x));
    const unsigned long long biased = (bits >> 52) & 0x7FFull;
    const unsigned long long fraction = bits & ((1ull << 52) - 1ull);
    if (biased == 0 && fraction == 0) {
        return;
    }
    const unsigned long long mant = biased == 0 ? fraction : (fraction | (1ull << 52));
    const int e = biased == 0 ? -1074 : static_cast<int>(biased) - 1075;
    const int p = e - kAccExp0;
    const int i = p >> 5;
    const int r = p & 31;
    const unsigned long long a = (mant & 0xFFFFFFFFull) << r;
    const unsigned long long b = (mant >> 32) << r;
    const unsigned long long d0 = a & 0xFFFFFFFFull;
    const unsigned long long d1 = (a >> 32) + (b & 0xFFFFFFFFull);
    const unsigned long long d2 = b >> 32;
    if (d0 != 0) atomicAdd(&acc[i], d0);
    if (d1 != 0) atomicAdd(&acc[i + 1], d1);
    if (d2 != 0) atomicAdd(&acc[i + 2], d2);
}

__host__ __device__ inline void acc_normalize(unsigned long long* acc) {
    unsigned long long carry = 0;
    for (int i = 0; i < kAccDigits; ++i) {
        const unsigned long long t = acc[i] + carry;
        acc[i] = t & 0xFFFFFFFFull;
        carry = t >> 32;
    }
}

// Correct rounding of a normalized accumulator (all digits < 2^32): keep the 53 bits from the top set bit down to
// q = max(msb - 52, 14), round to nearest with ties to even using the next bit and a sticky OR of the rest.
__host__ __device__ inline double acc_round_normalized(const unsigned long long* d) {
    int top = -1;
    for (int i = kAccDigits - 1; i >= 0; --i) {
        if (d[i] != 0) {
            int b = 31;
            while (((d[i] >> b) & 1ull) == 0) {
                --b;
            }
            top = i * 32 + b;
            break;
        }
    }
    if (top < 0) {
        return 0.0;
    }
    int q = top - 52;
    if (q < 14) {
        q = 14;
    }
    unsigned long long mant = 0;
    for (int k = top; k >= q; --k) {
        mant = (mant << 1) | ((d[k >> 5] >> (k & 31)) & 1ull);
    }
    const int half_index = q - 1;
    const unsigned long long half = (d[half_index >> 5] >> (half_index & 31)) & 1ull;
    bool sticky = false;
    const int word = half_index >> 5;
    for (int i = 0; i < word && !sticky; ++i) {
        sticky = d[i] != 0;
    }
    const int rem = half_index & 31;
    if (!sticky && rem != 0) {
        sticky = (d[word] & ((1ull << rem) - 1ull)) != 0;
    }
    if (half && (sticky || (mant & 1ull))) {
        mant += 1ull;
    }
    return ldexp(static_cast<double>(mant), q + kAccExp0);
}

// ------------------------------------------------------------------------------------------ 128-bit fixed point
// Per-vertex / per-arc sums across source tiles (betweenness, gradients): value * 2^64 as an unsigned 128-bit
// integer in (lo, hi) words. Integer adds commute, so the totals do not depend on the order in which CTAs finish.
__device__ __forceinline__ void fixed_add(unsigned long long* lo_hi, double x) {
    if (!(x > 0.0)) {
        return;
    }
    const double whole = floor(x);
    const unsigned long long hi = static_cast<unsigned long long>(whole);
    const unsigned long long lo = static_cast<unsigned long long>(ldexp(x - whole, 64));
    const unsigned long long old = atomicAdd(&lo_hi[0], lo);
    const unsigned long long carry = (old + lo < old) ? 1ull : 0ull;
    if (hi + carry != 0) {
        atomicAdd(&lo_hi[1], hi + carry);
    }
}

// The fixed-point words of a non-negative double (the same truncation as fixed_add).
__device__ __forceinline__ void fixed_parts(double x, unsigned long long& lo, unsigned long long& hi) {
    lo = 0ull;
    hi = 0ull;
    if (x > 0.0) {
        const double whole = floor(x);
        hi = static_cast<unsigned long long>(whole);
        lo = static_cast<unsigned long long>(ldexp(x - whole, 64));
    }
}

// Adds a fixed-point value given as words (e.g. an exact sum of fixed_parts) to a 128-bit accumulator.
__device__ __forceinline__ void fixed_add_parts(unsigned long long* lo_hi, unsigned long long lo, unsigned long long hi) {
    const unsigned long long old = atomicAdd(&lo_hi[0], lo);
    const unsigned long long carry = (old + lo < old) ? 1ull : 0ull;
    if (hi + carry != 0) {
        atomicAdd(&lo_hi[1], hi + carry);
    }
}

// Exact sum over the warp's lanes of 128-bit fixed-point values (integer adds: the result does not depend on which
// values sit in which lane); every lane receives it.
__device__ __forceinline__ void fixed_warp_sum(unsigned long long& lo, unsigned long long& hi) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o_lo = __shfl_xor_sync(0xFFFFFFFFu, lo, off);
        const unsigned long long o_hi = __shfl_xor_sync(0xFFFFFFFFu, hi, off);
        const unsigned long long s = lo + o_lo;
        hi += o_hi + (s < lo ? 1ull : 0ull);
        lo = s;
    }
}

__host__ __device__ inline double fixed_value(unsigned long long lo, unsigned long long hi) {
    return static_cast<double>(hi) + ldexp(static_cast<double>(lo), -64);
}

// ------------------------------------------------------------------------------------------ host helpers
struct Error {
    int status;
    std::string message;
};

void set_last_error(const std::string& message);
int fail(int status, const std::string& message);
int cuda_fail(cudaError_t err, const char* what);

// Runs the body of a C entry point and turns a host exception (an allocation that failed) into a status, so that no
// exception crosses the C ABI.
template <typename Body>
int guard_host(const char* entry, const Body& body) noexcept {
    try {
        return body();
    } catch (const std::bad_alloc&) {
        return fail(NGX_OUT_OF_MEMORY, std::string(entry) + ": host allocation failed");
    } catch (const std::exception& e) {
        return fail(NGX_OUT_OF_MEMORY, std::string(entry) + ": " + e.what());
    } catch (...) {
        return fail(NGX_OUT_OF_MEMORY, std::string(entry) + ": host failure");
    }
}

}  // namespace ngx

#define NGX_CUDA_TRY(call)                                  \
    do {                                                    \
        cudaError_t ngx_err_ = (call);                      \
        if (ngx_err_ != cudaSuccess) {                      \
            return ::ngx::cuda_fail(ngx_err_, #call);       \
        }                                                   \
    } while (0)
