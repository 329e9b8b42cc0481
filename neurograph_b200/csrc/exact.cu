// Host-side exact sums: accumulate doubles into, and round, the digit accumulators that the kernels build on the
// device (ngx_common.cuh). Used to merge the exact sums of several ranks (or runs) before the single rounding that
// the reference's AllPairsShortestPath.h:146-158 performs on its sequential sums.

#include <cmath>
#include <cstring>

#include "ngx_common.cuh"

static_assert(NGX_ACC_DIGITS == ngx::kAccDigits, "accumulator size mismatch");
static_assert(NGX_ACC_EXP0 == ngx::kAccExp0, "accumulator scale mismatch");

namespace ngx {
namespace {

// x = mant * 2^e (53-bit integer mant), added at absolute bit p = e - kAccExp0 into three 32-bit digits.
bool acc_add_host(unsigned long long* acc, double x) {
    if (!(x >= 0.0) || !std::isfinite(x)) {
        return false;
    }
    unsigned long long bits = 0;
    std::memcpy(&bits, &x, sizeof(bits));
    const unsigned long long biased = (bits >> 52) & 0x7FFull;
    const unsigned long long fraction = bits & ((1ull << 52) - 1ull);
    if (biased == 0 && fraction == 0) {
        return true;
    }
    const unsigned long long mant = biased == 0 ? fraction : (fraction | (1ull << 52));
    const int e = biased == 0 ? -1074 : static_cast<int>(biased) - 1075;
    const int p = e - kAccExp0;
    const int i = p >> 5;
    const int r = p & 31;
    const unsigned long long a = (mant & 0xFFFFFFFFull) << r;
    const unsigned long long b = (mant >> 32) << r;
    acc[i] += a & 0xFFFFFFFFull;
    acc[i + 1] += (a >> 32) + (b & 0xFFFFFFFFull);
    acc[i + 2] += b >> 32;
    return true;
}

}  // namespace
}  // namespace ngx

extern "C" {

int ngx_exact_accumulate(const double* values, int64_t count, uint64_t* digits) {
    if (digits == nullptr || (values == nullptr && count > 0) || count < 0) {
        return ngx::fail(NGX_INVALID_ARGUMENT, "ngx_exact_accumulate: NULL pointer or negative count");
    }
    auto* acc = reinterpret_cast<unsigned long long*>(digits);
    for (int64_t k = 0; k < count; ++k) {
        if (!ngx::acc_add_host(acc, values[k])) {
            ngx::acc_normalize(acc);
            return ngx::fail(NGX_INVALID_ARGUMENT, "ngx_exact_accumulate: values must be non-negative and finite");
        }
        if ((k & 0x3FFFFFFF) == 0x3FFFFFFF) {
            ngx::acc_normalize(acc);  // keep every word far below 2^64
        }
    }
    ngx::acc_normalize(acc);
    return NGX_OK;
}

double ngx_exact_round(uint64_t* digits) {
    if (digits == nullptr) {
        return 0.0;
    }
    auto* acc = reinterpret_cast<unsigned long long*>(digits);
    ngx::acc_normalize(acc);
    return ngx::acc_round_normalized(acc);
}

}  // extern "C"
