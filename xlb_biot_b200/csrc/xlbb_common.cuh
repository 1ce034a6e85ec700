// Shared device helpers of the xlbb kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace xlbb {

// D2Q8 velocity set of the elasticity lattice (reference src/lattice.py:124-127).
__host__ __device__ constexpr int cx8(int i) { return i == 0 ? 1 : i == 2 ? -1 : i == 4 ? 1 : i == 5 ? -1 : i == 6 ? -1 : i == 7 ? 1 : 0; }
__host__ __device__ constexpr int cy8(int i) { return i == 1 ? 1 : i == 3 ? -1 : i == 4 ? 1 : i == 5 ? 1 : i == 6 ? -1 : i == 7 ? -1 : 0; }
// D2Q9 velocity set of the Darcy lattice (src/lattice.py:128-131).
__host__ __device__ constexpr int cx9(int i) { return i == 3 ? 1 : i == 4 ? -1 : i == 5 ? 1 : i == 6 ? -1 : i == 7 ? 1 : i == 8 ? -1 : 0; }
__host__ __device__ constexpr int cy9(int i) { return i == 1 ? 1 : i == 2 ? -1 : i == 4 ? 1 : i == 5 ? -1 : i == 7 ? 1 : i == 8 ? -1 : 0; }
// D2Q9 weights (src/lattice.py:144-182): 4/9 rest, 1/9 axis, 1/36 diagonal.
template <typename T>
__host__ __device__ constexpr T w9(int i) {
    return i == 0 ? T(4.0 / 9.0) : (i == 1 || i == 2 || i == 3 || i == 6) ? T(1.0 / 9.0) : T(1.0 / 36.0);
}

template <typename T, int Q>
struct RulesView {
    int count;
    const int* row_ptr;
    const int* cell_x;
    const uint8_t* code;
    const T* cst;
    const uint32_t* mask;    // one bit per cell, words_per_row words per row
    const int* word_base;    // index of the first rule cell of each mask word
    int words_per_row;
    const uint32_t* push;    // per-cell push word of post-streaming rules (or NULL)
};

// Index of the rule of cell (x, y), or -1.  Rows are CSR, x sorted.
template <typename T, int Q>
__device__ __forceinline__ int find_rule(const RulesView<T, Q>& r, int y, int x) {
    if (r.count == 0) return -1;
    int lo = __ldg(r.row_ptr + y);
    const int end = __ldg(r.row_ptr + y + 1);
    int hi = end;
    if (lo == hi) return -1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(r.cell_x + mid) < x) lo = mid + 1; else hi = mid;
    }
    return (lo < end && __ldg(r.cell_x + lo) == x) ? lo : -1;
}

// Register-array element select by a runtime index without local memory.
template <typename T, int Q>
__device__ __forceinline__ T pick(const T (&v)[Q], int k) {
    T r = T(0);
#pragma unroll
    for (int j = 0; j < Q; ++j) r = (k == j) ? v[j] : r;
    return r;
}

// Rule value for direction d: base selected by the code, plus the constant.
template <typename T, int Q>
__device__ __forceinline__ T rule_value(uint8_t code, T cur, T src_val, T cst) {
    T base;
    if (code < Q) base = src_val;
    else if (code < 2 * Q) base = -src_val;
    else if (code == 2 * Q) base = T(0);
    else if (code == 2 * Q + 1) base = cur;
    else base = -cur;
    return base + cst;
}

__device__ __forceinline__ int wrap(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// 1 / feq in the KBC entropic products: correctly rounded in FP64; in FP32 the
// fast hardware reciprocal (__fdividef, within 2 ulp for feq's range), since
// the FP32 KBC collision is bound by these divisions.
template <typename T>
__device__ __forceinline__ T kbc_rcp(T x) { return T(1) / x; }
template <>
__device__ __forceinline__ float kbc_rcp<float>(float x) { return __fdividef(1.0f, x); }

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may be scheduled while its predecessor in the stream is still
// draining; it waits here, before touching any memory, until the predecessor
// has finished and its writes are visible (a no-op for an ordinary launch).
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Warp-wide FP64 sum (fixed butterfly order: deterministic), in every lane.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide FP64 sum (blockDim.x multiple of 32, <= 1024).
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        for (int i = 0; i < nw; ++i) s += sh[i];   // fixed order: deterministic
    }
    return s;
}

// The smoothers' mixing a * f + b * s with one fixed rounding (b * s rounded,
// then a fused multiply-add), the same in every sweep kernel, so that all launch
// forms of a sweep give bit-identical results.
template <typename T>
__device__ __forceinline__ T mix_ab(T a, T f, T b, T s) { return fma(a, f, b * s); }

// Block-wide FP64 sum for 2D blocks (warps follow the linear thread index;
// sh holds one double per warp): the total is returned in thread (0, 0).
__device__ __forceinline__ double block_sum_2d(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int lane = tid & 31, wid = tid >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (tid == 0) {
        const int nw = (blockDim.x * blockDim.y + 31) >> 5;
        for (int i = 0; i < nw; ++i) s += sh[i];   // fixed order: deterministic
    }
    return s;
}

}  // namespace xlbb
