// Persistent multigrid tail of a batch: the coarse levels of every instance of
// a periodic elasticity batch in ONE launch, one CTA per instance, all of the
// tail's levels resident in that CTA's shared memory.
//
// The batched V-cycle (batched.py) runs the fine levels of all instances with
// one launch per sweep/transfer and level; below a size the launches are
// latency-bound (a few thousand cells per instance).  From the level where an
// instance's remaining levels fit in shared memory, this kernel finishes the
// V-cycle of that instance (src/elasticity.py:1221-1312, restricted to the
// batch's periodic levels >= 1):
//   level j < last: k damped sweeps from zero, residual sweep, restriction
//                   (2 x 2 block sums) into level j + 1, the level below,
//                   injection of its correction, k damped sweeps;
//   last level:     2 k damped sweeps, the first from zero.
// The arithmetic is the batched kernels' operation by operation (collision
// elast_collide, mixing mix_ab, restriction and prolongation sums in the
// wider type), so the results equal the level-by-level launches bit for bit.
// Only CTA barriers are used: nothing waits on another CTA.
// ---------------------------------------------------------------------------

namespace xlbb {

static constexpr int TAIL_MAX_LEVELS = 12;
static constexpr int TAIL_THREADS = 256;

__host__ __device__ inline size_t tail_align(size_t b) { return (b + 15) & ~size_t(15); }

// Dynamic shared memory of a tail whose top grid is nx x ny with `levels`
// levels (the last in TC): X and R per level, a ping-pong/residual buffer of
// the top size in T and one of the last level in TC.
template <typename T, typename TC>
__host__ __device__ inline size_t tail_smem_bytes(int nx, int ny, int levels) {
    size_t b = 0;
    for (int j = 0; j < levels; ++j) {
        const size_t n = (size_t)(nx >> j) * (size_t)(ny >> j);
        b += 2 * tail_align(8 * n * (j == levels - 1 ? sizeof(TC) : sizeof(T)));
    }
    b += tail_align(8 * (size_t)nx * (size_t)ny * sizeof(T));
    const size_t nl = (size_t)(nx >> (levels - 1)) * (size_t)(ny >> (levels - 1));
    b += tail_align(8 * nl * sizeof(TC));
    return b;
}

// One damped sweep out = a f + b STEP(f - r) of a periodic nx x ny level held
// in shared memory (planes of nx * ny cells); zero_in: f taken as zero.
// elast_rates with every operation rounded on its own (no fused multiply-add):
// the batched sweeps' rates are computed on the host (to_batch_inst), and the
// tail reproduces them bit for bit.
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rn_div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rn_div(double a, double b) { return __ddiv_rn(a, b); }

template <typename T>
__device__ __forceinline__ void tail_rates(T lam, T mu, T& cs, T& cd, T& h, T& n) {
    const T s = rn_add(lam, mu);
    T g = rn_div(T(1.0), rn_sub(rn_mul(T(12.0), s), T(4.0)));
    if (g > T(100) || g < T(-100)) g = T(0);
    h = rn_add(T(0.25), rn_mul(T(0.5), g));
    n = rn_mul(T(-0.25), g);
    const T t = rn_mul(T(3), s);
    cs = rn_div(rn_sub(t, T(1)), rn_add(t, T(1)));
    const T m6 = rn_mul(T(6), mu);
    cd = rn_div(rn_sub(m6, T(1)), rn_add(m6, T(1)));
}

template <typename U>
__device__ __forceinline__ void tail_sweep(const U* fin, U* fout, const U* r, int nx, int ny, U a, U b, bool zero_in,
                                           U cs, U cd, U h, U n) {
    const int N = nx * ny;
    for (int c = threadIdx.x; c < N; c += blockDim.x) {
        const int x = c % nx, y = c / nx;
        U g[8], fs[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) g[i] = (zero_in ? U(0) : fin[c + i * N]) - r[c + i * N];
        elast_collide<U>(g, false, U(0), U(0), cs, cd, h, n, fs);
        const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
        const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int zx = cx8(i) > 0 ? xp : (cx8(i) < 0 ? xm : x);
            const int zy = cy8(i) > 0 ? yp : (cy8(i) < 0 ? ym : y);
            const int z = zy * nx + zx + i * N;
            const U fz = zero_in ? U(0) : fin[z];
            fout[z] = mix_ab(a, fz, b, fs[i]);
        }
    }
}

// 2 x 2 block sums of the fine residual into the coarse right-hand side.
template <typename Uf, typename Uc>
__device__ __forceinline__ void tail_restrict(const Uf* res, Uc* rc, int nxf, int nyf) {
    using Ts = typename std::conditional<(sizeof(Uf) > sizeof(Uc)), Uf, Uc>::type;
    const int ncx = nxf / 2, Nf = nxf * nyf, Nc = ncx * (nyf / 2);
    for (int e = threadIdx.x; e < Nc; e += blockDim.x) {
        const int X = e % ncx, Y = e / ncx;
        const int o = (2 * Y) * nxf + 2 * X;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const Uf* s = res + o + i * Nf;
            rc[e + i * Nc] = Uc(Ts(s[0]) + Ts(s[nxf]) + Ts(s[1]) + Ts(s[nxf + 1]));
        }
    }
}

// Injection of the coarse correction, added to the fine level.
template <typename Uf, typename Uc>
__device__ __forceinline__ void tail_prolong(Uf* ff, const Uc* fc, int nxf, int nyf) {
    const int ncx = nxf / 2, Nf = nxf * nyf, Nc = ncx * (nyf / 2);
    for (int e = threadIdx.x; e < Nf; e += blockDim.x) {
        const int x = e % nxf, y = e / nxf;
        const int oc = (y / 2) * ncx + x / 2;
#pragma unroll
        for (int i = 0; i < 8; ++i) ff[e + i * Nf] = Uf(ff[e + i * Nf] + fc[oc + i * Nc]);
    }
}

template <typename U>
__device__ __forceinline__ void tail_smooth(U* x, U* y, const U* r, int nx, int ny, U a, U b, int k, bool from_zero,
                                            U cs, U cd, U h, U n) {
    for (int s = 0; s < k; ++s) {
        tail_sweep<U>(s % 2 == 0 ? x : y, s % 2 == 0 ? y : x, r, nx, ny, a, b, from_zero && s == 0, cs, cd, h, n);
        __syncthreads();
    }
}

template <typename T, typename TC>
__global__ void __launch_bounds__(TAIL_THREADS) batched_tail_kernel(const XlbbBatchTail* __restrict__ tails,
                                                                     double gamma, int k, size_t smem_bytes) {
    grid_dep_wait();
    extern __shared__ __align__(128) unsigned char smem[];
    const XlbbBatchTail tl = tails[blockIdx.x];
    const int m = tl.levels;
    // a record that does not fit the launch is skipped (nothing is touched)
    if (m < 1 || m > TAIL_MAX_LEVELS || (tl.nx >> (m - 1)) < 1 || (tl.ny >> (m - 1)) < 1 ||
        ((tl.nx >> (m - 1)) << (m - 1)) != tl.nx || ((tl.ny >> (m - 1)) << (m - 1)) != tl.ny ||
        tail_smem_bytes<T, TC>(tl.nx, tl.ny, m) > smem_bytes) {
        if (threadIdx.x == 0) note_status(XLBB_EBADARG);
        return;
    }
    void* X[TAIL_MAX_LEVELS];
    void* R[TAIL_MAX_LEVELS];
    size_t off = 0;
    for (int j = 0; j < m; ++j) {
        const size_t bytes = 8 * (size_t)(tl.nx >> j) * (size_t)(tl.ny >> j) * (j == m - 1 ? sizeof(TC) : sizeof(T));
        X[j] = smem + off;
        off += tail_align(bytes);
        R[j] = smem + off;
        off += tail_align(bytes);
    }
    T* Y = reinterpret_cast<T*>(smem + off);
    off += tail_align(8 * (size_t)tl.nx * tl.ny * sizeof(T));
    TC* Yc = reinterpret_cast<TC*>(smem + off);

    // the top level's right-hand side from global memory
    {
        const int nx = tl.nx, ny = tl.ny, N = nx * ny;
        for (int c = threadIdx.x; c < N; c += blockDim.x) {
            const size_t o = (size_t)(c / nx) * tl.pitch + (c % nx);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (m == 1) static_cast<TC*>(R[0])[c + i * N] = static_cast<const TC*>(tl.resid)[o + i * tl.plane];
                else static_cast<T*>(R[0])[c + i * N] = static_cast<const T*>(tl.resid)[o + i * tl.plane];
            }
        }
    }
    __syncthreads();

    T cs, cd, h, n;
    tail_rates<T>(T(tl.lam), T(tl.mu), cs, cd, h, n);
    TC csc, cdc, hc, nc;
    tail_rates<TC>(TC(tl.lam), TC(tl.mu), csc, cdc, hc, nc);
    const T a = T(1.0 - gamma), b = T(gamma);
    const TC ac = TC(1.0 - gamma), bc = TC(gamma);

    // descend: smoothing from zero, residual, restriction
    for (int j = 0; j < m - 1; ++j) {
        T* x = static_cast<T*>(X[j]);
        const T* r = static_cast<const T*>(R[j]);
        const int nx = tl.nx >> j, ny = tl.ny >> j;
        tail_smooth<T>(x, Y, r, nx, ny, a, b, k, true, cs, cd, h, n);
        tail_sweep<T>(x, Y, r, nx, ny, T(1), T(-1), false, cs, cd, h, n);
        __syncthreads();
        if (j + 1 == m - 1) tail_restrict<T, TC>(Y, static_cast<TC*>(R[j + 1]), nx, ny);
        else tail_restrict<T, T>(Y, static_cast<T*>(R[j + 1]), nx, ny);
        __syncthreads();
    }
    // the instance's coarsest level: 2 k sweeps, the first from zero
    {
        const int nx = tl.nx >> (m - 1), ny = tl.ny >> (m - 1);
        tail_smooth<TC>(static_cast<TC*>(X[m - 1]), Yc, static_cast<const TC*>(R[m - 1]), nx, ny, ac, bc, 2 * k, true,
                        csc, cdc, hc, nc);
    }
    // ascend: injection of the correction, smoothing
    for (int j = m - 2; j >= 0; --j) {
        T* x = static_cast<T*>(X[j]);
        const int nx = tl.nx >> j, ny = tl.ny >> j;
        if (j + 1 == m - 1) tail_prolong<T, TC>(x, static_cast<const TC*>(X[j + 1]), nx, ny);
        else tail_prolong<T, T>(x, static_cast<const T*>(X[j + 1]), nx, ny);
        __syncthreads();
        tail_smooth<T>(x, Y, static_cast<const T*>(R[j]), nx, ny, a, b, k, false, cs, cd, h, n);
    }
    // the top level's correction back to global memory
    {
        const int nx = tl.nx, ny = tl.ny, N = nx * ny;
        for (int c = threadIdx.x; c < N; c += blockDim.x) {
            const size_t o = (size_t)(c / nx) * tl.pitch + (c % nx);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (m == 1) static_cast<TC*>(tl.f_out)[o + i * tl.plane] = static_cast<const TC*>(X[0])[c + i * N];
                else static_cast<T*>(tl.f_out)[o + i * tl.plane] = static_cast<const T*>(X[0])[c + i * N];
            }
        }
    }
}

}  // namespace xlbb
