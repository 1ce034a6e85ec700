// xlbb: B200 (sm_100a) kernels of the lattice-Boltzmann Biot hot path and
// their C ABI (include/xlbb.h).  Reference: s-lunowa/xlb-biot src/elasticity.py,
// src/darcy.py, src/poroelasticity.py.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>
#include <cstdlib>
#include <utility>
#include <algorithm>
#include <climits>

#include "xlbb.h"
#include "xlbb_common.cuh"
#include "xlbb_sweep.cuh"

namespace xlbb {

static thread_local std::string g_last_error;

static int fail(int code, const char* msg) {
    g_last_error = msg;
    return code;
}

static int check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
        return XLBB_ELAUNCH;
    }
    return XLBB_OK;
}

// Every kernel of the library is launched here, with programmatic stream
// serialization (programmatic dependent launch): the next kernel of a stream
// (or of a captured CUDA graph) may be scheduled while its predecessor drains,
// which hides most of the launch gap between the short dependent sweeps of the
// multigrid levels; each kernel starts with grid_dep_wait(), so it touches no
// memory before its predecessor has finished.  XLBB_PDL=0 in the environment
// launches ordinarily.  Errors surface through cudaGetLastError (check_launch).
static bool pdl_enabled() {
    static const bool on = [] {
        const char* v = getenv("XLBB_PDL");
        return !(v && v[0] == '0');
    }();
    return on;
}

template <typename... KArgs, typename... Args>
static void launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Offsets inside one plane are 32-bit in the kernels: a plane holds < 2^31 elements.
static bool grid_ok(const XlbbGrid* g) {
    return g && g->nx > 0 && g->ny > 0 && g->pitch >= g->nx && g->plane >= (long long)g->pitch * g->ny &&
           g->plane < (1LL << 31);
}

static int g_num_sms = 0;
static int num_sms() {
    if (g_num_sms == 0) {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        g_num_sms = n > 0 ? n : 148;
    }
    return g_num_sms;
}

template <typename T, int Q>
static RulesView<T, Q> rules_view(const XlbbRules& r) {
    RulesView<T, Q> v;
    v.count = r.row_ptr ? r.count : 0;
    v.row_ptr = r.row_ptr;
    v.cell_x = r.cell_x;
    v.code = r.code;
    v.cst = static_cast<const T*>(r.cst);
    v.mask = r.mask;
    v.word_base = r.word_base;
    v.words_per_row = r.words_per_row;
    v.push = r.push;
    if (v.count > 0 && (r.mask == nullptr || r.word_base == nullptr)) v.count = 0;
    return v;
}

static bool rules_ok(const XlbbRules& r, const XlbbGrid* g) {
    if (r.count <= 0 || r.row_ptr == nullptr) return true;
    return r.cell_x && r.code && r.cst && r.mask && r.word_base && r.words_per_row * 32 >= g->nx;
}

// Launch shapes of the sweeps, per kernel family (0: elasticity, 1: Darcy):
// collide-and-push by default (sweeps with fused reductions use push_fallback).
// (pipeline 4 measured no faster than 3 on single 1 M-cell grids: 3.5 waves of
// its 512-thread CTAs; it stays a launch shape the autotuner can pick)
static XlbbSweepConfig g_cfg[2] = {{128, 1, 1, 8, 3}, {128, 1, 1, 8, 3}};

static constexpr int WARP_COLS = 30;   // output columns of one warp of sweep_warp_kernel

static bool cfg_ok(const XlbbSweepConfig& c) {
    const bool depth_ok = c.pipeline == 1 ? (c.depth == 2 || c.depth == 4 || c.depth == 6) : (c.depth == 1 || c.depth == 2);
    return (c.tx == 128 || c.tx == 256) && depth_ok && c.ctas_per_sm >= 1 && c.ctas_per_sm <= 32 &&
           c.min_rows >= 1 && c.pipeline >= 0 && c.pipeline <= 4;
}

// Pipeline 3 (collide-and-push) runs sweeps without fused reductions; the
// others run on this row-marching shape.
static XlbbSweepConfig push_fallback(bool f32) { return XlbbSweepConfig{f32 ? 256 : 128, 1, 3, 8, 0}; }

// ---------------------------------------------------------------------------
// D2Q8 elasticity (src/elasticity.py:805-848 transfer matrices, :959-1000
// collision, :1002-1058 moments).
// ---------------------------------------------------------------------------
// T: arithmetic type; S: storage type of the fields (S = float with T = double
// is FP32 storage with FP64 arithmetic).
template <typename T, typename S = T>
struct ElastMat {
    T cs, cd, h, n;   // uniform relaxation rates and m_to_f coefficients
    const S* lam_f;   // optional per-cell Lame fields
    const S* mu_f;
};

template <typename T>
__host__ __device__ inline void elast_rates(T lam, T mu, T& cs, T& cd, T& h, T& n) {
    // src/elasticity.py:810-813, :829-830, :973-974
    T g = T(1.0) / (T(12.0) * (lam + mu) - T(4.0));
    if (g > T(100) || g < T(-100)) g = T(0);
    h = T(0.25) + T(0.5) * g;
    n = T(-0.25) * g;
    cs = (T(3) * (lam + mu) - T(1)) / (T(3) * (lam + mu) + T(1));
    cd = (T(6) * mu - T(1)) / (T(6) * mu + T(1));
}

template <typename T>
__device__ __forceinline__ void elast_collide(const T (&f)[8], bool hasF, T F0, T F1, T cs, T cd, T h, T n,
                                              T (&o)[8]) {
    const T m0 = f[0] - f[2] + f[4] - f[5] - f[6] + f[7];
    const T m1 = f[1] - f[3] + f[4] + f[5] - f[6] - f[7];
    const T m2 = f[0] + f[1] + f[2] + f[3] + T(2) * (f[4] + f[5] + f[6] + f[7]);
    const T m3 = f[0] - f[1] + f[2] - f[3];
    const T m4 = f[4] - f[5] + f[6] - f[7];
    // thirds and sixths by multiplication with the rounded constants (one
    // rounding each, like the division, at a fraction of its instructions);
    // the sums with one explicit fused multiply-add, so that every kernel
    // rounds them alike
    constexpr T third = T(1.0 / 3.0), sixth = T(1.0 / 6.0);
    T M0 = m0, M1 = m1, M5 = third * m0, M6 = third * m1;
    if (hasF) {
        M0 = m0 + F0;
        M1 = m1 + F1;
        M5 = fma(sixth, F0, M5);
        M6 = fma(sixth, F1, M6);
    }
    const T M2 = m2 * cs, M3 = m3 * cd, M4 = m4 * cd;
    o[0] = T(0.5) * M0 + h * M2 + T(0.25) * M3 - T(0.5) * M5;
    o[1] = T(0.5) * M1 + h * M2 - T(0.25) * M3 - T(0.5) * M6;
    o[2] = T(-0.5) * M0 + h * M2 + T(0.25) * M3 + T(0.5) * M5;
    o[3] = T(-0.5) * M1 + h * M2 - T(0.25) * M3 + T(0.5) * M6;
    o[4] = n * M2 + T(0.25) * M4 + T(0.25) * M5 + T(0.25) * M6;
    o[5] = n * M2 - T(0.25) * M4 - T(0.25) * M5 + T(0.25) * M6;
    o[6] = n * M2 + T(0.25) * M4 - T(0.25) * M5 - T(0.25) * M6;
    o[7] = n * M2 - T(0.25) * M4 + T(0.25) * M5 - T(0.25) * M6;
}

// T_: arithmetic type (registers, the post-collision ring, boundary-rule
// constants); S_: storage type of the fields in HBM.  S_ = float with
// T_ = double is the FP32-storage / FP64-arithmetic sweep (register-prefetch
// pipeline only).
template <typename T_, bool RESID, typename S_ = T_>
struct ElastPhys {
    using T = T_;
    using Storage = S_;
    static constexpr int Q = 8;
    __host__ __device__ static constexpr int cx(int i) { return cx8(i); }
    __host__ __device__ static constexpr int cy(int i) { return cy8(i); }
    struct Args {
        SweepGeom geom;
        const S_* f_in;
        S_* f_out;
        const S_* force;
        const S_* fext;
        const S_* resid;
        T a, b;
        ElastMat<T, S_> mat;
        RulesView<T, 8> pc, ps;
        double* sumsq;
        int bx0, bx1, by0, by1;
        S_* div_out;
        T div_scale;
        int mix;   // 0: out = S; 1: out = a f + b S
        int sumsq_diff;   // sumsq of (out - f_in) instead of out
        int ext_in_kernel = 0;   // the external force is computed by the kernel itself (not loaded)
        static constexpr int PMAX = 20;
        const S_* planes[PMAX];   // input planes in from_smem order (bulk-copy kernel)
        int np;
        // Plane pointers in fixed slots (f 0-7, resid 8-15, force 16-17, fext
        // 18-19; NULL when absent), so a kernel addresses plane i of a cell as
        // ip[i] + (32-bit cell offset) instead of base + i * plane.
        const S_* ip[20];
        S_* op[8];
    };
    __host__ __device__ static void fill_ptrs(Args& a) {
        const long long P = a.geom.plane;
        for (int i = 0; i < 8; ++i) {
            a.ip[i] = a.f_in + i * P;
            a.ip[8 + i] = a.resid ? a.resid + i * P : nullptr;
            a.op[i] = a.f_out + i * P;
        }
        a.ip[16] = a.force;
        a.ip[17] = a.force ? a.force + P : nullptr;
        a.ip[18] = a.fext;
        a.ip[19] = a.fext ? a.fext + P : nullptr;
    }
    struct In {
        T f[8];
        T r[RESID ? 8 : 1];
        T F0, F1;
    };
    // Input planes: f[0..7], resid[0..7] (RESID), force[0..1], fext[0..1].
    static int make_planes(Args& a) {
        int k = 0;
        for (int i = 0; i < 8; ++i) a.planes[k++] = a.f_in + i * a.geom.plane;
        if (RESID)
            for (int i = 0; i < 8; ++i) a.planes[k++] = a.resid + i * a.geom.plane;
        if (a.force) { a.planes[k++] = a.force; a.planes[k++] = a.force + a.geom.plane; }
        if (a.fext) { a.planes[k++] = a.fext; a.planes[k++] = a.fext + a.geom.plane; }
        a.np = k;
        return k;
    }
    __device__ static void from_smem(const Args& p, const T* s, int rs, int col, In& in) {
        int k = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) in.f[i] = s[(k++) * rs + col];
        if (RESID) {
#pragma unroll
            for (int i = 0; i < 8; ++i) in.r[i] = s[(k++) * rs + col];
        }
        T F0 = T(0), F1 = T(0);
        if (p.force) { F0 = s[k * rs + col]; F1 = s[(k + 1) * rs + col]; k += 2; }
        if (p.fext) {
            const T e0 = s[k * rs + col], e1 = s[(k + 1) * rs + col];
            if (p.force) { F0 = F0 + e0; F1 = F1 + e1; } else { F0 = e0; F1 = e1; }
        }
        in.F0 = F0;
        in.F1 = F1;
    }
    __device__ static void load(const Args& p, int y, int x, In& in) {
        const int o = y * p.geom.pitch + x;
#pragma unroll
        for (int i = 0; i < 8; ++i) in.f[i] = T(__ldg(p.ip[i] + o));
        if (RESID) {
#pragma unroll
            for (int i = 0; i < 8; ++i) in.r[i] = T(__ldg(p.ip[8 + i] + o));
        }
        T F0 = T(0), F1 = T(0);
        if (p.force) { F0 = T(__ldg(p.ip[16] + o)); F1 = T(__ldg(p.ip[17] + o)); }
        if (p.fext) {
            const T e0 = T(__ldg(p.ip[18] + o)), e1 = T(__ldg(p.ip[19] + o));
            if (p.force) { F0 = F0 + e0; F1 = F1 + e1; } else { F0 = e0; F1 = e1; }
        }
        in.F0 = F0;
        in.F1 = F1;
    }
    __device__ static void fin(const In& in, T (&g)[8]) {
#pragma unroll
        for (int i = 0; i < 8; ++i) g[i] = RESID ? in.f[i] - in.r[i] : in.f[i];
    }
    // Output population i of cell (zx, zy) (offset o) from its streamed-in
    // value s, with the store stage's algebra (collide-and-push sweep); returns
    // the value's term of the fused FP64 sum of squares (0 without one).
    template <bool SUMSQ>
    __device__ static double put(const Args& p, int i, int o, int zx, int zy, T s) {
        T v = s;
        T fz = T(0);
        if (p.mix || (SUMSQ && p.sumsq_diff)) fz = T(__ldg(p.ip[i] + o));
        if (p.mix) v = mix_ab(p.a, fz, p.b, s);
        const S_ sv = S_(v);
        p.op[i][o] = sv;
        if constexpr (SUMSQ) {
            if (zx < p.bx0 || zx >= p.bx1 || zy < p.by0 || zy >= p.by1) return 0.0;
            double d = (double)sv;
            if (p.sumsq_diff) d -= (double)S_(fz);
            return d * d;
        }
        return 0.0;
    }
    static bool push_ok(const Args& a) { return a.div_out == nullptr; }
    __device__ static T f_in(const In& in, int i) { return in.f[i]; }
    __device__ static void collide(const Args& p, int y, int x, const In& in, T (&o)[8]) {
        T g[8];
        fin(in, g);
        T cs = p.mat.cs, cd = p.mat.cd, h = p.mat.h, n = p.mat.n;
        if (p.mat.mu_f) {
            const int c = y * p.geom.pitch + x;
            elast_rates<T>(T(__ldg(p.mat.lam_f + c)), T(__ldg(p.mat.mu_f + c)), cs, cd, h, n);
        }
        elast_collide<T>(g, p.force != nullptr || p.fext != nullptr || p.ext_in_kernel, in.F0, in.F1, cs, cd, h, n, o);
    }
    template <bool PREV>
    __device__ static double store(const Args& p, int y, int x, T (&S)[8], const T* fprev) {
        const int o = y * p.geom.pitch + x;
        double acc = 0.0;
        T m2 = T(0);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            T v = S[i];
            if constexpr (PREV) {
                if (p.mix) v = mix_ab(p.a, fprev[i], p.b, S[i]);
            }
            const S_ sv = S_(v);
            p.op[i][o] = sv;
            double d = (double)sv;
            if constexpr (PREV) {
                if (p.sumsq_diff) d -= (double)S_(fprev[i]);
            }
            acc += d * d;
            m2 += (i < 4 ? T(1) : T(2)) * v;
        }
        if (p.div_out) p.div_out[o] = S_(p.div_scale * m2);
        const bool in_box = x >= p.bx0 && x < p.bx1 && y >= p.by0 && y < p.by1;
        return in_box ? acc : 0.0;
    }
};

// ---------------------------------------------------------------------------
// D2Q9 advection-diffusion-reaction BGK (src/darcy.py:106-129).
// ---------------------------------------------------------------------------
// T_: arithmetic type; St_: storage type of the fields (St_ = float with
// T_ = double is FP32 storage with FP64 arithmetic, the 'f64/f32' policy).
template <typename T_, typename St_ = T_, bool RES_ = false>
struct DarcyPhys {
    using T = T_;
    using St = St_;
    using Storage = St_;
    static constexpr int Q = 9;
    __host__ __device__ static constexpr int cx(int i) { return cx9(i); }
    __host__ __device__ static constexpr int cy(int i) { return cy9(i); }
    struct Args {
        SweepGeom geom;
        const St* f_in;
        St* f_out;
        T omega;
        const St* omega_f;
        const St* source;
        const St* ext;
        const St* resid;         // 9 planes subtracted from the input before the collision, or NULL
        RulesView<T, 9> pc, ps;
        double* sumsq;
        static constexpr int PMAX = 12;
        const St* planes[PMAX];  // input planes in from_smem order (bulk-copy kernel, St = T only)
        int np;
        // Plane pointers in fixed slots (f 0-8, omega 9, source 10, ext 11)
        const St* ip[12];
        St* op[9];
    };
    __host__ __device__ static void fill_ptrs(Args& a) {
        for (int i = 0; i < 9; ++i) {
            a.ip[i] = a.f_in + i * a.geom.plane;
            a.op[i] = a.f_out + i * a.geom.plane;
        }
        a.ip[9] = a.omega_f;
        a.ip[10] = a.source;
        a.ip[11] = a.ext;
    }
    struct In {
        T f[9];
        T S;
        T om;
    };
    // Input planes: f[0..8], omega (per cell), source, ext_source.
    static int make_planes(Args& a) {
        int k = 0;
        for (int i = 0; i < 9; ++i) a.planes[k++] = a.f_in + i * a.geom.plane;
        if (a.omega_f) a.planes[k++] = a.omega_f;
        if (a.source) a.planes[k++] = a.source;
        if (a.ext) a.planes[k++] = a.ext;
        a.np = k;
        return k;
    }
    __device__ static void from_smem(const Args& p, const T* s, int rs, int col, In& in) {
        int k = 0;
#pragma unroll
        for (int i = 0; i < 9; ++i) in.f[i] = s[(k++) * rs + col];
        in.om = p.omega_f ? s[(k++) * rs + col] : p.omega;
        T S = T(0);
        if (p.source) S = s[(k++) * rs + col];
        if (p.ext) S = p.source ? S + s[(k++) * rs + col] : s[(k++) * rs + col];
        in.S = S;
    }
    __device__ static void load(const Args& p, int y, int x, In& in) {
        const int o = y * p.geom.pitch + x;
#pragma unroll
        for (int i = 0; i < 9; ++i) in.f[i] = T(__ldg(p.ip[i] + o));
        T S = T(0);
        if (p.source) S = T(__ldg(p.ip[10] + o));
        if (p.ext) S = p.source ? S + T(__ldg(p.ip[11] + o)) : T(__ldg(p.ip[11] + o));
        in.S = S;
        in.om = p.omega_f ? T(__ldg(p.ip[9] + o)) : p.omega;
    }
    __device__ static void fin(const In& in, T (&g)[9]) {
#pragma unroll
        for (int i = 0; i < 9; ++i) g[i] = in.f[i];
    }
    template <bool SUMSQ>
    __device__ static double put(const Args& p, int i, int o, int, int, T s) {
        const St sv = St(s);
        p.op[i][o] = sv;
        if constexpr (SUMSQ) {
            const double d = (double)sv - (double)__ldg(p.ip[i] + o);
            return d * d;
        }
        return 0.0;
    }
    static bool push_ok(const Args&) { return true; }
    __device__ static T f_in(const In& in, int i) { return in.f[i]; }
    __device__ static void collide(const Args& p, int y, int x, const In& in, T (&o)[9]) {
        const bool hasS = p.source != nullptr || p.ext != nullptr;
        T f[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) f[i] = in.f[i];
        if constexpr (RES_) {   // the sweep of f - resid (the correction equation of a refinement step)
            const size_t o = (size_t)y * p.geom.pitch + x;
#pragma unroll
            for (int i = 0; i < 9; ++i) f[i] = f[i] - T(__ldg(p.resid + (o + (size_t)i * p.geom.plane)));
        }
        T rho = f[0];
#pragma unroll
        for (int i = 1; i < 9; ++i) rho += f[i];
        if (hasS) rho = rho + T(0.5) * in.S;
        const T om = in.om;
        const T sf = T(1) - T(0.5) * om;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const T feq = rho * w9<T>(i);
            T v = f[i] - om * (f[i] - feq);
            if (hasS) v = v + in.S * (sf * w9<T>(i));
            o[i] = v;
        }
    }
    template <bool PREV>
    __device__ static double store(const Args& p, int y, int x, T (&S)[9], const T* fprev) {
        const int o = y * p.geom.pitch + x;
        double acc = 0.0;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const St sv = St(S[i]);
            p.op[i][o] = sv;
            if constexpr (PREV) {
                const double d = (double)sv - (double)St(fprev[i]);
                acc += d * d;
            }
        }
        return acc;
    }
};

// ---------------------------------------------------------------------------
// D2Q9 fluid models of src/models.py: BGK (:20-34) and KBC (:48-72).
// rho = sum f, u = sum c f / rho (src/base.py:748-772), feq = rho w (1 + cu
// (1 + cu / 2) - usqr) with cu = 3 c.u, usqr = 3/2 |u|^2 (src/base.py:686-724).
// BGK: f* = f - omega (f - feq).  KBC: fneq = f - feq splits into the shear
// part dS (fdecompose_shear_d2q9, :127-154, times rho / 4) and dH = fneq - dS;
// with beta = omega / 2 and the entropic products <x, y> = sum x y / feq,
// gamma = 1 / beta - (2 - 1 / beta) <dS, dH> / (1e-32 + <dH, dH>) and
// f* = f - beta (2 dS + gamma dH).  Same planes, rules and sweep pipelines as
// the Darcy step; only the collision differs (no source terms: the fluid entry
// point rejects them).
// ---------------------------------------------------------------------------
template <typename T_, bool KBC>
struct FluidPhys : DarcyPhys<T_> {
    using T = T_;
    using Args = typename DarcyPhys<T_>::Args;
    using In = typename DarcyPhys<T_>::In;
    __device__ static void collide(const Args&, int, int, const In& in, T (&o)[9]) {
        T rho = in.f[0];
#pragma unroll
        for (int i = 1; i < 9; ++i) rho += in.f[i];
        // momentum: D2Q9 x-velocities (+) 3, 5, 7 and (-) 4, 6, 8; y (+) 1, 4, 7 and (-) 2, 5, 8
        const T jx = ((in.f[3] - in.f[4]) + (in.f[5] - in.f[6])) + (in.f[7] - in.f[8]);
        const T jy = ((in.f[1] - in.f[2]) + (in.f[4] - in.f[5])) + (in.f[7] - in.f[8]);
        // one reciprocal of rho instead of two divisions (u = j / rho)
        const T irho = T(1) / rho;
        const T ux = jx * irho, uy = jy * irho;
        const T usqr = T(1.5) * (ux * ux + uy * uy);
        const T om = in.om;
        T feq[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const T cu = T(3) * (T(cx9(i)) * ux + T(cy9(i)) * uy);
            feq[i] = rho * w9<T>(i) * (T(1) + cu * (T(1) + T(0.5) * cu) - usqr);
        }
        if constexpr (!KBC) {
#pragma unroll
            for (int i = 0; i < 9; ++i) o[i] = in.f[i] - om * (in.f[i] - feq[i]);
        } else {
            T fneq[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) fneq[i] = in.f[i] - feq[i];
            // momentum flux of fneq: axis directions 1-4 / 6 carry cx^2 or cy^2,
            // diagonals 4, 5, 7, 8 carry both and cx cy = -1 (4, 5) or +1 (7, 8)
            const T dg = ((fneq[4] + fneq[5]) + (fneq[7] + fneq[8]));
            const T pxx = (fneq[3] + fneq[6]) + dg;
            const T pyy = (fneq[1] + fneq[2]) + dg;
            const T pxy = (fneq[7] + fneq[8]) - (fneq[4] + fneq[5]);
            const T N = pxx - pyy;
            const T r4 = rho * T(0.25);
            T dS[9];
            dS[0] = T(0);
            dS[1] = -N * r4;
            dS[2] = -N * r4;
            dS[3] = N * r4;
            dS[6] = N * r4;
            dS[4] = -pxy * r4;
            dS[5] = -pxy * r4;
            dS[7] = pxy * r4;
            dS[8] = pxy * r4;
            // entropic products <x, y> = sum x y / feq with one reciprocal of
            // feq per direction shared by both products
            T sh = T(0), hh = T(0);
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                const T dH = fneq[i] - dS[i];
                const T ife = kbc_rcp<T>(feq[i]);
                sh += (dS[i] * dH) * ife;
                hh += (dH * dH) * ife;
            }
            const T beta = om * T(0.5);
            const T ib = T(1) / beta;
            const T gamma = ib - (T(2) - ib) * sh / (T(1e-32) + hh);
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                const T dH = fneq[i] - dS[i];
                o[i] = in.f[i] - beta * (T(2) * dS[i] + gamma * dH);
            }
        }
    }
};

#include "xlbb_push.cuh"
#include "xlbb_fluid3.cuh"
#include "xlbb_darcy4.cuh"

// Launch geometry of the sweeps: tx owned columns per CTA, strips of rows
// chosen so that the grid holds about ctas_per_sm CTAs per SM (one wave),
// never shorter than min_rows rows (each strip recomputes two halo rows).
struct WarpGrid {
    int nbx, nstrips, ctas;
};

static WarpGrid warp_grid(const XlbbGrid* g, const XlbbSweepConfig& c) {
    WarpGrid w;
    w.nbx = (g->nx + WARP_COLS - 1) / WARP_COLS;
    const int target = c.ctas_per_sm * 4 * num_sms();
    int ns = target / w.nbx;
    const int max_s = g->ny / c.min_rows > 0 ? g->ny / c.min_rows : 1;
    if (ns > max_s) ns = max_s;
    if (ns < 1) ns = 1;
    if (ns > g->ny) ns = g->ny;
    w.nstrips = ns;
    w.ctas = (w.nbx * ns + 3) / 4;
    return w;
}

static dim3 sweep_grid(const XlbbGrid* g, const XlbbSweepConfig& c) {
    if (c.pipeline == 2) return dim3(warp_grid(g, c).ctas, 1);
    const int nbx = (g->nx + c.tx - 1) / c.tx;
    const int target = c.ctas_per_sm * num_sms();
    int nby = target / nbx;
    const int max_by = g->ny / c.min_rows > 0 ? g->ny / c.min_rows : 1;
    if (nby > max_by) nby = max_by;
    if (nby < 1) nby = 1;
    if (nby > g->ny) nby = g->ny;
    return dim3(nbx, nby);
}

// The launch shape a sweep takes under config c: pipeline 3 collides and
// pushes only when the sweep is push-eligible (its post-streaming rules carry
// push words and it has no divergence side output); otherwise it runs on the
// row-marching fallback shape.  Every launcher and every partial-count query
// resolves the shape here, so a fused sum's partials are counted on the grid
// that wrote them.
static XlbbSweepConfig resolve_shape(XlbbSweepConfig c, bool push, bool f32) {
    if (c.pipeline == 3 && !push) return push_fallback(f32);
    return c;
}

// CTAs (= FP64 partials of a fused sum) of a launch with the resolved shape c.
static long long launch_ctas(const XlbbGrid* g, const XlbbSweepConfig& c) {
    if (c.pipeline == 3) return (long long)((g->nx + c.tx - 1) / c.tx) * g->ny;   // one per push block
    const dim3 a = sweep_grid(g, c);
    return (long long)a.x * a.y;
}

template <class Ph>
static bool push_eligible(const typename Ph::Args& a) {
    return Ph::push_ok(a) && (a.ps.count == 0 || a.ps.push != nullptr);
}

// Runtime (tx, depth) -> template instance.
template <class Ph, int TX, int D, bool PREV>
static void launch_bulk(dim3 grid, cudaStream_t st, const typename Ph::Args& a) {
    using T = typename Ph::T;
    static size_t configured = 0;   // max dynamic smem already granted to this instance
    const size_t bytes = bulk_smem_bytes<T, Ph::Q, TX, D>(a.np);
    auto k = sweep_bulk_kernel<Ph, TX, D, PREV>;
    if (bytes > configured) {
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        configured = bytes;
    }
    launch_k(k, grid, TX + 32, bytes, st, a);
}

// 16-byte alignment of every input plane and of the row pitch: the bulk copies need it.
template <class Ph>
static bool bulk_aligned(const typename Ph::Args& a) {
    using T = typename Ph::T;
    if ((a.geom.pitch * sizeof(T)) % 16 != 0) return false;
    for (int k = 0; k < a.np; ++k)
        if (reinterpret_cast<uintptr_t>(a.planes[k]) % 16 != 0) return false;
    return true;
}

// Collide and push: one thread per cell, tx threads per block along x, one row
// per block row; with fused partials, one FP64 partial per block.
template <class Ph>
static void launch_push(const XlbbSweepConfig& c, const XlbbGrid* g, cudaStream_t st, const typename Ph::Args& a) {
    const dim3 grid((g->nx + c.tx - 1) / c.tx, g->ny);
    if (a.sumsq) launch_k(push_kernel<Ph, true>, grid, c.tx, 0, st, a);
    else launch_k(push_kernel<Ph, false>, grid, c.tx, 0, st, a);
}

// Runtime (bulk, tx, depth) -> template instance.  The register-prefetch
// kernel takes depth 1..2, the bulk-copy ring depth 2, 4 or 6; FP64 uses
// tx = 128 (larger rings exceed the shared memory of one SM).
template <class Ph, bool PREV>
static void launch_sweep(XlbbSweepConfig c, const XlbbGrid* g, cudaStream_t st, typename Ph::Args& a) {
    constexpr bool F32 = sizeof(typename Ph::T) == 4;
    Ph::fill_ptrs(a);
    c = resolve_shape(c, push_eligible<Ph>(a), F32);
    if (c.pipeline == 3) {
        launch_push<Ph>(c, g, st, a);
        return;
    }
    const dim3 grid = sweep_grid(g, c);
    if (c.pipeline == 2) {
        const WarpGrid wg = warp_grid(g, c);
        if (c.depth == 2) launch_k(sweep_warp_kernel<Ph, 2, PREV>, wg.ctas, 128, 0, st, a, wg.nbx, wg.nstrips);
        else launch_k(sweep_warp_kernel<Ph, 1, PREV>, wg.ctas, 128, 0, st, a, wg.nbx, wg.nstrips);
        return;
    }
    constexpr bool SAME = std::is_same<typename Ph::T, typename Ph::Storage>::value;
    if constexpr (SAME) Ph::make_planes(a);
    if (c.pipeline == 1 && (!SAME || !bulk_aligned<Ph>(a))) {     // the bulk ring holds the arithmetic type
        c.pipeline = 0;
        c.depth = c.depth > 2 ? 2 : c.depth;
    }
    if constexpr (SAME) if (c.pipeline == 1) {
#define XLBB_BULK(TX_, D_)                                              \
    if (c.tx == TX_ && c.depth == D_) {                                  \
        launch_bulk<Ph, TX_, D_, PREV>(grid, st, a);                     \
        return;                                                          \
    }
        XLBB_BULK(128, 2) XLBB_BULK(128, 4)
        if constexpr (F32) { XLBB_BULK(128, 6) XLBB_BULK(256, 2) XLBB_BULK(256, 4) XLBB_BULK(256, 6) }
#undef XLBB_BULK
        launch_bulk<Ph, 128, 2, PREV>(grid, st, a);
        return;
    }
#define XLBB_CASE(TX_, D_)                                                            \
    if (c.tx == TX_ && c.depth == D_) {                                                \
        launch_k(sweep_kernel<Ph, TX_, D_, PREV>, grid, TX_ + 32, 0, st, a);                 \
        return;                                                                        \
    }
    XLBB_CASE(128, 1) XLBB_CASE(128, 2)
    if constexpr (F32) { XLBB_CASE(256, 1) XLBB_CASE(256, 2) }
#undef XLBB_CASE
    launch_k(sweep_kernel<Ph, 128, 1, PREV>, grid, 128 + 32, 0, st, a);
}

// FP32 storage / FP64 arithmetic: the register-prefetch kernel at tx = 128
// (c is a resolved row-marching shape).
template <class Ph, bool PREV>
static void launch_sweep_regs(const XlbbSweepConfig& c, const XlbbGrid* g, cudaStream_t st,
                              typename Ph::Args& a) {
    Ph::fill_ptrs(a);
    const dim3 grid = sweep_grid(g, c);
    if (c.depth == 2) launch_k(sweep_kernel<Ph, 128, 2, PREV>, grid, 128 + 32, 0, st, a);
    else launch_k(sweep_kernel<Ph, 128, 1, PREV>, grid, 128 + 32, 0, st, a);
}

// The configuration a launch actually uses (FP64 arithmetic caps tx at 128;
// the FP32-storage / FP64-arithmetic sweep has only the register-prefetch
// pipeline, depth <= 2).
static XlbbSweepConfig effective_cfg(int kernel, int dtype) {
    XlbbSweepConfig c = g_cfg[kernel];
    if (c.pipeline == 4) c.pipeline = 3;   // the four-column form is chosen per sweep (launch_elast)
    if ((dtype == XLBB_F64 || dtype == XLBB_F32_ACC64) && c.tx > 128) c.tx = 128;
    if (dtype == XLBB_F32_ACC64 && (c.pipeline == 1 || c.pipeline == 2)) {
        c.pipeline = 0;
        if (c.depth > 2) c.depth = 2;
    }
    return c;
}

// ---------------------------------------------------------------------------
// Small kernels: gradient, moments, equilibrium, transfers, reductions.
// ---------------------------------------------------------------------------
// src/darcy.py:104: grad = sum_i p_i * (-3 * scale * w_i * c_i), each term with
// one fused multiply-add (the same rounding in every kernel that forms it).
template <typename T>
__device__ __forceinline__ void gradient_sum(const T (&v)[9], T scale, T& gx, T& gy) {
    gx = T(0);
    gy = T(0);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const T k = T(-3) * scale * w9<T>(i);
        gx = fma(v[i], k * T(cx9(i)), gx);
        gy = fma(v[i], k * T(cy9(i)), gy);
    }
}

// Divergence moment of the populations of the cell at offset o
// (src/elasticity.py:1040-1058): c * m2 with c = -1.5 / (3 (lambda + mu) + 1).
template <typename T>
__device__ __forceinline__ T elast_div_at(const T* f, long long P, size_t o, const ElastMat<T>& mat, T lam, T mu,
                                          T div_scale) {
    T v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = f[o + i * P];
    const T m2 = v[0] + v[1] + v[2] + v[3] + T(2) * (v[4] + v[5] + v[6] + v[7]);
    T l = lam, m = mu;
    if (mat.mu_f) { l = mat.lam_f[o]; m = mat.mu_f[o]; }
    const T c = mat.mu_f ? T(-1.5) / (T(3) * (l + m) + T(1)) : div_scale;
    return c * m2;
}

template <typename T>
__global__ void gradient_kernel(SweepGeom G, const T* q, T scale, RulesView<T, 9> rules, const T* base, T* out) {
    grid_dep_wait();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= G.nx) return;
    T v[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const int xs = wrap(x - cx9(i), G.nx), ys = wrap(y - cy9(i), G.ny);
        v[i] = __ldg(q + (size_t)ys * G.pitch + xs);
    }
    const size_t o = (size_t)y * G.pitch + x;
    const int r = find_rule(rules, y, x);
    if (r >= 0) {
        const T qc = __ldg(q + o);   // every direction of the tiled input is q(x)
#pragma unroll
        for (int d = 0; d < 9; ++d) {
            const uint8_t code = __ldg(rules.code + (size_t)r * 9 + d);
            v[d] = rule_value<T, 9>(code, v[d], qc, rules.cst[(size_t)r * 9 + d]);
        }
    }
    T gx, gy;
    gradient_sum<T>(v, scale, gx, gy);
    if (base) {
        gx = base[o] + gx;
        gy = base[o + G.plane] + gy;
    }
    out[o] = gx;
    out[o + G.plane] = gy;
}

template <typename T>
__global__ void elast_moments_kernel(SweepGeom G, ElastMat<T> mat, T lam, T mu, const T* f, const T* force,
                                     const T* fext, T* eta, T* sigma, T* div, T div_scale) {
    grid_dep_wait();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= G.nx) return;
    const size_t o = (size_t)y * G.pitch + x;
    const long long P = G.plane;
    T v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = f[o + i * P];
    const T m0 = v[0] - v[2] + v[4] - v[5] - v[6] + v[7];
    const T m1 = v[1] - v[3] + v[4] + v[5] - v[6] - v[7];
    const T m2 = v[0] + v[1] + v[2] + v[3] + T(2) * (v[4] + v[5] + v[6] + v[7]);
    const T m3 = v[0] - v[1] + v[2] - v[3];
    const T m4 = v[4] - v[5] + v[6] - v[7];
    T l = lam, m = mu;
    if (mat.mu_f) { l = mat.lam_f[o]; m = mat.mu_f[o]; }
    if (eta) {
        T e0 = m0, e1 = m1;
        if (force) { e0 = e0 + T(0.5) * force[o]; e1 = e1 + T(0.5) * force[o + P]; }
        if (fext) { e0 = e0 + T(0.5) * fext[o]; e1 = e1 + T(0.5) * fext[o + P]; }
        eta[o] = e0;
        eta[o + P] = e1;
    }
    if (sigma) {
        const T cs = T(-1.5) * (l + m) / (T(3) * (l + m) + T(1));
        const T cd = T(-3) * m / (T(6) * m + T(1));
        const T ms = m2 * cs, md = m3 * cd;
        sigma[o] = ms + md;
        sigma[o + P] = (T(2) * cd) * m4;
        sigma[o + 2 * P] = ms - md;
    }
    if (div) div[o] = elast_div_at<T>(f, P, o, mat, lam, mu, div_scale);
}

// The Biot coupling force ext = base + G(div(f)) in one kernel: a 32 x 8 block
// forms the divergence of its cells and a one-cell halo (periodic wrap) in
// shared memory, then applies the Darcy gradient stencil with its boundary
// rules -- the arithmetic of elast_moments_kernel's divergence followed by
// gradient_kernel, without the divergence's round trip through memory or the
// second launch.
template <typename T>
__global__ void __launch_bounds__(256) elast_divgrad_kernel(SweepGeom G, ElastMat<T> mat, T lam, T mu, T div_scale,
                                                            const T* f, T scale, RulesView<T, 9> rules, const T* base,
                                                            T* out) {
    grid_dep_wait();
    constexpr int BX = 32, BY = 8;
    __shared__ T q[BY + 2][BX + 2];
    const int x0 = blockIdx.x * BX, y0 = blockIdx.y * BY;
    for (int k = threadIdx.y * BX + threadIdx.x; k < (BX + 2) * (BY + 2); k += BX * BY) {
        const int lx = k % (BX + 2), ly = k / (BX + 2);
        const int xs = ((x0 + lx - 1) % G.nx + G.nx) % G.nx, ys = ((y0 + ly - 1) % G.ny + G.ny) % G.ny;
        q[ly][lx] = elast_div_at<T>(f, G.plane, (size_t)ys * G.pitch + xs, mat, lam, mu, div_scale);
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= G.nx || y >= G.ny) return;
    T v[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) v[i] = q[threadIdx.y + 1 - cy9(i)][threadIdx.x + 1 - cx9(i)];
    const size_t o = (size_t)y * G.pitch + x;
    const int r = find_rule(rules, y, x);
    if (r >= 0) {
        const T qc = q[threadIdx.y + 1][threadIdx.x + 1];
#pragma unroll
        for (int d = 0; d < 9; ++d) {
            const uint8_t code = __ldg(rules.code + (size_t)r * 9 + d);
            v[d] = rule_value<T, 9>(code, v[d], qc, rules.cst[(size_t)r * 9 + d]);
        }
    }
    T gx, gy;
    gradient_sum<T>(v, scale, gx, gy);
    if (base) {
        gx = base[o] + gx;
        gy = base[o + G.plane] + gy;
    }
    out[o] = gx;
    out[o + G.plane] = gy;
}

// A damped smoothing sweep of the poroelastic multigrid in ONE kernel: the
// coupling force base + G(div f) of the sweep's own input (the stages of
// elast_divgrad_kernel: divergence of a 32 x 8 tile plus halo in shared
// memory, the gradient stencil with its rules) is handed to the
// collide-and-push sweep of the tile's cells as its external force, without
// the force's round trip through memory or a second launch.  The operations
// are those of xlbb_elast_divgrad followed by xlbb_elast_sweep on the
// collide-and-push launch, so the results are the same bit for bit.
template <typename T, bool RESID>
__global__ void __launch_bounds__(256) elast_divgrad_push_kernel(const typename ElastPhys<T, RESID>::Args p, T lam,
                                                                 T mu, T div_scale, T scale,
                                                                 RulesView<T, 9> grules, const T* base) {
    grid_dep_wait();
    constexpr int BX = 32, BY = 8;
    __shared__ T q[BY + 2][BX + 2];
    const SweepGeom& G = p.geom;
    const int x0 = blockIdx.x * BX, y0 = blockIdx.y * BY;
    for (int k = threadIdx.y * BX + threadIdx.x; k < (BX + 2) * (BY + 2); k += BX * BY) {
        const int lx = k % (BX + 2), ly = k / (BX + 2);
        const int xs = ((x0 + lx - 1) % G.nx + G.nx) % G.nx, ys = ((y0 + ly - 1) % G.ny + G.ny) % G.ny;
        q[ly][lx] = elast_div_at<T>(p.f_in, G.plane, (size_t)ys * G.pitch + xs, p.mat, lam, mu, div_scale);
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= G.nx || y >= G.ny) return;
    T v[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) v[i] = q[threadIdx.y + 1 - cy9(i)][threadIdx.x + 1 - cx9(i)];
    const size_t o = (size_t)y * G.pitch + x;
    const int r = find_rule(grules, y, x);
    if (r >= 0) {
        const T qc = q[threadIdx.y + 1][threadIdx.x + 1];
#pragma unroll
        for (int d = 0; d < 9; ++d) {
            const uint8_t code = __ldg(grules.code + (size_t)r * 9 + d);
            v[d] = rule_value<T, 9>(code, v[d], qc, grules.cst[(size_t)r * 9 + d]);
        }
    }
    T gx, gy;
    gradient_sum<T>(v, scale, gx, gy);
    if (base) {
        gx = base[o] + gx;
        gy = base[o + G.plane] + gy;
    }
    // as ElastPhys::load adds an external force to the static one
    const bool hasF = p.force != nullptr;
    push_cell<ElastPhys<T, RESID>, false>(p, y, x, [&](typename ElastPhys<T, RESID>::In& in) {
        in.F0 = hasF ? in.F0 + gx : gx;
        in.F1 = hasF ? in.F1 + gy : gy;
    });
}

template <typename T>
__global__ void elast_equilibrium_kernel(SweepGeom G, T lam, T mu, const T* lam_f, const T* mu_f, const T* eta,
                                         const T* sigma, const T* force, const T* fext, T* fo) {
    grid_dep_wait();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= G.nx) return;
    const size_t o = (size_t)y * G.pitch + x;
    const long long P = G.plane;
    T l = lam, m = mu;
    if (mu_f) { l = lam_f[o]; m = mu_f[o]; }
    T h, n, cs_, cd_;
    elast_rates<T>(l, m, cs_, cd_, h, n);
    T e0 = eta[o], e1 = eta[o + P];
    if (force) { e0 = e0 - T(0.5) * force[o]; e1 = e1 - T(0.5) * force[o + P]; }
    if (fext) { e0 = e0 - T(0.5) * fext[o]; e1 = e1 - T(0.5) * fext[o + P]; }
    const T cs = T(-1) - T(1) / (T(3) * (l + m));
    const T cd = T(-1) - T(1) / (T(6) * m);
    const T s0 = sigma[o], s1 = sigma[o + P], s2 = sigma[o + 2 * P];
    const T M0 = e0, M1 = e1, M2 = (s0 + s2) * cs, M3 = (s0 - s2) * cd, M4 = s1 * cd;
    const T M5 = e0 / T(3), M6 = e1 / T(3);
    fo[o] = T(0.5) * M0 + h * M2 + T(0.25) * M3 - T(0.5) * M5;
    fo[o + P] = T(0.5) * M1 + h * M2 - T(0.25) * M3 - T(0.5) * M6;
    fo[o + 2 * P] = T(-0.5) * M0 + h * M2 + T(0.25) * M3 + T(0.5) * M5;
    fo[o + 3 * P] = T(-0.5) * M1 + h * M2 - T(0.25) * M3 + T(0.5) * M6;
    fo[o + 4 * P] = n * M2 + T(0.25) * M4 + T(0.25) * M5 + T(0.25) * M6;
    fo[o + 5 * P] = n * M2 - T(0.25) * M4 - T(0.25) * M5 + T(0.25) * M6;
    fo[o + 6 * P] = n * M2 + T(0.25) * M4 - T(0.25) * M5 - T(0.25) * M6;
    fo[o + 7 * P] = n * M2 - T(0.25) * M4 + T(0.25) * M5 - T(0.25) * M6;
}

template <typename T>
__global__ void darcy_moments_kernel(SweepGeom G, const T* f, T omega, const T* omega_f, const T* src,
                                     const T* ext, T* rho, T* grad) {
    grid_dep_wait();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= G.nx) return;
    const size_t o = (size_t)y * G.pitch + x;
    const long long P = G.plane;
    T v[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) v[i] = f[o + i * P];
    if (rho) {
        T s = v[0];
#pragma unroll
        for (int i = 1; i < 9; ++i) s += v[i];
        if (src && ext) s = s + T(0.5) * (src[o] + ext[o]);
        else if (src) s = s + T(0.5) * src[o];
        else if (ext) s = s + T(0.5) * ext[o];
        rho[o] = s;
    }
    if (grad) {
        const T k = T(-3) * (omega_f ? omega_f[o] : omega);
        T gx = T(0), gy = T(0);
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            gx += v[i] * (k * T(cx9(i)));
            gy += v[i] * (k * T(cy9(i)));
        }
        grad[o] = gx;
        grad[o + P] = gy;
    }
}

// Tf: fine-level type, Tc: coarse-level type (a multigrid may run its coarsest
// level in FP64 under FP32 levels; the sum is formed in the wider type).
template <typename Tf, typename Tc>
__global__ void restrict_kernel(SweepGeom F, SweepGeom C, int q, int x0, int y0, int nix, int niy,
                                const Tf* __restrict__ res, Tc* __restrict__ rc) {
    grid_dep_wait();
    // one thread per coarse cell (all q planes); zero outside the coarse interior;
    // every plane's loads are issued before the first store (up to 9 planes at once)
    using Ts = typename std::conditional<(sizeof(Tf) > sizeof(Tc)), Tf, Tc>::type;
    const int X = blockIdx.x * blockDim.x + threadIdx.x;
    const int Y = blockIdx.y;
    if (X >= C.nx) return;
    const size_t oc = (size_t)Y * C.pitch + X;
    const int I = X - x0, J = Y - y0;
    const bool inside = I >= 0 && I < nix && J >= 0 && J < niy;
    const size_t of = inside ? (size_t)(y0 + 2 * J) * F.pitch + (x0 + 2 * I) : 0;
    for (int i0 = 0; i0 < q; i0 += 9) {
        Ts v[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            v[k] = Ts(0);
            if (inside && i0 + k < q) {
                const Tf* s = res + of + (size_t)(i0 + k) * F.plane;
                const Ts a = __ldg(s), b = __ldg(s + 1), c = __ldg(s + F.pitch), d = __ldg(s + F.pitch + 1);
                v[k] = a + c + b + d;
            }
        }
#pragma unroll
        for (int k = 0; k < 9; ++k)
            if (i0 + k < q) rc[oc + (size_t)(i0 + k) * C.plane] = Tc(v[k]);
    }
}

template <typename Tf, typename Tc>
__global__ void prolong_add_kernel(SweepGeom F, SweepGeom C, int q, int x0, int y0, int nfx, int nfy,
                                   const Tc* __restrict__ fc, Tf* __restrict__ ff) {
    grid_dep_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= nfx || j >= nfy) return;
    const size_t of = (size_t)(y0 + j) * F.pitch + (x0 + i);
    const size_t oc = (size_t)(y0 + j / 2) * C.pitch + (x0 + i / 2);
    for (int k0 = 0; k0 < q; k0 += 9) {      // loads of up to 9 planes before the stores
        Tf a[9];
        Tc c[9];
#pragma unroll
        for (int k = 0; k < 9; ++k)
            if (k0 + k < q) {
                a[k] = ff[of + (size_t)(k0 + k) * F.plane];
                c[k] = __ldg(fc + oc + (size_t)(k0 + k) * C.plane);
            }
#pragma unroll
        for (int k = 0; k < 9; ++k)
            if (k0 + k < q) ff[of + (size_t)(k0 + k) * F.plane] = Tf(a[k] + c[k]);
    }
}

template <typename T>
__global__ void sumsq_kernel(SweepGeom G, int nplanes, const T* d, int bx0, int bx1, int by0, int by1,
                             double* partials) {
    grid_dep_wait();
    __shared__ double red[8];
    double acc = 0.0;
    const long long n = (long long)(bx1 - bx0) * (by1 - by0);
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int y = by0 + (int)(e / (bx1 - bx0));
        const int x = bx0 + (int)(e % (bx1 - bx0));
        const size_t o = (size_t)y * G.pitch + x;
        for (int i = 0; i < nplanes; ++i) {
            const double v = (double)d[o + (size_t)i * G.plane];
            acc += v * v;
        }
    }
    const double s = block_sum(acc, red);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void reduce_sum_kernel(const double* p, int n, double* out) {
    grid_dep_wait();
    __shared__ double red[32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += p[i];
    const double s = block_sum(acc, red);
    if (threadIdx.x == 0) {
        *out = s;
        if (!isfinite(s)) note_status(XLBB_ENONFINITE);
    }
}

// Self-test of the bounded mbarrier wait: one thread waits on a barrier that
// nothing arrives at, with a limit of `polls`; the wait gives up, records
// XLBB_ETIMEOUT and the kernel returns (no copy is in flight, nothing hangs).
__global__ void wait_selftest_kernel(uint32_t polls, int* gave_up) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *gave_up = mbar_wait(&bar, 0, polls) ? 0 : 1;
    }
}

template <typename T>
__global__ void axpby_kernel(long long n, T a, const T* x, T b, const T* y, T* o) {
    grid_dep_wait();
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        o[i] = a * x[i] + b * y[i];
}

static SweepGeom geom(const XlbbGrid* g) { return SweepGeom{g->nx, g->ny, g->pitch, g->plane}; }

template <typename T, typename S = T>
static ElastMat<T, S> make_mat(const XlbbElastMaterial* m) {
    ElastMat<T, S> e;
    elast_rates<T>(T(m->lam), T(m->mu), e.cs, e.cd, e.h, e.n);
    e.lam_f = static_cast<const S*>(m->lam_field);
    e.mu_f = static_cast<const S*>(m->mu_field);
    return e;
}


// Kernel arguments of a D2Q9 sweep (Darcy or fluid policy; the fluid entry
// point rejects source planes before this is built).
template <class Ph>
static typename Ph::Args darcy_args(const XlbbGrid* g, const XlbbDarcySweep* s) {
    using T = typename Ph::T;
    using St = typename Ph::Storage;
    typename Ph::Args a;
    a.geom = geom(g);
    a.f_in = static_cast<const St*>(s->f_in);
    a.f_out = static_cast<St*>(s->f_out);
    a.omega = T(s->omega);
    a.omega_f = static_cast<const St*>(s->omega_field);
    a.source = static_cast<const St*>(s->source);
    a.ext = static_cast<const St*>(s->ext_source);
    a.resid = static_cast<const St*>(s->resid);
    a.pc = rules_view<T, 9>(s->pc);
    a.ps = rules_view<T, 9>(s->ps);
    a.sumsq = s->sumsq;
    return a;
}

// FP64 partials that a D2Q9 sweep with these arguments writes when it fuses
// its residual sum (the CTAs of the launch it takes).
template <typename T, typename St = T>
static constexpr int darcy_dtype() {
    return sizeof(T) == sizeof(St) ? (sizeof(T) == 4 ? XLBB_F32 : XLBB_F64) : XLBB_F32_ACC64;
}

template <typename T, typename St = T>
static long long darcy_partials_t(const XlbbGrid* g, const XlbbDarcySweep* s) {
    using Ph = DarcyPhys<T, St>;
    const typename Ph::Args a = darcy_args<Ph>(g, s);
    const XlbbSweepConfig c = effective_cfg(1, darcy_dtype<T, St>());
    return launch_ctas(g, resolve_shape(c, push_eligible<Ph>(a), sizeof(T) == 4));
}

// Whether a Darcy sweep takes the four-column kernel (launch pipeline 4):
// FP32 storage and arithmetic, no resid and no fused sum, post-streaming rules
// only with their push words, rows and planes of whole float4 (nx, pitch and
// plane multiples of 4; planes and push words 16-byte aligned).
static bool darcy4_ok(const XlbbGrid* g, const XlbbDarcySweep* s) {
    auto a16 = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
    const bool ps_rules = rules_view<float, 9>(s->ps).count > 0;
    return s->resid == nullptr && s->sumsq == nullptr && g->nx % 4 == 0 && g->pitch % 4 == 0 &&
           g->plane % 4 == 0 && a16(s->f_in) && a16(s->f_out) && a16(s->omega_field) && a16(s->source) &&
           a16(s->ext_source) && (!ps_rules || (s->ps.push != nullptr && a16(s->ps.push)));
}

template <typename T, typename St = T>
static int darcy_sweep_t(const XlbbGrid* g, const XlbbDarcySweep* s, cudaStream_t st) {
    if constexpr (sizeof(T) == 4 && sizeof(St) == 4) {
        if (g_cfg[1].pipeline == 4 && darcy4_ok(g, s)) {
            using Ph = DarcyPhys<float>;
            typename Ph::Args a = darcy_args<Ph>(g, s);
            Ph::fill_ptrs(a);
            launch_k(darcy_push4_kernel, dim3((g->nx + 127) / 128, (g->ny + DARCY4_ROWS - 1) / DARCY4_ROWS),
                     dim3(32, DARCY4_ROWS), 0, st, a);
            return check_launch("xlbb_darcy_sweep");
        }
    }
    const XlbbSweepConfig c = effective_cfg(1, darcy_dtype<T, St>());
    if (s->resid) {          // a separate instantiation: the plain sweep keeps its registers
        using Ph = DarcyPhys<T, St, true>;
        typename Ph::Args a = darcy_args<Ph>(g, s);
        if (s->sumsq) launch_sweep<Ph, true>(c, g, st, a);
        else launch_sweep<Ph, false>(c, g, st, a);
    } else {
        using Ph = DarcyPhys<T, St>;
        typename Ph::Args a = darcy_args<Ph>(g, s);
        if (s->sumsq) launch_sweep<Ph, true>(c, g, st, a);
        else launch_sweep<Ph, false>(c, g, st, a);
    }
    return check_launch("xlbb_darcy_sweep");
}

template <typename T, bool KBC>
static int fluid_sweep_t(const XlbbGrid* g, const XlbbDarcySweep* s, cudaStream_t st) {
    using Ph = FluidPhys<T, KBC>;
    typename Ph::Args a = darcy_args<Ph>(g, s);
    const XlbbSweepConfig c = effective_cfg(1, sizeof(T) == 4 ? XLBB_F32 : XLBB_F64);
    if (s->sumsq) launch_sweep<Ph, true>(c, g, st, a);
    else launch_sweep<Ph, false>(c, g, st, a);
    return check_launch("xlbb_fluid_sweep");
}

static bool grid3_ok(const XlbbGrid3* g) {
    return g && g->nx > 0 && g->ny > 0 && g->nz > 0 && g->pitch >= g->nx && g->ny <= 65535 && g->nz <= 65535 &&
           g->plane >= (long long)g->pitch * g->ny * g->nz && g->plane < (1LL << 31);
}

template <typename T, int Q, bool KBC = false>
static int fluid3_sweep_t(const XlbbGrid3* g, const XlbbDarcySweep* s, cudaStream_t st) {
    Fluid3Args<T, Q> a;
    a.nx = g->nx; a.ny = g->ny; a.nz = g->nz; a.pitch = g->pitch; a.plane = g->plane;
    a.f_in = static_cast<const T*>(s->f_in);
    a.f_out = static_cast<T*>(s->f_out);
    a.omega = T(s->omega);
    a.pc = rules_view<T, Q>(s->pc);
    a.ps = rules_view<T, Q>(s->ps);
    const dim3 grid((g->nx + FLUID3_THREADS - 1) / FLUID3_THREADS, g->ny, g->nz);
    if constexpr (KBC) {         // the collision-bound KBC sweep: bulk and rule cells as two launches
        launch_k(fluid3_bulk_kernel<T, Q, KBC>, grid, FLUID3_THREADS, 0, st, a);
        const long long nrules = (long long)a.pc.count + a.ps.count;
        if (nrules > 0)
            launch_k(fluid3_rules_kernel<T, Q, KBC>, dim3((unsigned)((nrules + FLUID3_THREADS - 1) / FLUID3_THREADS)),
                     FLUID3_THREADS, 0, st, a);
    } else if constexpr (FLUID3_LANE_RULES<T, Q, KBC>) {
        launch_k(fluid3_push19_kernel, grid, FLUID3_THREADS, 0, st, a);
    } else {
        launch_k(fluid3_push_kernel<T, Q, KBC>, grid, FLUID3_THREADS, 0, st, a);
    }
    return check_launch("xlbb_fluid3_sweep");
}

static inline dim3 row_grid(int nx, int ny, int bs) { return dim3((nx + bs - 1) / bs, ny); }

// ---------------------------------------------------------------------------
// Batched elasticity multigrid: many independent periodic instances of
// different sizes and materials in one launch per sweep.  CTAs loop over a
// work list of tiles (instance, owned columns, strip of rows); every tile is a
// sweep_strip of that instance's grid.
// ---------------------------------------------------------------------------
template <typename T, typename S = T>
struct BatchInst {
    const S* f_in;
    S* f_out;
    const S* force;
    const S* resid;
    SweepGeom geom;
    T cs, cd, h, n;
    int vec4;   // FP32 storage, nx / pitch / plane multiples of 4, 16-byte aligned planes
};

template <typename T, typename S = T>
static BatchInst<T, S> to_batch_inst(const XlbbBatchInstance& s) {
    BatchInst<T, S> b;
    b.f_in = static_cast<const S*>(s.f_in);
    b.f_out = static_cast<S*>(s.f_out);
    b.force = static_cast<const S*>(s.force);
    b.resid = static_cast<const S*>(s.resid);
    b.geom = SweepGeom{s.nx, s.ny, s.pitch, s.plane};
    elast_rates<T>(T(s.lam), T(s.mu), b.cs, b.cd, b.h, b.n);
    auto a16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    b.vec4 = sizeof(S) == 4 && s.nx % 4 == 0 && s.pitch % 4 == 0 && s.plane % 4 == 0 && a16(s.f_in) &&
             a16(s.f_out) && a16(s.force) && a16(s.resid);
    return b;
}

template <typename T, int TX, bool RESID, bool PREV, typename S = T>
__global__ void __launch_bounds__(TX + 32)
batched_elast_kernel(const BatchInst<T, S>* __restrict__ inst, const XlbbBatchTile* __restrict__ tiles, int ntiles,
                     T a, T b, int mix, int use_force, int sumsq_diff, double* tile_sumsq) {
    grid_dep_wait();
    using Ph = ElastPhys<T, RESID, S>;
    __shared__ T post[4][8][TX + 2];
    __shared__ double red[(TX + 32) / 32];
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        __syncthreads();   // the ring of the previous tile is no longer read
        const XlbbBatchTile tl = tiles[t];
        const BatchInst<T, S> I = inst[tl.inst];
        typename Ph::Args p;
        p.geom = I.geom;
        p.f_in = I.f_in;
        p.f_out = I.f_out;
        p.force = use_force ? I.force : nullptr;
        p.fext = nullptr;
        p.resid = I.resid;
        p.a = a;
        p.b = b;
        p.mat = ElastMat<T, S>{I.cs, I.cd, I.h, I.n, nullptr, nullptr};
        p.pc = RulesView<T, 8>{0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0, nullptr};
        p.ps = p.pc;
        p.sumsq = tile_sumsq;
        p.bx0 = 0; p.bx1 = I.geom.nx; p.by0 = 0; p.by1 = I.geom.ny;
        p.div_out = nullptr;
        p.div_scale = T(0);
        p.mix = mix;
        p.sumsq_diff = sumsq_diff;
        p.np = 0;
        Ph::fill_ptrs(p);
        const double acc = sweep_strip<Ph, TX, 1, PREV>(p, tl.x0, tl.ys, tl.ye, post);
        if (tile_sumsq != nullptr) {
            const double s = block_sum(acc, red);
            if (threadIdx.x < XLBB_BATCH_PARTS_PER_TILE)
                tile_sumsq[(size_t)t * XLBB_BATCH_PARTS_PER_TILE + threadIdx.x] = threadIdx.x == 0 ? s : 0.0;
        }
    }
}

// Volatile shared loads: a value read this way is not kept in a register
// beyond its use (the compiler can neither merge nor hoist the reads).
__device__ __forceinline__ unsigned long long lds64(const void* p) {
    unsigned long long v;
    asm volatile("ld.shared.u64 %0, [%1];" : "=l"(v) : "r"(smem_u32(p)));
    return v;
}
__device__ __forceinline__ unsigned lds32(const void* p) {
    unsigned v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)));
    return v;
}
template <typename T>
__device__ __forceinline__ T ldsT(const T* p) {
    if constexpr (sizeof(T) == 4) return __uint_as_float(lds32(p));
    else return __longlong_as_double((long long)lds64(p));
}
template <typename P_>
__device__ __forceinline__ P_* ldsP(P_* const* p) { return reinterpret_cast<P_*>(lds64(p)); }

// A warp's copy of its current tile and that tile's instance record, in
// shared memory: lane 0 fetches it once per tile, every lane reads the fields
// it needs with volatile shared loads right where it uses them.
template <typename T, typename S>
struct __align__(16) TileRec {
    const S* fi;
    S* fo;
    const S* fc;
    const S* rs;
    unsigned P;      // plane stride (the upload checks 8 planes fit in 32-bit offsets)
    int pitch, nx, ny;
    int x0, ys, ye, pad;
    T cs, cd, h, n;
};

// Lane 0 copies tile t's record into `d`; with `vec4`, an instance that does
// not qualify for the four-column kernel gets an empty row range and sets the
// status word.
template <typename T, typename S>
__device__ __forceinline__ void fill_tile_rec(TileRec<T, S>* d, const BatchInst<T, S>* __restrict__ inst,
                                              const XlbbBatchTile* __restrict__ tiles, int t, int use_force,
                                              bool resid, bool vec4) {
    const XlbbBatchTile tl = tiles[t];
    const BatchInst<T, S>& I = inst[tl.inst];
    const bool ok = !vec4 || (I.vec4 && (tl.x0 & 3) == 0);
    d->fi = I.f_in;
    d->fo = I.f_out;
    d->fc = use_force ? I.force : nullptr;
    d->rs = resid ? I.resid : nullptr;
    d->P = (unsigned)I.geom.plane;
    d->pitch = I.geom.pitch;
    d->nx = I.geom.nx;
    d->ny = I.geom.ny;
    d->x0 = tl.x0;
    d->ys = tl.ys;
    d->ye = ok ? tl.ye : tl.ys;
    d->cs = I.cs;
    d->cd = I.cd;
    d->h = I.h;
    d->n = I.n;
    if (!ok) note_status(XLBB_EBADARG);
}

__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Prefetch into L2 a warp's cells of the next tile's row (`n` cells per lane
// starting at column x): no registers stay held, the next row's loads are then
// served from L2.
template <typename T, typename S, bool RESID>
__device__ __forceinline__ void prefetch_tile_row(const TileRec<T, S>* rn, int w, int x, int zero_in) {
    const int yn = (int)lds32(&rn->ys) + w, xn = (int)lds32(&rn->x0) + x;
    if (yn >= (int)lds32(&rn->ye) || xn >= (int)lds32(&rn->nx)) return;
    const unsigned Pn = lds32(&rn->P), on = unsigned(yn * (int)lds32(&rn->pitch) + xn);
    const S* fin = ldsP(&rn->fi);
    if (!zero_in) {
#pragma unroll
        for (unsigned i = 0; i < 8; ++i) prefetch_l2(fin + (on + i * Pn));
    }
    const S* fcn = ldsP(&rn->fc);
    if (fcn) { prefetch_l2(fcn + on); prefetch_l2(fcn + (on + Pn)); }
    if constexpr (RESID) {
        const S* rsn = ldsP(&rn->rs);
#pragma unroll
        for (unsigned i = 0; i < 8; ++i) prefetch_l2(rsn + (on + i * Pn));
    }
}

// One cell of the batched collide-and-push sweep (periodic, no boundary rules):
// the arithmetic of ElastPhys's load / collide / put; plane i of the cell at
// offset o is fi + (i * P + o).  Split in its loads and the rest, so that the
// caller can overlap work with the loads' latency.
template <typename T>
struct BatchedCell {
    T g[8];
    T F0, F1;
    bool hasF;
};

// zero_in: the populations are taken as zero (not read) -- the first sweep of a
// coarse level, whose correction starts from zero; the same values as a
// zero-filled input, bit for bit.
template <typename T, bool RESID, typename S>
__device__ __forceinline__ void batched_cell_load(const TileRec<T, S>* r, int y, int x, BatchedCell<T>& c,
                                                  int zero_in) {
    const S* fi = ldsP(&r->fi);
    const unsigned P = lds32(&r->P);
    const unsigned o = unsigned(y * (int)lds32(&r->pitch) + x);
#pragma unroll
    for (unsigned i = 0; i < 8; ++i) c.g[i] = zero_in ? T(0) : T(__ldg(fi + (o + i * P)));
    if constexpr (RESID) {
        const S* rs = ldsP(&r->rs);
#pragma unroll
        for (unsigned i = 0; i < 8; ++i) c.g[i] = c.g[i] - T(__ldg(rs + (o + i * P)));
    }
    const S* fc = ldsP(&r->fc);
    c.hasF = fc != nullptr;
    c.F0 = T(0);
    c.F1 = T(0);
    if (fc) { c.F0 = T(__ldg(fc + o)); c.F1 = T(__ldg(fc + (o + P))); }
}

template <typename T, bool SUMSQ, typename S>
__device__ __forceinline__ double batched_cell_push(const TileRec<T, S>* r, const BatchedCell<T>& c, T a, T b, int mix,
                                                    int sumsq_diff, int y, int x, int zero_in) {
    T fs[8];
    elast_collide<T>(c.g, c.hasF, c.F0, c.F1, ldsT(&r->cs), ldsT(&r->cd), ldsT(&r->h), ldsT(&r->n), fs);
    const int pitch = (int)lds32(&r->pitch), nx = (int)lds32(&r->nx), ny = (int)lds32(&r->ny);
    const unsigned P = lds32(&r->P);
    const S* fi = ldsP(&r->fi);
    S* fo = ldsP(&r->fo);
    const int rm = (y == 0 ? ny - 1 : y - 1) * pitch, r0 = y * pitch, rp = (y == ny - 1 ? 0 : y + 1) * pitch;
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int zx = cx8(i) > 0 ? xp : (cx8(i) < 0 ? xm : x);
        const unsigned oz = unsigned((cy8(i) > 0 ? rp : (cy8(i) < 0 ? rm : r0)) + zx) + i * P;
        T v = fs[i];
        T fz = T(0);
        if ((mix || (SUMSQ && sumsq_diff)) && !zero_in) fz = T(__ldg(fi + oz));
        if (mix) v = mix_ab(a, fz, b, fs[i]);
        const S sv = S(v);
        fo[oz] = sv;
        if constexpr (SUMSQ) {
            double d = (double)sv;
            if (sumsq_diff) d -= (double)S(fz);
            acc += d * d;
        }
    }
    return acc;
}

// Collide-and-push form of the batched sweep: a block of 128 x 8 threads takes
// a tile, thread (tx, ty) its column x0 + tx and every 8th row from ys + ty
// (independent cells: no block barrier); with SUMSQ one FP64 partial per tile.
// Each warp keeps its tile record, and the next one, in shared memory: while
// the first row's loads are in flight lane 0 fetches the next tile's record
// and the warp prefetches its cells of the next tile into L2.  Measured on
// B200 (512 instances, 26 M cells, level-0 smoothing sweep): the record in
// shared memory beat every thread loading it into registers by 15%; CTAs held
// to 32 or 40 registers for more CTAs per SM, two rows per thread loaded
// before either is collided, and taller tiles were all slower.  The explicit
// minimum of one CTA per SM lets the compiler keep up to 64 registers per
// thread (more loads in flight per thread), which measured faster than its
// 32-register choice.
template <typename T, bool RESID, bool SUMSQ, typename S = T>
__global__ void __launch_bounds__(1024, 1)
batched_push_kernel(const BatchInst<T, S>* __restrict__ inst, const XlbbBatchTile* __restrict__ tiles, int ntiles,
                    T a, T b, int mix, int use_force, int sumsq_diff, double* tile_sumsq, int zero_in) {
    grid_dep_wait();
    __shared__ TileRec<T, S> rec[2][32];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, wid = tid >> 5;
    if (blockIdx.x >= ntiles) return;          // uniform over the block
    if ((tid & 31) == 0) fill_tile_rec(&rec[0][wid], inst, tiles, blockIdx.x, use_force, RESID, false);
    __syncwarp();
    // FP32 arithmetic overlaps the next tile's record and prefetch with the
    // loads; the FP64-arithmetic variants, at their 64-register limit, fetch
    // each record when they reach the tile (the overlap measured slower: spills)
    constexpr bool OVERLAP = sizeof(T) == 4;
    int k = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
        TileRec<T, S>* r = &rec[OVERLAP ? (k & 1) : 0][wid];
        TileRec<T, S>* rn = &rec[OVERLAP ? ((k + 1) & 1) : 0][wid];
        const int tn = t + gridDim.x;
        if constexpr (!OVERLAP) {
            if (k > 0) {
                if ((tid & 31) == 0) fill_tile_rec(r, inst, tiles, t, use_force, RESID, false);
                __syncwarp();
            }
        }
        bool pending = OVERLAP;                // the next record is still to be fetched
        const int x = (int)lds32(&r->x0) + threadIdx.x;
        const bool active = x < (int)lds32(&r->nx);
        double acc = 0.0;
        // warp-uniform loop (a warp spans one threadIdx.y); inactive lanes only join the next-tile work
        for (int y = (int)lds32(&r->ys) + threadIdx.y; y < (int)lds32(&r->ye); y += blockDim.y) {
            BatchedCell<T> c;
            if (active) batched_cell_load<T, RESID, S>(r, y, x, c, zero_in);
            if (pending) {
                pending = false;
                if (tn < ntiles && (tid & 31) == 0) fill_tile_rec(rn, inst, tiles, tn, use_force, RESID, false);
                __syncwarp();
                if (tn < ntiles) prefetch_tile_row<T, S, RESID>(rn, threadIdx.y, threadIdx.x, zero_in);
            }
            if (active) acc += batched_cell_push<T, SUMSQ, S>(r, c, a, b, mix, sumsq_diff, y, x, zero_in);
        }
        if (pending) {                          // a warp without a row in this tile
            if (tn < ntiles && (tid & 31) == 0) fill_tile_rec(rn, inst, tiles, tn, use_force, RESID, false);
            __syncwarp();
        }
        if constexpr (SUMSQ) {   // a partial per warp (no block barrier); every output is written once
            const double s = warp_sum(acc);
            if ((tid & 31) == 0) tile_sumsq[(size_t)t * XLBB_BATCH_PARTS_PER_TILE + wid] = s;
        }
        __syncwarp();                           // every lane is done with r before it is refilled
    }
}

// ---------------------------------------------------------------------------
// Four-column form of the batched sweep (FP32 storage): a warp takes one row
// of a 128-column tile, lane c the columns x0 + 4c .. x0 + 4c + 3, with float4
// loads and stores of every plane.  Streaming along x moves the values that
// cross a 4-column chunk between lanes by shuffles, so each destination chunk
// is written with one aligned float4 store; the mixing reads of the row's own
// directions (c_y = 0) are the lane's own inputs.  Where an instance spans
// several tiles, the one value of a direction that crosses a tile edge is
// written by its pusher with a scalar store, and the receiving lane writes the
// other three values of its chunk: every output is written exactly once, with
// the arithmetic of the scalar sweep.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

template <typename T>
__device__ __forceinline__ T mixv(int mix, T a, T fz, T b, T s) { return mix ? mix_ab(a, fz, b, s) : s; }

// `mid` runs once the row's loads are issued (work that overlaps their latency).
template <typename T, bool RESID, bool SUMSQ, class Mid>
__device__ __forceinline__ double batched_push_row4(const TileRec<T, float>* r, T a, T b, int mix, int sumsq_diff,
                                                    int y, int x, int lane, bool active, int nlan, bool single,
                                                    int zero_in, Mid&& mid) {
    const unsigned P = lds32(&r->P);
    const int pitch = (int)lds32(&r->pitch);
    const unsigned o = unsigned(y * pitch + x);
    const int ny = (int)lds32(&r->ny);
    const int yu = y == ny - 1 ? 0 : y + 1, yl = y == 0 ? ny - 1 : y - 1;
    const bool need_fz = mix || (SUMSQ && sumsq_diff);
    T ps[8][4];
    T f0[4], f2[4];   // the inputs of the directions that stay in the row (mixing)
    // the mixing inputs of the destination chunks in the rows above and below,
    // loaded with the row's own inputs (all loads of the row in flight at once)
    float4 fzv[8];
    {
        const float* fi = ldsP(&r->fi);
        float4 v[8];
#pragma unroll
        for (unsigned i = 0; i < 8; ++i)
            v[i] = active && !zero_in ? ldg4(fi + (o + i * P)) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            fzv[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (cy8(i) != 0 && need_fz && active && !zero_in)
                fzv[i] = ldg4(fi + (unsigned((cy8(i) > 0 ? yu : yl) * pitch + x) + unsigned(i) * P));
        }
        f0[0] = T(v[0].x); f0[1] = T(v[0].y); f0[2] = T(v[0].z); f0[3] = T(v[0].w);
        f2[0] = T(v[2].x); f2[1] = T(v[2].y); f2[2] = T(v[2].z); f2[3] = T(v[2].w);
        T g[4][8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            g[0][i] = T(v[i].x); g[1][i] = T(v[i].y); g[2][i] = T(v[i].z); g[3][i] = T(v[i].w);
        }
        if constexpr (RESID) {
            const float* rs = ldsP(&r->rs);
#pragma unroll
            for (unsigned i = 0; i < 8; ++i) {
                const float4 q = active ? ldg4(rs + (o + i * P)) : make_float4(0.f, 0.f, 0.f, 0.f);
                g[0][i] = g[0][i] - T(q.x); g[1][i] = g[1][i] - T(q.y);
                g[2][i] = g[2][i] - T(q.z); g[3][i] = g[3][i] - T(q.w);
            }
        }
        const float* fc = ldsP(&r->fc);
        float4 F0 = make_float4(0.f, 0.f, 0.f, 0.f), F1 = F0;
        if (fc && active) { F0 = ldg4(fc + o); F1 = ldg4(fc + (o + P)); }
        mid();
        const T F0j[4] = {T(F0.x), T(F0.y), T(F0.z), T(F0.w)}, F1j[4] = {T(F1.x), T(F1.y), T(F1.z), T(F1.w)};
        const T cs = ldsT(&r->cs), cd = ldsT(&r->cd), h = ldsT(&r->h), n = ldsT(&r->n);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            T fs[8];
            elast_collide<T>(g[j], fc != nullptr, F0j[j], F1j[j], cs, cd, h, n, fs);
#pragma unroll
            for (int i = 0; i < 8; ++i) ps[i][j] = fs[i];
        }
    }
    const int nx = (int)lds32(&r->nx);
    const float* fi = ldsP(&r->fi);
    float* fo = ldsP(&r->fo);
    const int src_l = lane == 0 ? nlan - 1 : lane - 1;          // chunk to the left (wrap inside one tile)
    const int src_r = lane >= nlan - 1 ? 0 : lane + 1;          // chunk to the right
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int cxi = cx8(i), cyi = cy8(i);
        const int yd = cyi > 0 ? yu : (cyi < 0 ? yl : y);
        T e[4];
        bool has0 = true, has3 = true;
        if (cxi > 0) {
            const T left = __shfl_sync(0xffffffffu, ps[i][3], src_l);
            e[0] = left; e[1] = ps[i][0]; e[2] = ps[i][1]; e[3] = ps[i][2];
            has0 = lane > 0 || single;
        } else if (cxi < 0) {
            const T right = __shfl_sync(0xffffffffu, ps[i][0], src_r);
            e[0] = ps[i][1]; e[1] = ps[i][2]; e[2] = ps[i][3]; e[3] = right;
            has3 = lane < nlan - 1 || single;
        } else {
            e[0] = ps[i][0]; e[1] = ps[i][1]; e[2] = ps[i][2]; e[3] = ps[i][3];
        }
        if (!active) continue;
        const unsigned od = unsigned(yd * pitch + x) + unsigned(i) * P;
        T fz[4] = {T(0), T(0), T(0), T(0)};
        if (need_fz) {
            if (cyi == 0) {
#pragma unroll
                for (int j = 0; j < 4; ++j) fz[j] = i == 0 ? f0[j] : f2[j];
            } else {
                fz[0] = T(fzv[i].x); fz[1] = T(fzv[i].y); fz[2] = T(fzv[i].z); fz[3] = T(fzv[i].w);
            }
        }
        float out[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) out[j] = float(mixv<T>(mix, a, fz[j], b, e[j]));
        if (has0 && has3) {
            *reinterpret_cast<float4*>(fo + od) = make_float4(out[0], out[1], out[2], out[3]);
        } else if (!has0) {   // element 0 comes from the tile to the left
            fo[od + 1] = out[1];
            *reinterpret_cast<float2*>(fo + od + 2) = make_float2(out[2], out[3]);
        } else {              // element 3 comes from the tile to the right
            *reinterpret_cast<float2*>(fo + od) = make_float2(out[0], out[1]);
            fo[od + 2] = out[2];
        }
        if constexpr (SUMSQ) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if ((j == 0 && !has0) || (j == 3 && !has3)) continue;
                double d = (double)out[j];
                if (sumsq_diff) d -= (double)float(fz[j]);
                acc += d * d;
            }
        }
        // the value that leaves the tile: one scalar store by its pusher
        if (!single && ((cxi > 0 && lane == nlan - 1) || (cxi < 0 && lane == 0))) {
            const int xd = cxi > 0 ? (x + 4 == nx ? 0 : x + 4) : (x == 0 ? nx - 1 : x - 1);
            const unsigned oz = unsigned(yd * pitch + xd) + unsigned(i) * P;
            const T sv = cxi > 0 ? ps[i][3] : ps[i][0];
            T fzs = T(0);
            if (need_fz && !zero_in) fzs = T(__ldg(fi + oz));
            const float w = float(mixv<T>(mix, a, fzs, b, sv));
            fo[oz] = w;
            if constexpr (SUMSQ) {
                double d = (double)w;
                if (sumsq_diff) d -= (double)float(fzs);
                acc += d * d;
            }
        }
    }
    return acc;
}


// 16 warps (one per row of a 16-row tile), up to 128 registers: the row's 16
// float4 loads stay in flight together.  While they are in flight, lane 0
// copies the warp's next tile record into the second slot and every lane asks
// L2 for its columns of the next tile's row (prefetch: no registers held), so
// the next row's loads are served from L2.  Measured on B200 against 8-warp
// CTAs held to 80 registers (three per SM) and CTAs held to 64: both slower
// (spills, or the mixing loads issued late).
template <typename T, bool RESID, bool SUMSQ>
__global__ void __launch_bounds__(512, 1)
batched_push4_kernel(const BatchInst<T, float>* __restrict__ inst, const XlbbBatchTile* __restrict__ tiles, int ntiles,
                     T a, T b, int mix, int use_force, int sumsq_diff, double* tile_sumsq, int zero_in) {
    grid_dep_wait();
    __shared__ TileRec<T, float> rec[2][16];
    const int lane = threadIdx.x, w = threadIdx.y;   // blockDim = (32, 16): a warp per tile row
    if (blockIdx.x >= ntiles) return;                 // uniform over the block
    if (lane == 0) fill_tile_rec(&rec[0][w], inst, tiles, blockIdx.x, use_force, RESID, true);
    __syncwarp();
    int k = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
        TileRec<T, float>* r = &rec[k & 1][w];
        TileRec<T, float>* rn = &rec[(k + 1) & 1][w];
        const int tn = t + gridDim.x;
        bool pending = true;                          // the next record is still to be fetched
        auto next = [&]() {
            if (!pending) return;
            pending = false;
            if (tn < ntiles && lane == 0) fill_tile_rec(rn, inst, tiles, tn, use_force, RESID, true);
            __syncwarp();
            if (tn < ntiles) {
                const int yn = (int)lds32(&rn->ys) + w, xn = (int)lds32(&rn->x0) + 4 * lane;
                if (yn < (int)lds32(&rn->ye) && xn < (int)lds32(&rn->nx)) {
                    const unsigned Pn = lds32(&rn->P), on = unsigned(yn * (int)lds32(&rn->pitch) + xn);
                    const float* fin = ldsP(&rn->fi);
                    if (!zero_in) {
#pragma unroll
                        for (unsigned i = 0; i < 8; ++i) prefetch_l2(fin + (on + i * Pn));
                    }
                    const float* fcn = ldsP(&rn->fc);
                    if (fcn) { prefetch_l2(fcn + on); prefetch_l2(fcn + (on + Pn)); }
                    if constexpr (RESID) {
                        const float* rsn = ldsP(&rn->rs);
#pragma unroll
                        for (unsigned i = 0; i < 8; ++i) prefetch_l2(rsn + (on + i * Pn));
                    }
                }
            }
        };
        const int x0 = (int)lds32(&r->x0), nx = (int)lds32(&r->nx);
        const int x = x0 + 4 * lane;
        const int nlan = min(32, (nx - x0) >> 2);
        const bool single = nx <= 128;           // the whole row is this warp's
        double acc = 0.0;
        for (int y = (int)lds32(&r->ys) + w; y < (int)lds32(&r->ye); y += blockDim.y)
            acc += batched_push_row4<T, RESID, SUMSQ>(r, a, b, mix, sumsq_diff, y, x, lane, lane < nlan, nlan, single,
                                                      zero_in, next);
        next();                                  // a warp without a row in this tile
        if constexpr (SUMSQ) {                   // a partial per warp (no block barrier)
            const double s = warp_sum(acc);
            if (lane == 0) {
                tile_sumsq[(size_t)t * XLBB_BATCH_PARTS_PER_TILE + w] = s;
                tile_sumsq[(size_t)t * XLBB_BATCH_PARTS_PER_TILE + 16 + w] = 0.0;
            }
        }
        __syncwarp();                            // every lane is done with r before it is refilled
    }
}

// The four-column sweep on one grid (pipeline 4): the batched form's row
// code on a tile per CTA (128 columns x 16 rows; the CTA's record, from the
// kernel parameters, in shared memory).  For periodic FP32 sweeps without
// boundary rules, per-cell material, side outputs or fused sums; bit-identical
// to the collide-and-push kernel.
template <bool RESID>
__global__ void __launch_bounds__(512, 1) grid_push4_kernel(const TileRec<float, float> rin, float a, float b, int mix) {
    grid_dep_wait();
    __shared__ TileRec<float, float> rec;
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        rec = rin;
        rec.x0 = blockIdx.x * 128;
        rec.ys = blockIdx.y * 16;
        rec.ye = min(rec.ys + 16, rin.ny);
    }
    __syncthreads();
    const int lane = threadIdx.x;
    const int x0 = blockIdx.x * 128, nx = rin.nx;
    const int x = x0 + 4 * lane;
    const int nlan = min(32, (nx - x0) >> 2);
    const int y = blockIdx.y * 16 + threadIdx.y;
    if (y < rin.ny)
        batched_push_row4<float, RESID, false>(&rec, a, b, mix, 0, y, x, lane, lane < nlan, nlan, nx <= 128, 0, [] {});
}

// Whether an FP32 sweep can take the four-column kernel: periodic (no rules),
// uniform material, no side output or fused sum, at most one force array,
// 16-byte aligned rows and planes, 8 planes within 32-bit offsets, and a grid
// of at least 64 K cells (smaller grids want one thread per cell).
template <class Args>
static bool grid_push4_ok(const XlbbGrid* g, const Args& a) {
    auto a16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    return a.pc.count == 0 && a.ps.count == 0 && a.mat.mu_f == nullptr && a.div_out == nullptr &&
           a.sumsq == nullptr && !(a.force && a.fext) && g->nx % 4 == 0 && g->pitch % 4 == 0 && g->plane % 4 == 0 &&
           g->plane < (1LL << 28) && (long long)g->nx * g->ny >= 65536 && a16(a.f_in) && a16(a.f_out) &&
           a16(a.force) && a16(a.fext) && a16(a.resid);
}

template <typename T, bool RESID, typename S = T>
static typename ElastPhys<T, RESID, S>::Args elast_args(const XlbbGrid* g, const XlbbElastMaterial* mat,
                                                        const XlbbElastSweep* s) {
    typename ElastPhys<T, RESID, S>::Args a;
    a.geom = geom(g);
    a.f_in = static_cast<const S*>(s->f_in);
    a.f_out = static_cast<S*>(s->f_out);
    a.force = s->use_force ? static_cast<const S*>(s->force) : nullptr;
    a.fext = static_cast<const S*>(s->fext);
    a.resid = static_cast<const S*>(s->resid);
    a.a = T(s->a);
    a.b = T(s->b);
    a.mix = (s->a == 0.0 && s->b == 1.0) ? 0 : 1;
    a.sumsq_diff = (s->sumsq != nullptr && s->sumsq_diff) ? 1 : 0;
    a.mat = make_mat<T, S>(mat);
    a.pc = rules_view<T, 8>(s->pc);
    a.ps = rules_view<T, 8>(s->ps);
    a.sumsq = s->sumsq;
    a.bx0 = s->bx0; a.bx1 = s->bx1; a.by0 = s->by0; a.by1 = s->by1;
    a.div_out = static_cast<S*>(s->div_out);
    a.div_scale = T(-1.5 / (3.0 * (mat->lam + mat->mu) + 1.0));
    return a;
}

template <typename T, bool RESID, bool PREV, typename S = T>
static int launch_elast(const XlbbGrid* g, const XlbbElastMaterial* mat, const XlbbElastSweep* s, cudaStream_t st) {
    using Ph = ElastPhys<T, RESID, S>;
    typename Ph::Args a = elast_args<T, RESID, S>(g, mat, s);
    if constexpr (sizeof(T) != sizeof(S)) {
        const XlbbSweepConfig c = resolve_shape(effective_cfg(0, XLBB_F32_ACC64), push_eligible<Ph>(a), false);
        if (c.pipeline == 3) {
            Ph::fill_ptrs(a);
            launch_push<Ph>(c, g, st, a);
        } else {
            launch_sweep_regs<Ph, PREV>(c, g, st, a);
        }
    } else {
        const XlbbSweepConfig c = effective_cfg(0, sizeof(T) == 4 ? XLBB_F32 : XLBB_F64);
        if constexpr (sizeof(T) == 4) {
            if (g_cfg[0].pipeline == 4 && grid_push4_ok(g, a)) {
                TileRec<float, float> r{};
                r.fi = a.f_in;
                r.fo = a.f_out;
                r.fc = a.force ? a.force : a.fext;
                r.rs = RESID ? a.resid : nullptr;
                r.P = (unsigned)g->plane;
                r.pitch = g->pitch;
                r.nx = g->nx;
                r.ny = g->ny;
                r.cs = a.mat.cs;
                r.cd = a.mat.cd;
                r.h = a.mat.h;
                r.n = a.mat.n;
                const dim3 grid((g->nx + 127) / 128, (g->ny + 15) / 16), blk(32, 16);
                launch_k(grid_push4_kernel<RESID>, grid, blk, 0, st, r, a.a, a.b, a.mix);
                return check_launch("xlbb_elast_sweep");
            }
        }
        launch_sweep<Ph, PREV>(c, g, st, a);
    }
    return check_launch("xlbb_elast_sweep");
}

template <typename T, typename S = T>
static int elast_sweep_t(const XlbbGrid* g, const XlbbElastMaterial* mat, const XlbbElastSweep* s, cudaStream_t st) {
    // the previous populations are kept when mixed or differenced
    const bool mix = !(s->a == 0.0 && s->b == 1.0) || (s->sumsq != nullptr && s->sumsq_diff);
    if (s->resid)
        return mix ? launch_elast<T, true, true, S>(g, mat, s, st) : launch_elast<T, true, false, S>(g, mat, s, st);
    return mix ? launch_elast<T, false, true, S>(g, mat, s, st) : launch_elast<T, false, false, S>(g, mat, s, st);
}

// FP64 partials that an elasticity sweep with these arguments writes with a
// fused sum (the four-column kernel never takes a fused sum).
template <typename T, typename S>
static long long elast_partials_t(const XlbbGrid* g, const XlbbElastMaterial* mat, const XlbbElastSweep* s,
                                  int dtype) {
    using Ph = ElastPhys<T, false, S>;
    const typename Ph::Args a = elast_args<T, false, S>(g, mat, s);
    const XlbbSweepConfig c = effective_cfg(0, dtype);
    return launch_ctas(g, resolve_shape(c, push_eligible<Ph>(a), sizeof(T) == 4));
}

// Restriction (2x2 block sums) and prolongation (injection, added) of every
// instance of a periodic batch; blockIdx.y = instance.
template <typename Tf, typename Tc>
__global__ void batched_restrict_kernel(const XlbbBatchTransfer* __restrict__ tr) {
    grid_dep_wait();
    const XlbbBatchTransfer T_ = tr[blockIdx.y];
    const Tf* __restrict__ res = static_cast<const Tf*>(T_.fine);
    Tc* __restrict__ rc = static_cast<Tc*>(T_.coarse);
    using Ts = typename std::conditional<(sizeof(Tf) > sizeof(Tc)), Tf, Tc>::type;
    const int ncx = T_.nx_f / 2, ncy = T_.ny_f / 2;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ncx * ncy; e += gridDim.x * blockDim.x) {
        const int X = e % ncx, Y = e / ncx;
        const size_t of = (size_t)(2 * Y) * T_.pitch_f + 2 * X, oc = (size_t)Y * T_.pitch_c + X;
        Ts v[8];      // every plane's loads before the first store
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const Tf* s = res + of + (size_t)i * T_.plane_f;
            v[i] = Ts(__ldg(s)) + Ts(__ldg(s + T_.pitch_f)) + Ts(__ldg(s + 1)) + Ts(__ldg(s + T_.pitch_f + 1));
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) rc[oc + (size_t)i * T_.plane_c] = Tc(v[i]);
    }
}

// With ``parts`` != NULL every block also writes its FP64 sums of the
// correction^2 and of the corrected populations^2 to parts[2 * block + {0, 1}]
// (block = blockIdx.y * gridDim.x + blockIdx.x).
template <typename Tf, typename Tc>
__global__ void batched_prolong_add_kernel(const XlbbBatchTransfer* __restrict__ tr, double* parts) {
    grid_dep_wait();
    __shared__ double red[8];
    const XlbbBatchTransfer T_ = tr[blockIdx.y];
    Tf* __restrict__ ff = static_cast<Tf*>(const_cast<void*>(T_.fine));
    const Tc* __restrict__ fc = static_cast<const Tc*>(T_.coarse);
    double cc = 0.0, nn = 0.0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < T_.nx_f * T_.ny_f; e += gridDim.x * blockDim.x) {
        const int x = e % T_.nx_f, y = e / T_.nx_f;
        const size_t of = (size_t)y * T_.pitch_f + x, oc = (size_t)(y / 2) * T_.pitch_c + x / 2;
        Tf a[8];      // every plane's loads before the first store
        Tc c[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            a[i] = ff[of + (size_t)i * T_.plane_f];
            c[i] = __ldg(fc + oc + (size_t)i * T_.plane_c);
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const Tf v = Tf(a[i] + c[i]);
            ff[of + (size_t)i * T_.plane_f] = v;
            cc += (double)c[i] * (double)c[i];
            nn += (double)v * (double)v;
        }
    }
    if (parts != nullptr) {
        const double a = block_sum(cc, red);
        const double b = block_sum(nn, red);
        if (threadIdx.x == 0) {
            const size_t blk = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
            parts[2 * blk] = a;
            parts[2 * blk + 1] = b;
        }
    }
}

// norms[2 i + k] = sum over the XLBB_PROLONG_BLOCKS blocks of instance i of
// parts[2 block + k]; one warp per instance, fixed order.
// Prolongation with a balanced block map: block b adds the coarse correction
// to elements [e0, e0 + 1024) of instance map[b].x (e0 = map[b].y; a thread
// takes 4 elements 256 apart), so that every block does the same work whatever
// the instance sizes.  With parts != NULL the block writes its FP64 sums of the
// correction^2 and of the corrected populations^2 to parts[b], parts[nb + b].
template <typename Tf, typename Tc>
__global__ void __launch_bounds__(256) batched_prolong_map_kernel(const XlbbBatchTransfer* __restrict__ tr,
                                                                  const int2* __restrict__ map, int nb,
                                                                  double* parts) {
    grid_dep_wait();
    __shared__ double red[8];
    const int2 m = map[blockIdx.x];
    const XlbbBatchTransfer T_ = tr[m.x];
    Tf* __restrict__ ff = static_cast<Tf*>(const_cast<void*>(T_.fine));
    const Tc* __restrict__ fc = static_cast<const Tc*>(T_.coarse);
    const int n = T_.nx_f * T_.ny_f;
    double cc = 0.0, nn = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int e = m.y + k * 256 + threadIdx.x;
        if (e < n) {
            const int x = e % T_.nx_f, y = e / T_.nx_f;
            const size_t of = (size_t)y * T_.pitch_f + x, oc = (size_t)(y / 2) * T_.pitch_c + x / 2;
            Tf a[8];      // every plane's loads before the first store
            Tc c[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                a[i] = ff[of + (size_t)i * T_.plane_f];
                c[i] = __ldg(fc + oc + (size_t)i * T_.plane_c);
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const Tf v = Tf(a[i] + c[i]);
                ff[of + (size_t)i * T_.plane_f] = v;
                cc += (double)c[i] * (double)c[i];
                nn += (double)v * (double)v;
            }
        }
    }
    if (parts != nullptr) {
        const double sa = block_sum(cc, red);
        const double sb = block_sum(nn, red);
        if (threadIdx.x == 0) {
            parts[blockIdx.x] = sa;
            parts[nb + blockIdx.x] = sb;
        }
    }
}

// The mean first moments of a batch's level-0 populations (the mean of
// sum_i c_i f_i over an instance's cells, the displacement mode that a
// periodic problem leaves undetermined).  In exact arithmetic the V-cycle
// from zero with a zero-mean force keeps it at zero (collision adds the
// force, streaming and the transfers conserve it, the restricted residual has
// none); FP32 rounding makes it drift.  moment_map: FP64 partial sums of
// sum_i cx_i f_i and sum_i cy_i f_i over a block's cells (block map as the
// prolongation's); shift_map: f_i -= (cx_i mx + cy_i my) / 6, which moves the
// first moments by (mx, my) and leaves the others unchanged (sum_i c_i c_i^T
// = 6 I on D2Q8, odd moments of c vanish).
template <typename T>
__global__ void __launch_bounds__(256) batched_moment_map_kernel(const XlbbBatchTransfer* __restrict__ tr,
                                                                  const int2* __restrict__ map, int nb,
                                                                  double* parts) {
    grid_dep_wait();
    __shared__ double red[8];
    const int2 m = map[blockIdx.x];
    const XlbbBatchTransfer T_ = tr[m.x];
    const T* __restrict__ ff = static_cast<const T*>(T_.fine);
    const int n = T_.nx_f * T_.ny_f;
    double sx = 0.0, sy = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int e = m.y + k * 256 + threadIdx.x;
        if (e < n) {
            const size_t of = (size_t)(e / T_.nx_f) * T_.pitch_f + e % T_.nx_f;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const double v = (double)__ldg(ff + of + (size_t)i * T_.plane_f);
                sx += cx8(i) * v;
                sy += cy8(i) * v;
            }
        }
    }
    const double a = block_sum(sx, red);
    const double b = block_sum(sy, red);
    if (threadIdx.x == 0) {
        parts[blockIdx.x] = a;
        parts[nb + blockIdx.x] = b;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) batched_shift_map_kernel(const XlbbBatchTransfer* __restrict__ tr,
                                                                 const int2* __restrict__ map,
                                                                 const double* __restrict__ sums) {
    grid_dep_wait();
    const int2 m = map[blockIdx.x];
    const XlbbBatchTransfer T_ = tr[m.x];
    T* __restrict__ ff = static_cast<T*>(const_cast<void*>(T_.fine));
    const int n = T_.nx_f * T_.ny_f;
    const double mx = sums[2 * m.x] / n, my = sums[2 * m.x + 1] / n;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int e = m.y + k * 256 + threadIdx.x;
        if (e < n) {
            const size_t of = (size_t)(e / T_.nx_f) * T_.pitch_f + e % T_.nx_f;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const size_t a = of + (size_t)i * T_.plane_f;
                ff[a] = T((double)ff[a] - (cx8(i) * mx + cy8(i) * my) / 6.0);
            }
        }
    }
}

// norms[2 i] = sum of parts[begin[i] .. begin[i+1]), norms[2 i + 1] the same
// over parts[nb + ...] (fixed order: deterministic).
__global__ void pair_segment_sum_kernel(const double* parts, int nb, const int* begin, int nseg, double* norms) {
    grid_dep_wait();
    __shared__ double red[8];
    const int i = blockIdx.x;
    if (i >= nseg) return;
    double a = 0.0, b = 0.0;
    for (int t = begin[i] + threadIdx.x; t < begin[i + 1]; t += blockDim.x) {
        a += parts[t];
        b += parts[nb + t];
    }
    const double sa = block_sum(a, red);
    const double sb = block_sum(b, red);
    if (threadIdx.x == 0) {
        norms[2 * i] = sa;
        norms[2 * i + 1] = sb;
    }
}

__global__ void prolong_norms_kernel(const double* parts, int ninst, double* norms) {
    grid_dep_wait();
    const int i = blockIdx.x;
    if (i >= ninst) return;
    static_assert(XLBB_PROLONG_BLOCKS == 32, "one lane per block");
    const size_t base = (size_t)i * XLBB_PROLONG_BLOCKS + threadIdx.x;
    double a = parts[2 * base], b = parts[2 * base + 1];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if (threadIdx.x == 0) {
        norms[2 * i] = a;
        norms[2 * i + 1] = b;
    }
}

// Per-instance FP64 sums of tile partials (tiles of one instance are contiguous).
__global__ void segment_sum_kernel(const double* parts, const int* begin, int ninst, double* out) {
    grid_dep_wait();
    __shared__ double red[8];
    const int i = blockIdx.x;
    if (i >= ninst) return;
    double acc = 0.0;
    for (int t = begin[i] + threadIdx.x; t < begin[i + 1]; t += blockDim.x) acc += parts[t];
    const double s = block_sum(acc, red);
    if (threadIdx.x == 0) out[i] = s;
}


}  // namespace xlbb

#include "xlbb_tail.cuh"

using namespace xlbb;

#define XLBB_STREAM(s) (static_cast<cudaStream_t>(s))

extern "C" {

int xlbb_version(void) { return 100; }

const char* xlbb_last_error(void) { return g_last_error.c_str(); }

// Upper bound on the FP64 partials of a sweep of this dtype on g under the
// current launch config (the larger of its collide-and-push and row-marching
// shapes): enough to size a partials buffer for any sweep.
int xlbb_elast_sweep_ctas(int dtype, const XlbbGrid* g) {
    if (!grid_ok(g) || (dtype != XLBB_F32 && dtype != XLBB_F64 && dtype != XLBB_F32_ACC64))
        return fail(XLBB_EBADARG, "xlbb_elast_sweep_ctas: bad argument");
    const XlbbSweepConfig c = effective_cfg(0, dtype);
    const bool f32 = dtype == XLBB_F32;
    const long long n = std::max(launch_ctas(g, resolve_shape(c, true, f32)), launch_ctas(g, resolve_shape(c, false, f32)));
    return n > INT_MAX ? fail(XLBB_EBADARG, "xlbb_elast_sweep_ctas: grid too large") : (int)n;
}

int xlbb_darcy_sweep_ctas(int dtype, const XlbbGrid* g) {
    if (!grid_ok(g) || (dtype != XLBB_F32 && dtype != XLBB_F64 && dtype != XLBB_F32_ACC64))
        return fail(XLBB_EBADARG, "xlbb_darcy_sweep_ctas: bad argument");
    const XlbbSweepConfig c = effective_cfg(1, dtype);
    const bool f32 = dtype == XLBB_F32;
    const long long n = std::max(launch_ctas(g, resolve_shape(c, true, f32)), launch_ctas(g, resolve_shape(c, false, f32)));
    return n > INT_MAX ? fail(XLBB_EBADARG, "xlbb_darcy_sweep_ctas: grid too large") : (int)n;
}

// Exactly the FP64 partials that a sweep with these arguments writes with a
// fused sum: the count to hand to xlbb_reduce_sum.
int xlbb_darcy_sweep_partials(int dtype, const XlbbGrid* g, const XlbbDarcySweep* s) {
    if (!grid_ok(g) || !s) return fail(XLBB_EBADARG, "xlbb_darcy_sweep_partials: bad argument");
    long long n;
    if (dtype == XLBB_F32) n = darcy_partials_t<float>(g, s);
    else if (dtype == XLBB_F64) n = darcy_partials_t<double>(g, s);
    else if (dtype == XLBB_F32_ACC64) n = darcy_partials_t<double, float>(g, s);
    else return fail(XLBB_EBADARG, "xlbb_darcy_sweep_partials: dtype");
    return n > INT_MAX ? fail(XLBB_EBADARG, "xlbb_darcy_sweep_partials: grid too large") : (int)n;
}

int xlbb_elast_sweep_partials(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat, const XlbbElastSweep* s) {
    if (!grid_ok(g) || !mat || !s) return fail(XLBB_EBADARG, "xlbb_elast_sweep_partials: bad argument");
    long long n;
    if (dtype == XLBB_F32) n = elast_partials_t<float, float>(g, mat, s, dtype);
    else if (dtype == XLBB_F64) n = elast_partials_t<double, double>(g, mat, s, dtype);
    else if (dtype == XLBB_F32_ACC64) n = elast_partials_t<double, float>(g, mat, s, dtype);
    else return fail(XLBB_EBADARG, "xlbb_elast_sweep_partials: dtype");
    return n > INT_MAX ? fail(XLBB_EBADARG, "xlbb_elast_sweep_partials: grid too large") : (int)n;
}

int xlbb_sweep_set_config(int kernel, const XlbbSweepConfig* cfg) {
    if ((kernel != 0 && kernel != 1) || !cfg || !cfg_ok(*cfg)) return fail(XLBB_EBADARG, "xlbb_sweep_set_config: bad argument");
    g_cfg[kernel] = *cfg;
    return XLBB_OK;
}

int xlbb_device_status(int* status, int reset) {
    if (!status) return fail(XLBB_EBADARG, "xlbb_device_status: bad argument");
    cudaError_t e = cudaMemcpyFromSymbol(status, g_xlbb_status, sizeof(int));
    if (e == cudaSuccess && reset) {
        const int zero = 0;
        e = cudaMemcpyToSymbol(g_xlbb_status, &zero, sizeof(int));
    }
    if (e != cudaSuccess) return fail(XLBB_ELAUNCH, cudaGetErrorString(e));
    return XLBB_OK;
}

int xlbb_sweep_get_config(int kernel, XlbbSweepConfig* cfg) {
    if ((kernel != 0 && kernel != 1) || !cfg) return fail(XLBB_EBADARG, "xlbb_sweep_get_config: bad argument");
    *cfg = g_cfg[kernel];
    return XLBB_OK;
}

int xlbb_elast_sweep(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat, const XlbbElastSweep* s,
                     void* stream) {
    if (!grid_ok(g) || !mat || !s || !s->f_in || !s->f_out) return fail(XLBB_EBADARG, "xlbb_elast_sweep: bad argument");
    if (s->f_in == s->f_out) return fail(XLBB_EBADARG, "xlbb_elast_sweep: f_in and f_out must differ");
    if (!rules_ok(s->pc, g) || !rules_ok(s->ps, g)) return fail(XLBB_EBADARG, "xlbb_elast_sweep: incomplete rules");

    if ((mat->mu_field == nullptr) != (mat->lam_field == nullptr))
        return fail(XLBB_EBADARG, "xlbb_elast_sweep: lam_field and mu_field go together");
    if (s->div_out && s->sumsq && effective_cfg(0, dtype).pipeline == 3)
        return fail(XLBB_EUNSUPPORTED, "xlbb_elast_sweep: div_out with sumsq needs a row-marching launch shape");
    if (dtype == XLBB_F32) return elast_sweep_t<float>(g, mat, s, XLBB_STREAM(stream));
    if (dtype == XLBB_F64) return elast_sweep_t<double>(g, mat, s, XLBB_STREAM(stream));
    if (dtype == XLBB_F32_ACC64) return elast_sweep_t<double, float>(g, mat, s, XLBB_STREAM(stream));
    return fail(XLBB_EUNSUPPORTED, "xlbb_elast_sweep: dtype");
}

int xlbb_elast_sweep_pipeline(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat, const XlbbElastSweep* s) {
    if (!grid_ok(g) || !mat || !s) return fail(XLBB_EBADARG, "xlbb_elast_sweep_pipeline: bad argument");
    if (dtype == XLBB_F32 && g_cfg[0].pipeline == 4) {
        const bool ok = s->resid ? grid_push4_ok(g, elast_args<float, true>(g, mat, s))
                                 : grid_push4_ok(g, elast_args<float, false>(g, mat, s));
        if (ok) return 4;
    }
    const XlbbSweepConfig c = effective_cfg(0, dtype);
    const bool push = push_eligible<ElastPhys<double, false>>(elast_args<double, false>(g, mat, s));
    return resolve_shape(c, push, dtype == XLBB_F32).pipeline;
}

int xlbb_darcy_sweep_pipeline(int dtype, const XlbbGrid* g, const XlbbDarcySweep* s) {
    if (!grid_ok(g) || !s || (dtype != XLBB_F32 && dtype != XLBB_F64 && dtype != XLBB_F32_ACC64))
        return fail(XLBB_EBADARG, "xlbb_darcy_sweep_pipeline: bad argument");
    if (dtype == XLBB_F32 && g_cfg[1].pipeline == 4 && darcy4_ok(g, s)) return 4;
    const XlbbSweepConfig c = effective_cfg(1, dtype);
    const bool push = push_eligible<DarcyPhys<double>>(darcy_args<DarcyPhys<double>>(g, s));
    return resolve_shape(c, push, dtype == XLBB_F32).pipeline;
}

int xlbb_darcy_sweep(int dtype, const XlbbGrid* g, const XlbbDarcySweep* s, void* stream) {
    if (!grid_ok(g) || !s || !s->f_in || !s->f_out) return fail(XLBB_EBADARG, "xlbb_darcy_sweep: bad argument");
    if (s->f_in == s->f_out) return fail(XLBB_EBADARG, "xlbb_darcy_sweep: f_in and f_out must differ");
    if (!rules_ok(s->pc, g) || !rules_ok(s->ps, g)) return fail(XLBB_EBADARG, "xlbb_darcy_sweep: incomplete rules");
    if (s->resid && s->pc.count > 0 && s->pc.row_ptr)
        return fail(XLBB_EUNSUPPORTED, "xlbb_darcy_sweep: resid with post-collision rules");

    if (dtype == XLBB_F32) return darcy_sweep_t<float>(g, s, XLBB_STREAM(stream));
    if (dtype == XLBB_F64) return darcy_sweep_t<double>(g, s, XLBB_STREAM(stream));
    if (dtype == XLBB_F32_ACC64) return darcy_sweep_t<double, float>(g, s, XLBB_STREAM(stream));
    return fail(XLBB_EUNSUPPORTED, "xlbb_darcy_sweep: dtype");
}

int xlbb_fluid_sweep(int dtype, const XlbbGrid* g, const XlbbDarcySweep* s, int model, void* stream) {
    if (!grid_ok(g) || !s || !s->f_in || !s->f_out) return fail(XLBB_EBADARG, "xlbb_fluid_sweep: bad argument");
    if (model != XLBB_FLUID_BGK && model != XLBB_FLUID_KBC) return fail(XLBB_EBADARG, "xlbb_fluid_sweep: model");
    if (s->f_in == s->f_out) return fail(XLBB_EBADARG, "xlbb_fluid_sweep: f_in and f_out must differ");
    if (s->source || s->ext_source || s->resid)
        return fail(XLBB_EBADARG, "xlbb_fluid_sweep: source and resid planes are not supported");
    if (!rules_ok(s->pc, g) || !rules_ok(s->ps, g)) return fail(XLBB_EBADARG, "xlbb_fluid_sweep: incomplete rules");

    const bool kbc = model == XLBB_FLUID_KBC;
    if (dtype == XLBB_F32)
        return kbc ? fluid_sweep_t<float, true>(g, s, XLBB_STREAM(stream)) : fluid_sweep_t<float, false>(g, s, XLBB_STREAM(stream));
    if (dtype == XLBB_F64)
        return kbc ? fluid_sweep_t<double, true>(g, s, XLBB_STREAM(stream)) : fluid_sweep_t<double, false>(g, s, XLBB_STREAM(stream));
    return fail(XLBB_EUNSUPPORTED, "xlbb_fluid_sweep: dtype");
}

int xlbb_fluid3_sweep(int dtype, const XlbbGrid3* g, const XlbbDarcySweep* s, int q, int model, void* stream) {
    if (!grid3_ok(g) || !s || !s->f_in || !s->f_out) return fail(XLBB_EBADARG, "xlbb_fluid3_sweep: bad argument");
    if (q != 19 && q != 27) return fail(XLBB_EBADARG, "xlbb_fluid3_sweep: q must be 19 or 27");
    if (model != XLBB_FLUID_BGK && !(model == XLBB_FLUID_KBC && q == 27))
        return fail(XLBB_EBADARG, "xlbb_fluid3_sweep: model (KBC needs q = 27)");
    if (s->f_in == s->f_out) return fail(XLBB_EBADARG, "xlbb_fluid3_sweep: f_in and f_out must differ");
    if (s->omega_field || s->source || s->ext_source || s->resid || s->sumsq)
        return fail(XLBB_EBADARG, "xlbb_fluid3_sweep: omega_field, source, ext_source, resid and sumsq must be NULL");
    const XlbbGrid rows = {g->nx, g->ny * g->nz, g->pitch, g->plane};
    if (!rules_ok(s->pc, &rows) || !rules_ok(s->ps, &rows)) return fail(XLBB_EBADARG, "xlbb_fluid3_sweep: incomplete rules");
    if (s->ps.count > 0 && s->ps.row_ptr && !s->ps.push)
        return fail(XLBB_EUNSUPPORTED, "xlbb_fluid3_sweep: PostStreaming rules without push words");
    const cudaStream_t st = XLBB_STREAM(stream);
    const bool kbc = model == XLBB_FLUID_KBC;
    if (dtype == XLBB_F32)
        return q == 19 ? fluid3_sweep_t<float, 19>(g, s, st)
                       : (kbc ? fluid3_sweep_t<float, 27, true>(g, s, st) : fluid3_sweep_t<float, 27>(g, s, st));
    if (dtype == XLBB_F64)
        return q == 19 ? fluid3_sweep_t<double, 19>(g, s, st)
                       : (kbc ? fluid3_sweep_t<double, 27, true>(g, s, st) : fluid3_sweep_t<double, 27>(g, s, st));
    return fail(XLBB_EUNSUPPORTED, "xlbb_fluid3_sweep: dtype");
}

int xlbb_darcy_gradient(int dtype, const XlbbGrid* g, const void* q, double scale, const XlbbRules* rules,
                        const void* base, void* out, void* stream) {
    if (!grid_ok(g) || !q || !out) return fail(XLBB_EBADARG, "xlbb_darcy_gradient: bad argument");
    XlbbRules none = {0, nullptr, nullptr, nullptr, nullptr};
    const XlbbRules& r = rules ? *rules : none;
    const dim3 grid = row_grid(g->nx, g->ny, 128);
    if (dtype == XLBB_F32)
        launch_k(gradient_kernel<float>, grid, 128, 0, XLBB_STREAM(stream), geom(g), (const float*)q, (float)scale,
                                                                      rules_view<float, 9>(r), (const float*)base, (float*)out);
    else if (dtype == XLBB_F64)
        launch_k(gradient_kernel<double>, grid, 128, 0, XLBB_STREAM(stream), geom(g), (const double*)q, scale,
                                                                       rules_view<double, 9>(r), (const double*)base, (double*)out);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_darcy_gradient: dtype");
    return check_launch("xlbb_darcy_gradient");
}

int xlbb_elast_moments(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat, const void* f, const void* force,
                       const void* fext, void* eta, void* sigma, void* div, double div_scale, void* stream) {
    if (!grid_ok(g) || !mat || !f) return fail(XLBB_EBADARG, "xlbb_elast_moments: bad argument");
    const dim3 grid = row_grid(g->nx, g->ny, 128);
    if (dtype == XLBB_F32)
        launch_k(elast_moments_kernel<float>, grid, 128, 0, XLBB_STREAM(stream), 
            geom(g), make_mat<float>(mat), (float)mat->lam, (float)mat->mu, (const float*)f, (const float*)force,
            (const float*)fext, (float*)eta, (float*)sigma, (float*)div, (float)div_scale);
    else if (dtype == XLBB_F64)
        launch_k(elast_moments_kernel<double>, grid, 128, 0, XLBB_STREAM(stream), 
            geom(g), make_mat<double>(mat), mat->lam, mat->mu, (const double*)f, (const double*)force,
            (const double*)fext, (double*)eta, (double*)sigma, (double*)div, div_scale);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_elast_moments: dtype");
    return check_launch("xlbb_elast_moments");
}

int xlbb_elast_divgrad(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat, double div_scale, const void* f,
                       double scale, const XlbbRules* rules, const void* base, void* out, void* stream) {
    if (!grid_ok(g) || !mat || !f || !out) return fail(XLBB_EBADARG, "xlbb_elast_divgrad: bad argument");
    XlbbRules none = {0, nullptr, nullptr, nullptr, nullptr};
    const XlbbRules& r = rules ? *rules : none;
    const dim3 grid((g->nx + 31) / 32, (g->ny + 7) / 8), blk(32, 8);
    if (dtype == XLBB_F32)
        launch_k(elast_divgrad_kernel<float>, grid, blk, 0, XLBB_STREAM(stream), geom(g), make_mat<float>(mat),
                 (float)mat->lam, (float)mat->mu, (float)div_scale, (const float*)f, (float)scale,
                 rules_view<float, 9>(r), (const float*)base, (float*)out);
    else if (dtype == XLBB_F64)
        launch_k(elast_divgrad_kernel<double>, grid, blk, 0, XLBB_STREAM(stream), geom(g), make_mat<double>(mat),
                 mat->lam, mat->mu, div_scale, (const double*)f, scale, rules_view<double, 9>(r),
                 (const double*)base, (double*)out);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_elast_divgrad: dtype");
    return check_launch("xlbb_elast_divgrad");
}

int xlbb_elast_sweep_divgrad(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat, const XlbbElastSweep* s,
                             double div_scale, double scale, const XlbbRules* grad_rules, void* stream) {
    if (!grid_ok(g) || !mat || !s || !s->f_in || !s->f_out || s->f_in == s->f_out)
        return fail(XLBB_EBADARG, "xlbb_elast_sweep_divgrad: bad argument");
    if (!rules_ok(s->pc, g) || !rules_ok(s->ps, g)) return fail(XLBB_EBADARG, "xlbb_elast_sweep_divgrad: incomplete rules");
    if ((mat->mu_field == nullptr) != (mat->lam_field == nullptr))
        return fail(XLBB_EBADARG, "xlbb_elast_sweep_divgrad: lam_field and mu_field go together");
    if (s->sumsq || s->div_out || (dtype != XLBB_F32 && dtype != XLBB_F64))
        return fail(XLBB_EUNSUPPORTED, "xlbb_elast_sweep_divgrad: fused sums, side outputs and mixed precision "
                                       "take xlbb_elast_divgrad + xlbb_elast_sweep");
    XlbbRules none = {0, nullptr, nullptr, nullptr, nullptr};
    const XlbbRules& gr = grad_rules ? *grad_rules : none;
    const dim3 grid((g->nx + 31) / 32, (g->ny + 7) / 8), blk(32, 8);
#define XLBB_DGP(T_, R_)                                                                                      \
    {                                                                                                         \
        using Ph = ElastPhys<T_, R_>;                                                                         \
        typename Ph::Args a = elast_args<T_, R_>(g, mat, s);                                                  \
        if (!push_eligible<Ph>(a))                                                                            \
            return fail(XLBB_EUNSUPPORTED, "xlbb_elast_sweep_divgrad: post-streaming rules without push words"); \
        const T_* base = static_cast<const T_*>(s->fext);                                                     \
        a.fext = nullptr;                                                                                     \
        a.ext_in_kernel = 1;                                                                                  \
        Ph::fill_ptrs(a);                                                                                     \
        launch_k(elast_divgrad_push_kernel<T_, R_>, grid, blk, 0, XLBB_STREAM(stream), a, (T_)mat->lam,        \
                 (T_)mat->mu, (T_)div_scale, (T_)scale, rules_view<T_, 9>(gr), base);                           \
    }
    if (dtype == XLBB_F32) {
        if (s->resid) XLBB_DGP(float, true) else XLBB_DGP(float, false)
    } else {
        if (s->resid) XLBB_DGP(double, true) else XLBB_DGP(double, false)
    }
#undef XLBB_DGP
    return check_launch("xlbb_elast_sweep_divgrad");
}

int xlbb_elast_equilibrium(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat, const void* eta,
                           const void* sigma, const void* force, const void* fext, void* f_out, void* stream) {
    if (!grid_ok(g) || !mat || !eta || !sigma || !f_out) return fail(XLBB_EBADARG, "xlbb_elast_equilibrium: bad argument");
    const dim3 grid = row_grid(g->nx, g->ny, 128);
    if (dtype == XLBB_F32)
        launch_k(elast_equilibrium_kernel<float>, grid, 128, 0, XLBB_STREAM(stream), 
            geom(g), (float)mat->lam, (float)mat->mu, (const float*)mat->lam_field, (const float*)mat->mu_field,
            (const float*)eta, (const float*)sigma, (const float*)force, (const float*)fext, (float*)f_out);
    else if (dtype == XLBB_F64)
        launch_k(elast_equilibrium_kernel<double>, grid, 128, 0, XLBB_STREAM(stream), 
            geom(g), mat->lam, mat->mu, (const double*)mat->lam_field, (const double*)mat->mu_field,
            (const double*)eta, (const double*)sigma, (const double*)force, (const double*)fext, (double*)f_out);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_elast_equilibrium: dtype");
    return check_launch("xlbb_elast_equilibrium");
}

int xlbb_darcy_moments(int dtype, const XlbbGrid* g, const void* f, double omega, const void* omega_field,
                       const void* source, const void* ext_source, void* rho, void* grad, void* stream) {
    if (!grid_ok(g) || !f) return fail(XLBB_EBADARG, "xlbb_darcy_moments: bad argument");
    const dim3 grid = row_grid(g->nx, g->ny, 128);
    if (dtype == XLBB_F32)
        launch_k(darcy_moments_kernel<float>, grid, 128, 0, XLBB_STREAM(stream), 
            geom(g), (const float*)f, (float)omega, (const float*)omega_field, (const float*)source,
            (const float*)ext_source, (float*)rho, (float*)grad);
    else if (dtype == XLBB_F64)
        launch_k(darcy_moments_kernel<double>, grid, 128, 0, XLBB_STREAM(stream), 
            geom(g), (const double*)f, omega, (const double*)omega_field, (const double*)source,
            (const double*)ext_source, (double*)rho, (double*)grad);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_darcy_moments: dtype");
    return check_launch("xlbb_darcy_moments");
}

int xlbb_restrict(int dtype_fine, int dtype_coarse, const XlbbGrid* fine, const XlbbGrid* coarse, int q, int x0,
                  int x1bc, int y0, int y1bc, const void* res, void* r_coarse, void* stream) {
    if (!grid_ok(fine) || !grid_ok(coarse) || !res || !r_coarse || q <= 0)
        return fail(XLBB_EBADARG, "xlbb_restrict: bad argument");
    const int nfx = fine->nx - x0 - x1bc, nfy = fine->ny - y0 - y1bc;
    if (nfx % 2 || nfy % 2 || coarse->nx != nfx / 2 + x0 + x1bc || coarse->ny != nfy / 2 + y0 + y1bc)
        return fail(XLBB_EBADARG, "xlbb_restrict: coarse grid does not match the fine interior");
    const dim3 grid = row_grid(coarse->nx, coarse->ny, 128);
    cudaStream_t st = XLBB_STREAM(stream);
#define XLBB_R(TF, TC) \
    launch_k(restrict_kernel<TF, TC>, grid, 128, 0, st, geom(fine), geom(coarse), q, x0, y0, nfx / 2, nfy / 2, (const TF*)res, (TC*)r_coarse)
    if (dtype_fine == XLBB_F32 && dtype_coarse == XLBB_F32) XLBB_R(float, float);
    else if (dtype_fine == XLBB_F32 && dtype_coarse == XLBB_F64) XLBB_R(float, double);
    else if (dtype_fine == XLBB_F64 && dtype_coarse == XLBB_F64) XLBB_R(double, double);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_restrict: dtype pair");
#undef XLBB_R
    return check_launch("xlbb_restrict");
}

int xlbb_prolong_add(int dtype_fine, int dtype_coarse, const XlbbGrid* fine, const XlbbGrid* coarse, int q, int x0,
                     int x1bc, int y0, int y1bc, const void* f_coarse, void* f_fine, void* stream) {
    if (!grid_ok(fine) || !grid_ok(coarse) || !f_coarse || !f_fine || q <= 0)
        return fail(XLBB_EBADARG, "xlbb_prolong_add: bad argument");
    const int nfx = fine->nx - x0 - x1bc, nfy = fine->ny - y0 - y1bc;
    if (nfx % 2 || nfy % 2 || coarse->nx != nfx / 2 + x0 + x1bc || coarse->ny != nfy / 2 + y0 + y1bc)
        return fail(XLBB_EBADARG, "xlbb_prolong_add: coarse grid does not match the fine interior");
    const dim3 grid = row_grid(nfx, nfy, 128);
    cudaStream_t st = XLBB_STREAM(stream);
#define XLBB_P(TF, TC) \
    launch_k(prolong_add_kernel<TF, TC>, grid, 128, 0, st, geom(fine), geom(coarse), q, x0, y0, nfx, nfy, (const TC*)f_coarse, (TF*)f_fine)
    if (dtype_fine == XLBB_F32 && dtype_coarse == XLBB_F32) XLBB_P(float, float);
    else if (dtype_fine == XLBB_F32 && dtype_coarse == XLBB_F64) XLBB_P(float, double);
    else if (dtype_fine == XLBB_F64 && dtype_coarse == XLBB_F64) XLBB_P(double, double);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_prolong_add: dtype pair");
#undef XLBB_P
    return check_launch("xlbb_prolong_add");
}

int xlbb_sumsq_ctas(const XlbbGrid* g) {
    (void)g;
    return 2 * num_sms();
}

int xlbb_sumsq(int dtype, const XlbbGrid* g, int nplanes, const void* data, int bx0, int bx1, int by0, int by1,
               double* partials, void* stream) {
    if (!grid_ok(g) || !data || !partials || nplanes <= 0 || bx0 < 0 || by0 < 0 || bx1 > g->nx || by1 > g->ny ||
        bx1 <= bx0 || by1 <= by0)
        return fail(XLBB_EBADARG, "xlbb_sumsq: bad argument");
    const int nb = xlbb_sumsq_ctas(g);
    if (dtype == XLBB_F32)
        launch_k(sumsq_kernel<float>, nb, 256, 0, XLBB_STREAM(stream), geom(g), nplanes, (const float*)data, bx0, bx1, by0,
                                                                 by1, partials);
    else if (dtype == XLBB_F64)
        launch_k(sumsq_kernel<double>, nb, 256, 0, XLBB_STREAM(stream), geom(g), nplanes, (const double*)data, bx0, bx1,
                                                                  by0, by1, partials);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_sumsq: dtype");
    return check_launch("xlbb_sumsq");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Darcy sweep + FP64 residual without caller-provided scratch.
//
// Some callers cannot allocate device memory: code running inside a CUDA
// graph being captured, a host runtime that hands this library only the
// buffers it owns (inputs and outputs), or a process whose allocator is not
// allowed to grow.  For them the per-CTA FP64 partial sums of the residual
// live in this file-scope device array (XLBB_NOALLOC_MAX_PARTIALS doubles,
// 128 KiB, held by every GPU that loads the library until the process exits).
// Host code only uses the array's device address, obtained once per device
// with cudaGetSymbolAddress while that device is current.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double g_noalloc_partials[XLBB_NOALLOC_MAX_PARTIALS];

static std::mutex g_noalloc_mutex;
static double* g_noalloc_addr[XLBB_NOALLOC_MAX_DEVICES] = {nullptr};

// Device address of the scratch array on the current device (looked up on the
// first call per device).
static int noalloc_scratch(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(XLBB_ELAUNCH, cudaGetErrorString(e));
    if (dev < 0 || dev >= XLBB_NOALLOC_MAX_DEVICES)
        return fail(XLBB_EUNSUPPORTED, "xlbb_darcy_sweep_residual_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_addr[dev] == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || p == nullptr) {
            g_last_error = std::string("xlbb_darcy_sweep_residual_noalloc: cudaGetSymbolAddress failed: ") +
                           cudaGetErrorString(e);
            return XLBB_ELAUNCH;
        }
        g_noalloc_addr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_addr[dev];
    return XLBB_OK;
}

extern "C" {

int xlbb_darcy_sweep_residual_noalloc(int dtype, const XlbbGrid* g, const XlbbDarcySweep* s, double* sumsq_out,
                                      void* stream) {
    if (!grid_ok(g) || !s || !sumsq_out) return fail(XLBB_EBADARG, "xlbb_darcy_sweep_residual_noalloc: bad argument");
    // the partials of the launch this sweep actually takes (push or row-marching shape)
    const int n = xlbb_darcy_sweep_partials(dtype, g, s);
    if (n < 0) return n;
    if (n > XLBB_NOALLOC_MAX_PARTIALS) {
        g_last_error = "xlbb_darcy_sweep_residual_noalloc: this sweep's launch has " + std::to_string(n) +
                       " CTAs, more than the " + std::to_string(XLBB_NOALLOC_MAX_PARTIALS) +
                       " partials of the built-in scratch (the collide-and-push shape has ceil(nx/tx)*ny CTAs; "
                       "a row-marching shape, xlbb_sweep_set_config pipeline 0-2, has about ctas_per_sm per SM)";
        return XLBB_EBADARG;
    }
    double* scratch = nullptr;
    const int rc = noalloc_scratch(&scratch);
    if (rc != XLBB_OK) return rc;
    XlbbDarcySweep local = *s;
    local.sumsq = scratch;      // the launch's n CTAs write slots 0..n-1 before the reduction reads them
    const int st = xlbb_darcy_sweep(dtype, g, &local, stream);
    if (st != XLBB_OK) return st;
    return xlbb_reduce_sum(scratch, n, sumsq_out, stream);
}

int xlbb_wait_selftest(unsigned polls, int* gave_up, void* stream) {
    if (!gave_up || polls == 0 || polls > (1u << 22)) return fail(XLBB_EBADARG, "xlbb_wait_selftest: bad argument");
    wait_selftest_kernel<<<1, 32, 0, XLBB_STREAM(stream)>>>(polls, gave_up);
    return check_launch("xlbb_wait_selftest");
}

int xlbb_reduce_sum(const double* partials, int n, double* out, void* stream) {
    if (!partials || !out || n <= 0) return fail(XLBB_EBADARG, "xlbb_reduce_sum: bad argument");
    launch_k(reduce_sum_kernel, 1, 1024, 0, XLBB_STREAM(stream), partials, n, out);
    return check_launch("xlbb_reduce_sum");
}

int xlbb_axpby(int dtype, long long n, double a, const void* x, double b, const void* y, void* out, void* stream) {
    if (n < 0 || (n > 0 && (!x || !y || !out))) return fail(XLBB_EBADARG, "xlbb_axpby: bad argument");
    if (n == 0) return XLBB_OK;
    long long nb = (n + 255) / 256;
    if (nb > 8 * num_sms()) nb = 8 * num_sms();
    if (dtype == XLBB_F32)
        launch_k(axpby_kernel<float>, (int)nb, 256, 0, XLBB_STREAM(stream), n, (float)a, (const float*)x, (float)b,
                                                                      (const float*)y, (float*)out);
    else if (dtype == XLBB_F64)
        launch_k(axpby_kernel<double>, (int)nb, 256, 0, XLBB_STREAM(stream), n, a, (const double*)x, b, (const double*)y,
                                                                       (double*)out);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_axpby: dtype");
    return check_launch("xlbb_axpby");
}


// ---------------------------------------------------------------------------
// Batched multigrid entry points.
// ---------------------------------------------------------------------------
int xlbb_batch_upload(int dtype, const XlbbBatchInstance* host, int ninst, void* dev, void* stream) {
    if (!host || !dev || ninst <= 0) return fail(XLBB_EBADARG, "xlbb_batch_upload: bad argument");
    for (int i = 0; i < ninst; ++i)   // the sweeps address the 8 planes of an instance with 32-bit offsets
        if (host[i].nx <= 0 || host[i].ny <= 0 || host[i].pitch < host[i].nx ||
            host[i].plane < (long long)host[i].pitch * host[i].ny || host[i].plane >= (1ll << 28))
            return fail(XLBB_EBADARG, "xlbb_batch_upload: instance geometry (plane must be below 2^28 elements)");
    if (dtype == XLBB_F32) {
        std::vector<BatchInst<float>> v(ninst);
        for (int i = 0; i < ninst; ++i) v[i] = to_batch_inst<float>(host[i]);
        cudaMemcpyAsync(dev, v.data(), sizeof(BatchInst<float>) * ninst, cudaMemcpyHostToDevice, XLBB_STREAM(stream));
        return cudaStreamSynchronize(XLBB_STREAM(stream)) == cudaSuccess ? XLBB_OK : fail(XLBB_ELAUNCH, "xlbb_batch_upload");
    }
    if (dtype == XLBB_F64) {
        std::vector<BatchInst<double>> v(ninst);
        for (int i = 0; i < ninst; ++i) v[i] = to_batch_inst<double>(host[i]);
        cudaMemcpyAsync(dev, v.data(), sizeof(BatchInst<double>) * ninst, cudaMemcpyHostToDevice, XLBB_STREAM(stream));
        return cudaStreamSynchronize(XLBB_STREAM(stream)) == cudaSuccess ? XLBB_OK : fail(XLBB_ELAUNCH, "xlbb_batch_upload");
    }
    if (dtype == XLBB_F32_ACC64) {
        std::vector<BatchInst<double, float>> v(ninst);
        for (int i = 0; i < ninst; ++i) v[i] = to_batch_inst<double, float>(host[i]);
        cudaMemcpyAsync(dev, v.data(), sizeof(BatchInst<double, float>) * ninst, cudaMemcpyHostToDevice,
                        XLBB_STREAM(stream));
        return cudaStreamSynchronize(XLBB_STREAM(stream)) == cudaSuccess ? XLBB_OK : fail(XLBB_ELAUNCH, "xlbb_batch_upload");
    }
    return fail(XLBB_EUNSUPPORTED, "xlbb_batch_upload: dtype");
}

int xlbb_batch_desc_bytes(int dtype) {
    if (dtype == XLBB_F64) return (int)sizeof(BatchInst<double>);
    if (dtype == XLBB_F32_ACC64) return (int)sizeof(BatchInst<double, float>);
    return (int)sizeof(BatchInst<float>);
}

}  // extern "C"

// Zero the input populations (8 planes) of every tile's cells: the
// row-marching form's stand-in for zero_in (it reads its input rows).
template <typename T, typename S>
__global__ void batched_zero_in_kernel(const BatchInst<T, S>* __restrict__ inst, const XlbbBatchTile* __restrict__ tiles,
                                       int ntiles) {
    grid_dep_wait();
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const XlbbBatchTile tl = tiles[t];
        const BatchInst<T, S>& I = inst[tl.inst];
        S* f = const_cast<S*>(I.f_in);
        const int x = tl.x0 + threadIdx.x;
        if (x >= I.geom.nx) continue;
        for (int y = tl.ys; y < tl.ye; ++y)
            for (int i = 0; i < 8; ++i) f[(size_t)y * I.geom.pitch + x + (size_t)i * I.geom.plane] = S(0);
    }
}

template <typename T, typename S = T>
static int batched_sweep_t(const void* inst, const XlbbBatchTile* tiles, int ntiles, int ctas, double a, double b,
                           int use_force, int has_resid, int sumsq_diff, double* tile_sumsq, int zero_in,
                           cudaStream_t st) {
    const int mix = (a == 0.0 && b == 1.0) ? 0 : 1;
    const bool prev = mix || (tile_sumsq && sumsq_diff);
    const BatchInst<T, S>* I = static_cast<const BatchInst<T, S>*>(inst);
    if (g_cfg[0].pipeline >= 3) {     // collide and push
        const dim3 blk(128, 8);
        // the CTAs loop over the tile list: launch at most one wave of resident CTAs
#define XLBB_BP(R, Q_)                                                                                        \
    do {                                                                                                      \
        static int resident = 0;                                                                              \
        if (resident == 0) {                                                                                  \
            int per_sm = 0;                                                                                   \
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_push_kernel<T, R, Q_, S>,          \
                                                          (int)(blk.x * blk.y), 0);                           \
            resident = (per_sm > 0 ? per_sm : 1) * num_sms();                                                 \
        }                                                                                                     \
        launch_k(batched_push_kernel<T, R, Q_, S>, ctas < resident ? ctas : resident, blk, 0, st,                   \
            I, tiles, ntiles, T(a), T(b), mix, use_force, sumsq_diff, tile_sumsq, zero_in);                   \
    } while (0)
        if (has_resid) { if (tile_sumsq) XLBB_BP(true, true); else XLBB_BP(true, false); }
        else { if (tile_sumsq) XLBB_BP(false, true); else XLBB_BP(false, false); }
#undef XLBB_BP
        return check_launch("xlbb_batched_elast_sweep");
    }
    if (zero_in) launch_k(batched_zero_in_kernel<T, S>, ctas, 128, 0, st, I, tiles, ntiles);
#define XLBB_B(R, P) \
    launch_k(batched_elast_kernel<T, 128, R, P, S>, ctas, 160, 0, st, I, tiles, ntiles, T(a), T(b), mix, use_force, \
                                                                 sumsq_diff, tile_sumsq)
    if (has_resid) { if (prev) XLBB_B(true, true); else XLBB_B(true, false); }
    else { if (prev) XLBB_B(false, true); else XLBB_B(false, false); }
#undef XLBB_B
    return check_launch("xlbb_batched_elast_sweep");
}

// Four-column batched sweep: CTAs of 32 x 16 threads (a warp per tile row),
// at most one wave of resident CTAs.
template <typename T>
static int batched_sweep4_t(const void* inst, const XlbbBatchTile* tiles, int ntiles, int ctas, double a, double b,
                            int use_force, int has_resid, int sumsq_diff, double* tile_sumsq, int zero_in,
                            cudaStream_t st) {
    const int mix = (a == 0.0 && b == 1.0) ? 0 : 1;
    const BatchInst<T, float>* I = static_cast<const BatchInst<T, float>*>(inst);
    const dim3 blk(32, 16);
#define XLBB_BP4(R, Q_)                                                                                       \
    do {                                                                                                      \
        static int resident = 0;                                                                              \
        if (resident == 0) {                                                                                  \
            int per_sm = 0;                                                                                   \
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_push4_kernel<T, R, Q_>,            \
                                                          (int)(blk.x * blk.y), 0);                           \
            resident = (per_sm > 0 ? per_sm : 1) * num_sms();                                                 \
        }                                                                                                     \
        launch_k(batched_push4_kernel<T, R, Q_>, ctas < resident ? ctas : resident, blk, 0, st,                     \
            I, tiles, ntiles, T(a), T(b), mix, use_force, sumsq_diff, tile_sumsq, zero_in);                   \
    } while (0)
    if (has_resid) { if (tile_sumsq) XLBB_BP4(true, true); else XLBB_BP4(true, false); }
    else { if (tile_sumsq) XLBB_BP4(false, true); else XLBB_BP4(false, false); }
#undef XLBB_BP4
    return check_launch("xlbb_batched_elast_sweep4");
}

extern "C" {

int xlbb_batched_elast_sweep(int dtype, const void* inst_dev, const XlbbBatchTile* tiles_dev, int ntiles, int ctas,
                             double a, double b, int use_force, int has_resid, int sumsq_diff, double* tile_sumsq,
                             int zero_in, void* stream) {
    if (!inst_dev || !tiles_dev || ntiles <= 0 || ctas <= 0) return fail(XLBB_EBADARG, "xlbb_batched_elast_sweep: bad argument");
    if (dtype == XLBB_F32)
        return batched_sweep_t<float>(inst_dev, tiles_dev, ntiles, ctas, a, b, use_force, has_resid, sumsq_diff,
                                      tile_sumsq, zero_in, XLBB_STREAM(stream));
    if (dtype == XLBB_F64)
        return batched_sweep_t<double>(inst_dev, tiles_dev, ntiles, ctas, a, b, use_force, has_resid, sumsq_diff,
                                       tile_sumsq, zero_in, XLBB_STREAM(stream));
    if (dtype == XLBB_F32_ACC64)
        return batched_sweep_t<double, float>(inst_dev, tiles_dev, ntiles, ctas, a, b, use_force, has_resid,
                                              sumsq_diff, tile_sumsq, zero_in, XLBB_STREAM(stream));
    return fail(XLBB_EUNSUPPORTED, "xlbb_batched_elast_sweep: dtype");
}

int xlbb_batched_elast_sweep4(int dtype, const void* inst_dev, const XlbbBatchTile* tiles_dev, int ntiles, int ctas,
                              double a, double b, int use_force, int has_resid, int sumsq_diff, double* tile_sumsq,
                              int zero_in, void* stream) {
    if (!inst_dev || !tiles_dev || ntiles <= 0 || ctas <= 0)
        return fail(XLBB_EBADARG, "xlbb_batched_elast_sweep4: bad argument");
    if (dtype == XLBB_F32)
        return batched_sweep4_t<float>(inst_dev, tiles_dev, ntiles, ctas, a, b, use_force, has_resid, sumsq_diff,
                                       tile_sumsq, zero_in, XLBB_STREAM(stream));
    return fail(XLBB_EUNSUPPORTED, "xlbb_batched_elast_sweep4: dtype (XLBB_F32 only)");
}

int xlbb_batched_restrict(int dtype_fine, int dtype_coarse, const XlbbBatchTransfer* tr_dev, int ninst, void* stream) {
    if (!tr_dev || ninst <= 0) return fail(XLBB_EBADARG, "xlbb_batched_restrict: bad argument");
    const dim3 grid(16, ninst);
    cudaStream_t st = XLBB_STREAM(stream);
    if (dtype_fine == XLBB_F32 && dtype_coarse == XLBB_F32) launch_k(batched_restrict_kernel<float, float>, grid, 256, 0, st, tr_dev);
    else if (dtype_fine == XLBB_F32 && dtype_coarse == XLBB_F64) launch_k(batched_restrict_kernel<float, double>, grid, 256, 0, st, tr_dev);
    else if (dtype_fine == XLBB_F64 && dtype_coarse == XLBB_F64) launch_k(batched_restrict_kernel<double, double>, grid, 256, 0, st, tr_dev);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_batched_restrict: dtype pair");
    return check_launch("xlbb_batched_restrict");
}

static int prolong_t(int dtype_fine, int dtype_coarse, const XlbbBatchTransfer* tr_dev, int ninst, double* parts,
                     cudaStream_t st) {
    const dim3 grid(XLBB_PROLONG_BLOCKS, ninst);
    if (dtype_fine == XLBB_F32 && dtype_coarse == XLBB_F32) launch_k(batched_prolong_add_kernel<float, float>, grid, 256, 0, st, tr_dev, parts);
    else if (dtype_fine == XLBB_F32 && dtype_coarse == XLBB_F64) launch_k(batched_prolong_add_kernel<float, double>, grid, 256, 0, st, tr_dev, parts);
    else if (dtype_fine == XLBB_F64 && dtype_coarse == XLBB_F64) launch_k(batched_prolong_add_kernel<double, double>, grid, 256, 0, st, tr_dev, parts);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_batched_prolong_add: dtype pair");
    return check_launch("xlbb_batched_prolong_add");
}

int xlbb_batched_prolong_add(int dtype_fine, int dtype_coarse, const XlbbBatchTransfer* tr_dev, int ninst, void* stream) {
    if (!tr_dev || ninst <= 0) return fail(XLBB_EBADARG, "xlbb_batched_prolong_add: bad argument");
    return prolong_t(dtype_fine, dtype_coarse, tr_dev, ninst, nullptr, XLBB_STREAM(stream));
}

int xlbb_batched_prolong_add_norms(int dtype_fine, int dtype_coarse, const XlbbBatchTransfer* tr_dev, int ninst,
                                   double* parts, double* norms, void* stream) {
    if (!tr_dev || ninst <= 0 || !parts || !norms)
        return fail(XLBB_EBADARG, "xlbb_batched_prolong_add_norms: bad argument");
    const int st_ = prolong_t(dtype_fine, dtype_coarse, tr_dev, ninst, parts, XLBB_STREAM(stream));
    if (st_ != XLBB_OK) return st_;
    launch_k(prolong_norms_kernel, ninst, 32, 0, XLBB_STREAM(stream), parts, ninst, norms);
    return check_launch("xlbb_batched_prolong_add_norms");
}

int xlbb_batched_prolong_add_map(int dtype_fine, int dtype_coarse, const XlbbBatchTransfer* tr_dev,
                                 const int* map_dev, int nblocks, double* parts, const int* begin_dev, int ninst,
                                 double* norms, void* stream) {
    if (!tr_dev || !map_dev || nblocks <= 0 || ((parts != nullptr) != (norms != nullptr)) ||
        (norms && (!begin_dev || ninst <= 0)))
        return fail(XLBB_EBADARG, "xlbb_batched_prolong_add_map: bad argument");
    cudaStream_t st = XLBB_STREAM(stream);
    const int2* map = reinterpret_cast<const int2*>(map_dev);
    if (dtype_fine == XLBB_F32 && dtype_coarse == XLBB_F32)
        launch_k(batched_prolong_map_kernel<float, float>, nblocks, 256, 0, st, tr_dev, map, nblocks, parts);
    else if (dtype_fine == XLBB_F32 && dtype_coarse == XLBB_F64)
        launch_k(batched_prolong_map_kernel<float, double>, nblocks, 256, 0, st, tr_dev, map, nblocks, parts);
    else if (dtype_fine == XLBB_F64 && dtype_coarse == XLBB_F64)
        launch_k(batched_prolong_map_kernel<double, double>, nblocks, 256, 0, st, tr_dev, map, nblocks, parts);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_batched_prolong_add_map: dtype pair");
    if (norms) launch_k(pair_segment_sum_kernel, ninst, 256, 0, st, (const double*)parts, nblocks, begin_dev, ninst,
                        norms);
    return check_launch("xlbb_batched_prolong_add_map");
}

int xlbb_batched_tail_smem(int dtype, int dtype_coarse, int nx, int ny, int levels) {
    if (nx < 1 || ny < 1 || levels < 1 || levels > TAIL_MAX_LEVELS || (nx >> (levels - 1)) < 1 ||
        (ny >> (levels - 1)) < 1)
        return fail(XLBB_EBADARG, "xlbb_batched_tail_smem: bad argument");
    size_t b;
    if (dtype == XLBB_F32 && dtype_coarse == XLBB_F32) b = tail_smem_bytes<float, float>(nx, ny, levels);
    else if (dtype == XLBB_F32 && dtype_coarse == XLBB_F64) b = tail_smem_bytes<float, double>(nx, ny, levels);
    else if (dtype == XLBB_F64 && dtype_coarse == XLBB_F64) b = tail_smem_bytes<double, double>(nx, ny, levels);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_batched_tail_smem: dtype pair");
    return b > (size_t)INT_MAX ? fail(XLBB_EBADARG, "xlbb_batched_tail_smem: too large") : (int)b;
}

int xlbb_batched_tail(int dtype, int dtype_coarse, const XlbbBatchTail* tails_dev, int count, int smem_bytes,
                      double gamma, int k_smooth, void* stream) {
    if (!tails_dev || count <= 0 || smem_bytes <= 0 || k_smooth < 2 || k_smooth % 2)
        return fail(XLBB_EBADARG, "xlbb_batched_tail: bad argument");
    static int optin = 0;
    if (optin == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) optin = 0;
    }
    if (smem_bytes > optin)
        return fail(XLBB_EBADARG, "xlbb_batched_tail: smem_bytes above the device's shared memory per block");
#define XLBB_TAIL(T_, TC_)                                                                                    \
    {                                                                                                         \
        static int configured = 0;                                                                            \
        auto k = batched_tail_kernel<T_, TC_>;                                                                \
        if (smem_bytes > configured) {                                                                        \
            if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes) != cudaSuccess) \
                return fail(XLBB_ELAUNCH, "xlbb_batched_tail: shared memory attribute");                      \
            configured = smem_bytes;                                                                          \
        }                                                                                                     \
        launch_k(k, count, TAIL_THREADS, (size_t)smem_bytes, XLBB_STREAM(stream), tails_dev, gamma, k_smooth,  \
                 (size_t)smem_bytes);                                                                         \
    }
    if (dtype == XLBB_F32 && dtype_coarse == XLBB_F32) XLBB_TAIL(float, float)
    else if (dtype == XLBB_F32 && dtype_coarse == XLBB_F64) XLBB_TAIL(float, double)
    else if (dtype == XLBB_F64 && dtype_coarse == XLBB_F64) XLBB_TAIL(double, double)
    else return fail(XLBB_EUNSUPPORTED, "xlbb_batched_tail: dtype pair");
#undef XLBB_TAIL
    return check_launch("xlbb_batched_tail");
}

int xlbb_batched_remove_mean_moment(int dtype, const XlbbBatchTransfer* tr_dev, const int* map_dev, int nblocks,
                                    double* parts, const int* begin_dev, int ninst, double* sums, void* stream) {
    if (!tr_dev || !map_dev || nblocks <= 0 || !parts || !begin_dev || ninst <= 0 || !sums)
        return fail(XLBB_EBADARG, "xlbb_batched_remove_mean_moment: bad argument");
    cudaStream_t st = XLBB_STREAM(stream);
    const int2* map = reinterpret_cast<const int2*>(map_dev);
    if (dtype == XLBB_F32) launch_k(batched_moment_map_kernel<float>, nblocks, 256, 0, st, tr_dev, map, nblocks, parts);
    else if (dtype == XLBB_F64)
        launch_k(batched_moment_map_kernel<double>, nblocks, 256, 0, st, tr_dev, map, nblocks, parts);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_batched_remove_mean_moment: dtype");
    launch_k(pair_segment_sum_kernel, ninst, 256, 0, st, (const double*)parts, nblocks, begin_dev, ninst, sums);
    if (dtype == XLBB_F32) launch_k(batched_shift_map_kernel<float>, nblocks, 256, 0, st, tr_dev, map, (const double*)sums);
    else launch_k(batched_shift_map_kernel<double>, nblocks, 256, 0, st, tr_dev, map, (const double*)sums);
    return check_launch("xlbb_batched_remove_mean_moment");
}

int xlbb_segment_sum(const double* parts, const int* begin_dev, int nseg, double* out, void* stream) {
    if (!parts || !begin_dev || !out || nseg <= 0) return fail(XLBB_EBADARG, "xlbb_segment_sum: bad argument");
    launch_k(segment_sum_kernel, nseg, 256, 0, XLBB_STREAM(stream), parts, begin_dev, nseg, out);
    return check_launch("xlbb_segment_sum");
}

}  // extern "C"

#include "xlbb_adjoint.cuh"
