// The D2Q9 advection-diffusion sweep in four-column form (launch pipeline 4
// of the Darcy family): a warp takes a 128-cell segment of one row, a lane
// four adjacent cells, every population plane (and the per-cell omega and
// source planes) moved with 16-byte loads and stores.  Streaming is arranged
// by destination: the float4 a lane stores for direction i at columns x..x+3
// of row y + cy_i holds the post-collision values of cells x - cx_i ..
// x + 3 - cx_i of row y, so along x a lane takes one value from its
// neighbour lane (warp shuffle) and the segment's first and last lanes take
// it from the cell just outside the segment, which they collide themselves
// (one extra cell per segment edge, periodic wrap at the row's ends).
// Everything else is the collide-and-push sweep's (xlbb_push.cuh): the same
// collision arithmetic per cell (DarcyPhys::collide), the same post-collision
// rules, and the same push words -- a float4 with a component that a rule
// cell rebuilds itself is stored component by component, and rule cells
// (push-word bit 16) write their rebuilt directions.  Bit-identical to the
// collide-and-push kernel.  Included inside namespace xlbb.
#pragma once

constexpr int DARCY4_ROWS = 8;          // rows (warps) per CTA

__device__ __forceinline__ float f4c(const float4& v, int j) {
    return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w));
}

__device__ __forceinline__ uint32_t u4c(const uint4& v, int j) {
    return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w));
}

// Post-collision populations of cell (y, x) from its inputs (the collision and
// post-collision rules of post_collision(), xlbb_push.cuh).
template <class Ph>
__device__ __forceinline__ void darcy4_post(const typename Ph::Args& p, int y, int x, const typename Ph::In& in,
                                            float (&fs)[9]) {
    Ph::collide(p, y, x, in, fs);
    if (p.pc.count > 0) {
        const int r = probe_rule(load_probe(p.pc, y, x), x);
        if (r >= 0) {
#pragma unroll
            for (int d = 0; d < 9; ++d) {
                const uint8_t code = __ldg(p.pc.code + (size_t)r * 9 + d);
                const int k = code < 9 ? code : (code < 18 ? code - 9 : 0);
                fs[d] = rule_value<float, 9>(code, fs[d], pick<float, 9>(in.f, k), p.pc.cst[(size_t)r * 9 + d]);
            }
        }
    }
}

// Inputs of the four cells x..x+3 of a row (16-byte loads).
struct Darcy4Loads {
    float4 f[9];
    float4 om, S;
};

template <class Ph>
__device__ __forceinline__ void darcy4_load(const typename Ph::Args& p, int o, Darcy4Loads& L) {
#pragma unroll
    for (int i = 0; i < 9; ++i) L.f[i] = __ldg(reinterpret_cast<const float4*>(p.ip[i] + o));
    L.om = p.omega_f ? __ldg(reinterpret_cast<const float4*>(p.ip[9] + o)) : make_float4(p.omega, p.omega, p.omega, p.omega);
    float4 S = make_float4(0.f, 0.f, 0.f, 0.f);
    if (p.source) S = __ldg(reinterpret_cast<const float4*>(p.ip[10] + o));
    if (p.ext) {
        const float4 e = __ldg(reinterpret_cast<const float4*>(p.ip[11] + o));
        // DarcyPhys::load: S = source + ext when both are present, else the one given
        S = p.source ? make_float4(S.x + e.x, S.y + e.y, S.z + e.z, S.w + e.w) : e;
    }
    L.S = S;
}

template <class Ph>
__device__ __forceinline__ void darcy4_in(const Darcy4Loads& L, int j, typename Ph::In& in) {
#pragma unroll
    for (int i = 0; i < 9; ++i) in.f[i] = f4c(L.f[i], j);
    in.S = f4c(L.S, j);
    in.om = f4c(L.om, j);
}

// One sweep; grid (ceil(nx / 128), ceil(ny / DARCY4_ROWS)), CTAs of 32 x DARCY4_ROWS.
// Needs nx, pitch and plane multiples of 4 and 16-byte aligned planes (darcy4_ok).
__global__ void __launch_bounds__(32 * DARCY4_ROWS) darcy_push4_kernel(const DarcyPhys<float>::Args p) {
    using Ph = DarcyPhys<float>;
    grid_dep_wait();
    const int lane = threadIdx.x;
    const int y = blockIdx.y * DARCY4_ROWS + threadIdx.y;
    if (y >= p.geom.ny) return;                       // a whole warp
    const int nx = p.geom.nx, ny = p.geom.ny, pitch = p.geom.pitch;
    const int x0 = blockIdx.x * 128;
    const int nl = min(32, (nx - x0) >> 2);           // lanes holding cells
    const bool act = lane < nl;
    const int x = x0 + 4 * (act ? lane : 0);
    const int o = y * pitch + x;
    const bool rules = p.ps.count > 0;
    // own cells: post-collision values v[j][i] of cell x + j
    float v[4][9];
    uint4 pw = make_uint4(0u, 0u, 0u, 0u);
    {
        Darcy4Loads L;
        darcy4_load<Ph>(p, o, L);
        if (rules) pw = __ldg(reinterpret_cast<const uint4*>(p.ps.push + (size_t)y * nx + x));
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            typename Ph::In in;
            darcy4_in<Ph>(L, j, in);
            darcy4_post<Ph>(p, y, x + j, in, v[j]);
        }
    }
    // the cells just outside the segment (periodic wrap): the first lane collides
    // the one on the left, the last lane the one on the right (a one-lane
    // segment both)
    float hl[9], hr[9];
    uint32_t pwl = 0u, pwr = 0u;
    if (lane == 0) {
        const int xh = x0 == 0 ? nx - 1 : x0 - 1;
        typename Ph::In in;
        Ph::load(p, y, xh, in);
        darcy4_post<Ph>(p, y, xh, in, hl);
        if (rules) pwl = __ldg(p.ps.push + (size_t)y * nx + xh);
    }
    if (lane == nl - 1) {
        const int xh = x0 + 4 * nl == nx ? 0 : x0 + 4 * nl;
        typename Ph::In in;
        Ph::load(p, y, xh, in);
        darcy4_post<Ph>(p, y, xh, in, hr);
        if (rules) pwr = __ldg(p.ps.push + (size_t)y * nx + xh);
    }
    // streaming, by destination: the float4 of direction i at columns x..x+3 of
    // row y + cy_i holds the values of cells x - cx_i .. x + 3 - cx_i
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const int yd = cy9(i) > 0 ? yp : (cy9(i) < 0 ? ym : y);
        float e[4];
        uint32_t sp[4];          // push words of the four source cells
        if (cx9(i) == 0) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                e[j] = v[j][i];
                sp[j] = u4c(pw, j);
            }
        } else if (cx9(i) > 0) {
            const float up = __shfl_up_sync(0xffffffffu, v[3][i], 1);
            const uint32_t upw = __shfl_up_sync(0xffffffffu, pw.w, 1);
            e[0] = lane == 0 ? hl[i] : up;
            sp[0] = lane == 0 ? pwl : upw;
#pragma unroll
            for (int j = 1; j < 4; ++j) {
                e[j] = v[j - 1][i];
                sp[j] = u4c(pw, j - 1);
            }
        } else {
            const float dn = __shfl_down_sync(0xffffffffu, v[0][i], 1);
            const uint32_t dpw = __shfl_down_sync(0xffffffffu, pw.x, 1);
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                e[j] = v[j + 1][i];
                sp[j] = u4c(pw, j + 1);
            }
            e[3] = lane == nl - 1 ? hr[i] : dn;
            sp[3] = lane == nl - 1 ? pwr : dpw;
        }
        if (act) {
            float* dst = p.op[i] + (yd * pitch + x);
            const uint32_t bit = 1u << i;
            if (!((sp[0] | sp[1] | sp[2] | sp[3]) & bit)) {
                *reinterpret_cast<float4*>(dst) = make_float4(e[0], e[1], e[2], e[3]);
            } else {             // a destination rebuilds this direction itself
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (!(sp[j] & bit)) dst[j] = e[j];
            }
        }
    }
    // the rule cells' post-streaming rules, from their own post-collision values
    if (rules && act) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (u4c(pw, j) & (1u << 16)) {
                const int xj = x + j;
                const int r = rule_at(p.ps, y, xj);
                const int oj = y * pitch + xj;
#pragma unroll
                for (int d = 0; d < 9; ++d) {
                    const uint8_t code = __ldg(p.ps.code + (size_t)r * 9 + d);
                    if (code != 19) {
                        const int k = code < 9 ? code : (code < 18 ? code - 9 : 0);
                        p.op[d][oj] = rule_value<float, 9>(code, 0.f, pick<float, 9>(v[j], k),
                                                           p.ps.cst[(size_t)r * 9 + d]);
                    }
                }
            }
        }
    }
}
