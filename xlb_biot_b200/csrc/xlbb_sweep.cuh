// Row-marching fused collide + stream sweep (sm_100a).
//
// A CTA owns TX consecutive output columns of a horizontal strip of rows.  It
// walks the strip row by row:  the post-collision populations of row y (the TX
// owned columns plus one halo column on each side, collided redundantly by an
// extra warp) go into a 4-slot shared-memory ring; once rows y-2..y are in the
// ring, row y-1 is streamed (pull from the ring), boundary rules are applied
// and the result is written.  The inputs of row y+D are prefetched into a
// D-deep register ring while row y is collided, so D rows of loads are in
// flight per thread; every population is read from HBM once and written once
// per sweep (plus one recomputed row at each strip end, served from L2).
// One __syncthreads per row; 4 ring slots make the ring race-free.
//
// Boundary rules are found without searching: a per-row bitmask word (one bit
// per cell) and the global index of the first rule in that word are loaded
// with the populations; the rule index is base + popc(mask below the bit).
#pragma once
#include "xlbb_common.cuh"

namespace xlbb {

struct SweepGeom {
    int nx, ny, pitch;
    long long plane;
};

// Rule lookup data of one cell, loaded D rows ahead.
struct RuleProbe {
    uint32_t mask;
    int base;
};

template <typename T, int Q>
__device__ __forceinline__ RuleProbe load_probe(const RulesView<T, Q>& r, int y, int x) {
    RuleProbe p{0u, 0};
    if (r.count > 0) {
        const size_t w = (size_t)y * r.words_per_row + (x >> 5);
        p.mask = __ldg(r.mask + w);
        p.base = __ldg(r.word_base + w);
    }
    return p;
}

__device__ __forceinline__ int probe_rule(const RuleProbe& p, int x) {
    const uint32_t bit = 1u << (x & 31);
    return (p.mask & bit) ? p.base + __popc(p.mask & (bit - 1u)) : -1;
}

// Phys must provide: T, Q, cx(i), cy(i), struct In, load(p, y, x, In&),
// collide(p, y, x, const In&, T (&fs)[Q]), fin(const In&, T (&g)[Q]) (the
// pre-collision input seen by post-collision rules), f_in(const In&, i) (the
// sweep input used by the mixing / difference terms) and store<PREV>(...).
template <class Phys, int TX, int D, bool PREV>
__global__ void __launch_bounds__(TX + 32) sweep_kernel(const typename Phys::Args p) {
    using T = typename Phys::T;
    constexpr int Q = Phys::Q;
    constexpr int NT = TX + 2;  // owned columns + 2 halo columns
    __shared__ T post[4][Q][NT];
    __shared__ double red[(TX + 32) / 32];

    const SweepGeom& G = p.geom;
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * TX;
    const int w = min(TX, G.nx - x0);
    // Thread -> ring column.  Threads [0, TX) own columns x0+tid (ring col tid+1);
    // the extra warp's lanes 0/1 collide the left/right halo columns.
    int rc, xg;
    bool active;
    if (tid < TX) {
        rc = tid + 1; xg = x0 + tid; active = tid < w;
    } else if (tid == TX) {
        rc = 0; xg = x0 - 1; active = true;
    } else if (tid == TX + 1) {
        rc = w + 1; xg = x0 + w; active = true;
    } else {
        rc = 0; xg = 0; active = false;
    }
    const bool owner = tid < w;
    const int xw = wrap(xg, G.nx);
    const int ys = (int)(((long long)blockIdx.y * G.ny) / gridDim.y);
    const int ye = (int)(((long long)(blockIdx.y + 1) * G.ny) / gridDim.y);

    typename Phys::In pf[D];      // register ring of prefetched rows
    RuleProbe pcp[D], psp[D];
    T fprev[PREV ? Q : 1];
    RuleProbe ps_prev{0u, 0};
    double acc = 0.0;
#pragma unroll
    for (int u = 0; u < D; ++u) {
        const int yy = ys - 1 + u;
        if (active && yy <= ye) {
            const int y = wrap(yy, G.ny);
            Phys::load(p, y, xw, pf[u]);
            pcp[u] = load_probe(p.pc, y, xw);
            psp[u] = load_probe(p.ps, y, xw);
        }
    }
    for (int base = ys - 1; base <= ye; base += D) {
#pragma unroll
        for (int u = 0; u < D; ++u) {
            const int yy = base + u;
            if (yy <= ye) {   // uniform over the block
                const int slot = (yy + 4) & 3;
                const int yc = wrap(yy, G.ny);
                const typename Phys::In cur = pf[u];
                const RuleProbe pcc = pcp[u], psc = psp[u];
                if (active && yy + D <= ye) {
                    const int yn = wrap(yy + D, G.ny);
                    Phys::load(p, yn, xw, pf[u]);
                    pcp[u] = load_probe(p.pc, yn, xw);
                    psp[u] = load_probe(p.ps, yn, xw);
                }
                if (active) {
                    T fs[Q];
                    Phys::collide(p, yc, xw, cur, fs);
                    const int r = probe_rule(pcc, xw);
                    if (r >= 0) {
                        T g[Q];
                        Phys::fin(cur, g);
#pragma unroll
                        for (int d = 0; d < Q; ++d) {
                            const uint8_t code = __ldg(p.pc.code + (size_t)r * Q + d);
                            const int k = code < Q ? code : (code < 2 * Q ? code - Q : 0);
                            fs[d] = rule_value<T, Q>(code, fs[d], pick<T, Q>(g, k), p.pc.cst[(size_t)r * Q + d]);
                        }
                    }
#pragma unroll
                    for (int i = 0; i < Q; ++i) post[slot][i][rc] = fs[i];
                }
                __syncthreads();
                if (owner && yy - 1 >= ys) {
                    const int yo = yy - 1;
                    const int so = (yo + 4) & 3;
                    T S[Q];
#pragma unroll
                    for (int i = 0; i < Q; ++i) S[i] = post[(yo - Phys::cy(i) + 4) & 3][i][rc - Phys::cx(i)];
                    const int r = probe_rule(ps_prev, xg);
                    if (r >= 0) {
#pragma unroll
                        for (int d = 0; d < Q; ++d) {
                            const uint8_t code = __ldg(p.ps.code + (size_t)r * Q + d);
                            const int k = code < Q ? code : (code < 2 * Q ? code - Q : 0);
                            S[d] = rule_value<T, Q>(code, S[d], post[so][k][rc], p.ps.cst[(size_t)r * Q + d]);
                        }
                    }
                    acc += Phys::template store<PREV>(p, yo, xg, S, fprev);
                }
                if (PREV) {
#pragma unroll
                    for (int i = 0; i < Q; ++i) fprev[i] = Phys::f_in(cur, i);
                }
                ps_prev = psc;
            }
        }
    }
    if (p.sumsq != nullptr) {
        const double s = block_sum(acc, red);
        if (tid == 0) p.sumsq[blockIdx.y * gridDim.x + blockIdx.x] = s;
    }
}

}  // namespace xlbb
