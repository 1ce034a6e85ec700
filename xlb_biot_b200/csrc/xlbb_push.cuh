// Collide-and-push sweep (launch pipeline 3).
//
// One thread per cell: load the cell's inputs, collide, apply the cell's
// post-collision rules, and write every post-collision population straight to
// the cell it streams to (z = x + c_i, periodic wrap), mixed with that cell's
// input as the sweep's algebra asks.  No shared memory, no barriers, no
// recomputed rows: every input is read once and every output written once.
// Post-streaming rules are resolved in the same kernel: a direction d that
// the destination's rule rebuilds from the destination's own post-collision
// values (source or zero codes) is written by the destination cell's thread,
// which has those values, and skipped by the pushing thread (a per-cell push
// word, built with the rule table, says which); rule tables whose "keep"
// codes transform the pushed value have no push word and use the row-marching
// sweep.  Each output is written exactly once, with the arithmetic of the
// row-marching sweep.  The fused FP64 sums of squares are the writers' sums
// (one partial per block); only the divergence side output needs the
// row-marching kernels.
// Included inside namespace xlbb, after the physics structs.
#pragma once

// Rule index of cell (zx, zy) in a bitmask-indexed rule table, or -1.
template <typename T, int Q>
__device__ __forceinline__ int rule_at(const RulesView<T, Q>& r, int zy, int zx) {
    const int w = zy * r.words_per_row + (zx >> 5);
    const uint32_t m = __ldg(r.mask + w);
    const uint32_t bit = 1u << (zx & 31);
    if (!(m & bit)) return -1;
    return __ldg(r.word_base + w) + __popc(m & (bit - 1u));
}

// Post-collision populations of cell (y, x): load, collide, post-collision rules
// (the arithmetic of the row-marching sweep's collide stage).
// (adj: a change of the loaded inputs before the collision, e.g. a force
// computed in the same kernel; the default changes nothing)
struct NoAdjust {
    template <class In>
    __device__ void operator()(In&) const {}
};

template <class Phys, class Adj = NoAdjust>
__device__ __forceinline__ void post_collision(const typename Phys::Args& p, int y, int x,
                                               typename Phys::T (&fs)[Phys::Q], const Adj& adj = Adj()) {
    using T = typename Phys::T;
    constexpr int Q = Phys::Q;
    typename Phys::In in;
    Phys::load(p, y, x, in);
    adj(in);
    Phys::collide(p, y, x, in, fs);
    if (p.pc.count > 0) {
        const int r = probe_rule(load_probe(p.pc, y, x), x);
        if (r >= 0) {
            T g[Q];
            Phys::fin(in, g);
#pragma unroll
            for (int d = 0; d < Q; ++d) {
                const uint8_t code = __ldg(p.pc.code + (size_t)r * Q + d);
                const int k = code < Q ? code : (code < 2 * Q ? code - Q : 0);
                fs[d] = rule_value<T, Q>(code, fs[d], pick<T, Q>(g, k), p.pc.cst[(size_t)r * Q + d]);
            }
        }
    }
}

// One cell of the collide-and-push sweep; returns the FP64 squares of the
// values it wrote (the sweep's fused sum: every output is written exactly once,
// so the writers' sums add up to the sum over all outputs).
template <class Phys, bool SUMSQ, class Adj = NoAdjust>
__device__ __forceinline__ double push_cell(const typename Phys::Args& p, int y, int x, const Adj& adj = Adj()) {
    using T = typename Phys::T;
    constexpr int Q = Phys::Q;
    const SweepGeom& G = p.geom;
    T fs[Q];
    post_collision<Phys>(p, y, x, fs, adj);
    const int ym = y == 0 ? G.ny - 1 : y - 1, yp = y == G.ny - 1 ? 0 : y + 1;
    const int xm = x == 0 ? G.nx - 1 : x - 1, xp = x == G.nx - 1 ? 0 : x + 1;
    // the cell's push word: directions rebuilt at their destination, own rules
    const uint32_t pw = p.ps.count > 0 ? __ldg(p.ps.push + y * G.nx + x) : 0u;
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int zx = Phys::cx(i) > 0 ? xp : (Phys::cx(i) < 0 ? xm : x);
        const int zy = Phys::cy(i) > 0 ? yp : (Phys::cy(i) < 0 ? ym : y);
        if (!(pw & (1u << i))) acc += Phys::template put<SUMSQ>(p, i, zy * G.pitch + zx, zx, zy, fs[i]);
    }
    if (pw & (1u << 16)) {       // this cell's post-streaming rules, from its own post-collision values
        const int r = rule_at(p.ps, y, x);
        const int o = y * G.pitch + x;
#pragma unroll
        for (int d = 0; d < Q; ++d) {
            const uint8_t code = __ldg(p.ps.code + (size_t)r * Q + d);
            if (code != 2 * Q + 1) {
                const int k = code < Q ? code : (code < 2 * Q ? code - Q : 0);
                acc += Phys::template put<SUMSQ>(p, d, o, x, y,
                                 rule_value<T, Q>(code, T(0), pick<T, Q>(fs, k), p.ps.cst[(size_t)r * Q + d]));
            }
        }
    }
    return acc;
}

template <class Phys, bool SUMSQ>
__global__ void __launch_bounds__(256) push_kernel(const typename Phys::Args p) {
    grid_dep_wait();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if constexpr (SUMSQ) {        // one FP64 partial per block
        __shared__ double red[8];
        const double acc = x < p.geom.nx ? push_cell<Phys, true>(p, y, x) : 0.0;
        const double s = block_sum(acc, red);
        if (threadIdx.x == 0) p.sumsq[blockIdx.y * gridDim.x + blockIdx.x] = s;
    } else {
        if (x < p.geom.nx) push_cell<Phys, false>(p, y, x);
    }
}
