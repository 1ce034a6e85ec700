// Collide-and-push sweep (launch pipeline 3).
//
// One thread per cell: load the cell's inputs, collide, apply the cell's
// post-collision rules, and write every post-collision population straight to
// the cell it streams to (z = x + c_i, periodic wrap), mixed with that cell's
// input as the sweep's algebra asks.  No shared memory, no barriers, no
// recomputed rows: every input is read once and every output written once
// (each destination receives exactly one population per direction).
// Post-streaming rules need the destination cell's own post-collision values,
// which another thread computed, so a second, sparse kernel over the rule
// cells recomputes them (same device functions, same arithmetic) and rewrites
// the directions the rules replace.  Sweeps that fuse an FP64 residual or a
// divergence output use the row-marching kernels instead.
// Included inside namespace xlbb, after the physics structs.
#pragma once

// Post-collision populations of cell (y, x): load, collide, post-collision rules
// (the arithmetic of the row-marching sweep's collide stage).
template <class Phys>
__device__ __forceinline__ void post_collision(const typename Phys::Args& p, int y, int x,
                                               typename Phys::T (&fs)[Phys::Q]) {
    using T = typename Phys::T;
    constexpr int Q = Phys::Q;
    typename Phys::In in;
    Phys::load(p, y, x, in);
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

template <class Phys>
__global__ void __launch_bounds__(256) push_kernel(const typename Phys::Args p) {
    using T = typename Phys::T;
    constexpr int Q = Phys::Q;
    const SweepGeom& G = p.geom;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= G.nx) return;
    T fs[Q];
    post_collision<Phys>(p, y, x, fs);
    const int xm = x == 0 ? G.nx - 1 : x - 1, xp = x == G.nx - 1 ? 0 : x + 1;
    const int rm = (y == 0 ? G.ny - 1 : y - 1) * G.pitch, r0 = y * G.pitch;
    const int rp = (y == G.ny - 1 ? 0 : y + 1) * G.pitch;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int zx = Phys::cx(i) > 0 ? xp : (Phys::cx(i) < 0 ? xm : x);
        const int zr = Phys::cy(i) > 0 ? rp : (Phys::cy(i) < 0 ? rm : r0);
        Phys::put(p, i, zr + zx, fs[i]);
    }
}

// Post-streaming rules of every rule cell (one thread per rule cell).
template <class Phys>
__global__ void push_fixup_kernel(const typename Phys::Args p) {
    using T = typename Phys::T;
    constexpr int Q = Phys::Q;
    const SweepGeom& G = p.geom;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= p.ps.count) return;
    int lo = 0, hi = G.ny - 1;              // the row y with row_ptr[y] <= r < row_ptr[y + 1]
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(p.ps.row_ptr + mid) <= r) lo = mid; else hi = mid - 1;
    }
    const int y = lo, x = __ldg(p.ps.cell_x + r);
    T post[Q];
    post_collision<Phys>(p, y, x, post);
    const int o = y * G.pitch + x;
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        const uint8_t code = __ldg(p.ps.code + (size_t)r * Q + d);
        const T cst = p.ps.cst[(size_t)r * Q + d];
        if (code == 2 * Q + 1 && cst == T(0)) continue;   // identity: the pushed value stands
        T cur = T(0);
        if (code >= 2 * Q + 1) {                           // needs the value streamed in: recompute its source
            T nb[Q];
            post_collision<Phys>(p, wrap(y - Phys::cy(d), G.ny), wrap(x - Phys::cx(d), G.nx), nb);
            cur = pick<T, Q>(nb, d);
        }
        const int k = code < Q ? code : (code < 2 * Q ? code - Q : 0);
        Phys::put(p, d, o, rule_value<T, Q>(code, cur, pick<T, Q>(post, k), cst));
    }
}
