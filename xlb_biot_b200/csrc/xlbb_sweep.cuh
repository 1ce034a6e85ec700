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
        const int w = y * r.words_per_row + (x >> 5);
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
// One CTA's strip: owned columns [x0, x0+TX) of rows [ys, ye) of the grid in
// ``p``.  Returns this thread's contribution to the FP64 sum of the strip.
// ``post`` is the CTA's 4-slot ring; callers synchronise before reusing it.
template <class Phys, int TX, int D, bool PREV>
__device__ __forceinline__ double sweep_strip(const typename Phys::Args& p, int x0, int ys, int ye,
                                              typename Phys::T (*post)[Phys::Q][TX + 2]) {
    using T = typename Phys::T;
    constexpr int Q = Phys::Q;
    const SweepGeom& G = p.geom;
    const int tid = threadIdx.x;
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
    return acc;
}

template <class Phys, int TX, int D, bool PREV>
__global__ void __launch_bounds__(TX + 32) sweep_kernel(const typename Phys::Args p) {
    grid_dep_wait();
    using T = typename Phys::T;
    constexpr int Q = Phys::Q;
    __shared__ T post[4][Q][TX + 2];
    __shared__ double red[(TX + 32) / 32];
    const int ys = (int)(((long long)blockIdx.y * p.geom.ny) / gridDim.y);
    const int ye = (int)(((long long)(blockIdx.y + 1) * p.geom.ny) / gridDim.y);
    const double acc = sweep_strip<Phys, TX, D, PREV>(p, blockIdx.x * TX, ys, ye, post);
    if (p.sumsq != nullptr) {
        const double s = block_sum(acc, red);
        if (threadIdx.x == 0) p.sumsq[blockIdx.y * gridDim.x + blockIdx.x] = s;
    }
}

}  // namespace xlbb

namespace xlbb {

// Status word of the bounded waits (0 = fine); read with xlbb_device_status().
__device__ int g_xlbb_status = 0;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Records a device error in g_xlbb_status unless an earlier one is there
// (the first error of a run is the one reported).
__device__ __forceinline__ void note_status(int code) { atomicCAS(&g_xlbb_status, 0, code); }

// Bounded wait on an mbarrier phase: gives up after `limit` polls (by default
// ~2^22, seconds), records XLBB_ETIMEOUT in g_xlbb_status and returns false;
// the caller runs on to its end.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = 1u << 22) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    note_status(-3);
    return false;
}

// 1D bulk copy global -> shared completing on an mbarrier (no multicast).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Dynamic shared memory of sweep_bulk_kernel.
template <typename T, int Q, int TX, int D>
__host__ __device__ constexpr size_t bulk_smem_bytes(int np) {
    return 128 + sizeof(T) * (size_t)(4 * Q * (TX + 2)) + sizeof(T) * (size_t)D * np * (TX + 4);
}

// Same sweep as sweep_kernel, but the inputs of row y+D are brought into a
// D-stage shared-memory ring by bulk copies (one per input plane, issued by one
// thread, completing on the stage's mbarrier) instead of register prefetch;
// the two halo cells use per-thread cp.async.  Loads in flight no longer cost
// registers, so deeper rings fit.  Requires 16-byte aligned planes and pitch.
template <class Phys, int TX, int D, bool PREV>
__global__ void __launch_bounds__(TX + 32) sweep_bulk_kernel(const typename Phys::Args p) {
    grid_dep_wait();
    using T = typename Phys::T;
    constexpr int Q = Phys::Q;
    constexpr int NT = TX + 2;
    constexpr int RS = TX + 4;            // raw ring row stride (16-byte multiple)
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
    T(*post)[Q][NT] = reinterpret_cast<T(*)[Q][NT]>(smem + 128);
    T* raw = reinterpret_cast<T*>(smem + 128 + sizeof(T) * 4 * Q * NT);
    __shared__ double red[(TX + 32) / 32];

    const SweepGeom& G = p.geom;
    const int np = p.np;
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * TX;
    const int w = min(TX, G.nx - x0);
    constexpr int VEC = 16 / sizeof(T);
    const uint32_t seg_bytes = (uint32_t)(((w + VEC - 1) / VEC) * VEC * sizeof(T));
    int rc, xg, col;
    bool active, halo;
    if (tid < TX) {
        rc = tid + 1; xg = x0 + tid; active = tid < w; col = tid; halo = false;
    } else if (tid == TX) {
        rc = 0; xg = x0 - 1; active = true; col = TX; halo = true;
    } else if (tid == TX + 1) {
        rc = w + 1; xg = x0 + w; active = true; col = TX + 1; halo = true;
    } else {
        rc = 0; xg = 0; active = false; col = 0; halo = false;
    }
    const bool owner = tid < w;
    const int xw = wrap(xg, G.nx);
    const int ys = (int)(((long long)blockIdx.y * G.ny) / gridDim.y);
    const int ye = (int)(((long long)(blockIdx.y + 1) * G.ny) / gridDim.y);
    const int r0 = ys - 1;

    // issue the loads of row `yy` into stage `s`
    auto issue = [&](int yy, int s) {
        const int y = wrap(yy, G.ny);
        T* dst = raw + (size_t)s * np * RS;
        if (tid == 0) {
            mbar_expect_tx(&bars[s], seg_bytes * (uint32_t)np);
            for (int k = 0; k < np; ++k)
                bulk_g2s(dst + (size_t)k * RS, p.planes[k] + (size_t)y * G.pitch + x0, seg_bytes, &bars[s]);
        }
        if (halo) {
            for (int k = 0; k < np; ++k)
                cp_async_elem<sizeof(T)>(dst + (size_t)k * RS + col, p.planes[k] + (size_t)y * G.pitch + xw);
        }
        if (halo) cp_async_commit();
    };

    if (tid == 0) {
        for (int s = 0; s < D; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    RuleProbe pcp[D], psp[D];
#pragma unroll
    for (int u = 0; u < D; ++u) {
        const int yy = r0 + u;
        if (yy <= ye) {
            issue(yy, u);
            if (active) {
                const int y = wrap(yy, G.ny);
                pcp[u] = load_probe(p.pc, y, xw);
                psp[u] = load_probe(p.ps, y, xw);
            }
        } else if (halo) {
            cp_async_commit();
        }
    }
    T fprev[PREV ? Q : 1];
    RuleProbe ps_prev{0u, 0};
    double acc = 0.0;
    for (int base = r0; base <= ye; base += D) {
#pragma unroll
        for (int u = 0; u < D; ++u) {
            const int yy = base + u;
            if (yy <= ye) {
                const int slot = (yy + 4) & 3;
                const int yc = wrap(yy, G.ny);
                const uint32_t parity = (uint32_t)(((yy - r0) / D) & 1);
                mbar_wait(&bars[u], parity);
                if (halo) cp_async_wait<D - 1>();
                typename Phys::In cur;
                const RuleProbe pcc = pcp[u], psc = psp[u];
                if (active) {
                    Phys::from_smem(p, raw + (size_t)u * np * RS, RS, col, cur);
                    if (yy + D <= ye) {
                        const int yn = wrap(yy + D, G.ny);
                        pcp[u] = load_probe(p.pc, yn, xw);
                        psp[u] = load_probe(p.ps, yn, xw);
                    }
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
                __syncthreads();   // ring slot consumed by everyone; post row visible
                if (yy + D <= ye) {
                    if (tid == 0) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    issue(yy + D, u);
                } else if (halo) {
                    cp_async_commit();
                }
                if (owner && yy - 1 >= ys) {
                    const int yo = yy - 1;
                    const int so = (yo + 4) & 3;
                    T S[Q];
#pragma unroll
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
                if (PREV && active) {
#pragma unroll
                    for (int i = 0; i < Q; ++i) fprev[i] = Phys::f_in(cur, i);
                }
                ps_prev = psc;
            }
        }
    }
    if (halo) cp_async_wait<0>();
    if (p.sumsq != nullptr) {
        const double s = block_sum(acc, red);
        if (tid == 0) p.sumsq[blockIdx.y * gridDim.x + blockIdx.x] = s;
    }
}

}  // namespace xlbb

namespace xlbb {

// Independent-warp sweep: each warp owns 30 output columns (lanes 1..30; lanes
// 0 and 31 collide the halo columns) of a strip of rows and keeps the last
// three post-collision rows in registers.  Streaming pulls x-neighbours with
// warp shuffles and y-neighbours from the register rows, so there is no
// shared memory and no block barrier; the inputs of row y+D are prefetched
// into a register ring.  Warps of one CTA are unrelated (different column
// blocks / strips).
template <class Phys, int D, bool PREV>
__global__ void __launch_bounds__(128) sweep_warp_kernel(const typename Phys::Args p, int nbx, int nstrips) {
    grid_dep_wait();
    using T = typename Phys::T;
    constexpr int Q = Phys::Q;
    constexpr int W = 30;
    __shared__ double red[4];
    const SweepGeom& G = p.geom;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int wg = blockIdx.x * 4 + wib;
    const bool live = wg < nbx * nstrips;           // warp-uniform
    const int cb = live ? wg % nbx : 0;
    const int sb = live ? wg / nbx : 0;
    const int x0 = cb * W;
    const int w = min(W, G.nx - x0);
    const int xg = x0 - 1 + lane;
    const bool active = live && lane <= w + 1;
    const bool owner = live && lane >= 1 && lane <= w;
    const int xw = wrap(xg, G.nx);
    const int ys = (int)(((long long)sb * G.ny) / nstrips);
    const int ye = live ? (int)(((long long)(sb + 1) * G.ny) / nstrips) : ys - 2;

    typename Phys::In pf[D];
    RuleProbe pcp[D], psp[D];
    T P0[Q], P1[Q], P2[Q];      // post-collision rows yy-2, yy-1, yy
    T fprev[PREV ? Q : 1];
    RuleProbe ps_prev{0u, 0};
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < Q; ++i) { P0[i] = T(0); P1[i] = T(0); P2[i] = T(0); }
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
            if (yy <= ye) {   // warp-uniform
                const int yc = wrap(yy, G.ny);
                const typename Phys::In cur = pf[u];
                const RuleProbe pcc = pcp[u], psc = psp[u];
                if (active && yy + D <= ye) {
                    const int yn = wrap(yy + D, G.ny);
                    Phys::load(p, yn, xw, pf[u]);
                    pcp[u] = load_probe(p.pc, yn, xw);
                    psp[u] = load_probe(p.ps, yn, xw);
                }
#pragma unroll
                for (int i = 0; i < Q; ++i) { P0[i] = P1[i]; P1[i] = P2[i]; }
                if (active) {
                    Phys::collide(p, yc, xw, cur, P2);
                    const int r = probe_rule(pcc, xw);
                    if (r >= 0) {
                        T g[Q];
                        Phys::fin(cur, g);
#pragma unroll
                        for (int d = 0; d < Q; ++d) {
                            const uint8_t code = __ldg(p.pc.code + (size_t)r * Q + d);
                            const int k = code < Q ? code : (code < 2 * Q ? code - Q : 0);
                            P2[d] = rule_value<T, Q>(code, P2[d], pick<T, Q>(g, k), p.pc.cst[(size_t)r * Q + d]);
                        }
                    }
                }
                if (yy - 1 >= ys) {   // warp-uniform: stream row yo = yy-1
                    const int yo = yy - 1;
                    T S[Q];
#pragma unroll
                    for (int i = 0; i < Q; ++i) {
                        const T v = Phys::cy(i) > 0 ? P0[i] : (Phys::cy(i) < 0 ? P2[i] : P1[i]);
                        S[i] = Phys::cx(i) == 0 ? v : __shfl_sync(0xffffffffu, v, (lane - Phys::cx(i)) & 31);
                    }
                    if (owner) {
                        const int r = probe_rule(ps_prev, xg);
                        if (r >= 0) {
#pragma unroll
                            for (int d = 0; d < Q; ++d) {
                                const uint8_t code = __ldg(p.ps.code + (size_t)r * Q + d);
                                const int k = code < Q ? code : (code < 2 * Q ? code - Q : 0);
                                S[d] = rule_value<T, Q>(code, S[d], pick<T, Q>(P1, k), p.ps.cst[(size_t)r * Q + d]);
                            }
                        }
                        acc += Phys::template store<PREV>(p, yo, xg, S, fprev);
                    }
                }
                if (PREV && active) {
#pragma unroll
                    for (int i = 0; i < Q; ++i) fprev[i] = Phys::f_in(cur, i);
                }
                ps_prev = psc;
            }
        }
    }
    if (p.sumsq != nullptr) {
        // one partial per warp slot: sumsq[blockIdx.x * 4 + warp]
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) red[wib] = acc;
        __syncthreads();
        if (threadIdx.x == 0) p.sumsq[blockIdx.x] = red[0] + red[1] + red[2] + red[3];
    }
}

}  // namespace xlbb
