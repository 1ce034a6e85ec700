// Three-dimensional fluid sweep: the step of src/base.py:809-846 with the BGK
// collision of src/models.py:9-34 on the D3Q19 and D3Q27 lattices, or the KBC
// collision of src/models.py:36-72 on D3Q27
// (velocity order and weights of src/lattice.py:132-182), the path of
// examples/performance/MLUPS3d.py.  One thread per cell collides and pushes
// every post-collision population to the cell it streams to (periodic wrap in
// x, y and z); PostCollision rules are applied before the push, PostStreaming
// rules through per-cell push words (as the 2D collide-and-push sweep does:
// directions a destination rebuilds from its own post-collision values are
// skipped by the pushing cell and written by the destination, whose push word
// carries the rule flag in bit 31).  Rows are (y, z) pairs, row = z ny + y.
// Included inside namespace xlbb.
#pragma once

// Velocity i of D3Q19 / D3Q27: the reference enumerates (x, y, z) over
// {0, -1, 1}^3 with x slowest; k3 is the position of velocity i in that
// 27-entry enumeration (D3Q19 leaves out the 8 corners k = 13, 14, 16, 17,
// 22, 23, 25, 26).
template <int Q>
__host__ __device__ constexpr int k3(int i) {
    return Q == 27 ? i
                   : (i <= 12 ? i : i == 13 ? 15 : i == 14 ? 18 : i == 15 ? 19 : i == 16 ? 20 : i == 17 ? 21 : 24);
}
__host__ __device__ constexpr int v3(int d) { return d == 0 ? 0 : (d == 1 ? -1 : 1); }
template <int Q>
__host__ __device__ constexpr int c3x(int i) { return v3(k3<Q>(i) / 9); }
template <int Q>
__host__ __device__ constexpr int c3y(int i) { return v3((k3<Q>(i) / 3) % 3); }
template <int Q>
__host__ __device__ constexpr int c3z(int i) { return v3(k3<Q>(i) % 3); }

// Weights by |c|^2: D3Q19 1/3, 2/36, 1/36; D3Q27 8/27, 2/27, 1/54, 1/216.
template <typename T, int Q>
__host__ __device__ constexpr T w3(int i) {
    return Q == 19
               ? ((c3x<Q>(i) * c3x<Q>(i) + c3y<Q>(i) * c3y<Q>(i) + c3z<Q>(i) * c3z<Q>(i)) == 0   ? T(1.0 / 3.0)
                  : (c3x<Q>(i) * c3x<Q>(i) + c3y<Q>(i) * c3y<Q>(i) + c3z<Q>(i) * c3z<Q>(i)) == 1 ? T(2.0 / 36.0)
                                                                                              : T(1.0 / 36.0))
               : ((c3x<Q>(i) * c3x<Q>(i) + c3y<Q>(i) * c3y<Q>(i) + c3z<Q>(i) * c3z<Q>(i)) == 0   ? T(8.0 / 27.0)
                  : (c3x<Q>(i) * c3x<Q>(i) + c3y<Q>(i) * c3y<Q>(i) + c3z<Q>(i) * c3z<Q>(i)) == 1 ? T(2.0 / 27.0)
                  : (c3x<Q>(i) * c3x<Q>(i) + c3y<Q>(i) * c3y<Q>(i) + c3z<Q>(i) * c3z<Q>(i)) == 2 ? T(1.0 / 54.0)
                                                                                              : T(1.0 / 216.0));
}

constexpr int FLUID3_THREADS = 128;    // threads per CTA (x extent of a CTA's row segment)

template <typename T, int Q>
struct Fluid3Args {
    int nx, ny, nz, pitch;
    long long plane;
    const T* f_in;
    T* f_out;
    T omega;
    RulesView<T, Q> pc, ps;
};

// Shear part of a D3Q27 non-equilibrium population per unit density
// (src/models.py:156-214): with the momentum flux Pi of fneq, N_xz = Pi_xx -
// Pi_zz and N_yz = Pi_yy - Pi_zz, the axis directions carry (2 N_xz - N_yz) / 6
// (x), (2 N_yz - N_xz) / 6 (y), -(N_xz + N_yz) / 6 (z), the face diagonals
// c_a c_b Pi_ab / 4, the rest population and the corners nothing.
template <typename T, int Q>
__device__ __forceinline__ T kbc_shear3(int i, T nxz, T nyz, T pxy, T pxz, T pyz) {
    const int ax = c3x<Q>(i) * c3x<Q>(i), ay = c3y<Q>(i) * c3y<Q>(i), az = c3z<Q>(i) * c3z<Q>(i);
    if (ax + ay + az == 1) {
        if (ax) return (T(2) * nxz - nyz) / T(6);
        if (ay) return (-nxz + T(2) * nyz) / T(6);
        return (-nxz - nyz) / T(6);
    }
    if (ax + ay + az == 2) {
        if (!az) return T(c3x<Q>(i) * c3y<Q>(i)) * (pxy / T(4));
        if (!ay) return T(c3x<Q>(i) * c3z<Q>(i)) * (pxz / T(4));
        return T(c3y<Q>(i) * c3z<Q>(i)) * (pyz / T(4));
    }
    return T(0);
}

// Rules, a warp per rule cell.  A cavity's x walls put one rule cell in a
// quarter of the warps, where it would keep its warp for Q dependent rule
// evaluations; instead the whole warp takes the rule cell's directions, one
// per lane (coalesced code and constant loads, source values read from the
// cell's shared-memory column), and shuffles move the cell's values in and
// out.  Warps with more than FLUID3_WARP_RULES rule cells are evaluated lane
// by lane (rolled loops through shared memory) where FLUID3_LANE_RULES says so.
constexpr uint32_t FLUID3_FULL = 0xffffffffu;
constexpr int FLUID3_WARP_RULES = 4;

template <typename T, int Q>
__device__ __forceinline__ T lane_value(const T (&v)[Q], int lane, int src_lane) {
    // v[lane] of lane src_lane, for every lane < Q
    T out = T(0);
#pragma unroll
    for (int j = 0; j < Q; ++j) {
        const T b = __shfl_sync(FLUID3_FULL, v[j], src_lane);
        if (lane == j) out = b;
    }
    return out;
}

template <typename T, int Q>
__device__ __forceinline__ void gather_lanes(T (&v)[Q], T val, int lane, int dst_lane) {
    // v[j] of lane dst_lane <- val of lane j, for j < Q
#pragma unroll
    for (int j = 0; j < Q; ++j) {
        const T b = __shfl_sync(FLUID3_FULL, val, j);
        if (lane == dst_lane) v[j] = b;
    }
}

// The FP32 D3Q19 BGK sweep also evaluates the warps made mostly of rule cells
// (y and z walls, lid) lane by lane, at the registers it takes without that
// path (fluid3_push19_kernel): on the 256^3 cavity 0.69 of the HBM copy
// bandwidth against 0.67.  On D3Q27 the same path cost more than it saved
// (0.59 against 0.65), so that sweep keeps the warp-per-rule-cell path only.
template <typename T, int Q, bool KBC>
constexpr bool FLUID3_LANE_RULES = sizeof(T) == 4 && Q == 19 && !KBC;

// The collision of one cell, in place: BGK (src/models.py:20-34) or KBC
// (src/models.py:47-72) with the second-order equilibrium.
template <typename T, int Q, bool KBC>
__device__ __forceinline__ void fluid3_collide(T (&f)[Q], const T om) {
    // src/base.py:748-772: rho = sum f, u = sum c f / rho (one reciprocal of rho)
    T rho = f[0], jx = T(0), jy = T(0), jz = T(0);
#pragma unroll
    for (int i = 1; i < Q; ++i) rho += f[i];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        if (c3x<Q>(i) > 0) jx += f[i]; else if (c3x<Q>(i) < 0) jx -= f[i];
        if (c3y<Q>(i) > 0) jy += f[i]; else if (c3y<Q>(i) < 0) jy -= f[i];
        if (c3z<Q>(i) > 0) jz += f[i]; else if (c3z<Q>(i) < 0) jz -= f[i];
    }
    const T irho = T(1) / rho;
    const T ux = jx * irho, uy = jy * irho, uz = jz * irho;
    const T usqr = T(1.5) * (ux * ux + uy * uy + uz * uz);
    if constexpr (!KBC) {
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const T cu = T(3) * (T(c3x<Q>(i)) * ux + T(c3y<Q>(i)) * uy + T(c3z<Q>(i)) * uz);
            const T feq = rho * w3<T, Q>(i) * (T(1) + cu * (T(1) + T(0.5) * cu) - usqr);
            f[i] = f[i] - om * (f[i] - feq);
        }
    } else {
        // src/models.py:47-72
        T fe[Q];
        T pxx = T(0), pxy = T(0), pxz = T(0), pyy = T(0), pyz = T(0), pzz = T(0);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const T cu = T(3) * (T(c3x<Q>(i)) * ux + T(c3y<Q>(i)) * uy + T(c3z<Q>(i)) * uz);
            fe[i] = rho * w3<T, Q>(i) * (T(1) + cu * (T(1) + T(0.5) * cu) - usqr);
            const T fn = f[i] - fe[i];
            if (c3x<Q>(i)) pxx += fn;
            if (c3y<Q>(i)) pyy += fn;
            if (c3z<Q>(i)) pzz += fn;
            if (c3x<Q>(i) * c3y<Q>(i) > 0) pxy += fn; else if (c3x<Q>(i) * c3y<Q>(i) < 0) pxy -= fn;
            if (c3x<Q>(i) * c3z<Q>(i) > 0) pxz += fn; else if (c3x<Q>(i) * c3z<Q>(i) < 0) pxz -= fn;
            if (c3y<Q>(i) * c3z<Q>(i) > 0) pyz += fn; else if (c3y<Q>(i) * c3z<Q>(i) < 0) pyz -= fn;
        }
        const T nxz = pxx - pzz, nyz = pyy - pzz;
        // entropic products <x, y> = sum x y / feq, one reciprocal of feq per
        // direction shared by both products
        T sh = T(0), hh = T(0);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const T dS = kbc_shear3<T, Q>(i, nxz, nyz, pxy, pxz, pyz) * rho;
            const T dH = (f[i] - fe[i]) - dS;
            const T ife = kbc_rcp<T>(fe[i]);
            sh += (dS * dH) * ife;
            hh += (dH * dH) * ife;
        }
        const T beta = om * T(0.5);
        const T ib = T(1) / beta;
        const T gamma = ib - (T(2) - ib) * sh / (T(1e-32) + hh);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const T dS = kbc_shear3<T, Q>(i, nxz, nyz, pxy, pxz, pyz) * rho;
            const T dH = (f[i] - fe[i]) - dS;
            f[i] = f[i] - beta * (T(2) * dS + gamma * dH);
        }
    }
}

template <typename T, int Q, bool KBC>
__device__ __forceinline__ void fluid3_sweep_body(const Fluid3Args<T, Q>& p) {
    static_assert(!KBC || Q == 27, "the KBC collision is defined on D3Q27");
    static_assert(Q <= 32, "a warp takes one direction per lane");
    __shared__ T stage[Q][FLUID3_THREADS];
    // post-collision values of the lane-by-lane rule path (below)
    __shared__ T post[FLUID3_LANE_RULES<T, Q, KBC> ? Q : 1][FLUID3_THREADS];
    grid_dep_wait();
    const int t = threadIdx.x, lane = t & 31, wbase = t & ~31;
    const int x = blockIdx.x * blockDim.x + t, y = blockIdx.y, z = blockIdx.z;
    // every lane stays to the end (warp-wide shuffles); lanes past the row's
    // end compute on the rest state and touch no memory
    const bool valid = x < p.nx;
    const int xs = valid ? x : p.nx - 1;
    const int row = z * p.ny + y;
    const size_t o = (size_t)row * p.pitch + xs;
    const long long P = p.plane;
    // rule lookups and push word first: independent of the populations
    const int rpc = (valid && p.pc.count > 0) ? probe_rule(load_probe(p.pc, row, xs), xs) : -1;
    const uint32_t pw = (valid && p.ps.count > 0) ? __ldg(p.ps.push + (size_t)row * p.nx + xs) : 0u;
    // f: the cell's populations, collided in place
    T f[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i] = valid ? __ldg(p.f_in + (o + (size_t)i * P)) : w3<T, Q>(i);
    if (rpc >= 0) {              // a rule cell keeps its inputs for its post-collision rules
#pragma unroll
        for (int k = 0; k < Q; ++k) stage[k][t] = f[k];
    }
    fluid3_collide<T, Q, KBC>(f, p.omega);
    // post-collision rules (source values: the step's input, staged above)
    uint32_t todo = __ballot_sync(FLUID3_FULL, rpc >= 0);
    if constexpr (FLUID3_LANE_RULES<T, Q, KBC>) {
        if (__popc(todo) > FLUID3_WARP_RULES) {     // a warp of rule cells: lane by lane, rolled loop
            if (rpc >= 0) {
#pragma unroll
                for (int k = 0; k < Q; ++k) post[k][t] = f[k];
#pragma unroll 1
                for (int d = 0; d < Q; ++d) {
                    const uint8_t code = __ldg(p.pc.code + (size_t)rpc * Q + d);
                    const int k = code < Q ? code : (code < 2 * Q ? code - Q : 0);
                    post[d][t] = rule_value<T, Q>(code, post[d][t], stage[k][t], p.pc.cst[(size_t)rpc * Q + d]);
                }
#pragma unroll
                for (int k = 0; k < Q; ++k) f[k] = post[k][t];
            }
            todo = 0;
        }
    }
    if (todo) {
        __syncwarp();
        do {
            const int l = __ffs(todo) - 1;
            todo &= todo - 1;
            const int r = __shfl_sync(FLUID3_FULL, rpc, l);
            const T cur = lane_value<T, Q>(f, lane, l);
            T val = cur;
            if (lane < Q) {
                const uint8_t code = __ldg(p.pc.code + (size_t)r * Q + lane);
                const int k = code < Q ? code : (code < 2 * Q ? code - Q : 0);
                val = rule_value<T, Q>(code, cur, stage[k][wbase + l], p.pc.cst[(size_t)r * Q + lane]);
            }
            gather_lanes<T, Q>(f, val, lane, l);
        } while (todo);
    }
    if (valid) {
        const int xm = x == 0 ? p.nx - 1 : x - 1, xp = x == p.nx - 1 ? 0 : x + 1;
        const int ym = y == 0 ? p.ny - 1 : y - 1, yp = y == p.ny - 1 ? 0 : y + 1;
        const int zm = z == 0 ? p.nz - 1 : z - 1, zp = z == p.nz - 1 ? 0 : z + 1;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int dx = c3x<Q>(i) > 0 ? xp : (c3x<Q>(i) < 0 ? xm : x);
            const int dy = c3y<Q>(i) > 0 ? yp : (c3y<Q>(i) < 0 ? ym : y);
            const int dz = c3z<Q>(i) > 0 ? zp : (c3z<Q>(i) < 0 ? zm : z);
            if (!(pw & (1u << i))) p.f_out[((size_t)(dz * p.ny + dy) * p.pitch + dx) + (size_t)i * P] = f[i];
        }
    }
    // the flagged cells' post-streaming rules, from their own post-collision values
    const bool flagged = (pw >> 31) & 1u;
    todo = __ballot_sync(FLUID3_FULL, flagged);
    if (todo) {
        const int rps = flagged ? rule_at(p.ps, row, xs) : -1;
        __syncwarp();            // the post-collision rules' reads of stage are done
        if (flagged) {
#pragma unroll
            for (int k = 0; k < Q; ++k) stage[k][t] = f[k];
        }
        __syncwarp();
        if constexpr (FLUID3_LANE_RULES<T, Q, KBC>) {
            if (__popc(todo) > FLUID3_WARP_RULES) {     // a warp of rule cells: lane by lane, rolled loop
                if (flagged) {
#pragma unroll 1
                    for (int d = 0; d < Q; ++d) {
                        const uint8_t code = __ldg(p.ps.code + (size_t)rps * Q + d);
                        if (code != 2 * Q + 1) {
                            const int k = code < Q ? code : (code < 2 * Q ? code - Q : 0);
                            p.f_out[o + (size_t)d * P] =
                                rule_value<T, Q>(code, T(0), stage[k][t], p.ps.cst[(size_t)rps * Q + d]);
                        }
                    }
                }
                todo = 0;
            }
        }
        while (todo) {
            const int l = __ffs(todo) - 1;
            todo &= todo - 1;
            const int r = __shfl_sync(FLUID3_FULL, rps, l);
            if (lane < Q) {
                const uint8_t code = __ldg(p.ps.code + (size_t)r * Q + lane);
                if (code != 2 * Q + 1) {
                    const int k = code < Q ? code : (code < 2 * Q ? code - Q : 0);
                    const size_t ol = (size_t)row * p.pitch + (blockIdx.x * blockDim.x + wbase + l);
                    p.f_out[ol + (size_t)lane * P] =
                        rule_value<T, Q>(code, T(0), stage[k][wbase + l], p.ps.cst[(size_t)r * Q + lane]);
                }
            }
        }
    }
}

template <typename T, int Q, bool KBC>
__global__ void __launch_bounds__(FLUID3_THREADS) fluid3_push_kernel(const Fluid3Args<T, Q> p) {
    fluid3_sweep_body<T, Q, KBC>(p);
}

// FP32 D3Q19 BGK, compiled for 9 CTAs per SM: the 56 registers it takes without
// the lane-by-lane rule path.  (An explicit bound on the other sweeps changed
// their code for the worse: D3Q27 at the same 72 registers 0.53 against 0.64.)
__global__ void __launch_bounds__(FLUID3_THREADS, 9) fluid3_push19_kernel(const Fluid3Args<float, 19> p) {
    fluid3_sweep_body<float, 19, false>(p);
}

// ---------------------------------------------------------------------------
// The same step as two launches: every cell without a rule in a kernel with
// no rule code at all, then the rule cells, one thread each, from the rule
// tables (a cell with both kinds of rule is taken once, by its post-collision
// rule).  The two write disjoint outputs: every output is written once, by
// the cell it streams from or by its own post-streaming rule.  The KBC sweep
// runs this way (its collision takes fewer registers without rule code: 1.56
// against 1.75 ms on the 256^3 D3Q27 cavity); for BGK the fused kernel above
// is faster (D3Q19 0.69 against 0.58, D3Q27 0.64 against 0.58 of the HBM copy
// bandwidth: the rule cells of the x walls, scattered one per row, cost the
// separate launch more than the warp-shared rule path).
// ---------------------------------------------------------------------------

template <typename T, int Q>
__device__ __forceinline__ void fluid3_push_all(const Fluid3Args<T, Q>& p, int x, int y, int z, uint32_t pw,
                                                const T (&f)[Q]) {
    const long long P = p.plane;
    const int xm = x == 0 ? p.nx - 1 : x - 1, xp = x == p.nx - 1 ? 0 : x + 1;
    const int ym = y == 0 ? p.ny - 1 : y - 1, yp = y == p.ny - 1 ? 0 : y + 1;
    const int zm = z == 0 ? p.nz - 1 : z - 1, zp = z == p.nz - 1 ? 0 : z + 1;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int dx = c3x<Q>(i) > 0 ? xp : (c3x<Q>(i) < 0 ? xm : x);
        const int dy = c3y<Q>(i) > 0 ? yp : (c3y<Q>(i) < 0 ? ym : y);
        const int dz = c3z<Q>(i) > 0 ? zp : (c3z<Q>(i) < 0 ? zm : z);
        if (!(pw & (1u << i))) p.f_out[((size_t)(dz * p.ny + dy) * p.pitch + dx) + (size_t)i * P] = f[i];
    }
}

template <typename T, int Q, bool KBC>
__global__ void __launch_bounds__(FLUID3_THREADS) fluid3_bulk_kernel(const Fluid3Args<T, Q> p) {
    grid_dep_wait();
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
    if (x >= p.nx) return;
    const int row = z * p.ny + y;
    const size_t o = (size_t)row * p.pitch + x;
    const uint32_t pw = p.ps.count > 0 ? __ldg(p.ps.push + (size_t)row * p.nx + x) : 0u;
    const bool pc_rule = p.pc.count > 0 && probe_rule(load_probe(p.pc, row, x), x) >= 0;
    T f[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i] = __ldg(p.f_in + (o + (size_t)i * p.plane));
    if (pc_rule || ((pw >> 31) & 1u)) return;     // a rule cell: fluid3_rules_kernel
    fluid3_collide<T, Q, KBC>(f, p.omega);
    fluid3_push_all<T, Q>(p, x, y, z, pw, f);
}

// Row of rule r of a CSR rule table over `rows` rows.
template <typename T, int Q>
__device__ __forceinline__ int fluid3_rule_row(const RulesView<T, Q>& rv, int r, int rows) {
    int lo = 0, hi = rows;       // the last row whose first rule is <= r
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(rv.row_ptr + mid) <= r) lo = mid; else hi = mid;
    }
    return lo;
}

template <typename T, int Q, bool KBC>
__global__ void __launch_bounds__(FLUID3_THREADS) fluid3_rules_kernel(const Fluid3Args<T, Q> p) {
    __shared__ T stage[Q][FLUID3_THREADS];
    grid_dep_wait();
    const int t = threadIdx.x;
    const int r = blockIdx.x * blockDim.x + t;
    const int npc = p.pc.count, nps = p.ps.count, rows = p.ny * p.nz;
    if (r >= npc + nps) return;
    int row, x, rpc = -1;
    if (r < npc) {
        rpc = r;
        row = fluid3_rule_row(p.pc, r, rows);
        x = __ldg(p.pc.cell_x + r);
    } else {
        const int q = r - npc;
        row = fluid3_rule_row(p.ps, q, rows);
        x = __ldg(p.ps.cell_x + q);
        if (npc > 0 && probe_rule(load_probe(p.pc, row, x), x) >= 0) return;   // taken by its post-collision rule
    }
    const int y = row % p.ny, z = row / p.ny;
    const size_t o = (size_t)row * p.pitch + x;
    const long long P = p.plane;
    const uint32_t pw = nps > 0 ? __ldg(p.ps.push + (size_t)row * p.nx + x) : 0u;
    T f[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i] = __ldg(p.f_in + (o + (size_t)i * P));
    if (rpc >= 0) {              // the inputs its post-collision rules read, indexed at run time
#pragma unroll
        for (int k = 0; k < Q; ++k) stage[k][t] = f[k];
    }
    fluid3_collide<T, Q, KBC>(f, p.omega);
    if (rpc >= 0) {
#pragma unroll
        for (int d = 0; d < Q; ++d) {
            const uint8_t code = __ldg(p.pc.code + (size_t)rpc * Q + d);
            const int k = code < Q ? code : (code < 2 * Q ? code - Q : 0);
            f[d] = rule_value<T, Q>(code, f[d], stage[k][t], p.pc.cst[(size_t)rpc * Q + d]);
        }
    }
    fluid3_push_all<T, Q>(p, x, y, z, pw, f);
    if ((pw >> 31) & 1u) {       // its post-streaming rules, from its own post-collision values
        const int rps = rule_at(p.ps, row, x);
#pragma unroll
        for (int k = 0; k < Q; ++k) stage[k][t] = f[k];
#pragma unroll
        for (int d = 0; d < Q; ++d) {
            const uint8_t code = __ldg(p.ps.code + (size_t)rps * Q + d);
            if (code != 2 * Q + 1) {
                const int k = code < Q ? code : (code < 2 * Q ? code - Q : 0);
                p.f_out[o + (size_t)d * P] = rule_value<T, Q>(code, T(0), stage[k][t], p.ps.cst[(size_t)rps * Q + d]);
            }
        }
    }
}
