// Hand-written adjoints (transposes) of the sweeps and stencils of the Biot
// step, for gradients of a misfit with respect to per-cell material fields.
//
// Every forward kernel is affine in the populations for fixed material, so its
// adjoint is the transposed linear map:
//   sweep:    out = a f + b PS(stream(PC(C g + B F, g)), post),  g = f - resid
//   adjoint:  pull lam_out from the cells the populations streamed to
//             (z = y + c_i), undo the post-streaming rules (a rule that
//             overwrote a direction passes nothing back through the stream;
//             a rule that copied another direction of the same cell passes its
//             adjoint to that direction), undo the post-collision rules, and
//             apply C^T per cell.
// The parameter gradients (lambda, mu of the collision; omega of the Darcy
// BGK) accumulate in FP64 per cell from the forward sweep's inputs.
// One thread per cell; gathers read every adjoint value exactly once.
#pragma once

namespace xlbb {

// Factor the adjoint of a post-streaming (or gradient) rule passes back
// through the stream for direction d: 1 without a rule, +-1 for the "keep"
// codes, 0 when the rule replaced the value.
template <typename T, int Q>
__device__ __forceinline__ T rule_keep_factor(const RulesView<T, Q>& r, int y, int x, int d) {
    const int k = find_rule(r, y, x);
    if (k < 0) return T(1);
    const uint8_t code = __ldg(r.code + (size_t)k * Q + d);
    if (code == 2 * Q + 1) return T(1);
    if (code == 2 * Q + 2) return T(-1);
    return T(0);
}

// Factor the adjoint of rule table r passes back through the stream from
// (zy, zx) for direction d of the cell at (y, x) = (zy, zx) - c_d: with the
// table's push words (word of the source cell, bit d set when the value was
// rebuilt at the destination) one coalesced load per cell, else a search.
template <typename T, int Q>
__device__ __forceinline__ T gather_factor(const RulesView<T, Q>& r, uint32_t pw, int zy, int zx, int d) {
    if (r.count == 0) return T(1);
    if (r.push) return (pw >> d) & 1u ? T(0) : T(1);
    return rule_keep_factor<T, Q>(r, zy, zx, d);
}

// Rule index of the cell itself (bitmask probe with push words' bit 16 as a
// first filter).
template <typename T, int Q>
__device__ __forceinline__ int own_rule(const RulesView<T, Q>& r, uint32_t pw, int y, int x) {
    if (r.count == 0) return -1;
    if (r.push && !((pw >> 16) & 1u)) return -1;
    return probe_rule(load_probe(r, y, x), x);
}

// Adjoint of the rules of one cell applied to v (in place): the adjoint that
// flows to the rules' source directions is added to src[].
template <typename T, int Q>
__device__ __forceinline__ void rules_transpose(const RulesView<T, Q>& r, int rule, T (&v)[Q], T (&src)[Q]) {
    if (rule < 0) return;
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        const uint8_t code = __ldg(r.code + (size_t)rule * Q + d);
        if (code == 2 * Q + 1) continue;
        if (code == 2 * Q + 2) { v[d] = -v[d]; continue; }
        if (code < 2 * Q) {
            const int k = code < Q ? code : code - Q;
            const T s = code < Q ? v[d] : -v[d];
#pragma unroll
            for (int j = 0; j < Q; ++j)
                if (j == k) src[j] += s;
        }
        v[d] = T(0);
    }
}

template <typename T>
struct ElastAdjArgs {
    SweepGeom geom;
    const T* lam_out;
    T* lam_f;
    T* lam_resid;
    T* lam_force;
    double* g_lam;
    double* g_mu;
    const T* f_in;
    const T* resid;
    const T* force;
    const T* fext;
    T a, b;
    ElastMat<T> mat;
    T lam_u, mu_u;
    RulesView<T, 8> pc, ps;
};

template <typename T>
__global__ void elast_sweep_adjoint_kernel(const ElastAdjArgs<T> p) {
    grid_dep_wait();
    const SweepGeom& G = p.geom;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= G.nx) return;
    const size_t o = (size_t)y * G.pitch + x;
    const long long P = G.plane;
    // adjoint of the post-collision populations of this cell
    const uint32_t pw = p.ps.count > 0 && p.ps.push ? __ldg(p.ps.push + y * G.nx + x) : 0u;
    T lp[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int zx = wrap(x + cx8(i), G.nx), zy = wrap(y + cy8(i), G.ny);
        const T v = __ldg(p.lam_out + (size_t)zy * G.pitch + zx + i * P);
        lp[i] = p.b * (v * gather_factor<T, 8>(p.ps, pw, zy, zx, i));
    }
    T lo[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) lo[i] = __ldg(p.lam_out + o + i * P);
    if (p.ps.count > 0) {
        const int r = own_rule<T, 8>(p.ps, pw, y, x);
        if (r >= 0) {   // post-streaming rules of this cell read its own post-collision values
            T v[8], add[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) { v[i] = p.b * lo[i]; add[i] = T(0); }
            rules_transpose<T, 8>(p.ps, r, v, add);
#pragma unroll
            for (int i = 0; i < 8; ++i) lp[i] += add[i];
        }
    }
    // post-collision rules: lp -> adjoint of the collision output, lge -> adjoint of g
    T lge[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) lge[i] = T(0);
    if (p.pc.count > 0) rules_transpose<T, 8>(p.pc, probe_rule(load_probe(p.pc, y, x), x), lp, lge);
    // rates of this cell
    T lam = p.lam_u, mu = p.mu_u;
    T cs = p.mat.cs, cd = p.mat.cd, h = p.mat.h, n = p.mat.n;
    if (p.mat.mu_f) {
        lam = __ldg(p.mat.lam_f + o);
        mu = __ldg(p.mat.mu_f + o);
        elast_rates<T>(lam, mu, cs, cd, h, n);
    }
    const T A = lp[0] + lp[1] + lp[2] + lp[3], B = lp[4] + lp[5] + lp[6] + lp[7];
    const T lM0 = T(0.5) * (lp[0] - lp[2]), lM1 = T(0.5) * (lp[1] - lp[3]);
    const T lM2 = h * A + n * B;
    const T lM3 = T(0.25) * (lp[0] - lp[1] + lp[2] - lp[3]);
    const T lM4 = T(0.25) * (lp[4] - lp[5] + lp[6] - lp[7]);
    const T lM5 = T(-0.5) * lp[0] + T(0.5) * lp[2] + T(0.25) * (lp[4] - lp[5] - lp[6] + lp[7]);
    const T lM6 = T(-0.5) * lp[1] + T(0.5) * lp[3] + T(0.25) * (lp[4] + lp[5] - lp[6] - lp[7]);
    const T lm0 = lM0 + T(1.0 / 3.0) * lM5, lm1 = lM1 + T(1.0 / 3.0) * lM6;   // transposes of the collision's thirds
    const T lm2 = cs * lM2, lm3 = cd * lM3, lm4 = cd * lM4;
    T lg[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const T w2 = i < 4 ? T(1) : T(2);
        const T c3 = i < 4 ? ((i & 1) ? T(-1) : T(1)) : T(0);
        const T c4 = i < 4 ? T(0) : ((i & 1) ? T(-1) : T(1));
        lg[i] = T(cx8(i)) * lm0 + T(cy8(i)) * lm1 + w2 * lm2 + c3 * lm3 + c4 * lm4 + lge[i];
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) p.lam_f[o + i * P] = p.a * lo[i] + lg[i];
    if (p.lam_resid) {
#pragma unroll
        for (int i = 0; i < 8; ++i) p.lam_resid[o + i * P] = p.lam_resid[o + i * P] - lg[i];
    }
    // the collision with F absent is the same map as with F = 0: the adjoint
    // of the force is defined either way
    if (p.lam_force) {
        p.lam_force[o] = lM0 + T(1.0 / 6.0) * lM5;
        p.lam_force[o + P] = lM1 + T(1.0 / 6.0) * lM6;
    }
    if (p.g_mu) {
        // moments of the forward sweep's pre-collision input g = f - resid
        T g[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            g[i] = __ldg(p.f_in + o + i * P);
            if (p.resid) g[i] -= __ldg(p.resid + o + i * P);
        }
        const double m2 = (double)(g[0] + g[1] + g[2] + g[3] + T(2) * (g[4] + g[5] + g[6] + g[7]));
        const double m3 = (double)(g[0] - g[1] + g[2] - g[3]);
        const double m4 = (double)(g[4] - g[5] + g[6] - g[7]);
        const double s = (double)lam + (double)mu;
        const double dcs = 6.0 / ((3.0 * s + 1.0) * (3.0 * s + 1.0));
        const double dcd = 12.0 / ((6.0 * (double)mu + 1.0) * (6.0 * (double)mu + 1.0));
        const double graw = 1.0 / (12.0 * s - 4.0);
        const double dg = (graw > 100.0 || graw < -100.0) ? 0.0 : -12.0 * graw * graw;
        const double M2 = m2 * (double)cs;
        const double dJ_ds = (double)A * (0.5 * dg * M2 + (double)h * m2 * dcs) +
                             (double)B * (-0.25 * dg * M2 + (double)n * m2 * dcs);
        const double dJ_dcd = (double)lM3 * m3 + (double)lM4 * m4;
        p.g_lam[o] += dJ_ds;
        p.g_mu[o] += dJ_ds + dJ_dcd * dcd;
    }
}

template <typename T>
struct DarcyAdjArgs {
    SweepGeom geom;
    const T* lam_out;
    T* lam_f;
    T* lam_source;
    double* g_omega;
    const T* f_in;
    T omega;
    const T* omega_f;
    const T* source;
    const T* ext;
    RulesView<T, 9> pc, ps;
};

template <typename T>
__global__ void darcy_sweep_adjoint_kernel(const DarcyAdjArgs<T> p) {
    grid_dep_wait();
    const SweepGeom& G = p.geom;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= G.nx) return;
    const size_t o = (size_t)y * G.pitch + x;
    const long long P = G.plane;
    const uint32_t pw = p.ps.count > 0 && p.ps.push ? __ldg(p.ps.push + y * G.nx + x) : 0u;
    T lp[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const int zx = wrap(x + cx9(i), G.nx), zy = wrap(y + cy9(i), G.ny);
        const T v = __ldg(p.lam_out + (size_t)zy * G.pitch + zx + i * P);
        lp[i] = v * gather_factor<T, 9>(p.ps, pw, zy, zx, i);
    }
    if (p.ps.count > 0) {
        const int r = own_rule<T, 9>(p.ps, pw, y, x);
        if (r >= 0) {
            T v[9], add[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) { v[i] = __ldg(p.lam_out + o + i * P); add[i] = T(0); }
            rules_transpose<T, 9>(p.ps, r, v, add);
#pragma unroll
            for (int i = 0; i < 9; ++i) lp[i] += add[i];
        }
    }
    T lge[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) lge[i] = T(0);
    if (p.pc.count > 0) rules_transpose<T, 9>(p.pc, probe_rule(load_probe(p.pc, y, x), x), lp, lge);
    const T om = p.omega_f ? __ldg(p.omega_f + o) : p.omega;
    T W = T(0);
#pragma unroll
    for (int i = 0; i < 9; ++i) W += w9<T>(i) * lp[i];
#pragma unroll
    for (int i = 0; i < 9; ++i) p.lam_f[o + i * P] = (T(1) - om) * lp[i] + om * W + lge[i];
    if (p.lam_source) p.lam_source[o] = W;   // d o_i / d S = w_i (also at S = 0)
    if (p.g_omega) {
        double sf = 0.0, lf = 0.0;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const T fi = __ldg(p.f_in + o + i * P);
            sf += (double)fi;
            lf += (double)lp[i] * (double)fi;
        }
        p.g_omega[o] += -lf + (double)W * sf;
    }
}

// lam_q += G^T lam_grad for the Darcy gradient stencil with its boundary rules
// (G(q)(x) = sum_d K_d V_d(x), V_d(x) = q(x - c_d) or a rule of (q(x - c_d), q(x))).
template <typename T>
__global__ void gradient_adjoint_kernel(SweepGeom G, const T* lg, T scale, RulesView<T, 9> rules, T* lq) {
    grid_dep_wait();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= G.nx) return;
    const size_t o = (size_t)y * G.pitch + x;
    T acc = T(0);
    const uint32_t pw = rules.count > 0 && rules.push ? __ldg(rules.push + y * G.nx + x) : 0u;
#pragma unroll
    for (int d = 1; d < 9; ++d) {
        const int zx = wrap(x + cx9(d), G.nx), zy = wrap(y + cy9(d), G.ny);
        const size_t oz = (size_t)zy * G.pitch + zx;
        const T k = T(-3) * scale * w9<T>(d);
        const T v = k * (T(cx9(d)) * __ldg(lg + oz) + T(cy9(d)) * __ldg(lg + oz + G.plane));
        acc += v * gather_factor<T, 9>(rules, pw, zy, zx, d);
    }
    if (rules.count > 0) {
        const int r = own_rule<T, 9>(rules, pw, y, x);
        if (r >= 0) {   // rules of this cell whose source is q(x) itself
            const T gx = __ldg(lg + o), gy = __ldg(lg + o + G.plane);
#pragma unroll
            for (int d = 0; d < 9; ++d) {
                const uint8_t code = __ldg(rules.code + (size_t)r * 9 + d);
                if (code < 18) {
                    const T k = T(-3) * scale * w9<T>(d);
                    const T v = k * (T(cx9(d)) * gx + T(cy9(d)) * gy);
                    acc += code < 9 ? v : -v;
                }
            }
        }
    }
    lq[o] += acc;
}

// lam_f += adjoint of eta = (sum c_i f_i) (+ forces, handled by the caller)
// and of div = c(x) sum w2_i f_i; parameter gradients of c(x) = -1.5 / (3 (lam + mu) + 1).
template <typename T>
__global__ void elast_moments_adjoint_kernel(SweepGeom G, ElastMat<T> mat, T lam_u, T mu_u, T div_scale,
                                             const T* f, const T* lam_eta, const T* lam_div, T* lam_f,
                                             double* g_lam, double* g_mu) {
    grid_dep_wait();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= G.nx) return;
    const size_t o = (size_t)y * G.pitch + x;
    const long long P = G.plane;
    T lam = lam_u, mu = mu_u, c = div_scale;
    if (mat.mu_f) {
        lam = mat.lam_f[o];
        mu = mat.mu_f[o];
        c = T(-1.5) / (T(3) * (lam + mu) + T(1));
    }
    const T e0 = lam_eta ? lam_eta[o] : T(0), e1 = lam_eta ? lam_eta[o + P] : T(0);
    const T ld = lam_div ? lam_div[o] : T(0);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const T w2 = i < 4 ? T(1) : T(2);
        lam_f[o + i * P] += T(cx8(i)) * e0 + T(cy8(i)) * e1 + c * w2 * ld;
    }
    if (g_mu && lam_div) {
        double m2 = 0.0;
#pragma unroll
        for (int i = 0; i < 8; ++i) m2 += (i < 4 ? 1.0 : 2.0) * (double)f[o + i * P];
        const double s = (double)lam + (double)mu;
        const double dc = 4.5 / ((3.0 * s + 1.0) * (3.0 * s + 1.0));
        const double v = (double)ld * m2 * dc;
        g_lam[o] += v;
        g_mu[o] += v;
    }
}

// lam_f += adjoint of rho = sum f (+ sources, handled by the caller) and of
// grad = -3 omega sum c_i f_i; g_omega += d/d omega.
template <typename T>
__global__ void darcy_moments_adjoint_kernel(SweepGeom G, const T* f, T omega, const T* omega_f, const T* lam_rho,
                                             const T* lam_grad, T* lam_f, double* g_omega) {
    grid_dep_wait();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= G.nx) return;
    const size_t o = (size_t)y * G.pitch + x;
    const long long P = G.plane;
    const T om = omega_f ? omega_f[o] : omega;
    const T lr = lam_rho ? lam_rho[o] : T(0);
    const T gx = lam_grad ? lam_grad[o] : T(0), gy = lam_grad ? lam_grad[o + P] : T(0);
    double dom = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const T cg = T(cx9(i)) * gx + T(cy9(i)) * gy;
        lam_f[o + i * P] += lr + T(-3) * om * cg;
        if (g_omega && lam_grad) dom += -3.0 * (double)cg * (double)f[o + i * P];
    }
    if (g_omega && lam_grad) g_omega[o] += dom;
}

// Transpose of the Biot coupling force of a multigrid level,
// ext = fe + G(c(x) m2(f), scale): one kernel for G^T (the gradient stencil
// with its rules, gathered at this cell) followed by the divergence's
// transpose at this cell: lam_f += c w2 (G^T lam_ext), lam_fe += lam_ext, and
// the divergence scale's material gradient (needs the forward f).
template <typename T>
__global__ void divgrad_adjoint_kernel(SweepGeom G, ElastMat<T> mat, T lam_u, T mu_u, T div_scale, T scale,
                                       RulesView<T, 9> rules, const T* lg, const T* f, T* lam_f, T* lam_fe,
                                       double* g_lam, double* g_mu) {
    grid_dep_wait();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= G.nx) return;
    const size_t o = (size_t)y * G.pitch + x;
    const long long P = G.plane;
    T acc = T(0);                       // (G^T lam_ext)(x), as gradient_adjoint_kernel
    const uint32_t pw = rules.count > 0 && rules.push ? __ldg(rules.push + y * G.nx + x) : 0u;
#pragma unroll
    for (int d = 1; d < 9; ++d) {
        const int zx = wrap(x + cx9(d), G.nx), zy = wrap(y + cy9(d), G.ny);
        const size_t oz = (size_t)zy * G.pitch + zx;
        const T k = T(-3) * scale * w9<T>(d);
        const T v = k * (T(cx9(d)) * __ldg(lg + oz) + T(cy9(d)) * __ldg(lg + oz + P));
        acc += v * gather_factor<T, 9>(rules, pw, zy, zx, d);
    }
    const T gx = __ldg(lg + o), gy = __ldg(lg + o + P);
    if (rules.count > 0) {
        const int r = own_rule<T, 9>(rules, pw, y, x);
        if (r >= 0) {
#pragma unroll
            for (int d = 0; d < 9; ++d) {
                const uint8_t code = __ldg(rules.code + (size_t)r * 9 + d);
                if (code < 18) {
                    const T k = T(-3) * scale * w9<T>(d);
                    const T v = k * (T(cx9(d)) * gx + T(cy9(d)) * gy);
                    acc += code < 9 ? v : -v;
                }
            }
        }
    }
    if (lam_fe) {
        lam_fe[o] += gx;
        lam_fe[o + P] += gy;
    }
    T lam = lam_u, mu = mu_u, c = div_scale;
    if (mat.mu_f) {
        lam = mat.lam_f[o];
        mu = mat.mu_f[o];
        c = T(-1.5) / (T(3) * (lam + mu) + T(1));
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) lam_f[o + i * P] += c * (i < 4 ? T(1) : T(2)) * acc;
    if (g_mu) {
        double m2 = 0.0;
#pragma unroll
        for (int i = 0; i < 8; ++i) m2 += (i < 4 ? 1.0 : 2.0) * (double)f[o + i * P];
        const double s = (double)lam + (double)mu;
        const double v = (double)acc * m2 * (4.5 / ((3.0 * s + 1.0) * (3.0 * s + 1.0)));
        g_lam[o] += v;
        g_mu[o] += v;
    }
}

}  // namespace xlbb

extern "C" {

int xlbb_elast_sweep_adjoint(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat,
                             const XlbbElastSweepAdjoint* s, void* stream) {
    using namespace xlbb;
    if (!grid_ok(g) || !mat || !s || !s->lam_out || !s->lam_f) return fail(XLBB_EBADARG, "xlbb_elast_sweep_adjoint: bad argument");
    if (s->lam_out == s->lam_f) return fail(XLBB_EBADARG, "xlbb_elast_sweep_adjoint: lam_out and lam_f must differ");
    if ((s->g_lam == nullptr) != (s->g_mu == nullptr) || (s->g_mu && !s->f_in))
        return fail(XLBB_EBADARG, "xlbb_elast_sweep_adjoint: parameter gradients need g_lam, g_mu and f_in");
    if (!rules_ok(s->pc, g) || !rules_ok(s->ps, g)) return fail(XLBB_EBADARG, "xlbb_elast_sweep_adjoint: incomplete rules");
    if ((mat->mu_field == nullptr) != (mat->lam_field == nullptr))
        return fail(XLBB_EBADARG, "xlbb_elast_sweep_adjoint: lam_field and mu_field go together");
    const dim3 grid((g->nx + 127) / 128, g->ny);
    cudaStream_t st = XLBB_STREAM(stream);
#define XLBB_ADJ(T)                                                                 \
    {                                                                               \
        ElastAdjArgs<T> a;                                                          \
        a.geom = geom(g);                                                           \
        a.lam_out = (const T*)s->lam_out;                                           \
        a.lam_f = (T*)s->lam_f;                                                     \
        a.lam_resid = (T*)s->lam_resid;                                             \
        a.lam_force = (T*)s->lam_force;                                             \
        a.g_lam = s->g_lam;                                                         \
        a.g_mu = s->g_mu;                                                           \
        a.f_in = (const T*)s->f_in;                                                 \
        a.resid = (const T*)s->resid;                                               \
        a.force = s->use_force ? (const T*)s->force : nullptr;                      \
        a.fext = (const T*)s->fext;                                                 \
        a.a = T(s->a);                                                              \
        a.b = T(s->b);                                                              \
        a.mat = make_mat<T>(mat);                                                   \
        a.lam_u = T(mat->lam);                                                      \
        a.mu_u = T(mat->mu);                                                        \
        a.pc = rules_view<T, 8>(s->pc);                                             \
        a.ps = rules_view<T, 8>(s->ps);                                             \
        launch_k(elast_sweep_adjoint_kernel<T>, grid, 128, 0, st, a);                     \
    }
    if (dtype == XLBB_F32) XLBB_ADJ(float)
    else if (dtype == XLBB_F64) XLBB_ADJ(double)
    else return fail(XLBB_EUNSUPPORTED, "xlbb_elast_sweep_adjoint: dtype");
#undef XLBB_ADJ
    return check_launch("xlbb_elast_sweep_adjoint");
}

int xlbb_darcy_sweep_adjoint(int dtype, const XlbbGrid* g, const XlbbDarcySweepAdjoint* s, void* stream) {
    using namespace xlbb;
    if (!grid_ok(g) || !s || !s->lam_out || !s->lam_f) return fail(XLBB_EBADARG, "xlbb_darcy_sweep_adjoint: bad argument");
    if (s->lam_out == s->lam_f) return fail(XLBB_EBADARG, "xlbb_darcy_sweep_adjoint: lam_out and lam_f must differ");
    if (s->g_omega && !s->f_in) return fail(XLBB_EBADARG, "xlbb_darcy_sweep_adjoint: g_omega needs f_in");
    if (!rules_ok(s->pc, g) || !rules_ok(s->ps, g)) return fail(XLBB_EBADARG, "xlbb_darcy_sweep_adjoint: incomplete rules");
    const dim3 grid((g->nx + 127) / 128, g->ny);
    cudaStream_t st = XLBB_STREAM(stream);
#define XLBB_ADJ(T)                                                   \
    {                                                                 \
        DarcyAdjArgs<T> a;                                            \
        a.geom = geom(g);                                             \
        a.lam_out = (const T*)s->lam_out;                             \
        a.lam_f = (T*)s->lam_f;                                       \
        a.lam_source = (T*)s->lam_source;                             \
        a.g_omega = s->g_omega;                                       \
        a.f_in = (const T*)s->f_in;                                   \
        a.omega = T(s->omega);                                        \
        a.omega_f = (const T*)s->omega_field;                         \
        a.source = (const T*)s->source;                               \
        a.ext = (const T*)s->ext_source;                              \
        a.pc = rules_view<T, 9>(s->pc);                               \
        a.ps = rules_view<T, 9>(s->ps);                               \
        launch_k(darcy_sweep_adjoint_kernel<T>, grid, 128, 0, st, a);       \
    }
    if (dtype == XLBB_F32) XLBB_ADJ(float)
    else if (dtype == XLBB_F64) XLBB_ADJ(double)
    else return fail(XLBB_EUNSUPPORTED, "xlbb_darcy_sweep_adjoint: dtype");
#undef XLBB_ADJ
    return check_launch("xlbb_darcy_sweep_adjoint");
}

int xlbb_darcy_gradient_adjoint(int dtype, const XlbbGrid* g, const void* lam_grad, double scale,
                                const XlbbRules* rules, void* lam_q, void* stream) {
    using namespace xlbb;
    if (!grid_ok(g) || !lam_grad || !lam_q || !rules) return fail(XLBB_EBADARG, "xlbb_darcy_gradient_adjoint: bad argument");
    if (!rules_ok(*rules, g)) return fail(XLBB_EBADARG, "xlbb_darcy_gradient_adjoint: incomplete rules");
    const dim3 grid((g->nx + 127) / 128, g->ny);
    cudaStream_t st = XLBB_STREAM(stream);
    if (dtype == XLBB_F32)
        launch_k(gradient_adjoint_kernel<float>, grid, 128, 0, st, geom(g), (const float*)lam_grad, (float)scale,
                                                             rules_view<float, 9>(*rules), (float*)lam_q);
    else if (dtype == XLBB_F64)
        launch_k(gradient_adjoint_kernel<double>, grid, 128, 0, st, geom(g), (const double*)lam_grad, scale,
                                                              rules_view<double, 9>(*rules), (double*)lam_q);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_darcy_gradient_adjoint: dtype");
    return check_launch("xlbb_darcy_gradient_adjoint");
}

int xlbb_elast_moments_adjoint(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat, const void* f,
                               const void* lam_eta, const void* lam_div, double div_scale, void* lam_f,
                               double* g_lam, double* g_mu, void* stream) {
    using namespace xlbb;
    if (!grid_ok(g) || !mat || !lam_f || (!lam_eta && !lam_div)) return fail(XLBB_EBADARG, "xlbb_elast_moments_adjoint: bad argument");
    if ((g_lam == nullptr) != (g_mu == nullptr) || (g_mu && !f))
        return fail(XLBB_EBADARG, "xlbb_elast_moments_adjoint: parameter gradients need g_lam, g_mu and f");
    const dim3 grid((g->nx + 127) / 128, g->ny);
    cudaStream_t st = XLBB_STREAM(stream);
    if (dtype == XLBB_F32)
        launch_k(elast_moments_adjoint_kernel<float>, grid, 128, 0, st, 
            geom(g), make_mat<float>(mat), (float)mat->lam, (float)mat->mu, (float)div_scale, (const float*)f,
            (const float*)lam_eta, (const float*)lam_div, (float*)lam_f, g_lam, g_mu);
    else if (dtype == XLBB_F64)
        launch_k(elast_moments_adjoint_kernel<double>, grid, 128, 0, st, 
            geom(g), make_mat<double>(mat), mat->lam, mat->mu, div_scale, (const double*)f,
            (const double*)lam_eta, (const double*)lam_div, (double*)lam_f, g_lam, g_mu);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_elast_moments_adjoint: dtype");
    return check_launch("xlbb_elast_moments_adjoint");
}

int xlbb_darcy_moments_adjoint(int dtype, const XlbbGrid* g, const void* f, double omega, const void* omega_field,
                               const void* lam_rho, const void* lam_grad, void* lam_f, double* g_omega,
                               void* stream) {
    using namespace xlbb;
    if (!grid_ok(g) || !lam_f || (!lam_rho && !lam_grad) || (g_omega && !f))
        return fail(XLBB_EBADARG, "xlbb_darcy_moments_adjoint: bad argument");
    const dim3 grid((g->nx + 127) / 128, g->ny);
    cudaStream_t st = XLBB_STREAM(stream);
    if (dtype == XLBB_F32)
        launch_k(darcy_moments_adjoint_kernel<float>, grid, 128, 0, st, 
            geom(g), (const float*)f, (float)omega, (const float*)omega_field, (const float*)lam_rho,
            (const float*)lam_grad, (float*)lam_f, g_omega);
    else if (dtype == XLBB_F64)
        launch_k(darcy_moments_adjoint_kernel<double>, grid, 128, 0, st, 
            geom(g), (const double*)f, omega, (const double*)omega_field, (const double*)lam_rho,
            (const double*)lam_grad, (double*)lam_f, g_omega);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_darcy_moments_adjoint: dtype");
    return check_launch("xlbb_darcy_moments_adjoint");
}

int xlbb_divgrad_adjoint(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat, const void* lam_ext,
                         double scale, const XlbbRules* rules, const void* f, void* lam_f, void* lam_fe,
                         double* g_lam, double* g_mu, void* stream) {
    using namespace xlbb;
    if (!grid_ok(g) || !mat || !lam_ext || !lam_f || !rules) return fail(XLBB_EBADARG, "xlbb_divgrad_adjoint: bad argument");
    if ((g_lam == nullptr) != (g_mu == nullptr) || (g_mu && !f))
        return fail(XLBB_EBADARG, "xlbb_divgrad_adjoint: parameter gradients need g_lam, g_mu and f");
    if (!rules_ok(*rules, g)) return fail(XLBB_EBADARG, "xlbb_divgrad_adjoint: incomplete rules");
    const dim3 grid((g->nx + 127) / 128, g->ny);
    cudaStream_t st = XLBB_STREAM(stream);
    const double div_scale = -1.5 / (3.0 * (mat->lam + mat->mu) + 1.0);
    if (dtype == XLBB_F32)
        launch_k(divgrad_adjoint_kernel<float>, grid, 128, 0, st, 
            geom(g), make_mat<float>(mat), (float)mat->lam, (float)mat->mu, (float)div_scale, (float)scale,
            rules_view<float, 9>(*rules), (const float*)lam_ext, (const float*)f, (float*)lam_f, (float*)lam_fe,
            g_lam, g_mu);
    else if (dtype == XLBB_F64)
        launch_k(divgrad_adjoint_kernel<double>, grid, 128, 0, st, 
            geom(g), make_mat<double>(mat), mat->lam, mat->mu, div_scale, scale, rules_view<double, 9>(*rules),
            (const double*)lam_ext, (const double*)f, (double*)lam_f, (double*)lam_fe, g_lam, g_mu);
    else return fail(XLBB_EUNSUPPORTED, "xlbb_divgrad_adjoint: dtype");
    return check_launch("xlbb_divgrad_adjoint");
}

}  // extern "C"
