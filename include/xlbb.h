/*
 * xlbb.h -- C ABI of the B200 (sm_100a) lattice-Boltzmann Biot hot path.
 *
 * The reference (s-lunowa/xlb-biot) is pure Python/JAX; its "interface" for
 * this path is the set of solver methods listed beside each entry point below
 * (file:line inside the reference project).  Every entry point:
 *   - takes device pointers owned by the caller plus a cudaStream_t (as void*),
 *   - is stream-ordered and asynchronous, allocates nothing,
 *   - returns XLBB_OK (0) or a negative XLBB_E* code; a thread-local message is
 *     kept for xlbb_last_error().
 *
 * Memory layout of every field ("SoA"): component planes of a (ny x pitch)
 * row-major grid, x fastest:  value(x, y, i) = base[i*plane + y*pitch + x],
 * with pitch >= nx and plane >= ny*pitch.  The Python layer exposes such a
 * buffer to users as a tensor of the reference's shape (nx, ny, q).
 */
#ifndef XLBB_H
#define XLBB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XLBB_OK 0
#define XLBB_EBADARG (-1)
#define XLBB_ELAUNCH (-2)
#define XLBB_ETIMEOUT (-3)
#define XLBB_ENONFINITE (-4)
#define XLBB_EUNSUPPORTED (-5)

#define XLBB_F32 0
#define XLBB_F64 1
#define XLBB_F32_ACC64 2   /* FP32 storage, FP64 arithmetic and rule constants (elasticity
                              and Darcy sweeps: the "f64/f32" precision policy) */

typedef struct {
    int nx, ny;        /* logical grid size (cells)                        */
    int pitch;         /* row stride in elements                           */
    long long plane;   /* component-plane stride in elements               */
} XlbbGrid;

/*
 * Boundary rules compiled on the host from the reference's BC objects.
 * Rule cells are stored CSR-by-row: the cells of row y are
 * cell_x[row_ptr[y] .. row_ptr[y+1]) sorted by x.  For each rule cell and
 * direction d, code[r*q+d] selects the base value and cst[r*q+d] is added:
 *   0..q-1      : +src[code]        (src = pre-collision input for a
 *   q..2q-1     : -src[code-q]       post-collision rule, own post-collision
 *   2q          : 0                  populations for a post-streaming rule)
 *   2q+1        : +current value    (collision output / streamed value)
 *   2q+2        : -current value
 */
typedef struct {
    int count;
    const int* row_ptr;      /* ny+1 entries */
    const int* cell_x;       /* count entries */
    const uint8_t* code;     /* count*q entries */
    const void* cst;         /* count*q entries, compute dtype */
    const uint32_t* mask;    /* ny*words_per_row words: bit (x%32) of word x/32 set on rule cells */
    const int* word_base;    /* rule index of the first rule cell of each mask word */
    int words_per_row;       /* >= ceil(nx/32) */
    /* Post-streaming rules, for the collide-and-push sweep (may be NULL: that
     * sweep then uses the row-marching kernel): one word per cell (index
     * y*nx + x), bit d set when direction d pushed from this cell lands where a
     * rule rebuilds it, bit 16 set on rule cells.  Only built when every
     * "current value" code is +current with constant 0. */
    const uint32_t* push;
} XlbbRules;

/*
 * Launch shape of the fused sweeps (kernel 0: elasticity, 1: Darcy):
 * tx owned columns per CTA (128 or 256), strips sized for ctas_per_sm CTAs per
 * SM but never shorter than min_rows rows, and the pipeline:
 *   0: CTA row ring in shared memory, register prefetch of depth (1, 2) rows;
 *   1: as 0, inputs in a shared-memory ring of depth (2, 4, 6) rows filled by
 *      cp.async.bulk copies on mbarriers (needs 16-byte aligned planes and
 *      pitch, otherwise pipeline 0 is used);
 *   2: independent warps of 30 output columns (tx ignored), post-collision
 *      rows in registers, streaming by warp shuffles, no barrier; register
 *      prefetch of depth (1, 2) rows; ctas_per_sm counts CTAs of 4 warps;
 *   3: collide and push (the default): one thread per cell, CTAs of tx
 *      columns of one row; depth, ctas_per_sm and min_rows are not used;
 *   4: as 3, except that FP32 elasticity sweeps of
 *      at least 64 K cells without boundary rules, per-cell material, side
 *      outputs or fused sums, with at most one force array and 16-byte
 *      aligned rows and planes, run four columns per lane (float4 loads and
 *      stores, streaming along x by warp shuffles); same results.
 * FP64 sweeps cap tx at 128.
 */
typedef struct {
    int tx, depth, ctas_per_sm, min_rows, pipeline;
} XlbbSweepConfig;

int xlbb_sweep_set_config(int kernel, const XlbbSweepConfig* cfg);
int xlbb_sweep_get_config(int kernel, XlbbSweepConfig* cfg);

/* Device status word: 0, or the first error a kernel recorded since the last
 * reset -- XLBB_ETIMEOUT if a bounded wait gave up, XLBB_ENONFINITE if
 * xlbb_reduce_sum produced NaN or Inf (a diverged or corrupted field),
 * XLBB_EBADARG if xlbb_batched_elast_sweep4 skipped an instance that does not
 * qualify.  Synchronous; reset != 0 clears it. */
int xlbb_device_status(int* status, int reset);
/* Self-test of the bounded waits (no counterpart in the reference): one
 * kernel waits on an mbarrier that nothing completes, with a limit of `polls`
 * (1 .. 2^22), gives up, records XLBB_ETIMEOUT in the status word, writes 1
 * to the device int *gave_up and returns.  No copy is in flight, so nothing
 * hangs; the context stays usable. */
int xlbb_wait_selftest(unsigned polls, int* gave_up, void* stream);

typedef struct {
    double lam, mu;          /* uniform Lame parameters (lattice units)       */
    const void* lam_field;   /* optional per-cell lambda (1 plane) or NULL    */
    const void* mu_field;    /* optional per-cell mu (1 plane) or NULL        */
} XlbbElastMaterial;

/*
 * One D2Q8 elasticity sweep, fused collide + post-collision BCs + stream +
 * post-streaming BCs, with the multigrid smoother algebra folded in:
 *     g   = f_in - resid                      (resid may be NULL)
 *     out = a * f_in + b * STEP(g)
 * a=0,b=1 is LBMElasticity._step (src/elasticity.py:1169-1219);
 * a=1-gamma,b=gamma the damped smoothing sweep of _mg_step (:1258-1267);
 * a=1,b=-1 the residual f - STEP(f - r) (:1285-1286).
 * STEP applies force (if use_force) + fext as in collision() (:959-1000).
 * If sumsq != NULL, each CTA writes sum(out^2) (sumsq_diff = 0) or
 * sum((out - f_in)^2) (sumsq_diff = 1) over the box [bx0,bx1)x[by0,by1) into
 * sumsq[cta] (FP64; reduce with xlbb_reduce_sum); the buffer needs
 * xlbb_elast_sweep_ctas() entries, the reduction the exact count
 * xlbb_elast_sweep_partials().  If div_out != NULL the divergence moment of out
 * (update_divergence, :1040-1058) is written as a side output.
 */
typedef struct {
    const void* f_in;
    void* f_out;
    const void* force;       /* static force (2 planes) or NULL */
    int use_force;
    const void* fext;        /* external force (2 planes) or NULL */
    const void* resid;       /* residual (8 planes, zero outside the interior) or NULL */
    double a, b;
    XlbbRules pc, ps;
    double* sumsq;
    int bx0, bx1, by0, by1;
    void* div_out;
    int sumsq_diff;
} XlbbElastSweep;

int xlbb_elast_sweep(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat,
                     const XlbbElastSweep* s, void* stream);
/* Upper bound on the FP64 partials of any elasticity sweep of this dtype on g
 * under the current launch config (size of a partials buffer). */
int xlbb_elast_sweep_ctas(int dtype, const XlbbGrid* g);
/* Exactly the partials that xlbb_elast_sweep with these arguments writes when
 * s->sumsq is set (the CTAs of the launch it takes: collide-and-push, or the
 * row-marching shape when its post-streaming rules have no push words or it
 * writes div_out); pass this count to xlbb_reduce_sum. */
int xlbb_elast_sweep_partials(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat,
                              const XlbbElastSweep* s);
/* The pipeline (XlbbSweepConfig numbering; 0 for the row-marching kernel)
 * that xlbb_elast_sweep would run for these arguments now (diagnostic). */
int xlbb_elast_sweep_pipeline(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat,
                              const XlbbElastSweep* s);

/*
 * One D2Q9 advection-diffusion-reaction BGK sweep (AdvectionDiffusionReactionBGK.step,
 * src/darcy.py:131-171 with collision :106-129): omega uniform or per cell.
 * If sumsq != NULL each CTA writes sum((out - f_in)^2) (FP64 convergence residual).
 */
typedef struct {
    const void* f_in;
    void* f_out;
    double omega;
    const void* omega_field; /* per-cell omega (1 plane) or NULL */
    const void* source;      /* static source (1 plane) or NULL */
    const void* ext_source;  /* external source (1 plane) or NULL */
    XlbbRules pc, ps;
    double* sumsq;
    const void* resid;       /* 9 planes r or NULL: the sweep collides f - r (a
                                refinement step's correction equation); not
                                with post-collision rules (XLBB_EUNSUPPORTED) */
} XlbbDarcySweep;

int xlbb_darcy_sweep(int dtype, const XlbbGrid* g, const XlbbDarcySweep* s, void* stream);
/* Upper bound on the FP64 partials of any D2Q9 sweep of this dtype on g under
 * the current launch config (size of a partials buffer). */
int xlbb_darcy_sweep_ctas(int dtype, const XlbbGrid* g);
/* Exactly the partials that xlbb_darcy_sweep / xlbb_fluid_sweep with these
 * arguments writes when s->sumsq is set; pass this count to xlbb_reduce_sum. */
int xlbb_darcy_sweep_partials(int dtype, const XlbbGrid* g, const XlbbDarcySweep* s);
/* The pipeline (XlbbSweepConfig numbering) that xlbb_darcy_sweep would run
 * for these arguments now (diagnostic). */
int xlbb_darcy_sweep_pipeline(int dtype, const XlbbGrid* g, const XlbbDarcySweep* s);

/*
 * One fused D2Q9 fluid step (replaces BGKSim.collision, src/models.py:20-34, or
 * KBCSim.collision, :48-72, inside LBMBase.step, src/base.py:809-846):
 * collision with the second-order equilibrium of src/base.py:686-724,
 * PostCollision rules, streaming, PostStreaming rules.  Same argument block as
 * xlbb_darcy_sweep (omega uniform or per cell); source, ext_source and resid
 * must be NULL (XLBB_EBADARG otherwise).  sumsq, when set, has
 * xlbb_darcy_sweep_ctas(dtype, g) entries, of which it writes
 * xlbb_darcy_sweep_partials(dtype, g, s).
 */
#define XLBB_FLUID_BGK 0
#define XLBB_FLUID_KBC 1
int xlbb_fluid_sweep(int dtype, const XlbbGrid* g, const XlbbDarcySweep* s, int model, void* stream);

/*
 * Three-dimensional grid: nz planes of ny rows; row (y, z) is y + ny * z, cell
 * (x, y, z) at (y + ny * z) * pitch + x, population i at i * plane further.
 * Rule tables over such a grid index rows the same way (ny * nz rows).
 */
typedef struct {
    int nx, ny, nz, pitch;
    long long plane;
} XlbbGrid3;

/*
 * One fused D3Q19 (q = 19) or D3Q27 (q = 27) fluid step: model XLBB_FLUID_BGK
 * (BGKSim.collision, src/models.py:20-34) on either lattice, XLBB_FLUID_KBC
 * (KBCSim.collision, :47-72, shear decomposition :156-214) on D3Q27 only;
 * inside LBMBase.step, src/base.py:809-846, on the lattices of
 * src/lattice.py:132-182: collision, PostCollision rules,
 * streaming with periodic wrap in x, y and z, PostStreaming rules.  Uniform
 * omega only; omega_field, source, ext_source, resid and sumsq must be NULL
 * (XLBB_EBADARG), and PostStreaming rules need their push words
 * (XLBB_EUNSUPPORTED otherwise).  Replaces the step that
 * examples/performance/MLUPS3d.py times.
 */
int xlbb_fluid3_sweep(int dtype, const XlbbGrid3* g, const XlbbDarcySweep* s, int q, int model, void* stream);

/*
 * Darcy sweep plus its FP64 convergence residual, allocating nothing.
 * No counterpart in the reference: it exists for callers that cannot allocate
 * device memory (inside a CUDA-graph capture, host runtimes that hand the
 * library only the buffers they own, processes with a fixed memory budget).
 * The caller passes the sweep's inputs and outputs as for xlbb_darcy_sweep
 * (s->sumsq is ignored) plus sumsq_out, one device double that receives
 * sum((f_out - f_in)^2).  The per-CTA partial sums go to a scratch array built
 * into the library: XLBB_NOALLOC_MAX_PARTIALS doubles (128 KiB) held by every
 * GPU that loads the library until exit; a sweep whose launch has more CTAs
 * (xlbb_darcy_sweep_partials) is rejected with XLBB_EBADARG.  Under the
 * default collide-and-push shape that is ceil(nx / 128) * ny > 16384, e.g.
 * every grid of 2048 x 2048 or more; row-marching shapes (pipelines 0-2) have
 * about ctas_per_sm CTAs per SM at any size.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress), so make that first call
 * before any stream capture.  All calls share the array, which keeps the last
 * call's contents (each used slot is rewritten before it is read, so nothing
 * needs clearing); calls that overlap on the GPU (concurrent streams) race.
 */
#define XLBB_NOALLOC_MAX_PARTIALS 16384
#define XLBB_NOALLOC_MAX_DEVICES 64
int xlbb_darcy_sweep_residual_noalloc(int dtype, const XlbbGrid* g, const XlbbDarcySweep* s,
                                      double* sumsq_out, void* stream);

/*
 * Isotropic 9-point gradient of a scalar field with the ADR (anti-)bounce-back
 * rules applied to the shifted copies (AdvectionDiffusionReactionBGK.gradient,
 * src/darcy.py:75-104):  out = base + gradient(q, scale)  (2 planes; base may
 * be NULL, out may alias base).
 */
int xlbb_darcy_gradient(int dtype, const XlbbGrid* g, const void* q, double scale,
                        const XlbbRules* rules, const void* base, void* out, void* stream);

/*
 * Elasticity macroscopic fields (LBMElasticity.update_macroscopic :1002-1038,
 * update_divergence :1040-1058).  eta = m10,m01 + 0.5*(force + fext);
 * any output may be NULL.  div is computed from f (not f + force).
 */
int xlbb_elast_moments(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat,
                       const void* f, const void* force, const void* fext,
                       void* eta, void* sigma, void* div, double div_scale, void* stream);

/*
 * The Biot coupling force out = base + G(div(f), scale) in one kernel: the
 * divergence of xlbb_elast_moments followed by the gradient of
 * xlbb_darcy_gradient (with its rules), bit for bit, without the divergence's
 * round trip through memory (poroelasticity's nonlinear force,
 * src/poroelasticity.py:324, evaluated before every elasticity sweep).
 * base may be NULL; out must not alias f.
 */
int xlbb_elast_divgrad(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat, double div_scale,
                       const void* f, double scale, const XlbbRules* rules, const void* base,
                       void* out, void* stream);
/*
 * A poroelastic smoothing sweep in one kernel: xlbb_elast_divgrad of the
 * sweep's own input s->f_in (base = s->fext, gradient rules grad_rules)
 * handed to xlbb_elast_sweep as its external force, on the collide-and-push
 * launch -- the smoothing and residual sweeps of _mg_step with the nonlinear
 * force of src/poroelasticity.py:324 (src/elasticity.py:1258-1305), the same
 * values bit for bit, one launch instead of two and no force field in memory.
 * XLBB_F32 / XLBB_F64 only; XLBB_EUNSUPPORTED for fused sums (s->sumsq),
 * s->div_out, or post-streaming rules without push words (use the two calls).
 */
int xlbb_elast_sweep_divgrad(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat,
                             const XlbbElastSweep* s, double div_scale, double scale,
                             const XlbbRules* grad_rules, void* stream);

/* Elasticity equilibrium (LBMElasticity.equilibrium :909-957). */
int xlbb_elast_equilibrium(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat,
                           const void* eta, const void* sigma, const void* force,
                           const void* fext, void* f_out, void* stream);

/*
 * Darcy macroscopic fields (update_macroscopic, src/darcy.py:36-73):
 * rho = sum f + 0.5*(source + ext_source); grad = -3*omega*sum c_i f_i.
 */
int xlbb_darcy_moments(int dtype, const XlbbGrid* g, const void* f, double omega,
                       const void* omega_field, const void* source, const void* ext_source,
                       void* rho, void* grad, void* stream);

/*
 * Multigrid transfers (LBMElasticity._restrict :850-865, _prolong :878-894).
 * Interior box of the fine grid: [x0, nx_f - x1bc) x [y0, ny_f - y1bc) with the
 * same BC offsets on the coarse grid.  restrict writes the 2x2 block SUMS into
 * the coarse grid's interior and zeros outside it; prolong_add adds the coarse
 * interior, injected, into the fine interior.
 */
int xlbb_restrict(int dtype_fine, int dtype_coarse, const XlbbGrid* fine, const XlbbGrid* coarse, int q,
                  int x0, int x1bc, int y0, int y1bc, const void* res, void* r_coarse, void* stream);
int xlbb_prolong_add(int dtype_fine, int dtype_coarse, const XlbbGrid* fine, const XlbbGrid* coarse, int q,
                     int x0, int x1bc, int y0, int y1bc, const void* f_coarse, void* f_fine, void* stream);
/* dtype pairs (fine, coarse): (F32, F32), (F32, F64) -- an FP64 coarsest level
 * under FP32 levels -- and (F64, F64). */

/*
 * Batched elasticity multigrid (no counterpart in the reference, which runs
 * one instance per solver object): many independent periodic D2Q8 instances
 * of different sizes and Lame parameters advance in one launch per sweep.
 * xlbb_batch_upload converts host instance records into the device
 * descriptor array `dev` (xlbb_batch_desc_bytes(dtype) bytes each; the caller
 * owns it).  A sweep runs every tile of `tiles_dev`: tile = (instance, x0,
 * row range), CTAs of 128 owned columns looping over the list (`ctas` is an
 * upper bound: at most one wave of resident CTAs is launched); the algebra is
 * the one of xlbb_elast_sweep (out = a f + b STEP(f - resid)); tile_sumsq
 * (XLBB_BATCH_PARTS_PER_TILE doubles per tile -- a partial per warp, no block
 * barrier --, or NULL) receives sum(out^2) / sum((out - f_in)^2), reduced per
 * instance by xlbb_segment_sum over the ranges begin[i]..begin[i+1] of
 * partials (tile ranges times XLBB_BATCH_PARTS_PER_TILE).
 * zero_in != 0 takes every f_in as zero without reading it (the first sweep of
 * a coarse level, whose correction starts from zero): the results of a
 * zero-filled input, bit for bit, without the fill and the reads.
 */
typedef struct {
    const void* f_in;
    void* f_out;
    const void* force;       /* static force (2 planes) or NULL */
    const void* resid;       /* residual (8 planes) or NULL */
    int nx, ny, pitch;
    long long plane;
    double lam, mu;
} XlbbBatchInstance;

typedef struct {
    int inst, x0, ys, ye;
} XlbbBatchTile;

#define XLBB_BATCH_PARTS_PER_TILE 32

typedef struct {
    const void* fine;        /* fine residual (restrict) / fine populations (prolong) */
    void* coarse;            /* coarse residual (restrict) / coarse correction (prolong) */
    int nx_f, ny_f, pitch_f, pitch_c;
    long long plane_f, plane_c;
} XlbbBatchTransfer;

int xlbb_batch_desc_bytes(int dtype);
int xlbb_batch_upload(int dtype, const XlbbBatchInstance* host, int ninst, void* dev, void* stream);
int xlbb_batched_elast_sweep(int dtype, const void* inst_dev, const XlbbBatchTile* tiles_dev, int ntiles,
                             int ctas, double a, double b, int use_force, int has_resid, int sumsq_diff,
                             double* tile_sumsq, int zero_in, void* stream);
/*
 * The same sweep by the four-column kernel (dtype XLBB_F32 only): a warp
 * takes a tile row, a lane four adjacent columns, with
 * 16-byte loads and stores and streaming along x by warp shuffles.  Every
 * instance must store FP32 with nx, pitch and plane multiples of 4 and 16-byte
 * aligned planes (xlbb_batch_upload records whether it does); the tiles of one
 * that does not are skipped and the device status word is set to
 * XLBB_EBADARG.  Results equal xlbb_batched_elast_sweep's.
 */
int xlbb_batched_elast_sweep4(int dtype, const void* inst_dev, const XlbbBatchTile* tiles_dev, int ntiles,
                              int ctas, double a, double b, int use_force, int has_resid, int sumsq_diff,
                              double* tile_sumsq, int zero_in, void* stream);
int xlbb_batched_restrict(int dtype_fine, int dtype_coarse, const XlbbBatchTransfer* tr_dev, int ninst,
                          void* stream);
int xlbb_batched_prolong_add(int dtype_fine, int dtype_coarse, const XlbbBatchTransfer* tr_dev, int ninst,
                             void* stream);
/*
 * Prolongation plus the FP64 norms that track the smooth error: as
 * xlbb_batched_prolong_add, and norms[2 i] = sum over instance i of the
 * prolongated correction^2, norms[2 i + 1] = sum of the corrected fine
 * populations^2 (deterministic).  parts: caller scratch of
 * 2 * XLBB_PROLONG_BLOCKS * ninst doubles.
 */
#define XLBB_PROLONG_BLOCKS 32
int xlbb_batched_prolong_add_norms(int dtype_fine, int dtype_coarse, const XlbbBatchTransfer* tr_dev, int ninst,
                                   double* parts, double* norms, void* stream);
/*
 * The same prolongation with a balanced block map: block b adds the coarse
 * correction to elements [map[2 b + 1], + 1024) (cell index y * nx_f + x) of
 * instance map[2 b] of tr_dev -- the caller gives each instance
 * ceil(nx_f * ny_f / 1024) consecutive blocks, so every block does the same
 * work whatever the instance sizes.  With norms != NULL (then parts, begin_dev
 * and ninst too), norms[2 i] / norms[2 i + 1] receive the FP64 sums of the
 * correction^2 / of the corrected populations^2 over instance i's blocks
 * begin_dev[i] .. begin_dev[i + 1] (deterministic); parts: caller scratch of
 * 2 * nblocks doubles.
 */
int xlbb_batched_prolong_add_map(int dtype_fine, int dtype_coarse, const XlbbBatchTransfer* tr_dev,
                                 const int* map_dev, int nblocks, double* parts, const int* begin_dev, int ninst,
                                 double* norms, void* stream);
int xlbb_segment_sum(const double* parts, const int* begin_dev, int nseg, double* out, void* stream);
/*
 * Removes the mean first moments (the mean of sum_i c_i f_i, the rigid
 * displacement mode a periodic problem leaves undetermined) from the level-0
 * populations of a batch: the fine fields of tr_dev (their coarse fields are
 * not used), block map and begin_dev as for xlbb_batched_prolong_add_map;
 * sums[2 i] / sums[2 i + 1] receive the FP64 moment sums of instance i before
 * the shift; parts: caller scratch of 2 * nblocks doubles.  No counterpart in
 * the reference (whose FP64 iteration keeps this mode at zero to rounding):
 * the V-cycle from zero with a zero-mean force conserves it in exact
 * arithmetic, and FP32 rounding makes it drift over hundreds of cycles.
 */
int xlbb_batched_remove_mean_moment(int dtype, const XlbbBatchTransfer* tr_dev, const int* map_dev, int nblocks,
                                    double* parts, const int* begin_dev, int ninst, double* sums, void* stream);

/*
 * Persistent multigrid tail of a periodic batch (the recursion of
 * LBMElasticity._mg_step, src/elasticity.py:1221-1312, below a level): one
 * launch finishes the V-cycle of every listed instance from its tail's top
 * level down to its coarsest level and back, one CTA per instance with all of
 * the tail's levels in shared memory (CTA barriers only).  Per level above the
 * last: k_smooth damped sweeps (1 - gamma, gamma) from zero, the residual
 * sweep, 2 x 2 block-sum restriction, the level below, injection of its
 * correction, k_smooth damped sweeps; the last level: 2 k_smooth damped
 * sweeps, the first from zero.  Reads each record's top-level right-hand
 * side `resid` and writes its correction `f_out` (both in the top level's
 * dtype: dtype_coarse when the tail has one level, else dtype); the results
 * equal the level-by-level batched launches'.  dtype / dtype_coarse:
 * (XLBB_F32, XLBB_F32), (XLBB_F32, XLBB_F64) or (XLBB_F64, XLBB_F64).
 * smem_bytes: the largest xlbb_batched_tail_smem of the records (at most the
 * device's opt-in shared memory per block); a record that needs more, or
 * whose grid is not divisible by 2^(levels - 1), is skipped and the device
 * status word set to XLBB_EBADARG.  k_smooth even, >= 2.
 */
typedef struct {
    const void* resid;       /* top level's right-hand side (8 planes)             */
    void* f_out;             /* top level's correction (8 planes)                  */
    int nx, ny, pitch;       /* top level grid and row pitch (elements)            */
    long long plane;         /* plane stride (elements)                            */
    int levels;              /* levels of the tail, 1 .. 12 (the last: the coarsest) */
    double lam, mu;          /* Lame parameters (lattice units)                    */
} XlbbBatchTail;
int xlbb_batched_tail_smem(int dtype, int dtype_coarse, int nx, int ny, int levels);
int xlbb_batched_tail(int dtype, int dtype_coarse, const XlbbBatchTail* tails_dev, int count, int smem_bytes,
                      double gamma, int k_smooth, void* stream);

/*
 * Adjoints (transposed linear maps) for gradients of a misfit with respect to
 * per-cell material fields.  No counterpart in the reference (which has no
 * adjoint).  Each call takes the adjoint of a forward kernel's output and
 * produces the adjoints of its inputs; parameter gradients accumulate per cell
 * in FP64 and need the forward call's inputs.
 *
 * xlbb_elast_sweep_adjoint: transpose of xlbb_elast_sweep with the same a, b,
 * rules and material: lam_f = a lam_out + lam_g (written), lam_resid -= lam_g
 * (if not NULL), lam_force = adjoint of the total force force + fext
 * (2 planes, written, if not NULL), g_lam / g_mu += d/d lambda, d/d mu of the
 * collision at every cell (if not NULL; need f_in, resid, force, fext of the
 * forward call).
 */
typedef struct {
    const void* lam_out;     /* adjoint of the sweep's output (8 planes) */
    void* lam_f;             /* adjoint of f_in (8 planes, written) */
    void* lam_resid;         /* adjoint of resid (8 planes, accumulated) or NULL */
    void* lam_force;         /* adjoint of the total force (2 planes, written) or NULL */
    double* g_lam;           /* per-cell gradient accumulators (FP64) or NULL */
    double* g_mu;
    const void* f_in;        /* forward inputs (parameter gradients only) */
    const void* resid;
    const void* force;
    int use_force;
    const void* fext;
    double a, b;
    XlbbRules pc, ps;
} XlbbElastSweepAdjoint;

int xlbb_elast_sweep_adjoint(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat,
                             const XlbbElastSweepAdjoint* s, void* stream);

/* Transpose of xlbb_darcy_sweep: lam_f (written), lam_source = adjoint of the
 * total source (1 plane, written, or NULL), g_omega += d/d omega per cell. */
typedef struct {
    const void* lam_out;
    void* lam_f;
    void* lam_source;
    double* g_omega;
    const void* f_in;
    double omega;
    const void* omega_field;
    const void* source;
    const void* ext_source;
    XlbbRules pc, ps;
} XlbbDarcySweepAdjoint;

int xlbb_darcy_sweep_adjoint(int dtype, const XlbbGrid* g, const XlbbDarcySweepAdjoint* s, void* stream);

/* lam_q += G^T lam_grad, G = xlbb_darcy_gradient with the same scale and rules. */
int xlbb_darcy_gradient_adjoint(int dtype, const XlbbGrid* g, const void* lam_grad, double scale,
                                const XlbbRules* rules, void* lam_q, void* stream);

/* lam_f += adjoint of eta (without forces) and of the divergence moment;
 * g_lam / g_mu += derivative of the divergence scale (need f). */
int xlbb_elast_moments_adjoint(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat, const void* f,
                               const void* lam_eta, const void* lam_div, double div_scale, void* lam_f,
                               double* g_lam, double* g_mu, void* stream);

/* lam_f += adjoint of rho (without sources) and of grad = -3 omega sum c f;
 * g_omega += d/d omega (needs f). */
int xlbb_darcy_moments_adjoint(int dtype, const XlbbGrid* g, const void* f, double omega,
                               const void* omega_field, const void* lam_rho, const void* lam_grad, void* lam_f,
                               double* g_omega, void* stream);

/* Transpose of a multigrid level's Biot coupling force
 * ext = fe + G(div(f), scale) (xlbb_darcy_gradient of xlbb_elast_moments'
 * divergence, with the gradient's rules): lam_f += div^T G^T lam_ext,
 * lam_fe += lam_ext (if not NULL), g_lam / g_mu += derivative of the
 * divergence scale (need the forward f).  One kernel. */
int xlbb_divgrad_adjoint(int dtype, const XlbbGrid* g, const XlbbElastMaterial* mat, const void* lam_ext,
                         double scale, const XlbbRules* rules, const void* f, void* lam_f, void* lam_fe,
                         double* g_lam, double* g_mu, void* stream);

/* Deterministic FP64 sum of n partials (fixed order) into *out. */
int xlbb_reduce_sum(const double* partials, int n, double* out, void* stream);

/* Sum of squares of nplanes planes over a box, into partials[] (one per CTA; see
 * xlbb_sumsq_ctas) -- the norm of substract/residual fields at any level. */
int xlbb_sumsq(int dtype, const XlbbGrid* g, int nplanes, const void* data,
               int bx0, int bx1, int by0, int by1, double* partials, void* stream);
int xlbb_sumsq_ctas(const XlbbGrid* g);

/* out = a*x + b*y elementwise over n elements (n contiguous elements). */
int xlbb_axpby(int dtype, long long n, double a, const void* x, double b, const void* y,
               void* out, void* stream);

const char* xlbb_last_error(void);
int xlbb_version(void);

#ifdef __cplusplus
}
#endif
#endif /* XLBB_H */
