/* hfk.h - C ABI of the B200 engine for HyperFEMKernels' hot path.
 *
 * The reference (MultiSimOLab/HyperFEMKernels.jl) is Julia; its host side keeps capturing and
 * lowering the Gridap weak form and calls these functions with `ccall` in place of its own
 * element loops. Citations are file:line in the reference repository.
 *
 * Conventions (those of the reference's arrays, so that Julia passes them without copies):
 *  - arrays are column-major with the reference's logical shapes;
 *  - cell_dof_ids is (ndl, ncells) Int32 with ndl = 3*nn and ldof = c*nn + n (the CONTIG layout of
 *    FieldTable, src/tables.jl:181-182); > 0 = free dof id (1-based), < 0 = -(Dirichlet index);
 *  - free-dof vectors have length nfree, Dirichlet vectors length ndir;
 *  - CSC patterns are Julia's SparseMatrixCSC{Float64,Int}: colptr/rowval Int64 1-based;
 *  - every vector argument may be a host pointer or a device pointer (CUDA device or managed
 *    memory); the library detects which and copies host data through its own device buffers;
 *  - every function returns HFK_OK (0) or an error code; hfk_last_error() gives the message,
 *    prefixed "HyperFEMKernels: " like the reference's exceptions;
 *  - numerical failure (a non-finite tangent, an indefinite level) is a status output, not an
 *    error code (src/pmultigrid.jl:331-335, src/solvers.jl:114-121);
 *  - a handle is not reentrant: calls on one handle must not overlap (src/assembly.jl:363-367).
 *    Each handle launches on its own CUDA stream (hfk_problem_set_stream to choose it).
 */
#ifndef HFK_H
#define HFK_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HFK_OK 0
#define HFK_ERR_ARG 1
#define HFK_ERR_CUDA 2
#define HFK_ERR_STATE 3
#define HFK_ERR_UNSUPPORTED 4
#define HFK_ERR_NUMERIC 5
#define HFK_ERR_PATTERN 6
#define HFK_ERR_INTERNAL 7

/* pointwise laws the host recognised from the captured tree (src/tree.jl:253-283) */
#define HFK_LAW_SVK 1            /* St Venant-Kirchhoff P(F) = F S(E); params lambda, mu[, body x y z] */
#define HFK_LAW_LINEAR_ELASTIC 2 /* sigma = lambda tr(H) I + mu (H + H'); params lambda, mu[, body] */

/* matrix-free formulations */
#define HFK_MF_STORED 0    /* reference partial assembly: T, inv(Jt), dV stored per point (src/matrixfree.jl:14-23) */
#define HFK_MF_RECOMPUTE 1 /* tangent re-evaluated from the state at every product (no per-point storage) */

typedef struct hfk_problem hfk_problem;
typedef struct hfk_transfer hfk_transfer;
typedef struct hfk_pmg hfk_pmg;

/* Message of the last error on this thread. */
const char* hfk_last_error(void);
/* Library version (major*10000 + minor*100 + patch). */
int hfk_version(void);

/* ---- operator: one volume group of a 3-component Lagrangian field on hexahedra ----------------
 * Replaces the construction of KernelOperator (src/assembly.jl:630-666) for a group whose law the
 * host recognised: the field layout (FieldLayout/cell_dof_matrix, src/assembly.jl:20-30,
 * src/tables.jl:329-342), the geometry (GeoTable, src/tables.jl:42-106), the reference tables
 * (FieldTable, src/tables.jl:171-237), and the tensor-product structure found numerically from xq
 * and Nt (TPTable, src/tensorproduct.jl:55-91). Cells are coloured at construction
 * (color_cells, src/coloring.jl:4-28).
 *   nn nodes per cell (Q^3), np quadrature points (P^3), ng geometry nodes (8: trilinear map)
 *   xq (3, np) reference points; w (np) weights; Nt (nn, np); dNt (nn, 3, np); dMt (ng, 3, np)
 *   coords (3, ng, ncells) vertex coordinates; cell_dof_ids (3*nn, ncells) */
int hfk_problem_create(hfk_problem** out, int nn, int np, int ng, int ncells, const double* xq, const double* w,
                       const double* Nt, const double* dNt, const double* dMt, const double* coords,
                       const int32_t* cell_dof_ids, int64_t nfree, int64_t ndir, int law, const double* params,
                       int nparams);
int hfk_problem_destroy(hfk_problem* p);
/* Cheap update(op, res, jac) of the same structure: new law parameters, tables/pattern/colours kept
 * (src/assembly.jl:693-744). */
int hfk_problem_set_params(hfk_problem* p, const double* params, int nparams);
/* Launch on `stream` (a cudaStream_t) from now on; NULL restores the handle's own stream. On
 * cudaStreamLegacy (the legacy default stream, which cannot be captured) a p-multigrid or slot over
 * this problem runs its cycle uncaptured. */
int hfk_problem_set_stream(hfk_problem* p, void* stream);
int hfk_problem_info(hfk_problem* p, int64_t* nfree, int* Q, int* P, int* ncolors, int64_t* nnz);
/* Scatter of the sum-factorised kernels (residual, products): colour by colour with plain
 * read-modify-writes (deterministic, the reference's race-free colouring, src/coloring.jl:1-3), or
 * one launch over all cells with FP64 atomics (the summation order, hence the last bit, varies
 * between runs). AUTO (default) is autotuned per kernel mode and precision on the first call (the
 * atomic or the colour-by-colour scatter, 2 or 4 warps per CTA, timed with CUDA events; on B200
 * the atomic scatter usually wins: one launch, no read of the output before the write); COLOURED
 * gives bit-reproducible results. The nodal blocks, the assembled Jacobian (one launch over all
 * cells) and the restriction of a transfer whose fine level is this problem scatter atomically
 * unless COLOURED is set. */
#define HFK_SCATTER_AUTO 0
#define HFK_SCATTER_COLOURED 1
#define HFK_SCATTER_ATOMIC 2
int hfk_problem_set_scatter(hfk_problem* p, int mode);
/* Launch shape under an explicit scatter mode (COLOURED or ATOMIC; AUTO tunes its own): kernel 0,
 * the line-mapped kernels with 2 or 4 warps per CTA (default 4); kernel 1, the point-parallel
 * matrix-free product with one cell per CTA (warps = 0) or 8 warps per CTA; kernel 2, the FP32
 * product of Q2 cells (3^3 Gauss points) with both sum-factorisation contractions as GEMMs on the
 * tensor cores (tcgen05.mma kind::tf32, operands split hi + lo for FP32 accuracy, 128 cells per
 * CTA; warps ignored); kernel 3, the matrix-free product of Q1 cells (2^3 Gauss points) by a
 * warp-synchronous kernel, 8 lanes per cell, one per point, the nodal sums by shuffles (warps
 * ignored). With kernels 2 and 3 the other kernels take the line-mapped shape of 4 warps. Under
 * AUTO the tensor-core product is a candidate of the FP32 product, kept only when its result
 * agrees with the line-mapped kernel's to 1e-5, and the Q1 kernel a candidate of every Q1 product. */
int hfk_problem_set_launch(hfk_problem* p, int kernel, int warps);
/* Kernel of the assembled Jacobian (hfk_jacobian) on 27-node cells: 0 (default) forms the element
 * blocks of a symmetric tangent (the recognised laws) on the FP64 FMA pipe, a 27 x 162 register-
 * tiled product per cell; 1 forms them on the FP64 tensor cores (mma m8n8k4 f64, 8 x 8 tiles). Both
 * give the reference's jacobian! (src/assembly.jl:918-927) to round-off; no counterpart in the
 * reference. */
int hfk_problem_set_assembly_kernel(hfk_problem* p, int kernel);
/* The batched CG (hfk_solve_cg_batched) on this operator: on = 1 (default) runs the iterations after
 * the second as one CUDA graph launch whose while node loops on the device (the iteration, captured
 * from the engine's launches, ends with a kernel that sets the loop condition: a problem still
 * active and the iteration limit not reached), so the host launches once and waits instead of
 * reading a flag count every iteration; on = 0 keeps the host-driven loop. Same iterates either
 * way. No counterpart in the reference. */
int hfk_problem_set_solve_graph(hfk_problem* p, int on);
/* The autotuner's choice for a kernel (mode 0: matrix-free product, 1: residual, 2: stored-tangent
 * product; precision HFK_FP64 / HFK_FP32): atomic = 1/0 (scatter), kernel = 0 (line-mapped: a
 * warp's lanes on the tensor lines of a few cells), 1 (point-parallel product: one thread per
 * quadrature point), 2 (the FP32 Q2 product on the tensor cores) or 3 (the warp-synchronous Q1
 * product), warps per CTA; atomic = -1 if that kernel has not run under AUTO yet. No
 * counterpart in the reference. */
int hfk_problem_tuning(hfk_problem* p, int mode, int precision, int* atomic, int* kernel, int* warps);

/* KernelFunctional (src/functionals.jl:10-27) for the recognised laws at the state (x, dvals):
 * HFK_FUNCTIONAL_ENERGY = Σ_cells Σ_q Ψ(F) dV, the stored energy (reduce = :sum; SVK
 * Ψ = μ E:E + λ/2 (tr E)², linear elasticity the same with E = sym ∇u; body-force work excluded:
 * it is the linear term of the load vector), HFK_FUNCTIONAL_MIN_DETF = min over the quadrature
 * points of det F (reduce = :min, unweighted: the injectivity check of a line search). One launch
 * of the sum-factorised cell kernel and a deterministic reduction. */
#define HFK_FUNCTIONAL_ENERGY 0
#define HFK_FUNCTIONAL_MIN_DETF 1
int hfk_functional(hfk_problem* p, const double* x, const double* dvals, int kind, double* out);
/* Number of kernels this handle launched so far (launch accounting for benchmarks). */
int hfk_launch_count(hfk_problem* p, int64_t* count);

/* Kernel timing, a measurement aid with no counterpart in the reference. With on = 1, every
 * element-kernel launch sequence of hfk_residual, hfk_jacobian, hfk_mf_apply and hfk_mf_apply_f32
 * (the cell kernels, without the zero-fill of the output) is bracketed by CUDA events on the
 * handle's stream; nothing waits on them. hfk_problem_kernel_time waits for the last one, returns
 * the summed milliseconds and the number of bracketed sequences since timing was switched on or
 * last read, and starts a new count. */
int hfk_problem_set_timing(hfk_problem* p, int on);
int hfk_problem_kernel_time(hfk_problem* p, double* ms, int64_t* count);
/* Bounded device waits of this problem's kernels that ran out since the last call (the tensor-core
 * product's waits for its MMAs; a kernel whose wait runs out skips its remaining work, frees its
 * tensor memory and returns), then cleared. 0 in a healthy run; no counterpart in the reference. */
int hfk_problem_device_errors(hfk_problem* p, int* errors);

/* FP64 throughput of the current device in TFLOP/s, measured by two microkernels on every SM:
 * the FP64 tensor-core MMA (mma m8n8k4 f64, the instruction of the assembly's element products)
 * and the FP64 FMA pipe (best of three runs each, about 0.5 s in all). The denominator of the
 * FP64 roofline fractions; no counterpart in the reference. */
int hfk_device_peak_fp64(double* dmma_tflops, double* dfma_tflops);

/* Colour of every cell, 1-based (color_cells, src/coloring.jl:4-28; bit-exact greedy first fit). */
int hfk_colors(hfk_problem* p, int32_t* color_of_cell);

/* Sparsity pattern of the Jacobian and the positions of the element entries
 * (sparsity/full_keys!/cell_positions!, src/assembly.jl:773-899). Built on the GPU;
 * identical to the reference's sorted-key construction. */
int hfk_pattern_build(hfk_problem* p, int64_t* nnz);
/* sparsity_pattern(op) (src/assembly.jl:768): colptr (nfree+1), rowval (nnz), 1-based. */
int hfk_pattern_get(hfk_problem* p, int64_t* colptr, int64_t* rowval);
/* nonzero_positions(op) (src/assembly.jl:771): (ndl*ndl, ncells) Int32, 1-based, 0 = not stored;
 * entry ii + ndl*jj of a cell = (test ii, trial jj). */
int hfk_nonzero_positions(hfk_problem* p, int32_t* nzpos);

/* residual!(b, op, x) (src/assembly.jl:909-916): b (nfree) = assembled residual at the free values
 * x and Dirichlet values dvals. FP64. */
int hfk_residual(hfk_problem* p, const double* x, const double* dvals, double* b);
/* jacobian!(A, op, x) (src/assembly.jl:918-927): nzval (nnz) of the CSC Jacobian in rowval order
 * (zero-filled, then the fused element kernels: one launch with atomic adds by default, colour by
 * colour, bit-reproducible, under HFK_SCATTER_COLOURED). FP64. */
int hfk_jacobian(hfk_problem* p, const double* x, const double* dvals, double* nzval);

/* prepare!(mf, x) / jacobian!(mf, op, x) (src/matrixfree.jl:97-100, :140-159): bind the state.
 * mode HFK_MF_STORED stores T, inv(Jt), dV per point as the reference does; HFK_MF_RECOMPUTE keeps
 * only the state and re-evaluates the tangent inside every product. */
int hfk_mf_prepare(hfk_problem* p, const double* x, const double* dvals, int mode);
/* mul!(y, mf, dx) (src/matrixfree.jl:246-260): y = J(x) dx on free dofs (Dirichlet increments zero),
 * sum-factorised. FP64. */
int hfk_mf_apply(hfk_problem* p, const double* dx, double* y);
/* The same product in FP32 (state, increment and result in FP32; mixed-precision smoothers). */
int hfk_mf_apply_f32(hfk_problem* p, const float* dx, float* y);
/* y[i] = J dx[i] for count vectors (the reference's mul! of src/matrixfree.jl:246-260, applied to
 * a stream of inputs): host vectors are copied in and out on two copy streams of their own, with
 * two staging slots per direction, so that the copies of vectors i + 1 and i - 1 overlap the
 * product of vector i (host buffers must be page-locked for the copies to overlap anything).
 * Device pointers skip their copies. The copies start after the work already queued on the
 * problem's stream, later work on it follows them, and the call returns when every y[i] is
 * written. The staging buffers (4 n doubles) are allocated on the first call. */
int hfk_mf_apply_many(hfk_problem* p, int count, const double* const* dx, double* const* y);

/* BlockJacobi nodal blocks of the prepared tangent (field_blocks/block_diagonal!/invert_blocks!,
 * src/preconditioners.jl:151-327); ok = 0 if a block is not finite. */
int hfk_blocks_update(hfk_problem* p, int* ok);
/* ldiv!(y, BlockJacobiState, r) (src/preconditioners.jl:329-344). */
int hfk_blocks_apply(hfk_problem* p, const double* r, double* y);
/* Replace the nodal blocks B (3, 3, nblocks; the numbering of hfk_blocks_get) and invert them, as
 * invert_blocks! does (src/preconditioners.jl:284-305); ok = 0 if a block is not finite. A subdomain
 * of a partitioned mesh passes its blocks summed with the other subdomains' partial blocks of the
 * nodes they share. Requires hfk_blocks_update once (it numbers the blocks). */
int hfk_blocks_set(hfk_problem* p, const double* B, int* ok);
/* Blocks as the reference stores them: dofs (3, nblocks) 1-based (0 = fixed component), B and Binv
 * (3, 3, nblocks). Any output may be NULL; nblocks is always written. */
int hfk_blocks_get(hfk_problem* p, int* nblocks, int32_t* dofs, double* B, double* Binv);

/* eigenvalue_bounds(mf, BlockJacobi; k, b) (src/preconditioners.jl:374-389): Ritz bounds of the
 * block-preconditioned tangent after k Arnoldi steps from `start` (NULL = the Chebyshev start vector
 * sin(1+0.7i)+0.3cos(2.3i), src/smoothers.jl:68-71). FP64. */
int hfk_eigenvalue_bounds(hfk_problem* p, int k, const double* start, double* lmin, double* lmax);
/* Eigenvalues (real, imaginary parts) of an n x n upper Hessenberg matrix (column-major), the eigvals
 * call of eigenvalue_bounds (src/preconditioners.jl:386); host only. */
int hfk_hessenberg_eigvals(int n, const double* H, double* re, double* im);
/* smooth!(x, ChebyshevState, rhs; zero_guess, residual) (src/smoothers.jl:116-146) on [a, b]:
 * `degree` steps; residual may be NULL. FP64. */
int hfk_chebyshev_smooth(hfk_problem* p, double a, double b, int degree, const double* rhs, double* x,
                         int zero_guess, double* residual);

/* Allocation-free smooth!: the same smoothing as hfk_chebyshev_smooth, for callers that cannot allocate
 * device memory once their solver is set up (a host drawing every GPU buffer from a fixed, pre-sized
 * pool, or an application that forbids allocation after set-up; cudaMalloc/cudaFree synchronise the
 * device and can fail once memory is committed). No counterpart in the reference. It allocates
 * nothing: its three work vectors live in one file-scope device array sized for
 * HFK_NOALLOC_MAX_DOFS free dofs (3 * 2^19 doubles = 12 MiB, held on every GPU that loads the
 * library until the process exits); larger operators are rejected with HFK_ERR_ARG. rhs, x and
 * residual (NULL allowed) must be device pointers on the operator's GPU. The launch-shape autotuner
 * does not run inside this call: a product not tuned yet runs with the default shape (atomic scatter,
 * 4 warps per CTA). The first call on a device does the set-up (it
 * resolves the array's device address with cudaGetSymbolAddress); make that first call before any
 * stream capture. Every call shares the array and starts by clearing it; calls that overlap on the
 * GPU (from other streams or threads) race on it. The call returns after the smoothing has finished. */
#define HFK_NOALLOC_MAX_DOFS 524288
int hfk_chebyshev_smooth_noalloc(hfk_problem* p, double a, double b, int degree, const double* rhs, double* x,
                                 int zero_guess, double* residual);

/* ---- transfers between nested levels on one mesh (src/transfers.jl) --------------------------
 * E (nn_f, nn_c): coarse basis at the fine nodes; Einj (nn_c, nn_f): fine basis at the coarse
 * nodes (TransferField, src/transfers.jl:57-131). When E is a tensor product E1 x E1 x E1 (checked
 * entry by entry at creation), prolongation and restriction run sum-factorised, one warp per cell. */
int hfk_transfer_create(hfk_transfer** out, hfk_problem* fine, hfk_problem* coarse, const double* E,
                        const double* Einj);
int hfk_transfer_destroy(hfk_transfer* t);
/* Replace the multiplicity of every fine free dof (the number of cells containing it, `cells_of`,
 * src/transfers.jl:27, :124-127) that the restriction divides by. A subdomain of a partitioned mesh
 * passes the counts over the whole mesh, so that its partial restrictions sum to the global one; each
 * count must be at least the number of this level's cells that contain the dof. */
int hfk_transfer_set_multiplicity(hfk_transfer* t, const int32_t* mult);
/* prolongate!(yf, P, xc) (src/transfers.jl:238-245) */
int hfk_prolongate(hfk_transfer* t, const double* xc, double* yf);
/* restrict!(yc, P, yf) (src/transfers.jl:252-259) */
int hfk_restrict(hfk_transfer* t, const double* yf, double* yc);
/* inject!(xc, dc, P, xf, df) (src/transfers.jl:285-313) */
int hfk_inject(hfk_transfer* t, const double* xf, const double* df, double* xc, double* dc);

/* ---- p-multigrid (src/pmultigrid.jl) ---------------------------------------------------------
 * levels[0] is the working level (its state is bound by hfk_pmg_update), levels[nlevels-1] the
 * assembled coarse level (solved by a Cholesky factorisation on the GPU, hand-written over the
 * band of the matrix and stored in band form, and two block triangular solves per cycle, in place
 * of the reference's LUSolver); transfers[l] goes from level l+1 to level l. Chebyshev(degree, range,
 * inflate, eig_iters) as src/smoothers.jl:21-33. precision HFK_FP64 or HFK_FP32: the arithmetic of
 * the smoothers and products on the levels above the coarse one (the coarse solve is always FP64). */
#define HFK_FP64 0
#define HFK_FP32 1
/* The hierarchy runs every level on level 0's stream while it exists; destroy it before its levels. */
int hfk_pmg_create(hfk_pmg** out, int nlevels, hfk_problem* const* levels, hfk_transfer* const* transfers,
                   int degree, double range, double inflate, int eig_iters, int coarse_every, int precision);
int hfk_pmg_destroy(hfk_pmg* m);
/* update_levels! + smoother updates (src/pmultigrid.jl:168-221, :298-313): inject the fine state
 * (x, dvals), prepare every level, extract blocks and intervals, assemble and factorise the coarse
 * level every coarse_every updates. ok = 0 when a level is not usable (NaN tangent, indefinite). */
int hfk_pmg_update(hfk_pmg* m, const double* x, const double* dvals, int* ok);
/* ldiv!(y, PMultigridState, r) (src/pmultigrid.jl:316-338): one V-cycle; NaN when not ok. */
int hfk_pmg_vcycle(hfk_pmg* m, const double* r, double* y);
/* Counters and times (ms) of a hierarchy: out[9] = updates, coarse factorisations, V-cycles, time in
 * updates, in coarse assembly + factorisation, in block extraction, in eigenvalue estimates, in
 * V-cycles, in the Cholesky factorisation alone. The
 * V-cycle is replayed from a CUDA graph captured on the second cycle after each update. Cycles run
 * inside the device-driven loop of a batched solve (hfk_problem_set_solve_graph) are counted but
 * not timed (a graph loop body holds no events). */
int hfk_pmg_stats(hfk_pmg* m, double* out);
/* State of the last update: ok (preconditioner_ok, src/solvers.jl:105-106) and, when it failed,
 * whether it met an indefinite tangent: finite nodal blocks and a finite Ritz estimate with a
 * non-positive value on some smoothing level (preconditioner_indefinite, src/pmultigrid.jl:342-343,
 * the signal a Newton with a switching tangent reads). hfk_solve_cg reports the same flag in
 * `indefinite` when it returns without iterating on a failed preconditioner. */
int hfk_pmg_status(hfk_pmg* m, int* ok, int* indefinite);
/* Interval and Ritz values of a level's smoother (with segments: the extreme Ritz values over the
 * segments and the interval of the largest). */
int hfk_pmg_level_info(hfk_pmg* m, int level, double* lmin, double* lmax, double* a, double* b);
/* A one-level preconditioner slot on the prepared operator `op`, for hfk_solve_cg / hfk_solve_gmres
 * (the reference's preconditioner slots, src/preconditioners.jl): HFK_SLOT_LAGGED_ASSEMBLED, the
 * operator's tangent assembled on the GPU and factorised (Cholesky over the band, FP64, memory
 * about 8 n (b + 64) bytes for the lower bandwidth b) at the first update and then every `every` updates (LaggedAssembled(LUSolver();
 * every), :41-97; a stale factor between builds); HFK_SLOT_BLOCK_JACOBI, the nodal 3x3 block
 * inverses of the tangent at every update (BlockJacobi, :151-344; `every` ignored). The slot is an
 * hfk_pmg handle with one level: updated by hfk_pmg_update, applied by the solvers or
 * hfk_pmg_vcycle, builds counted by hfk_pmg_stats (out[1]), released by hfk_pmg_destroy. */
#define HFK_SLOT_LAGGED_ASSEMBLED 0
#define HFK_SLOT_BLOCK_JACOBI 1
int hfk_slot_create(hfk_pmg** out, hfk_problem* op, int kind, int every);
/* Coarse solve of the hierarchy: HFK_COARSE_CHOLESKY (default; the assembled coarse level, band
 * Cholesky, in place of the reference's LUSolver, src/pmultigrid.jl:212-219) or HFK_COARSE_CG:
 * `iters` steps of block-Jacobi CG per segment on the matrix-free coarse level from zero (scalars on
 * the device, inside the captured cycle; a variable preconditioner, so use the flexible CG). The
 * second serves hierarchies whose coarse level is too large for a direct factor (many batched
 * problems); it has no counterpart in the reference. Takes effect at the next hfk_pmg_update. */
/* Ritz values (extremes) of a level's eigenvalue estimate per segment (nseg entries each; NaN
 * for a level without a smoother or before the first update). */
int hfk_pmg_segment_bounds(hfk_pmg* m, int level, double* lmin, double* lmax);
/* Inner product of the smoothers' eigenvalue estimate: HFK_EIG_EUCLIDEAN (default; the reference's
 * Arnoldi, src/preconditioners.jl:374-389) or HFK_EIG_PRECONDITIONED: the same Arnoldi in the
 * P^-1 inner product, in which J P^-1 is self-adjoint, so that H is symmetric and the Ritz values
 * lie inside the spectrum (a Lanczos estimate). An option of this engine. Takes effect at the next
 * hfk_pmg_update. */
#define HFK_EIG_EUCLIDEAN 0
#define HFK_EIG_PRECONDITIONED 1
int hfk_pmg_set_eig_inner(hfk_pmg* m, int mode);
#define HFK_COARSE_CHOLESKY 0
#define HFK_COARSE_CG 1
int hfk_pmg_set_coarse(hfk_pmg* m, int mode, int iters);
/* Test knob of the coarse solve's bounded waits (no counterpart in the reference): the block
 * triangular solves give up a wait after `polls` polls (0 = the default of 4 194 304), and with
 * skip_first = 1 the next forward solve starts its step tickets at 1, so that step 0 never runs
 * and the steps after it wait in vain: the wait runs out, the kernel sets its error word and
 * returns, and the V-cycle returns HFK_ERR_INTERNAL ("... timed out"). Nothing faults or hangs. */
int hfk_pmg_test_coarse_wait(hfk_pmg* m, int polls, int skip_first);

/* ---- learned correction (no counterpart in the reference) ------------------------------------
 * A per-node MLP (16 -> 64 -> 64 -> 3, tanh, BF16 weights read by the forward pass, FP32 master
 * weights, FP32 accumulation) whose output delta, scaled, is added to the V-cycle's result y after
 * each cycle with the step omega = (delta . s) / (delta . A delta) per segment (s = r - A y), the
 * step that minimises the energy error of y along delta; omega = 0 (the plain cycle) when delta is
 * not a descent direction. Features per
 * node: residual after the cycle s, its block-Jacobi value, the cycle's input r and output y (each
 * group scaled by its RMS), log lambda, log mu. Training pairs (features, remaining error A^-1 s)
 * come from the plain cycle (hfk_pmg_mlp_sample); training is Adam on the GPU (hfk_mlp_train). */
typedef struct hfk_mlp hfk_mlp;
int hfk_mlp_create(hfk_mlp** out, uint64_t seed);
int hfk_mlp_destroy(hfk_mlp* m);
/* Number of parameters (flat vector: W1 (64x16 row-major), b1, W2 (64x64), b2, W3 (3x64), b3). */
int hfk_mlp_num_params(void);
int hfk_mlp_get_weights(hfk_mlp* m, float* w);
int hfk_mlp_set_weights(hfk_mlp* m, const float* w);
/* out (n x 3) = MLP(feats (n x 16)), device pointers. */
int hfk_mlp_forward(hfk_mlp* m, const float* feats, int64_t n, float* out);
/* Gradient of the mean squared error over n samples (device samples; grad may be host memory). */
int hfk_mlp_grad(hfk_mlp* m, const float* feats, const float* targets, int64_t n, float* grad, float* loss);
/* `steps` Adam steps on consecutive minibatches of `batch` samples (wrapping), learning rate lr. */
int hfk_mlp_train(hfk_mlp* m, const float* feats, const float* targets, int64_t n, int steps, int64_t batch, float lr,
                  float* last_loss);
/* Attach (or detach with NULL) the network to a hierarchy's cycle. */
int hfk_pmg_set_mlp(hfk_pmg* m, hfk_mlp* net);
/* Corrections tried and accepted since the network was attached. */
int hfk_pmg_mlp_stats(hfk_pmg* m, int64_t* tried, int64_t* accepted);
/* One set of training samples for the residual r (device): features (nblocks x 16) and targets
 * (nblocks x 3, the remaining error after the plain cycle, solved to rtol); nsamples = nblocks. */
int hfk_pmg_mlp_sample(hfk_pmg* m, const double* r, float* feats, float* targets, int* nsamples, double rtol);

/* ---- Krylov (src/solvers.jl) ----------------------------------------------------------------
 * MatrixFreeSolver.solve! (src/solvers.jl:111-159) with an FP64 (flexible) CG on the prepared
 * operator `op` preconditioned by `prec` (NULL = none): stops when ||b - J x|| <= atol + rtol ||b||
 * (true residual). flexible != 0 uses the Polak-Ribiere beta (a variable preconditioner, e.g. a
 * mixed-precision V-cycle). x is the initial guess on input. A non-positive curvature stops with
 * converged = 0 and indefinite = 1; an unusable preconditioner returns at once, iters = 0. */
/* MatrixFreeSolver.solve! with krylov = :gmres or :fgmres (src/solvers.jl:128-131; Krylov.jl's
 * gmres!/fgmres! with right preconditioning and restart): restarted GMRES on the device, classical
 * Gram-Schmidt with one reorthogonalisation, Givens rotations on the host; `restart` iterations per
 * cycle (the reference's memory, default 50). flexible != 0 is FGMRES (the preconditioned basis is
 * kept: any, also variable, preconditioner); flexible = 0 is GMRES (x += N^-1 (V y) at the end of
 * a cycle: a fixed preconditioner). Stops when ||b - J x|| <= atol + rtol ||b|| on the true
 * residual, computed at the end of every cycle. x is the initial guess on input; an unusable
 * preconditioner returns at once with iters = 0. */
int hfk_solve_gmres(hfk_problem* op, hfk_pmg* prec, const double* b, double* x, double rtol, double atol, int maxiter,
                    int restart, int flexible, int* iters, int* converged, double* relres);
int hfk_solve_cg(hfk_problem* op, hfk_pmg* prec, const double* b, double* x, double rtol, double atol, int maxiter,
                 int flexible, int* iters, int* converged, int* indefinite, double* relres);

/* ---- batched problems (no counterpart in the reference: many independent solves at once) -------
 * A problem handle may hold several independent problems ("segments") as one disjoint union of
 * meshes: segment s owns the free dofs [dof_off[s], dof_off[s+1]) and the cells
 * [cell_off[s], cell_off[s+1]) (cell_off may be NULL when params is NULL; with it, the call checks
 * that no cell of a segment touches another segment's free dofs). params (2, nseg): lambda, mu per
 * segment (NULL keeps the problem's parameters for every cell). Every kernel launch covers all
 * segments; reductions, Chebyshev intervals (eigenvalue_bounds per segment,
 * src/preconditioners.jl:374-389) and the Krylov scalars are per segment. Set the same segments on
 * every level before building a hierarchy. */
int hfk_problem_set_segments(hfk_problem* p, int nseg, const int64_t* dof_off, const int32_t* cell_off,
                             const double* params);
int hfk_problem_segments(hfk_problem* p, int* nseg);
/* Per-cell law parameters lm (2, ncells) host array (lambda, mu of each cell); NULL returns to the
 * problem's parameters. */
int hfk_problem_set_cell_params(hfk_problem* p, const double* lm);
/* out[s] = a . b over segment s (host or device pointers; out has nseg entries). */
int hfk_segment_dots(hfk_problem* p, const double* a, const double* b, double* out);
/* x[i] *= f[segment of i] (x a device vector; f host, nseg entries). */
int hfk_segment_scale(hfk_problem* p, double* x, const double* f);
/* MatrixFreeSolver.solve! (src/solvers.jl:111-159) on every segment at once: one (flexible) CG per
 * segment with its own tolerance atol + rtol ||b_s||, stopping test and curvature check, all
 * segments advancing in the same launches. iters, converged, indefinite, relres: nseg entries
 * (host); sweeps: the number of iterations of the common loop. */
int hfk_solve_cg_batched(hfk_problem* op, hfk_pmg* prec, const double* b, double* x, double rtol, double atol,
                         int maxiter, int flexible, int* iters, int* converged, int* indefinite, double* relres,
                         int* sweeps);

/* ---- Oseen–BDF step, Taylor–Hood P2–P1 on affine tetrahedra (test/common.jl:164-228) ----------
 * The volume terms of the reference's Oseen problem: a((u,p),(v,q)) with SUPG/PSPG/LSIC
 * stabilisation and l((v,q)) with the BDF history and the elementwise Laplacian of uⁿ, assembled
 * as the reference's residual!/jacobian! do (src/assembly.jl:909-927): residual = a(x, .) - l(.)
 * at the free dofs, Jacobian = the CSC nonzeros of a (the form is linear in x). Inputs:
 *   nq points, w (nq); P2 tables N2 (10, nq), dN2 (10, 3, nq), reference Hessians H2 (10, 3, 3);
 *   P1 tables N1 (4, nq), dN1 (4, 3, nq); coords (3, 4, ncells) vertices; cell_dof_ids
 *   (34, ncells): velocity c*10 + n (P2 node n: 4 vertices then the edges 01 02 03 12 13 23),
 *   pressure 30 + n; params = rho, mu, dt, bdf2 (1: BDF2 coefficients, 0: backward Euler).
 * The history uⁿ, uⁿ⁻¹ (free and Dirichlet values, trial-space numbering, pressure entries
 * ignored) gives w = 2uⁿ - uⁿ⁻¹ (BDF2), the history term f and the τ of test/common.jl:196-198. */
typedef struct hfk_oseen hfk_oseen;
int hfk_oseen_create(hfk_oseen** out, int ncells, int nq, const double* w, const double* N2, const double* dN2,
                     const double* H2, const double* N1, const double* dN1, const double* coords,
                     const int32_t* cell_dof_ids, int64_t nfree, int64_t ndir, const double* params, int nparams);
int hfk_oseen_destroy(hfk_oseen* o);
/* update(op, res, jac) for the step (src/assembly.jl:693-744): new rho, mu, dt, bdf2; tables,
 * pattern and colours kept. */
int hfk_oseen_set_params(hfk_oseen* o, const double* params, int nparams);
int hfk_oseen_set_scatter(hfk_oseen* o, int mode);
int hfk_oseen_set_history(hfk_oseen* o, const double* un, const double* und, const double* unm1, const double* unm1d);
/* sparsity (src/assembly.jl:773-818): nnz, then colptr (nfree + 1) and rowval, Int64 1-based. */
int hfk_oseen_pattern(hfk_oseen* o, int64_t* nnz);
int hfk_oseen_pattern_get(hfk_oseen* o, int64_t* colptr, int64_t* rowval);
int hfk_oseen_residual(hfk_oseen* o, const double* x, const double* dvals, double* b);
int hfk_oseen_jacobian(hfk_oseen* o, double* nzval);
int hfk_oseen_launch_count(hfk_oseen* o, int64_t* count);
/* The outlet boundary group of the reference's Oseen problem (test/common.jl:194-210):
 * -∫ ρ negpart(w·n)(u·v) dΓ (backflow) + ∫ ZA (u·n)(v·n) dΓ (Robin) in a, -∫ Pc (v·n) dΓ
 * (Windkessel pressure) in l, added to the residual and the Jacobian. Per facet: its cell, the
 * local face (opposite local vertex f), the area and the outward unit normal (3, nfacets); nq facet
 * points with weights w summing to 1 and the cell's P2 values at them for each local face,
 * N (10, nq, 4). nfacets = 0 removes the group. */
int hfk_oseen_set_outlet(hfk_oseen* o, int nfacets, const int32_t* cells, const int32_t* faces, const double* areas,
                         const double* normals, int nq, const double* w, const double* N, double Pc, double ZA);

#ifdef __cplusplus
}
#endif
#endif
