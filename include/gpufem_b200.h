/*
 * gpufem_b200 — C-ABI of the B200 (sm_100a) implementation of gpufem's hot path:
 * per-element stiffness integration (Q4, Q8, Brick8, Brick20), scatter of Ke into a
 * column-major ELL matrix, and the ELL SpMV / dot / axpy loop of (preconditioned) CG.
 *
 * Every entry point takes plain pointers and sizes, returns a gf_status, never aborts
 * and never exits.  gf_last_error() gives the message of the last failure on a context.
 * One context owns one CUDA stream and all device memory it allocates; contexts are
 * independent (no global state) and a context must be driven by one host thread at a
 * time.  Calls are synchronous unless the name says otherwise.
 *
 * Reference interfaces replaced (paths within fpaboim/gpufem):
 *   FemData::Init                    src/FEM/FemData.cc:122-194      -> gf_mesh_create
 *   femColor (METIS dual + greedy)   src/FEM/femColor.cc:79-191      -> gf_mesh_color
 *   StiffAlgo::CalcGlobalStiffness   src/FEM/StiffAlgo.h:46          -> gf_assemble
 *     (StiffAlgoCPU.cc:58-284, StiffAlgoGpuOmp.cc:49-323, gpuFEM_*.cl)
 *   ELLmatrix storage                src/SPRmatrix/ELLmatrix.h:35-89 -> gf_ell_view / gf_ell_download
 *   FEM::ApplyConstraint             src/FEM/fem.cc:112-167          -> gf_apply_constraints
 *   FemData::CalcForceVector         src/FEM/FemData.cc:370-385      -> gf_set_nodal_loads
 *   ELLmatrix::Axy / AxyGPU          src/SPRmatrix/ELLmatrix.cc:194-285 -> gf_spmv
 *   SPRmatrix::CG / CPU_CG / SolveCgGpu  SPRmatrix.cc:374-480, ELLmatrix.cc:289-459 -> gf_solve
 *   SPRmatrix::SetElem/AddElem/GetElem   SPRmatrix.h:71-73           -> gf_ell_upload (host-built ELL)
 */
#ifndef GPUFEM_B200_H_
#define GPUFEM_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define GF_API __attribute__((visibility("default")))
#else
#define GF_API
#endif

typedef enum gf_status {
  GF_OK = 0,
  GF_ERR_INVALID_ARG = 1,   /* bad pointer, size, enum or mesh data            */
  GF_ERR_OOM = 2,           /* device or pinned allocation failed               */
  GF_ERR_NOT_CONVERGED = 3, /* iteration or time cap reached before tolerance   */
  GF_ERR_STALLED = 4,       /* solver made no progress / breakdown (p.Ap <= 0)  */
  GF_ERR_CUDA = 5,          /* a CUDA runtime call failed                       */
  GF_ERR_STATE = 6,         /* call out of order (e.g. assemble before mesh)    */
  GF_ERR_UNSUPPORTED = 7    /* mesh outside the kernels' limits                 */
} gf_status;

/* Element families, same numbering idea as FileIO::ElemType (src/Utils/fileIO.h:40-46)
 * but 0-based.  Node order within an element is the reference's natural-coordinate
 * order (src/FEM/StiffAlgo.cc:47-202); connectivity is 1-based as in FileIO/FemData. */
typedef enum gf_elem_type { GF_Q4 = 0, GF_Q8 = 1, GF_BRICK8 = 2, GF_BRICK20 = 3 } gf_elem_type;

/* 2-D constitutive law (FemData::CalcConstituitiveData, src/FEM/FemData.cc:322-365).
 * Ignored for 3-D elements. */
typedef enum gf_analysis { GF_PLANE_STRESS = 0, GF_PLANE_STRAIN = 1 } gf_analysis;

/* Value type of an assembled matrix / vector. */
typedef enum gf_dtype { GF_F64 = 0, GF_F32 = 1 } gf_dtype;

/* Scatter schedule of gf_assemble. */
typedef enum gf_scatter {
  GF_SCATTER_COLOR = 0,  /* colour classes in turn, plain read-modify-write (no atomics) */
  GF_SCATTER_ATOMIC = 1, /* all elements at once, red.global.add into K               */
  GF_SCATTER_OWNER = 2,  /* owner computes: each CTA owns a node range, sums the blocks
                            of its rows in shared memory and writes every K entry once
                            (no colouring, no global atomics, no zero-fill)            */
  GF_SCATTER_AUTO = 3    /* the fastest of the above for the element type, as measured
                            on B200: OWNER for Q4 and Q8, ATOMIC for Brick8 and Brick20
                            (OWNER with GF_ENGINE_TF32_MMA)                           */
} gf_scatter;

/* Element-integration engine of gf_assemble (FP32 only; FP64 always uses CUDA cores). */
typedef enum gf_engine {
  GF_ENGINE_CUDA_CORE = 0, /* FP32/FP64 FMA                                             */
  GF_ENGINE_TF32_MMA = 1   /* per-element Gram matrix M = G diag(w) G^T on tensor cores
                              (mma.sync TF32, three products hi*hi + hi*lo + lo*hi,
                              FP32 accumulate; within the FP32 tolerance).  Colour and
                              atomic schedules only (AUTO picks atomic); OWNER returns
                              GF_ERR_UNSUPPORTED.  Slower than CUDA cores on B200.    */
} gf_engine;

/* Constraint treatment (FEM::ConstraintMode, src/FEM/fem.h:51-54). */
typedef enum gf_bc_mode {
  GF_BC_PENALTY = 0,     /* reference PEN: K_dd <- (1e4 * max_i K_ii) * K_dd, f unchanged */
  GF_BC_ELIMINATION = 1  /* symmetric elimination: zero row+column, K_dd = 1, f_d = 0     */
} gf_bc_mode;

typedef enum gf_solver {
  GF_SOLVER_CG = 0,          /* reference CPU_CG semantics: plain CG, x0 = 0, stop on
                                r.r <= eps^2 * r0.r0; runs in the dtype of `matrix`      */
  GF_SOLVER_PCG = 1,         /* Jacobi-preconditioned CG in the dtype of `matrix`        */
  GF_SOLVER_MIXED_PCG = 2,   /* Jacobi-PCG whose SpMVs read the FP32 matrix K32, with
                                FP64 vectors and FP64 residual replacement on K64
                                (r = f - K64 u) every 10x drop; finishes in FP64 PCG when
                                the true residual stops falling. Needs K64 and K32.       */
  GF_SOLVER_LEARNED_FCG = 3, /* FP64 flexible CG on K64 with the learned (message-passing)
                                preconditioner, falling back to Jacobi-PCG when it breaks
                                down or stalls. Needs K64 and gf_lp_init.                 */
  GF_SOLVER_MIXED_PCG32 = 4, /* as MIXED_PCG with FP32 vectors as well (half the vector
                                traffic; for moderately conditioned systems)              */
  GF_SOLVER_TWOLEVEL_PCG = 5, /* PCG with the two-level preconditioner (gf_twolevel_setup);
                                needs a mesh-built pattern.  matrix = GF_F64: FP64 PCG on
                                K64; GF_F32: SpMVs on K32 with FP64 vectors and reliable
                                updates on K64 as in MIXED_PCG (needs K64 and K32)       */
  GF_SOLVER_TWOLEVEL_PCG32 = 6 /* two-level PCG with the recursion in FP32 (K32 SpMVs, FP32
                                vectors, FP64 dot products and scalars) and FP64 reliable
                                updates r = f - K64 u; needs K64 and K32 (matrix ignored) */
} gf_solver;

typedef struct gf_solve_opts {
  int32_t solver;        /* gf_solver                                              */
  int32_t matrix;        /* gf_dtype used by CG / PCG                              */
  int32_t max_iter;      /* total inner iterations cap (0 -> 10000)                */
  double tol;            /* relative residual target ||f - K u|| / ||f||           */
  double inner_tol;      /* MIXED/LEARNED: inner relative reduction per refinement
                            step (0 -> 1e-4)                                        */
  int32_t max_outer;     /* MIXED/LEARNED: refinement steps cap (0 -> 50)          */
  int32_t check_every;   /* iterations between host convergence checks (0 -> 16)   */
  double max_seconds;    /* wall-time cap (0 -> none)                               */
} gf_solve_opts;

typedef struct gf_solve_info {
  int32_t iterations;    /* inner iterations performed (all refinement steps)      */
  int32_t outer;         /* refinement steps (MIXED/LEARNED), else 1               */
  int32_t fallback;      /* LEARNED: 1 if Jacobi-PCG took over                      */
  int32_t status;        /* gf_status of the solve                                  */
  double rel_residual;   /* final ||f - K u|| / ||f|| in FP64 on the FP64 matrix
                            (in the matrix dtype for CG / PCG on FP32)              */
  double seconds;        /* device time of the solve                                */
} gf_solve_info;

typedef struct gf_ctx gf_ctx;

/* ---- context ------------------------------------------------------------------ */
GF_API gf_status gf_create(gf_ctx** ctx, int32_t device);
GF_API gf_status gf_destroy(gf_ctx* ctx);
GF_API const char* gf_last_error(const gf_ctx* ctx);
GF_API const char* gf_version(void);
/* Device time (seconds) of the last timed phase: assemble, spmv, solve or lp_apply. */
GF_API double gf_last_device_seconds(const gf_ctx* ctx);
/* The last gf_assemble split by kernel (device seconds): for GF_SCATTER_OWNER the
 * geometry kernel and the owner kernel; for the other schedules 0 and the whole. */
GF_API gf_status gf_last_assembly_split(const gf_ctx* ctx, double* geometry_seconds,
                                        double* scatter_seconds);
/* Kernel launches issued by this context since creation (for accounting). */
GF_API int64_t gf_kernel_launches(const gf_ctx* ctx);
/* Synchronise the context's stream. */
GF_API gf_status gf_sync(gf_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that order their own work
 * with the context's: work they enqueue on it runs between the context's calls. */
GF_API gf_status gf_stream(gf_ctx* ctx, void** stream);

/* ---- mesh (FemData::Init) --------------------------------------------------------
 * coords: nnodes*dim doubles, packed xy / xyz (dim = 2 for Q4/Q8, 3 for bricks).
 * connect: nelem*nen int32, 1-based node ids, element-major.
 * ngauss: Gauss points per direction, 2 or 3 (FemData::CalcGaussVectors).
 * E_elem: nelem Young's moduli, or NULL for the scalar E.  Replaces any previous mesh. */
GF_API gf_status gf_mesh_create(gf_ctx* ctx, int32_t elem_type, int32_t nnodes,
                                const double* coords, int32_t nelem,
                                const int32_t* connect, int32_t ngauss, double E,
                                const double* E_elem, double nu, int32_t analysis);
/* Update per-element moduli (or the scalar E when E_elem is NULL) without
 * rebuilding the pattern. */
GF_API gf_status gf_mesh_set_modulus(gf_ctx* ctx, double E, const double* E_elem);

/* Colour schedule for GF_SCATTER_COLOR.  elem_color: nelem colours (0-based) from the
 * caller, or NULL to compute the reference's greedy first-fit colouring of the element
 * dual graph (elements sharing >= 1 node are adjacent; femColor.cc:103-191).  Returns
 * the number of colours.  A caller colouring is validated (no two elements of a colour
 * share a node) and rejected with GF_ERR_INVALID_ARG otherwise. */
GF_API gf_status gf_mesh_color(gf_ctx* ctx, const int32_t* elem_color, int32_t* ncolors);
/* Colour on the device instead (Jones–Plassmann rounds with pseudo-random priorities
 * from `seed`, first-fit colours; at most 256 colours).  Same validity as gf_mesh_color,
 * usually a few more colours than the greedy host order, no host pass over the dual
 * graph.  Builds the ELL pattern first if needed (it walks the node incidence lists).
 * No reference counterpart beyond femColor's role (femColor.cc:79-191). */
GF_API gf_status gf_mesh_color_device(gf_ctx* ctx, uint64_t seed, int32_t* ncolors);
/* Copy the colour of each element (0-based) to host. */
GF_API gf_status gf_mesh_get_colors(gf_ctx* ctx, int32_t* elem_color);

/* ---- ELL pattern (symbolic) --------------------------------------------------------
 * Topological pattern: row r (dof of node a) holds every dof of every node sharing an
 * element with a, columns strictly increasing.  Column-major: entry (row, slot) at
 * slot*n + row.  width = max row length.  Slots past rownnz hold col = row, value 0.  */
GF_API gf_status gf_ell_build_pattern(gf_ctx* ctx, int32_t* n, int32_t* width,
                                      int64_t* nnz);

/* ---- numeric assembly (StiffAlgo::CalcGlobalStiffness) ------------------------------
 * Computes Ke = sum_gp B^T D B detJ w for every element and scatters it into the ELL
 * values of dtype `dtype`.  Builds the pattern and the colouring on first use.  */
GF_API gf_status gf_assemble(gf_ctx* ctx, int32_t dtype, int32_t scatter, int32_t engine);
/* Round the FP64 matrix into the FP32 matrix (same pattern). */
GF_API gf_status gf_ell_convert_f64_to_f32(gf_ctx* ctx);

/* Device pointers of the assembled matrix (owned by the context). */
GF_API gf_status gf_ell_view(gf_ctx* ctx, int32_t dtype, int32_t* n, int32_t* width,
                             const int32_t** rownnz, const int32_t** colidx,
                             const void** values);
/* Version of the values of the matrix of `dtype`: a per-context counter that grows every
 * time those values change (assembly, constraints, conversion, upload).  No counterpart in
 * the reference, whose ELLmatrix lives in host memory: a host-side cache of the device
 * matrix (the reference-side ELLmatrixCUDA adapter) compares it to tell that it is stale. */
GF_API gf_status gf_ell_version(gf_ctx* ctx, int32_t dtype, int64_t* version);
/* Copy to host: rownnz[n], colidx[n*width], values[n*width] (dtype-sized). */
GF_API gf_status gf_ell_download(gf_ctx* ctx, int32_t dtype, int32_t* rownnz,
                                 int32_t* colidx, void* values);
/* Diagonal K(i, i) of the matrix of `dtype` into a host buffer of n doubles (0 where a row
 * has no diagonal entry); the device-side form of the reference's GetElem(i, i) scan
 * (SPRmatrix::GetElem, src/SPRmatrix/ELLmatrix.cc:142-159). */
GF_API gf_status gf_ell_diagonal(gf_ctx* ctx, int32_t dtype, double* diag);
/* Replace the matrix with a host-built ELL (n, width, rownnz, colidx, FP64 values);
 * fills both the FP64 and FP32 matrices.  Slots past rownnz are ignored. */
GF_API gf_status gf_ell_upload(gf_ctx* ctx, int32_t n, int32_t width,
                               const int32_t* rownnz, const int32_t* colidx,
                               const double* values);

/* ---- loads and constraints ----------------------------------------------------------
 * supports: nsup rows of (dim+1) int32: node id (1-based), then 1 = fixed per component
 * (FileIO::extractNodeSupports layout).  loads: nload rows of (dim+1) doubles: node id,
 * then force components; a nonzero component SETS f[dof] (CalcForceVector semantics). */
GF_API gf_status gf_set_supports(gf_ctx* ctx, int32_t nsup, const int32_t* supports);
GF_API gf_status gf_set_nodal_loads(gf_ctx* ctx, int32_t nload, const double* loads);
/* Full right-hand side (n doubles), replacing the nodal loads. */
GF_API gf_status gf_set_force(gf_ctx* ctx, const double* f);
GF_API gf_status gf_get_force(gf_ctx* ctx, double* f);
/* Apply the supports to the assembled matrices present (FP64 and/or FP32). */
GF_API gf_status gf_apply_constraints(gf_ctx* ctx, int32_t mode);

/* ---- solve --------------------------------------------------------------------------- */
/* y = K x on device pointers of dtype `dtype` (x, y: n entries; x 16-byte aligned, as
 * every device allocation is: 2-D meshes read x in pairs, GF_ERR_INVALID_ARG otherwise). */
GF_API gf_status gf_spmv(gf_ctx* ctx, int32_t dtype, const void* x, void* y);
/* Host-buffer SpMV (n doubles in, n doubles out), computed in `dtype`. */
GF_API gf_status gf_spmv_host(gf_ctx* ctx, int32_t dtype, const double* x, double* y);
GF_API gf_status gf_solve(gf_ctx* ctx, const gf_solve_opts* opts, gf_solve_info* info);
/* Solution of the last solve (n doubles). */
GF_API gf_status gf_get_solution(gf_ctx* ctx, double* u);
/* r = f - K64 (u_hi + u_lo) in double-double arithmetic (compensated products and sums,
 * rounded to FP64 once), for iterative refinement of a solution held as an unevaluated sum
 * of two doubles; the residual r = b - A x that SPRmatrix::CPU_CG (SPRmatrix.cc:405-480)
 * starts from, computed accurately enough to certify solutions whose true residual is
 * below FP64 roundoff of K u.  u_hi, u_lo and r are DEVICE pointers (n doubles, on this
 * context's device); f is the context's force vector.  rel_residual (host, may be NULL)
 * receives ||r|| / ||f||. */
GF_API gf_status gf_residual_dd(gf_ctx* ctx, const double* u_hi, const double* u_lo, double* r,
                                double* rel_residual);
/* Device pointer of the FP64 solution. */
GF_API gf_status gf_solution_view(gf_ctx* ctx, const double** u);

/* ---- learned preconditioner (no counterpart in the reference) ---------------------------
 * M(r) = D^-1 r + c * y, c = rms(D^-1 r), y from a 3-layer message-passing network over
 * the node graph of K (nodes sharing an element).  Per-node input features (4*dim):
 * rho/c, v1/c, v2/c, log(d/geomean d) with rho = D^-1 r, v1 = D^-1 K rho, v2 = D^-1 K v1.
 * Input layer (4*dim -> 64), three layers h' = relu(Ws h + Wn mean_neighbours(h) + b)
 * (hidden width 64), output layer (64 -> dim) initialised to zero (an untrained network
 * is Jacobi).  Weights are BF16 in use with an FP32 master copy; activations and
 * accumulation are FP32.  Used by GF_SOLVER_LEARNED_FCG.
 * Parameter layout: W0[64][4 dim], b0[64], then per layer Ws[64][64], Wn[64][64], b[64],
 * then Wout[dim][64], bout[dim]. */
#define GF_LP_LOSS_ERROR 0    /* sum d (M(r) - e)^2 / sum d e^2 (default) */
#define GF_LP_LOSS_RESIDUAL 1 /* sum (K (e - M(r)))^2 / d / sum (K e)^2 / d */
GF_API int64_t gf_lp_num_params(int32_t dim);
GF_API gf_status gf_lp_init(gf_ctx* ctx, int32_t dim, uint64_t seed);
GF_API gf_status gf_lp_get_weights(gf_ctx* ctx, float* w);
GF_API gf_status gf_lp_set_weights(gf_ctx* ctx, const float* w);
/* Training pairs (r_k, e_k = u* - x_k) from Jacobi-PCG on the current FP64 matrix and
 * force: one pair every `every` iterations of a run to `tol`, up to npairs (u* from a run
 * to tol * 1e-3).  Replaces previously collected pairs. */
GF_API gf_status gf_lp_collect(gf_ctx* ctx, int32_t npairs, int32_t every, double tol,
                               int32_t max_iter);
/* Random training pairs: e_k = xi / sqrt(d) with xi standard normal (counter-based,
 * from seed), r_k = K e_k.  Errors white in the D-norm make the error loss weigh every
 * eigenmode of D^-1 K alike (a sparse-approximate-inverse objective).  Replaces
 * previously collected pairs; GF_ERR_UNSUPPORTED with the coarse correction on. */
GF_API gf_status gf_lp_collect_random(gf_ctx* ctx, int32_t npairs, uint64_t seed);
/* Adam steps (lr, batch pairs per step) on the collected pairs with the loss chosen by
 * gf_lp_set_loss (d = diag K).  *final_loss = mean loss of the last step. */
GF_API gf_status gf_lp_train(gf_ctx* ctx, int32_t steps, int32_t batch, float lr, uint64_t seed,
                             float* final_loss);
/* z = M(r) on FP32 device vectors of n entries; gf_last_device_seconds then gives the
 * device time of this one application. */
GF_API gf_status gf_lp_apply(gf_ctx* ctx, const float* r, float* z);
/* on != 0: the learned preconditioner works with the two-level coarse correction
 * (gf_twolevel_setup): gf_lp_collect records its pairs from two-level PCG runs with the
 * coarse correction of each residual taken off the error (the network learns what the
 * coarse space misses), and GF_SOLVER_LEARNED_FCG applies M(r) + P Ac^-1 P^T r, falling
 * back to two-level PCG.  Needs a mesh-built pattern. */
GF_API gf_status gf_lp_set_coarse(gf_ctx* ctx, int32_t on);
/* Training loss (GF_LP_LOSS_*) of gf_lp_train and gf_lp_loss_grad.  The residual loss
 * weighs the error by K D^-1 K instead of D: it rewards reducing the rough part of the
 * error, the part a local operator can reach. */
GF_API gf_status gf_lp_set_loss(gf_ctx* ctx, int32_t loss);
/* Loss of one (r, e) pair (FP32 device vectors) and its gradient w.r.t. every parameter
 * (host buffer of gf_lp_num_params floats, or NULL); weights unchanged. */
GF_API gf_status gf_lp_loss_grad(gf_ctx* ctx, const float* r, const float* e, float* loss,
                                 float* grad);

/* ---- two-level preconditioner (no counterpart in the reference) ------------------------
 * M r = D^-1 r + P (P^T K P)^-1 P^T r.  Nodes are grouped into aggregates by the boxes of a
 * regular grid over the mesh's bounding box (box side s chosen so that the coarse space has
 * at most target_coarse unknowns); P holds, per aggregate, its dim translations and
 * dim(dim-1)/2 rotations about the aggregate's centroid c (offsets (x - c) / s), with the
 * rows of constrained dofs zero.  P^T K P is assembled and inverted on the device (FP64,
 * regularised by 1e-10 * its largest diagonal entry; a zero diagonal entry becomes 1).  Built
 * for the current FP64 matrix and supports; rebuilt by the next TWOLEVEL_PCG solve after
 * either changes.  target_coarse 0 = n / 128 within [192, 3072]; at most 4096.  *ncoarse may be NULL. */
GF_API gf_status gf_twolevel_setup(gf_ctx* ctx, int32_t target_coarse, int32_t* ncoarse);
/* z = M r on HOST vectors of n doubles (builds the coarse space if needed). */
GF_API gf_status gf_twolevel_apply(gf_ctx* ctx, const double* r, double* z);
/* Aggregate (0-based, in box order) of every node, and the box side s. */
GF_API gf_status gf_twolevel_aggregates(gf_ctx* ctx, int32_t* node_agg, double* box_side);

/* ---- sharded solve ----------------------------------------------------------------------
 * No counterpart in the reference (it runs one device).  One context per rank holds the
 * rank's local mesh — its owned nodes first, then a halo of the nodes its elements share
 * with other ranks — assembled as usual, so the owned rows of K are exact.  gf_dist_pcg is
 * Jacobi-PCG over the owned dofs (x0 = 0, stop when r.r <= tol^2 b.b summed over ranks)
 * with every vector and scalar on the device and no host synchronisation per iteration:
 * the caller's callbacks enqueue the collectives on the context's stream (`stream`,
 * a cudaStream_t) and return at once (non-zero return = failure).
 *   gf_allreduce_fn: sum `count` doubles at the device address in place over all ranks.
 *   gf_halo_fn: send the packed owned values `send` (n_send doubles, in the order of
 *     send_dofs) to the ranks that hold them as halo, and receive the halo values `recv`
 *     (n_recv doubles, in the order of recv_dofs).
 * Every rank must call gf_dist_pcg with the same options; all ranks then make the same
 * callbacks in the same order and stop at the same iteration.  The solution (owned dofs;
 * halo dofs 0) is read with gf_get_solution; info->rel_residual is the recursive one. */
typedef int32_t (*gf_allreduce_fn)(double* values, int32_t count, void* stream, void* user);
typedef int32_t (*gf_halo_fn)(const double* send, double* recv, void* stream, void* user);
/* send_dofs: owned local dofs whose values the neighbours need, packed per neighbour as
 * the caller's halo callback expects; recv_dofs: halo local dofs filled from them. */
GF_API gf_status gf_dist_set_halo(gf_ctx* ctx, int32_t n_owned, int32_t n_send,
                                  const int32_t* send_dofs, int32_t n_recv,
                                  const int32_t* recv_dofs);
GF_API gf_status gf_dist_pcg(gf_ctx* ctx, const gf_solve_opts* opts, gf_allreduce_fn allreduce,
                             gf_halo_fn halo, void* user, gf_solve_info* info);

/* ---- allocation-free solve -------------------------------------------------------------
 * No counterpart in the reference.  FP64 Jacobi-PCG (x0 = 0, stop when the recursive
 * residual satisfies r.r <= tol^2 b.b, or after max_iter iterations) for callers that
 * cannot allocate GPU memory: applications whose framework hands out every device byte
 * from its own arena, or loops in which a cudaMalloc/cudaFree and the device-wide
 * synchronisation it can cause are not allowed.  It allocates nothing and takes no
 * context: every pointer is a caller-owned DEVICE buffer (the column-major ELL matrix as
 * gf_ell_view describes it, b and x of n doubles) and `stream` is the caller's CUDA stream
 * (NULL = legacy default stream).  Its work vectors live in one fixed __device__ array
 * sized for n <= GF_PCG_NOALLOC_MAX_N (about 10.5 MB, held by every GPU that loads the
 * library until the process exits); larger n returns GF_ERR_INVALID_ARG, and so does an
 * ELL whose row lengths fall outside [0, width] or whose stored columns fall outside
 * [0, n) (checked on the device before the solve starts).  All calls share
 * that array: calls whose GPU work overlaps (other streams, other threads) race.  The first
 * call on a device looks up the array's address (cudaGetSymbolAddress) and should come
 * before any stream capture.  Returns when done; *iterations and *rel_residual (true FP64
 * ||b - K x|| / ||b||) may be NULL. */
#define GF_PCG_NOALLOC_MAX_N 262144
GF_API gf_status gf_pcg_noalloc(int32_t n, int32_t width, const int32_t* rownnz,
                                const int32_t* colidx, const double* values, const double* b,
                                double* x, double tol, int32_t max_iter, void* stream,
                                int32_t* iterations, double* rel_residual);

#ifdef __cplusplus
}
#endif
#endif /* GPUFEM_B200_H_ */
