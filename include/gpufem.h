/*
 * gpufem.h — C ABI of the B200 shell-analysis hot path (libgpufem.so).
 *
 * The reference (smdogroup/gpu_fem) is a header-only C++ template library
 * with no C ABI; each entry point below replaces the member function or
 * driver step cited beside it. A C++ facade that keeps the reference's class
 * names (ElementAssembler, BsrMat, DeviceVec, HostVec, ILUk_Preconditioner)
 * lives in include/gpufem/gpufem.hpp.
 *
 * Conventions
 *  - All functions return gf_status; nothing calls exit().
 *  - Device pointers are caller-owned and never freed by the library.
 *    Handles (gf_assembler, gf_bsr, gf_precond, gf_solver, gf_batch) are
 *    library-owned and released with their destroy call.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *    Work on distinct handles may run concurrently from different threads.
 *  - Nodal vectors at the boundary are in the caller's (natural) node order,
 *    6 DOF per node, AoS (6*node + dof) as in include/linalg/vec.h:47-57.
 *    The BSR matrix is stored in the solver ordering (perm[old] = new), with
 *    6x6 row-major blocks values[36*blk + 6*r + c] (include/linalg/bsr_mat.h:217-223)
 *    and 32-bit rowPtr/colPtr (include/linalg/bsr_utils.h:16).
 *  - All assembly arithmetic is FP64.
 */
#ifndef GPUFEM_H
#define GPUFEM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gf_status {
  GF_OK = 0,
  GF_INVALID_ARG = 1,
  GF_OOM = 2,
  GF_ZERO_PIVOT = 3,
  GF_NOT_CONVERGED = 4,
  GF_NAN = 5,
  GF_TIMEOUT = 6,
  GF_CUDA_ERROR = 7,
  GF_NO_DEVICE = 8,
  GF_OVER_BUDGET = 9
} gf_status;

/* Per-element isotropic shell data; same fields and meaning as
 * ShellIsotropicData (include/shell/data.h:8-47). */
typedef struct gf_shell_data {
  double E, nu, thick, tOffset;
  double refAxis[3];
  int32_t has_ref_axis;
  int32_t pad;
} gf_shell_data;

/* Mesh description (host arrays, copied by gf_assembler_create). Replaces
 * the ElementAssembler constructor arguments (include/assembler.h:31-34). */
typedef struct gf_mesh_desc {
  int32_t num_nodes;           /* num_geo_nodes == num_vars_nodes */
  int32_t num_elements;
  const int32_t* conn;         /* 4 per element, tensor-product node order */
  const double* xpts;          /* 3 per node */
  const int32_t* bcs;          /* natural DOF indices (6*node + dof) */
  int32_t num_bcs;
  const gf_shell_data* data;   /* one per element */
  int32_t ordering;            /* GF_ORDER_* */
  int32_t rcm_root;            /* RCM root node (reference uses 0) */
  double qorder_p;             /* GF_ORDER_QORDER: window = bandwidth / p (0: p = 1) */
  uint64_t qorder_seed;        /* GF_ORDER_QORDER: seed of the window shuffles */
} gf_mesh_desc;

/* Node orderings of the solver: natural (the caller's numbering), RCM
 * (TacsComputeRCMOrder, include/linalg/reordering_utils.h:189-291, root
 * rcm_root), and q-ordering (examples/iterative/gmres.cu:159-215) made
 * deterministic: the RCM order cut into windows of floor(bandwidth / p)
 * positions (bandwidth of the RCM-ordered pattern, getBandWidth,
 * include/linalg/bsr_utils.h:655-670), each window's positions permuted by a
 * Fisher-Yates shuffle (from its last position down, position i swapped with
 * lo + x mod (i - lo + 1)) drawing x from one MT19937-64 stream seeded with
 * qorder_seed; the reference seeds from std::random_device. */
enum { GF_ORDER_NATURAL = 0, GF_ORDER_RCM = 1, GF_ORDER_QORDER = 2 };

/* GF_ASSEMBLE_ATOMIC: scatter with FP64 atomics in one launch over all
 * element chunks (the reference's scatter, include/linalg/bsr_mat.h:229-276)
 * instead of the coloured, bitwise-reproducible schedule (one launch per
 * colour); the outputs are zeroed first unless GF_ASSEMBLE_ADD is set, and
 * sums are taken in arrival order. */
enum {
  GF_ASSEMBLE_OVERWRITE = 0,
  GF_ASSEMBLE_ADD = 1,
  GF_ASSEMBLE_FUSE_BCS = 2,
  GF_ASSEMBLE_ATOMIC = 4
};

typedef struct gf_assembler gf_assembler;
typedef struct gf_bsr gf_bsr;
typedef struct gf_precond gf_precond;
typedef struct gf_batch gf_batch;

/* ---- library --------------------------------------------------------- */
const char* gf_status_string(gf_status s);
const char* gf_version(void);
/* Last CUDA error text seen by the library on this thread ("" if none). */
const char* gf_last_error(void);
/* Number of kernels the library has launched in this process (all threads). */
long long gf_launch_count(void);
/* Sweep timing for benchmarks (no reference counterpart). While enabled,
 * the two triangular-sweep launches of every preconditioner apply are
 * bracketed by CUDA events on their stream, and the sweeps add their
 * algorithmic bytes (the compulsory unique traffic: stored blocks: 36 values
 * + column index; rows: row pointer + right-hand side + result) to a device
 * counter.
 * Enabling or disabling resets the totals. Meant for a benchmark driving
 * the library from one host thread. */
gf_status gf_timing_enable(int32_t enable);
/* Totals since the last enable: event time of the sweep pairs (ms), sweep
 * launches and algorithmic bytes. Waits for the recorded events. */
gf_status gf_timing_read(double* sweep_ms, long long* sweep_launches, double* sweep_bytes);

/* ---- assembler ------------------------------------------------------- */
/* ElementAssembler(...) (include/assembler.h:31-73) + BsrData(...)
 * (include/linalg/bsr_utils.h:46-62) + post_reordering_update (:84-103).
 * Builds the block pattern, the optional RCM ordering
 * (include/linalg/reordering_utils.h:272-291), elemIndMap
 * (include/linalg/bsr_utils.h:809-870), the coloured scatter schedule and
 * uploads the mesh to the current device. */
gf_status gf_assembler_create(const gf_mesh_desc* desc, gf_assembler** out);
/* The node ordering gf_assembler_create would use for this mesh
 * (perm[natural node] = solver row, num_nodes entries). Host only: needs no
 * GPU. */
/* Which parts of the assembler's symbolic setup ran on the GPU: the node
 * pattern (get_row_col_ptrs, include/linalg/bsr_utils.h:430-476) and the
 * elemIndMap (get_elem_ind_map, :809-870); 0 where the host computed them (a
 * node with more than 64 elements, or a device failure). Any pointer may be
 * NULL. The node ordering and the scatter colouring are host algorithms. */
gf_status gf_assembler_setup_info(const gf_assembler* a, int32_t* pattern_on_gpu,
                                  int32_t* elem_map_on_gpu);
gf_status gf_order_nodes(const gf_mesh_desc* desc, int32_t* perm);
gf_status gf_assembler_destroy(gf_assembler* a);
/* get_num_nodes / get_num_elements / get_num_vars (include/assembler.h:117-118, :309-310) */
int32_t gf_assembler_num_nodes(const gf_assembler* a);
int32_t gf_assembler_num_elements(const gf_assembler* a);
int32_t gf_assembler_num_vars(const gf_assembler* a);
int32_t gf_assembler_nnzb(const gf_assembler* a);
/* BsrData public fields (include/linalg/bsr_utils.h:395-403), host copies:
 * rowPtr[nnodes+1], colPtr[nnzb], perm[nnodes] (perm[old] = new),
 * elemIndMap[16*nelems]; any pointer may be NULL. */
gf_status gf_assembler_get_pattern(const gf_assembler* a, int32_t* rowPtr, int32_t* colPtr,
                                   int32_t* perm, int32_t* elemIndMap);
/* Scatter schedule: chunk id, chunk colour, element colour and first-touch
 * mask per element; chunk colour / element colour counts. Host copies. */
gf_status gf_assembler_get_schedule(const gf_assembler* a, int32_t* elem_chunk,
                                    int32_t* chunk_color, int32_t* elem_color,
                                    uint32_t* first_touch, int32_t* num_chunk_colors,
                                    int32_t* num_chunks);
/* set_variables (include/assembler.h:191-195): d_vars is natural-order,
 * 6*num_nodes doubles on the device; copied (not referenced). */
gf_status gf_set_variables(gf_assembler* a, const double* d_vars, void* stream);
/* Replace the per-element thickness (device pointer, natural element order,
 * num_elements doubles); other material data is kept. Lets one assembler
 * (pattern, ordering, schedule) serve many thickness fields on one mesh. */
gf_status gf_assembler_set_thickness(gf_assembler* a, const double* d_thick, void* stream);
/* add_residual (include/assembler.h:232-264, kernel base/elem_group.cuh:17-97):
 * d_res (natural order) = R(u)  (or += with GF_ASSEMBLE_ADD). */
gf_status gf_add_residual(gf_assembler* a, double* d_res, int32_t flags, void* stream);
/* add_jacobian (include/assembler.h:267-305, kernel base/elem_group.cuh:103-211):
 * K(u) into the BSR values (overwrite, or += with GF_ASSEMBLE_ADD) and R(u)
 * into d_res (may be NULL). GF_ASSEMBLE_FUSE_BCS applies the Dirichlet
 * rows/columns of apply_bcs(Mat) and zeroes BC entries of d_res in the same
 * pass. */
gf_status gf_add_jacobian(gf_assembler* a, double* d_res, gf_bsr* mat, int32_t flags,
                          void* stream);
/* add_jacobian with a per-call element thickness field (device pointer,
 * natural element order) instead of the assembler's own, so one assembler
 * can assemble many thickness fields concurrently on different streams. */
gf_status gf_add_jacobian_thick(gf_assembler* a, const double* d_thick, double* d_res,
                                gf_bsr* mat, int32_t flags, void* stream);
/* add_energy (include/assembler.h:198-229; the reference GPU kernel is an
 * empty stub, base/elem_group.cuh:11-13): *h_energy = U(u). */
gf_status gf_add_energy(gf_assembler* a, double* h_energy, void* stream);
/* apply_bcs(Vec) (include/assembler.h:119-136, vec.cuh:3-13). */
gf_status gf_apply_bcs_vec(gf_assembler* a, double* d_vec, void* stream);
/* apply_bcs(Mat) (include/assembler.h:137-154, bsr_mat.cuh:1-104). */
gf_status gf_apply_bcs_mat(gf_assembler* a, gf_bsr* mat, void* stream);

/* ---- BDF mesh input -------------------------------------------------- */
/* A 4-node shell mesh read from a NASTRAN bulk-data file: the data
 * TACSMeshLoader::scanBDFFile + getAssemblerCreatorData
 * (include/mesh/TACSMeshLoader.h:188-225) hand to createFromBDF
 * (include/assembler.h:92-115). GRID / GRID* (CP = CD = 0), CQUAD4 / CQUADR
 * and SPC / SPC* entries in small-field, large-field or free-field format;
 * nodes and elements are numbered by ascending file id; element nodes are in
 * tensor order (G1 G2 G4 G3); bcs are natural DOF indices (6 node + dof).
 * component[e] is the element's property id (PID). Other element types give
 * GF_INVALID_ARG with the reason in gf_last_error. Host only. */
typedef struct gf_bdf_mesh {
  int32_t num_nodes, num_elements, num_bcs;
  const int32_t* conn;       /* 4 per element */
  const double* xpts;        /* 3 per node */
  const int32_t* bcs;        /* ascending, unique */
  const int32_t* component;  /* one per element */
  void* impl;                /* owned by the library */
} gf_bdf_mesh;
gf_status gf_bdf_read(const char* path, gf_bdf_mesh** out);
gf_status gf_bdf_free(gf_bdf_mesh* mesh);

/* ---- BSR matrix ------------------------------------------------------ */
/* createBsrMat (include/linalg/bsr_mat.h:354-357): values zeroed. */
gf_status gf_bsr_create(gf_assembler* a, gf_bsr** out);
gf_status gf_bsr_destroy(gf_bsr* m);
/* getPtr (bsr_mat.h:31-32): device pointer to nnzb*36 doubles. */
double* gf_bsr_values(gf_bsr* m);
gf_status gf_bsr_zero(gf_bsr* m, void* stream);
/* cusparseDbsrmv as used at examples/iterative/gmres.cu:498-509:
 * y = alpha A x + beta y, vectors in the solver ordering. */
gf_status gf_bsr_spmv(gf_bsr* m, double alpha, const double* d_x, double beta, double* d_y,
                      void* stream);
/* Natural-order <-> solver-order vector permutation (permute_vec_kernel,
 * vec.cuh:15-34; bsr_pre_solve / bsr_post_solve, solve_utils.h:4-17).
 * direction 0: out[perm[i]] = in[i]; 1: out[i] = in[perm[i]]. */
gf_status gf_permute_vec(gf_assembler* a, const double* d_in, double* d_out, int32_t direction,
                         void* stream);

/* ---- ILU preconditioner ---------------------------------------------- */
enum { GF_PREC_FP64 = 0, GF_PREC_FP32 = 1 };
/* ILUk_Preconditioner (include/linalg/precond.h:5-55) with the symbolic
 * ILU(k) of computeILUk (include/linalg/bsr_utils.h:678-807); fill_level 0
 * keeps A's pattern (ILU(0)). precision selects FP64 or FP32 factors.
 * Fails (GF_INVALID_ARG or GF_CUDA_ERROR with the reason in gf_last_error)
 * if a factor row holds more blocks than one shared-memory stage of the
 * triangular sweep: about 260 blocks in FP64 and 440 in FP32, or 170 and
 * 290 for triangles whose levels are split over two CTAs. */
gf_status gf_precond_create(gf_assembler* a, int32_t fill_level, int32_t precision,
                            gf_precond** out);
/* Which triangular-sweep kernel solves a triangle of the factor (sweep
 * argument of gf_precond_create_ex; no reference counterpart, cuSPARSE's
 * bsrsv2 picks its own level scheme):
 *  GF_SWEEP_DATAFLOW  one CTA per problem; each row waits only for the rows
 *                     it multiplies (shared-memory result ring), no block
 *                     barriers between levels;
 *  GF_SWEEP_LEVEL     level-synchronous chunks, split over a 2-CTA cluster
 *                     when a chunk-cost model says it pays (levels with
 *                     more rows than one CTA's warps or more blocks than its
 *                     stage);
 *  GF_SWEEP_AUTO      the level-synchronous kernel (the faster of the two
 *                     on the batched plate workload on B200).
 * The dataflow kernel needs its result ring and stages to fit one CTA's
 * shared memory: a factor whose rows reach back more than ~1000 positions
 * in level order does not fit.
 * Both give the same z up to the rounding of different summation orders. */
enum { GF_SWEEP_AUTO = 0, GF_SWEEP_DATAFLOW = 1, GF_SWEEP_LEVEL = 2 };
/* gf_precond_create with a choice of sweep kernel. GF_SWEEP_DATAFLOW fails
 * with GF_INVALID_ARG (text in gf_last_error) where the dataflow kernel does
 * not fit. */
gf_status gf_precond_create_ex(gf_assembler* a, int32_t fill_level, int32_t precision,
                               int32_t sweep, gf_precond** out);
gf_status gf_precond_destroy(gf_precond* p);
/* The sweep kernel of the L and U triangles (GF_SWEEP_DATAFLOW or
 * GF_SWEEP_LEVEL) and, for dataflow triangles, the result ring's slots. Any
 * pointer may be NULL. */
gf_status gf_precond_sweeps(const gf_precond* p, int32_t* kind_L, int32_t* kind_U,
                            int32_t* ring_L, int32_t* ring_U);
/* copyValues + numeric factorization (precond.h:35-44; cusparseDbsrilu02 at
 * examples/iterative/gmres.cu:426-457). A dataflow kernel on the device: one
 * warp per row, rows taken in level order, each step waiting only for the
 * row it reads (bounded waits; GF_TIMEOUT if one runs out). The factor is
 * bitwise reproducible run to run. */
gf_status gf_precond_factor(gf_precond* p, gf_bsr* A, void* stream);
/* z = U^{-1} L^{-1} r (two cusparseDbsrsv2_solve calls,
 * examples/iterative/gmres.cu:522-532), solver ordering. */
gf_status gf_precond_apply(gf_precond* p, const double* d_r, double* d_z, void* stream);
/* As gf_precond_apply, but the call allocates no device memory. No
 * counterpart in the reference. For callers that must not allocate while
 * they run: a serving loop that reserved its HBM up front, or host code
 * whose streams must not be stalled by the device-wide synchronisation an
 * allocation or free can cause.
 * The intermediate vector y = L^{-1} r lives in one fixed device array of
 * GF_NOALLOC_MAX_DOUBLES doubles (2 MiB) inside the library; problems with
 * 6 * num_nodes above that return GF_INVALID_ARG (text in gf_last_error) and
 * run nothing. No entry of the array needs to start at zero: the lower
 * sweep writes every entry the upper sweep reads.
 * The first call on a device (with that device current) looks up the
 * array's address on that device; make that first call before any stream
 * capture. All calls in the process share the one array per device, which
 * keeps the last call's contents; calls whose work overlaps on the GPU
 * (different streams, no ordering between them) race on it. */
#define GF_NOALLOC_MAX_DOUBLES 262144
gf_status gf_precond_apply_noalloc(gf_precond* p, const double* d_r, double* d_z, void* stream);
/* Reads and clears the status flags the preconditioner's kernels recorded
 * since the last read: GF_TIMEOUT when a bounded device-side wait of a
 * triangular sweep or of the factorization ran out (the apply's z is then
 * incomplete), GF_ZERO_PIVOT for a singular diagonal block, else GF_OK.
 * gf_precond_apply and gf_precond_apply_noalloc do not wait for the GPU, so
 * their flags are reported here, or by the next gf_precond_factor /
 * gf_gmres_solve on this preconditioner, which read and clear them too.
 * Synchronises `stream`. No counterpart in the reference (which exits on
 * errors, include/cuda_utils.h:35-43). */
gf_status gf_precond_status(gf_precond* p, void* stream);
/* How the triangular work of this preconditioner is laid out on the GPU:
 * CTAs that share each sweep chunk's rows (1 or 2) for L and U, the CTAs the
 * dataflow factorization runs on when this preconditioner is factored alone
 * (1 to 128; in a batch the SMs are shared out by the problems' block
 * updates), and the number of chunks of each triangle (a chunk holds rows of one level; a
 * level with more blocks than a chunk's stage spans several). Any pointer
 * may be NULL. No reference counterpart (cuSPARSE's bsrsv2 level analysis is
 * internal). */
/* Where and how long the preconditioner's setup ran: whether its ILU(k)
 * pattern was computed on the GPU (1; 0 when the host computed it: fill 0,
 * a row whose column window exceeds the GPU kernel's 4096, or a device
 * failure), the wall time of that pattern and of the whole
 * gf_precond_create (ms). Any pointer may be NULL. No reference counterpart
 * (computeILUk, include/linalg/bsr_utils.h:678-807, runs on the host). */
gf_status gf_precond_setup_info(const gf_precond* p, int32_t* symbolic_on_gpu, double* symbolic_ms,
                                double* setup_ms);
gf_status gf_precond_layout(const gf_precond* p, int32_t* nsplit_L, int32_t* nsplit_U,
                            int32_t* fac_ctas, int32_t* chunks_L, int32_t* chunks_U);
/* Pattern, level count and factor copy for checking. rowPtr/colPtr may be
 * NULL; values receives nnzb_pc*36 entries with the diagonal blocks holding
 * U_ii^{-1}. */
gf_status gf_precond_info(const gf_precond* p, int32_t* nnzb, int32_t* num_levels_L,
                          int32_t* num_levels_U);
gf_status gf_precond_get(const gf_precond* p, int32_t* rowPtr, int32_t* colPtr,
                         double* h_values);

/* ---- GMRES / iterative refinement ------------------------------------ */
typedef struct gf_solve_opts {
  int32_t restart;        /* m (reference: 30, examples/iterative/gmres.cu:33) */
  int32_t max_iters;      /* total Arnoldi steps */
  double rtol;            /* ||b - A x||_2 / ||b||_2 target (FP64 A) */
  int32_t side;           /* 0 left (reference), 1 right preconditioning */
  int32_t mixed;          /* 0: FP64 GMRES and SpMV (the preconditioner
                              applies in its own precision, FP64 or FP32
                              factors); 1: FP32 SpMV + FP32 ILU inside an
                              inner GMRES under FP64 iterative refinement */
  double inner_rtol;      /* inner tolerance per refinement step (mixed) */
  int32_t max_refine;     /* max refinement steps (mixed) */
  int32_t check_every;    /* host polls convergence every k steps */
} gf_solve_opts;

typedef struct gf_solve_stats {
  int32_t iterations;     /* Arnoldi steps */
  int32_t restarts;
  int32_t refinements;
  int32_t status;         /* gf_status of the solve */
  double rel_residual;    /* final ||b - A x|| / ||b|| in FP64 */
  double time_ms;
} gf_solve_stats;

void gf_solve_opts_default(gf_solve_opts* o);
/* The ILU-GMRES driver of examples/iterative/gmres.cu:468-771 (bugs fixed:
 * dot length nvars, m+1 basis vectors, restarts): solves A x = b with the
 * BSR matrix A (BCs applied) and a factored preconditioner. d_b / d_x are in
 * natural order; permutation happens inside. d_x is the initial guess on
 * entry. Device-resident: no host round trip per Arnoldi step. */
gf_status gf_gmres_solve(gf_assembler* a, gf_bsr* A, gf_precond* p, const double* d_b,
                         double* d_x, const gf_solve_opts* opts, gf_solve_stats* stats,
                         void* stream);

/* fill_level of gf_precond_create(_ex) that keeps every fill block: the
 * complete block LU factor (no entry dropped), i.e. a direct solver. */
#define GF_FILL_FULL 0x7fffffff
/* CUSPARSE::direct_LU_solve_old (include/linalg/solvers/cusparse.h:16-192):
 * the reference factors the matrix with bsrilu02 on a full-fill pattern (a
 * complete block LU without pivoting) and runs two bsrsv2 triangular solves.
 * Here: the symbolic full fill of A's pattern in the assembler's ordering,
 * the block LU on the GPU (the ILU kernels with nothing dropped), the two
 * triangular sweeps, then FP64 refinement through the same factor: four
 * steps of right-preconditioned GMRES from x = 0, the first of which is
 * x = (LU)^{-1} b (residuals with the FP64 A). d_b / d_x in
 * natural order; stats->rel_residual is the final ||b - A x|| / ||b||.
 * Returns GF_OK, GF_ZERO_PIVOT, GF_NAN or a CUDA / argument error; factor
 * rows longer than the sweep kernels' shared-memory stages (large
 * bandwidths) give GF_INVALID_ARG with the reason in gf_last_error. The
 * factor is built and released inside the call; for repeated solves with
 * one matrix, create a GF_FILL_FULL preconditioner and use gf_gmres_solve. */
gf_status gf_direct_solve(gf_assembler* a, gf_bsr* A, const double* d_b, double* d_x,
                          gf_solve_stats* stats, void* stream);

/* ---- batched uneven solves ------------------------------------------- */
/* A batch of independent problems (assembler + BSR matrix + preconditioner
 * each) solved together: SpMV, ILU factorization and both triangular sweeps
 * run as one launch over the whole batch (merged level order), GMRES keeps
 * per-problem Arnoldi states and per-problem reductions, so every problem's
 * result is bitwise the same alone and in any batch. No reference
 * counterpart: the reference solves one problem per driver
 * (examples/iterative/gmres.cu). The handles must outlive the batch, and
 * all preconditioners of a batch must have the same precision
 * (GF_INVALID_ARG otherwise). */
gf_status gf_batch_create(int32_t n, gf_assembler* const* asms, gf_bsr* const* mats,
                          gf_precond* const* pcs, gf_batch** out);
gf_status gf_batch_destroy(gf_batch* b);
/* add_jacobian with fused BCs for every problem: one launch per colour over
 * all problems (or one launch with gf_batch_set_scatter(GF_ASSEMBLE_ATOMIC)).
 * The per-problem launch parameters are cached in the batch and uploaded
 * again (with a synchronisation of `stream`) only when they change. Calls on
 * one batch must not overlap. */
gf_status gf_batch_assemble(gf_batch* b, void* stream);
/* As gf_batch_assemble with a per-problem thickness field (d_thick[k] may be
 * NULL to use the assembler's own). Passing the same pointers every call
 * keeps the cached parameters; new pointers re-upload them. */
gf_status gf_batch_assemble_ex(gf_batch* b, const double* const* d_thick, void* stream);
/* Numeric ILU(k) of every problem in one level-ordered launch. */
/* Scatter of the batch's assembly (gf_batch_assemble / _ex): 0 (default)
 * runs each colour of all problems in one launch (coloured, bitwise
 * reproducible), GF_ASSEMBLE_ATOMIC runs all chunks of all problems in one
 * launch with FP64 atomics. No reference counterpart. */
gf_status gf_batch_set_scatter(gf_batch* b, int32_t flags);
gf_status gf_batch_factor(gf_batch* b, void* stream);
/* Solve every problem: d_b[k], d_x[k] device pointers (natural order,
 * d_x[k] is the initial guess); stats[k] per problem (may be NULL). */
gf_status gf_batch_solve(gf_batch* b, const double* const* d_b, double* const* d_x,
                         const gf_solve_opts* opts, gf_solve_stats* stats, void* stream);

/* ---- failure injection for tests ------------------------------------- */
/* Sets, on the current device, the bound of the device-side waits that end
 * when a bulk copy lands, a partner CTA arrives or a row that is read is
 * final (wait_ns; 0 restores the default of 2 s), and whether the kernels
 * skip publishing (skip_meetings != 0): CTA rank 1 of every split triangle
 * skips its arrivals on the partner's meeting barriers, the factorization
 * never publishes the first row of its order and the dataflow sweep's warp
 * 0 never publishes its rows, which makes the bounded waits run out so that
 * the launch reports GF_TIMEOUT. The waits that drain a CTA's own copies
 * in flight keep the 2 s bound, and both CTAs of a cluster still meet on the
 * final cluster barrier, so nothing hangs. Process-wide for the device: set
 * it only while no other work of this library runs there, and restore it
 * with gf_test_set_waits(0, 0). No reference counterpart. */
gf_status gf_test_set_waits(unsigned long long wait_ns, int32_t skip_meetings);

#ifdef __cplusplus
}
#endif
#endif /* GPUFEM_H */
