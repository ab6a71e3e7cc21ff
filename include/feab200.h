/*
 * feab200 -- C ABI of the B200 (sm_100a) hex8 linear-elastic library.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and returns an
 * int status (FEAB_OK on success).  Pointers named d_* / device arrays are device
 * memory owned by the caller; the library never frees caller memory.  Scratch memory
 * is passed in by the caller (sizes from the *_bytes queries), so the library itself
 * performs no cudaMalloc.  Work is enqueued on the given stream; functions documented
 * as "synchronous" also wait for it and read small results back to the host.
 *
 * Device-side failures (degenerate element, zero diagonal, capacity) are written to a
 * caller-provided feab_device_status in device memory: the first failure wins and
 * records the offending element/node/row index.
 *
 * The reference (abhi2k16/computation-suite, fea_engine) is pure Python; each entry
 * point names the reference function whose work it replaces (file:line inside
 * fea_engine/src/fea_engine/ unless stated).
 */
#ifndef FEAB200_H
#define FEAB200_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (map to the reference's Python exceptions, see the Python layer) ---- */
#define FEAB_OK 0
#define FEAB_BAD_ARG 1              /* ValueError  (bad sizes / indices)                   */
#define FEAB_DEGENERATE_ELEMENT 2   /* ValueError  mesh_transform.py:327-332 (|detJ|<1e-300) */
#define FEAB_ZERO_DIAGONAL 3        /* ValueError  iterative_solvers.py:199-200            */
#define FEAB_NOT_SPD 4              /* LinAlgError iterative_solvers.py:450-454 (pAp <= 0) */
#define FEAB_NOT_CONVERGED 5        /* RuntimeError iterative_solvers.py:478-481           */
#define FEAB_CUDA_ERROR 6           /* RuntimeError (CUDA launch / runtime failure)        */
#define FEAB_CAPACITY 7             /* ValueError  node valence beyond the kernels' limit  */
#define FEAB_SCRATCH_LIMIT 8        /* ValueError  n beyond feab_pcg_solve_noalloc's fixed scratch */

#define FEAB_HEX8_KE_PACKED 324     /* doubles per element: the 36 upper 3x3 node blocks   */
#define FEAB_HEX8_KE_FULL 576       /* doubles per element: full 24x24, row major          */
#define FEAB_MAX_NODE_ELEMS 64      /* elements per node supported by the topology kernels */
#define FEAB_MAX_NODE_NBRS 128      /* distinct neighbour nodes per node                   */

typedef struct feab_device_status {
  int32_t code;      /* 0 = OK, else the first FEAB_* failure */
  int32_t reserved;
  int64_t index;     /* element / node / row that failed */
} feab_device_status;

/* Reduced stiffness in CSR form.  Rows of one mesh node share one column pattern; a
 * group is a run of consecutive rows with identical col_idx (group_ptr may be NULL:
 * every row is then its own group). */
typedef struct feab_csr {
  int32_t n;                 /* rows = columns                     */
  int32_t n_groups;          /* groups in group_ptr (ignored if NULL) */
  int64_t nnz;
  const int32_t* row_ptr;    /* n+1                                */
  const int32_t* col_idx;    /* nnz, sorted within each row        */
  const double* vals64;      /* nnz                                */
  const float* vals32;       /* nnz, FP32 copy (mixed precision) or NULL */
  const int32_t* group_ptr;  /* n_groups+1 or NULL                 */
} feab_csr;

#define FEAB_PREC_FP64 0     /* plain FP64 PCG: the reference recurrence, FP64 throughout        */
#define FEAB_PREC_MIXED 1    /* FP64 vectors/scalars; SpMV on 48-bit values in difference form;   */
                             /* FP64 reliable residual replacement (needs a feab_diff_operator)  */
#define FEAB_PREC_FP32 2     /* FP32 values and p/r/Ap/x-correction, FP64 scalars, FP64 reliable */
                             /* residual replacement folding into an FP64 solution               */

/* Difference-form operator built from the FP64 CSR by feab_diff_operator_build (storage is
 * caller memory, feab_diff_operator_bytes).  Applies y_a = sum_{b!=a} K_ab (x_b - x_a) + S_a x_a
 * with K_ab rounded to 44 mantissa bits (7 bytes each: vhi, vlo, vlo2) and S_a = sum_b K_ab
 * accumulated in FP64,
 * evaluated as sum_{b!=a} K_ab x_b + T_a x_a with T_a = S_a - W_a, W_a = sum_{b!=a} K_ab over the
 * rounded values: the same value, so the same rounding error; S holds T.
 * Layout per node row group g (the f rows of one node): its off-node columns, padded to a
 * multiple of 4 (Lp_g), start at goff[g] in tcol; its values start at voff[g], row-major
 * (f rows x Lp_g), so every 4-column quad is one 16-byte (vhi) + 8-byte (vlo) + 4-byte (vlo2)
 * load.  Padding columns point at the node's own first free DOF with value 0.  (44 bits keep the
 * operator's FP64 residual floor far below 1e-9 on every mesh tried, so the mixed block-PCG
 * keeps FP64's iteration count; 36 bits, the single-right-hand-side sliced operator's width,
 * leave it above 1e-9 on some meshes and moduli.) */
typedef struct feab_diff_operator {
  int32_t* tcol;     /* sum Lp_g: column | (DOF component << 30)            */
  uint32_t* vhi;     /* sum f_g Lp_g: upper 32 bits of the rounded double   */
  uint16_t* vlo;     /* sum f_g Lp_g: next 16 bits                          */
  uint8_t* gmask;    /* n_groups: free-DOF mask of the group's node         */
  double* S;         /* 3 n: own-node terms T = S - W per DOF component      */
  int32_t* goff;     /* n_groups + 1: first tagged column of each group     */
  int32_t* voff;     /* n_groups + 1: first value of each group             */
  uint8_t* vlo2;     /* sum f_g Lp_g: the 8 bits below vlo                  */
} feab_diff_operator;

/* Sliced (SELL-32) node-group operator for the single-right-hand-side PCG, built from the CSR
 * by feab_sell_operator_build into caller storage (feab_sell_operator_bytes).  Node row groups
 * are cut into slices of 32; lane l of a warp owns group 32 s + l, and slice s holds W_s column
 * steps (a multiple of 4) from step soff[s].  Steps come in blocks of 4; for the block starting
 * at step b, lane l's 4 columns are tcol[b * 32 + 4 l + u] and its row-k values are at
 * (3 b + 4 k) * 32 + 4 l + u (u = 0..3), so each lane reads 16 contiguous bytes per load and
 * each warp 512 contiguous bytes.
 *   kind FEAB_PREC_FP64:  v64 holds the FP64 values; all columns (plain y = K x).
 *   kind FEAB_PREC_MIXED: vhi/vlo hold the values rounded to 36 mantissa bits; own-node columns
 *                         are left out and K is applied in difference form with the row-block
 *                         sums S (as feab_diff_operator); tcol carries the DOF component.
 * Steps past a group's length point at the node's own first free DOF with value 0. */
typedef struct feab_sell_operator {
  int32_t kind;      /* FEAB_PREC_FP64 or FEAB_PREC_MIXED                       */
  int32_t n_slices;  /* ceil(n_groups / 32)                                     */
  int32_t* soff;     /* n_slices + 1: first column step of each slice           */
  int32_t* tcol;     /* 32 per step                                             */
  double* v64;       /* FP64 kind: 96 per step                                  */
  uint32_t* vhi;     /* MIXED kind: 96 per step                                 */
  uint16_t* vlo;     /* MIXED kind: 96 per step                                 */
  uint8_t* gmask;    /* MIXED kind: n_groups free-DOF masks                     */
  double* S;         /* MIXED kind: 3 n own-node terms T = S - W               */
  int16_t* tcol16;   /* 32 per step: column - the lane's first row, when every  */
                     /* such offset fits 16 bits (NULL otherwise); the SpMV    */
                     /* then reads these 2-byte offsets instead of tcol        */
} feab_sell_operator;

typedef struct feab_pcg_params {
  double tol;                /* on ||b - A x|| / ||b||  (||b|| := 1 when b == 0)          */
  int32_t maxiter;           /* <= 0: 10 n, as iterative_solvers.py:393-394              */
  int32_t precision;         /* FEAB_PREC_*                                              */
  double reliable_delta;     /* mixed: FP64 residual replacement when ||r|| < delta*rmax  */
  int32_t chunk;             /* iterations per CUDA-graph launch (<= 0: default 16)      */
  int32_t use_dinv;          /* 1: Jacobi preconditioner (method="pcg"), 0: plain CG     */
  int32_t lanes_per_group;   /* SpMV lanes per node row group: 4, 8, 16 or 32 (else 16)  */
  int32_t reserved;
} feab_pcg_params;

typedef struct feab_pcg_result {
  int32_t status;            /* FEAB_OK / FEAB_NOT_SPD / FEAB_NOT_CONVERGED / ...        */
  int32_t iters;             /* CG iterations (the reference's n_iter)                   */
  int32_t reliable_updates;  /* mixed: FP64 residual replacements performed              */
  int32_t graph_launches;    /* CUDA-graph replays (each holds 3*chunk kernels)          */
  double relres;             /* final ||r||/||b|| (mixed: the FP64 true residual)        */
  double bnorm;
} feab_pcg_result;

/* ---------------------------------------------------------------- library */
int32_t feab_abi_version(void);
const char* feab_status_string(int32_t code);
/* Make `device` current for this host thread in the library's own CUDA runtime (the
 * library links the runtime statically; its current device is independent of the caller's). */
int32_t feab_set_device(int32_t device);
/* Kernels this library has launched in this process (graph replays count their kernels). */
uint64_t feab_launch_count(void);

/* ---------------------------------------------------------------- topology
 * Replaces the pattern part of scatter_global_stiffness' COO->CSR + [ix_(free,free)]
 * (vectorized_assembly.py:217-262, solver.py:1977-1978).  The resulting row_ptr/col_idx
 * equal SciPy's sorted int32 CSR of the reduced matrix bit for bit. */

/* Scratch bytes needed by the topology calls for a mesh of this size. */
size_t feab_topology_scratch_bytes(int32_t n_nodes, int64_t n_elem);

/* Node -> element incidence, each node's list sorted by element id.
 * conn: n_elem*8 int32 node ids.  inc_ptr: n_nodes+1, inc_elem: 8*n_elem.
 * Synchronous: *max_elems_out = largest node valence (FEAB_CAPACITY if above
 * FEAB_MAX_NODE_ELEMS). */
int32_t feab_node_incidence(const int32_t* conn, int64_t n_elem, int32_t n_nodes, int32_t* inc_ptr,
                            int32_t* inc_elem, void* scratch, size_t scratch_bytes,
                            feab_device_status* status, int32_t* max_elems_out, cudaStream_t stream);

/* Sorted node adjacency (a node is its own neighbour).  Call with nbr_idx == NULL to
 * fill nbr_ptr (n_nodes+1) and get *total_out / *max_nbrs_out (synchronous), then again
 * with nbr_idx (total entries) to fill it. */
int32_t feab_node_adjacency(const int32_t* conn, const int32_t* inc_ptr, const int32_t* inc_elem,
                            int32_t n_nodes, int32_t* nbr_ptr, int32_t* nbr_idx, void* scratch,
                            size_t scratch_bytes, feab_device_status* status, int64_t* total_out,
                            int32_t* max_nbrs_out, cudaStream_t stream);

/* CSR pattern of the free x free block.  free_map[3*node+k] = reduced row of that DOF or
 * -1 when fixed (fix_dofs, solver.py:1109-1176).  Call with col_idx == NULL to fill
 * row_ptr (n_free+1) and group_ptr (n_groups+1, may be NULL) and get *nnz_out,
 * *n_groups_out (synchronous); then again with col_idx to fill the columns. */
int32_t feab_csr_pattern(const int32_t* nbr_ptr, const int32_t* nbr_idx, int32_t n_nodes,
                         const int32_t* free_map, int32_t n_free, int32_t* row_ptr,
                         int32_t* group_ptr, int32_t* col_idx, void* scratch, size_t scratch_bytes,
                         int64_t* nnz_out, int32_t* n_groups_out, cudaStream_t stream);

/* ---------------------------------------------------------------- element kernel
 * ke = sum over the 2x2x2 Gauss points of B^T D B detJ w (signed detJ), per element,
 * times scale[e] when scale != NULL.  Replaces Hex8Solid3D.stiffness / B_matrix
 * (elements/base.py:494-514, elements/solids.py:130-163) and the batched
 * MeshTransformation + tensorized_element_stiffness einsum (mesh_transform.py:280-437,
 * vectorized_assembly.py:165-214).  D: 36 doubles in HOST memory (symmetric 6x6, Voigt
 * xx,yy,zz,xy,yz,zx).  layout: FEAB_HEX8_KE_PACKED (36 upper node blocks (a<=b), block
 * (a,b) at a*8-a*(a-1)/2+(b-a), each 3x3 row major) or FEAB_HEX8_KE_FULL. */
int32_t feab_hex8_element_stiffness(const double* coords, const int32_t* conn, int64_t n_elem,
                                    const double* D_host, const double* scale, double thickness,
                                    double* ke_out, int32_t layout, feab_device_status* status,
                                    cudaStream_t stream);

/* The same for Hex8SolidBbar (elements/solids.py:225-257): B replaced by the mean-dilatation
 * B-bar = B - (m m^T / 3) B + (m m^T / 3) sum_q B detJ w / sum_q detJ w, m = [1 1 1 0 0 0], at
 * the same 8 Gauss points (signed detJ in both sums). */
int32_t feab_hex8_bbar_element_stiffness(const double* coords, const int32_t* conn, int64_t n_elem,
                                         const double* D_host, const double* scale, double thickness,
                                         double* ke_out, int32_t layout, feab_device_status* status,
                                         cudaStream_t stream);

/* Consistent mass of every element (Element.mass, elements/base.py:711-731, through
 * FESystem.assemble_mass, solver.py:699-740): me = sum_q Nm^T R Nm |detJ| w thickness (times
 * scale[e] when scale != NULL), i.e. node block (a, b) = m_ab R thickness with
 * m_ab = sum_q N_a N_b |detJ| w.  R_host: the 3x3 density matrix (9 doubles, HOST memory,
 * symmetric, e.g. rho I).  Same layouts as feab_hex8_element_stiffness, so feab_assemble_csr
 * assembles M on the stiffness pattern. */
int32_t feab_hex8_element_mass(const double* coords, const int32_t* conn, int64_t n_elem, const double* R_host,
                               const double* scale, double thickness, double* me_out, int32_t layout,
                               feab_device_status* status, cudaStream_t stream);

/* ---------------------------------------------------------------- assembly
 * Deterministic gather assembly of the reduced CSR values from packed element
 * matrices: each entry is summed over its elements in ascending element order.
 * Also writes the FP32 copy (vals32 may be NULL) and the Jacobi inverse diagonal
 * 1/diag (dinv64/dinv32 may be NULL; zero diagonal -> FEAB_ZERO_DIAGONAL).
 * Replaces the COO duplicate summation of scatter_global_stiffness
 * (vectorized_assembly.py:254-262) / the LIL scatter (solver.py:684-697) and
 * jacobi_preconditioner (iterative_solvers.py:193-202). */
int32_t feab_assemble_csr(const double* ke_packed, const int32_t* conn, const int32_t* inc_ptr,
                          const int32_t* inc_elem, const int32_t* nbr_ptr, const int32_t* nbr_idx,
                          int32_t n_nodes, int32_t max_nbrs, const int32_t* free_map,
                          const int32_t* row_ptr, double* vals64, float* vals32, double* dinv64,
                          float* dinv32, feab_device_status* status, cudaStream_t stream);

/* y = K v over all 3*n_nodes DOFs, element by element from packed element matrices
 * (node-centric gather, deterministic).  Used for the Dirichlet RHS correction
 * F_f - K[free,fixed] u_fixed (solver.py:1496-1511) and for residual checks. */
int32_t feab_hex8_apply(const double* ke_packed, const int32_t* conn, const int32_t* inc_ptr,
                        const int32_t* inc_elem, int32_t n_nodes, const double* v, double* y,
                        cudaStream_t stream);

/* ---------------------------------------------------------------- PCG
 * Jacobi-preconditioned CG, the recurrence of preconditioned_cg
 * (iterative_solvers.py:362-481) and _cg_torch (torch_sparse_solver.py:165-202).
 * FEAB_PREC_FP64 follows the reference step for step in FP64, through the CSR or, when `sell`
 * (kind FEAB_PREC_FP64) is given, through the sliced operator.  FEAB_PREC_MIXED needs `sell` of
 * kind FEAB_PREC_MIXED; FEAB_PREC_FP32 uses the CSR's vals32.  The precisions other than FP64
 * declare convergence only on an FP64 residual b - K x computed with the FP64 values.
 * Synchronous: returns when the solve has finished; *result holds the outcome. */
size_t feab_pcg_workspace_bytes(int32_t n, int32_t precision);

/* Difference-form operator for the batched block-PCG (feab_block_pcg_solve); upper bound from
 * the sizes alone (no device work); needs nnz + 3 n_groups < 2^31. */
size_t feab_diff_operator_bytes(int32_t n, int64_t nnz, int32_t n_groups);

/* dof_of[r] = original DOF of reduced row r (free_dofs, solver.py:1400-1401).  A needs
 * group_ptr. */
int32_t feab_diff_operator_build(const feab_csr* A, const int32_t* dof_of, void* storage, size_t storage_bytes,
                                 feab_diff_operator* out, cudaStream_t stream);

int32_t feab_pcg_solve(const feab_csr* A, const feab_sell_operator* sell, const double* dinv64,
                       const float* dinv32, const double* b, const double* x0, double* x,
                       const feab_pcg_params* params, void* workspace, size_t workspace_bytes,
                       feab_pcg_result* result, cudaStream_t stream);

/* Allocation-free FP64 PCG.  No counterpart in the reference: it exists for callers that
 * cannot allocate device memory -- a host that hands all device memory to its own pool and
 * forbids libraries from calling cudaMalloc (which would fail or fragment that pool), a
 * thread that must not block on the implicit device synchronisation cudaMalloc/cudaFree can
 * cause, or an environment that forbids allocation after start-up.  Same algorithm, arguments
 * and result as feab_pcg_solve with precision FEAB_PREC_FP64, but the workspace is a fixed
 * 32 MiB array in the library's device memory (feab_pcg_noalloc_scratch_bytes), held by every
 * GPU that loads the library until the process exits; n above feab_pcg_noalloc_max_n() is
 * rejected with FEAB_SCRATCH_LIMIT before anything is launched.  The limit depends on the SM
 * count of the device (the per-block partials grow with it): about 838 thousand rows on a
 * 148-SM B200; query it at run time.  The function calls no cudaMalloc/cudaFree/cudaHostAlloc
 * and creates no stream, event or graph: it launches the plain CSR step kernels in chunks and
 * reads the done flag into a stack variable (the allocating entry point's sliced operator and
 * CUDA graph are faster).  Every call looks up the array's device address on the current device
 * (cudaGetSymbolAddress; no allocation); the first call on a device also loads the library's
 * device code there, so make it before any stream capture.  All calls on a device
 * share the one array and it keeps the previous call's contents (each call re-initialises what
 * must start at zero), so calls that overlap on the GPU -- on different streams or threads --
 * race and must be serialised by the caller.  Synchronous. */
size_t feab_pcg_noalloc_scratch_bytes(void);
int32_t feab_pcg_noalloc_max_n(void);
int32_t feab_pcg_solve_noalloc(const feab_csr* A, const double* dinv64, const double* b, const double* x0,
                               double* x, const feab_pcg_params* params, feab_pcg_result* result,
                               cudaStream_t stream);

/* Storage for a sliced operator of the CSR A (n rows, n_groups node groups) whose longest row has
 * max_row_len entries (81 for hex8 meshes). */
size_t feab_sell_operator_bytes(int32_t n, int32_t n_groups, int32_t max_row_len, int32_t kind);

/* Builds the sliced operator (A needs group_ptr; dof_of as for feab_diff_operator_build, only
 * read for the MIXED kind).  FEAB_BAD_ARG if a row is longer than max_row_len.  Synchronous. */
int32_t feab_sell_operator_build(const feab_csr* A, const int32_t* dof_of, int32_t kind, int32_t max_row_len,
                                 void* storage, size_t storage_bytes, feab_sell_operator* out, cudaStream_t stream);

/* y = A x (x, y double) through the sliced operator: the same product as the CSR SpMV
 * `A @ p` of preconditioned_cg (iterative_solvers.py:448), in FP64 or the mixed difference form. */
int32_t feab_sell_spmv(const feab_csr* A, const feab_sell_operator* op, const double* x, double* y,
                       cudaStream_t stream);

/* y = A x with the PCG's SpMV kernel (same code and launch shape as one PCG step's SpMV).
 * FEAB_PREC_FP64: x, y double, vals64; FEAB_PREC_FP32: x, y float, vals32;
 * FEAB_PREC_MIXED: x, y double, difference form through a MIXED sliced operator (sell);
 * FEAB_PREC_FP64 with an FP64 sliced operator: the sliced product instead of the CSR one.
 * Replaces the CSR SpMV `A @ p` of preconditioned_cg (iterative_solvers.py:448) /
 * `K_t @ x` of torch_sparse_cg_solve (torch_sparse_solver.py:255-256). */
int32_t feab_csr_spmv(const feab_csr* A, const feab_sell_operator* sell, int32_t precision, int32_t lanes_per_group,
                      const void* x, void* y, cudaStream_t stream);

/* ---------------------------------------------------------------- batched multi-RHS PCG
 * Many independent problems in one block-diagonal K (e.g. disconnected meshes assembled as
 * one mesh), each with a panel of right-hand sides.  Vectors are row-major n x k panels
 * (k in {1,2,4,8,16,32,64}); problem p owns the row groups of its work items.  Each column
 * runs its own CG recurrence (preconditioned_cg, iterative_solvers.py:434-481) -- the
 * iterative counterpart of solve_batched / solve_static_batched (batched_solve.py:44-164),
 * which factorise once for many columns.  precision: FEAB_PREC_FP64 or FEAB_PREC_MIXED
 * (diff != NULL).  X and the workspace must be 16-byte aligned.  Synchronous; per-column iterations / FP64
 * relative residuals and per-problem status go to the optional host arrays. */
typedef struct feab_batch {
  int32_t n_problems;
  int32_t k;                       /* panel width                                   */
  int32_t n_items;
  int32_t reserved;
  const int32_t* item_problem;     /* n_items: problem of the work item             */
  const int32_t* item_group0;      /* n_items: first row group                      */
  const int32_t* item_group1;      /* n_items: one past the last row group          */
  const int32_t* problem_items;    /* n_problems+1: items of p are [p, p+1)          */
  const int32_t* problem_cols;     /* n_problems: active RHS columns (<= k)          */
} feab_batch;

size_t feab_block_pcg_workspace_bytes(int32_t n, int32_t k, int32_t n_problems, int32_t n_items);

/* ---------------------------------------------------------------- node tiles of the block SpMM
 * FEAB_TILE_GROUPS consecutive node row groups of one problem form a tile, which one warp
 * applies: it walks the union of the tiles' column lists and gathers each panel row once for
 * every group of the tile that has the column (consecutive nodes of a structured hex8 mesh share
 * 2/3 of their neighbours, so a 4-group tile gathers half the panel rows its groups would gather
 * one by one).  Tile t covers groups tile_g0[t] .. tile_g0[t+1]-1 (tiles start at each problem's
 * first group and every FEAB_TILE_GROUPS groups after it); its union columns are
 * ucol[uoff[t] .. uoff[t+1]), grouped by mask (every column of mask 1, then of mask 2, ...,
 * ascending within a mask), padded to a multiple of 4 with mask 0; bit j of umask[u] says that
 * group tile_g0[t] + j has column ucol[u].  Values follow in the same order:
 * from value 3 * poff[t], for each union column, for each set bit j ascending, rows 0..2 of group
 * tile_g0[t] + j (rows past the group's free DOFs are 0).  FEAB_PREC_FP64: the CSR's FP64 values
 * (own-node columns included) in v64.  FEAB_PREC_MIXED: the feab_diff_operator's off-node columns
 * and 44-bit values in vhi / vlo / vlo2 (the own-node term comes from that operator's S). */
#define FEAB_TILE_GROUPS 4
#define FEAB_TILE_CHUNK 64   /* union columns the SpMM stages at a time */

typedef struct feab_tile_operator {
  int32_t n_tiles;
  int32_t precision;     /* FEAB_PREC_FP64 or FEAB_PREC_MIXED                         */
  int32_t n_groups;
  int32_t reserved;
  int32_t* tile_g0;      /* n_tiles + 1: first row group of each tile                  */
  int32_t* group_tile;   /* n_groups: tile of each row group                           */
  int32_t* uoff;         /* n_tiles + 1: first union column (a multiple of 4)          */
  int32_t* poff;         /* n_tiles + 1: first (column, group) pair                    */
  int32_t* ucol;         /* union columns                                              */
  int32_t* upair;        /* per union column: its first pair within the tile           */
  uint8_t* umask;        /* per union column: the groups of the tile that have it      */
  double* v64;           /* FEAB_PREC_FP64: 3 values per pair                          */
  uint32_t* vhi;         /* FEAB_PREC_MIXED: 3 values per pair, 44-bit as in           */
  uint16_t* vlo;         /*   feab_diff_operator                                       */
  uint8_t* vlo2;
  int32_t* cptr;         /* n_tiles + 1: first chunk of each tile                      */
  int32_t* chunk;        /* 4 per chunk (FEAB_TILE_CHUNK union columns of a tile):     */
                         /*   first union column, columns, first value, values        */
} feab_tile_operator;

/* Scratch for feab_tile_operator_build. */
size_t feab_tile_scratch_bytes(int32_t n_groups, int32_t n_problems);

/* Tiles of A's node row groups (A needs group_ptr), never crossing a problem boundary:
 * problem_groups (device, n_problems + 1) are the first row group of each problem and n_groups.
 * precision FEAB_PREC_MIXED needs diff (built from A).  Call with storage == NULL to get
 * *bytes_out (synchronous: the unions are counted on the device), then again with that much
 * storage (16-byte aligned) to build *out (synchronous).  Needs fewer than 2^31 union columns
 * and 2^31 values. */
int32_t feab_tile_operator_build(const feab_csr* A, const feab_diff_operator* diff, const int32_t* problem_groups,
                                 int32_t n_problems, int32_t precision, void* scratch, size_t scratch_bytes,
                                 void* storage, size_t storage_bytes, size_t* bytes_out, feab_tile_operator* out,
                                 cudaStream_t stream);

/* tiles (optional, of the solve's precision, built with this batch's problem boundaries): the
 * SpMM of every CG step walks node tiles instead of single row groups; work items must then
 * start and end on tile boundaries (items of a multiple of FEAB_TILE_GROUPS groups from each
 * problem's first group do).  The mixed solve's FP64 residual replacements use A and diff. */
int32_t feab_block_pcg_solve(const feab_csr* A, const feab_diff_operator* diff, const feab_tile_operator* tiles,
                             const feab_batch* batch, const double* dinv64, const double* B, double* X,
                             const feab_pcg_params* params, void* workspace, size_t workspace_bytes,
                             int32_t* iters_out, double* relres_out, int32_t* status_out, cudaStream_t stream);

/* Y = A X for a row-major n x k panel X (k in {1,2,4,8,16,32,64}; X 16-byte aligned for
 * k = 64): the block-PCG's SpMM on the plain CSR (FP64 values, node row groups required) on its
 * own, through the node tiles when tiles (FEAB_PREC_FP64) is given.  Applies K_ff or M_ff to the
 * whole block of vectors of the modal subspace iteration (the products eigsh makes inside
 * FESystem.solve_modal, solver.py:2047-2114).  Asynchronous. */
int32_t feab_block_spmm(const feab_csr* A, const feab_tile_operator* tiles, const double* X, double* Y, int32_t k,
                        cudaStream_t stream);

/* ---------------------------------------------------------------- POD Gram + eigensolve
 * Replaces the FP64 economy SVD of PodBasis._fit_standard (rom_engine/src/rom_engine/pod.py:
 * 140-147) for the singular values: G = X^T X with X (n x 64, FP32, row major, 16-byte
 * aligned) split into bf16 hi + lo on the tensor cores (tcgen05.mma, TMEM accumulator),
 * G = hi^T hi + hi^T lo + lo^T hi, FP64 across chunks and CTAs (deterministic); then the FP64
 * eigenvalues of G (squared singular values).  *error_flag (device int, zero it first) is
 * set if a bounded wait timed out. */
size_t feab_gram_workspace_bytes(int64_t n, int32_t k);

int32_t feab_gram_bf16x3(const float* X, int64_t n, int32_t k, double* G, void* workspace, size_t workspace_bytes,
                         int32_t* error_flag, cudaStream_t stream);

/* G = X^T X (64 x 64, FP64) on the tensor cores with exact products: X (n x 64, FP32, row major,
 * 16-byte aligned) is split per CTA row range and column into seven signed 7-bit integer digits
 * below a power-of-two column scale, the digit products are summed exactly in int32 by
 * tcgen05.mma kind::i8, and the scaled sums are combined in FP64 (the integer-slice method of
 * Ootomo, Ozaki & Yokota 2024).  Inputs keep 49 bits below their CTA's column maximum, so G has
 * FP64-level accuracy -- enough for the trailing singular values of PodBasis._fit_standard's FP64
 * SVD (rom_engine/src/rom_engine/pod.py:140-147).  The workspace of feab_gram_bf16x3;
 * *error_flag (device int, zero it first) is set if a bounded wait timed out.  Asynchronous;
 * deterministic. */
int32_t feab_gram_int8(const float* X, int64_t n, int32_t k, double* G, void* workspace, size_t workspace_bytes,
                       int32_t* error_flag, cudaStream_t stream);

/* G = X^T X (64 x 64, FP64) accumulated in FP64 on the CUDA cores, for X (n x 64, row major)
 * of FP32 (x_bytes = 4) or FP64 (x_bytes = 8) values; the same workspace as feab_gram_bf16x3.
 * The accurate Gram for snapshot sets whose spectrum decays faster than FP32 accumulation
 * resolves (the FP64 SVD of PodBasis._fit_standard, rom_engine/src/rom_engine/pod.py:140-147,
 * gets such trailing singular values right).  Asynchronous on the stream; deterministic. */
int32_t feab_gram_fp64(const void* X, int32_t x_bytes, int64_t n, int32_t k, double* G, void* workspace,
                       size_t workspace_bytes, cudaStream_t stream);

/* C = X^T Y (k x k, row major, FP64) for row-major n x k FP64 panels X and Y with leading
 * dimensions ldx, ldy (k <= 64): the Rayleigh-Ritz projections Y^T K Y and Y^T M Y of the modal
 * subspace iteration (the dense products behind eigsh in FESystem.solve_modal, solver.py:
 * 2047-2114).  Per-CTA partials in the workspace (feab_panel_gram_workspace_bytes(n)) are summed
 * in a fixed order, so C is deterministic.  Asynchronous. */
size_t feab_panel_gram_workspace_bytes(int64_t n);
int32_t feab_panel_gram(const double* X, int32_t ldx, const double* Y, int32_t ldy, int64_t n, int32_t k, double* C,
                        void* workspace, size_t workspace_bytes, cudaStream_t stream);

/* Z = Y V for a row-major n x k FP64 panel Y (leading dimension ldy, k <= 64) and a row-major
 * k x m matrix V (m <= 64), into the n x m panel Z (leading dimension ldz; Z must not be Y):
 * the Ritz vectors of the modal subspace iteration and the POD modes X V / sigma
 * (rom_engine/src/rom_engine/pod.py:140-160).  Asynchronous. */
int32_t feab_panel_small(const double* Y, int32_t ldy, int64_t n, int32_t k, const double* V, int32_t m, double* Z,
                         int32_t ldz, cudaStream_t stream);

/* Cyclic Jacobi eigensolver (one CTA, FP64) for a symmetric k x k matrix (k <= 64) in device
 * memory: eigenvalues descending into evals, eigenvectors (columns) into evecs (may be NULL).
 * A is overwritten.  *sweeps_out (device int, may be NULL) receives the sweeps used. */
int32_t feab_symeig_jacobi(double* A, int32_t k, double* evals, double* evecs, int32_t max_sweeps,
                           int32_t* sweeps_out, cudaStream_t stream);

/* ---------------------------------------------------------------- SIMP adjoint
 * out[e] = -p (1-rho_min) rho_e^(p-1) * lam_e^T K0_e u_e, with K0_e recomputed from the
 * coordinates and D (unit modulus) at the Gauss points as sum_q eps(lam)^T D eps(u)
 * detJ w.  lam == u gives the compliance sensitivity dC/drho
 * (compliance_sensitivity_closed_form, topopt.py:161-177, simp_scale_grad :85-93);
 * a general lam (an adjoint solution) gives the VJP of rho -> K(rho) u used by
 * compliance_sensitivity_via_adjoint (topopt.py:180-232).  u, lam: 3*n_nodes. */
int32_t feab_hex8_simp_vjp(const double* coords, const int32_t* conn, int64_t n_elem,
                           const double* D_host, const double* rho, double penal, double rho_min,
                           const double* u, const double* lam, double* out,
                           feab_device_status* status, cudaStream_t stream);

/* ---------------------------------------------------------------- SIMP optimality-criteria loop
 * The steps of topology_optimize_compliance (fea_engine/src/fea_engine/topopt.py:298-379) after
 * the solve and dC/drho (feab_pcg_solve, feab_hex8_simp_vjp).
 *
 * feab_element_centroids: centroids (n_elem x 3) = mean of the 8 corner coordinates
 * (mesh.nodes[conn].mean(axis=1), topopt.py:352).
 *
 * feab_filter_build: the filter weights H[e, j] = max(0, radius - |c_e - c_j|) of
 * build_filter_weights (topopt.py:235-243) as a CSR over elements (columns ascending, only the
 * positive entries), with rowsum[e] = sum_j H[e, j].  Two phases: with idx == NULL it counts,
 * writes ptr (n_elem + 1) and *nnz_out (host) and synchronises (scratch:
 * feab_filter_scratch_bytes); with idx != NULL it fills idx / w (nnz) and rowsum (n_elem),
 * asynchronously (scratch unused).  Every pair of centroids is compared once per phase. */
int32_t feab_element_centroids(const double* coords, const int32_t* conn, int64_t n_elem, double* centroids,
                               cudaStream_t stream);

size_t feab_filter_scratch_bytes(int64_t n_elem);

int32_t feab_filter_build(const double* centroids, int64_t n_elem, double radius, int32_t* ptr, int32_t* idx,
                          double* w, double* rowsum, int64_t* nnz_out, void* scratch, size_t scratch_bytes,
                          cudaStream_t stream);

/* out[e] = sum_j H[e, j] rho_j dc_j / max(max(rho_e, eps) rowsum[e], eps)
 * (apply_sensitivity_filter, topopt.py:246-253).  out must not alias rho or dc. */
int32_t feab_filter_apply(const int32_t* ptr, const int32_t* idx, const double* w, const double* rowsum,
                          int64_t n_elem, const double* rho, const double* dc, double eps, double* out,
                          cudaStream_t stream);

/* oc_update (topopt.py:259-295): dc clipped to <= -1e-12; the bracket [1e-12, l2] on the volume
 * multiplier is doubled (at most 60 times) until mean(rho_try) <= volume_fraction, then bisected
 * until (l2 - l1) < bisection_tol * max(l2, 1) or max_bisection_iter steps, with
 * rho_try = clip(clip(rho sqrt(-dc / l), rho - move, rho + move), rho_min_bound, rho_max_bound).
 * rho_new receives the last bisection step's densities and *max_change (device double)
 * max |rho_new - rho|.  Runs on the device with no host synchronisation (a fixed sequence of
 * step kernels that return at once after convergence); workspace: feab_oc_workspace_bytes. */
size_t feab_oc_workspace_bytes(int64_t n_elem);

int32_t feab_oc_update(const double* rho, const double* dc, int64_t n_elem, double volume_fraction, double move,
                       double rho_min_bound, double rho_max_bound, double bisection_tol,
                       int32_t max_bisection_iter, double* rho_new, double* max_change, void* workspace,
                       size_t workspace_bytes, cudaStream_t stream);

/* ---------------------------------------------------------------- strain / stress recovery
 * Replaces recovery._recover / stress / strain / von_mises for Hex8 blocks
 * (fea_engine/src/fea_engine/recovery.py:196-227 _block_batched, :258-334 _recover,
 * :365-420 stress / strain / _mises / von_mises; FESystem.stress / strain / von_mises,
 * solver.py:413-430).  At the 2x2x2 Gauss points val = D B u (D_host != NULL: stress) or
 * B u (D_host == NULL: engineering strain), Voigt order xx, yy, zz, xy, yz, xz.
 * nodal (n_nodes x 6): lumped L2 projection to the corners,
 *   sum_e sum_q N_a |detJ| w val / sum_e sum_q N_a |detJ| w, summed over the node's elements in
 *   ascending element order (nodes with no element get 0);
 * elem (n_elem x 6): sum_q |detJ| w val / sum_q |detJ| w;
 * nodal_vm / elem_vm: the von Mises stress of those (stress only).  Any of the four outputs
 * may be NULL (not all).  u: 3*n_nodes.  inc_ptr / inc_elem: feab_node_incidence.  scratch:
 * feab_hex8_recover_scratch_bytes(n_elem) bytes of device memory (8 doubles per element
 * corner).  conn, nodal and scratch must be 16-byte aligned.  Asynchronous on the stream; a
 * degenerate element sets status. */
size_t feab_hex8_recover_scratch_bytes(int64_t n_elem);

int32_t feab_hex8_recover(const double* coords, const int32_t* conn, int64_t n_elem, int32_t n_nodes,
                          const int32_t* inc_ptr, const int32_t* inc_elem, const double* D_host,
                          const double* u, double* nodal, double* nodal_vm, double* elem,
                          double* elem_vm, void* scratch, size_t scratch_bytes,
                          feab_device_status* status, cudaStream_t stream);

/* ---------------------------------------------------------------- direct solve (banded Cholesky)
 * Replaces the sparse direct solve of FESystem.solve_static() with method=None:
 * FESystem._sparse_lu_solve (solver.py:1681-1724, SuperLU splu of K_ff, then a singularity test
 * on the pivots: min |U_ii| < tol * max |U_ii|).  K_ff is SPD, so its LU without pivoting is
 * its Cholesky factorisation and U_ii = L_ii^2; the same pivot test is reported.
 *
 * The rows are first renumbered (iperm: old row -> new row, a fill-reducing order such as
 * reverse Cuthill-McKee) so that every nonzero lies within `bandwidth` of the diagonal.  The
 * lower band is stored as 64 x 64 tiles: block row I (rows 64 I .. 64 I + 63) keeps the tiles of
 * block columns I - bands .. I, tile (I, d) (block column I - d) at
 * tiles + (I * (bands + 1) + d) * 4096, row major, where tiles = storage + 256 bytes (the first
 * 256 bytes hold the factorisation's status and pivot range).  After the band, n_tiles more tiles
 * hold the inverses of the diagonal factor tiles.  Rows past n are identity rows. */
#define FEAB_BAND_TILE 64
#define FEAB_BAND_HEADER_BYTES 256

typedef struct feab_band {
  int32_t n;          /* rows                                                  */
  int32_t n_tiles;    /* block rows: ceil(n / 64)                              */
  int32_t bands;      /* sub-diagonal tile columns kept: ceil(bandwidth / 64)  */
  int32_t reserved;
  void* storage;      /* feab_band_bytes(n, bandwidth) bytes of device memory, 256-byte aligned */
} feab_band;

/* The largest |iperm[i] - iperm[j]| over the nonzeros (i, j) of A.  scratch: 2 int32 of device
 * memory.  An iperm entry outside [0, n) returns FEAB_BAD_ARG.  Synchronous. */
int32_t feab_band_width(const feab_csr* A, const int32_t* iperm, int32_t* scratch, int32_t* bandwidth_out,
                        cudaStream_t stream);

/* Bytes of band storage (header, band tiles, inverse diagonal tiles) for n rows and the given
 * bandwidth (0 if n <= 0). */
size_t feab_band_bytes(int32_t n, int32_t bandwidth);

/* Fills B with the lower band of the renumbered A; B->n, B->n_tiles and B->bands are set from
 * n and bandwidth, B->storage must be set by the caller.  An entry outside the band returns
 * FEAB_BAD_ARG.  Synchronous. */
int32_t feab_band_assemble(const feab_csr* A, const int32_t* iperm, int32_t bandwidth, feab_band* B,
                           cudaStream_t stream);

/* In-place Cholesky factorisation B = L L^T (tile by tile, on the stream; synchronous).
 * pivots_out[0] / [1]: the smallest and largest pivot L_ii^2 of rows < n.  A pivot <= 0 returns
 * FEAB_NOT_SPD (the factor is then not usable). */
int32_t feab_band_cholesky(feab_band* B, double* pivots_out, cudaStream_t stream);

/* x = (L L^T)^{-1} b in the renumbered order (b, x and work: n_tiles * 64 doubles of device
 * memory; the entries of b past n must be 0, and those of x past n are 0).  Asynchronous. */
int32_t feab_band_solve(const feab_band* B, const double* b, double* x, double* work, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* FEAB200_H */
