/*
 * qdkp -- C ABI of the B200 eight-band k.p eigensolve library (libqdkp.so, sm_100a).
 *
 * Drop-in boundary for qd3Dsolver's eigensolve hot path. The reference is pure Python; its
 * "interface" for this path is two Python entry points, and the functions below are what a
 * ctypes / cffi binding of those entry points calls:
 *
 *   kp_pryor.confined_hamiltonian(ops, fields, n_bands, hole_convention, strain,
 *                                 include_hydrostatic, interband_strain)   kp_pryor.py:363-466
 *       -> qdkp_operator_create / qdkp_operator_update_diagonal / qdkp_operator_destroy
 *   H @ X  (scipy CSR times a block, eigensolvers.py:86,98,307-308; scipy lobpcg.py:788)
 *       -> qdkp_apply, qdkp_apply_host
 *   eigensolvers.folded_operator(A, sigma)                                 eigensolvers.py:301-310
 *       -> qdkp_apply(..., QDKP_APPLY_FOLDED)
 *   eigensolvers.solve_interior / solve_lowest (scipy.sparse.linalg.lobpcg inside)
 *                                            eigensolvers.py:200-268, 313-372
 *       -> qdkp_lobpcg_workspace_size / qdkp_lobpcg_solve
 *   eigensolvers.residual_norms / rayleigh_quotients                       eigensolvers.py:76-101
 *       -> qdkp_residuals
 *
 * Conventions
 *   - Every function returns an int status: QDKP_OK (0) or a negative QDKP_ERR_* code;
 *     qdkp_last_error() returns the message of the last failure on the calling thread.
 *   - Grids are C-ordered (x slowest, z fastest); a coefficient field is n_sites doubles.
 *   - Vector blocks are row-major (n, m) complex arrays with a leading dimension ld >= m
 *     (numpy's C-ordered complex128 / complex64 layout); row = band * n_sites + site (band-major,
 *     kp_confined.py:66 with sp.bmat at kp_pryor.py:466).
 *   - "dev" pointers are CUDA device pointers on the operator's device; "stream" is a
 *     cudaStream_t passed as void* (NULL = legacy default stream).
 *   - The library allocates device memory only inside qdkp_operator_create (its coefficient
 *     fields). Every other buffer, workspaces included, belongs to the caller.
 */
#ifndef QDKP_H
#define QDKP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  QDKP_OK = 0,
  QDKP_ERR_ARG = -1,
  QDKP_ERR_CUDA = -2,
  QDKP_ERR_UNSUPPORTED = -3,
  QDKP_ERR_WORKSPACE = -4,
  QDKP_ERR_NUMERIC = -5
};

/* operator flags (kp_pryor.confined_hamiltonian keyword arguments) */
enum {
  QDKP_HOLE_CONVENTION = 1,  /* negate a 6- or 4-band operator (kp_pryor.py:239-240, 464) */
  QDKP_STRAIN = 2,           /* Bir-Pikus shear terms from the strain fields (kp_pryor.py:419-424) */
  QDKP_INTERBAND_STRAIN = 4, /* Pryor's u, v terms, 8-band only (kp_pryor.py:439-454) */
  QDKP_NEGATE = 8            /* apply -H (eigensolvers.solve_lowest_hole, eigensolvers.py:385) */
};

/* arithmetic of a vector block */
enum { QDKP_C128 = 0, QDKP_C64 = 1 };

/* qdkp_apply modes: Y = H X, Y = (H - sigma) X, Y = (H - sigma)^2 X */
enum { QDKP_APPLY_PLAIN = 0, QDKP_APPLY_SHIFTED = 1, QDKP_APPLY_FOLDED = 2 };

/* order of the 15 coefficient fields handed to qdkp_operator_create (kp_pryor.material_fields
 * keys plus the six strain components, kp_pryor.py:564-593, strain_fourier.py:84-139) */
enum {
  QDKP_FIELD_GAMMA1 = 0, QDKP_FIELD_GAMMA2, QDKP_FIELD_GAMMA3, QDKP_FIELD_P0, QDKP_FIELD_EC,
  QDKP_FIELD_EV, QDKP_FIELD_DELTA_SO, QDKP_FIELD_B, QDKP_FIELD_D, QDKP_FIELD_EXX,
  QDKP_FIELD_EYY, QDKP_FIELD_EZZ, QDKP_FIELD_EXY, QDKP_FIELD_EYZ, QDKP_FIELD_EZX,
  QDKP_FIELD_COUNT
};

typedef struct qdkp_operator qdkp_operator;

/* Number of CUDA kernels this library has launched in the process (diagnostic counter). */
int64_t qdkp_kernel_launches(void);

/* Last error message of the calling thread ("" if none). */
const char* qdkp_last_error(void);

/* Library version string. */
const char* qdkp_version(void);

/*
 * Build the device-resident operator; replaces kp_pryor.confined_hamiltonian
 * (kp_pryor.py:363-466) with `ops` = GridOperators(shape=(nx,ny,nz), h, periodic=False,
 * scheme='central') (kp_confined.py:398-454). fields[i] points to n_sites host doubles in
 * QDKP_FIELD_* order. Fields a model does not use may be NULL (P0 for 6/4 bands, strain when
 * QDKP_STRAIN is clear). The include_hydrostatic keyword is applied by the caller by folding
 * a_c Tr(eps) into Ec and -a_v Tr(eps) into Ev before the call (the same sum, kp_pryor.py:425-428).
 * n_bands is 8, 6 or 4 (kp_pryor.py:70).
 */
int qdkp_operator_create(int nx, int ny, int nz, double h, int n_bands, int flags,
                         const double* const* fields, int device, qdkp_operator** out);

/* Replace the Ec / Ev fields in place (Hartree or piezo potential updates that change only the
 * diagonal, as pryor_fig6.eight_band_states does per iteration, pryor_fig6.py:97-106).
 * Either pointer may be NULL to keep that field. Host doubles, n_sites each. */
int qdkp_operator_update_diagonal(qdkp_operator* op, const double* Ec, const double* Ev);

/* Grid shape, size and the nonzero count of the equivalent CSR (H.shape / H.nnz in
 * pryor_fig4.py:148, heterostructure.py:842,988). Any output pointer may be NULL. */
int qdkp_operator_info(const qdkp_operator* op, int* nx, int* ny, int* nz, int* n_bands,
                       int64_t* n, int64_t* nnz);

int qdkp_operator_destroy(qdkp_operator* op);

/* Structural nonzero count of the CSR kp_pryor.confined_hamiltonian assembles for this grid
 * and flags (every stencil coupling counted, clipped at the walls). scipy additionally drops
 * entries whose value cancels to exactly 0 (e.g. diagonal strain terms on symmetry planes), so
 * the reference's H.nnz is at most this. Needs no GPU. */
int64_t qdkp_structural_nnz(int nx, int ny, int nz, int n_bands, int flags);

/*
 * Y = op(X) on device blocks: X (n, m) with leading dimension ldx, Y (n, m) with ldy, both
 * complex128 (precision QDKP_C128) or complex64 (QDKP_C64). mode QDKP_APPLY_FOLDED needs a
 * workspace of n * m complex elements of the same precision (ws, ws_bytes); the other modes
 * take ws = NULL. X and Y must not overlap.
 */
int qdkp_apply(const qdkp_operator* op, const void* X, int64_t ldx, void* Y, int64_t ldy,
               int m, double sigma, int mode, int precision, void* ws, size_t ws_bytes,
               void* stream);

/*
 * No counterpart in the reference (its folded operator is a Python closure). Allocation-free
 * variant of qdkp_apply(..., QDKP_APPLY_FOLDED): Y = (H - sigma)^2 X with the intermediate
 * (H - sigma) X held in a fixed device array built into the library, so the caller passes only
 * X and Y. It is for callers that cannot allocate device memory when they apply the operator:
 * bindings from languages with no device allocator of their own, code running where the
 * implicit device synchronisation of cudaMalloc is not allowed (callbacks, latency-critical
 * loops), or processes whose device memory is managed by another runtime.
 *   - Limit: n * m complex elements must fit QDKP_NOALLOC_SCRATCH_BYTES (64 MiB: 4 Mi complex128
 *     or 8 Mi complex64 elements); larger blocks are rejected with QDKP_ERR_WORKSPACE and a
 *     message, and must use qdkp_apply with a workspace.
 *   - Every GPU that loads libqdkp.so keeps those 64 MiB until the process exits.
 *   - The first call on a device looks up the array's device address (cudaGetSymbolAddress,
 *     with that device current); make that first call before any stream capture. The address
 *     is kept for the life of the process: a device reset (cudaDeviceReset) invalidates it, so
 *     do not use this entry point on a device after resetting it.
 *   - The call makes the operator's device current and restores the caller's current device.
 *   - No cudaMalloc, cudaFree or other allocating routine is called.
 *   - All calls share the one array, which keeps the last call's contents; calls that overlap
 *     on the GPU (different streams or threads, without ordering between them) race on it.
 *     Nothing needs clearing: each call writes every element it later reads.
 */
#define QDKP_NOALLOC_SCRATCH_BYTES (64ull << 20)
size_t qdkp_apply_folded_noalloc_max_elems(int precision);
int qdkp_apply_folded_noalloc(const qdkp_operator* op, const void* X, int64_t ldx, void* Y,
                              int64_t ldy, int m, double sigma, int precision, void* stream);

/*
 * H.X kernel selection (no counterpart in the reference, which multiplies an assembled CSR).
 * Eight-band operators are applied by a staged kernel: a CTA owns a (y, z) tile of sites and a
 * few columns, walks along x and keeps a ring of x planes in shared memory. Tiles 0..3 fill the
 * ring with cp.async (both precisions); tiles 4..11 (complex64 only) fill it with bulk tensor
 * copies (TMA) and give every thread two columns of a site; tiles 12..16 (complex64 only) do the
 * same with a producer warp and per-slot full/empty barriers, the record read from global
 * memory by the threads of its site. A block the tensor maps cannot
 * describe (odd leading dimension, a base not 16-byte aligned, fewer columns than a tile or a
 * grid smaller than a tile) falls back to a cp.async tile. The tile is chosen by a heuristic
 * unless set here or by qdkp_operator_tune; QDKP_TILE_DIRECT selects the unstaged
 * one-thread-per-(site, column) kernel (always used for 6- and 4-band slices). The choice is per
 * operator and precision.
 */
enum { QDKP_TILE_AUTO = -1, QDKP_TILE_DIRECT = -2, QDKP_TILE_COUNT = 17 };
int qdkp_operator_set_tile(qdkp_operator* op, int precision, int tile);
int qdkp_operator_get_tile(const qdkp_operator* op, int precision, int* tile);
/* Autotuner: times every tile shape and the direct kernel on the caller's device blocks X, Y
 * (n x m, `precision`) with `reps` launches each, keeps the fastest for this operator and
 * precision, and writes the per-candidate seconds per launch to seconds[QDKP_TILE_COUNT + 1]
 * (may be NULL; index QDKP_TILE_COUNT is the direct kernel; -1 marks a candidate that does not
 * apply to this block or precision). Y is overwritten. Synchronous. */
int qdkp_operator_tune(qdkp_operator* op, const void* X, int64_t ldx, void* Y, int64_t ldy,
                       int m, int precision, int reps, double* seconds, void* stream);

/* Kernels that wait on their own bulk copies give up after about a second if a copy never lands
 * (a fault elsewhere on the device) and set a device flag instead of hanging. *fault receives the
 * flag of `device` (0 = none); clear = 1 resets it. Synchronous; the current device is kept. */
int qdkp_device_fault(int device, int clear, int* fault);

/* Workspace bytes qdkp_apply_host needs for an (n, m) complex128 block in `mode`. */
size_t qdkp_apply_host_workspace_size(const qdkp_operator* op, int m, int mode);

/* The same apply on HOST complex128 buffers (the `A @ X` a scipy LinearOperator performs):
 * copies X to the device workspace, applies, copies Y back; synchronous on `stream`. */
int qdkp_apply_host(const qdkp_operator* op, const void* X_host, void* Y_host, int m,
                    double sigma, int mode, void* ws, size_t ws_bytes, void* stream);

/*
 * LOBPCG (scipy.sparse.linalg.lobpcg as called by eigensolvers.py:247-248, 352-353:
 * B = None, Y = None, largest = False) on A = op (folded = 0) or A = (op - sigma)^2
 * (folded = 1, eigensolvers.folded_operator). All vectors stay on the device.
 */
typedef struct {
  int block;             /* sizeX, columns of X0 */
  int folded;            /* 1: A = (H - sigma)^2 (solve_interior), 0: A = H (solve_lowest) */
  double sigma;
  double tol;            /* residual tolerance on A; <= 0 selects sqrt(eps) * n (scipy) */
  int maxiter;
  int restart_control;   /* forced restart when the mean residual exceeds 2^this x best (20) */
  int precision;         /* QDKP_C128 (plain) or QDKP_C64 (search directions in complex64) */
  int verbosity;         /* 0 = silent */
  int time_hx;           /* 1: time every H X launch with CUDA events (info->hx_seconds) */
  int stall_iterations;  /* batched engine only: > 0 stops a slot (status QDKP_LOBPCG_MAXITER)
                            once its best mean residual is this many iterations old; used to end
                            a complex64 search phase that has reached its rounding floor */
} qdkp_lobpcg_params;

typedef struct {
  int iterations;          /* len(residualNormsHistory) as scipy returns it */
  int best_iteration;
  int status;              /* QDKP_LOBPCG_* below */
  int explicit_gram;       /* 1 once the Gram matrices were formed explicitly */
  double best_mean_residual;
  double seconds;          /* wall time inside qdkp_lobpcg_solve */
  int64_t hx_applications; /* H X column applications (folded counts two per column) */
  int64_t hx_launches;     /* H X kernel launches */
  double hx_seconds;       /* summed CUDA-event time of those launches (time_hx = 1) */
  double hx_bytes;         /* algorithmic bytes of those launches: N (15 s_f + 2*8 m s_c) each */
} qdkp_lobpcg_info;

enum {
  QDKP_LOBPCG_CONVERGED = 0,        /* every residual below tol */
  QDKP_LOBPCG_MAXITER = 1,          /* ran out of iterations; best iterate returned */
  QDKP_LOBPCG_RCHOL_BREAKDOWN = 2,  /* Cholesky of the residual Gram failed (scipy breaks) */
  QDKP_LOBPCG_EIGH_BREAKDOWN = 3,   /* the restart Rayleigh-Ritz eigh failed (scipy breaks) */
  QDKP_LOBPCG_NONFINITE = 4         /* a residual became NaN/inf */
};

/* Workspace bytes qdkp_lobpcg_solve needs for an n x block problem. */
size_t qdkp_lobpcg_workspace_size(const qdkp_operator* op, const qdkp_lobpcg_params* prm);

/*
 * Run LOBPCG. X0 (device, n x block complex128, leading dimension block) is the start block
 * and is not modified. On return lambda[block] (host) holds the final Ritz values of A in
 * ascending order and V (device, n x block complex128) the Ritz vectors of the best iterate
 * after the final Rayleigh-Ritz (scipy lobpcg.py:1009-1060); resid_history (host, may be
 * NULL) receives (maxiter + 3) x block residual norms, row-major, info->iterations rows used.
 */
int qdkp_lobpcg_solve(const qdkp_operator* op, const qdkp_lobpcg_params* prm, const void* X0,
                      double* lambda, void* V, double* resid_history, qdkp_lobpcg_info* info,
                      void* ws, size_t ws_bytes, void* stream);

/*
 * Batched LOBPCG engine (no counterpart in the reference, which solves one operator at a time):
 * many folded or plain eight-band solves resident on the GPU, advanced together one LOBPCG
 * iteration (the same scipy iteration as qdkp_lobpcg_solve) per tick, with every decision taken
 * on the device. Slots are admitted and retired between steps; each slot's workspace
 * (qdkp_engine_slot_workspace_size bytes) belongs to the caller and must stay alive until the
 * slot is retired. A solve gives the same result alone and in any mix.
 */
typedef struct qdkp_engine qdkp_engine;
int qdkp_engine_create(int max_slots, int device, qdkp_engine** out);
int qdkp_engine_destroy(qdkp_engine* e);
size_t qdkp_engine_slot_workspace_size(const qdkp_operator* op, const qdkp_lobpcg_params* prm);
/* Admit one solve: orthonormalises X0 (device, n x block complex128) and runs the initial
 * Rayleigh-Ritz step (synchronous on `stream`). *slot receives the slot id. */
int qdkp_engine_admit(qdkp_engine* e, const qdkp_operator* op, const qdkp_lobpcg_params* prm,
                      const void* X0, void* ws, size_t ws_bytes, void* stream, int* slot);
/* Launch `ticks` iterations of every running slot (asynchronous on `stream`). The tick sequence
 * is fixed for a slot layout, so by default it is captured once per layout (and tick count) as
 * a CUDA graph and replayed on the engine's own stream, ordered after `stream` and before later
 * work on it by events. */
int qdkp_engine_step(qdkp_engine* e, int ticks, void* stream);
/* 0: launch the tick kernels directly on the caller's stream instead of replaying a graph. */
int qdkp_engine_set_graphs(qdkp_engine* e, int enable);
/* state[max_slots]: -1 free, 1 running, 0 stopped (status[] gives QDKP_LOBPCG_*);
 * iterations[] = iterations started so far. Synchronous. */
int qdkp_engine_poll(qdkp_engine* e, int* state, int* status, int* iterations, void* stream);
/* Final Rayleigh-Ritz on the slot's best iterate (lobpcg.py:1009-1060): lambda[block] (host),
 * V (device, n x block complex128), residuals[block] (host, may be NULL); frees the slot. */
int qdkp_engine_retire(qdkp_engine* e, int slot, double* lambda, void* V, double* residuals,
                       qdkp_lobpcg_info* info, void* stream);

/*
 * The tall-skinny block products of scipy's LOBPCG (the Gram assembly X^H A X, X^H A R, ... at
 * lobpcg.py:833-880 and the Ritz updates X Cx + R Cr + P Cp at lobpcg.py:921-973), on device
 * blocks of complex128 (FP64 tensor-core MMA) or complex64 (split-precision TF32 tensor-core MMA
 * accumulated in FP32, partial sums in FP64).
 *   qdkp_block_gram:   out (host, P x Q complex128, row-major) = A^H B, A (n x P, lda), B (n x Q)
 *   qdkp_block_update: Y (n x q) = A (n x P) C, C (host, P x q complex128, row-major)
 * Synchronous on `stream`; workspaces from the *_workspace_size functions. Complex64 updates (here
 * and in the engine) run on the split-TF32 mma.sync kernel unless the environment variable
 * QDKP_C64_UPDATE=tcgen05 selects the tcgen05 / TMEM pipeline; it is read once per process.
 */
size_t qdkp_block_gram_workspace_size(int P, int Q);
int qdkp_block_gram(const void* A, int64_t lda, int P, const void* B, int64_t ldb, int Q,
                    int64_t n, int precision, double* out, void* ws, size_t ws_bytes,
                    void* stream);
size_t qdkp_block_update_workspace_size(int P, int q);
int qdkp_block_update(const void* A, int64_t lda, int P, const double* C, int q, int64_t n,
                      void* Y, int64_t ldy, int precision, void* ws, size_t ws_bytes,
                      void* stream);

/*
 * The Rayleigh-Ritz eigensolve of a LOBPCG iteration, eigh(gramA, gramB) (scipy lobpcg.py:891-909):
 * A, B host n x n complex128 Hermitian (row-major; B NULL for
 * the identity), n <= 72. All n eigenpairs (nwant = n) by Householder + QL, or only the nwant
 * smallest (1 <= nwant < n) by multisection and inverse iteration, the form the LOBPCG iterations
 * use (they keep the block-size smallest). w (host, n doubles) ascending in its first nwant
 * entries; V (host, n x n complex128, row-major) eigenvectors in its first nwant columns,
 * B-orthonormal. Returns QDKP_OK, or QDKP_ERR_NUMERIC when B is not positive definite or the
 * spectrum is not finite. Synchronous on `stream`; workspace qdkp_block_eigh_workspace_size(n).
 */
size_t qdkp_block_eigh_workspace_size(int n);
int qdkp_block_eigh(const double* A, const double* B, int n, int nwant, double* w, double* V,
                    void* ws, size_t ws_bytes, void* stream);

/*
 * Rayleigh quotients and residual norms of H for the columns of V (device, n x k complex128,
 * leading dimension ldv): rq[j] = v^H H v / v^H v and res[j] = ||H v_j - E_j v_j|| on the
 * normalised v_j, with E = E_in if non-NULL else rq (eigensolvers.residual_norms /
 * rayleigh_quotients, eigensolvers.py:76-101). rq and res are host arrays of k doubles.
 * Workspace: qdkp_residuals_workspace_size bytes.
 */
size_t qdkp_residuals_workspace_size(const qdkp_operator* op, int k);
int qdkp_residuals(const qdkp_operator* op, const void* V, int64_t ldv, int k,
                   const double* E_in, double* rq, double* res, void* ws, size_t ws_bytes,
                   void* stream);

/*
 * Localisation and Kramers pairing of eigenvector blocks (pryor_fig4.localization,
 * pryor_fig4.py:179-193, and pryor_fig4.kramers_levels, pryor_fig4.py:222-236).
 * V: device (n, k) block, complex128 or complex64 (`precision`), leading dimension ldv, rows
 * band-major as H's; mask: device array of n_sites bytes, nonzero inside the dot.
 * loc[k] (host): sum over dot sites and bands of |V_j|^2 over the same sum over every site.
 * E (host, may be NULL): k energies in the order to pair; consecutive entries form a pair, and
 * levels[k/2], level_loc[k/2] receive each pair's mean energy and mean localisation and
 * *worst_split the largest within-pair |E_2p+1 - E_2p|. Sums run in a fixed order: the result is
 * the same for any launch and any other work on the GPU. Synchronous; k <= 128.
 */
size_t qdkp_state_summary_workspace_size(const qdkp_operator* op, int k);
int qdkp_state_summary(const qdkp_operator* op, const void* V, int64_t ldv, int k, int precision,
                       const unsigned char* mask, const double* E, double* loc, double* levels,
                       double* level_loc, double* worst_split, void* ws, size_t ws_bytes,
                       void* stream);

/*
 * Local band edges at k = 0 from the operator's own fields (kp_pryor.local_band_edges,
 * kp_pryor.py:469-531, with the hydrostatic shift already in Ev, and kp_pryor.hole_sigma,
 * kp_pryor.py:156-191): per site the three Kramers-paired levels v1 >= v2 >= v3 of the 6x6
 * valence block (Ev, delta_so, the Bir-Pikus terms of the strain fields with b and d).
 * levels (device, 3 x n_sites doubles, may be NULL) receives v1, v2, v3; *top_v1 (host) the
 * largest v1 over the sites where mask (device, n_sites bytes, may be NULL for every site) is
 * nonzero -- hole_sigma with margin 0; *kramers_split (host, may be NULL) the largest splitting
 * within a level pair over all sites. Operators of 8 or 6 bands. Synchronous.
 */
size_t qdkp_local_band_edges_workspace_size(const qdkp_operator* op);
int qdkp_local_band_edges(const qdkp_operator* op, const unsigned char* mask, double* levels,
                          double* top_v1, double* kramers_split, void* ws, size_t ws_bytes,
                          void* stream);

/*
 * Host input producers on the device: the homogeneous Fourier strain of a dot
 * (strain_fourier.solve_strain, strain_fourier.py:142-235) and the first-order piezoelectric
 * potential (piezoelectric.potential with polarization / charge_density, piezoelectric.py:59-99),
 * on the periodic (nx, ny, nz) cell of spacing h (C order, z fastest).
 *   qdkp_fourier_strain: mask (device, n_sites bytes); strain (device, 6 x n_sites doubles) gets
 *     the ELASTIC strain exx, eyy, ezz, exy, eyz, ezx (tensor shear convention).
 *   qdkp_piezo_potential: strain (device, 6 x n_sites, that order), e14 (device field, n_sites),
 *     scalar eps_r; phi (device, n_sites) in volts.
 * The 3-D transforms are cuFFT double-complex plans, made once per grid shape (cuFFT keeps its
 * own small tables on the device) and run with the work area in the caller's workspace.
 * Asynchronous on `stream`.
 */
/*
 * Inhomogeneous elastic strain by the FD (Q1 finite-element) energy minimisation of
 * elasticity_fd.solve_strain_fd (elasticity_fd.py:211-419): trilinear hexahedra with 2x2x2 Gauss
 * quadrature on the periodic (nx, ny, nz) cell of spacing h, the dot (mask, device, n_sites
 * bytes, on element centres) with its own cubic constants C_dot[3] = (C11, C12, C44) and the
 * matrix with C_matrix[3], the dilatational eigenstrain -eps_star inside the dot; solved by CG
 * preconditioned with the exact Fourier inverse of the volume-averaged homogeneous operator, to
 * ||r|| / ||f|| < tol or maxiter iterations. strain (device, 6 x n_sites) gets the ELASTIC strain
 * exx, eyy, ezz, exy, eyz, ezx at the element centres; total (device, may be NULL) the total
 * strain (no eigenstrain term). info (host) receives iterations, relative residual, the dropped
 * preconditioner modes (1 = only k = 0), a breakdown code (0 none; 1 preconditioner not positive
 * definite; 2 non-positive curvature; 3 preconditioner lost definiteness) and converged
 * (residual below tol, no breakdown, no dropped mode but k = 0). Synchronous on `stream`.
 */
typedef struct {
  int iterations;
  double residual;
  int modes_dropped;
  int breakdown;
  int converged;
} qdkp_fd_info;
size_t qdkp_fd_strain_workspace_size(int nx, int ny, int nz);
int qdkp_fd_strain(int nx, int ny, int nz, double h, const unsigned char* mask, double eps_star,
                   const double* C_dot, const double* C_matrix, double tol, int maxiter,
                   double* strain, double* total, qdkp_fd_info* info, void* ws, size_t ws_bytes,
                   void* stream);

size_t qdkp_fourier_strain_workspace_size(int nx, int ny, int nz);
int qdkp_fourier_strain(int nx, int ny, int nz, double h, const unsigned char* mask,
                        double eps_star, double C11, double C12, double C44, double* strain,
                        void* ws, size_t ws_bytes, void* stream);
size_t qdkp_piezo_potential_workspace_size(int nx, int ny, int nz);
int qdkp_piezo_potential(int nx, int ny, int nz, double h, const double* strain,
                         const double* e14, double eps_r, double sign, double* phi, void* ws,
                         size_t ws_bytes, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* QDKP_H */
