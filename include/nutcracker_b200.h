/*
 * nutcracker_b200.h - C-ABI of the B200 (sm_100a) variational-MPS sweep path.
 *
 * Level 0: drop-in replacements for the Fortran-ABI numeric kernels that the
 * reference's C++ layer binds in sources/common/core.cpp (declared there as
 * extern "C" with trailing underscores).  Same names, same argument order and
 * meaning: every scalar is passed by pointer, buffers are column-major
 * complex128 (layout-compatible with std::complex<double>), MPO indices are
 * uint32 (from,to) pairs, 1-based, and outputs are caller-allocated HOST
 * buffers.  Each call copies its inputs to the GPU, runs the CUDA kernels and
 * copies the outputs back.  Unlike the reference (which calls Fortran `stop`
 * on LAPACK errors), no entry point ever exits the process: failures are
 * reported through the return code where the reference has one, and always
 * through nc_last_status()/nc_last_error().
 *
 * Level 1: device-resident chain handle (nc_chain_*), the performance
 * drop-in for Nutcracker::Chain (includes/nutcracker/chain.hpp:115-235):
 * sites, environments and projectors stay in HBM across sweeps.
 */
#ifndef NUTCRACKER_B200_H
#define NUTCRACKER_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } nc_complex; /* == std::complex<double> */

/* ---- error reporting --------------------------------------------------- */
/* Status of the last call on this host thread (0 = success). */
int nc_last_status(void);
/* Message of the last failing call on this host thread ("" if none). */
const char* nc_last_error(void);
/* Kernels this library has launched on this host thread's context. */
uint64_t nc_launch_count(void);
/* Library version string. */
const char* nc_version(void);
/* Enqueue this thread's work on `stream` (a cudaStream_t; NULL is the
   legacy default stream).  Returns a status code. */
int nc_set_stream(void* stream);
/* Go back to the library's own non-blocking stream (the initial state). */
int nc_use_own_stream(void);
/* Wait for this thread's stream.  Returns a status code. */
int nc_synchronize(void);
/* Start timing every complex GEMM of at least `min_flops` algorithmic flops
   with CUDA events on this thread's stream. */
int nc_profile_begin(double min_flops);
/* Stop timing; report the number of timed FP64 complex GEMMs, their summed
   device time (ms) and summed algorithmic flops (8*M*N*K per complex
   product). */
int nc_profile_end(uint64_t* launches, double* total_ms, double* total_flops);
/* Without stopping: the same totals for one kind of timed GEMM, kind 0 =
   FP64 complex GEMM, kind 1 = tcgen05 3xTF32 GEMM (flops counted as the
   TF32 tensor work, 2*M*Nr*Kr per segment, three segments per product). */
int nc_profile_query(int kind, uint64_t* launches, double* total_ms, double* total_flops);

/* Device-pointer effective-Hamiltonian product y = H_eff x for one site
   (the strategy-3 `operate_on` of core.f95:2529-2556 without projectors):
   L (bl,bl,cl), R (br,br,cr), x and y (br,bl,d), W (d,d,nnz), idx (2,nnz)
   1-based, all in device memory.  Scratch comes from the library's device
   arena.  Asynchronous on this thread's stream; returns a status code. */
int nc_heff_apply_dev(uint32_t bl, uint32_t br, uint32_t cl, uint32_t cr, uint32_t d, uint32_t nnz,
                      const uint32_t* idx_dev, const void* W_dev, const void* L_dev,
                      const void* R_dev, const void* x_dev, void* y_dev);

/* Precision form of nc_heff_apply_dev: the two complex contractions run on
   the tcgen05 tensor cores in 3xTF32 (each operand split into two TF32
   halves, three products, FP32 accumulation); the input, output and the
   sparse-MPO mix stay FP64.  Relative error ~1e-6 of |H_eff x|.  Device
   pointers as for nc_heff_apply_dev; synchronises this thread's stream
   before returning.  Returns a status code. */
int nc_heff_apply_mixed_dev(uint32_t bl, uint32_t br, uint32_t cl, uint32_t cr, uint32_t d, uint32_t nnz,
                            const uint32_t* idx_dev, const void* W_dev, const void* L_dev,
                            const void* R_dev, const void* x_dev, void* y_dev);

/* Device-pointer environment update for one site: side 0 is
   contract_sos_left (L (bl,bl,cl) -> L' (br,br,cr), core.f95:623-677),
   side 1 is contract_sos_right (R (br,br,cr) -> R' (bl,bl,cl),
   core.f95:679-848); psi (br,bl,d).  mixed = 0 runs the FP64 path, mixed = 1
   the precision form (3xTF32 tensor-core contractions, FP64 input/output;
   synchronises this thread's stream).  Returns a status code. */
int nc_env_update_dev(int side, int mixed, uint32_t bl, uint32_t br, uint32_t cl, uint32_t cr, uint32_t d,
                      uint32_t nnz, const uint32_t* idx_dev, const void* W_dev, const void* env_dev,
                      const void* psi_dev, void* out_dev);

/* Device-pointer gauge move (norm_denorm_going_right_ / _left_ of
   core.f95:2708-2878, QR gauge): direction > 0 left-normalises A (bm,bl,dl)
   into out_A and lets B (br,bm,dr) absorb the factor into out_B; direction < 0
   right-normalises B into out_B and lets A absorb the factor into out_A.  All
   buffers in device memory; inputs are not modified.  Asynchronous on this
   thread's stream; returns a status code. */
int nc_gauge_move_dev(int direction, uint32_t bl, uint32_t bm, uint32_t br, uint32_t dl, uint32_t dr,
                      const void* A_dev, const void* B_dev, void* out_A_dev, void* out_B_dev);

/* C = A B for column-major complex128 device matrices A (M x K), B (K x N),
   C (M x N) on the tcgen05 tensor cores: 3xTF32 when `three` is nonzero,
   else one TF32 product.  The GEMM under the precision form, exposed for
   testing; synchronises this thread's stream.  Returns a status code. */
int nc_tc_zgemm_dev(uint32_t M, uint32_t N, uint32_t K, const void* A_dev, const void* B_dev,
                    void* C_dev, int three);

/* No counterpart in the reference; for tests of the failure path.  Sets
   the time limit of every mbarrier wait in the tcgen05 GEMM (default 2 s,
   here in nanoseconds, at least 1000) and, when skip_first_load is nonzero,
   makes tile (0,0,0) of the following GEMMs leave its first K stage
   unloaded, so that a wait runs out: the kernel then stops issuing, leaves
   through its final barrier and frees its tensor memory, and the host call
   reports NC_ERR_TIMEOUT.  Process-wide; restore (2000000000, 0) after use.
   Returns a status code. */
int nc_test_tc32_wait(uint64_t wait_ns, int skip_first_load);

/* No counterpart in the reference.  The same H_eff product as
   nc_heff_apply_dev for callers that cannot let the library allocate
   device memory (a fixed memory budget, or code where a cudaMalloc/cudaFree
   would stall the device): it allocates nothing and takes its scratch from
   one fixed 64 MiB device array compiled into the library, which every GPU
   that loads the library holds until exit.  A call needs
   16*(br*bl*cl*d + br*cr*bl*d) bytes of it; larger calls return an error
   and launch nothing.  Work is enqueued on `stream` (a cudaStream_t, NULL =
   legacy default stream).  The first call on each device looks the array's
   device address up (cudaGetSymbolAddress); make it before any stream
   capture.  All calls share the array and each rewrites it completely, so
   nothing needs clearing, but calls that overlap on the GPU race: order them
   on one stream.  The (from, to) indices in idx_dev stay on the device and
   are not range-checked: each pair must satisfy 1 <= from <= cl and
   1 <= to <= cr.  Every dimension must be at least 1 (checked).
   Returns a status code. */
int nc_heff_apply_dev_noalloc(uint32_t bl, uint32_t br, uint32_t cl, uint32_t cr, uint32_t d,
                              uint32_t nnz, const uint32_t* idx_dev, const void* W_dev,
                              const void* L_dev, const void* R_dev, const void* x_dev,
                              void* y_dev, void* stream);

/* ---- Level 0: contractions (sources/common/core.cpp:33-526) ------------- */

/* core.cpp:33-45 (compute_expectation_): <psi|H|psi> at one site. */
void compute_expectation_(const uint32_t* bl, const uint32_t* br, const uint32_t* cl,
                          const uint32_t* cr, const uint32_t* d, const nc_complex* left_environment,
                          const nc_complex* state_site_tensor, const uint32_t* number_of_matrices,
                          const uint32_t* sparse_operator_indices,
                          const nc_complex* sparse_operator_matrices,
                          const nc_complex* right_environment, nc_complex* expectation);

/* core.cpp:75-86 (compute_optimization_matrix_): dense H_eff, (br*bl*d)^2. */
void compute_optimization_matrix_(const uint32_t* bl, const uint32_t* br, const uint32_t* cl,
                                  const uint32_t* cr, const uint32_t* d,
                                  const nc_complex* left_environment,
                                  const uint32_t* number_of_matrices,
                                  const uint32_t* sparse_operator_indices,
                                  const nc_complex* sparse_operator_matrices,
                                  const nc_complex* right_environment,
                                  nc_complex* optimization_matrix);

/* core.cpp:139-144 (construct_left_exp_boundary_). */
void construct_left_exp_boundary_(const uint32_t* b, const uint32_t* c,
                                  const nc_complex* state_boundary,
                                  const nc_complex* operator_boundary,
                                  nc_complex* left_expectation_boundary);
/* core.cpp:161-166 (construct_right_exp_boundary_). */
void construct_right_exp_boundary_(const uint32_t* b, const uint32_t* c,
                                   const nc_complex* state_boundary,
                                   const nc_complex* operator_boundary,
                                   nc_complex* right_expectation_boundary);
/* core.cpp:183-189 (contract_expectation_boundaries_). */
void contract_expectation_boundaries_(const uint32_t* b, const uint32_t* c,
                                      const nc_complex* left_boundary,
                                      const nc_complex* right_boundary, nc_complex* expectation);

/* core.cpp:235-247 (contract_sos_left_): new left environment (br,br,cr). */
void contract_sos_left_(const uint32_t* bl, const uint32_t* br, const uint32_t* cl,
                        const uint32_t* cr, const uint32_t* d, const nc_complex* left_environment,
                        const uint32_t* number_of_matrices, const uint32_t* sparse_operator_indices,
                        const nc_complex* sparse_operator_matrices,
                        const nc_complex* state_site_tensor, nc_complex* new_left_environment);
/* core.cpp:272-284 (contract_sos_right_): new right environment (bl,bl,cl). */
void contract_sos_right_(const uint32_t* bl, const uint32_t* br, const uint32_t* cl,
                         const uint32_t* cr, const uint32_t* d, const nc_complex* right_environment,
                         const uint32_t* number_of_matrices, const uint32_t* sparse_operator_indices,
                         const nc_complex* sparse_operator_matrices,
                         const nc_complex* state_site_tensor, nc_complex* new_right_environment);
/* core.cpp:309-318 (contract_vs_left_). */
void contract_vs_left_(const uint32_t* b_left_old, const uint32_t* b_right_old,
                       const uint32_t* b_left_new, const uint32_t* b_right_new, const uint32_t* d,
                       const nc_complex* left_environment,
                       const nc_complex* normalized_projector_site_tensor,
                       const nc_complex* normalized_state_site_tensor,
                       nc_complex* new_left_environment);
/* core.cpp:340-349 (contract_vs_right_). */
void contract_vs_right_(const uint32_t* b_left_old, const uint32_t* b_right_old,
                        const uint32_t* b_left_new, const uint32_t* b_right_new, const uint32_t* d,
                        const nc_complex* right_environment,
                        const nc_complex* normalized_projector_site_tensor,
                        const nc_complex* normalized_state_site_tensor,
                        nc_complex* new_right_environment);
/* core.cpp:517-526 (form_overlap_vector_). */
void form_overlap_vector_(const uint32_t* b_left_old, const uint32_t* b_right_old,
                          const uint32_t* b_left_new, const uint32_t* b_right_new,
                          const uint32_t* d, const nc_complex* left_environment,
                          const nc_complex* right_environment,
                          const nc_complex* unnormalized_projector_site_tensor,
                          nc_complex* overlap_vector);
/* core.cpp:498-504 (form_overlap_site_tensor_). */
void form_overlap_site_tensor_(const uint32_t* br, const uint32_t* bl, const uint32_t* d,
                               const nc_complex* state_site_tensor,
                               nc_complex* overlap_site_tensor);

/* core.cpp:210-231 (contract_matrix_left_): L' (br,br) = M L M^H. */
void contract_matrix_left_(const uint32_t* bl, const uint32_t* br, const nc_complex* left_environment,
                           const nc_complex* matrix, nc_complex* new_left_environment);
/* core.cpp:400-427 (extend_state_vector_fragment_, used by flat.cpp):
   new (br,dr,dl) = sum_m site(br,m,dr) old(m,dl). */
void extend_state_vector_fragment_(const uint32_t* bm, const uint32_t* br, const uint32_t* dl,
                                   const uint32_t* dr, const nc_complex* old_state_vector_fragment,
                                   const nc_complex* site_tensor, nc_complex* new_state_vector_fragment);
/* core.cpp:785-818 (increase_bandwidth_with_environment_): the infinite-chain
   routine; exported so the reference's C++ layer links, and always fails with
   NC_ERR_ARG (the infinite chain is not supported). */
void increase_bandwidth_with_environment_(const uint32_t* b, const uint32_t* c, const uint32_t* d,
                                          const uint32_t* new_b, const nc_complex* old_state_site_tensor,
                                          const nc_complex* old_left_exp_environment,
                                          const nc_complex* old_right_exp_environment,
                                          nc_complex* new_state_site_tensor, nc_complex* new_left_exp_environment,
                                          nc_complex* new_right_exp_environment);

/* ---- Level 0: site eigen-solve and projectors (core.cpp:109-441, 676-774) -------- */

/* core.cpp:676-693 (optimize_): the site eigen-solve.  Returns the
   reference's info code: 0 success, 5 orthogonal dimension too large,
   10 no room left by the projectors, 11 guess inside the projector space,
   -14 (as uint32) no convergence within `number_of_iterations` restart
   cycles; 0xFFFFFFFF on an argument/CUDA error (see nc_last_error()).
   `which` is the 2-character ARPACK selector "SR", "LR" or "LM"; on output
   number_of_iterations holds the number of H_eff products (0 when the
   orthogonal space has at most 4 dimensions, like the reference's dense
   strategy 1). */
uint32_t optimize_(const uint32_t* bl, const uint32_t* br, const uint32_t* cl, const uint32_t* cr,
                   const uint32_t* d, const nc_complex* left_environment,
                   const uint32_t* number_of_matrices, const uint32_t* sparse_operator_indices,
                   const nc_complex* sparse_operator_matrices, const nc_complex* right_environment,
                   const uint32_t* number_of_projectors, const uint32_t* number_of_reflectors,
                   const uint32_t* orthogonal_subspace_dimension, const nc_complex* reflectors,
                   const nc_complex* coefficients, const uint32_t* swaps, const char* which,
                   const double* tol, uint32_t* number_of_iterations, const nc_complex* guess,
                   nc_complex* result, nc_complex* eigenvalue, double* normal);

/* core.cpp:371-378 (convert_vectors_to_reflectors_): pivoted Householder QR
   of `m` overlap vectors of length `n`, in place; rank and swaps out. */
void convert_vectors_to_reflectors_(const uint32_t* n, const uint32_t* m, nc_complex* vectors,
                                    uint32_t* rank, nc_complex* coefficients, uint32_t* swaps);

/* core.cpp:431-441 (filter_components_outside_orthog_): output = the input
   with its components in the projector space removed. */
void filter_components_outside_orthog_(const uint32_t* full_space_dimension,
                                       const uint32_t* number_of_projectors,
                                       const uint32_t* number_of_reflectors,
                                       const uint32_t* orthogonal_subspace_dimension,
                                       const nc_complex* reflectors, const nc_complex* coefficients,
                                       const uint32_t* swaps, const nc_complex* input,
                                       nc_complex* output);

/* core.cpp:109-118 (compute_overlap_with_projectors_): the Fortran routine
   writes a real overlap; it is returned in overlap->re with overlap->im = 0. */
void compute_overlap_with_projectors_(const uint32_t* number_of_projectors,
                                      const uint32_t* number_of_reflectors,
                                      const nc_complex* reflectors, const nc_complex* coefficients,
                                      const uint32_t* swaps, const uint32_t* vector_size,
                                      const nc_complex* vector, nc_complex* overlap);

/* core.cpp:769-774 (random_projector_matrix_): reflectors of random
   projector vectors (seeded device generator instead of gfortran rand()). */
void random_projector_matrix_(const uint32_t* projector_length, const uint32_t* number_of_projectors,
                              uint32_t* rank, nc_complex* reflectors, nc_complex* coefficients,
                              uint32_t* swaps);

/* Lanczos basis size used by optimize_ on this thread (default 24). */
int nc_set_krylov_dimension(int m);

/* ---- Level 0: gauge moves and random sites (core.cpp:463-662, 735-757) --
   norm_denorm_going_left_/right_, norm_for_left_/right_ and
   form_norm_overlap_tensors_ return the reference's exact polar factor
   (U V^H of the site matrix's SVD; the neighbour absorbs U S U^H, as
   zgesdd gives them in core.f95:2708-2960), computed on the device as a
   Householder QR followed by the QDWH polar iteration on the small square
   factor.  A rank-deficient site has no unique polar factor; there, and
   after nc_set_level0_gauge(0), these entry points use the device chain's
   Householder-QR gauge (A = P Q with Q row-orthonormal): the outputs then
   differ from the reference element-wise by a unitary on the shared bond,
   and every contraction of the pair (state, energies, environments,
   overlaps) is identical.  Return 0 on success, a nonzero status
   otherwise. */

/* No counterpart in the reference.  Selects the gauge of the Level-0 moves
   above on this thread: nonzero (default) = exact polar factor, 0 = the
   faster Householder-QR gauge.  Returns a status code. */
int nc_set_level0_gauge(int exact_polar);

/* core.cpp:580-589 (norm_denorm_going_left_): site_tensor_to_normalize
   (br,bm,dr) becomes right-normalised, site_tensor_to_denormalize (bm,bl,dl)
   absorbs the factor. */
int32_t norm_denorm_going_left_(const uint32_t* bl, const uint32_t* bm, const uint32_t* br,
                                const uint32_t* dl, const uint32_t* dr,
                                const nc_complex* site_tensor_to_denormalize,
                                const nc_complex* site_tensor_to_normalize,
                                nc_complex* denormalized_site_tensor,
                                nc_complex* normalized_site_tensor);
/* core.cpp:609-618 (norm_denorm_going_right_): site_tensor_to_normalize
   (bm,bl,dl) becomes left-normalised, site_tensor_to_denormalize (br,bm,dr)
   absorbs the factor. */
int32_t norm_denorm_going_right_(const uint32_t* bl, const uint32_t* bm, const uint32_t* br,
                                 const uint32_t* dl, const uint32_t* dr,
                                 const nc_complex* site_tensor_to_normalize,
                                 const nc_complex* site_tensor_to_denormalize,
                                 nc_complex* normalized_site_tensor,
                                 nc_complex* denormalized_site_tensor);
/* core.cpp:638-643 (norm_for_left_): left-normalised factor of a site. */
int32_t norm_for_left_(const uint32_t* br, const uint32_t* bl, const uint32_t* d,
                       const nc_complex* site_tensor, nc_complex* normalized_site_tensor);
/* core.cpp:657-662 (norm_for_right_): right-normalised factor of a site. */
int32_t norm_for_right_(const uint32_t* br, const uint32_t* bl, const uint32_t* d,
                        const nc_complex* site_tensor, nc_complex* normalized_site_tensor);
/* core.cpp:548-559 (increase_bandwidth_between_): grow the bond between a
   normalised site (bm,bl,dl) and its right neighbour (br,bm,dr) to new_bm;
   outputs (new_bm,bl,dl) carrying the weight and (br,new_bm,dr) right-
   normalised. */
int32_t increase_bandwidth_between_(const uint32_t* bl, const uint32_t* bm, const uint32_t* br,
                                    const uint32_t* dl, const uint32_t* dr, const uint32_t* new_bm,
                                    const nc_complex* site_tensor_to_normalize,
                                    const nc_complex* site_tensor_to_denormalize,
                                    nc_complex* normalized_site_tensor,
                                    nc_complex* denormalized_site_tensor);
/* core.cpp:735-740 (rand_norm_state_site_tensor_): right-normalised random
   site (seeded device generator). */
void rand_norm_state_site_tensor_(const uint32_t* br, const uint32_t* bl, const uint32_t* d,
                                  nc_complex* state_site_tensor);
/* core.cpp:752-757 (rand_unnorm_state_site_tensor_): random site of unit norm. */
void rand_unnorm_state_site_tensor_(const uint32_t* br, const uint32_t* bl, const uint32_t* d,
                                    nc_complex* state_site_tensor);
/* core.cpp:463-475 (form_norm_overlap_tensors_): the projector sites of one
   bond (left-normalised and centre overlap sites of site 1, site 2 with the
   factor absorbed, right-normalised overlap site of site 2). */
void form_norm_overlap_tensors_(const uint32_t* bl, const uint32_t* bm, const uint32_t* br,
                                const uint32_t* dl, const uint32_t* dr,
                                const nc_complex* unnormalized_state_tensor_1,
                                const nc_complex* right_norm_state_tensor_2,
                                nc_complex* left_norm_overlap_tensor_1,
                                nc_complex* unnormalized_overlap_tensor_1,
                                nc_complex* unnormalized_state_tensor_2,
                                nc_complex* right_norm_overlap_tensor_2);

/* ---- Level 1: device-resident chain (chain.hpp:115-235) ---------------- */

/* ChainOptions (chain_options.hpp:11-48); nc_chain_options_init fills the
   reference defaults of chain_options.cpp:21-30. */
typedef struct {
    uint32_t maximum_number_of_iterations;
    double sanity_check_threshold;
    double site_convergence_threshold;
    double sweep_convergence_threshold;
    double chain_convergence_threshold;
    uint32_t initial_bandwidth_dimension;
    uint32_t bandwidth_increment;     /* new bandwidth = old + increment */
    char optimizer_mode[4];           /* "<v", ">v" or ">m" */
    uint32_t krylov_dimension;        /* Lanczos basis size (default 24) */
    uint64_t seed;                    /* random initial states */
    uint32_t strict;                  /* nonzero: a failed site solve is an error */
    uint32_t time_phases;             /* nonzero: synchronise and time each phase (diagnostics) */
    uint32_t precision;               /* 0: plain FP64 form (default); 1: precision form: sweeps with
                                         3xTF32 tensor-core contractions (FP64 Krylov, eigenproblem
                                         and energies), and sweep_until_converged closes with FP64
                                         refinement sweeps to the options' thresholds */
    uint32_t maximum_sweeps;          /* sweepUntilConverged: 0 (default) sweeps until the energy
                                         settles, without bound, as base_chain.cpp:112-123 does;
                                         k > 0: a call that has not settled after k sweeps fails
                                         with NC_ERR_NUMERIC ("sweeps did not converge") */
} nc_chain_options;

/* One MPO site (OperatorSite, tensors.hpp:1641-1854): indices (2,nnz)
   1-based (from,to); matrices (d,d,nnz) column-major, host memory. */
typedef struct {
    uint32_t physical_dimension, left_dimension, right_dimension, number_of_matrices;
    const uint32_t* indices;
    const nc_complex* matrices;
} nc_operator_site;

typedef struct {
    uint32_t number_of_sites, current_site, bandwidth_dimension, maximum_bandwidth_dimension;
    uint32_t number_of_projectors;
    uint64_t sweeps, site_solves, matvecs, moves, failures;
    int32_t last_failure;             /* optimizer failure kind, 0 = none */
    double energy;
    /* seconds spent per phase when time_phases is set: site solves, gauge
       moves, environment updates, projector matrices */
    double seconds_solve, seconds_gauge, seconds_environment, seconds_projector;
    uint64_t mixed_sweeps;            /* sweeps run in the precision form */
    uint32_t precision;               /* current precision (0 FP64, 1 mixed) */
} nc_chain_info;

typedef struct nc_chain nc_chain;

void nc_chain_options_init(nc_chain_options* options);
/* Chain(Operator, ChainOptions): copies the operator to the GPU and resets
   to a random state (chain.cpp:37-48).  NULL on error (see nc_last_error). */
nc_chain* nc_chain_create(uint32_t number_of_sites, const nc_operator_site* sites,
                          const nc_chain_options* options);
void nc_chain_free(nc_chain* chain);
/* chain.cpp:175-237 */
int nc_chain_reset(nc_chain* chain);
/* Reset from an explicit state: bond dimensions (N+1 entries, both ends 1)
   and host site tensors (br,bl,d), site 0 the centre, the rest right-
   normalised. */
int nc_chain_set_state(nc_chain* chain, const uint32_t* bond_dimensions,
                       const nc_complex* const* sites);
int nc_chain_optimize_site(nc_chain* chain);                 /* base_chain.cpp:81-110 */
int nc_chain_perform_optimization_sweep(nc_chain* chain);    /* chain.cpp:147-163 */
int nc_chain_sweep_until_converged(nc_chain* chain);         /* base_chain.cpp:112-123 */
int nc_chain_optimize_chain(nc_chain* chain);                /* base_chain.cpp:64-79 */
/* No counterpart in the reference: `n` levels at the chain's current bond
   dimension (sweepUntilConverged per level, then the level becomes a
   projector and the chain resets, as solveForMultipleLevels does around
   optimizeChain, chain.cpp:301-310, but without bond growth).  energies
   receives n values. */
int nc_chain_solve_levels_at_bandwidth(nc_chain* chain, uint32_t n, double* energies);
/* No counterpart in the reference: estimated device bytes of a chain of this
   operator at options->initial_bandwidth_dimension for `levels` levels
   (buffers, solver scratch, gauge plans, 25% margin); host-only. */
int nc_chain_footprint_bytes(uint32_t number_of_sites, const nc_operator_site* sites,
                             const nc_chain_options* options, uint32_t levels, uint64_t* bytes);
/* No counterpart in the reference: switch the precision of the following
   sweeps (0 FP64, 1 precision form).  Going back to FP64 rebuilds every
   environment in FP64 and resets the energy to the FP64 expectation value
   of the current state. */
int nc_chain_set_precision(nc_chain* chain, uint32_t precision);
int nc_chain_increase_bandwidth_dimension(nc_chain* chain, uint32_t new_dimension); /* chain.cpp:75-122 */
int nc_chain_construct_and_add_projector_from_state(nc_chain* chain);  /* chain.cpp:63-73 */
/* Checkpoint / resume: the chain's state (centre moved to site 0) in the
   StateBuffer layout of nutcracker.proto (first site MIDDLE, the rest RIGHT).
   nc_chain_serialize_state returns the byte count and writes the bytes when
   capacity suffices (out may be NULL to query); 0 on error.
   nc_chain_deserialize_state resets the chain to such a state (its own sites'
   physical dimensions) and recomputes the environments and the energy. */
size_t nc_chain_serialize_state(nc_chain* chain, void* out, size_t capacity);
int nc_chain_deserialize_state(nc_chain* chain, const void* data, size_t length);
/* Signals (base_chain.hpp:54-60, chain.hpp:151): `fn` runs on the calling
   thread when the event happens, in connection order; it may call the
   nc_chain_* query functions.  value: the site solve's H_eff products
   (success), the failure kind (failure), the sweep count (sweep performed),
   else 0.  nc_chain_connect returns a connection id (> 0) or -1. */
enum {
    NC_SIGNAL_OPTIMIZE_SITE_SUCCESS = 1,
    NC_SIGNAL_OPTIMIZE_SITE_FAILURE = 2,
    NC_SIGNAL_SWEEP_PERFORMED = 3,
    NC_SIGNAL_SWEEPS_CONVERGED = 4,
    NC_SIGNAL_CHAIN_OPTIMIZED = 5,
    NC_SIGNAL_CHAIN_RESET = 6
};
typedef void (*nc_chain_signal_fn)(nc_chain* chain, int signal, int64_t value, void* user);
int64_t nc_chain_connect(nc_chain* chain, int signal, nc_chain_signal_fn fn, void* user);
int nc_chain_disconnect(nc_chain* chain, int64_t connection);
/* solveForEigenvalues (chain.cpp:292-310): `eigenvalues` receives n levels. */
int nc_chain_solve_for_eigenvalues(nc_chain* chain, uint32_t number_of_levels, double* eigenvalues);
int nc_chain_move_to(nc_chain* chain, uint32_t site);        /* chain.cpp:124-133 */
int nc_chain_get_energy(nc_chain* chain, double* energy);
int nc_chain_compute_expectation_value(nc_chain* chain, double* value);
int nc_chain_get_info(nc_chain* chain, nc_chain_info* info);
/* Copies site i to host `out` (may be NULL) and writes dims (br,bl,d). */
int nc_chain_get_site(nc_chain* chain, uint32_t i, nc_complex* out, uint32_t* dims);

/* ---- Serving loop (no counterpart in the reference) ---------------------

   Continuous batching of independent MPO solves on one GPU.  Requests wait
   in arrival order; a pool of worker threads, each with its own stream and
   device arena, starts the request at the head of the queue as soon as a
   worker is free and the request's estimated footprint
   (nc_chain_footprint_bytes) fits in the memory budget beside the requests
   already running (a request larger than the budget runs alone).  Each
   request keeps its MPS and environments on the device for all of its
   sweeps, solves `levels` levels at options->initial_bandwidth_dimension
   (nc_chain_solve_levels_at_bandwidth) and releases its memory without
   synchronising the device.  Results depend only on the request's own
   inputs, so they are the same alone and in the mix. */
#define NC_SERVER_MAX_LEVELS 8
typedef struct {
    uint32_t max_inflight;          /* worker threads = requests running at once (default 16) */
    uint64_t memory_budget_bytes;   /* 0: 80% of the device memory free at creation */
} nc_server_options;
typedef struct {
    int32_t status;                 /* 0 or the failing call's status code */
    uint32_t levels, bandwidth_dimension;
    double energies[NC_SERVER_MAX_LEVELS];
    double seconds_queued, seconds_run, seconds_total;   /* submit -> start -> done */
    uint64_t footprint_bytes, sweeps;
    char message[128];              /* error message when status != 0 */
} nc_request_result;
typedef struct {
    uint64_t submitted, completed, failed, in_flight, queued;
    double p50_seconds, p99_seconds, mean_seconds;       /* time to converged (submit -> done) */
    double solves_per_second, window_seconds;            /* completed / (first submit -> last done) */
    uint64_t peak_bytes_in_flight, memory_budget_bytes;
} nc_server_stats;
typedef struct nc_server nc_server;

void nc_server_options_init(nc_server_options* options);
/* Starts the worker threads on the current device.  NULL on error. */
nc_server* nc_server_create(const nc_server_options* options);
/* Copies the operator and options; returns the request id (> 0) or -1. */
int64_t nc_server_submit(nc_server* server, uint32_t number_of_sites, const nc_operator_site* sites,
                         const nc_chain_options* options, uint32_t levels);
/* 0 and the result when done, 1 while queued or running, else an error. */
int nc_server_poll(nc_server* server, int64_t id, nc_request_result* result);
/* Blocks until the request is done. */
int nc_server_wait(nc_server* server, int64_t id, nc_request_result* result);
/* Blocks until no request is queued or running. */
int nc_server_drain(nc_server* server);
int nc_server_get_stats(nc_server* server, nc_server_stats* stats);
/* Finishes the queued requests, stops the workers and frees the server. */
void nc_server_free(nc_server* server);

/* ---- Batched form (no counterpart in the reference) ----------------------

   Many independent chains (each its own operator, number of sites and bond
   dimension) swept in lockstep on one GPU.  Every chain runs the reference's
   single-site sweep (chain.cpp:147-163) until its sweep energy settles
   (base_chain.cpp:112-123); the per-site work is that of optimize_
   (core.f95:2131-2609) and contract_sos_left/right (core.f95:623-848).
   Each contraction stage of all chains' site solves, gauge moves and
   environment updates is one persistent launch over a work list spanning
   the chains; the tile shape of every problem comes from a table keyed by
   (stage, bond dimension, MPO bond dimension, physical dimension) that the
   autotuner below fills.  A Lanczos iteration of every chain is one CUDA
   graph replay.  The chains start from seeded random states (one seed per
   chain), every reduction runs in a fixed order within its chain, so a
   chain's energies are the same alone and in any batch.  Ground states only
   (no projectors). */
typedef struct {
    uint32_t precision;               /* 1 (default): contractions in complex FP32 (complex64 products;
                                         FP64 Krylov basis, reorthogonalisation, projected problem,
                                         gauge moves and energies), sweeps until the relative energy
                                         change is below 1e-7 (at most 50); 0: FP64 throughout */
    uint32_t refine;                  /* precision 1: then rebuild every environment in FP64 and sweep
                                         in FP64 to sweep_convergence_threshold (default 1) */
    uint32_t krylov_dimension;        /* Lanczos basis before an explicit restart, 2..24 (default 16) */
    uint32_t maximum_number_of_iterations;   /* restarts before a site solve fails (default 100) */
    double sanity_check_threshold;    /* acceptance rule of base_chain.cpp:97-103 (default 1e-12) */
    double site_convergence_threshold;   /* Ritz residual <= tol * |theta| (default 1e-12) */
    double sweep_convergence_threshold;  /* relative sweep-energy change (default 1e-12) */
    uint32_t maximum_sweeps;          /* FP64 sweeps per chain, 0 (default): no bound; a chain that
                                         reaches it stops and reports converged = 0 */
    uint64_t seed;                    /* seed of every chain when no per-chain seeds are given */
    uint32_t time_phases;             /* nonzero: synchronise after the moves and after the solves of
                                         every global step and time them (diagnostics) */
} nc_batch_options;
typedef struct {
    double energy;                    /* the last accepted site energy of the final sweep */
    uint32_t sweeps, mixed_sweeps, fp64_sweeps;
    uint32_t converged;               /* 0: stopped by maximum_sweeps */
    uint32_t bandwidth_dimension, reserved;
    uint64_t site_solves;
} nc_batch_chain_result;
typedef struct {
    uint32_t chains, reserved;
    uint64_t global_steps;            /* lockstep actions (each: moves of the chains that move, then
                                         a site solve of every chain still sweeping) */
    uint64_t lanczos_iterations;      /* Lanczos graph replays (one iteration of every chain) */
    uint64_t graph_launches;
    uint64_t kernel_launches;         /* kernels launched, graph nodes included */
    uint64_t device_bytes;            /* the batch's device allocation */
    double seconds;                   /* wall time of the last nc_batch_solve */
    double seconds_moves, seconds_solves;   /* with time_phases: gauge moves + environments, site solves */
    uint64_t continued_solves;        /* site solves carried into a following step (a step gives every
                                         solving chain at most 8 Lanczos iterations) */
    uint64_t max_iterations_per_step; /* most Lanczos iterations one global step ran */
    double seconds_replays;           /* with time_phases: device time of the Lanczos graph replays */
} nc_batch_stats;
typedef struct nc_batch nc_batch;

void nc_batch_options_init(nc_batch_options* options);
/* Copies every chain's operator to the device and allocates all of the
   batch's device memory (one allocation; nothing is allocated while it
   solves).  sites[c] points at chain c's number_of_sites[c] operator sites;
   bandwidth_dimensions[c] is its bond dimension (bond dimension x physical
   dimension <= 512); seeds may be NULL (options->seed for every chain).
   NULL on error. */
nc_batch* nc_batch_create(uint32_t number_of_chains, const uint32_t* number_of_sites,
                          const nc_operator_site* const* sites, const uint32_t* bandwidth_dimensions,
                          const uint64_t* seeds, const nc_batch_options* options);
void nc_batch_free(nc_batch* batch);
/* Tile table: `count` entries of five int32 (stage, bond dimension, MPO bond
   dimension, physical dimension, tile configuration); a problem takes the
   entry of its stage, MPO and physical dimension whose bond dimension is
   nearest its own (power-of-two buckets), else a size rule.  Stages: 0 H_eff
   first product, 1 H_eff last product, 2 left environment, 3 and 4 right
   environment, 5 gauge-factor absorption. */
int nc_batch_set_tile_table(nc_batch* batch, const int32_t* entries, uint32_t count);
/* Random initial states, then sweeps until every chain has settled. */
int nc_batch_solve(nc_batch* batch);
/* One result per chain, in creation order. */
int nc_batch_get_results(nc_batch* batch, nc_batch_chain_result* results);
int nc_batch_get_stats(nc_batch* batch, nc_batch_stats* stats);
/* Autotuner measurement: seconds per launch of one grouped launch holding
   `problems` copies of `stage`'s interior-site products at (bond dimension
   chi, MPO bond dimension D, physical dimension d), for each tile
   configuration (nc_batch_tile_configs entries). */
int nc_batch_autotune_stage(uint32_t stage, uint32_t chi, uint32_t D, uint32_t d, uint32_t problems,
                            uint32_t reps, uint32_t precision, double* seconds_per_config);
/* Number of tile configurations; rows/cols (may be NULL) receive their output
   tile shapes. */
uint32_t nc_batch_tile_configs(int32_t* rows, int32_t* cols);

/* ---- YAML operator format (yaml.cpp:169-306, README:27-187) ----------------
   The input format of the reference's `nutcracker` program: a "sites" list of
   {physical dimension, left dimension, right dimension, matrices: [{from, to,
   data}]} and a 1-based "sequence" ordering them into the chain.  Complex
   entries are a scalar (real), [re, im] or {real: re, imag: im}; the d*d data
   list is stored as written into the site's (d,d) column-major block.
   Host-only (no GPU needed). */
typedef struct nc_parsed_operator nc_parsed_operator;
/* Parses the first YAML document of `text` (`length` bytes).  `location`
   (NULL or "") selects the operator inside the document by slash-separated
   keys (--input-location).  NULL on error; nc_last_error() then holds the
   reference's message (e.g. "The 'from' index is too high. (4 > 3)"). */
nc_parsed_operator* nc_yaml_read_operator(const char* text, size_t length, const char* location);
uint32_t nc_parsed_operator_number_of_sites(const nc_parsed_operator* op);
/* The chain's sites in order, ready for nc_chain_create / nc_server_submit;
   valid until nc_parsed_operator_free. */
const nc_operator_site* nc_parsed_operator_sites(const nc_parsed_operator* op);
void nc_parsed_operator_free(nc_parsed_operator* op);
/* The protobuf operator format (OperatorBuffer of nutcracker.proto, 0-based
   sequence; protobuf.cpp:41-99, 110-131): the input of the command-line
   program's protobuf format.  NULL on error (nc_last_error()). */
nc_parsed_operator* nc_protobuf_read_operator(const void* data, size_t length);
/* Writes the operator in the YAML format (identical sites listed once, with
   the sequence); returns the text length and copies at most capacity-1 bytes
   plus a NUL into `out` (out may be NULL to query the length). */
size_t nc_yaml_write_operator(uint32_t number_of_sites, const nc_operator_site* sites, char* out, size_t capacity);

#ifdef __cplusplus
}
#endif

#endif /* NUTCRACKER_B200_H */
