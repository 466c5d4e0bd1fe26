// Internal declarations of the device-resident chain.
#pragma once

#include <cstdint>

#include "nc_common.cuh"

namespace nc {

// OptimizerFailure kinds (includes/nutcracker/optimizer.hpp:35-143)
enum ChainFailure : int {
    NC_FAIL_NONE = 0,
    NC_FAIL_UNABLE_TO_CONVERGE = 1,
    NC_FAIL_TOO_MANY_PROJECTORS = 2,
    NC_FAIL_GUESS_IN_PROJECTOR_SPACE = 3,
    NC_FAIL_EIGENVALUE_NOT_EXPECTATION = 4,
    NC_FAIL_COMPLEX_EIGENVALUE = 5,
    NC_FAIL_VANISHING_EIGENVECTOR = 6,
    NC_FAIL_EIGENVECTOR_IN_PROJECTOR_SPACE = 7,
    NC_FAIL_REGRESSIVE_EIGENVALUE = 8,
    NC_FAIL_UNKNOWN = 9,
};

// ChainOptions (includes/nutcracker/chain_options.hpp:11-48), defaults of
// chain_options.cpp:21-30.
struct ChainOptions {
    uint32_t maximum_number_of_iterations = 10000;
    double sanity_check_threshold = 1e-12;
    double site_convergence_threshold = 1e-12;
    double sweep_convergence_threshold = 1e-12;
    double chain_convergence_threshold = 1e-12;
    uint32_t initial_bandwidth_dimension = 1;
    uint32_t bandwidth_increment = 1;   // computeNewBandwidthDimension = b + increment
    int mode = 0;                       // WHICH_SR ("<v"), WHICH_LR (">v"), WHICH_LM (">m")
    int krylov_dim = 24;
    uint64_t seed = 1;
    bool strict = false;                // raise on a site failure instead of keeping the old site
    bool time_phases = false;           // synchronise and time each phase
    int precision = 0;                  // 0: all FP64; 1: precision form (mixed sweeps + FP64 refinement)
    uint32_t maximum_sweeps = 0;        // sweep_until_converged bound per call; 0 = none (the reference's loop)
};

// Thresholds of the mixed sweeps (the FP64 refinement uses the options'):
// the 3xTF32 products carry ~1e-6 relative error, so the Lanczos residual is
// taken to 1e-5 (the Ritz value is still accurate to ~1e-10 relative), the
// eigenvalue/expectation sanity check to 1e-5, and the mixed sweeps stop at a
// 1e-7 relative energy change or after kMixedMaxSweeps sweeps.
constexpr double kMixedSiteTol = 1e-5;
constexpr double kMixedSanity = 1e-5;
constexpr double kMixedSweepTol = 1e-7;
constexpr int kMixedMaxSweeps = 50;

struct OperatorSiteDesc {
    uint32_t d, cl, cr, nnz;
    const uint32_t* idx;   // host (2,nnz), 1-based
    const cplx* W;         // host (d,d,nnz)
};

struct ChainStats {
    uint64_t sweeps = 0, site_solves = 0, matvecs = 0, moves = 0, failures = 0, mixed_sweeps = 0;
    int last_failure = 0;
    double t_solve = 0, t_gauge = 0, t_env = 0, t_proj = 0;
};

}  // namespace nc
