// Internal (C++) interface of the CUDA path.  All pointers are device
// pointers; every routine enqueues on ctx.stream and returns without a host
// synchronisation unless it returns a host value.
#pragma once

#include "nc_common.cuh"

namespace nc {

// Runs launch(); when ctx.profile is on and the work is at least
// profile_min_flops, brackets it with CUDA events on ctx.stream and records
// (flops, kind) for nc_profile_end / nc_profile_query.
template <typename F>
void profile_launch(Context& ctx, double flops, int kind, F&& launch) {
    if (!ctx.profile || flops < ctx.profile_min_flops) {
        launch();
        return;
    }
    if (ctx.prof_used == ctx.prof_start.size()) {
        cudaEvent_t a, b;
        NC_CUDA(cudaEventCreate(&a));
        NC_CUDA(cudaEventCreate(&b));
        ctx.prof_start.push_back(a);
        ctx.prof_stop.push_back(b);
        ctx.prof_flops.push_back(0);
        ctx.prof_kind.push_back(0);
    }
    const size_t i = ctx.prof_used++;
    ctx.prof_flops[i] = flops;
    ctx.prof_kind[i] = kind;
    NC_CUDA(cudaEventRecord(ctx.prof_start[i], ctx.stream));
    launch();
    NC_CUDA(cudaEventRecord(ctx.prof_stop[i], ctx.stream));
}

enum Op { OP_N = 0, OP_T = 1, OP_C = 2 };

struct ZGemmParams {
    int opA, opB;
    int M, N, K;
    const cplx* A; long long lda, sA0, sA1;
    const cplx* B; long long ldb, sB0, sB1;
    cplx* C; long long ldc, sC0, sC1;
    int nb0, batch;   // batch index b = b0 + nb0*b1; nb0 = 0: one level (b0 = b)
    cplx alpha, beta;
    int kchunk, nsplit;  // split-K (set by zgemm(p, ctx); 0/1 = none)
    cplx* ws;            // split-K partials
};

ZGemmParams zgemm_params(int opA, int opB, int M, int N, int K, const cplx* A, long long lda,
                         const cplx* B, long long ldb, cplx* C, long long ldc);
// Plain launch on stream s (no split-K).
void zgemm(const ZGemmParams& p, cudaStream_t s);
// Launch with automatic split-K when the tile grid is small (workspace from ctx.arena).
void zgemm(const ZGemmParams& p, Context& ctx);
void scale_strided(const ZGemmParams& p, cudaStream_t s);

// One MPO site on the device: W (d,d,nnz) column-major, idx (2,nnz) 1-based.
struct MpoSite {
    int d = 0, cl = 0, cr = 0, nnz = 0;
    const uint32_t* idx = nullptr;
    const cplx* W = nullptr;
};

// ---- sparse-MPO contractions (contract.cu) ---------------------------------
size_t heff_workspace_elems(int bl, int br, const MpoSite& op);
// y = H_eff x for x, y of shape (br,bl,d).  ws: heff_workspace_elems complex.
void heff_apply(Context& ctx, int bl, int br, const MpoSite& op, const cplx* L, const cplx* R,
                const cplx* x, cplx* y, cplx* ws);
// The same product launched on stream s with caller-provided scratch only.
void heff_apply_stream(cudaStream_t s, int bl, int br, const MpoSite& op, const cplx* L, const cplx* R,
                       const cplx* x, cplx* y, cplx* ws);
// New left environment (br,br,cr) from L (bl,bl,cl) and psi (br,bl,d).
void sos_left(Context& ctx, int bl, int br, const MpoSite& op, const cplx* L, const cplx* psi,
              cplx* Lnew);
// New right environment (bl,bl,cl) from R (br,br,cr) and psi (br,bl,d).
void sos_right(Context& ctx, int bl, int br, const MpoSite& op, const cplx* R, const cplx* psi,
               cplx* Rnew);
void vs_left(Context& ctx, int blo, int bro, int bln, int brn, int d, const cplx* Lov,
             const cplx* P, const cplx* S, cplx* out);
void vs_right(Context& ctx, int blo, int bro, int bln, int brn, int d, const cplx* Rov,
              const cplx* P, const cplx* S, cplx* out);
void overlap_vector(Context& ctx, int blo, int bro, int bln, int brn, int d, const cplx* Lov,
                    const cplx* Rov, const cplx* P, cplx* out);
// out(l,s,r) = conj(S(r,l,s))
void overlap_site_from_state(Context& ctx, int br, int bl, int d, const cplx* S, cplx* out);
// sum_{i,j,k} L(j,i,k) R(i,j,k) -> *result (device)
void contract_exp_boundaries(Context& ctx, int b, int c, const cplx* L, const cplx* R,
                             cplx* result);

// <psi|H|psi> at one site -> *result (device), via one H_eff product.
void expectation_dev(Context& ctx, int bl, int br, const MpoSite& op, const cplx* L, const cplx* psi,
                     const cplx* R, cplx* result);

// ---- vector kernels (vector.cu) --------------------------------------------
// out = permute(in) for 3-index column-major tensors: out axis k = in axis perm[k].
void permute3(Context& ctx, const cplx* in, int n0, int n1, int n2, const int perm[3],
              bool conj, cplx* out);
// result[0] = sum conj(x) y (deterministic two-pass reduction).
void zdotc(Context& ctx, long long n, const cplx* x, const cplx* y, cplx* result);
// result[0] = sum |x|^2 (as .x; .y = 0)
void znrm2sq(Context& ctx, long long n, const cplx* x, cplx* result);
void zcopy(Context& ctx, long long n, const cplx* x, cplx* y);
void zfill(Context& ctx, long long n, cplx v, cplx* y);
// y = a*x + y with a read from device scalar (a_dev) times host factor s
void zaxpy_dev(Context& ctx, long long n, const cplx* a_dev, double s, const cplx* x, cplx* y);
void zscal_host(Context& ctx, long long n, cplx a, cplx* x);
// x *= 1/sqrt(nrm2sq_dev->x)
void znormalize_dev(Context& ctx, long long n, const cplx* nrm2sq_dev, cplx* x);
// Reads one device complex to the host (synchronises ctx.stream).
cplx read_scalar(Context& ctx, const cplx* dev);
void read_scalars(Context& ctx, const void* dev, size_t bytes, void* host);
// Fills x with seeded uniform (-0.5,0.5] real and imaginary parts.
void zrandom(Context& ctx, long long n, uint64_t seed, cplx* x);

// ---- projector algebra (householder.cu) -------------------------------------
constexpr int kMaxProjectors = 16;

// ProjectorMatrix (includes/nutcracker/projectors.hpp:93-203) on the device.
struct DevProjector {
    int nproj = 0, nrefl = 0;
    long long n = 0, orth_dim = 0;
    const cplx* refl = nullptr;     // (n, nproj) column-major reflectors + R
    const cplx* tau = nullptr;      // (nrefl)
    std::vector<uint32_t> swaps;    // host copy, 1-based, size nrefl
};
// x <- x Q (conj_trans=false) or x Q^H for the 1 x n row vector x.
void apply_q_row(Context& ctx, const DevProjector& P, cplx* x, bool conj_trans);
// out = unproject(project(in)) (core.f95:1866-1909); in may equal out.
void filter_outside(Context& ctx, const DevProjector& P, const cplx* in, cplx* out);
// core.f95:1266-1339; synchronises.
double overlap_with_projectors(Context& ctx, const DevProjector& P, const cplx* x);
// Reduced-space positions removed by the filter, in order.
std::vector<long long> removed_positions(const DevProjector& P);
// U (n x r) orthonormal basis of the removed space (r = n - orth_dim).
void removed_basis(Context& ctx, const DevProjector& P, cplx* U);
// unproject_from_orthogonal_space of the reduced unit vector e_j.
void unproject_unit(Context& ctx, const DevProjector& P, long long reduced_index, cplx* out);
// zgeqp3 + rank rule (core.f95:1341-1435); A (m x n) overwritten with the
// reflectors and R; returns the rank; swaps gets min(m,n) 1-based entries.
int convert_vectors_to_reflectors_dev(Context& ctx, long long m, int n, cplx* A, cplx* tau_dev,
                                      std::vector<uint32_t>& swaps);

// ---- QR and gauge moves (qr.cu) ----------------------------------------------
// Householder QR of A (m x n, ld m, m >= n, m <= 2048): R left in the upper
// triangle of A; optional explicit Q (m x n) and R (n x n, zeros below,
// conjugated if conjR).
void householder_qr(Context& ctx, int m, int n, cplx* A, cplx* Q, cplx* R, bool conjR);

// ---- tcgen05 3xTF32 complex GEMM (tc32.cu) ---------------------------------
// One operand of the real GEMM: rows x Kr floats, Kr contiguous, row stride
// ld floats, batch planes sbatch floats apart (0: shared by every batch),
// held as the TF32 pair big + small.
struct TcOperand {
    const float* big = nullptr;
    const float* small = nullptr;
    long long ld = 0, sbatch = 0;
};
// D[z] = sum_segments A_s[z] B_s[z]^T (M x Nr, FP32 accumulate), read as
// complex (columns 2n, 2n+1 = Re, Im of column n) and stored to
// C[z*sz + m*sm + n*sn] as complex128 (c_fp64) or complex64.
struct TcGemm {
    TcOperand A, B;
    int M = 0, Nr = 0, Kr = 0, batch = 1;
    void* C = nullptr;
    long long sm = 0, sn = 0, sz = 0;
    bool c_fp64 = false;
    bool three = true;   // false: big x big only (one TF32 product)
};
void tc_gemm(Context& ctx, const TcGemm& g);
// Synchronises ctx.stream; raises NC_ERR_TIMEOUT if a tc32 pipeline wait expired.
void tc_check(Context& ctx);
// Test hook: the limit of every tc32 mbarrier wait (ns) and the switch that
// leaves the first K stage of tile (0,0,0) unloaded (its wait then runs out).
void tc_test_fault(unsigned long long wait_ns, int skip_first_load);

// ---- precision form of the site products (mixed.cu) ------------------------
// Tensor-core operands of one site's H_eff (environments expanded once per
// site) and the scratch of one product, all inside one float buffer of
// mixed_heff_floats() elements.
struct MixedHeff {
    int bl = 0, br = 0;
    MpoSite op;
    long long ldL = 0, ldR = 0, ldX = 0, ldU = 0;
    float *Lb = nullptr, *Ls = nullptr;   // stage-A B operand: rows 2*bl*cl, K 2*bl
    float *Rb = nullptr, *Rs = nullptr;   // stage-C B operand: rows 2*br, K 2*br*cr
    float *Xb = nullptr, *Xs = nullptr;   // stage-A A operand: d planes of br rows
    float2* T = nullptr;                  // stage-A output (br, bl*cl, d) complex64
    float *Ub = nullptr, *Us = nullptr;   // stage-C A operand: d planes of bl rows
};
size_t mixed_heff_floats(int bl, int br, const MpoSite& op);
void mixed_heff_prepare(Context& ctx, int bl, int br, const MpoSite& op, const cplx* L, const cplx* R,
                        float* buf, MixedHeff* h);
// y = H_eff x (x, y complex128 (br,bl,d)) with 3xTF32 tensor-core contractions.
void heff_apply_mixed(Context& ctx, const MixedHeff& h, const cplx* x, cplx* y);
// <psi|H_eff|psi> with the precision-form product.
void expectation_mixed(Context& ctx, const MixedHeff& h, const cplx* psi, cplx* result);
// Environment updates (sos_left / sos_right) in the precision form.
void sos_left_mixed(Context& ctx, int bl, int br, const MpoSite& op, const cplx* L, const cplx* psi, cplx* Lnew);
void sos_right_mixed(Context& ctx, int bl, int br, const MpoSite& op, const cplx* R, const cplx* psi, cplx* Rnew);
// C (M x N) = A (M x K) B (K x N), column-major complex128, through tc_gemm;
// three = false uses one TF32 product.  Synchronises and checks tc_check.
void tc_zgemm(Context& ctx, int M, int N, int K, const cplx* A, const cplx* B, cplx* C, bool three);
// Second stream for the neighbour's absorption of the gauge factor: the GEMM
// waits on `ready` (recorded on ctx.stream after the QR), runs on `stream` and
// records `done`, which the caller waits on before it reads the absorbed site.
struct AbsorbAsync {
    cudaStream_t stream;
    cudaEvent_t ready, done;
};
// A (bm,bl,dl) -> normA left-normalised; B (br,bm,dr) absorbs the factor
// (on async->stream when async is given).
void gauge_right(Context& ctx, int bl, int bm, int br, int dl, int dr, const cplx* A, const cplx* B,
                 cplx* normA, cplx* denormB, const AbsorbAsync* async = nullptr);
// B (br,bm,dr) -> normB right-normalised; A (bm,bl,dl) absorbs the factor.
void gauge_left(Context& ctx, int bl, int bm, int br, int dl, int dr, const cplx* A, const cplx* B,
                cplx* denormA, cplx* normB, const AbsorbAsync* async = nullptr);
// The same moves with the reference's exact polar factor (polar.cu): the
// normalised site is U V^H of the site matrix's SVD and the neighbour absorbs
// U S U^H, as zgesdd gives them (core.f95:2708-2960); a rank-deficient site
// falls back to the QR gauge above.
void gauge_right_polar(Context& ctx, int bl, int bm, int br, int dl, int dr, const cplx* A, const cplx* B,
                       cplx* normA, cplx* denormB);
void gauge_left_polar(Context& ctx, int bl, int bm, int br, int dl, int dr, const cplx* A, const cplx* B,
                      cplx* denormA, cplx* normB);
// Polar decomposition A = U H of a square n x n matrix (n <= 1024) by QDWH;
// false if it did not converge to an isometry (A rank-deficient).
bool polar_qdwh(Context& ctx, int n, const cplx* A, cplx* U, cplx* H);
void rand_norm_site(Context& ctx, int br, int bl, int d, uint64_t seed, cplx* out);
void rand_unnorm_site(Context& ctx, int br, int bl, int d, uint64_t seed, cplx* out);
void increase_bandwidth(Context& ctx, int bl, int bm, int br, int dl, int dr, int new_bm, uint64_t seed,
                        const cplx* A, const cplx* B, cplx* outA, cplx* outB);

// ---- Krylov eigensolver (lanczos.cu) -----------------------------------------
// w -= sum_i h_i V_i and h = V^H w helpers (V: k columns of length n, ld n).
void multi_dotc(Context& ctx, long long n, int k, const cplx* V, const cplx* w, cplx* h);
void multi_axpy(Context& ctx, long long n, int k, const cplx* V, const cplx* h, double sign, cplx* w);

enum Which { WHICH_SR = 0, WHICH_LR = 1, WHICH_LM = 2 };
int parse_which(const char* which);

struct EigenStats {
    int matvecs = 0;
    int restarts = 0;
};

// The site eigen-solve of core.f95:1911-2609 on the device.  Returns the
// reference's info code (0, 5, 10, 11, -14).  With `mixed` (prepared for the
// same L, R) every H_eff product runs in the precision form; the Krylov
// basis, its reorthogonalisation and the projected eigenproblem stay FP64.
int optimize_site(Context& ctx, int bl, int br, const MpoSite& op, const cplx* L, const cplx* R,
                  const DevProjector& P, int which, double tol, int maxit, const cplx* guess,
                  cplx* result, double* eigenvalue, double* normal, EigenStats* stats,
                  const MixedHeff* mixed = nullptr);


}  // namespace nc
