// Device side of the batched form (batched.cu): many independent chains
// swept in lockstep, every contraction stage one persistent launch over a
// work list that spans all chains.
//
// Work lists live in fixed device buffers; their lengths are read on the
// device, so one captured CUDA graph replays a Lanczos iteration for any
// set of chains, sites and bond dimensions the host writes into them.
#pragma once

#include "nc_common.cuh"

namespace nc {
namespace batch {

// ---- grouped complex GEMM ---------------------------------------------------
// C = op(A) op(B) (+ C), column-major complex128 storage; the products run
// in FP64 (prec 0) or in complex FP32 (prec 1: operands rounded to FP32 as
// they are staged, FP32 accumulation, FP64 output).
enum GOp { G_N = 0, G_T = 1, G_C = 2 };

// Tile configurations (BM x BN output tile, 256 threads, BK = 8).  The
// autotuner picks one per (stage, chi, D, d); index into kTileM / kTileN.
constexpr int kTileConfigs = 5;
constexpr int kTileM[kTileConfigs] = {16, 32, 64, 32, 64};
constexpr int kTileN[kTileConfigs] = {16, 32, 32, 64, 64};
constexpr int kGemmThreads = 256;
constexpr int kGemmBK = 8;
// shared memory: two stages of A (BK x BM) and B (BK x BN) tiles in FP64
constexpr size_t kGemmSmem = 2 * (size_t)kGemmBK * (64 + 64) * sizeof(cplx);   // 32 KB

struct GProb {
    int M, N, K;
    int opA, opB;
    int cfg;          // tile configuration
    int prec;         // 0 FP64, 1 complex FP32
    int chain;        // solver flag index: the problem is skipped when done[chain]
    int accumulate;   // C += op(A) op(B)
    int tiles_n;      // tiles along N (tile t -> tm = t / tiles_n, tn = t % tiles_n)
    int use_jsel;     // A += jsel[chain] * a_jstride (the Lanczos vector being expanded)
    int b_kdiv;       // op(B) = B (opB == G_N): row k at (k % b_kdiv) + (k / b_kdiv) * b_kstride (0: row k)
    const cplx* A;
    long long lda, a_jstride;
    const cplx* B;
    long long ldb, b_kstride;
    cplx* C;
    long long ldc;
};

// ---- sparse-MPO mix over a chain's site ---------------------------------------
// mode 0 (H_eff and the left environment update):
//   U(r,k2,j,b) = sum_{n: to(n)=k2} sum_a W(a,b,n) T(r,j,k1(n),a)
//   T (br,bl,cl,d), U (br,cr,bl,d)
// mode 1 (right environment update):
//   Z(x,r,a,k1) = sum_{n: from(n)=k1} sum_b W(a,b,n) Y(x,b,r,k2(n))
//   Y (bl,d,br,cr), Z (bl,br,d,cl)
constexpr int kMixMaxNnz = 64;
constexpr int kMixMaxD = 4;
constexpr int kMixChunk = 1024;   // output elements per work item
struct MixProb {
    int mode;
    int chain;
    int br, bl, cl, cr, d, nnz;
    const uint32_t* idx;
    const cplx* W;
    const cplx* in;
    cplx* out;
    long long total;   // output elements
};

// ---- per-chain vector chunks (Lanczos basis, norms) -------------------------
constexpr int kVecChunk = 2048;   // elements per chunk
constexpr int kMaxKrylov = 24;    // basis vectors kept before an explicit restart
struct VChunk {
    int chain;
    int off;   // element offset inside the chain's vectors
    int len;
};

// ---- Householder QR of one chain's site matrix (one CTA) -------------------
// X(i, j) = conj(src[(i % p) * s0 + (i / p) * s2 + j * s1]), i < m, j < n;
// on return the same locations hold conj(Q(i, j)) (Q m x n with orthonormal
// columns, X = Q R) and R (n x n, conjugated when conj_r) is in rbuf.  With
// random_seed != 0 the input X is a seeded random matrix instead.
struct QrProb {
    int chain;
    int m, n;
    int p;
    long long s0, s1, s2;
    cplx* site;   // src and dst
    cplx* X;      // m x n workspace
    cplx* Q;      // m x n workspace
    cplx* tau;    // n
    cplx* rbuf;   // n x n
    int conj_r;
    unsigned long long random_seed;
};
constexpr int kQrThreads = 512;

}  // namespace batch
}  // namespace nc
