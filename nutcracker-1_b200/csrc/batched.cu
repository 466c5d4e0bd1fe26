// Batched form: many independent chains swept in lockstep on one GPU.
//
// Every chain runs the reference's single-site sweep (chain.cpp:147-163,
// base_chain.cpp:81-123: optimise the centre, move it right to the last
// site, then left to the first, until the sweep energy settles) on its own
// operator, sites and bond dimensions.  The chains do not wait for one
// another: at each global step every chain that is still sweeping takes its
// own next action (a gauge move plus environment update, then a site
// solve), and each stage of those actions is ONE launch over a work list
// spanning every chain:
//
//   grouped_gemm_kernel  persistent; tiles of every (chain, problem) of a
//                        stage; the tile shape of each problem comes from
//                        the autotuned table (stage, chi, D, d)
//   grouped_mix_kernel   the sparse-MPO mix of every chain's site
//   lz_*_kernel          Lanczos steps: CGS2 reorthogonalisation over
//                        per-chain vector chunks, then one thread per chain
//                        for the tridiagonal Ritz problem and the decision
//   batched_qr_kernel    one CTA per moving chain: Householder QR of the
//                        site matrix, explicit Q, R for the neighbour
//
// A Lanczos iteration (three contraction stages plus eight vector and
// decision kernels) is captured once as a CUDA graph and replayed: the work
// lists live in fixed device buffers whose lengths are read on the device.
//
// Precision: the batched workload's complex64 products (prec 1: the
// contractions in complex FP32, the Krylov basis, its reorthogonalisation,
// the projected problem, the gauge moves and the energies in FP64), followed
// by FP64 refinement sweeps (every environment rebuilt in FP64) as in the
// precision form of the single chain; prec 0 runs everything in FP64.
//
// A chain's result depends only on its own inputs: every reduction runs in
// a fixed order within the chain, and the random initial state is seeded
// per chain, so a chain gives the same energies alone and in any batch.
//
// There is no counterpart in the reference (which solves one chain per
// process); the per-site work is that of core.f95:2131-2609 (optimize_) and
// core.f95:623-848 (contract_sos_left/right), and the per-chain driver that
// of chain.cpp:147-163 and base_chain.cpp:112-123.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>


#include "batched_kernels.cuh"
#include "nc_abi_util.h"
#include "nc_common.cuh"
#include "nc_ritz.cuh"
#include "nutcracker_b200.h"

namespace nc {
namespace batch {
namespace {


// ---------------------------------------------------------------------------
// Per-chain Lanczos state (read by every stage: a finished chain is skipped)
// ---------------------------------------------------------------------------
constexpr int kKeepMax = 8;   // Ritz vectors kept by a thick restart

struct LzChain {
    cplx* V;      // (kMaxKrylov + 1) vectors of length n
    cplx* w;      // residual / scratch vector
    cplx* x;      // the site: initial guess, and the result when accepted
    cplx* Y;      // (kKeepMax + 1) vectors: the kept Ritz vectors and the residual at a restart
    long long n;
    double tol;
    int cstart, ccount;   // the chain's chunks in the chunk list
    int m_max;            // basis size before a thick restart
    int keep;             // Ritz vectors kept by a restart
    int maxit;            // restarts before the solve fails
};

struct LzState {
    int j;          // index of the vector being expanded
    int done;       // 1: converged, failed or not solving this step
    int stall;      // 1: basis full, waiting for a restart
    int adv;        // 1: the next basis vector is to be written
    int restarts, matvecs, fail, accept;
    int fin;        // 1: the solve's result has been taken (or there is no solve)
    double theta, res, beta, tnorm, xnorm, energy;
    cplx h1[kMaxKrylov + 1], h2[kMaxKrylov + 1];
    double wn2;
};

// The projected problem of one chain (nc_ritz.cuh): its kept decomposition,
// the ordered Ritz vectors S (column r at S[kMaxKrylov * r]) and values.
struct LzRitz {
    double state[2 * kMaxKrylov * kMaxKrylov];
    double S[kMaxKrylov * kMaxKrylov];
    double theta[kMaxKrylov];
};

// ---------------------------------------------------------------------------
// Grouped complex GEMM
// ---------------------------------------------------------------------------
template <typename R>
struct CR;
template <>
struct CR<float> {
    typedef float2 T;
};
template <>
struct CR<double> {
    typedef double2 T;
};

template <typename R>
__device__ __forceinline__ typename CR<R>::T to_r(cplx v);
template <>
__device__ __forceinline__ float2 to_r<float>(cplx v) {
    return make_float2((float)v.x, (float)v.y);
}
template <>
__device__ __forceinline__ double2 to_r<double>(cplx v) {
    return v;
}

template <typename R, int BM, int BN>
__device__ __forceinline__ void gemm_tile(const GProb& P, const cplx* __restrict__ A, int tm, int tn,
                                          unsigned char* smem_raw) {
    typedef typename CR<R>::T C2;
    constexpr int BK = kGemmBK, TM = BM / 16, TN = BN / 16;
    constexpr int AL = (BM * BK + kGemmThreads - 1) / kGemmThreads;
    constexpr int BL = (BN * BK + kGemmThreads - 1) / kGemmThreads;
    C2* As = reinterpret_cast<C2*>(smem_raw);   // [2][BK][BM]
    C2* Bs = As + 2 * BK * BM;                   // [2][BK][BN]
    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    const int m0 = tm * BM, n0 = tn * BN;
    const int M = P.M, N = P.N, K = P.K;
    const cplx* __restrict__ B = P.B;
    C2 ra[AL], rb[BL];
    auto a_coord = [&](int e, int& m, int& k) {
        if (P.opA == G_N) { m = e % BM; k = e / BM; }
        else { k = e % BK; m = e / BK; }
    };
    auto b_coord = [&](int e, int& k, int& n) {
        if (P.opB == G_N) { k = e % BK; n = e / BK; }
        else { n = e % BN; k = e / BN; }
    };
    auto load = [&](int k0) {
#pragma unroll
        for (int q = 0; q < AL; ++q) {
            const int e = tid + q * kGemmThreads;
            cplx x = cmake(0, 0);
            if (e < BM * BK) {
                int m, k;
                a_coord(e, m, k);
                const int gm = m0 + m, gk = k0 + k;
                if (gm < M && gk < K) {
                    x = (P.opA == G_N) ? A[gm + (long long)gk * P.lda] : A[gk + (long long)gm * P.lda];
                    if (P.opA == G_C) x.y = -x.y;
                }
            }
            ra[q] = to_r<R>(x);
        }
#pragma unroll
        for (int q = 0; q < BL; ++q) {
            const int e = tid + q * kGemmThreads;
            cplx x = cmake(0, 0);
            if (e < BN * BK) {
                int k, n;
                b_coord(e, k, n);
                const int gk = k0 + k, gn = n0 + n;
                if (gk < K && gn < N) {
                    if (P.opB == G_N) {
                        const long long row =
                            P.b_kdiv ? (long long)(gk % P.b_kdiv) + (long long)(gk / P.b_kdiv) * P.b_kstride : gk;
                        x = B[row + (long long)gn * P.ldb];
                    } else {
                        x = B[gn + (long long)gk * P.ldb];
                        if (P.opB == G_C) x.y = -x.y;
                    }
                }
            }
            rb[q] = to_r<R>(x);
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int q = 0; q < AL; ++q) {
            const int e = tid + q * kGemmThreads;
            if (e < BM * BK) {
                int m, k;
                a_coord(e, m, k);
                As[(buf * BK + k) * BM + m] = ra[q];
            }
        }
#pragma unroll
        for (int q = 0; q < BL; ++q) {
            const int e = tid + q * kGemmThreads;
            if (e < BN * BK) {
                int k, n;
                b_coord(e, k, n);
                Bs[(buf * BK + k) * BN + n] = rb[q];
            }
        }
    };
    R accr[TM][TN], acci[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) accr[i][j] = acci[i][j] = 0;
    const int ktiles = (K + BK - 1) / BK;
    load(0);
    store(0);
    __syncthreads();
    for (int kt = 0; kt < ktiles; ++kt) {
        const int buf = kt & 1;
        const bool more = kt + 1 < ktiles;
        if (more) load((kt + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            C2 a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = As[(buf * BK + kk) * BM + tx + 16 * i];
#pragma unroll
            for (int j = 0; j < TN; ++j) b[j] = Bs[(buf * BK + kk) * BN + ty + 16 * j];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) {
                    accr[i][j] = fma(a[i].x, b[j].x, fma(-a[i].y, b[j].y, accr[i][j]));
                    acci[i][j] = fma(a[i].x, b[j].y, fma(a[i].y, b[j].x, acci[i][j]));
                }
        }
        if (more) store(buf ^ 1);
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int m = m0 + tx + 16 * i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int n = n0 + ty + 16 * j;
            if (n >= N) continue;
            cplx* dst = P.C + m + (long long)n * P.ldc;
            cplx v = cmake((double)accr[i][j], (double)acci[i][j]);
            if (P.accumulate) v = cadd(v, *dst);
            *dst = v;
        }
    }
}

template <typename R>
__device__ __forceinline__ void gemm_dispatch(const GProb& P, const cplx* A, int tm, int tn, unsigned char* smem) {
    switch (P.cfg) {
        case 0: gemm_tile<R, 16, 16>(P, A, tm, tn, smem); break;
        case 1: gemm_tile<R, 32, 32>(P, A, tm, tn, smem); break;
        case 2: gemm_tile<R, 64, 32>(P, A, tm, tn, smem); break;
        case 3: gemm_tile<R, 32, 64>(P, A, tm, tn, smem); break;
        default: gemm_tile<R, 64, 64>(P, A, tm, tn, smem); break;
    }
}

// Persistent: block b takes tiles b, b + grid, ...; tile t belongs to
// problem tile_prob[t] and is its (t - prefix[problem])-th tile.
// (The stage bodies below take the block's index vb among nvb blocks; each
// kernel runs one of them over its whole grid.)
__device__ __forceinline__ void gemm_phase(const GProb* __restrict__ probs, const int* __restrict__ prefix,
                                           const int* __restrict__ tile_prob, const int* __restrict__ ntiles,
                                           const LzState* __restrict__ st, unsigned char* smem, int vb, int nvb) {
    __shared__ GProb P;
    __shared__ int s_local;
    const int total = *ntiles;
    for (int t = vb; t < total; t += nvb) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const int p = tile_prob[t];
            P = probs[p];
            s_local = t - prefix[p];
        }
        __syncthreads();
        if (st && (st[P.chain].done || st[P.chain].stall)) continue;
        const cplx* A = P.A;
        if (P.use_jsel) A += (long long)st[P.chain].j * P.a_jstride;
        const int tm = s_local / P.tiles_n, tn = s_local % P.tiles_n;
        if (P.prec) gemm_dispatch<float>(P, A, tm, tn, smem);
        else gemm_dispatch<double>(P, A, tm, tn, smem);
    }
}

__global__ void __launch_bounds__(kGemmThreads, 2) grouped_gemm_kernel(const GProb* __restrict__ probs,
                                                                    const int* __restrict__ prefix,
                                                                    const int* __restrict__ tile_prob,
                                                                    const int* __restrict__ ntiles,
                                                                    const LzState* __restrict__ st) {
    extern __shared__ __align__(16) unsigned char smem[];
    gemm_phase(probs, prefix, tile_prob, ntiles, st, smem, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// Grouped sparse-MPO mix (FP64 accumulation)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mix_phase(const MixProb* __restrict__ probs, const int2* __restrict__ items,
                                          const int* __restrict__ nitems, const LzState* __restrict__ st, int vb,
                                          int nvb) {
    __shared__ cplx Ws[kMixMaxNnz * kMixMaxD * kMixMaxD];
    __shared__ int k1s[kMixMaxNnz], k2s[kMixMaxNnz];
    __shared__ MixProb P;
    __shared__ int s_item;
    const int total = *nitems;
    for (int t = vb; t < total; t += nvb) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const int2 it = items[t];
            P = probs[it.x];
            s_item = it.y;
        }
        __syncthreads();
        if (st && (st[P.chain].done || st[P.chain].stall)) continue;
        const int d = P.d, nnz = P.nnz;
        for (int i = threadIdx.x; i < nnz * d * d; i += blockDim.x) Ws[i] = P.W[i];
        for (int i = threadIdx.x; i < nnz; i += blockDim.x) {
            k1s[i] = (int)P.idx[2 * i] - 1;
            k2s[i] = (int)P.idx[2 * i + 1] - 1;
        }
        __syncthreads();
        const long long e0 = (long long)s_item * kMixChunk;
        const long long e1 = min(e0 + kMixChunk, P.total);
        const int br = P.br, bl = P.bl, cl = P.cl, cr = P.cr;
        if (P.mode == 0) {
            const long long sT_j = br, sT_k = (long long)br * bl, sT_a = (long long)br * bl * cl;
            for (long long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                long long q = e;
                const int r = (int)(q % br); q /= br;
                const int k2 = (int)(q % cr); q /= cr;
                const int j = (int)(q % bl); q /= bl;
                const int b = (int)q;
                double ar = 0, ai = 0;
                const cplx* Tb = P.in + r + j * sT_j;
                for (int n = 0; n < nnz; ++n) {
                    if (k2s[n] != k2) continue;
                    const cplx* Tk = Tb + k1s[n] * sT_k;
                    for (int a = 0; a < d; ++a) {
                        const cplx w = Ws[(n * d + b) * d + a], tv = Tk[a * sT_a];
                        ar = fma(w.x, tv.x, fma(-w.y, tv.y, ar));
                        ai = fma(w.x, tv.y, fma(w.y, tv.x, ai));
                    }
                }
                P.out[e] = cmake(ar, ai);
            }
        } else {
            const long long sY_b = bl, sY_r = (long long)bl * d, sY_k = (long long)bl * d * br;
            for (long long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
                long long q = e;
                const int x = (int)(q % bl); q /= bl;
                const int r = (int)(q % br); q /= br;
                const int a = (int)(q % d); q /= d;
                const int k1 = (int)q;
                double ar = 0, ai = 0;
                const cplx* Yb = P.in + x + r * sY_r;
                for (int n = 0; n < nnz; ++n) {
                    if (k1s[n] != k1) continue;
                    const cplx* Yk = Yb + k2s[n] * sY_k;
                    for (int b = 0; b < d; ++b) {
                        const cplx w = Ws[(n * d + b) * d + a], yv = Yk[b * sY_b];
                        ar = fma(w.x, yv.x, fma(-w.y, yv.y, ar));
                        ai = fma(w.x, yv.y, fma(w.y, yv.x, ai));
                    }
                }
                P.out[e] = cmake(ar, ai);
            }
        }
    }
}

__global__ void __launch_bounds__(256) grouped_mix_kernel(const MixProb* __restrict__ probs,
                                                          const int2* __restrict__ items,
                                                          const int* __restrict__ nitems,
                                                          const LzState* __restrict__ st) {
    mix_phase(probs, items, nitems, st, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// Lanczos over every chain (FP64 basis, CGS2 reorthogonalisation)
// ---------------------------------------------------------------------------
constexpr int kLzT = 256;
constexpr int kLzW = kLzT / 32;
constexpr int kPartStride = kMaxKrylov + 1;   // complex partials per chunk

// Sums acc[0..nk) over the block and writes them to out[0..nk).
template <int NK>
__device__ __forceinline__ void block_sum_c(double (&ar)[NK], double (&ai)[NK], int nk, cplx* red /*[kLzW][NK]*/,
                                            cplx* out) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NK; ++k) {
        if (k < nk) {
            double x = ar[k], y = ai[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                x += __shfl_down_sync(0xffffffffu, x, o);
                y += __shfl_down_sync(0xffffffffu, y, o);
            }
            if (lane == 0) red[wid * NK + k] = cmake(x, y);
        }
    }
    __syncthreads();
    if (threadIdx.x < nk) {
        double x = 0, y = 0;
        for (int w = 0; w < kLzW; ++w) {
            const cplx v = red[w * NK + threadIdx.x];
            x += v.x;
            y += v.y;
        }
        out[threadIdx.x] = cmake(x, y);
    }
    __syncthreads();
}

// PASS 0: part = V^H w;  PASS 1: w -= V h1, part = V^H w;  PASS 2: w -= V h2, part[0] = |w|^2.
// Each thread keeps its (at most kVecChunk / kLzT) elements of w in
// registers; the dot products run four basis vectors at a time, so that every
// thread has many independent loads in flight, each a fixed-order sum over
// the chunk.
constexpr int kEpt = kVecChunk / kLzT;
template <int PASS>
__device__ __forceinline__ void cgs_phase(const VChunk* __restrict__ chunks, const int* __restrict__ nchunks,
                                          const LzChain* __restrict__ ch, LzState* __restrict__ st,
                                          cplx* __restrict__ part, int vb, int nvb) {
    __shared__ cplx red[kLzW * (kMaxKrylov + 1)];
    __shared__ cplx hs[kMaxKrylov + 1];
    const int total = *nchunks;
    for (int t = vb; t < total; t += nvb) {
        const VChunk c = chunks[t];
        const LzState& S = st[c.chain];
        if (S.done || S.stall) continue;
        const LzChain C = ch[c.chain];
        const int nk = S.j + 1;
        __syncthreads();
        if (PASS > 0 && threadIdx.x < nk) hs[threadIdx.x] = (PASS == 1) ? S.h1[threadIdx.x] : S.h2[threadIdx.x];
        __syncthreads();
        const int end = c.off + c.len;
        cplx wv[kEpt];
#pragma unroll
        for (int e = 0; e < kEpt; ++e) {
            const int i = c.off + threadIdx.x + e * kLzT;
            wv[e] = (i < end) ? C.w[i] : cmake(0, 0);
        }
        if (PASS > 0) {
            double nr[1] = {0}, ni[1] = {0};
            for (int k = 0; k < nk; ++k) {
                const cplx h = hs[k];
                const cplx* Vk = C.V + (long long)k * C.n;
#pragma unroll
                for (int e = 0; e < kEpt; ++e) {
                    const int i = c.off + threadIdx.x + e * kLzT;
                    if (i < end) {
                        const cplx v = Vk[i];
                        wv[e].x -= v.x * h.x - v.y * h.y;
                        wv[e].y -= v.x * h.y + v.y * h.x;
                    }
                }
            }
#pragma unroll
            for (int e = 0; e < kEpt; ++e) {
                const int i = c.off + threadIdx.x + e * kLzT;
                if (i < end) {
                    C.w[i] = wv[e];
                    nr[0] = fma(wv[e].x, wv[e].x, fma(wv[e].y, wv[e].y, nr[0]));
                }
            }
            if (PASS == 2) block_sum_c<1>(nr, ni, 1, red, part + (long long)t * kPartStride);
        }
        if constexpr (PASS < 2) for (int k0 = 0; k0 < nk; k0 += 4) {
            const int kc = min(4, nk - k0);
            double ar[4] = {0, 0, 0, 0}, ai[4] = {0, 0, 0, 0};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (q < kc) {
                    const cplx* Vk = C.V + (long long)(k0 + q) * C.n;
#pragma unroll
                    for (int e = 0; e < kEpt; ++e) {
                        const int i = c.off + threadIdx.x + e * kLzT;
                        if (i < end) {
                            const cplx v = Vk[i];   // conj(v) * w
                            ar[q] = fma(v.x, wv[e].x, fma(v.y, wv[e].y, ar[q]));
                            ai[q] = fma(v.x, wv[e].y, fma(-v.y, wv[e].x, ai[q]));
                        }
                    }
                }
            }
            block_sum_c<4>(ar, ai, kc, red, part + (long long)t * kPartStride + k0);
        }
    }
}

template <int PASS>
__global__ void __launch_bounds__(kLzT) lz_cgs_kernel(const VChunk* __restrict__ chunks, const int* __restrict__ nchunks,
                                                      const LzChain* __restrict__ ch, LzState* __restrict__ st,
                                                      cplx* __restrict__ part) {
    cgs_phase<PASS>(chunks, nchunks, ch, st, part, blockIdx.x, gridDim.x);
}

// Per chain (one warp): h = sum of the chain's chunk partials in chunk order.
template <int PASS>
__device__ __forceinline__ void reduce_chain(int c, int lane, const LzChain* __restrict__ ch, LzState* __restrict__ st,
                                             const cplx* __restrict__ part) {
    LzState& S = st[c];
    if (S.done || S.stall) return;
    const int nk = (PASS < 2) ? S.j + 1 : 1;
    if (lane >= nk) return;
    const LzChain C = ch[c];
    double x = 0, y = 0;
    for (int q = 0; q < C.ccount; ++q) {
        const cplx v = part[(long long)(C.cstart + q) * kPartStride + lane];
        x += v.x;
        y += v.y;
    }
    if (PASS == 0) S.h1[lane] = cmake(x, y);
    else if (PASS == 1) S.h2[lane] = cmake(x, y);
    else S.wn2 = x;
}

template <int PASS>
__global__ void lz_reduce_kernel(int nchains, const LzChain* __restrict__ ch, LzState* __restrict__ st,
                                 const cplx* __restrict__ part) {
    const int c = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
    if (c < nchains) reduce_chain<PASS>(c, lane, ch, st, part);
}

// One warp per chain: column j of the projected matrix from the
// reorthogonalisation coefficients, the Ritz pairs (warm-started Jacobi,
// nc_ritz.cuh), and the decision: converged (ARPACK's rule, Ritz estimate
// <= tol * max(|theta|, eps^(2/3)), or the Krylov space exhausted or
// invariant), basis full (thick restart), or advance.
__device__ __forceinline__ void ritz_chain(int c, RitzSmem<kMaxKrylov>& w, const LzChain* __restrict__ ch,
                                           LzState* __restrict__ st, LzRitz* __restrict__ rz) {
    LzState& S = st[c];
    if (S.done || S.stall) return;
    const LzChain C = ch[c];
    const int j = S.j;
    LzRitz& R = rz[c];
    const RitzResult r =
        ritz_update_warp<kMaxKrylov, false>(w, j + 1, R.state, S.h1, S.h2, fmax(S.wn2, 0.0), RITZ_SR, R.S,
                                            kMaxKrylov, R.theta);
    if ((threadIdx.x & 31) != 0) return;
    S.matvecs++;
    S.theta = r.theta;
    S.res = r.res;
    S.beta = r.beta;
    S.tnorm = r.tnorm;
    const double eps = 2.220446049250313e-16;
    const double eps23 = 3.666852862501036e-11;   // eps^(2/3), ARPACK's floor
    const double anorm = fmax(fabs(r.theta), eps23);
    if (r.res <= C.tol * anorm || (long long)(j + 1) >= C.n || r.beta <= 1e3 * eps * fmax(r.tnorm, 1e-300)) {
        S.done = 1;
    } else if (j + 1 >= C.m_max) {
        S.stall = 1;
    } else {
        S.adv = 1;
    }
}

__global__ void __launch_bounds__(32) lz_ritz_kernel(int nchains, const LzChain* __restrict__ ch,
                                                     LzState* __restrict__ st, LzRitz* __restrict__ rz,
                                                     int* __restrict__ active) {
    __shared__ RitzSmem<kMaxKrylov> w;
    const int c = blockIdx.x;
    if (c == 0 && threadIdx.x == 0) *active = 0;
    if (c < nchains) ritz_chain(c, w, ch, st, rz);
}

// V_{j+1} = w / beta_j for the chains that advance.
__device__ __forceinline__ void next_phase(const VChunk* __restrict__ chunks, const int* __restrict__ nchunks,
                                                       const LzChain* __restrict__ ch, const LzState* __restrict__ st, int vb, int nvb) {
    const int total = *nchunks;
    for (int t = vb; t < total; t += nvb) {
        const VChunk c = chunks[t];
        const LzState& S = st[c.chain];
        if (!S.adv) continue;
        const LzChain C = ch[c.chain];
        const double f = 1.0 / S.beta;
        cplx* vn = C.V + (long long)(S.j + 1) * C.n;
        for (int i = c.off + threadIdx.x; i < c.off + c.len; i += kLzT) vn[i] = cscale(C.w[i], f);
    }
}

__global__ void __launch_bounds__(kLzT) lz_next_kernel(const VChunk* __restrict__ chunks, const int* __restrict__ nchunks,
                                                       const LzChain* __restrict__ ch, const LzState* __restrict__ st) {
    next_phase(chunks, nchunks, ch, st, blockIdx.x, gridDim.x);
}

__global__ void lz_inc_kernel(int nchains, LzState* __restrict__ st, int* __restrict__ active) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchains) return;
    LzState& S = st[c];
    if (S.adv) {
        S.j++;
        S.adv = 0;
    }
    if (!S.done && !S.stall) atomicAdd(active, 1);
}

// ---- solve set-up, restarts and the result ------------------------------------

// Per chain: solving[c] = 1 starts a solve, 2 continues the one in progress,
// 0 sits this step out.
__global__ void lz_init_kernel(int nchains, const int* __restrict__ solving, LzState* __restrict__ st) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchains) return;
    LzState& S = st[c];
    if (solving[c] == 2) return;
    const bool start = solving[c] == 1;
    S.j = 0;
    S.done = start ? 0 : 1;
    S.stall = 0;
    S.adv = 0;
    S.restarts = 0;
    S.matvecs = 0;
    S.fail = 0;
    S.accept = 0;
    S.fin = start ? 0 : 1;
}

// After a step's iterations: the chains whose solve ended (converged or
// failed) and whose result was taken this step are reported to the host,
// with their energies.
__global__ void lz_finish_kernel(int nchains, const int* __restrict__ solving, LzState* __restrict__ st,
                                 int* __restrict__ finished, double* __restrict__ energy) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchains) return;
    LzState& S = st[c];
    const int f = (solving[c] && S.done && !S.fin) ? 1 : 0;
    if (f) S.fin = 1;
    finished[c] = f;
    energy[c] = S.energy;
}

// MODE 0: V_0 = x (the guess), part = |x|^2   (chains with !done)
// MODE 2: w = V S(:,0) (the wanted Ritz vector), part = |w|^2   (chains with done && !fail, solving)
template <int MODE>
__global__ void __launch_bounds__(kLzT) lz_form_kernel(const VChunk* __restrict__ chunks, const int* __restrict__ nchunks,
                                                       const LzChain* __restrict__ ch, const LzState* __restrict__ st,
                                                       const LzRitz* __restrict__ rz, const int* __restrict__ solving,
                                                       cplx* __restrict__ part) {
    __shared__ cplx red[kLzW * (kMaxKrylov + 1)];
    __shared__ double ss[kMaxKrylov];
    const int total = *nchunks;
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const VChunk c = chunks[t];
        const LzState& S = st[c.chain];
        const bool on = (MODE == 0) ? (solving[c.chain] == 1 && !S.done)
                                    : (solving[c.chain] && S.done && !S.fin && !S.fail);
        if (!on) continue;
        const LzChain C = ch[c.chain];
        const int nk = S.j + 1;
        __syncthreads();
        if (MODE > 0 && threadIdx.x < nk) ss[threadIdx.x] = rz[c.chain].S[threadIdx.x];
        __syncthreads();
        double ar[1] = {0}, ai[1] = {0};
        for (int i = c.off + threadIdx.x; i < c.off + c.len; i += kLzT) {
            cplx v;
            if (MODE == 0) {
                v = C.x[i];
                C.V[i] = v;
            } else {
                double vr = 0, vi = 0;
                for (int k = 0; k < nk; ++k) {
                    const cplx b = C.V[(long long)k * C.n + i];
                    vr = fma(ss[k], b.x, vr);
                    vi = fma(ss[k], b.y, vi);
                }
                v = cmake(vr, vi);
                C.w[i] = v;
            }
            ar[0] = fma(v.x, v.x, fma(v.y, v.y, ar[0]));
        }
        block_sum_c<1>(ar, ai, 1, red, part + (long long)t * kPartStride);
    }
}

// Per chain, after lz_form_kernel<MODE>: the norm of the formed vector.
//   MODE 0: xnorm (a vanishing guess fails the solve)
//   MODE 2: acceptance rule (base_chain.cpp:97-103) and the energy
template <int MODE>
__global__ void lz_norm_kernel(int nchains, const LzChain* __restrict__ ch, LzState* __restrict__ st,
                               const int* __restrict__ solving, const cplx* __restrict__ part, double sanity) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchains) return;
    LzState& S = st[c];
    const bool on = (MODE == 0) ? (solving[c] == 1 && !S.done) : (solving[c] && S.done && !S.fin && !S.fail);
    if (!on) return;
    const LzChain C = ch[c];
    double x = 0;
    for (int q = 0; q < C.ccount; ++q) x += part[(long long)(C.cstart + q) * kPartStride].x;
    const double nrm = sqrt(x);
    S.xnorm = nrm;
    if (MODE == 0) {
        if (!(nrm > 1e-280)) {
            S.done = 1;
            S.fail = 1;
        }
    } else {
        const double e0 = S.energy, ev = S.theta;
        const double aa = fabs(e0), bb = fabs(ev);
        const bool outside = (aa + bb) / 2 > sanity && fabs(aa - bb) / (aa + bb + sanity) > sanity;
        S.accept = ((e0 >= 0 && ev >= 0) || (e0 <= 0 && ev <= 0) || outside || isnan(e0)) && nrm > 1e-280;
        if (S.accept) S.energy = ev;
    }
}

// MODE 0: V_0 /= |V_0|;  MODE 2: x = w / |w| for an accepted result.
template <int MODE>
__global__ void __launch_bounds__(kLzT) lz_scale_kernel(const VChunk* __restrict__ chunks, const int* __restrict__ nchunks,
                                                        const LzChain* __restrict__ ch, const LzState* __restrict__ st,
                                                        const int* __restrict__ solving) {
    const int total = *nchunks;
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const VChunk c = chunks[t];
        const LzState& S = st[c.chain];
        const LzChain C = ch[c.chain];
        if (MODE == 0) {
            if (solving[c.chain] != 1 || S.done) continue;
            const double f = 1.0 / S.xnorm;
            for (int i = c.off + threadIdx.x; i < c.off + c.len; i += kLzT) C.V[i] = cscale(C.V[i], f);
        } else {
            if (!(solving[c.chain] && S.done && !S.fin && !S.fail && S.accept)) continue;
            const double f = 1.0 / S.xnorm;
            for (int i = c.off + threadIdx.x; i < c.off + c.len; i += kLzT) C.x[i] = cscale(C.w[i], f);
        }
    }
}

// ---- thick restart (Wu & Simon 2000), for the chains whose basis is full ---
// Y_i = V S(:,i) for the `keep` wanted Ritz vectors, Y_keep = w / beta (the
// residual direction, orthogonal to them).
__device__ __forceinline__ void restart_form_phase(const VChunk* __restrict__ chunks,
                                                               const int* __restrict__ nchunks,
                                                               const LzChain* __restrict__ ch,
                                                               const LzState* __restrict__ st,
                                                               const LzRitz* __restrict__ rz, int vb, int nvb) {
    __shared__ double ss[kKeepMax * kMaxKrylov];
    const int total = *nchunks;
    for (int t = vb; t < total; t += nvb) {
        const VChunk c = chunks[t];
        const LzState& S = st[c.chain];
        if (S.done || !S.stall) continue;
        const LzChain C = ch[c.chain];
        const int m = S.j + 1;
        __syncthreads();
        for (int e = threadIdx.x; e < C.keep * kMaxKrylov; e += kLzT) ss[e] = rz[c.chain].S[e];
        __syncthreads();
        const double fb = 1.0 / S.beta;
        for (int i = c.off + threadIdx.x; i < c.off + c.len; i += kLzT) {
            for (int q = 0; q < C.keep; ++q) {
                double vr = 0, vi = 0;
                for (int k = 0; k < m; ++k) {
                    const cplx b = C.V[(long long)k * C.n + i];
                    const double f = ss[q * kMaxKrylov + k];
                    vr = fma(f, b.x, vr);
                    vi = fma(f, b.y, vi);
                }
                C.Y[(long long)q * C.n + i] = cmake(vr, vi);
            }
            C.Y[(long long)C.keep * C.n + i] = cscale(C.w[i], fb);
        }
    }
}

__global__ void __launch_bounds__(kLzT) lz_restart_form_kernel(const VChunk* __restrict__ chunks,
                                                               const int* __restrict__ nchunks,
                                                               const LzChain* __restrict__ ch,
                                                               const LzState* __restrict__ st,
                                                               const LzRitz* __restrict__ rz) {
    restart_form_phase(chunks, nchunks, ch, st, rz, blockIdx.x, gridDim.x);
}

// V_0..V_keep = Y_0..Y_keep.
__device__ __forceinline__ void restart_copy_phase(const VChunk* __restrict__ chunks,
                                                               const int* __restrict__ nchunks,
                                                               const LzChain* __restrict__ ch,
                                                               const LzState* __restrict__ st, int vb, int nvb) {
    const int total = *nchunks;
    for (int t = vb; t < total; t += nvb) {
        const VChunk c = chunks[t];
        const LzState& S = st[c.chain];
        if (S.done || !S.stall) continue;
        const LzChain C = ch[c.chain];
        for (int q = 0; q <= C.keep; ++q)
            for (int i = c.off + threadIdx.x; i < c.off + c.len; i += kLzT)
                C.V[(long long)q * C.n + i] = C.Y[(long long)q * C.n + i];
    }
}

__global__ void __launch_bounds__(kLzT) lz_restart_copy_kernel(const VChunk* __restrict__ chunks,
                                                               const int* __restrict__ nchunks,
                                                               const LzChain* __restrict__ ch,
                                                               const LzState* __restrict__ st) {
    restart_copy_phase(chunks, nchunks, ch, st, blockIdx.x, gridDim.x);
}

// Per chain (one block): the projected matrix becomes diag(theta_0 ..
// theta_{keep-1}) and the expansion continues from V_keep; after maxit
// restarts the solve fails (info -14 of the reference, core.f95:2565-2607).
__global__ void lz_restart_state_kernel(int nchains, const LzChain* __restrict__ ch, LzState* __restrict__ st,
                                        LzRitz* __restrict__ rz) {
    const int c = blockIdx.x;
    if (c >= nchains) return;
    LzState& S = st[c];
    if (S.done || !S.stall) return;
    const LzChain C = ch[c];
    const bool fail = S.restarts + 1 >= C.maxit;
    if (!fail) ritz_restart_state<kMaxKrylov>(C.keep, rz[c].theta, rz[c].state);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (fail) {
            S.done = 1;
            S.fail = 1;
        } else {
            S.restarts++;
            S.j = C.keep;
        }
        S.stall = 0;
    }
}

// ---- site normalisation (the new centre after a move) -----------------------
struct NormJob {
    cplx* x;
    int cstart, ccount;
};
__global__ void __launch_bounds__(kLzT) norm_partial_kernel(const VChunk* __restrict__ chunks, const int* __restrict__ nchunks,
                                                            const NormJob* __restrict__ jobs, cplx* __restrict__ part) {
    __shared__ cplx red[kLzW * (kMaxKrylov + 1)];
    const int total = *nchunks;
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const VChunk c = chunks[t];
        const cplx* x = jobs[c.chain].x;
        double ar[1] = {0}, ai[1] = {0};
        for (int i = c.off + threadIdx.x; i < c.off + c.len; i += kLzT) {
            const cplx v = x[i];
            ar[0] = fma(v.x, v.x, fma(v.y, v.y, ar[0]));
        }
        block_sum_c<1>(ar, ai, 1, red, part + (long long)t * kPartStride);
    }
}
__global__ void __launch_bounds__(kLzT) norm_scale_kernel(const VChunk* __restrict__ chunks, const int* __restrict__ nchunks,
                                                          const NormJob* __restrict__ jobs,
                                                          const cplx* __restrict__ part) {
    const int total = *nchunks;
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const VChunk c = chunks[t];
        const NormJob J = jobs[c.chain];
        double s = 0;
        for (int q = 0; q < J.ccount; ++q) s += part[(long long)(J.cstart + q) * kPartStride].x;
        const double f = (s > 0) ? 1.0 / sqrt(s) : 1.0;
        for (int i = c.off + threadIdx.x; i < c.off + c.len; i += kLzT) J.x[i] = cscale(J.x[i], f);
    }
}

// ---------------------------------------------------------------------------
// Householder QR of each moving chain's site matrix (one CTA per chain)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double unit_rand(uint64_t seed, uint64_t i) {
    return (double)(mix64(seed + 0x9E3779B97F4A7C15ull * (i + 1)) >> 11) * (1.0 / 9007199254740992.0) - 0.5;
}

constexpr int kQrWarps = kQrThreads / 32;
constexpr int kQrMaxRows = 512;

__global__ void __launch_bounds__(kQrThreads) batched_qr_kernel(const QrProb* __restrict__ probs,
                                                                const int* __restrict__ nprobs) {
    __shared__ QrProb P;
    __shared__ cplx xs[2][kQrMaxRows];   // column j (unscaled, rows > j), double-buffered
    __shared__ cplx piv[2][kQrMaxRows];  // row j of the trailing columns (index k), double-buffered
    __shared__ cplx sk[kQrMaxRows];      // per-column sums s_k = sum_{i>j} conj(x_i) X(i,k)
    const int total = *nprobs;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        __syncthreads();
        if (tid == 0) P = probs[t];
        __syncthreads();
        const int m = P.m, n = P.n;
        cplx* X = P.X;
        // load X
        for (long long e = tid; e < (long long)m * n; e += kQrThreads) {
            const int i = (int)(e % m), j = (int)(e / m);
            cplx v;
            if (P.random_seed) {
                v = cmake(unit_rand(P.random_seed, 2 * e), unit_rand(P.random_seed, 2 * e + 1));
            } else {
                const cplx s = P.site[(long long)(i % P.p) * P.s0 + (long long)(i / P.p) * P.s2 + (long long)j * P.s1];
                v = cconj(s);
            }
            X[e] = v;
        }
        __syncthreads();
        for (int i = tid; i < m; i += kQrThreads) xs[0][i] = X[i];
        for (int k = tid; k < n; k += kQrThreads) piv[0][k] = X[(long long)k * m];
        __syncthreads();
        for (int j = 0; j < n; ++j) {
            const int pb = j & 1;
            // phase 1: s_k = sum_{i>j} conj(x_i) X(i,k) for the warp's columns k >= j
            for (int k = j + warp; k < n; k += kQrWarps) {
                const cplx* Xk = X + (long long)k * m;
                double sr = 0, si = 0;
                for (int i = j + 1 + lane; i < m; i += 32) {
                    const cplx x = xs[pb][i], a = (k == j) ? x : Xk[i];
                    sr = fma(x.x, a.x, fma(x.y, a.y, sr));
                    si = fma(x.x, a.y, fma(-x.y, a.x, si));
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    sr += __shfl_xor_sync(0xffffffffu, sr, o);
                    si += __shfl_xor_sync(0xffffffffu, si, o);
                }
                if (lane == 0) sk[k] = cmake(sr, si);
            }
            __syncthreads();
            // the reflector (zlarfg), computed by every thread
            const double xnorm2 = sk[j].x;
            const cplx alpha = piv[pb][j];
            cplx tau = cmake(0, 0), scale = cmake(1, 0), diag = alpha;
            const bool reflect = !(xnorm2 == 0.0 && alpha.y == 0.0);
            if (reflect) {
                const double beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2), alpha.x);
                const cplx den = cmake(alpha.x - beta, alpha.y);
                const double dd = den.x * den.x + den.y * den.y;
                tau = cmake((beta - alpha.x) / beta, -alpha.y / beta);
                scale = cmake(den.x / dd, -den.y / dd);
                diag = cmake(beta, 0);
            }
            if (tid == 0) P.tau[j] = tau;
            // phase 2: H^H applied to the trailing columns; column j scaled
            const int np = pb ^ 1;
            for (int k = j + warp; k < n; k += kQrWarps) {
                cplx* Xk = X + (long long)k * m;
                if (k == j) {
                    for (int i = j + 1 + lane; i < m; i += 32) Xk[i] = cmul(xs[pb][i], scale);
                    if (lane == 0) Xk[j] = diag;
                    continue;
                }
                if (!reflect) {
                    if (k == j + 1)
                        for (int i = j + 1 + lane; i < m; i += 32) xs[np][i] = Xk[i];
                    if (lane == 0) piv[np][k] = (j + 1 < m) ? Xk[j + 1] : cmake(0, 0);
                    continue;
                }
                // w_k = X(j,k) + conj(scale) s_k;  f = conj(tau) w_k
                const cplx wk = cadd(piv[pb][k], cmul(cconj(scale), sk[k]));
                const cplx f = cmul(cconj(tau), wk);
                const cplx g = cmul(scale, f);
                if (lane == 0) Xk[j] = csub(piv[pb][k], f);
                for (int i = j + 1 + lane; i < m; i += 32) {
                    const cplx v = csub(Xk[i], cmul(xs[pb][i], g));
                    Xk[i] = v;
                    if (k == j + 1) xs[np][i] = v;
                    if (i == j + 1) piv[np][k] = v;
                }
                if (j + 1 >= m && lane == 0) piv[np][k] = cmake(0, 0);
            }
            __syncthreads();
        }
        // R (n x n, upper), conjugated for the left move
        for (long long e = tid; e < (long long)n * n; e += kQrThreads) {
            const int i = (int)(e % n), j = (int)(e / n);
            cplx v = (i <= j) ? X[i + (long long)j * m] : cmake(0, 0);
            if (P.conj_r) v = cconj(v);
            P.rbuf[e] = v;
        }
        // explicit Q = H_0 ... H_{n-1} applied to the first n columns of I;
        // the columns are independent, so each warp owns its columns
        cplx* Q = P.Q;
        for (int k = warp; k < n; k += kQrWarps) {
            cplx* Qk = Q + (long long)k * m;
            for (int i = lane; i < m; i += 32) Qk[i] = cmake(i == k ? 1.0 : 0.0, 0.0);
            __syncwarp();
            for (int j = min(k, n - 1); j >= 0; --j) {
                const cplx tj = P.tau[j];
                if (tj.x == 0.0 && tj.y == 0.0) continue;
                const cplx* Xj = X + (long long)j * m;
                double sr = 0, si = 0;
                for (int i = j + lane; i < m; i += 32) {
                    const cplx v = (i == j) ? cmake(1, 0) : Xj[i], q = Qk[i];   // conj(v) q
                    sr = fma(v.x, q.x, fma(v.y, q.y, sr));
                    si = fma(v.x, q.y, fma(-v.y, q.x, si));
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    sr += __shfl_xor_sync(0xffffffffu, sr, o);
                    si += __shfl_xor_sync(0xffffffffu, si, o);
                }
                const cplx f = cmul(tj, cmake(sr, si));
                for (int i = j + lane; i < m; i += 32) {
                    const cplx v = (i == j) ? cmake(1, 0) : Xj[i];
                    Qk[i] = csub(Qk[i], cmul(v, f));
                }
                __syncwarp();
            }
        }
        __syncthreads();
        for (long long e = tid; e < (long long)m * n; e += kQrThreads) {
            const int i = (int)(e % m), j = (int)(e / m);
            P.site[(long long)(i % P.p) * P.s0 + (long long)(i / P.p) * P.s2 + (long long)j * P.s1] = cconj(Q[e]);
        }
    }
}

// Seeded random site (the centre of a new chain): x = random, normalised later.
__global__ void random_fill_kernel(cplx* x, long long n, uint64_t seed) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        x[e] = cmake(unit_rand(seed, 2 * e), unit_rand(seed, 2 * e + 1));
}

__global__ void set_one_kernel(cplx* const* ptrs, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) *ptrs[i] = cmake(1, 0);
}

}  // namespace
}  // namespace batch
}  // namespace nc

// ===========================================================================
// Host side: the lockstep engine
// ===========================================================================
namespace nc {
namespace batch {
namespace {

constexpr double kMixedSiteTol = 1e-5;     // site tolerance of the complex64 sweeps
constexpr double kMixedSweepTol = 1e-7;    // their sweep-energy hand-over test
constexpr double kMixedSanity = 1e-5;
constexpr int kMixedMaxSweeps = 50;

// Stages of the tile table (the autotuner's key is (stage, chi, D, d)).
enum Stage {
    ST_HEFF_A = 0,     // T = psi_a [L_1..L_cl]   (also the left environment update)
    ST_HEFF_C = 1,     // out_b = [R_1..R_cr] U_b
    ST_ENV_LEFT = 2,   // L'_k2 = U_k2 psi^H
    ST_ENV_Y = 3,      // Y = psi^H [R_1..R_cr]
    ST_ENV_RIGHT = 4,  // R'_k1 = Z_k1 Pp
    ST_ABSORB = 5,     // the neighbour absorbs the gauge factor
    ST_COUNT = 6
};

inline bool outside_tolerance(double a, double b, double tol) {
    // utilities.hpp:418-420
    return (std::fabs(a) + std::fabs(b)) / 2 > tol && std::fabs(a - b) / (std::fabs(a) + std::fabs(b) + tol) > tol;
}

// Bond dimensions of an open chain at `requested` (the same profile as the
// single chain's reset, chain.cpp:175-237).
std::vector<int> bond_profile(int requested, const std::vector<int>& p) {
    NC_ARG(requested > 0, "requested bandwidth must be > 0");
    const size_t mid = (p.size() + 1) / 2;
    auto side = [&](bool rev) {
        std::vector<int> out{1};
        long long prod = 1;
        for (size_t i = 0; i < mid; ++i) {
            prod *= p[rev ? p.size() - 1 - i : i];
            if (prod >= requested) break;
            out.push_back((int)prod);
        }
        return out;
    };
    std::vector<int> fwd = side(false), rev = side(true);
    NC_ARG(!(fwd.size() == mid + 1 || rev.size() == mid + 1),
           "requested bandwidth dimension too large: " + std::to_string(requested));
    std::vector<int> seq = fwd;
    for (size_t i = 0; i < p.size() + 1 - fwd.size() - rev.size(); ++i) seq.push_back(requested);
    for (auto it = rev.rbegin(); it != rev.rend(); ++it) seq.push_back(*it);
    return seq;
}

int chi_bucket(int chi) {
    int b = 8;
    while (b < chi && b < 1024) b <<= 1;
    return b;
}

// Tile configuration when the table has no entry: the smallest tile that
// covers a 64 x 64 block, smaller tiles for small outputs.
int default_cfg(int M, int N) {
    if (M <= 16 && N <= 16) return 0;
    if (M <= 32 && N <= 32) return 1;
    if (M <= 32) return 3;
    if (N <= 32) return 2;
    return 4;
}

struct TileTable {
    struct Entry { int stage, chi, D, d, cfg; };
    std::vector<Entry> entries;
    int lookup(int stage, int chi, int D, int d, int M, int N) const {
        const int b = chi_bucket(chi);
        int best = -1, bestdist = 1 << 30;
        for (const Entry& e : entries) {
            if (e.stage != stage || e.D != D || e.d != d) continue;
            const int dist = std::abs(chi_bucket(e.chi) - b);
            if (dist < bestdist) { bestdist = dist; best = e.cfg; }
        }
        if (best < 0 || best >= kTileConfigs) return default_cfg(M, N);
        return best;
    }
};

// Device arrays in one allocation each, grown only outside graph capture.
template <class T>
struct DevArray {
    T* p = nullptr;
    size_t cap = 0;
    void reserve(size_t n) {
        if (n <= cap) return;
        if (p) NC_CUDA(cudaFree(p));
        NC_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
        cap = n;
    }
    ~DevArray() { if (p) cudaFree(p); }
};

// Pinned staging of the per-step uploads: host data is copied into pinned
// memory and the copy is enqueued asynchronously (a copy from pageable memory
// waits for the stream, which would serialise the host with the device at
// every upload).  The area is reused from its start after each
// synchronisation of the stream; when it runs out it synchronises itself.
struct Stager {
    char* base = nullptr;
    size_t cap = 0, used = 0;
    ~Stager() { if (base) cudaFreeHost(base); }
    void reset() { used = 0; }
    void copy(void* dst, const void* src, size_t bytes, cudaStream_t s) {
        if (!bytes) return;
        size_t off = (used + 255) & ~(size_t)255;
        if (off + bytes > cap) {
            NC_CUDA(cudaStreamSynchronize(s));
            off = 0;
            if (bytes > cap) {
                if (base) NC_CUDA(cudaFreeHost(base));
                base = nullptr;
                cap = std::max(bytes, (size_t)16 << 20);
                NC_CUDA(cudaMallocHost(&base, cap));
            }
        }
        std::memcpy(base + off, src, bytes);
        used = off + bytes;
        NC_CUDA(cudaMemcpyAsync(dst, base + off, bytes, cudaMemcpyHostToDevice, s));
    }
};

// A grouped-GEMM work list: problems, tile prefix sums, tile -> problem map.
struct GemmList {
    std::vector<GProb> h;
    std::vector<int> h_prefix, h_tile;
    DevArray<GProb> d_probs;
    DevArray<int> d_prefix, d_tile, d_count;
    void clear() { h.clear(); }
    void add(GProb g) {
        if (g.M <= 0 || g.N <= 0) return;
        const int bm = kTileM[g.cfg], bn = kTileN[g.cfg];
        g.tiles_n = (g.N + bn - 1) / bn;
        h.push_back(g);
        (void)bm;
    }
    int tiles_of(const GProb& g) const { return ((g.M + kTileM[g.cfg] - 1) / kTileM[g.cfg]) * g.tiles_n; }
    // Uploads the list (the device buffers keep their addresses once reserved).
    void upload(Stager& sg, cudaStream_t s) {
        h_prefix.assign(h.size() + 1, 0);
        for (size_t i = 0; i < h.size(); ++i) h_prefix[i + 1] = h_prefix[i] + tiles_of(h[i]);
        const int total = h_prefix.back();
        h_tile.resize(std::max(total, 1));
        for (size_t i = 0; i < h.size(); ++i)
            for (int t = h_prefix[i]; t < h_prefix[i + 1]; ++t) h_tile[t] = (int)i;
        NC_ARG(h.size() <= d_probs.cap && (size_t)total <= d_tile.cap, "batched work list exceeds its capacity");
        if (!h.empty()) {
            sg.copy(d_probs.p, h.data(), h.size() * sizeof(GProb), s);
            sg.copy(d_prefix.p, h_prefix.data(), h_prefix.size() * sizeof(int), s);
            sg.copy(d_tile.p, h_tile.data(), (size_t)total * sizeof(int), s);
        }
        h_total = total;
        sg.copy(d_count.p, &h_total, sizeof(int), s);
    }
    int h_total = 0;
    void reserve(size_t probs, size_t tiles) {
        d_probs.reserve(probs);
        d_prefix.reserve(probs + 1);
        d_tile.reserve(tiles);
        d_count.reserve(1);
    }
};

struct MixList {
    std::vector<MixProb> h;
    std::vector<int2> h_items;
    DevArray<MixProb> d_probs;
    DevArray<int2> d_items;
    DevArray<int> d_count;
    int h_total = 0;
    void clear() { h.clear(); }
    void add(const MixProb& m) { h.push_back(m); }
    void upload(Stager& sg, cudaStream_t s) {
        h_items.clear();
        for (size_t i = 0; i < h.size(); ++i) {
            const long long chunks = (h[i].total + kMixChunk - 1) / kMixChunk;
            for (long long c = 0; c < chunks; ++c) h_items.push_back(make_int2((int)i, (int)c));
        }
        NC_ARG(h.size() <= d_probs.cap && h_items.size() <= d_items.cap, "batched mix list exceeds its capacity");
        if (!h.empty()) {
            sg.copy(d_probs.p, h.data(), h.size() * sizeof(MixProb), s);
            sg.copy(d_items.p, h_items.data(), h_items.size() * sizeof(int2), s);
        }
        h_total = (int)h_items.size();
        sg.copy(d_count.p, &h_total, sizeof(int), s);
    }
    void reserve(size_t probs, size_t items) {
        d_probs.reserve(probs);
        d_items.reserve(items);
        d_count.reserve(1);
    }
};

struct ChunkList {
    std::vector<VChunk> h;
    DevArray<VChunk> d;
    DevArray<int> d_count;
    int h_total = 0;
    void clear() { h.clear(); }
    // Appends the chunks of one chain's vector of length n; returns (start, count).
    std::pair<int, int> add(int chain, long long n) {
        const int start = (int)h.size();
        for (long long off = 0; off < n; off += kVecChunk)
            h.push_back(VChunk{chain, (int)off, (int)std::min<long long>(kVecChunk, n - off)});
        return {start, (int)h.size() - start};
    }
    void upload(Stager& sg, cudaStream_t s) {
        NC_ARG(h.size() <= d.cap, "batched chunk list exceeds its capacity");
        if (!h.empty()) sg.copy(d.p, h.data(), h.size() * sizeof(VChunk), s);
        h_total = (int)h.size();
        sg.copy(d_count.p, &h_total, sizeof(int), s);
    }
    void reserve(size_t n) {
        d.reserve(n);
        d_count.reserve(1);
    }
};

struct MpoDev {
    int d, cl, cr, nnz;
    const uint32_t* idx;
    const cplx* W;
};

struct ChainHost {
    int N = 0;
    int chi = 0;
    uint64_t seed = 0;
    std::vector<int> phys, bonds;
    std::vector<MpoDev> ops;
    std::vector<cplx*> site, L, R;
    cplx *spare = nullptr, *T = nullptr, *U = nullptr, *V = nullptr, *w = nullptr, *Y = nullptr;
    cplx *X = nullptr, *Q = nullptr, *tau = nullptr, *rbuf = nullptr;
    size_t max_site = 0;
    // sweep state
    int cur = 0, dir = 1;
    bool optimized = false, converged = false, solving = false;
    int sweeps = 0, phase_sweeps = 0, mixed_sweeps = 0, fp64_sweeps = 0;
    double prev = NAN, energy = NAN;
    bool unconverged = false;
    uint64_t matvecs = 0, failures = 0, site_solves = 0;
    int bl(int i) const { return bonds[i]; }
    int br(int i) const { return bonds[i + 1]; }
    size_t site_elems(int i) const { return (size_t)bonds[i + 1] * bonds[i] * phys[i]; }
};

size_t align_up(size_t x) { return (x + 31) & ~(size_t)31; }   // complex elements (512 bytes)

}  // namespace

struct Engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    nc_batch_options opt{};
    std::vector<ChainHost> chains;
    TileTable tiles;
    int sms = 148;
    char* pool = nullptr;
    size_t pool_bytes = 0;

    GemmList g_a, g_c, g_mv1, g_mv2;   // H_eff stages A and C; move lists 1 (absorb + env first) and 2 (env final)
    MixList m_h, m_mv;
    ChunkList lz_chunks, nrm_chunks;
    DevArray<LzChain> d_lz;
    DevArray<LzState> d_st;
    DevArray<LzRitz> d_rz;
    DevArray<int> d_solving, d_active, d_finished;
    DevArray<double> d_energy;
    DevArray<cplx> d_part, d_part_n;
    DevArray<NormJob> d_norm_jobs;
    DevArray<QrProb> d_qr;
    DevArray<int> d_qr_count;
    DevArray<cplx*> d_ones;
    std::vector<LzChain> h_lz;
    std::vector<int> h_solving;
    std::vector<NormJob> h_norm_jobs;
    std::vector<QrProb> h_qr;
    int* h_active = nullptr;   // pinned
    int* h_finished = nullptr;   // pinned, one per chain
    double* h_energy = nullptr;   // pinned, one per chain
    LzState* h_state = nullptr;   // pinned, used for stats reads

    Stager stager;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int grid_gemm = 0, grid_mix = 0, grid_vec = 0, grid_qr = 0;

    // statistics
    uint64_t global_steps = 0, lanczos_iterations = 0, graph_launches = 0, launches = 0;
    uint64_t continued_solves = 0, max_iterations_per_step = 0;
    double seconds = 0, seconds_moves = 0, seconds_solves = 0;   // the last two with time_phases
    double seconds_replays = 0;   // device time of the Lanczos graph replays (time_phases)
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;

    ~Engine() {
        if (ev_a) cudaEventDestroy(ev_a);
        if (ev_b) cudaEventDestroy(ev_b);
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        if (pool) cudaFree(pool);
        if (h_active) cudaFreeHost(h_active);
        if (h_finished) cudaFreeHost(h_finished);
        if (h_energy) cudaFreeHost(h_energy);
        if (h_state) cudaFreeHost(h_state);
        if (stream) cudaStreamDestroy(stream);
    }

    // ---- set-up -----------------------------------------------------------
    void create(uint32_t nch, const uint32_t* nsites, const nc_operator_site* const* sites, const uint32_t* bw,
                const uint64_t* seeds, const nc_batch_options& o) {
        NC_ARG(nch >= 1, "a batch needs at least one chain");
        opt = o;
        NC_ARG(opt.krylov_dimension >= 2 && opt.krylov_dimension <= kMaxKrylov,
               "krylov_dimension must be in [2, 24]");
        NC_ARG(opt.precision <= 1, "precision must be 0 or 1");
        NC_CUDA(cudaGetDevice(&device));
        NC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        NC_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        chains.resize(nch);
        // sizes
        size_t total = 0;
        size_t mpo_bytes = 0;
        for (uint32_t c = 0; c < nch; ++c) {
            ChainHost& ch = chains[c];
            NC_ARG(nsites[c] >= 2, "every chain needs at least two sites");
            ch.N = (int)nsites[c];
            ch.chi = (int)bw[c];
            ch.seed = seeds ? seeds[c] : opt.seed;
            ch.phys.resize(ch.N);
            for (int i = 0; i < ch.N; ++i) {
                const nc_operator_site& s = sites[c][i];
                NC_ARG(s.physical_dimension >= 1 && s.physical_dimension <= (uint32_t)kMixMaxD,
                       "physical dimension must be in [1, 4]");
                NC_ARG(s.number_of_matrices >= 1 && s.number_of_matrices <= (uint32_t)kMixMaxNnz,
                       "operator site: number of matrices must be in [1, 64]");
                NC_ARG(s.left_dimension >= 1 && s.right_dimension >= 1, "operator site dimensions must be >= 1");
                NC_ARG((i == 0) == (s.left_dimension == 1) || s.left_dimension == 1, "bad operator boundary");
                for (uint32_t k = 0; k < s.number_of_matrices; ++k) {
                    NC_ARG(s.indices[2 * k] >= 1 && s.indices[2 * k] <= s.left_dimension,
                           "operator index 'from' out of range");
                    NC_ARG(s.indices[2 * k + 1] >= 1 && s.indices[2 * k + 1] <= s.right_dimension,
                           "operator index 'to' out of range");
                }
                if (i > 0) NC_ARG(sites[c][i - 1].right_dimension == s.left_dimension, "operator bond dimensions disagree");
                ch.phys[i] = (int)s.physical_dimension;
                mpo_bytes += align_up(2 * (size_t)s.number_of_matrices * sizeof(uint32_t) / 16 + 1) * 16 +
                             align_up((size_t)s.physical_dimension * s.physical_dimension * s.number_of_matrices) * 16;
            }
            NC_ARG(sites[c][0].left_dimension == 1 && sites[c][ch.N - 1].right_dimension == 1,
                   "the first operator site needs left dimension 1 and the last right dimension 1");
            ch.bonds = bond_profile(ch.chi, ch.phys);
            size_t ms = 1, mt = 1, mu = 1, mb = 1;
            for (int i = 0; i < ch.N; ++i) {
                const nc_operator_site& s = sites[c][i];
                ms = std::max(ms, ch.site_elems(i));
                mt = std::max(mt, ch.site_elems(i) * s.left_dimension);
                mu = std::max(mu, ch.site_elems(i) * s.right_dimension);
                mb = std::max<size_t>(mb, std::max(ch.bl(i), ch.br(i)));
                NC_ARG((size_t)ch.bl(i) * ch.phys[i] <= (size_t)kQrMaxRows && (size_t)ch.br(i) * ch.phys[i] <= (size_t)kQrMaxRows,
                       "batched chains need bond dimension x physical dimension <= 512");
            }
            ch.max_site = ms;
            size_t env = 0;
            for (int i = 0; i < ch.N; ++i) {
                env += align_up((size_t)ch.bl(i) * ch.bl(i) * sites[c][i].left_dimension);
                env += align_up((size_t)ch.br(i) * ch.br(i) * sites[c][i].right_dimension);
            }
            total += (size_t)(ch.N + 1) * align_up(ms)                    // sites + spare
                     + env                                                // environments
                     + align_up(mt) + align_up(mu)                        // T, U
                     + (size_t)(kMaxKrylov + 2) * align_up(ms)            // V, w
                     + (size_t)(kKeepMax + 1) * align_up(ms)              // Y (thick restart)
                     + 2 * align_up(ms) + align_up(mb) + align_up(mb * mb);   // X, Q, tau, R
        }
        pool_bytes = total * sizeof(cplx) + mpo_bytes + 4096;
        NC_CUDA(cudaMalloc(&pool, pool_bytes));
        char* cursor = pool;
        auto take = [&](size_t elems) {
            cplx* p = reinterpret_cast<cplx*>(cursor);
            cursor += align_up(elems) * sizeof(cplx);
            return p;
        };
        size_t nchunk_cap = 0, ntile_a = 0, ntile_c = 0, nmv1 = 0, nmv2 = 0, nmix_items = 0;
        for (uint32_t c = 0; c < nch; ++c) {
            ChainHost& ch = chains[c];
            ch.ops.resize(ch.N);
            for (int i = 0; i < ch.N; ++i) {
                const nc_operator_site& s = sites[c][i];
                MpoDev& op = ch.ops[i];
                op.d = (int)s.physical_dimension;
                op.cl = (int)s.left_dimension;
                op.cr = (int)s.right_dimension;
                op.nnz = (int)s.number_of_matrices;
                uint32_t* idx = reinterpret_cast<uint32_t*>(cursor);
                cursor += align_up(2 * (size_t)op.nnz * sizeof(uint32_t) / 16 + 1) * 16;
                NC_CUDA(cudaMemcpyAsync(idx, s.indices, 2 * (size_t)op.nnz * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
                cplx* W = take((size_t)op.d * op.d * op.nnz);
                NC_CUDA(cudaMemcpyAsync(W, s.matrices, (size_t)op.d * op.d * op.nnz * sizeof(cplx), cudaMemcpyHostToDevice,
                                        stream));
                op.idx = idx;
                op.W = W;
            }
            ch.site.resize(ch.N);
            for (int i = 0; i < ch.N; ++i) ch.site[i] = take(ch.max_site);
            ch.spare = take(ch.max_site);
            ch.L.resize(ch.N);
            ch.R.resize(ch.N);
            size_t mt = 1, mu = 1, mb = 1;
            for (int i = 0; i < ch.N; ++i) {
                ch.L[i] = take((size_t)ch.bl(i) * ch.bl(i) * ch.ops[i].cl);
                ch.R[i] = take((size_t)ch.br(i) * ch.br(i) * ch.ops[i].cr);
                mt = std::max(mt, ch.site_elems(i) * ch.ops[i].cl);
                mu = std::max(mu, ch.site_elems(i) * ch.ops[i].cr);
                mb = std::max<size_t>(mb, std::max(ch.bl(i), ch.br(i)));
            }
            ch.T = take(mt);
            ch.U = take(mu);
            ch.V = take((size_t)(kMaxKrylov + 1) * align_up(ch.max_site));
            ch.w = take(ch.max_site);
            ch.Y = take((size_t)(kKeepMax + 1) * align_up(ch.max_site));
            ch.X = take(ch.max_site);
            ch.Q = take(ch.max_site);
            ch.tau = take(mb);
            ch.rbuf = take(mb * mb);
            // work-list capacities (every tile counted at the smallest tile shape)
            size_t ta = 0, tc = 0, t1 = 0, t2 = 0, mi = 0;
            for (int i = 0; i < ch.N; ++i) {
                const long long bl = ch.bl(i), br = ch.br(i), d = ch.phys[i], cl = ch.ops[i].cl, cr = ch.ops[i].cr;
                auto tl = [](long long M, long long N) { return (size_t)(((M + 15) / 16) * ((N + 15) / 16)); };
                ta = std::max(ta, (size_t)d * tl(br, bl * cl));
                tc = std::max(tc, (size_t)d * tl(br, bl));
                // move list 1: absorb (either direction) + first environment stage
                const size_t absorb = std::max((size_t)d * tl(br, br), tl(bl, bl * d)) + 4 * tl(br, br) + 4 * tl(bl, bl * 4);
                t1 = std::max(t1, absorb + std::max((size_t)d * tl(br, bl * cl), tl(bl * d, br * cr)));
                t2 = std::max(t2, std::max((size_t)cr * tl(br, br), (size_t)cl * tl(bl, bl)));
                mi = std::max(mi, (size_t)((ch.site_elems(i) * std::max(cl, cr) + kMixChunk - 1) / kMixChunk));
            }
            ntile_a += ta;
            ntile_c += tc;
            nmv1 += t1;
            nmv2 += t2;
            nmix_items += mi;
            nchunk_cap += (ch.max_site + kVecChunk - 1) / kVecChunk;
        }
        NC_ARG((size_t)(cursor - pool) <= pool_bytes, "batched pool sizing");
        const size_t B = nch;
        g_a.reserve(4 * B, ntile_a);
        g_c.reserve(4 * B, ntile_c);
        g_mv1.reserve(12 * B, nmv1);
        g_mv2.reserve(kMixMaxNnz * B, nmv2);
        m_h.reserve(B, nmix_items);
        m_mv.reserve(B, nmix_items);
        lz_chunks.reserve(nchunk_cap);
        nrm_chunks.reserve(nchunk_cap);
        d_lz.reserve(B);
        d_st.reserve(B);
        d_rz.reserve(B);
        d_solving.reserve(B);
        d_finished.reserve(B);
        d_energy.reserve(B);
        d_active.reserve(1);
        d_part.reserve(nchunk_cap * kPartStride);
        d_part_n.reserve(nchunk_cap * kPartStride);
        d_norm_jobs.reserve(B);
        d_qr.reserve(B);
        d_qr_count.reserve(1);
        d_ones.reserve(2 * B);
        h_lz.assign(B, LzChain{});
        h_solving.assign(B, 0);
        h_norm_jobs.assign(B, NormJob{nullptr, 0, 0});
        NC_CUDA(cudaMallocHost(&h_active, sizeof(int)));
        NC_CUDA(cudaMallocHost(&h_finished, B * sizeof(int)));
        NC_CUDA(cudaMallocHost(&h_energy, B * sizeof(double)));
        NC_CUDA(cudaMallocHost(&h_state, B * sizeof(LzState)));
        NC_CUDA(cudaMemsetAsync(d_st.p, 0, B * sizeof(LzState), stream));
        // persistent grids from the occupancy of each kernel
        int occ = 0;
        NC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, grouped_gemm_kernel, kGemmThreads, kGemmSmem));
        grid_gemm = sms * std::max(1, occ);
        NC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, grouped_mix_kernel, 256, 0));
        grid_mix = sms * std::max(1, occ);
        NC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, lz_cgs_kernel<1>, kLzT, 0));
        grid_vec = sms * std::max(1, occ);
        NC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batched_qr_kernel, kQrThreads, 0));
        grid_qr = sms * std::max(1, occ);
        // a small batch has fewer work items than a full persistent grid: launch
        // no more CTAs than the largest work list can give work to
        auto cap = [](int grid, size_t items) { return (int)std::max<size_t>(1, std::min<size_t>(grid, items)); };
        grid_gemm = cap(grid_gemm, std::max(std::max(ntile_a, ntile_c), std::max(nmv1, nmv2)));
        grid_mix = cap(grid_mix, nmix_items);
        grid_vec = cap(grid_vec, nchunk_cap);

        NC_CUDA(cudaStreamSynchronize(stream));
    }

    // ---- stage builders -------------------------------------------------------
    GProb gp(int chain, int stage, const ChainHost& ch, int site, int prec, int M, int N, int K, int opA, const cplx* A,
             long long lda, int opB, const cplx* B, long long ldb, cplx* C, long long ldc) const {
        GProb g{};
        g.M = M; g.N = N; g.K = K;
        g.opA = opA; g.opB = opB;
        g.prec = prec;
        g.chain = chain;
        g.A = A; g.lda = lda;
        g.B = B; g.ldb = ldb;
        g.C = C; g.ldc = ldc;
        const int chi = std::max(ch.bl(site), ch.br(site));
        const int D = std::max(ch.ops[site].cl, ch.ops[site].cr);
        g.cfg = tiles.lookup(stage, chi, D, ch.phys[site], M, N);
        return g;
    }

    // Left environment of site i+1 from L_i and site i (sos_left), into the lists.
    void add_env_left(int c, int i, int prec) {
        ChainHost& ch = chains[c];
        const MpoDev& op = ch.ops[i];
        const int bl = ch.bl(i), br = ch.br(i), d = op.d, cl = op.cl, cr = op.cr;
        for (int a = 0; a < d; ++a)
            g_mv1.add(gp(c, ST_HEFF_A, ch, i, prec, br, bl * cl, bl, G_N, ch.site[i] + (size_t)a * br * bl, br, G_N,
                         ch.L[i], bl, ch.T + (size_t)a * br * bl * cl, br));
        MixProb m{};
        m.mode = 0; m.chain = c; m.br = br; m.bl = bl; m.cl = cl; m.cr = cr; m.d = d; m.nnz = op.nnz;
        m.idx = op.idx; m.W = op.W; m.in = ch.T; m.out = ch.U; m.total = (long long)br * cr * bl * d;
        m_mv.add(m);
        for (int k2 = 0; k2 < cr; ++k2)
            g_mv2.add(gp(c, ST_ENV_LEFT, ch, i, prec, br, br, bl * d, G_N, ch.U + (size_t)k2 * br, (long long)br * cr, G_C,
                         ch.site[i], br, ch.L[i + 1] + (size_t)k2 * br * br, br));
    }

    // Right environment of site i-1 from R_i and site i (sos_right).
    void add_env_right(int c, int i, int prec) {
        ChainHost& ch = chains[c];
        const MpoDev& op = ch.ops[i];
        const int bl = ch.bl(i), br = ch.br(i), d = op.d, cl = op.cl, cr = op.cr;
        // Y (bl*d x br*cr) = psi^H [R_1..R_cr]  -> U buffer
        g_mv1.add(gp(c, ST_ENV_Y, ch, i, prec, bl * d, br * cr, br, G_C, ch.site[i], br, G_N, ch.R[i], br, ch.U,
                     (long long)bl * d));
        MixProb m{};
        m.mode = 1; m.chain = c; m.br = br; m.bl = bl; m.cl = cl; m.cr = cr; m.d = d; m.nnz = op.nnz;
        m.idx = op.idx; m.W = op.W; m.in = ch.U; m.out = ch.T; m.total = (long long)bl * br * d * cl;
        m_mv.add(m);
        for (int k1 = 0; k1 < cl; ++k1) {
            GProb g = gp(c, ST_ENV_RIGHT, ch, i, prec, bl, bl, br * d, G_N, ch.T + (size_t)k1 * bl * br * d, bl, G_N,
                         ch.site[i], br, ch.R[i - 1] + (size_t)k1 * bl * bl, bl);
            g.b_kdiv = br;
            g.b_kstride = (long long)br * bl;
            g_mv2.add(g);
        }
    }

    void run_gemm(GemmList& g, const LzState* st) {
        grouped_gemm_kernel<<<grid_gemm, kGemmThreads, kGemmSmem, stream>>>(g.d_probs.p, g.d_prefix.p, g.d_tile.p,
                                                                             g.d_count.p, st);
        NC_CHECK_LAUNCH();
        launches++;
    }
    void run_mix(MixList& m, const LzState* st) {
        grouped_mix_kernel<<<grid_mix, 256, 0, stream>>>(m.d_probs.p, m.d_items.p, m.d_count.p, st);
        NC_CHECK_LAUNCH();
        launches++;
    }

    // Normalise one vector per listed chain (nrm_chunks / h_norm_jobs filled).
    void run_normalise() {
        nrm_chunks.upload(stager, stream);
        stager.copy(d_norm_jobs.p, h_norm_jobs.data(), h_norm_jobs.size() * sizeof(NormJob), stream);
        norm_partial_kernel<<<grid_vec, kLzT, 0, stream>>>(nrm_chunks.d.p, nrm_chunks.d_count.p, d_norm_jobs.p,
                                                           d_part_n.p);
        NC_CHECK_LAUNCH();
        norm_scale_kernel<<<grid_vec, kLzT, 0, stream>>>(nrm_chunks.d.p, nrm_chunks.d_count.p, d_norm_jobs.p,
                                                         d_part_n.p);
        NC_CHECK_LAUNCH();
        launches += 2;
    }

    void run_qr() {
        const int n = (int)h_qr.size();
        if (n == 0) return;
        stager.copy(d_qr.p, h_qr.data(), h_qr.size() * sizeof(QrProb), stream);
        stager.copy(d_qr_count.p, &qr_count_host, sizeof(int), stream);
        batched_qr_kernel<<<std::min(grid_qr, n), kQrThreads, 0, stream>>>(d_qr.p, d_qr_count.p);
        NC_CHECK_LAUNCH();
        launches++;
    }
    int qr_count_host = 0;

    QrProb qr_prob(int c, cplx* site, int m, int n, int p, long long s0, long long s1, long long s2, int conj_r,
                   unsigned long long seed) {
        ChainHost& ch = chains[c];
        QrProb q{};
        q.chain = c; q.m = m; q.n = n; q.p = p; q.s0 = s0; q.s1 = s1; q.s2 = s2;
        q.site = site; q.X = ch.X; q.Q = ch.Q; q.tau = ch.tau; q.rbuf = ch.rbuf;
        q.conj_r = conj_r; q.random_seed = seed;
        return q;
    }

    // ---- initial states and environment rebuilds ------------------------------
    // Every chain: random right-normalised sites N-1..1 (seeded per chain and
    // site), a random normalised centre at site 0, trivial boundaries, and the
    // right environments built from the last site down (lockstep over sites).
    void reset_all(int prec) {
        std::vector<cplx*> ones;
        for (auto& ch : chains) {
            ones.push_back(ch.L[0]);
            ones.push_back(ch.R[ch.N - 1]);
        }
        stager.copy(d_ones.p, ones.data(), ones.size() * sizeof(cplx*), stream);
        set_one_kernel<<<((int)ones.size() + 255) / 256, 256, 0, stream>>>(d_ones.p, (int)ones.size());
        NC_CHECK_LAUNCH();
        // the centre
        nrm_chunks.clear();
        for (size_t c = 0; c < chains.size(); ++c) {
            ChainHost& ch = chains[c];
            const long long n = (long long)ch.site_elems(0);
            random_fill_kernel<<<std::max(1, (int)std::min<long long>((n + 255) / 256, 64)), 256, 0, stream>>>(
                ch.site[0], n, seed_of(ch, 0));
            NC_CHECK_LAUNCH();
            auto r = nrm_chunks.add((int)c, n);
            h_norm_jobs[c] = NormJob{ch.site[0], r.first, r.second};
        }
        run_normalise();
        int nmax = 0;
        for (auto& ch : chains) nmax = std::max(nmax, ch.N);
        for (int t = 0; t < nmax - 1; ++t) {
            h_qr.clear();
            g_mv1.clear(); g_mv2.clear(); m_mv.clear();
            for (size_t c = 0; c < chains.size(); ++c) {
                ChainHost& ch = chains[c];
                const int i = ch.N - 1 - t;
                if (i < 1) continue;
                // right-normalised random site: conj(Q) of a random (br*d x bl) matrix
                const int br = ch.br(i), bl = ch.bl(i), d = ch.phys[i];
                h_qr.push_back(qr_prob((int)c, ch.site[i], br * d, bl, br, 1, br, (long long)br * bl, 0, seed_of(ch, i)));
                add_env_right((int)c, i, prec);
            }
            qr_count_host = (int)h_qr.size();
            run_qr();
            upload_moves();
            run_gemm(g_mv1, nullptr);
            run_mix(m_mv, nullptr);
            run_gemm(g_mv2, nullptr);
        }
        for (auto& ch : chains) {
            ch.cur = 0;
            ch.dir = 1;
            ch.optimized = false;
        }
    }

    // Every environment of the current state rebuilt at `prec` (centre at 0).
    void refresh_all(int prec) {
        int nmax = 0;
        for (auto& ch : chains) {
            NC_ARG(ch.cur == 0, "batched refresh needs the centre at site 0");
            nmax = std::max(nmax, ch.N);
        }
        for (int t = 0; t < nmax - 1; ++t) {
            g_mv1.clear(); g_mv2.clear(); m_mv.clear();
            for (size_t c = 0; c < chains.size(); ++c) {
                ChainHost& ch = chains[c];
                const int i = ch.N - 1 - t;
                if (i >= 1) add_env_right((int)c, i, prec);
            }
            upload_moves();
            run_gemm(g_mv1, nullptr);
            run_mix(m_mv, nullptr);
            run_gemm(g_mv2, nullptr);
        }
    }

    void upload_moves() {
        g_mv1.upload(stager, stream);
        g_mv2.upload(stager, stream);
        m_mv.upload(stager, stream);
    }

    uint64_t seed_of(const ChainHost& ch, int site) const {
        uint64_t z = ch.seed * 0x9E3779B97F4A7C15ull + (uint64_t)(site + 1) * 0xD1B54A32D192ED03ull;
        z ^= z >> 29;
        return z | 1ull;   // never 0 (0 means "load from the site")
    }

    // ---- one lockstep action: moves, then solves --------------------------------
    void do_moves(const std::vector<int>& movers, int prec) {
        if (movers.empty()) return;
        h_qr.clear();
        g_mv1.clear(); g_mv2.clear(); m_mv.clear();
        nrm_chunks.clear();
        for (int c : movers) {
            ChainHost& ch = chains[c];
            const int i = ch.cur;
            if (ch.dir > 0) {
                // site i -> left-normalised; site i+1 absorbs Rt^H (gauge_right)
                const int bm = ch.br(i), bl = ch.bl(i), dl = ch.phys[i];
                const int K = bl * dl;
                NC_ARG(K >= bm, "not enough degrees of freedom to normalize");
                h_qr.push_back(qr_prob(c, ch.site[i], K, bm, K, bm, 1, 0, 0, 0));
                const int brn = ch.br(i + 1), dr = ch.phys[i + 1];
                for (int s = 0; s < dr; ++s)
                    g_mv1.add(gp(c, ST_ABSORB, ch, i + 1, 0, brn, bm, bm, G_N, ch.site[i + 1] + (size_t)s * brn * bm, brn,
                                 G_C, ch.rbuf, bm, ch.spare + (size_t)s * brn * bm, brn));
                add_env_left(c, i, prec);
            } else {
                // site i -> right-normalised; site i-1 absorbs conj(Rt) (gauge_left)
                const int br = ch.br(i), bm = ch.bl(i), dr = ch.phys[i];
                const int K = br * dr;
                NC_ARG(K >= bm, "not enough degrees of freedom to normalize");
                h_qr.push_back(qr_prob(c, ch.site[i], K, bm, br, 1, br, (long long)br * bm, 1, 0));
                const int bll = ch.bl(i - 1), dl = ch.phys[i - 1];
                g_mv1.add(gp(c, ST_ABSORB, ch, i - 1, 0, bm, bll * dl, bm, G_N, ch.rbuf, bm, G_N, ch.site[i - 1], bm,
                             ch.spare, bm));
                add_env_right(c, i, prec);
            }
        }
        qr_count_host = (int)h_qr.size();
        run_qr();
        upload_moves();
        run_gemm(g_mv1, nullptr);
        run_mix(m_mv, nullptr);
        run_gemm(g_mv2, nullptr);
        // the absorbing neighbour becomes the centre: swap in and normalise
        for (int c : movers) {
            ChainHost& ch = chains[c];
            const int j = ch.cur + ch.dir;
            std::swap(ch.site[j], ch.spare);
            ch.cur = j;
            auto r = nrm_chunks.add(c, (long long)ch.site_elems(j));
            h_norm_jobs[c] = NormJob{ch.site[j], r.first, r.second};
        }
        run_normalise();
    }

    void capture_graph() {
        if (graph_exec) return;
        const int B = (int)chains.size();
        const int cb = (B + 7) / 8, tb = (B + 255) / 256;
        LzState* st = d_st.p;
        NC_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        grouped_gemm_kernel<<<grid_gemm, kGemmThreads, kGemmSmem, stream>>>(g_a.d_probs.p, g_a.d_prefix.p,
                                                                             g_a.d_tile.p, g_a.d_count.p, st);
        grouped_mix_kernel<<<grid_mix, 256, 0, stream>>>(m_h.d_probs.p, m_h.d_items.p, m_h.d_count.p, st);
        grouped_gemm_kernel<<<grid_gemm, kGemmThreads, kGemmSmem, stream>>>(g_c.d_probs.p, g_c.d_prefix.p,
                                                                             g_c.d_tile.p, g_c.d_count.p, st);
        lz_cgs_kernel<0><<<grid_vec, kLzT, 0, stream>>>(lz_chunks.d.p, lz_chunks.d_count.p, d_lz.p, st, d_part.p);
        lz_reduce_kernel<0><<<cb, 256, 0, stream>>>(B, d_lz.p, st, d_part.p);
        lz_cgs_kernel<1><<<grid_vec, kLzT, 0, stream>>>(lz_chunks.d.p, lz_chunks.d_count.p, d_lz.p, st, d_part.p);
        lz_reduce_kernel<1><<<cb, 256, 0, stream>>>(B, d_lz.p, st, d_part.p);
        lz_cgs_kernel<2><<<grid_vec, kLzT, 0, stream>>>(lz_chunks.d.p, lz_chunks.d_count.p, d_lz.p, st, d_part.p);
        lz_reduce_kernel<2><<<cb, 256, 0, stream>>>(B, d_lz.p, st, d_part.p);
        lz_ritz_kernel<<<B, 32, 0, stream>>>(B, d_lz.p, st, d_rz.p, d_active.p);
        lz_next_kernel<<<grid_vec, kLzT, 0, stream>>>(lz_chunks.d.p, lz_chunks.d_count.p, d_lz.p, st);
        // thick restart of the chains whose basis filled in this iteration
        lz_restart_form_kernel<<<grid_vec, kLzT, 0, stream>>>(lz_chunks.d.p, lz_chunks.d_count.p, d_lz.p, st, d_rz.p);
        lz_restart_copy_kernel<<<grid_vec, kLzT, 0, stream>>>(lz_chunks.d.p, lz_chunks.d_count.p, d_lz.p, st);
        lz_restart_state_kernel<<<B, 32, 0, stream>>>(B, d_lz.p, st, d_rz.p);
        lz_inc_kernel<<<tb, 256, 0, stream>>>(B, st, d_active.p);
        cudaError_t e = cudaStreamEndCapture(stream, &graph);
        NC_CUDA(e);
        NC_CHECK_LAUNCH();
        NC_CUDA(cudaGraphInstantiate(&graph_exec, graph, 0));
    }
    static constexpr int kGraphKernels = 15;

    int read_active() {
        NC_CUDA(cudaMemcpyAsync(h_active, d_active.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
        NC_CUDA(cudaStreamSynchronize(stream));
        return *h_active;
    }

    // One step of the site solves: `starting` chains begin a solve at their
    // centre (the guess is the site), `continuing` ones carry on with the
    // basis they have.  Every solving chain gets at most `iteration_cap`
    // Lanczos iterations in this step (thick restarts happen inside the
    // graph); a chain whose solve ends (converged or failed) has its result
    // taken and is returned in `finished` with its energy, the others continue
    // in the next step, so one slow solve does not hold the other chains.
    void do_solves(const std::vector<int>& starting, const std::vector<int>& continuing, int prec,
                   double site_tol, double sanity, std::vector<int>& finished) {
        finished.clear();
        if (starting.empty() && continuing.empty()) return;
        const int B = (int)chains.size();
        const int tb = (B + 255) / 256;
        g_a.clear(); g_c.clear(); m_h.clear(); lz_chunks.clear();
        std::fill(h_solving.begin(), h_solving.end(), 0);
        for (int c = 0; c < B; ++c) h_lz[c].ccount = 0;
        auto add = [&](int c, int flag) {
            ChainHost& ch = chains[c];
            const int i = ch.cur;
            const MpoDev& op = ch.ops[i];
            const int bl = ch.bl(i), br = ch.br(i), d = op.d, cl = op.cl, cr = op.cr;
            const long long n = (long long)br * bl * d;
            for (int a = 0; a < d; ++a) {
                // A = V_j(:,:,a): the basis is packed at stride n
                GProb g = gp(c, ST_HEFF_A, ch, i, prec, br, bl * cl, bl, G_N, ch.V + (size_t)a * br * bl, br, G_N, ch.L[i],
                             bl, ch.T + (size_t)a * br * bl * cl, br);
                g.use_jsel = 1;
                g.a_jstride = n;
                g_a.add(g);
            }
            MixProb m{};
            m.mode = 0; m.chain = c; m.br = br; m.bl = bl; m.cl = cl; m.cr = cr; m.d = d; m.nnz = op.nnz;
            m.idx = op.idx; m.W = op.W; m.in = ch.T; m.out = ch.U; m.total = (long long)br * cr * bl * d;
            m_h.add(m);
            for (int b = 0; b < d; ++b)
                g_c.add(gp(c, ST_HEFF_C, ch, i, prec, br, bl, br * cr, G_N, ch.R[i], br, G_N,
                           ch.U + (size_t)b * br * cr * bl, (long long)br * cr, ch.w + (size_t)b * br * bl, br));
            auto r = lz_chunks.add(c, n);
            LzChain& z = h_lz[c];
            z.V = ch.V; z.w = ch.w; z.x = ch.site[i]; z.n = n; z.tol = site_tol;
            z.cstart = r.first; z.ccount = r.second;
            z.m_max = (int)opt.krylov_dimension;
            z.keep = std::max(1, std::min(std::max(4, z.m_max / 3), z.m_max - 2));
            z.Y = ch.Y;
            z.maxit = (int)std::max<uint32_t>(1, opt.maximum_number_of_iterations);
            h_solving[c] = flag;
        };
        for (int c : starting) add(c, 1);
        for (int c : continuing) add(c, 2);
        g_a.upload(stager, stream);
        g_c.upload(stager, stream);
        m_h.upload(stager, stream);
        lz_chunks.upload(stager, stream);
        stager.copy(d_lz.p, h_lz.data(), B * sizeof(LzChain), stream);
        stager.copy(d_solving.p, h_solving.data(), B * sizeof(int), stream);
        capture_graph();
        LzState* st = d_st.p;
        lz_init_kernel<<<tb, 256, 0, stream>>>(B, d_solving.p, st);
        lz_form_kernel<0><<<grid_vec, kLzT, 0, stream>>>(lz_chunks.d.p, lz_chunks.d_count.p, d_lz.p, st, d_rz.p, d_solving.p,
                                                         d_part.p);
        lz_norm_kernel<0><<<tb, 256, 0, stream>>>(B, d_lz.p, st, d_solving.p, d_part.p, sanity);
        lz_scale_kernel<0><<<grid_vec, kLzT, 0, stream>>>(lz_chunks.d.p, lz_chunks.d_count.p, d_lz.p, st, d_solving.p);
        NC_CHECK_LAUNCH();
        launches += 4;
        const int check_every = 4;
        uint64_t iters = 0;
        if (opt.time_phases) {
            if (!ev_a) {
                NC_CUDA(cudaEventCreate(&ev_a));
                NC_CUDA(cudaEventCreate(&ev_b));
            }
            NC_CUDA(cudaEventRecord(ev_a, stream));
        }
        for (int it = 0; it < iteration_cap; ++it) {
            NC_CUDA(cudaGraphLaunch(graph_exec, stream));
            graph_launches++;
            lanczos_iterations++;
            iters++;
            launches += kGraphKernels;
            if ((it + 1) % check_every == 0 && read_active() == 0) break;
        }
        max_iterations_per_step = std::max(max_iterations_per_step, iters);
        if (opt.time_phases) {
            NC_CUDA(cudaEventRecord(ev_b, stream));
            NC_CUDA(cudaEventSynchronize(ev_b));
            float ms = 0;
            NC_CUDA(cudaEventElapsedTime(&ms, ev_a, ev_b));
            seconds_replays += ms * 1e-3;
        }
        // the results of the solves that ended
        lz_form_kernel<2><<<grid_vec, kLzT, 0, stream>>>(lz_chunks.d.p, lz_chunks.d_count.p, d_lz.p, st, d_rz.p, d_solving.p,
                                                         d_part.p);
        lz_norm_kernel<2><<<tb, 256, 0, stream>>>(B, d_lz.p, st, d_solving.p, d_part.p, sanity);
        lz_scale_kernel<2><<<grid_vec, kLzT, 0, stream>>>(lz_chunks.d.p, lz_chunks.d_count.p, d_lz.p, st, d_solving.p);
        lz_finish_kernel<<<tb, 256, 0, stream>>>(B, d_solving.p, st, d_finished.p, d_energy.p);
        NC_CHECK_LAUNCH();
        launches += 4;
        NC_CUDA(cudaMemcpyAsync(h_finished, d_finished.p, B * sizeof(int), cudaMemcpyDeviceToHost, stream));
        NC_CUDA(cudaMemcpyAsync(h_energy, d_energy.p, B * sizeof(double), cudaMemcpyDeviceToHost, stream));
        NC_CUDA(cudaStreamSynchronize(stream));
        stager.reset();   // every staged upload has been consumed
        for (int c = 0; c < B; ++c)
            if (h_solving[c] && h_finished[c]) {
                finished.push_back(c);
                chains[c].energy = h_energy[c];
            }
    }
    int iteration_cap = 8;

    // ---- sweeps ---------------------------------------------------------------
    // Every chain sweeps (chain.cpp:147-163) until its sweep energy settles
    // (base_chain.cpp:112-123) at `sweep_tol`, or `max_sweeps` (0: no bound).
    // A chain that has settled idles until every chain has.
    void phase(int prec, double site_tol, double sweep_tol, double sanity, uint32_t max_sweeps) {
        const int B = (int)chains.size();
        for (auto& ch : chains) {
            ch.cur = 0;
            ch.dir = 1;
            ch.optimized = false;
            ch.converged = false;
            ch.solving = false;
            ch.phase_sweeps = 0;
            ch.prev = NAN;
        }
        std::vector<int> movers, starting, continuing, finished;
        for (;;) {
            movers.clear();
            starting.clear();
            continuing.clear();
            for (int c = 0; c < B; ++c) {
                ChainHost& ch = chains[c];
                if (ch.converged) continue;
                if (ch.solving) {
                    continuing.push_back(c);
                    continue;
                }
                if (ch.optimized) {
                    if (ch.dir > 0 && ch.cur + 1 >= ch.N) ch.dir = -1;
                    movers.push_back(c);
                }
                starting.push_back(c);
            }
            if (starting.empty() && continuing.empty()) break;
            global_steps++;
            continued_solves += continuing.size();
            if (opt.time_phases) {
                auto t0 = std::chrono::steady_clock::now();
                do_moves(movers, prec);
                NC_CUDA(cudaStreamSynchronize(stream));
                auto t1 = std::chrono::steady_clock::now();
                do_solves(starting, continuing, prec, site_tol, sanity, finished);
                auto t2 = std::chrono::steady_clock::now();
                seconds_moves += std::chrono::duration<double>(t1 - t0).count();
                seconds_solves += std::chrono::duration<double>(t2 - t1).count();
            } else {
                do_moves(movers, prec);
                do_solves(starting, continuing, prec, site_tol, sanity, finished);
            }
            for (int c : starting) chains[c].solving = true;
            for (int c : finished) {
                ChainHost& ch = chains[c];
                ch.solving = false;
                ch.optimized = true;
                ch.site_solves++;
                if (!(ch.dir < 0 && ch.cur == 0)) continue;
                // a sweep has ended at site 0
                ch.dir = 1;
                ch.sweeps++;
                ch.phase_sweeps++;
                if (prec) ch.mixed_sweeps++;
                else ch.fp64_sweeps++;
                const double now = ch.energy;
                if (!std::isnan(ch.prev) && !outside_tolerance(ch.prev, now, sweep_tol)) {
                    ch.converged = true;
                } else if (max_sweeps && (uint32_t)ch.phase_sweeps >= max_sweeps) {
                    ch.converged = true;
                    ch.unconverged = true;
                }
                ch.prev = now;
            }
        }
        read_states();
    }

    // Energies and solver counters of every chain (synchronises).
    void read_states() {
        const int B = (int)chains.size();
        NC_CUDA(cudaMemcpyAsync(h_state, d_st.p, B * sizeof(LzState), cudaMemcpyDeviceToHost, stream));
        NC_CUDA(cudaStreamSynchronize(stream));
        for (int c = 0; c < B; ++c) {
            h_energy[c] = h_state[c].energy;
            chains[c].energy = h_state[c].energy;
        }
    }

    void solve() {
        const auto t0 = std::chrono::steady_clock::now();
        const int prec = (int)opt.precision;
        // random initial states; energies reset (NaN: the first solve is accepted)
        init_energies();
        reset_all(prec);
        if (prec) {
            phase(1, std::max(opt.site_convergence_threshold, kMixedSiteTol), kMixedSweepTol,
                  std::max(opt.sanity_check_threshold, kMixedSanity), kMixedMaxSweeps);
            if (opt.refine) {
                for (auto& ch : chains) ch.unconverged = false;
                refresh_all(0);
                phase(0, opt.site_convergence_threshold, opt.sweep_convergence_threshold, opt.sanity_check_threshold,
                      opt.maximum_sweeps);
            }
        } else {
            phase(0, opt.site_convergence_threshold, opt.sweep_convergence_threshold, opt.sanity_check_threshold,
                  opt.maximum_sweeps);
        }
        NC_CUDA(cudaStreamSynchronize(stream));
        seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    void init_energies() {
        const int B = (int)chains.size();
        for (int c = 0; c < B; ++c) {
            h_state[c] = LzState{};
            h_state[c].energy = NAN;
            h_state[c].done = 1;
        }
        NC_CUDA(cudaMemcpyAsync(d_st.p, h_state, B * sizeof(LzState), cudaMemcpyHostToDevice, stream));
        NC_CUDA(cudaStreamSynchronize(stream));
        for (auto& ch : chains) {
            ch.sweeps = ch.mixed_sweeps = ch.fp64_sweeps = 0;
            ch.unconverged = false;
            ch.site_solves = 0;
        }
    }
};

// ---------------------------------------------------------------------------
// Autotuner support: one grouped launch of `problems` copies of a stage's
// interior-site shape at (chi, D, d), timed per tile configuration.
// ---------------------------------------------------------------------------
void stage_shape(int stage, int chi, int D, int d, int& M, int& N, int& K, int& opA, int& opB, int& count) {
    const int bl = chi, br = chi, cl = D, cr = D;
    opA = G_N; opB = G_N; count = 1;
    switch (stage) {
        case ST_HEFF_A: M = br; N = bl * cl; K = bl; count = d; break;
        case ST_HEFF_C: M = br; N = bl; K = br * cr; count = d; break;
        case ST_ENV_LEFT: M = br; N = br; K = bl * d; opB = G_C; count = cr; break;
        case ST_ENV_Y: M = bl * d; N = br * cr; K = br; opA = G_C; break;
        case ST_ENV_RIGHT: M = bl; N = bl; K = br * d; count = cl; break;
        default: M = br; N = chi; K = chi; opB = G_C; count = d; break;   // ST_ABSORB (right move)
    }
}

}  // namespace batch
}  // namespace nc

using nc::batch::Engine;

struct nc_batch {
    Engine e;
};

extern "C" {

void nc_batch_options_init(nc_batch_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->precision = 1;
    o->refine = 1;
    o->krylov_dimension = 24;
    o->maximum_number_of_iterations = 100;
    o->sanity_check_threshold = 1e-12;
    o->site_convergence_threshold = 1e-12;
    o->sweep_convergence_threshold = 1e-12;
    o->maximum_sweeps = 0;
    o->seed = 1;
}

nc_batch* nc_batch_create(uint32_t number_of_chains, const uint32_t* number_of_sites,
                          const nc_operator_site* const* sites, const uint32_t* bandwidth_dimensions,
                          const uint64_t* seeds, const nc_batch_options* options) {
    NC_ABI_BEGIN
    NC_ARG(number_of_chains >= 1 && number_of_sites && sites && bandwidth_dimensions, "nc_batch_create: bad arguments");
    nc_batch_options o;
    nc_batch_options_init(&o);
    if (options) o = *options;
    std::unique_ptr<nc_batch> b(new nc_batch());
    b->e.create(number_of_chains, number_of_sites, sites, bandwidth_dimensions, seeds, o);
    return b.release();
    NC_ABI_END
    return nullptr;
}

void nc_batch_free(nc_batch* b) { delete b; }

int nc_batch_set_tile_table(nc_batch* b, const int32_t* entries, uint32_t count) {
    NC_ABI_BEGIN
    NC_ARG(b && (entries || count == 0), "nc_batch_set_tile_table: bad arguments");
    b->e.tiles.entries.clear();
    for (uint32_t i = 0; i < count; ++i) {
        const int32_t* x = entries + 5 * (size_t)i;
        NC_ARG(x[0] >= 0 && x[0] < nc::batch::ST_COUNT, "tile table: bad stage");
        NC_ARG(x[4] >= 0 && x[4] < nc::batch::kTileConfigs, "tile table: bad tile configuration");
        b->e.tiles.entries.push_back({x[0], x[1], x[2], x[3], x[4]});
    }
    NC_ABI_END
    return nc::g_status;
}

int nc_batch_solve(nc_batch* b) {
    NC_ABI_BEGIN
    NC_ARG(b, "nc_batch_solve: null batch");
    b->e.solve();
    NC_ABI_END
    return nc::g_status;
}

int nc_batch_get_results(nc_batch* b, nc_batch_chain_result* out) {
    NC_ABI_BEGIN
    NC_ARG(b && out, "nc_batch_get_results: bad arguments");
    for (size_t c = 0; c < b->e.chains.size(); ++c) {
        const auto& ch = b->e.chains[c];
        const auto& s = b->e.h_state[c];
        nc_batch_chain_result& r = out[c];
        r.energy = ch.energy;
        r.sweeps = (uint32_t)ch.sweeps;
        r.mixed_sweeps = (uint32_t)ch.mixed_sweeps;
        r.fp64_sweeps = (uint32_t)ch.fp64_sweeps;
        r.site_solves = ch.site_solves;
        r.converged = ch.unconverged ? 0u : 1u;
        r.bandwidth_dimension = (uint32_t)ch.chi;
        (void)s;
    }
    NC_ABI_END
    return nc::g_status;
}

int nc_batch_get_stats(nc_batch* b, nc_batch_stats* st) {
    NC_ABI_BEGIN
    NC_ARG(b && st, "nc_batch_get_stats: bad arguments");
    std::memset(st, 0, sizeof(*st));
    st->chains = (uint32_t)b->e.chains.size();
    st->global_steps = b->e.global_steps;
    st->lanczos_iterations = b->e.lanczos_iterations;
    st->graph_launches = b->e.graph_launches;
    st->kernel_launches = b->e.launches;
    st->seconds = b->e.seconds;
    st->seconds_moves = b->e.seconds_moves;
    st->seconds_solves = b->e.seconds_solves;
    st->seconds_replays = b->e.seconds_replays;
    st->continued_solves = b->e.continued_solves;
    st->max_iterations_per_step = b->e.max_iterations_per_step;
    st->device_bytes = b->e.pool_bytes;
    NC_ABI_END
    return nc::g_status;
}

int nc_batch_autotune_stage(uint32_t stage, uint32_t chi, uint32_t D, uint32_t d, uint32_t problems, uint32_t reps,
                            uint32_t precision, double* seconds_per_config) {
    using namespace nc::batch;
    NC_ABI_BEGIN
    NC_ARG(stage < (uint32_t)ST_COUNT && chi >= 1 && chi <= 256 && D >= 1 && D <= 16 && d >= 1 && d <= 4 &&
               problems >= 1 && problems <= 4096 && reps >= 1 && seconds_per_config,
           "nc_batch_autotune_stage: bad arguments");
    int M, N, K, opA, opB, count;
    stage_shape((int)stage, (int)chi, (int)D, (int)d, M, N, K, opA, opB, count);
    const size_t ea = (size_t)M * K, eb = (size_t)K * N, ec = (size_t)M * N;
    cudaStream_t s;
    NC_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct Guard {
        cudaStream_t s;
        std::vector<void*> ptrs;
        cudaEvent_t a = nullptr, b = nullptr;
        ~Guard() {
            if (a) cudaEventDestroy(a);
            if (b) cudaEventDestroy(b);
            for (void* p : ptrs) cudaFree(p);
            cudaStreamDestroy(s);
        }
    } g{s, {}};
    nc::cplx *A, *B, *C;
    NC_CUDA(cudaMalloc(&A, ea * problems * sizeof(nc::cplx)));
    g.ptrs.push_back(A);
    NC_CUDA(cudaMalloc(&B, eb * problems * sizeof(nc::cplx)));
    g.ptrs.push_back(B);
    NC_CUDA(cudaMalloc(&C, ec * count * problems * sizeof(nc::cplx)));
    g.ptrs.push_back(C);
    random_fill_kernel<<<256, 256, 0, s>>>(A, (long long)ea * problems, 11);
    random_fill_kernel<<<256, 256, 0, s>>>(B, (long long)eb * problems, 12);
    NC_CHECK_LAUNCH();
    int dev = 0, sms = 0, occ = 0;
    NC_CUDA(cudaGetDevice(&dev));
    NC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    NC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, grouped_gemm_kernel, kGemmThreads, kGemmSmem));
    const int grid = sms * std::max(1, occ);
    NC_CUDA(cudaEventCreate(&g.a));
    NC_CUDA(cudaEventCreate(&g.b));
    GemmList list;
    Stager sg;
    list.reserve((size_t)problems * count, (size_t)problems * count * ((M + 15) / 16) * ((N + 15) / 16));
    for (int cfg = 0; cfg < kTileConfigs; ++cfg) {
        list.clear();
        for (uint32_t p = 0; p < problems; ++p)
            for (int q = 0; q < count; ++q) {
                GProb x{};
                x.M = M; x.N = N; x.K = K; x.opA = opA; x.opB = opB; x.cfg = cfg; x.prec = (int)precision;
                x.A = A + ea * p; x.lda = (opA == G_N) ? M : K;
                x.B = B + eb * p; x.ldb = (opB == G_N) ? K : N;
                x.C = C + ec * ((size_t)p * count + q); x.ldc = M;
                list.add(x);
            }
        list.upload(sg, s);
        for (int w = 0; w < 2; ++w)
            grouped_gemm_kernel<<<grid, kGemmThreads, kGemmSmem, s>>>(list.d_probs.p, list.d_prefix.p, list.d_tile.p,
                                                                       list.d_count.p, nullptr);
        NC_CHECK_LAUNCH();
        NC_CUDA(cudaEventRecord(g.a, s));
        for (uint32_t r = 0; r < reps; ++r)
            grouped_gemm_kernel<<<grid, kGemmThreads, kGemmSmem, s>>>(list.d_probs.p, list.d_prefix.p, list.d_tile.p,
                                                                       list.d_count.p, nullptr);
        NC_CHECK_LAUNCH();
        NC_CUDA(cudaEventRecord(g.b, s));
        NC_CUDA(cudaEventSynchronize(g.b));
        float ms = 0;
        NC_CUDA(cudaEventElapsedTime(&ms, g.a, g.b));
        seconds_per_config[cfg] = ms * 1e-3 / reps;
    }
    NC_ABI_END
    return nc::g_status;
}

uint32_t nc_batch_tile_configs(int32_t* rows, int32_t* cols) {
    using namespace nc::batch;
    for (int i = 0; i < kTileConfigs; ++i) {
        if (rows) rows[i] = kTileM[i];
        if (cols) cols[i] = kTileN[i];
    }
    return (uint32_t)kTileConfigs;
}

}  // extern "C"
