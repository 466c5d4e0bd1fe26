// Gauge moves on the device: blocked Householder QR and its uses.
//
// The reference moves the orthogonality centre with the polar factor of an
// SVD (zgesdd, core.f95:2708-2960): A = (U S U^H)(U V^H).  Energies, overlaps
// and environments are invariant under any gauge A = P Q with Q having
// orthonormal rows, so the device path uses the Householder QR of A^H
// instead (A^H = Qt Rt, Q = Qt^H, P = Rt^H): it is backward stable for
// rank-deficient sites (Schmidt values down to zero), needs no iterative SVD
// and maps onto GEMMs.
//
// QR layout: right-looking blocked Householder, outer blocks of NB=64 columns
// (trailing update = three complex GEMMs through the compact WY form
// I - V T V^H), inner panels of JB=4 columns factorised by one CTA with the
// panel held in registers (mp <= 2048 rows) and updated inside the outer
// block by a per-column kernel.  Q is formed explicitly by backward
// accumulation of the block reflectors (zungqr order).
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "nc_common.cuh"
#include "nc_kernels.h"

namespace nc {

namespace {

constexpr int JB = 4;      // panel width
constexpr int NB = 64;     // outer block width
constexpr int PT = 256;    // panel threads
constexpr int PMAXROWS = 8;  // rows per thread -> mp <= 2048

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* red, double* out) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) red[wid * NV + k] = x;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0;
        for (int w = 0; w < PT / 32; ++w) s += red[w * NV + threadIdx.x];
        out[threadIdx.x] = s;
    }
    __syncthreads();
}

// Factor the mp x jb panel at A (ld lda), jb <= JB.  Writes R (upper part)
// and the reflector tails back to A, the unit-diagonal reflectors to V
// (ld ldv, rows 0..mp-1), tau, and the JB x JB compact-WY T.
template <int ROWS>
__global__ void __launch_bounds__(PT) panel_qr_kernel(int mp, int jb, cplx* __restrict__ A, long long lda,
                                                      cplx* __restrict__ V, long long ldv,
                                                      cplx* __restrict__ tau_out, cplx* __restrict__ Tout) {
    __shared__ double red[(PT / 32) * 2 * JB * JB];
    __shared__ double outv[2 * JB * JB];
    __shared__ cplx s_alpha;
    __shared__ cplx s_tau[JB];
    const int tid = threadIdx.x;
    cplx a[ROWS][JB];
#pragma unroll
    for (int r = 0; r < ROWS; ++r) {
        int row = tid + r * PT;
#pragma unroll
        for (int c = 0; c < JB; ++c) a[r][c] = (row < mp && c < jb) ? A[row + c * lda] : cmake(0, 0);
    }
#pragma unroll
    for (int c = 0; c < JB; ++c) {  // unrolled so that a[][c] stays in registers
        if (c >= jb) break;
        double p[1] = {0.0};
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            int row = tid + r * PT;
            if (row > c && row < mp) p[0] += cabs2(a[r][c]);
            if (row == c) s_alpha = a[r][c];
        }
        block_sum<1>(p, red, outv);
        const double xnorm2 = outv[0];
        const cplx alpha = s_alpha;
        cplx t = cmake(0, 0), scale = cmake(1, 0), diag = alpha;
        if (!(xnorm2 == 0.0 && alpha.y == 0.0)) {
            double beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2), alpha.x);
            t = cmake((beta - alpha.x) / beta, -alpha.y / beta);
            cplx den = cmake(alpha.x - beta, alpha.y);
            double dd = den.x * den.x + den.y * den.y;
            scale = cmake(den.x / dd, -den.y / dd);
            diag = cmake(beta, 0);
        }
        double w[2 * JB];
#pragma unroll
        for (int k = 0; k < 2 * JB; ++k) w[k] = 0;
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            int row = tid + r * PT;
            cplx v = cmake(0, 0);
            if (row == c) { a[r][c] = diag; v = cmake(1, 0); }
            else if (row > c && row < mp) { a[r][c] = cmul(a[r][c], scale); v = a[r][c]; }
            cplx vc = cconj(v);
#pragma unroll
            for (int c2 = 0; c2 < JB; ++c2) {
                if (c2 > c) {
                    cplx q = cmul(vc, a[r][c2]);
                    w[2 * c2] += q.x;
                    w[2 * c2 + 1] += q.y;
                }
            }
        }
        block_sum<2 * JB>(w, red, outv);
        const cplx tc = cconj(t);
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            int row = tid + r * PT;
            if (row < c || row >= mp) continue;
            cplx v = (row == c) ? cmake(1, 0) : a[r][c];
#pragma unroll
            for (int c2 = 0; c2 < JB; ++c2) {
                if (c2 > c && c2 < jb) {
                    cplx wc = cmake(outv[2 * c2], outv[2 * c2 + 1]);
                    a[r][c2] = csub(a[r][c2], cmul(tc, cmul(v, wc)));
                }
            }
        }
        if (tid == 0) s_tau[c] = t;
        __syncthreads();
    }
    // write back and Gram matrix of the reflectors
    double g[2 * JB * JB];
#pragma unroll
    for (int k = 0; k < 2 * JB * JB; ++k) g[k] = 0;
#pragma unroll
    for (int r = 0; r < ROWS; ++r) {
        int row = tid + r * PT;
        if (row >= mp) continue;
        cplx v[JB];
#pragma unroll
        for (int c = 0; c < JB; ++c) {
            v[c] = (c >= jb || row < c) ? cmake(0, 0) : (row == c ? cmake(1, 0) : a[r][c]);
            if (c < jb) {
                A[row + c * lda] = a[r][c];
                V[row + c * ldv] = v[c];
            }
        }
#pragma unroll
        for (int k = 0; k < JB; ++k)
#pragma unroll
            for (int c = 0; c < JB; ++c) {
                if (k < c) {
                    cplx q = cmul(cconj(v[k]), v[c]);
                    g[2 * (k + JB * c)] += q.x;
                    g[2 * (k + JB * c) + 1] += q.y;
                }
            }
    }
    block_sum<2 * JB * JB>(g, red, outv);
    if (tid == 0) {
        // compact WY (zlarft, forward/columnwise): T(c,c) = tau_c,
        // T(0:c,c) = -tau_c T(0:c,0:c) V(:,0:c)^H v_c
        cplx T[JB][JB];
        for (int i = 0; i < JB; ++i)
            for (int j = 0; j < JB; ++j) T[i][j] = cmake(0, 0);
        for (int c = 0; c < jb; ++c) {
            cplx tc = s_tau[c];
            T[c][c] = tc;
            for (int k = 0; k < c; ++k) {
                cplx acc = cmake(0, 0);
                for (int l = k; l < c; ++l)
                    acc = cadd(acc, cmul(T[k][l], cmake(outv[2 * (l + JB * c)], outv[2 * (l + JB * c) + 1])));
                T[k][c] = cscale(cmul(tc, acc), -1.0);
            }
        }
        for (int i = 0; i < JB; ++i)
            for (int j = 0; j < JB; ++j) Tout[i + JB * j] = T[i][j];
        for (int c = 0; c < jb; ++c) tau_out[c] = s_tau[c];
    }
}

// Apply the panel's (I - V T V^H)^H to nc columns of A (one block per column):
// a -= V T^H (V^H a).
__global__ void __launch_bounds__(PT) panel_apply_kernel(int mp, int jb, const cplx* __restrict__ V,
                                                         long long ldv, const cplx* __restrict__ T,
                                                         cplx* __restrict__ A, long long lda) {
    __shared__ double red[(PT / 32) * 2 * JB];
    __shared__ double outv[2 * JB];
    cplx* col = A + (long long)blockIdx.x * lda;
    double w[2 * JB];
#pragma unroll
    for (int k = 0; k < 2 * JB; ++k) w[k] = 0;
    for (int row = threadIdx.x; row < mp; row += PT) {
        cplx x = col[row];
#pragma unroll
        for (int c = 0; c < JB; ++c) {
            if (c < jb) {
                cplx q = cmul(cconj(V[row + c * ldv]), x);
                w[2 * c] += q.x;
                w[2 * c + 1] += q.y;
            }
        }
    }
    block_sum<2 * JB>(w, red, outv);
    // w2 = T^H w
    cplx w2[JB];
#pragma unroll
    for (int i = 0; i < JB; ++i) {
        cplx acc = cmake(0, 0);
        for (int k = 0; k <= i && k < jb; ++k)
            acc = cadd(acc, cmul(cconj(T[k + JB * i]), cmake(outv[2 * k], outv[2 * k + 1])));
        w2[i] = acc;
    }
    for (int row = threadIdx.x; row < mp; row += PT) {
        cplx x = col[row];
#pragma unroll
        for (int c = 0; c < JB; ++c)
            if (c < jb) x = csub(x, cmul(V[row + c * ldv], w2[c]));
        col[row] = x;
    }
}

// Compact-WY T (nb x nb) from G = V^H V (nb x nb) and tau, one CTA.
__global__ void build_t_kernel(int nb, const cplx* __restrict__ G, const cplx* __restrict__ tau,
                               cplx* __restrict__ T, int ldt) {
    // thread k owns row k of T; the diagonal is written by thread 0 and read
    // Uses T^{-1} = striu(V^H V) + diag(1/tau) (the compact-WY identity of
    // Puglisi 1992 / Joffrain et al. 2006): thread j back-substitutes column
    // j of T independently, T(i,j) = -tau_i sum_{l=i+1..j} G(i,l) T(l,j),
    // T(j,j) = tau_j (a zero tau gives a zero row and column, as it should).
    const int j = threadIdx.x;
    if (j >= nb) return;
    cplx col[NB];
    for (int i = 0; i < nb; ++i) col[i] = cmake(0, 0);
    col[j] = tau[j];
    for (int i = j - 1; i >= 0; --i) {
        cplx acc = cmake(0, 0);
        for (int l = i + 1; l <= j; ++l) acc = cadd(acc, cmul(G[i + nb * l], col[l]));
        col[i] = cscale(cmul(tau[i], acc), -1.0);
    }
    for (int i = 0; i < NB; ++i) T[i + (long long)ldt * j] = (i < nb) ? col[i] : cmake(0, 0);
    if (j == 0)
        for (int c = nb; c < NB; ++c)
            for (int i = 0; i < NB; ++i) T[i + (long long)ldt * c] = cmake(0, 0);
}

__global__ void identity_cols(long long m, int n, cplx* __restrict__ Q) {
    const long long total = m * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long r = e % m, c = e / m;
        Q[e] = (r == c) ? cmake(1, 0) : cmake(0, 0);
    }
}

// R (n x n, zeros below) from the upper triangle of A (ld lda), optionally conjugated.
__global__ void extract_r(int n, const cplx* __restrict__ A, long long lda, bool conj, cplx* __restrict__ R) {
    const long long total = (long long)n * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int r = (int)(e % n), c = (int)(e / n);
        cplx v = (r <= c) ? A[r + c * lda] : cmake(0, 0);
        R[e] = conj ? cconj(v) : v;
    }
}

unsigned gsz(long long n) {
    return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 16));
}

void launch_panel(Context& ctx, int mp, int jb, cplx* A, long long lda, cplx* V, long long ldv, cplx* tau,
                  cplx* T) {
    const int rows = (mp + PT - 1) / PT;
    if (rows <= 1) panel_qr_kernel<1><<<1, PT, 0, ctx.stream>>>(mp, jb, A, lda, V, ldv, tau, T);
    else if (rows <= 2) panel_qr_kernel<2><<<1, PT, 0, ctx.stream>>>(mp, jb, A, lda, V, ldv, tau, T);
    else if (rows <= 4) panel_qr_kernel<4><<<1, PT, 0, ctx.stream>>>(mp, jb, A, lda, V, ldv, tau, T);
    else panel_qr_kernel<8><<<1, PT, 0, ctx.stream>>>(mp, jb, A, lda, V, ldv, tau, T);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

}  // namespace

void householder_qr(Context& ctx, int m, int n, cplx* A, cplx* Q, cplx* R, bool conjR) {
    NC_ARG(m >= n && n >= 1, "householder_qr: need m >= n >= 1");
    NC_ARG(m <= PT * PMAXROWS, "householder_qr: at most 2048 rows (bond x physical dimension)");
    Arena& ar = ctx.scratch();
    ArenaFrame f(ar);
    const long long lda = m;
    cplx* V = ar.alloc_n<cplx>((size_t)m * n);
    cplx* tau = ar.alloc_n<cplx>(n);
    const int nblocks = (n + NB - 1) / NB;
    cplx* Tb = ar.alloc_n<cplx>((size_t)nblocks * NB * NB);
    cplx* T4 = ar.alloc_n<cplx>(JB * JB);
    cplx* G = ar.alloc_n<cplx>(NB * NB);
    cplx* W = ar.alloc_n<cplx>((size_t)NB * n);
    cplx* W2 = ar.alloc_n<cplx>((size_t)NB * n);
    zfill(ctx, (long long)m * n, cmake(0, 0), V);

    for (int ob = 0; ob < nblocks; ++ob) {
        const int j0 = ob * NB;
        const int nb = std::min(NB, n - j0);
        const int mp = m - j0;
        // inner panels
        for (int jj = j0; jj < j0 + nb; jj += JB) {
            const int jb = std::min(JB, j0 + nb - jj);
            launch_panel(ctx, m - jj, jb, A + jj + jj * lda, lda, V + jj + jj * (long long)m, m, tau + jj, T4);
            const int rest = j0 + nb - (jj + jb);
            if (rest > 0) {
                panel_apply_kernel<<<rest, PT, 0, ctx.stream>>>(m - jj, jb, V + jj + jj * (long long)m, m, T4,
                                                                A + jj + (jj + jb) * lda, lda);
                NC_CHECK_LAUNCH();
                ctx.launches++;
            }
        }
        // compact WY T for the outer block
        const cplx* Vb = V + j0 + j0 * (long long)m;
        zgemm(zgemm_params(OP_C, OP_N, nb, nb, mp, Vb, m, Vb, m, G, nb), ctx);
        cplx* T = Tb + (size_t)ob * NB * NB;
        build_t_kernel<<<1, NB, 0, ctx.stream>>>(nb, G, tau + j0, T, NB);
        NC_CHECK_LAUNCH();
        ctx.launches++;
        // trailing update: A2 -= V T^H (V^H A2)
        const int nt = n - (j0 + nb);
        if (nt > 0) {
            cplx* A2 = A + j0 + (j0 + nb) * lda;
            zgemm(zgemm_params(OP_C, OP_N, nb, nt, mp, Vb, m, A2, lda, W, nb), ctx);
            zgemm(zgemm_params(OP_C, OP_N, nb, nt, nb, T, NB, W, nb, W2, nb), ctx);
            ZGemmParams p = zgemm_params(OP_N, OP_N, mp, nt, nb, Vb, m, W2, nb, A2, lda);
            p.alpha = cmake(-1, 0);
            p.beta = cmake(1, 0);
            zgemm(p, ctx);
        }
    }
    if (R) {
        extract_r<<<gsz((long long)n * n), 256, 0, ctx.stream>>>(n, A, lda, conjR, R);
        NC_CHECK_LAUNCH();
        ctx.launches++;
    }
    if (Q) {
        identity_cols<<<gsz((long long)m * n), 256, 0, ctx.stream>>>(m, n, Q);
        NC_CHECK_LAUNCH();
        ctx.launches++;
        for (int ob = nblocks - 1; ob >= 0; --ob) {
            const int j0 = ob * NB;
            const int nb = std::min(NB, n - j0);
            const int mp = m - j0;
            const int nq = n - j0;
            const cplx* Vb = V + j0 + j0 * (long long)m;
            const cplx* T = Tb + (size_t)ob * NB * NB;
            cplx* Qs = Q + j0 + j0 * (long long)m;
            // Qs = (I - V T V^H) Qs
            zgemm(zgemm_params(OP_C, OP_N, nb, nq, mp, Vb, m, Qs, m, W, nb), ctx);
            zgemm(zgemm_params(OP_N, OP_N, nb, nq, nb, T, NB, W, nb, W2, nb), ctx);
            ZGemmParams p = zgemm_params(OP_N, OP_N, mp, nq, nb, Vb, m, W2, nb, Qs, m);
            p.alpha = cmake(-1, 0);
            p.beta = cmake(1, 0);
            zgemm(p, ctx);
        }
    }
}

// ---------------------------------------------------------------------------
// gauge moves (core.f95:2708-2960 semantics, QR gauge)
// ---------------------------------------------------------------------------

// A QR of one shape recorded as a CUDA graph: a gauge move issues a few
// hundred short kernels (the panels are latency bound), so replaying a
// pre-recorded graph removes the per-launch host overhead.  The plan owns its
// input/output buffers and a private workspace arena, so the pointers baked
// into the graph stay valid and are never shared with other work.
struct QrPlan {
    int m = 0, n = 0;
    bool conjR = false;
    Arena arena;
    cplx* X = nullptr;   // input (m x n), overwritten
    cplx* Q = nullptr;   // explicit Q (m x n)
    cplx* R = nullptr;   // R (n x n), conjugated if conjR
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t kernels = 0;
    ~QrPlan() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

namespace {
QrPlan& qr_plan(Context& ctx, int m, int n, bool conjR) {
    thread_local std::vector<std::unique_ptr<QrPlan>> plans;
    for (auto& p : plans)
        if (p->m == m && p->n == n && p->conjR == conjR) return *p;
    auto p = std::make_unique<QrPlan>();
    p->m = m; p->n = n; p->conjR = conjR;
    p->X = p->arena.alloc_n<cplx>((size_t)m * n);
    p->Q = p->arena.alloc_n<cplx>((size_t)m * n);
    p->R = p->arena.alloc_n<cplx>((size_t)n * n);
    plans.push_back(std::move(p));
    return *plans.back();
}

// Run the QR of plan.X; the first run of a shape executes directly (so the
// private arena grows to its final size) and then records the graph.
void qr_run(Context& ctx, QrPlan& P) {
    if (P.exec) {
        NC_CUDA(cudaGraphLaunch(P.exec, ctx.stream));
        ctx.launches += P.kernels;
        return;
    }
    const bool prof = ctx.profile;
    ctx.profile = false;
    ctx.ws_override = &P.arena;
    try {
        householder_qr(ctx, P.m, P.n, P.X, P.Q, P.R, P.conjR);
        const uint64_t l0 = ctx.launches;
        NC_CUDA(cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeRelaxed));
        try {
            householder_qr(ctx, P.m, P.n, P.X, P.Q, P.R, P.conjR);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(ctx.stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        NC_CUDA(cudaStreamEndCapture(ctx.stream, &P.graph));
        P.kernels = ctx.launches - l0;
        ctx.launches = l0;
        NC_CUDA(cudaGraphInstantiate(&P.exec, P.graph, 0));
    } catch (...) {
        ctx.ws_override = nullptr;
        ctx.profile = prof;
        throw;
    }
    ctx.ws_override = nullptr;
    ctx.profile = prof;
}
}  // namespace

void gauge_right(Context& ctx, int bl, int bm, int br, int dl, int dr, const cplx* A, const cplx* B,
                 cplx* normA, cplx* denormB) {
    const int K = bl * dl;
    NC_ARG(K >= bm, "not enough degrees of freedom to normalize");
    QrPlan& P = qr_plan(ctx, K, bm, false);
    const int p_t[3] = {1, 0, 2};
    permute3(ctx, A, bm, K, 1, p_t, true, P.X);             // X = A^H  (K x bm)
    qr_run(ctx, P);                                          // A^H = Qt Rt
    permute3(ctx, P.Q, K, bm, 1, p_t, true, normA);         // normA = Qt^H
    if (B && denormB) {
        // denormB_s = B_s Rt^H  (neighbour absorbs P = Rt^H on its left index)
        ZGemmParams p = zgemm_params(OP_N, OP_C, br, bm, bm, B, br, P.R, bm, denormB, br);
        p.batch = dr;
        p.sA0 = (long long)br * bm; p.sB0 = 0; p.sC0 = (long long)br * bm;
        zgemm(p, ctx);
    }
}

void gauge_left(Context& ctx, int bl, int bm, int br, int dl, int dr, const cplx* A, const cplx* B,
                cplx* denormA, cplx* normB) {
    const int K = br * dr;
    NC_ARG(K >= bm, "not enough degrees of freedom to normalize");
    QrPlan& P = qr_plan(ctx, K, bm, true);
    const cplx* Rc = P.R;
    const int p_rs[3] = {0, 2, 1};
    permute3(ctx, B, br, bm, dr, p_rs, true, P.X);           // X((r,s),m) = conj(B(r,m,s))
    qr_run(ctx, P);                                          // Rc = conj(Rt)
    permute3(ctx, P.Q, br, dr, bm, p_rs, true, normB);       // normB(r,m,s) = conj(Qt((r,s),m))
    if (A && denormA) {
        // denormA = conj(Rt) * A  (as bm x bl*dl)
        zgemm(zgemm_params(OP_N, OP_N, bm, bl * dl, bm, Rc, bm, A, bm, denormA, bm), ctx);
    }
}

void rand_norm_site(Context& ctx, int br, int bl, int d, uint64_t seed, cplx* out) {
    // core.f95:2634-2659: columns l of the (br*d x bl) workspace orthonormal
    NC_ARG(br * d >= bl, "not enough degrees of freedom to normalize");
    ArenaFrame f(ctx.arena);
    const int K = br * d;
    cplx* X = ctx.arena.alloc_n<cplx>((size_t)K * bl);
    cplx* Qt = ctx.arena.alloc_n<cplx>((size_t)K * bl);
    zrandom(ctx, (long long)K * bl, seed, X);
    householder_qr(ctx, K, bl, X, Qt, nullptr, false);
    const int p_rs[3] = {0, 2, 1};
    permute3(ctx, Qt, br, d, bl, p_rs, false, out);  // state(r,l,s) = ws(r,s,l)
}

void rand_unnorm_site(Context& ctx, int br, int bl, int d, uint64_t seed, cplx* out) {
    // core.f95:2661-2671
    const long long n = (long long)br * bl * d;
    zrandom(ctx, n, seed, out);
    ArenaFrame f(ctx.arena);
    cplx* nr = ctx.arena.alloc_n<cplx>(1);
    znrm2sq(ctx, n, out, nr);
    znormalize_dev(ctx, n, nr, out);
}

void increase_bandwidth(Context& ctx, int bl, int bm, int br, int dl, int dr, int new_bm, uint64_t seed,
                        const cplx* A, const cplx* B, cplx* outA, cplx* outB) {
    // core.f95:3090-3144
    ArenaFrame f(ctx.arena);
    cplx* M = ctx.arena.alloc_n<cplx>((size_t)new_bm * bm);
    cplx* X = ctx.arena.alloc_n<cplx>((size_t)new_bm * bm);
    zrandom(ctx, (long long)new_bm * bm, seed, X);
    householder_qr(ctx, new_bm, bm, X, M, nullptr, false);   // isometry new_bm x bm
    cplx* e1 = ctx.arena.alloc_n<cplx>((size_t)new_bm * bl * dl);
    cplx* e2 = ctx.arena.alloc_n<cplx>((size_t)br * new_bm * dr);
    zgemm(zgemm_params(OP_N, OP_N, new_bm, bl * dl, bm, M, new_bm, A, bm, e1, new_bm), ctx);
    ZGemmParams p = zgemm_params(OP_N, OP_C, br, new_bm, bm, B, br, M, new_bm, e2, br);
    p.batch = dr;
    p.sA0 = (long long)br * bm; p.sB0 = 0; p.sC0 = (long long)br * new_bm;
    zgemm(p, ctx);
    gauge_left(ctx, bl, new_bm, br, dl, dr, e1, e2, outA, outB);
}

}  // namespace nc
