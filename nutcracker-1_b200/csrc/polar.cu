// Exact polar gauge moves for the Level-0 drop-in entry points.
//
// The reference normalises a site with the polar factor of an SVD
// (zgesdd, core.f95:2708-2960): for the site matrix M = U S V^H the
// normalised site is U V^H and the neighbour absorbs H = U S U^H (conj(H)
// in the reference's index order).  The device-resident chain uses the
// cheaper Householder-QR gauge (qr.cu), which gives a gauge-equivalent but
// element-wise different site; the Level-0 entry points
// (norm_denorm_going_left_/right_, norm_for_left_/right_) return the
// reference's tensors, computed here as
//
//   M^H = Qt Rt          (Householder QR, qr.cu; Rt square, bm x bm)
//   Rt  = Up Hp          (polar factor of the small square factor: QDWH)
//   =>  M = Hp (Qt Up)^H,  so  U V^H = (Qt Up)^H  and  H = Hp.
//
// QDWH (Nakatsukasa, Bai and Gygi, "Optimizing Halley's iteration for
// computing the matrix polar decomposition", SIAM J. Matrix Anal. Appl. 31,
// 2010), QR form: X_0 = Rt / ||Rt||_F and
//   [sqrt(c_k) X_k; I] = [Q1; Q2] R,
//   X_{k+1} = (b_k/c_k) X_k + (a_k - b_k/c_k)/sqrt(c_k) Q1 Q2^H,
// with the dynamically weighted (a_k, b_k, c_k) from a lower bound l_k of the
// smallest singular value (started at 1e-15, so at most six iterations for
// any condition number up to 1e15).  It stops when ||X_{k+1} - X_k||_F <=
// (5 eps)^(1/3) (the convergence is cubic).  Hp = Up^H Rt, made exactly
// Hermitian.  The polar factor is unique when M has full row rank; for a
// rank-deficient site (a Schmidt value at zero) it is not, QDWH returns a
// partial isometry, and the move falls back to the QR gauge (still an exact
// isometry and the same state).
#include <algorithm>
#include <cmath>

#include "nc_common.cuh"
#include "nc_kernels.h"

namespace nc {

namespace {

// S (2n x n) = [s X; I]
__global__ void stack_kernel(int n, double s, const cplx* __restrict__ X, cplx* __restrict__ S) {
    const long long total = 2LL * n * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % (2 * n)), j = (int)(e / (2 * n));
        S[e] = (i < n) ? cscale(X[i + (long long)n * j], s) : cmake((i - n == j) ? 1.0 : 0.0, 0.0);
    }
}

// D = X - Y
__global__ void diff_kernel(long long n, const cplx* __restrict__ X, const cplx* __restrict__ Y,
                            cplx* __restrict__ D) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x)
        D[e] = csub(X[e], Y[e]);
}

// H <- (H + H^H) / 2, optionally conjugated, written to out
__global__ void hermitize_kernel(int n, const cplx* __restrict__ H, bool conj, cplx* __restrict__ out) {
    const long long total = (long long)n * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % n), j = (int)(e / n);
        const cplx a = H[i + (long long)n * j], b = H[j + (long long)n * i];
        cplx v = cmake(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
        if (conj) v.y = -v.y;
        out[e] = v;
    }
}

// G = U^H U - I, for the isometry check
__global__ void minus_identity_kernel(int n, cplx* __restrict__ G) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
        G[e + (long long)n * e].x -= 1.0;
}

unsigned grid_of(long long total) {
    return (unsigned)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 8));
}

double host_norm(Context& ctx, long long n, const cplx* x) {
    ArenaFrame f(ctx.arena);
    cplx* r = ctx.arena.alloc_n<cplx>(1);
    znrm2sq(ctx, n, x, r);
    return std::sqrt(read_scalar(ctx, r).x);
}

// QDWH weights from the lower bound l of the smallest singular value.
void qdwh_weights(double l, double* a, double* b, double* c) {
    const double l2 = l * l;
    const double dd = std::cbrt(4.0 * (1.0 - l2) / (l2 * l2));
    const double sq = std::sqrt(1.0 + dd);
    *a = sq + 0.5 * std::sqrt(8.0 - 4.0 * dd + 8.0 * (2.0 - l2) / (l2 * sq));
    *b = (*a - 1.0) * (*a - 1.0) / 4.0;
    *c = *a + *b - 1.0;
}

}  // namespace

bool polar_qdwh(Context& ctx, int n, const cplx* A, cplx* U, cplx* H) {
    NC_ARG(n >= 1 && 2 * n <= 2048, "polar: the square factor must be at most 1024 x 1024");
    ArenaFrame f(ctx.arena);
    const long long nn = (long long)n * n;
    cplx* S = ctx.arena.alloc_n<cplx>(2 * nn);
    cplx* Q = ctx.arena.alloc_n<cplx>(2 * nn);
    cplx* Xold = ctx.arena.alloc_n<cplx>(nn);
    cplx* D = ctx.arena.alloc_n<cplx>(nn);
    const double alpha = host_norm(ctx, nn, A);   // ||A||_F >= ||A||_2
    if (!(alpha > 0.0) || !std::isfinite(alpha)) return false;
    zcopy(ctx, nn, A, U);
    zscal_host(ctx, nn, cmake(1.0 / alpha, 0.0), U);
    const double eps = 2.220446049250313e-16;
    const double stop = std::cbrt(5.0 * eps);
    double l = 1e-15;
    bool converged = false;
    for (int it = 0; it < 12 && !converged; ++it) {
        double a, b, c;
        qdwh_weights(l, &a, &b, &c);
        stack_kernel<<<grid_of(2 * nn), 256, 0, ctx.stream>>>(n, std::sqrt(c), U, S);
        NC_CHECK_LAUNCH();
        householder_qr(ctx, 2 * n, n, S, Q, nullptr, false);
        zcopy(ctx, nn, U, Xold);
        // U = (b/c) U + (a - b/c)/sqrt(c) Q1 Q2^H
        ZGemmParams p = zgemm_params(OP_N, OP_C, n, n, n, Q, 2 * n, Q + n, 2 * n, U, n);
        p.alpha = cmake((a - b / c) / std::sqrt(c), 0.0);
        p.beta = cmake(b / c, 0.0);
        zgemm(p, ctx);
        l = std::min(1.0, l * (a + b * l * l) / (1.0 + c * l * l));
        diff_kernel<<<grid_of(nn), 256, 0, ctx.stream>>>(nn, U, Xold, D);
        NC_CHECK_LAUNCH();
        ctx.launches += 2;
        const double dn = host_norm(ctx, nn, D);
        if (!std::isfinite(dn)) return false;
        converged = dn <= stop && std::fabs(1.0 - l) <= 10 * eps;
    }
    // H = U^H A, Hermitian part
    zgemm(zgemm_params(OP_C, OP_N, n, n, n, U, n, A, n, D, n), ctx);
    hermitize_kernel<<<grid_of(nn), 256, 0, ctx.stream>>>(n, D, false, H);
    NC_CHECK_LAUNCH();
    // isometry check: ||U^H U - I||_F small (fails for rank-deficient A)
    zgemm(zgemm_params(OP_C, OP_N, n, n, n, U, n, U, n, D, n), ctx);
    minus_identity_kernel<<<grid_of(n), 256, 0, ctx.stream>>>(n, D);
    NC_CHECK_LAUNCH();
    ctx.launches += 2;
    const double orth = host_norm(ctx, nn, D);
    return converged && orth <= 1e-12 * std::sqrt((double)n);
}

void gauge_right_polar(Context& ctx, int bl, int bm, int br, int dl, int dr, const cplx* A, const cplx* B,
                       cplx* normA, cplx* denormB) {
    const int K = bl * dl;
    NC_ARG(K >= bm, "not enough degrees of freedom to normalize");
    NC_ARG(K <= 2048, "polar gauge: bl*dl must be at most 2048");
    ArenaFrame f(ctx.arena);
    cplx* X = ctx.arena.alloc_n<cplx>((size_t)K * bm);
    cplx* Qt = ctx.arena.alloc_n<cplx>((size_t)K * bm);
    cplx* Rt = ctx.arena.alloc_n<cplx>((size_t)bm * bm);
    cplx* Up = ctx.arena.alloc_n<cplx>((size_t)bm * bm);
    cplx* Hp = ctx.arena.alloc_n<cplx>((size_t)bm * bm);
    cplx* G = ctx.arena.alloc_n<cplx>((size_t)K * bm);
    const int p_t[3] = {1, 0, 2};
    permute3(ctx, A, bm, K, 1, p_t, true, X);               // X = M^H  (K x bm)
    householder_qr(ctx, K, bm, X, Qt, Rt, false);           // M^H = Qt Rt
    if (!polar_qdwh(ctx, bm, Rt, Up, Hp)) {
        gauge_right(ctx, bl, bm, br, dl, dr, A, B, normA, denormB);   // rank-deficient: QR gauge
        return;
    }
    zgemm(zgemm_params(OP_N, OP_N, K, bm, bm, Qt, K, Up, bm, G, K), ctx);   // G = Qt Up
    if (B && denormB) {
        // denormB_s = B_s Hp  (the neighbour absorbs H on its left index)
        ZGemmParams p = zgemm_params(OP_N, OP_N, br, bm, bm, B, br, Hp, bm, denormB, br);
        p.batch = dr;
        p.sA0 = (long long)br * bm; p.sB0 = 0; p.sC0 = (long long)br * bm;
        zgemm(p, ctx);
    }
    permute3(ctx, G, K, bm, 1, p_t, true, normA);           // normA = G^H = U V^H
}

void gauge_left_polar(Context& ctx, int bl, int bm, int br, int dl, int dr, const cplx* A, const cplx* B,
                      cplx* denormA, cplx* normB) {
    const int K = br * dr;
    NC_ARG(K >= bm, "not enough degrees of freedom to normalize");
    NC_ARG(K <= 2048, "polar gauge: br*dr must be at most 2048");
    ArenaFrame f(ctx.arena);
    cplx* X = ctx.arena.alloc_n<cplx>((size_t)K * bm);
    cplx* Qt = ctx.arena.alloc_n<cplx>((size_t)K * bm);
    cplx* Rt = ctx.arena.alloc_n<cplx>((size_t)bm * bm);
    cplx* Up = ctx.arena.alloc_n<cplx>((size_t)bm * bm);
    cplx* Hp = ctx.arena.alloc_n<cplx>((size_t)bm * bm);
    cplx* Hc = ctx.arena.alloc_n<cplx>((size_t)bm * bm);
    cplx* G = ctx.arena.alloc_n<cplx>((size_t)K * bm);
    const int p_rs[3] = {0, 2, 1};
    permute3(ctx, B, br, bm, dr, p_rs, true, X);            // X((r,s),m) = conj(B(r,m,s)) = ws^H
    householder_qr(ctx, K, bm, X, Qt, Rt, false);           // ws^H = Qt Rt
    if (!polar_qdwh(ctx, bm, Rt, Up, Hp)) {
        gauge_left(ctx, bl, bm, br, dl, dr, A, B, denormA, normB);    // rank-deficient: QR gauge
        return;
    }
    zgemm(zgemm_params(OP_N, OP_N, K, bm, bm, Qt, K, Up, bm, G, K), ctx);   // G = Qt Up
    if (A && denormA) {
        // denormA = conj(H) A  (as bm x bl*dl)
        hermitize_kernel<<<grid_of((long long)bm * bm), 256, 0, ctx.stream>>>(bm, Hp, true, Hc);
        NC_CHECK_LAUNCH();
        ctx.launches++;
        zgemm(zgemm_params(OP_N, OP_N, bm, bl * dl, bm, Hc, bm, A, bm, denormA, bm), ctx);
    }
    permute3(ctx, G, br, dr, bm, p_rs, true, normB);        // normB(r,m,s) = conj(G((r,s),m))
}

}  // namespace nc
