// The site eigen-solve (replaces ARPACK znaupd/zneupd, core.f95:2049-2609).
//
// A restarted Lanczos method with full (twice-iterated classical
// Gram-Schmidt) reorthogonalisation, run in the full site space on the
// operator P H P, where P projects onto the orthogonal complement of the
// lower levels (the reference works in reduced coordinates of the same
// subspace through zunmqr; both describe the same restricted operator, so the
// eigenpairs coincide).  Everything that touches vectors of length n runs on
// the GPU: the H_eff product (contract.cu), the projector filter, the
// reorthogonalisation (multi-dot / multi-axpy, HBM-bound) and the small
// projected problem (Sturm multisection + inverse iteration for the
// tridiagonal matrix, one warp).  The host only reads back three scalars per
// step to decide convergence.
//
// Convergence follows ARPACK's rule: the Ritz estimate beta_j |s_j| must be
// <= tol * |theta| with tol >= machine epsilon.  `maxit` bounds the number of
// restart cycles (ARPACK's iparam(3)); exhausting it returns -14 as the
// reference does (core.f95:2565-2607).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "nc_common.cuh"
#include "nc_kernels.h"
#include "nc_ritz.cuh"

namespace nc {

namespace {

constexpr int RT = 256;
constexpr int RB = 296;       // 2 x 148 SMs
constexpr int KC = 8;         // vectors per multi-dot chunk
constexpr int MAXM = 128;     // largest multi-dot / multi-axpy width

__global__ void multi_dot_partial(long long n, int k, const cplx* __restrict__ V,
                                  const cplx* __restrict__ w, cplx* __restrict__ part) {
    // part[(chunk*KC + i) * gridDim.x + block]
    __shared__ double sr[KC][RT / 32], si[KC][RT / 32];
    const int c0 = blockIdx.y * KC;
    const int kc = min(KC, k - c0);
    double ar[KC], ai[KC];
#pragma unroll
    for (int i = 0; i < KC; ++i) ar[i] = ai[i] = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        cplx b = w[e];
#pragma unroll
        for (int i = 0; i < KC; ++i) {
            if (i < kc) {
                cplx a = V[(size_t)(c0 + i) * n + e];
                ar[i] += a.x * b.x + a.y * b.y;
                ai[i] += a.x * b.y - a.y * b.x;
            }
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < KC; ++i) {
        double r = ar[i], im = ai[i];
        for (int o = 16; o > 0; o >>= 1) {
            r += __shfl_down_sync(0xffffffffu, r, o);
            im += __shfl_down_sync(0xffffffffu, im, o);
        }
        if (lane == 0) { sr[i][wid] = r; si[i][wid] = im; }
    }
    __syncthreads();
    if (threadIdx.x < KC) {
        int i = threadIdx.x;
        if (i < kc) {
            double r = 0, im = 0;
            for (int q = 0; q < RT / 32; ++q) { r += sr[i][q]; im += si[i][q]; }
            part[(size_t)(c0 + i) * gridDim.x + blockIdx.x] = cmake(r, im);
        }
    }
}

__global__ void multi_dot_final(int nb, const cplx* __restrict__ part, cplx* __restrict__ h) {
    __shared__ double sr[RT], si[RT];
    const cplx* p = part + (size_t)blockIdx.x * nb;
    double r = 0, im = 0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) { r += p[i].x; im += p[i].y; }
    sr[threadIdx.x] = r; si[threadIdx.x] = im;
    __syncthreads();
    for (int s = RT / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) { sr[threadIdx.x] += sr[threadIdx.x + s]; si[threadIdx.x] += si[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) h[blockIdx.x] = cmake(sr[0], si[0]);
}

__global__ void multi_axpy_kernel(long long n, int k, const cplx* __restrict__ V,
                                  const cplx* __restrict__ h, double sign, cplx* __restrict__ w) {
    __shared__ cplx hs[MAXM];
    for (int i = threadIdx.x; i < k; i += blockDim.x) hs[i] = cscale(h[i], sign);
    __syncthreads();
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        cplx acc = w[e];
        for (int i = 0; i < k; ++i) acc = cadd(acc, cmul(hs[i], V[(size_t)i * n + e]));
        w[e] = acc;
    }
}

// One classical Gram-Schmidt pass against V_0..V_{k-1} in one launch:
// out = w - sum_i hsub_i V_i (hsub may be null: out is not written), then
// h = V^H out over the updated vector.  Blocks (x: elements, y: chunks of KC
// vectors) store partial sums; the last block to finish adds them in block
// order (fixed, so the result does not depend on block timing).  Every chunk
// forms the updated vector itself; chunk 0 writes it.
__global__ void __launch_bounds__(RT) cgs_pass_kernel(long long n, int k, const cplx* __restrict__ V,
                                                      const cplx* __restrict__ w, const cplx* __restrict__ hsub,
                                                      cplx* __restrict__ out, cplx* __restrict__ part,
                                                      unsigned* __restrict__ counter, cplx* __restrict__ h) {
    __shared__ cplx hs[MAXM];
    __shared__ double sr[KC][RT / 32], si[KC][RT / 32];
    __shared__ bool last;
    if (hsub)
        for (int i = threadIdx.x; i < k; i += blockDim.x) hs[i] = hsub[i];
    __syncthreads();
    const int c0 = blockIdx.y * KC;
    const int kc = min(KC, k - c0);
    double ar[KC], ai[KC];
#pragma unroll
    for (int i = 0; i < KC; ++i) ar[i] = ai[i] = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        cplx b = w[e];
        if (hsub) {
            for (int i = 0; i < k; ++i) b = csub(b, cmul(hs[i], V[(size_t)i * n + e]));
            if (blockIdx.y == 0) out[e] = b;
        }
#pragma unroll
        for (int i = 0; i < KC; ++i) {
            if (i < kc) {
                const cplx a = V[(size_t)(c0 + i) * n + e];
                ar[i] += a.x * b.x + a.y * b.y;
                ai[i] += a.x * b.y - a.y * b.x;
            }
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < KC; ++i) {
        double r = ar[i], im = ai[i];
        for (int o = 16; o > 0; o >>= 1) {
            r += __shfl_down_sync(0xffffffffu, r, o);
            im += __shfl_down_sync(0xffffffffu, im, o);
        }
        if (lane == 0) { sr[i][wid] = r; si[i][wid] = im; }
    }
    __syncthreads();
    const unsigned nblocks = gridDim.x * gridDim.y;
    if (threadIdx.x < KC) {
        const int i = threadIdx.x;
        if (i < kc) {
            double r = 0, im = 0;
            for (int q = 0; q < RT / 32; ++q) { r += sr[i][q]; im += si[i][q]; }
            part[(size_t)(c0 + i) * gridDim.x + blockIdx.x] = cmake(r, im);
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == nblocks - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        double r = 0, im = 0;
        for (unsigned b = 0; b < gridDim.x; ++b) {
            const cplx p = __ldcg(&part[(size_t)i * gridDim.x + b]);
            r += p.x; im += p.y;
        }
        h[i] = cmake(r, im);
    }
    if (threadIdx.x == 0) *counter = 0;
}

// out = w - sum_i hsub_i V_i and nrm2 = |out|^2 in one launch (last-block
// reduction as in cgs_pass_kernel).
__global__ void __launch_bounds__(RT) axpy_norm_kernel(long long n, int k, const cplx* __restrict__ V,
                                                       const cplx* __restrict__ w, const cplx* __restrict__ hsub,
                                                       cplx* __restrict__ out, cplx* __restrict__ part,
                                                       unsigned* __restrict__ counter, cplx* __restrict__ nrm2) {
    __shared__ cplx hs[MAXM];
    __shared__ double s[RT];
    __shared__ bool last;
    for (int i = threadIdx.x; i < k; i += blockDim.x) hs[i] = hsub[i];
    __syncthreads();
    double acc = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        cplx b = w[e];
        for (int i = 0; i < k; ++i) b = csub(b, cmul(hs[i], V[(size_t)i * n + e]));
        out[e] = b;
        acc += b.x * b.x + b.y * b.y;
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int st = RT / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) s[threadIdx.x] += s[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[blockIdx.x] = cmake(s[0], 0);
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    acc = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) acc += __ldcg(&part[i]).x;
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int st = RT / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) s[threadIdx.x] += s[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        nrm2[0] = cmake(s[0], 0);
        *counter = 0;
    }
}

__global__ void random_kernel(long long n, uint64_t seed, cplx* __restrict__ x) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        // splitmix64 of (seed, index) -> two uniforms in (-0.5, 0.5]
        uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(2 * e + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        double u1 = (double)(z >> 11) * (1.0 / 9007199254740992.0);
        uint64_t y = z + 0x9E3779B97F4A7C15ull;
        y = (y ^ (y >> 30)) * 0xBF58476D1CE4E5B9ull;
        y = (y ^ (y >> 27)) * 0x94D049BB133111EBull;
        y ^= y >> 31;
        double u2 = (double)(y >> 11) * (1.0 / 9007199254740992.0);
        x[e] = cmake(0.5 - u1, 0.5 - u2);
    }
}

// ---- projected (Rayleigh-Ritz) problem (nc_ritz.cuh) ---------------------------
constexpr int MAXT = 32;   // largest projected problem
constexpr int RITZ_STATE = 2 * MAXT * MAXT;

struct RitzOut {
    double theta, res, beta, tnorm;
    int sweeps, pad;
};

// after a thick restart: A = diag(theta_0 .. theta_{k-1}), Z = I
__global__ void restart_t_kernel(int k, const double* __restrict__ theta, double* __restrict__ state) {
    ritz_restart_state<MAXT>(k, theta, state);
}

// Adds column m-1 of T to the kept decomposition and diagonalises (one warp);
// theta[] and S (m x m complex, column-major) receive the ordered Ritz pairs,
// out the wanted pair's value and Ritz estimate.
__global__ void ritz_kernel(int m, double* __restrict__ state, const cplx* __restrict__ h1,
                            const cplx* __restrict__ h2, const cplx* __restrict__ nrm2, int which,
                            RitzOut* __restrict__ out, cplx* __restrict__ S, double* __restrict__ theta) {
    __shared__ RitzSmem<MAXT> w;
    const RitzResult r = ritz_update_warp<MAXT, true>(w, m, state, h1, h2, nrm2[0].x, which, S, m, theta);
    if (threadIdx.x == 0) {
        out->theta = r.theta;
        out->res = r.res;
        out->beta = r.beta;
        out->tnorm = r.tnorm;
        out->sweeps = r.sweeps;
    }
}


__global__ void scale_by_inv_sqrt(long long n, const cplx* __restrict__ nrm2, const cplx* __restrict__ in,
                                  cplx* __restrict__ out) {
    double f = 1.0 / sqrt(nrm2[0].x);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x)
        out[e] = cscale(in[e], f);
}

// Dense Hermitian eigen-solve by cyclic complex Jacobi, one thread (n <= 8).
__global__ void small_herm_eig(int n, const cplx* __restrict__ Ain, int which, double* ev,
                               cplx* __restrict__ vec) {
    if (threadIdx.x != 0) return;
    cplx A[8][8], V[8][8];
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            // Hermitian part (the matrix is Hermitian up to rounding)
            cplx x = Ain[i + n * j], y = Ain[j + n * i];
            A[i][j] = cmake(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
            V[i][j] = cmake(i == j ? 1.0 : 0.0, 0.0);
        }
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0, diag = 0;
        for (int i = 0; i < n; ++i) {
            diag += A[i][i].x * A[i][i].x;
            for (int j = i + 1; j < n; ++j) off += cabs2(A[i][j]);
        }
        if (off <= 1e-34 * (diag + 1e-300)) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                double r = sqrt(cabs2(A[p][q]));
                if (r < 1e-300) continue;
                cplx ph = cmake(A[p][q].x / r, A[p][q].y / r);   // e^{i phi}
                cplx phc = cconj(ph);                              // e^{-i phi}
                double app = A[p][p].x, aqq = A[q][q].x;
                double tau = (aqq - app) / (2 * r);
                double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1 + tau * tau));
                double c = 1 / sqrt(1 + t * t), s = t * c;
                // G = D R: columns (c, -s e^{-i phi}) and (s, c e^{-i phi})
                cplx g00 = cmake(c, 0), g01 = cmake(s, 0);
                cplx g10 = cscale(phc, -s), g11 = cscale(phc, c);
                for (int k = 0; k < n; ++k) {
                    cplx akp = A[k][p], akq = A[k][q];
                    A[k][p] = cadd(cmul(akp, g00), cmul(akq, g10));
                    A[k][q] = cadd(cmul(akp, g01), cmul(akq, g11));
                    cplx vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = cadd(cmul(vkp, g00), cmul(vkq, g10));
                    V[k][q] = cadd(cmul(vkp, g01), cmul(vkq, g11));
                }
                for (int k = 0; k < n; ++k) {
                    cplx apk = A[p][k], aqk = A[q][k];
                    A[p][k] = cadd(cmul(cconj(g00), apk), cmul(cconj(g10), aqk));
                    A[q][k] = cadd(cmul(cconj(g01), apk), cmul(cconj(g11), aqk));
                }
                A[p][q] = cmake(0, 0);
                A[q][p] = cmake(0, 0);
            }
    }
    int best = 0;
    for (int i = 1; i < n; ++i) {
        double a = A[i][i].x, b = A[best][best].x;
        bool better = (which == WHICH_SR) ? (a < b) : (which == WHICH_LR) ? (a > b) : (fabs(a) > fabs(b));
        if (better) best = i;
    }
    ev[0] = A[best][best].x;
    for (int i = 0; i < n; ++i) vec[i] = V[i][best];
}

unsigned g1(long long n) {
    return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 16));
}

}  // namespace

int parse_which(const char* which) {
    if (which[0] == 'S' && which[1] == 'R') return WHICH_SR;
    if (which[0] == 'L' && which[1] == 'R') return WHICH_LR;
    if (which[0] == 'L' && which[1] == 'M') return WHICH_LM;
    throw Error(NC_ERR_ARG, std::string("invalid eigenvalue request: ") + which[0] + which[1]);
}

void zrandom(Context& ctx, long long n, uint64_t seed, cplx* x) {
    random_kernel<<<g1(n), 256, 0, ctx.stream>>>(n, seed, x);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

void multi_dotc(Context& ctx, long long n, int k, const cplx* V, const cplx* w, cplx* h) {
    if (k <= 0) return;
    NC_ARG(k <= MAXM, "multi_dotc: too many vectors");
    ArenaFrame f(ctx.arena);
    int nb = (int)std::min<long long>(RB, std::max<long long>(1, (n + RT - 1) / RT));
    cplx* part = ctx.arena.alloc_n<cplx>((size_t)nb * ((k + KC - 1) / KC) * KC);
    dim3 grid(nb, (k + KC - 1) / KC);
    multi_dot_partial<<<grid, RT, 0, ctx.stream>>>(n, k, V, w, part);
    NC_CHECK_LAUNCH();
    multi_dot_final<<<k, RT, 0, ctx.stream>>>(nb, part, h);
    NC_CHECK_LAUNCH();
    ctx.launches += 2;
}

void multi_axpy(Context& ctx, long long n, int k, const cplx* V, const cplx* h, double sign, cplx* w) {
    if (k <= 0) return;
    NC_ARG(k <= MAXM, "multi_axpy: too many vectors");
    multi_axpy_kernel<<<g1(n), 256, 0, ctx.stream>>>(n, k, V, h, sign, w);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

namespace {

// P filter through an explicit orthonormal basis U (n x r) of the removed space.
struct Filter {
    const cplx* U = nullptr;
    int r = 0;
    cplx* h = nullptr;
    void apply(Context& ctx, long long n, cplx* w) const {
        if (r == 0) return;
        multi_dotc(ctx, n, r, U, w, h);
        multi_axpy(ctx, n, r, U, h, -1.0, w);
    }
};

}  // namespace

int optimize_site(Context& ctx, int bl, int br, const MpoSite& op, const cplx* L, const cplx* R,
                  const DevProjector& P, int which, double tol, int maxit, const cplx* guess,
                  cplx* result, double* eigenvalue, double* normal, EigenStats* stats, const MixedHeff* mixed) {
    const long long n = (long long)br * bl * op.d;
    const long long orth_dim = P.nproj ? P.orth_dim : n;
    EigenStats st;
    *eigenvalue = 0;
    *normal = 0;
    // guards of core.f95:1954-1983
    if (orth_dim > n) return 5;
    double overlap = (P.nproj > 0) ? overlap_with_projectors(ctx, P, guess) : 0.0;
    if (orth_dim <= 0) return 10;
    if (orth_dim < n && overlap > 1e-7) return 11;

    ArenaFrame frame(ctx.arena);
    cplx* ws = mixed ? nullptr : ctx.arena.alloc_n<cplx>(heff_workspace_elems(bl, br, op));
    // y = H_eff x: FP64, or the precision form when `mixed` is given
    auto apply = [&](const cplx* x, cplx* y) {
        if (mixed) heff_apply_mixed(ctx, *mixed, x, y);
        else heff_apply(ctx, bl, br, op, L, R, x, y, ws);
    };
    Filter filt;
    if (P.nproj > 0 && orth_dim < n) {
        filt.r = (int)(n - orth_dim);
        cplx* U = ctx.arena.alloc_n<cplx>((size_t)filt.r * n);
        removed_basis(ctx, P, U);
        filt.U = U;
        filt.h = ctx.arena.alloc_n<cplx>(filt.r);
    }

    if (orth_dim <= 4) {
        // strategy 1 (core.f95:2049-2129): dense eigen-solve in the orthogonal space
        const int k = (int)orth_dim;
        cplx* B = ctx.arena.alloc_n<cplx>((size_t)k * n);
        cplx* HB_ = ctx.arena.alloc_n<cplx>((size_t)k * n);
        cplx* M = ctx.arena.alloc_n<cplx>((size_t)k * k);
        for (int q = 0; q < k; ++q) {
            unproject_unit(ctx, P, q, B + (size_t)q * n);
            apply(B + (size_t)q * n, HB_ + (size_t)q * n);
        }
        for (int q = 0; q < k; ++q) multi_dotc(ctx, n, k, B, HB_ + (size_t)q * n, M + (size_t)q * k);
        double* ev = ctx.arena.alloc_n<double>(1);
        cplx* c = ctx.arena.alloc_n<cplx>(k);
        small_herm_eig<<<1, 1, 0, ctx.stream>>>(k, M, which, ev, c);
        NC_CHECK_LAUNCH();
        ctx.launches++;
        zfill(ctx, n, cmake(0, 0), result);
        multi_axpy(ctx, n, k, B, c, 1.0, result);
        read_scalars(ctx, ev, sizeof(double), eigenvalue);
        cplx* nr = ctx.arena.alloc_n<cplx>(1);
        znrm2sq(ctx, n, result, nr);
        *normal = std::sqrt(read_scalar(ctx, nr).x);
        st.matvecs = k;
        if (stats) *stats = st;
        return 0;
    }

    // ---- thick-restart Lanczos (Wu & Simon 2000) with full reorthogonalisation
    const int m_max = (int)std::min<long long>(std::min(MAXT, ctx.krylov_dim), orth_dim);
    const int keep = std::max(1, std::min(std::max(4, m_max / 3), m_max - 2));
    cplx* V = ctx.arena.alloc_n<cplx>((size_t)(m_max + 1) * n);
    cplx* w = ctx.arena.alloc_n<cplx>(n);
    cplx* Y = ctx.arena.alloc_n<cplx>((size_t)keep * n);
    cplx* h1 = ctx.arena.alloc_n<cplx>(m_max + 1);
    cplx* h2 = ctx.arena.alloc_n<cplx>(m_max + 1);
    cplx* nr = ctx.arena.alloc_n<cplx>(1);
    double* T = ctx.arena.alloc_n<double>(RITZ_STATE);   // kept eigen-decomposition of T
    double* theta = ctx.arena.alloc_n<double>(MAXT);
    cplx* S = ctx.arena.alloc_n<cplx>(MAXT * MAXT);
    RitzOut* ro = ctx.arena.alloc_n<RitzOut>(1);

    const double eps = 2.220446049250313e-16;
    const double tol_eff = std::max(tol, eps);
    const double eps23 = std::pow(eps, 2.0 / 3.0);
    uint64_t seed = 0x5EEDull + (uint64_t)n * 7919ull;

    // CGS2 of v against V_0..V_{k-1}, then the P filter: h1 = V^H v,
    // h2 = V^H (v - V h1), v <- v - V h1 - V h2, nr = |v|^2, in three launches
    cplx* vtmp = ctx.arena.alloc_n<cplx>(n);
    const int cgs_nb = (int)std::min<long long>(RB, std::max<long long>(1, (n + RT - 1) / RT));
    cplx* cgs_part = ctx.arena.alloc_n<cplx>((size_t)cgs_nb * (MAXT / KC + 1) * KC);
    unsigned* counter = ctx.reduction_counter();
    auto orthogonalise = [&](cplx* v, int k) {
        NC_ARG(k <= MAXT + 1, "Krylov basis too large");
        const dim3 grid(cgs_nb, (k + KC - 1) / KC);
        cgs_pass_kernel<<<grid, RT, 0, ctx.stream>>>(n, k, V, v, nullptr, nullptr, cgs_part, counter, h1);
        NC_CHECK_LAUNCH();
        cgs_pass_kernel<<<grid, RT, 0, ctx.stream>>>(n, k, V, v, h1, vtmp, cgs_part, counter, h2);
        NC_CHECK_LAUNCH();
        axpy_norm_kernel<<<cgs_nb, RT, 0, ctx.stream>>>(n, k, V, vtmp, h2, v, cgs_part, counter, nr);
        NC_CHECK_LAUNCH();
        ctx.launches += 3;
        if (filt.r > 0) {
            filt.apply(ctx, n, v);
            znrm2sq(ctx, n, v, nr);
        }
    };
    // starting vector: the projected guess (core.f95:2454), or random if it vanishes
    zcopy(ctx, n, guess, V);
    filt.apply(ctx, n, V);
    znrm2sq(ctx, n, V, nr);
    if (!(read_scalar(ctx, nr).x > 1e-280)) {
        zrandom(ctx, n, seed++, V);
        filt.apply(ctx, n, V);
        znrm2sq(ctx, n, V, nr);
    }
    scale_by_inv_sqrt<<<g1(n), 256, 0, ctx.stream>>>(n, nr, V, V);
    NC_CHECK_LAUNCH();
    restart_t_kernel<<<1, 256, 0, ctx.stream>>>(0, theta, T);
    NC_CHECK_LAUNCH();
    ctx.launches += 2;

    int restarts = 0;
    int j = 0;
    for (;;) {
        cplx* vj = V + (size_t)j * n;
        apply(vj, w);
        filt.apply(ctx, n, w);
        ++st.matvecs;
        orthogonalise(w, j + 1);
        ritz_kernel<<<1, 32, 0, ctx.stream>>>(j + 1, T, h1, h2, nr, which, ro, S, theta);
        NC_CHECK_LAUNCH();
        ctx.launches++;
        RitzOut rr;
        read_scalars(ctx, ro, sizeof(RitzOut), &rr);
        const double anorm = std::max(std::fabs(rr.theta), eps23);
        if (rr.res <= tol_eff * anorm || j + 1 >= orth_dim) {
            // Ritz vector x = V s_0, cleaned of projector-space rounding and normalised
            zfill(ctx, n, cmake(0, 0), result);
            multi_axpy(ctx, n, j + 1, V, S, 1.0, result);
            filt.apply(ctx, n, result);
            znrm2sq(ctx, n, result, nr);
            scale_by_inv_sqrt<<<g1(n), 256, 0, ctx.stream>>>(n, nr, result, result);
            NC_CHECK_LAUNCH();
            ctx.launches++;
            *eigenvalue = rr.theta;
            znrm2sq(ctx, n, result, nr);
            *normal = std::sqrt(read_scalar(ctx, nr).x);
            st.restarts = restarts;
            if (stats) *stats = st;
            return 0;
        }
        if (j + 1 == m_max) {
            // thick restart: keep the `keep` wanted Ritz vectors, continue from the residual
            if (++restarts >= maxit) {
                st.restarts = restarts;
                if (stats) *stats = st;
                return -14;
            }
            zgemm(zgemm_params(OP_N, OP_N, (int)std::min<long long>(n, 1LL << 30), keep, j + 1, V, n, S, j + 1, Y, n),
                  ctx);
            zcopy(ctx, (long long)keep * n, Y, V);
            scale_by_inv_sqrt<<<g1(n), 256, 0, ctx.stream>>>(n, nr, w, V + (size_t)keep * n);
            NC_CHECK_LAUNCH();
            restart_t_kernel<<<1, 256, 0, ctx.stream>>>(keep, theta, T);
            NC_CHECK_LAUNCH();
            ctx.launches += 2;
            j = keep;
            continue;
        }
        cplx* vn = V + (size_t)(j + 1) * n;
        if (rr.beta <= 1e3 * eps * std::max(rr.tnorm, 1e-300)) {
            // invariant subspace: continue with a fresh random direction
            zrandom(ctx, n, seed++, vn);
            filt.apply(ctx, n, vn);
            orthogonalise(vn, j + 1);
            scale_by_inv_sqrt<<<g1(n), 256, 0, ctx.stream>>>(n, nr, vn, vn);
        } else {
            scale_by_inv_sqrt<<<g1(n), 256, 0, ctx.stream>>>(n, nr, w, vn);
        }
        NC_CHECK_LAUNCH();
        ctx.launches++;
        ++j;
    }
}

}  // namespace nc
