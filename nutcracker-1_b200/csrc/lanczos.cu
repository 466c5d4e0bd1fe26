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

namespace nc {

namespace {

constexpr int RT = 256;
constexpr int RB = 296;       // 2 x 148 SMs
constexpr int KC = 8;         // vectors per multi-dot chunk
constexpr int MAXM = 128;     // largest Krylov basis

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

// Sturm count: number of eigenvalues of the symmetric tridiagonal (a, b) below x.
__device__ int sturm_count(int m, const double* a, const double* b2, double x, double pivmin) {
    int c = 0;
    double q = a[0] - x;
    if (fabs(q) <= pivmin) q = -pivmin;
    if (q < 0) ++c;
    for (int i = 1; i < m; ++i) {
        q = a[i] - x - b2[i - 1] / q;
        if (fabs(q) <= pivmin) q = -pivmin;
        if (q < 0) ++c;
    }
    return c;
}

// k-th smallest eigenvalue (0-based) by 33-way multisection in one warp.
__device__ double kth_eigenvalue(int m, const double* a, const double* b2, int k, double lo, double hi,
                                 double pivmin) {
    const int lane = threadIdx.x & 31;
    for (int it = 0; it < 64; ++it) {
        double width = hi - lo;
        if (width <= 2.2e-16 * (fabs(lo) + fabs(hi)) + pivmin) break;
        double x = lo + width * (double)(lane + 1) / 33.0;
        int c = sturm_count(m, a, b2, x, pivmin);
        unsigned mask = __ballot_sync(0xffffffffu, c >= k + 1);
        int f = mask ? (__ffs(mask) - 1) : 32;
        double xf = __shfl_sync(0xffffffffu, x, f < 32 ? f : 0);
        double xl = __shfl_sync(0xffffffffu, x, f > 0 ? f - 1 : 0);
        double nhi = (f < 32) ? xf : hi;
        double nlo = (f > 0) ? xl : lo;
        if (nhi == hi && nlo == lo) break;
        hi = nhi;
        lo = nlo;
    }
    return 0.5 * (lo + hi);
}

// Inverse iteration for the eigenvector of T at theta (dgttrf/dgtts2-style
// elimination with partial pivoting; zero pivots replaced by eps*||T||).
__device__ void tridiag_eigvec(int m, const double* a, const double* b, double theta, double tnorm,
                               double* s) {
    double dl[MAXM], dd[MAXM], du[MAXM], du2[MAXM];
    int piv[MAXM];
    const double tiny = 2.2e-16 * (tnorm > 0 ? tnorm : 1.0);
    for (int i = 0; i < m; ++i) {
        dd[i] = a[i] - theta;
        if (i < m - 1) { dl[i] = b[i]; du[i] = b[i]; }
        du2[i] = 0;
        piv[i] = i;
    }
    for (int i = 0; i < m - 1; ++i) {
        if (fabs(dd[i]) >= fabs(dl[i])) {
            if (dd[i] == 0) dd[i] = tiny;
            double f = dl[i] / dd[i];
            dl[i] = f;
            dd[i + 1] -= f * du[i];
            du2[i] = 0;
        } else {
            double f = dd[i] / dl[i];
            dd[i] = dl[i];
            dl[i] = f;
            double t = du[i];
            du[i] = dd[i + 1];
            dd[i + 1] = t - f * dd[i + 1];
            if (i < m - 2) {
                du2[i] = du[i + 1];
                du[i + 1] = -f * du[i + 1];
            }
            piv[i] = i + 1;
        }
    }
    if (dd[m - 1] == 0) dd[m - 1] = tiny;
    for (int i = 0; i < m; ++i) s[i] = 1.0 / sqrt((double)m) * (1.0 + 0.01 * (i % 7));
    for (int it = 0; it < 3; ++it) {
        // forward: L
        for (int i = 0; i < m - 1; ++i) {
            if (piv[i] == i) {
                s[i + 1] -= dl[i] * s[i];
            } else {
                double t = s[i];
                s[i] = s[i + 1];
                s[i + 1] = t - dl[i] * s[i];
            }
        }
        // backward: U
        s[m - 1] /= dd[m - 1];
        if (m > 1) s[m - 2] = (s[m - 2] - du[m - 2] * s[m - 1]) / dd[m - 2];
        for (int i = m - 3; i >= 0; --i) s[i] = (s[i] - du[i] * s[i + 1] - du2[i] * s[i + 2]) / dd[i];
        double nr = 0;
        for (int i = 0; i < m; ++i) nr += s[i] * s[i];
        nr = sqrt(nr);
        for (int i = 0; i < m; ++i) s[i] /= nr;
    }
    // fix the sign for determinism: largest-magnitude component positive
    int imax = 0;
    for (int i = 1; i < m; ++i) if (fabs(s[i]) > fabs(s[imax])) imax = i;
    if (s[imax] < 0) for (int i = 0; i < m; ++i) s[i] = -s[i];
}

struct TriOut {
    double theta, s_last, beta, tnorm;
};

// One warp: finalise alpha_j, beta_j from the CGS coefficients, solve the
// (j+1)-dimensional tridiagonal problem for the wanted Ritz pair.
__global__ void lanczos_tridiag(int j, double* alpha, double* beta, const cplx* __restrict__ h1,
                                const cplx* __restrict__ h2, const cplx* __restrict__ nrm2,
                                int which, TriOut* out, cplx* __restrict__ s_out) {
    __shared__ double a[MAXM], b[MAXM], b2[MAXM];
    const int lane = threadIdx.x;
    if (lane == 0) {
        alpha[j] = h1[j].x + h2[j].x;
        beta[j] = sqrt(nrm2[0].x);
    }
    __syncwarp();
    const int m = j + 1;
    for (int i = lane; i < m; i += 32) {
        a[i] = alpha[i];
        b[i] = (i < m - 1) ? beta[i] : 0.0;
        b2[i] = b[i] * b[i];
    }
    __syncwarp();
    double lo = 1e300, hi = -1e300, tn = 0;
    for (int i = 0; i < m; ++i) {
        double r = (i > 0 ? fabs(b[i - 1]) : 0) + (i < m - 1 ? fabs(b[i]) : 0);
        lo = fmin(lo, a[i] - r);
        hi = fmax(hi, a[i] + r);
        tn = fmax(tn, fabs(a[i]) + r);
    }
    double pad = 2.2e-16 * tn * 4 + 1e-300;
    lo -= pad;
    hi += pad;
    double pivmin = 1e-300 + 2.2e-16 * 2.2e-16 * tn * tn;
    double th;
    if (which == WHICH_SR) {
        th = kth_eigenvalue(m, a, b2, 0, lo, hi, pivmin);
    } else if (which == WHICH_LR) {
        th = kth_eigenvalue(m, a, b2, m - 1, lo, hi, pivmin);
    } else {
        double t0 = kth_eigenvalue(m, a, b2, 0, lo, hi, pivmin);
        double t1 = kth_eigenvalue(m, a, b2, m - 1, lo, hi, pivmin);
        th = (fabs(t1) > fabs(t0)) ? t1 : t0;  // core.f95:446-456 picks the larger magnitude
    }
    if (lane == 0) {
        double s[MAXM];
        tridiag_eigvec(m, a, b, th, tn, s);
        for (int i = 0; i < m; ++i) s_out[i] = cmake(s[i], 0);
        out->theta = th;
        out->s_last = s[m - 1];
        out->beta = beta[j];
        out->tnorm = tn;
    }
}

__global__ void set_beta_zero(double* beta, int j) { beta[j] = 0.0; }

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
                  cplx* result, double* eigenvalue, double* normal, EigenStats* stats) {
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
    cplx* ws = ctx.arena.alloc_n<cplx>(heff_workspace_elems(bl, br, op));
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
            heff_apply(ctx, bl, br, op, L, R, B + (size_t)q * n, HB_ + (size_t)q * n, ws);
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

    const int m_max = (int)std::min<long long>(std::min(MAXM, ctx.krylov_dim), orth_dim);
    cplx* V = ctx.arena.alloc_n<cplx>((size_t)(m_max + 1) * n);
    cplx* w = ctx.arena.alloc_n<cplx>(n);
    cplx* h1 = ctx.arena.alloc_n<cplx>(m_max + 1);
    cplx* h2 = ctx.arena.alloc_n<cplx>(m_max + 1);
    cplx* nr = ctx.arena.alloc_n<cplx>(1);
    double* alpha = ctx.arena.alloc_n<double>(m_max + 1);
    double* beta = ctx.arena.alloc_n<double>(m_max + 1);
    cplx* s = ctx.arena.alloc_n<cplx>(m_max + 1);
    TriOut* tri = ctx.arena.alloc_n<TriOut>(1);

    const double eps = 2.220446049250313e-16;
    const double tol_eff = std::max(tol, eps);
    const double eps23 = std::pow(eps, 2.0 / 3.0);
    uint64_t seed = 0x5EEDull + (uint64_t)n * 7919ull;

    // starting vector: the projected guess (core.f95:2454), or random if it vanishes
    auto start_vector = [&](cplx* v, const cplx* src) {
        if (src) zcopy(ctx, n, src, v);
        else zrandom(ctx, n, seed++, v);
        filt.apply(ctx, n, v);
        znrm2sq(ctx, n, v, nr);
        return read_scalar(ctx, nr).x;
    };
    double g2 = start_vector(V, guess);
    if (!(g2 > 1e-280)) g2 = start_vector(V, nullptr);
    scale_by_inv_sqrt<<<g1(n), 256, 0, ctx.stream>>>(n, nr, V, V);
    NC_CHECK_LAUNCH();
    ctx.launches++;

    int restarts = 0;
    for (;;) {
        int jlast = -1;
        bool converged = false;
        TriOut T{};
        for (int j = 0; j < m_max; ++j) {
            cplx* vj = V + (size_t)j * n;
            heff_apply(ctx, bl, br, op, L, R, vj, w, ws);
            filt.apply(ctx, n, w);
            ++st.matvecs;
            // twice-iterated classical Gram-Schmidt against V_0..V_j
            multi_dotc(ctx, n, j + 1, V, w, h1);
            multi_axpy(ctx, n, j + 1, V, h1, -1.0, w);
            multi_dotc(ctx, n, j + 1, V, w, h2);
            multi_axpy(ctx, n, j + 1, V, h2, -1.0, w);
            znrm2sq(ctx, n, w, nr);
            lanczos_tridiag<<<1, 32, 0, ctx.stream>>>(j, alpha, beta, h1, h2, nr, which, tri, s);
            NC_CHECK_LAUNCH();
            ctx.launches++;
            read_scalars(ctx, tri, sizeof(TriOut), &T);
            jlast = j;
            const double res = std::fabs(T.beta * T.s_last);
            const double anorm = std::max(std::fabs(T.theta), eps23);
            if (res <= tol_eff * anorm || j + 1 >= orth_dim) {
                converged = true;
                break;
            }
            if (j + 1 == m_max) break;
            cplx* vn = V + (size_t)(j + 1) * n;
            if (T.beta <= 1e3 * eps * std::max(T.tnorm, 1e-300)) {
                // invariant subspace: continue with a fresh random direction
                start_vector(vn, nullptr);
                multi_dotc(ctx, n, j + 1, V, vn, h1);
                multi_axpy(ctx, n, j + 1, V, h1, -1.0, vn);
                multi_dotc(ctx, n, j + 1, V, vn, h1);
                multi_axpy(ctx, n, j + 1, V, h1, -1.0, vn);
                znrm2sq(ctx, n, vn, nr);
                scale_by_inv_sqrt<<<g1(n), 256, 0, ctx.stream>>>(n, nr, vn, vn);
                set_beta_zero<<<1, 1, 0, ctx.stream>>>(beta, j);
                NC_CHECK_LAUNCH();
                ctx.launches += 2;
            } else {
                scale_by_inv_sqrt<<<g1(n), 256, 0, ctx.stream>>>(n, nr, w, vn);
                NC_CHECK_LAUNCH();
                ctx.launches++;
            }
        }
        // Ritz vector x = V s (normalised)
        zfill(ctx, n, cmake(0, 0), result);
        multi_axpy(ctx, n, jlast + 1, V, s, 1.0, result);
        znrm2sq(ctx, n, result, nr);
        if (converged) {
            scale_by_inv_sqrt<<<g1(n), 256, 0, ctx.stream>>>(n, nr, result, result);
            NC_CHECK_LAUNCH();
            ctx.launches++;
            *eigenvalue = T.theta;
            znrm2sq(ctx, n, result, nr);
            *normal = std::sqrt(read_scalar(ctx, nr).x);
            st.restarts = restarts;
            if (stats) *stats = st;
            return 0;
        }
        ++restarts;
        if (restarts >= maxit) {
            st.restarts = restarts;
            if (stats) *stats = st;
            return -14;
        }
        scale_by_inv_sqrt<<<g1(n), 256, 0, ctx.stream>>>(n, nr, result, V);
        NC_CHECK_LAUNCH();
        ctx.launches++;
    }
}

}  // namespace nc
