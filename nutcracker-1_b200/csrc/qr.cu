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
// I - V T V^H).  Each block is factorised by one thread-block cluster of up
// to 16 CTAs with the block held in registers (mp <= 2048 rows); devices
// that cannot co-schedule such a cluster use inner panels of JB=4 columns
// (one CTA each) and a per-column update kernel.  Q is formed explicitly by
// backward accumulation of the block reflectors (zungqr order).
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include <cooperative_groups.h>

#include "nc_common.cuh"
#include "nc_kernels.h"

namespace nc {

namespace cg = cooperative_groups;

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

// Compact-WY T (nb x nb, forward/columnwise: H_0 H_1 ... = I - V T V^H) from
// the strict upper part of G = V^H V and tau, by recursive doubling: with T
// known on two adjacent diagonal blocks a, b of size s,
//   T(a,b) = -T(a,a) G(a,b) T(b,b)
// (the block form of the zlarft recurrence; Puglisi 1992, Joffrain et al.
// 2006), so six levels of small block products build the 64 x 64 T.  One
// CTA, T, G and the level's products in shared memory.
constexpr int BT_T = 1024;
constexpr size_t BT_SMEM = sizeof(cplx) * ((size_t)2 * NB * (NB + 1) + NB * NB / 2);

// G is either a matrix (ld nb) or, with nparts > 0, the sum of nparts NB x NB
// partial Gram blocks (ld NB, stride NB*NB) added in index order.
__global__ void __launch_bounds__(BT_T) build_t_kernel(int nb, const cplx* __restrict__ G, int nparts,
                                                      const cplx* __restrict__ tau, cplx* __restrict__ T,
                                                      int ldt) {
    extern __shared__ __align__(16) unsigned char bt_smem[];
    cplx* Ts = reinterpret_cast<cplx*>(bt_smem);   // [NB][NB+1]
    cplx* Gs = Ts + NB * (NB + 1);                   // [NB][NB+1], strict upper part
    cplx* Xs = Gs + NB * (NB + 1);                   // one level's G(a,b) T(b,b) blocks
    const int tid = threadIdx.x;
    for (int e = tid; e < NB * NB; e += BT_T) {
        const int i = e % NB, j = e / NB;
        cplx g = cmake(0, 0);
        if (i < j && j < nb) {
            if (nparts > 0) {
                double r0 = 0, i0 = 0, r1 = 0, i1 = 0;   // two interleaved chains, fixed order
                int c = 0;
                for (; c + 1 < nparts; c += 2) {
                    const cplx a = G[(size_t)c * NB * NB + i + NB * j];
                    const cplx b = G[(size_t)(c + 1) * NB * NB + i + NB * j];
                    r0 += a.x; i0 += a.y; r1 += b.x; i1 += b.y;
                }
                if (c < nparts) {
                    const cplx a = G[(size_t)c * NB * NB + i + NB * j];
                    r0 += a.x; i0 += a.y;
                }
                g = cmake(r0 + r1, i0 + i1);
            } else {
                g = G[i + (long long)nb * j];
            }
        }
        Gs[i * (NB + 1) + j] = g;
        Ts[i * (NB + 1) + j] = (i == j && i < nb) ? tau[i] : cmake(0, 0);
    }
    __syncthreads();
    for (int s = 1; s < NB; s <<= 1) {
        const int per = s * s, total = (NB / (2 * s)) * per;
        for (int e = tid; e < total; e += BT_T) {   // X = G(a,b) T(b,b), T(b,b) upper
            const int pr = e / per, rem = e % per, i = rem / s, j = rem % s;
            const int a0 = 2 * pr * s, b0 = a0 + s;
            double xr = 0, xi = 0;
            for (int l = 0; l <= j; ++l) {
                const cplx g = Gs[(a0 + i) * (NB + 1) + b0 + l], t = Ts[(b0 + l) * (NB + 1) + b0 + j];
                xr = fma(g.x, t.x, fma(-g.y, t.y, xr));
                xi = fma(g.x, t.y, fma(g.y, t.x, xi));
            }
            Xs[e] = cmake(xr, xi);
        }
        __syncthreads();
        for (int e = tid; e < total; e += BT_T) {   // T(a,b) = -T(a,a) X, T(a,a) upper
            const int pr = e / per, rem = e % per, i = rem / s, j = rem % s;
            const int a0 = 2 * pr * s, b0 = a0 + s;
            double tr = 0, ti = 0;
            for (int l = i; l < s; ++l) {
                const cplx t = Ts[(a0 + i) * (NB + 1) + a0 + l], x = Xs[pr * per + l * s + j];
                tr = fma(t.x, x.x, fma(-t.y, x.y, tr));
                ti = fma(t.x, x.y, fma(t.y, x.x, ti));
            }
            Ts[(a0 + i) * (NB + 1) + b0 + j] = cmake(-tr, -ti);
        }
        __syncthreads();
    }
    for (int e = tid; e < NB * NB; e += BT_T) {
        const int i = e % NB, j = e / NB;
        T[i + (long long)ldt * j] = Ts[i * (NB + 1) + j];
    }
}

void launch_build_t(Context& ctx, int nb, const cplx* G, const cplx* tau, cplx* T, int nparts = 0) {
    NC_SET_SMEM_ONCE(build_t_kernel, BT_SMEM);
    build_t_kernel<<<1, BT_T, BT_SMEM, ctx.stream>>>(nb, G, nparts, tau, T, NB);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

// ---------------------------------------------------------------------------
// One block reflector applied to one block of at most NB columns,
//   C <- (I - V T V^H)^H C = C - V T^H (V^H C)     (V mp x nb, C mp x nc),
// and the Gram matrix V^H V of the block, for the critical path of the
// look-ahead QR.  The products are small (64 x 64 outputs, K = mp <= 2048),
// so instead of split-K GEMMs on a handful of tiles they run as
//   refl_partial_kernel: per 32-row chunk, the 64 x 64 partial of V^H C
//                        (one CTA per chunk, operands staged in shared memory);
//   refl_w2_kernel:      per column k, the chunk partials summed in chunk order
//                        and W2(:,k) = T^H W(:,k);
//   refl_apply_kernel:   per 32-row chunk, C -= V W2.
// The Gram matrix is refl_partial_kernel with C = V, its partials summed by
// build_t_kernel.  Every sum runs in a fixed order (bit-reproducible).
// ---------------------------------------------------------------------------
constexpr int RC = 32;                                     // rows per chunk
constexpr int RT = 256;                                    // threads
constexpr int RL = NB + 1;                                 // padded shared-memory row
constexpr size_t RP_SMEM = sizeof(cplx) * 2 * RC * RL;     // V and C chunks
constexpr size_t RA_SMEM = sizeof(cplx) * (NB + RC) * RL;  // W2 and the V chunk

__global__ void __launch_bounds__(RT) refl_partial_kernel(int mp, int nb, const cplx* __restrict__ V, long long ldv,
                                                          const cplx* __restrict__ C, long long ldc, int nc,
                                                          cplx* __restrict__ part) {
    extern __shared__ __align__(16) unsigned char rp_smem[];
    cplx* Vs = reinterpret_cast<cplx*>(rp_smem);   // [RC][RL]
    cplx* Cs = Vs + RC * RL;                         // [RC][RL]
    const int r0 = blockIdx.x * RC, tid = threadIdx.x;
    for (int e = tid; e < RC * NB; e += RT) {
        const int r = e % RC, c = e / RC, row = r0 + r;
        Vs[r * RL + c] = (row < mp && c < nb) ? V[row + ldv * c] : cmake(0, 0);
        Cs[r * RL + c] = (row < mp && c < nc) ? C[row + ldc * c] : cmake(0, 0);
    }
    __syncthreads();
    const int k = tid % NB, i0 = (tid / NB) * (NB / 4);   // 16 outputs (i0..i0+15, k) per thread
    double ar[NB / 4], ai[NB / 4];
#pragma unroll
    for (int q = 0; q < NB / 4; ++q) ar[q] = ai[q] = 0;
    for (int r = 0; r < RC; ++r) {
        const cplx c = Cs[r * RL + k];
#pragma unroll
        for (int q = 0; q < NB / 4; ++q) {
            const cplx v = Vs[r * RL + i0 + q];   // conj(v) * c
            ar[q] = fma(v.x, c.x, fma(v.y, c.y, ar[q]));
            ai[q] = fma(v.x, c.y, fma(-v.y, c.x, ai[q]));
        }
    }
    cplx* out = part + (size_t)blockIdx.x * NB * NB;
#pragma unroll
    for (int q = 0; q < NB / 4; ++q) out[i0 + q + NB * k] = cmake(ar[q], ai[q]);
}

__global__ void __launch_bounds__(RT) refl_w2_kernel(int nparts, int nb, const cplx* __restrict__ part,
                                                     const cplx* __restrict__ T, int ldt, cplx* __restrict__ W2) {
    __shared__ cplx red[RT / NB][NB];
    __shared__ cplx Ws[NB];
    const int k = blockIdx.x, tid = threadIdx.x, i = tid % NB, q = tid / NB;
    double sr = 0, si = 0;
    for (int c = q; c < nparts; c += RT / NB) {
        const cplx a = part[(size_t)c * NB * NB + i + NB * k];
        sr += a.x;
        si += a.y;
    }
    red[q][i] = cmake(sr, si);
    __syncthreads();
    if (q == 0) {
        cplx w = red[0][i];
#pragma unroll
        for (int g = 1; g < RT / NB; ++g) w = cadd(w, red[g][i]);
        Ws[i] = w;
    }
    __syncthreads();
    if (q == 0) {
        // W2(i,k) = sum_{l <= i} conj(T(l,i)) W(l,k)   (T upper triangular)
        double wr = 0, wi = 0;
        if (i < nb)
            for (int l = 0; l <= i; ++l) {
                const cplx t = T[l + (long long)ldt * i], w = Ws[l];
                wr = fma(t.x, w.x, fma(t.y, w.y, wr));
                wi = fma(t.x, w.y, fma(-t.y, w.x, wi));
            }
        W2[i + NB * k] = cmake(wr, wi);
    }
}

__global__ void __launch_bounds__(RT) refl_apply_kernel(int mp, int nb, const cplx* __restrict__ V, long long ldv,
                                                        const cplx* __restrict__ W2, cplx* __restrict__ C,
                                                        long long ldc, int nc) {
    extern __shared__ __align__(16) unsigned char ra_smem[];
    cplx* Ws = reinterpret_cast<cplx*>(ra_smem);   // [NB][RL]: Ws[l * RL + k] = W2(l,k)
    cplx* Vs = Ws + NB * RL;                         // [RC][RL]
    const int r0 = blockIdx.x * RC, tid = threadIdx.x;
    for (int e = tid; e < NB * NB; e += RT) {
        const int l = e % NB, kk = e / NB;
        Ws[l * RL + kk] = (l < nb && kk < nc) ? W2[l + NB * kk] : cmake(0, 0);
    }
    for (int e = tid; e < RC * NB; e += RT) {
        const int r = e % RC, c = e / RC, row = r0 + r;
        Vs[r * RL + c] = (row < mp && c < nb) ? V[row + ldv * c] : cmake(0, 0);
    }
    __syncthreads();
    const int k = tid % NB, rq = (tid / NB) * (RC / 4);   // rows rq..rq+7 of column k
    if (k >= nc) return;
    double ar[RC / 4], ai[RC / 4];
#pragma unroll
    for (int q = 0; q < RC / 4; ++q) ar[q] = ai[q] = 0;
    for (int l = 0; l < NB; ++l) {
        const cplx w = Ws[l * RL + k];
#pragma unroll
        for (int q = 0; q < RC / 4; ++q) {
            const cplx v = Vs[(rq + q) * RL + l];
            ar[q] = fma(v.x, w.x, fma(-v.y, w.y, ar[q]));
            ai[q] = fma(v.x, w.y, fma(v.y, w.x, ai[q]));
        }
    }
#pragma unroll
    for (int q = 0; q < RC / 4; ++q) {
        const int row = r0 + rq + q;
        if (row < mp) {
            cplx& c = C[row + ldc * k];
            c = cmake(c.x - ar[q], c.y - ai[q]);
        }
    }
}

int refl_chunks(int mp) { return (mp + RC - 1) / RC; }

void refl_attrs() {
    NC_SET_SMEM_ONCE(refl_partial_kernel, RP_SMEM);
    NC_SET_SMEM_ONCE(refl_apply_kernel, RA_SMEM);
}

// part (refl_chunks(mp) x NB x NB) = chunk partials of V^H C.
void launch_refl_partial(Context& ctx, int mp, int nb, const cplx* V, long long ldv, const cplx* C, long long ldc,
                         int nc, cplx* part) {
    refl_attrs();
    refl_partial_kernel<<<refl_chunks(mp), RT, RP_SMEM, ctx.stream>>>(mp, nb, V, ldv, C, ldc, nc, part);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

// C -= V T^H (V^H C), from the chunk partials of V^H C.
void launch_refl_finish(Context& ctx, int mp, int nb, const cplx* V, long long ldv, const cplx* T, int ldt,
                        const cplx* part, cplx* W2, cplx* C, long long ldc, int nc) {
    refl_attrs();
    refl_w2_kernel<<<nc, RT, 0, ctx.stream>>>(refl_chunks(mp), nb, part, T, ldt, W2);
    NC_CHECK_LAUNCH();
    refl_apply_kernel<<<refl_chunks(mp), RT, RA_SMEM, ctx.stream>>>(mp, nb, V, ldv, W2, C, ldc, nc);
    NC_CHECK_LAUNCH();
    ctx.launches += 2;
}

// ---------------------------------------------------------------------------
// One outer block (mp x nb, nb <= NB) factorised by a thread-block cluster.
//
// The rows are split over the C CTAs of one cluster (at most CQ_MAXR rows
// each, held in registers: thread (k, g) owns column k at rows g + 8i), so
// the whole block needs one launch instead of NB/JB panel and update
// launches.  Column j needs a single cluster-wide reduction: every CTA forms,
// over its rows below the diagonal,
//   s_k = sum_r conj(x_r) P(r,k)   for k >= j   (x = column j)
// which gives the column norm (k = j) and the reflector products with the
// trailing columns (k > j: w_k = P(j,k) + conj(scale) s_k), because
// v = e_j + scale * x; warps whose columns all lie left of j sit the column
// out (the Gram matrix V^H V of the compact-WY T is one GEMM after the
// kernel).  Each CTA stores its partial sums (and CTA 0,
// which holds the pivot rows, row j) into every CTA's shared memory (DSMEM,
// double-buffered by column parity) and one cluster barrier publishes them;
// each CTA then reduces the C partials with the same tree, so all CTAs
// derive bit-identical reflectors.  Reflector tails stay unscaled; the scale
// of column k is applied on use and at write-back.  The only waits are the
// hardware block and cluster barriers.
// ---------------------------------------------------------------------------
constexpr int CQ_T = 512;             // threads per CTA
constexpr int CQ_G = CQ_T / NB;       // lanes per column (row interleave)
constexpr int CQ_MAXC = 16;           // CTAs per cluster (non-portable size)
constexpr int CQ_MAXR = 128;          // rows per CTA -> mp <= 2048
constexpr int CQ_RPT = CQ_MAXR / CQ_G;  // rows per thread
__global__ void __launch_bounds__(CQ_T, 1)
cluster_block_qr_kernel(int mp, int nb, int rows_per_cta, cplx* __restrict__ A, long long lda,
                        cplx* __restrict__ V, long long ldv, cplx* __restrict__ tau_out) {
    __shared__ cplx recv[2][CQ_MAXC][NB];   // partial sums by source CTA, per column parity
    __shared__ cplx piv[2][NB];             // pivot row as received, per column parity
    __shared__ cplx pivst[2][NB];           // pivot row staged by its owners (CTA 0)
    __shared__ cplx xs[2][CQ_MAXR];         // column j of this CTA's rows
    __shared__ cplx colscale[NB];
    __shared__ cplx taus[NB];
    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    const int tid = threadIdx.x, k = tid / CQ_G, g = tid % CQ_G;
    const int row0 = rank * rows_per_cta;
    const int nr = max(0, min(rows_per_cta, mp - row0));
    // Row j (< nb) always lies in CTA 0: rows_per_cta >= nb whenever C > 1
    // (mp > CQ_MAXR (C-1)), and mp >= nb when C == 1.
    const bool top = (rank == 0);

    cplx a[CQ_RPT];
#pragma unroll
    for (int i = 0; i < CQ_RPT; ++i) {
        const int r = g + CQ_G * i;
        a[i] = (r < nr && k < nb) ? A[(row0 + r) + (long long)k * lda] : cmake(0, 0);
    }
    if (k == 0) {
#pragma unroll
        for (int i = 0; i < CQ_RPT; ++i) xs[0][g + CQ_G * i] = a[i];
    }
    if (top && g == 0) pivst[0][k] = a[0];   // row 0
    cluster.sync();

    for (int j = 0; j < nb; ++j) {
        const int p = j & 1;
        // Only columns k >= j take part in column j; a warp whose four
        // columns all lie left of j (k = 4*warp .. 4*warp + 3) skips it.
        const bool wactive = 4 * (tid >> 5) + 3 >= j;
        if (wactive) {
            // phase 1: partial sums over this CTA's rows below the diagonal.
            // Only CTA 0's first NB rows can lie on or above the diagonal.
            double s0r = 0, s0i = 0, s1r = 0, s1i = 0;
#pragma unroll
            for (int i = 0; i < CQ_RPT; i += 2) {
                const int r0 = g + CQ_G * i, r1 = r0 + CQ_G;
                const cplx x0 = xs[p][r0], x1 = xs[p][r1];
                const bool u0 = !top || r0 >= NB || r0 > j, u1 = !top || r1 >= NB || r1 > j;
                if (u0) {
                    s0r = fma(x0.x, a[i].x, fma(x0.y, a[i].y, s0r));
                    s0i = fma(x0.x, a[i].y, fma(-x0.y, a[i].x, s0i));
                }
                if (u1) {
                    s1r = fma(x1.x, a[i + 1].x, fma(x1.y, a[i + 1].y, s1r));
                    s1i = fma(x1.x, a[i + 1].y, fma(-x1.y, a[i + 1].x, s1i));
                }
            }
            double sr = s0r + s1r, si = s0i + s1i;
#pragma unroll
            for (int o = 1; o < CQ_G; o <<= 1) {
                sr += __shfl_xor_sync(0xffffffffu, sr, o);
                si += __shfl_xor_sync(0xffffffffu, si, o);
            }
            // phase 2: push to every CTA of the cluster (DSMEM stores)
            if (k >= j) {
                const cplx part = cmake(sr, si);
                const cplx pv = top ? pivst[p][k] : cmake(0, 0);
                for (int d = g; d < C; d += CQ_G) {
                    cluster.map_shared_rank(&recv[p][rank][0], d)[k] = part;
                    if (top) cluster.map_shared_rank(&piv[p][0], d)[k] = pv;
                }
            }
        }
        cluster.sync();   // release/acquire: publishes the partial sums
        if (wactive) {
            // phase 3: the CQ_G lanes of column k split the sources; a fixed
            // reduction tree keeps every CTA bit-identical
            cplx Sk = cmake(0, 0), Sj = cmake(0, 0);
            for (int c = g; c < C; c += CQ_G) {
                Sk = cadd(Sk, recv[p][c][k]);
                Sj = cadd(Sj, recv[p][c][j]);
            }
#pragma unroll
            for (int o = 1; o < CQ_G; o <<= 1) {
                Sk.x += __shfl_xor_sync(0xffffffffu, Sk.x, o);
                Sk.y += __shfl_xor_sync(0xffffffffu, Sk.y, o);
                Sj.x += __shfl_xor_sync(0xffffffffu, Sj.x, o);
            }
            const double xnorm2 = Sj.x;
            const cplx alpha = piv[p][j];
            const cplx pk = piv[p][k];
            cplx t = cmake(0, 0), scale = cmake(1, 0), diag = alpha;
            const bool reflect = !(xnorm2 == 0.0 && alpha.y == 0.0);
            if (reflect) {
                const double beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2), alpha.x);
                const cplx den = cmake(alpha.x - beta, alpha.y);
                const double ib = 1.0 / beta;
                const double idd = 1.0 / (den.x * den.x + den.y * den.y);
                t = cmake((beta - alpha.x) * ib, -alpha.y * ib);
                scale = cmake(den.x * idd, -den.y * idd);
                diag = cmake(beta, 0);
            }
            if (k == j && g == 0) {
                colscale[j] = scale;
                taus[j] = t;
            }
            // phase 4: apply H_j^H = I - conj(tau) v v^H to the trailing columns
            if (reflect && k > j && k < nb) {
                const cplx cf = cmul(cconj(t), cadd(pk, cmul(cconj(scale), Sk)));
                const cplx ef = cmul(scale, cf);
                if (top) {
#pragma unroll
                    for (int i = 0; i < CQ_RPT; ++i) {
                        const int r = g + CQ_G * i;
                        if (r < NB && r == j) a[i] = csub(a[i], cf);
                        else if (r >= NB || r > j) a[i] = csub(a[i], cmul(xs[p][r], ef));
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < CQ_RPT; ++i) a[i] = csub(a[i], cmul(xs[p][g + CQ_G * i], ef));
                }
            }
            if (top && k >= j) {
                // diagonal of R, and stage row j+1 for the next pivot broadcast
#pragma unroll
                for (int i = 0; i < CQ_RPT / 2; ++i) {   // rows < NB
                    const int r = g + CQ_G * i;
                    if (k == j && r == j) a[i] = diag;
                    if (r == j + 1) pivst[p ^ 1][k] = a[i];
                }
            }
            if (k == j + 1) {
#pragma unroll
                for (int i = 0; i < CQ_RPT; ++i) xs[p ^ 1][g + CQ_G * i] = a[i];
            }
        }
        __syncthreads();
    }

    {
#pragma unroll
        for (int i = 0; i < CQ_RPT; ++i) {
            const int r = g + CQ_G * i, prow = row0 + r;
            if (r < nr && k < nb) {
                cplx v = a[i];
                if (prow > k) v = cmul(v, colscale[k]);
                A[prow + (long long)k * lda] = v;
                V[prow + (long long)k * ldv] = (prow > k) ? v : cmake(prow == k ? 1.0 : 0.0, 0);
            }
        }
        if (rank == 0)
            for (int c = tid; c < nb; c += CQ_T) tau_out[c] = taus[c];
    }
    cluster.sync();   // no CTA leaves while another may still write its shared memory
}

// Cluster launch support (size CQ_MAXC needs the non-portable opt-in); a
// device that cannot co-schedule the cluster uses the per-panel path.
// The attribute and the answer belong to each device, so both are kept per
// device (the first 64; others are probed on every call).
bool cluster_qr_probe() {
    if (cudaFuncSetAttribute(cluster_block_qr_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
        cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CQ_MAXC);
    cfg.blockDim = dim3(CQ_T);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CQ_MAXC;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, cluster_block_qr_kernel, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return nclusters >= 1;
}

bool cluster_qr_available() {
    static std::atomic<int> state[64];   // 0 unknown, 1 available, 2 not available
    int dev = 0;
    NC_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return cluster_qr_probe();
    int s = state[dev].load(std::memory_order_acquire);
    if (s == 0) {
        s = cluster_qr_probe() ? 1 : 2;
        state[dev].store(s, std::memory_order_release);
    }
    return s == 1;
}

void launch_cluster_block(Context& ctx, int mp, int nb, cplx* A, long long lda, cplx* V, long long ldv,
                          cplx* tau) {
    const int C = std::max(1, std::min(CQ_MAXC, (mp + CQ_MAXR - 1) / CQ_MAXR));
    const int rows = (mp + C - 1) / C;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(CQ_T);
    cfg.stream = ctx.stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    NC_CUDA(cudaLaunchKernelEx(&cfg, cluster_block_qr_kernel, mp, nb, rows, A, lda, V, ldv, tau));
    ctx.launches++;
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
    const bool use_cluster = cluster_qr_available();
    if (!use_cluster) zfill(ctx, (long long)m * n, cmake(0, 0), V);
    for (int ob = 0; ob < nblocks; ++ob) {
        const int j0 = ob * NB;
        const int nb = std::min(NB, n - j0);
        const int mp = m - j0;
        const cplx* Vb = V + j0 + j0 * (long long)m;
        cplx* T = Tb + (size_t)ob * NB * NB;
        if (use_cluster) {
            launch_cluster_block(ctx, mp, nb, A + j0 + j0 * lda, lda, V + j0 + j0 * (long long)m, m, tau + j0);
            zgemm(zgemm_params(OP_C, OP_N, nb, nb, mp, Vb, m, Vb, m, G, nb), ctx);
        } else {
            for (int jj = j0; jj < j0 + nb; jj += JB) {
                const int jb = std::min(JB, j0 + nb - jj);
                launch_panel(ctx, m - jj, jb, A + jj + jj * lda, lda, V + jj + jj * (long long)m, m, tau + jj,
                             T4);
                const int rest = j0 + nb - (jj + jb);
                if (rest > 0) {
                    panel_apply_kernel<<<rest, PT, 0, ctx.stream>>>(m - jj, jb, V + jj + jj * (long long)m, m,
                                                                    T4, A + jj + (jj + jb) * lda, lda);
                    NC_CHECK_LAUNCH();
                    ctx.launches++;
                }
            }
            zgemm(zgemm_params(OP_C, OP_N, nb, nb, mp, Vb, m, Vb, m, G, nb), ctx);
        }
        // compact WY T for the outer block from G = V^H V (strict upper part)
        launch_build_t(ctx, nb, G, tau + j0, T);
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

// Look-ahead form of householder_qr for the gauge moves (cluster path only).
// The main stream (ctx) runs the critical path: factor block k, build T_k,
// then apply reflector k to block k+1 only, so that block k+1 can be
// factorised next.  The side stream applies reflector k to the remaining
// columns and accumulates Q forwards, Q <- Q (I - V_k T_k V_k^H) on an m x m
// Q, while the main stream factors the following blocks on the cluster's
// 16 SMs.  Forward accumulation costs about twice the flops of the backward
// order but overlaps the panels instead of following them.  ev: 2 + 2*nblocks
// events (fork, join, then per block: T_k ready, bulk update k done).
void householder_qr_lookahead(Context& ctx, Context& side, cudaEvent_t* ev, int m, int n, cplx* A, cplx* Q,
                              cplx* R, bool conjR) {
    NC_ARG(m >= n && n >= 1 && m <= CQ_MAXC * CQ_MAXR, "householder_qr: need 1 <= n <= m <= 2048");
    Arena& ar = ctx.scratch();
    ArenaFrame f(ar);
    const long long lda = m;
    const int nblocks = (n + NB - 1) / NB;
    cplx* V = ar.alloc_n<cplx>((size_t)m * n);
    cplx* tau = ar.alloc_n<cplx>(n);
    cplx* Tb = ar.alloc_n<cplx>((size_t)nblocks * NB * NB);
    cplx* Gpart = ar.alloc_n<cplx>((size_t)refl_chunks(m) * NB * NB);
    cplx* Wpart = ar.alloc_n<cplx>((size_t)refl_chunks(m) * NB * NB);
    cplx* W2m = ar.alloc_n<cplx>(NB * NB);
    cplx* Ws = ar.alloc_n<cplx>((size_t)NB * n);
    cplx* W2s = ar.alloc_n<cplx>((size_t)NB * n);
    cplx* QW = ar.alloc_n<cplx>((size_t)m * NB);
    cplx* QW2 = ar.alloc_n<cplx>((size_t)m * NB);
    cplx* Qf = ar.alloc_n<cplx>((size_t)m * m);
    const uint64_t side0 = side.launches;

    NC_CUDA(cudaEventRecord(ev[0], ctx.stream));   // fork
    NC_CUDA(cudaStreamWaitEvent(side.stream, ev[0], 0));
    identity_cols<<<gsz((long long)m * m), 256, 0, side.stream>>>(m, m, Qf);
    NC_CHECK_LAUNCH();
    side.launches++;
    for (int ob = 0; ob < nblocks; ++ob) {
        const int j0 = ob * NB, nb = std::min(NB, n - j0), mp = m - j0;
        const cplx* Vb = V + j0 + j0 * (long long)m;
        cplx* T = Tb + (size_t)ob * NB * NB;
        cudaEvent_t ev_t = ev[2 + 2 * ob], ev_bulk = ev[3 + 2 * ob];
        // main: factor block ob, then T_ob from the chunk partials of V^H V
        launch_cluster_block(ctx, mp, nb, A + j0 + j0 * lda, lda, V + j0 + j0 * (long long)m, m, tau + j0);
        launch_refl_partial(ctx, mp, nb, Vb, m, Vb, m, nb, Gpart);
        launch_build_t(ctx, nb, Gpart, tau + j0, T, refl_chunks(mp));
        NC_CUDA(cudaEventRecord(ev_t, ctx.stream));
        const int j1 = j0 + nb, nb1 = (ob + 1 < nblocks) ? std::min(NB, n - j1) : 0;
        if (nb1 > 0) {
            // main: reflector ob on block ob+1, after the side stream's update of
            // those columns by reflector ob-1
            if (ob > 0) NC_CUDA(cudaStreamWaitEvent(ctx.stream, ev[3 + 2 * (ob - 1)], 0));
            cplx* A1 = A + j0 + j1 * lda;
            launch_refl_partial(ctx, mp, nb, Vb, m, A1, lda, nb1, Wpart);
            launch_refl_finish(ctx, mp, nb, Vb, m, T, NB, Wpart, W2m, A1, lda, nb1);
        }
        // side: reflector ob on the columns after block ob+1, then Q
        NC_CUDA(cudaStreamWaitEvent(side.stream, ev_t, 0));
        const int jr = j1 + nb1, nt = n - jr;
        if (nt > 0) {
            cplx* A2 = A + j0 + jr * lda;
            zgemm(zgemm_params(OP_C, OP_N, nb, nt, mp, Vb, m, A2, lda, Ws, nb), side);
            zgemm(zgemm_params(OP_C, OP_N, nb, nt, nb, T, NB, Ws, nb, W2s, nb), side);
            ZGemmParams p = zgemm_params(OP_N, OP_N, mp, nt, nb, Vb, m, W2s, nb, A2, lda);
            p.alpha = cmake(-1, 0);
            p.beta = cmake(1, 0);
            zgemm(p, side);
        }
        NC_CUDA(cudaEventRecord(ev_bulk, side.stream));
        // Qf(:, j0:) -= (Qf(:, j0:) V_ob) T_ob V_ob^H
        cplx* Qs = Qf + j0 * (long long)m;
        zgemm(zgemm_params(OP_N, OP_N, m, nb, mp, Qs, m, Vb, m, QW, m), side);
        zgemm(zgemm_params(OP_N, OP_N, m, nb, nb, QW, m, T, NB, QW2, m), side);
        ZGemmParams q = zgemm_params(OP_N, OP_C, m, mp, nb, QW2, m, Vb, m, Qs, m);
        q.alpha = cmake(-1, 0);
        q.beta = cmake(1, 0);
        zgemm(q, side);
    }
    NC_CUDA(cudaEventRecord(ev[1], side.stream));   // join
    NC_CUDA(cudaStreamWaitEvent(ctx.stream, ev[1], 0));
    ctx.launches += side.launches - side0;
    if (R) {
        extract_r<<<gsz((long long)n * n), 256, 0, ctx.stream>>>(n, A, lda, conjR, R);
        NC_CHECK_LAUNCH();
        ctx.launches++;
    }
    if (Q) NC_CUDA(cudaMemcpyAsync(Q, Qf, sizeof(cplx) * (size_t)m * n, cudaMemcpyDeviceToDevice, ctx.stream));
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
    // look-ahead: the thread's second stream (side_context) with this plan's
    // split-K arena, and the plan's events
    bool lookahead = false;
    Arena side_arena;
    std::vector<cudaEvent_t> ev;
    // single-block shapes are run directly: recording a graph saves nothing
    bool capture = true;
    cplx* X = nullptr;   // input (m x n), overwritten
    cplx* Q = nullptr;   // explicit Q (m x n)
    cplx* R = nullptr;   // R (n x n), conjugated if conjR
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t kernels = 0;
    ~QrPlan() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
};

namespace {
// Second stream of this host thread for the look-ahead QR (one per thread,
// shared by the thread's plans, which run one at a time).
Context& side_context() {
    thread_local Context* c = new Context();   // lives until process exit, like Context::get()
    return *c;
}

QrPlan& qr_plan(Context& ctx, int m, int n, bool conjR) {
    thread_local std::vector<std::unique_ptr<QrPlan>> plans;
    for (auto& p : plans)
        if (p->m == m && p->n == n && p->conjR == conjR) return *p;
    auto p = std::make_unique<QrPlan>();
    p->m = m; p->n = n; p->conjR = conjR;
    p->X = p->arena.alloc_n<cplx>((size_t)m * n);
    p->Q = p->arena.alloc_n<cplx>((size_t)m * n);
    p->R = p->arena.alloc_n<cplx>((size_t)n * n);
    if (cluster_qr_available()) {
        p->lookahead = true;
        p->ev.resize(4 + 2 * ((n + NB - 1) / NB));   // the last two fork/join the priority stream
        for (cudaEvent_t& e : p->ev) NC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    p->capture = n > NB;
    plans.push_back(std::move(p));
    return *plans.back();
}

// Highest-priority stream of this host thread for the critical path of the
// recorded look-ahead QR (panels, T, next-block updates).  Graph nodes keep
// the priority of the stream they were captured from (the graph is
// instantiated with cudaGraphInstantiateFlagUseNodePriority), so a pending
// cluster launch is dispatched ahead of the trailing-update GEMMs of the
// second stream as SMs drain.  Null when the stream cannot be created.
cudaStream_t priority_stream() {
    thread_local cudaStream_t s = [] {
        int least = 0, greatest = 0;
        cudaStream_t st = nullptr;
        if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
            cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, greatest) != cudaSuccess) {
            cudaGetLastError();
            st = nullptr;
        }
        return st;
    }();
    return s;
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
    Context& side = side_context();
    side.ws_override = &P.side_arena;
    auto once = [&] {
        if (P.lookahead && P.capture)
            householder_qr_lookahead(ctx, side, P.ev.data(), P.m, P.n, P.X, P.Q, P.R, P.conjR);
        else
            householder_qr(ctx, P.m, P.n, P.X, P.Q, P.R, P.conjR);
    };
    if (!P.capture) {
        try {
            once();
        } catch (...) {
            ctx.ws_override = nullptr;
            ctx.profile = prof;
            throw;
        }
        ctx.ws_override = nullptr;
        ctx.profile = prof;
        return;
    }
    try {
        once();
        const uint64_t l0 = ctx.launches;
        const cudaStream_t home = ctx.stream;
        const cudaStream_t hp = P.lookahead ? priority_stream() : nullptr;
        NC_CUDA(cudaStreamBeginCapture(home, cudaStreamCaptureModeRelaxed));
        try {
            if (hp) {
                NC_CUDA(cudaEventRecord(P.ev[P.ev.size() - 2], home));
                NC_CUDA(cudaStreamWaitEvent(hp, P.ev[P.ev.size() - 2], 0));
                ctx.stream = hp;
            }
            once();
            if (hp) {
                NC_CUDA(cudaEventRecord(P.ev[P.ev.size() - 1], hp));
                ctx.stream = home;
                NC_CUDA(cudaStreamWaitEvent(home, P.ev[P.ev.size() - 1], 0));
            }
        } catch (...) {
            ctx.stream = home;
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(home, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        NC_CUDA(cudaStreamEndCapture(home, &P.graph));
        P.kernels = ctx.launches - l0;
        ctx.launches = l0;
        NC_CUDA(cudaGraphInstantiateWithFlags(&P.exec, P.graph, cudaGraphInstantiateFlagUseNodePriority));
    } catch (...) {
        ctx.ws_override = nullptr;
        ctx.profile = prof;
        throw;
    }
    ctx.ws_override = nullptr;
    ctx.profile = prof;
}
}  // namespace

// The absorption GEMM of the gauge factor, on ctx.stream or, with `as`, on
// the second stream after the QR that produced the factor.
static void absorb_factor(Context& ctx, const ZGemmParams& p, const AbsorbAsync* as) {
    if (!as) {
        zgemm(p, ctx);
        return;
    }
    NC_CUDA(cudaEventRecord(as->ready, ctx.stream));
    NC_CUDA(cudaStreamWaitEvent(as->stream, as->ready, 0));
    zgemm(p, as->stream);
    ctx.launches++;
    NC_CUDA(cudaEventRecord(as->done, as->stream));
}

void gauge_right(Context& ctx, int bl, int bm, int br, int dl, int dr, const cplx* A, const cplx* B,
                 cplx* normA, cplx* denormB, const AbsorbAsync* async) {
    const int K = bl * dl;
    NC_ARG(K >= bm, "not enough degrees of freedom to normalize");
    QrPlan& P = qr_plan(ctx, K, bm, false);
    const int p_t[3] = {1, 0, 2};
    permute3(ctx, A, bm, K, 1, p_t, true, P.X);             // X = A^H  (K x bm)
    qr_run(ctx, P);                                          // A^H = Qt Rt
    if (B && denormB) {
        // denormB_s = B_s Rt^H  (neighbour absorbs P = Rt^H on its left index)
        ZGemmParams p = zgemm_params(OP_N, OP_C, br, bm, bm, B, br, P.R, bm, denormB, br);
        p.batch = dr;
        p.sA0 = (long long)br * bm; p.sB0 = 0; p.sC0 = (long long)br * bm;
        absorb_factor(ctx, p, async);
    }
    permute3(ctx, P.Q, K, bm, 1, p_t, true, normA);         // normA = Qt^H
}

void gauge_left(Context& ctx, int bl, int bm, int br, int dl, int dr, const cplx* A, const cplx* B,
                cplx* denormA, cplx* normB, const AbsorbAsync* async) {
    const int K = br * dr;
    NC_ARG(K >= bm, "not enough degrees of freedom to normalize");
    QrPlan& P = qr_plan(ctx, K, bm, true);
    const cplx* Rc = P.R;
    const int p_rs[3] = {0, 2, 1};
    permute3(ctx, B, br, bm, dr, p_rs, true, P.X);           // X((r,s),m) = conj(B(r,m,s))
    qr_run(ctx, P);                                          // Rc = conj(Rt)
    if (A && denormA) {
        // denormA = conj(Rt) * A  (as bm x bl*dl)
        absorb_factor(ctx, zgemm_params(OP_N, OP_N, bm, bl * dl, bm, Rc, bm, A, bm, denormA, bm), async);
    }
    permute3(ctx, P.Q, br, dr, bm, p_rs, true, normB);       // normB(r,m,s) = conj(Qt((r,s),m))
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
