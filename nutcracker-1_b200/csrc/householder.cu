// Projector (excited-state) algebra on the device.
//
// The reference stores the span of the lower levels' overlap vectors as the
// column-pivoted Householder QR of those vectors (zgeqp3, core.f95:1341-1435)
// and moves vectors in and out of the orthogonal complement with zunmqr
// (core.f95:1513-1664).  Vectors are treated as 1 x n ROW vectors multiplied
// from the right: project = swap(x Q)[r:], unproject = unswap([0, y]) Q^H,
// with Q = H_1 ... H_k, H_i = I - tau_i v_i v_i^H, v_i(i) = 1 and
// v_i(j<i) = 0.  Each reflector costs one reduction and one update pass over
// the vector (HBM-bound).  For the eigensolver the removed space is also
// materialised once per site as r orthonormal columns U (u_p = e_{sigma(p)} Q^H),
// turning the filter into one multi-dot and one multi-axpy.
#include <algorithm>
#include <cmath>

#include "nc_common.cuh"
#include "nc_kernels.h"

namespace nc {

namespace {

constexpr int HT = 256;
constexpr int HB = 592;

// s = sum_{j>=i} x_j v(j), v(i) = 1 (no conjugation), partial sums per block
__global__ void house_dot_partial(long long n, int i, const cplx* __restrict__ x,
                                  const cplx* __restrict__ v, cplx* __restrict__ part) {
    __shared__ double sr[HT], si[HT];
    double ar = 0, ai = 0;
    for (long long e = (long long)i + blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        cplx vv = (e == i) ? cmake(1, 0) : v[e];
        cplx p = cmul(x[e], vv);
        ar += p.x; ai += p.y;
    }
    sr[threadIdx.x] = ar; si[threadIdx.x] = ai;
    __syncthreads();
    for (int s = HT / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) { sr[threadIdx.x] += sr[threadIdx.x + s]; si[threadIdx.x] += si[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = cmake(sr[0], si[0]);
}

__global__ void reduce_to(int nb, const cplx* __restrict__ part, cplx* __restrict__ out) {
    __shared__ double sr[HT], si[HT];
    double ar = 0, ai = 0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) { ar += part[i].x; ai += part[i].y; }
    sr[threadIdx.x] = ar; si[threadIdx.x] = ai;
    __syncthreads();
    for (int s = HT / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) { sr[threadIdx.x] += sr[threadIdx.x + s]; si[threadIdx.x] += si[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = cmake(sr[0], si[0]);
}

// x_j -= f * s * conj(v(j)) for j >= i, f = tau_i (Q) or conj(tau_i) (Q^H)
__global__ void house_update(long long n, int i, const cplx* __restrict__ s_dev,
                             const cplx* __restrict__ tau, bool conj_tau, const cplx* __restrict__ v,
                             cplx* __restrict__ x) {
    cplx t = tau[i];
    if (conj_tau) t = cconj(t);
    cplx c = cmul(t, s_dev[0]);
    for (long long e = (long long)i + blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        cplx vv = (e == i) ? cmake(1, 0) : v[e];
        x[e] = csub(x[e], cmul(c, cconj(vv)));
    }
}

struct SwapSpec {
    int ns, zero_first;
    int sw[kMaxProjectors];
};

// swap_inplace, zero the first `zero_first` entries, unswap_inplace (core.f95:464-506)
__global__ void swap_zero_unswap(SwapSpec sp, cplx* __restrict__ x) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = 0; i < sp.ns; ++i) {
        int j = sp.sw[i] - 1;
        if (j != i) { cplx t = x[i]; x[i] = x[j]; x[j] = t; }
    }
    for (int i = 0; i < sp.zero_first; ++i) x[i] = cmake(0, 0);
    for (int i = sp.ns - 1; i >= 0; --i) {
        int j = sp.sw[i] - 1;
        if (j != i) { cplx t = x[i]; x[i] = x[j]; x[j] = t; }
    }
}

__global__ void set_unit(cplx* x, long long pos) { x[pos] = cmake(1, 0); }

// weights = R^T p[:nrefl] (R upper triangle of the reflector matrix), overlap = ||weights||
__global__ void overlap_weights(int nrefl, long long ld, const cplx* __restrict__ refl,
                                const cplx* __restrict__ p, const cplx* __restrict__ extra,
                                int nextra, double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double acc = 0;
    for (int c = 0; c < nrefl; ++c) {
        cplx w = cmake(0, 0);
        for (int r = 0; r <= c; ++r) w = cadd(w, cmul(refl[r + ld * c], p[r]));
        acc += cabs2(w);
    }
    for (int c = 0; c < nextra; ++c) acc += cabs2(extra[c]);
    out[0] = sqrt(acc);
}

// non-conjugated dot partial sums: sum x_j y_j
__global__ void dotu_partial(long long n, const cplx* __restrict__ x, const cplx* __restrict__ y,
                             cplx* __restrict__ part) {
    __shared__ double sr[HT], si[HT];
    double ar = 0, ai = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        cplx p = cmul(x[e], y[e]);
        ar += p.x; ai += p.y;
    }
    sr[threadIdx.x] = ar; si[threadIdx.x] = ai;
    __syncthreads();
    for (int s = HT / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) { sr[threadIdx.x] += sr[threadIdx.x + s]; si[threadIdx.x] += si[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = cmake(sr[0], si[0]);
}

void house_apply_one(Context& ctx, long long n, int i, const cplx* v, const cplx* tau, bool conj_tau,
                     cplx* x, cplx* part, cplx* s) {
    house_dot_partial<<<HB, HT, 0, ctx.stream>>>(n, i, x, v, part);
    NC_CHECK_LAUNCH();
    reduce_to<<<1, HT, 0, ctx.stream>>>(HB, part, s);
    NC_CHECK_LAUNCH();
    unsigned g = (unsigned)std::max<long long>(1, std::min<long long>((n - i + 255) / 256, 148 * 16));
    house_update<<<g, 256, 0, ctx.stream>>>(n, i, s, tau, conj_tau, v, x);
    NC_CHECK_LAUNCH();
    ctx.launches += 3;
}

SwapSpec make_swapspec(const DevProjector& P, int zero_first) {
    SwapSpec sp;
    sp.ns = (int)P.swaps.size();
    NC_ARG(sp.ns <= kMaxProjectors, "too many projectors");
    for (int i = 0; i < sp.ns; ++i) sp.sw[i] = (int)P.swaps[i];
    sp.zero_first = zero_first;
    return sp;
}

}  // namespace

void apply_q_row(Context& ctx, const DevProjector& P, cplx* x, bool conj_trans) {
    if (P.nrefl == 0) return;
    ArenaFrame f(ctx.arena);
    cplx* part = ctx.arena.alloc_n<cplx>(HB);
    cplx* s = ctx.arena.alloc_n<cplx>(1);
    if (!conj_trans) {
        for (int i = 0; i < P.nrefl; ++i) house_apply_one(ctx, P.n, i, P.refl + (size_t)i * P.n, P.tau, false, x, part, s);
    } else {
        for (int i = P.nrefl - 1; i >= 0; --i)
            house_apply_one(ctx, P.n, i, P.refl + (size_t)i * P.n, P.tau, true, x, part, s);
    }
}

void filter_outside(Context& ctx, const DevProjector& P, const cplx* in, cplx* out) {
    if (out != in) zcopy(ctx, P.n, in, out);
    if (P.nproj == 0) return;
    apply_q_row(ctx, P, out, false);
    SwapSpec sp = make_swapspec(P, (int)(P.n - P.orth_dim));
    swap_zero_unswap<<<1, 1, 0, ctx.stream>>>(sp, out);
    NC_CHECK_LAUNCH();
    ctx.launches++;
    apply_q_row(ctx, P, out, true);
}

double overlap_with_projectors(Context& ctx, const DevProjector& P, const cplx* x) {
    // core.f95:1266-1339
    if (P.nproj == 0) return 0.0;
    ArenaFrame f(ctx.arena);
    cplx* p = ctx.arena.alloc_n<cplx>(P.n);
    zcopy(ctx, P.n, x, p);
    apply_q_row(ctx, P, p, false);  // swap followed by unswap is the identity
    int nextra = P.nproj - P.nrefl;
    cplx* extra = ctx.arena.alloc_n<cplx>(std::max(1, nextra));
    cplx* part = ctx.arena.alloc_n<cplx>(HB);
    for (int c = 0; c < nextra; ++c) {
        dotu_partial<<<HB, HT, 0, ctx.stream>>>(P.n, P.refl + (size_t)(P.nrefl + c) * P.n, p, part);
        NC_CHECK_LAUNCH();
        reduce_to<<<1, HT, 0, ctx.stream>>>(HB, part, extra + c);
        NC_CHECK_LAUNCH();
        ctx.launches += 2;
    }
    double* out = ctx.arena.alloc_n<double>(1);
    overlap_weights<<<1, 1, 0, ctx.stream>>>(P.nrefl, P.n, P.refl, p, extra, nextra, out);
    NC_CHECK_LAUNCH();
    ctx.launches++;
    double v;
    read_scalars(ctx, out, sizeof(double), &v);
    return v;
}

std::vector<long long> removed_positions(const DevProjector& P) {
    const int ns = (int)P.swaps.size();
    std::vector<long long> arr(ns);
    for (int i = 0; i < ns; ++i) arr[i] = i;
    for (int i = 0; i < ns; ++i) {
        int j = (int)P.swaps[i] - 1;
        if (j != i) std::swap(arr[i], arr[j]);
    }
    const long long r = P.n - P.orth_dim;
    std::vector<long long> out;
    for (long long q = 0; q < r; ++q) out.push_back(q < ns ? arr[q] : q);
    return out;
}

void removed_basis(Context& ctx, const DevProjector& P, cplx* U) {
    std::vector<long long> pos = removed_positions(P);
    for (size_t q = 0; q < pos.size(); ++q) {
        cplx* u = U + q * (size_t)P.n;
        zfill(ctx, P.n, cmake(0, 0), u);
        set_unit<<<1, 1, 0, ctx.stream>>>(u, pos[q]);
        NC_CHECK_LAUNCH();
        ctx.launches++;
        apply_q_row(ctx, P, u, true);
    }
}

void unproject_unit(Context& ctx, const DevProjector& P, long long reduced_index, cplx* out) {
    // unproject_from_orthogonal_space (core.f95:1591-1664) applied to e_j of the reduced space
    zfill(ctx, P.n, cmake(0, 0), out);
    const long long start = P.n - P.orth_dim;  // 0-based first orthogonal coordinate
    set_unit<<<1, 1, 0, ctx.stream>>>(out, start + reduced_index);
    NC_CHECK_LAUNCH();
    ctx.launches++;
    if (P.nproj == 0) return;
    // unswap_inplace on the leading entries: follow where the unit entry moves
    long long pos = start + reduced_index;
    for (int i = (int)P.swaps.size() - 1; i >= 0; --i) {
        long long j = (long long)P.swaps[i] - 1;
        if (j == i) continue;
        if (pos == i) pos = j;
        else if (pos == j) pos = i;
    }
    if (pos != start + reduced_index) {
        zfill(ctx, P.n, cmake(0, 0), out);
        set_unit<<<1, 1, 0, ctx.stream>>>(out, pos);
        NC_CHECK_LAUNCH();
        ctx.launches++;
    }
    apply_q_row(ctx, P, out, true);
}

// ---------------------------------------------------------------------------
// convert_vectors_to_reflectors (core.f95:1341-1435): column-pivoted
// Householder QR of an m x n block of overlap vectors (n small), then the
// reference's rank/swap rule on the row norms of R.
// ---------------------------------------------------------------------------
namespace {

__global__ void colnorm2_partial(long long m, long long row0, const cplx* __restrict__ col,
                                 cplx* __restrict__ part) {
    __shared__ double sr[HT];
    double a = 0;
    for (long long e = row0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m;
         e += (long long)gridDim.x * blockDim.x)
        a += cabs2(col[e]);
    sr[threadIdx.x] = a;
    __syncthreads();
    for (int s = HT / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sr[threadIdx.x] += sr[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = cmake(sr[0], 0);
}

__global__ void swap_cols(long long m, cplx* __restrict__ a, cplx* __restrict__ b) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m;
         e += (long long)gridDim.x * blockDim.x) {
        cplx t = a[e]; a[e] = b[e]; b[e] = t;
    }
}

__global__ void scale_from(long long m, long long row0, cplx f, cplx* __restrict__ col) {
    for (long long e = row0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m;
         e += (long long)gridDim.x * blockDim.x)
        col[e] = cmul(f, col[e]);
}

__global__ void set_value(cplx* p, cplx v) { *p = v; }

// s = v^H a over rows >= i (v(i) = 1), partial sums
__global__ void house_dotc_partial(long long m, long long i, const cplx* __restrict__ v,
                                   const cplx* __restrict__ a, cplx* __restrict__ part) {
    __shared__ double sr[HT], si[HT];
    double ar = 0, ai = 0;
    for (long long e = i + blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m;
         e += (long long)gridDim.x * blockDim.x) {
        cplx vv = (e == i) ? cmake(1, 0) : v[e];
        cplx p = cmul(cconj(vv), a[e]);
        ar += p.x; ai += p.y;
    }
    sr[threadIdx.x] = ar; si[threadIdx.x] = ai;
    __syncthreads();
    for (int s = HT / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) { sr[threadIdx.x] += sr[threadIdx.x + s]; si[threadIdx.x] += si[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = cmake(sr[0], si[0]);
}

// a -= f s v over rows >= i, f given on host, s on device
__global__ void house_left_update(long long m, long long i, cplx f, const cplx* __restrict__ s_dev,
                                  const cplx* __restrict__ v, cplx* __restrict__ a) {
    cplx c = cmul(f, s_dev[0]);
    for (long long e = i + blockIdx.x * (long long)blockDim.x + threadIdx.x; e < m;
         e += (long long)gridDim.x * blockDim.x) {
        cplx vv = (e == i) ? cmake(1, 0) : v[e];
        a[e] = csub(a[e], cmul(c, vv));
    }
}

double dev_colnorm2(Context& ctx, long long m, long long row0, const cplx* col, cplx* part, cplx* s) {
    colnorm2_partial<<<HB, HT, 0, ctx.stream>>>(m, row0, col, part);
    NC_CHECK_LAUNCH();
    reduce_to<<<1, HT, 0, ctx.stream>>>(HB, part, s);
    NC_CHECK_LAUNCH();
    ctx.launches += 2;
    return read_scalar(ctx, s).x;
}

}  // namespace

int convert_vectors_to_reflectors_dev(Context& ctx, long long m, int n, cplx* A, cplx* tau_dev,
                                      std::vector<uint32_t>& swaps) {
    swaps.clear();
    if (n == 0) return 0;
    NC_ARG(n <= kMaxProjectors, "convert_vectors_to_reflectors: too many vectors");
    const int k = (int)std::min<long long>(m, n);
    ArenaFrame f(ctx.arena);
    cplx* part = ctx.arena.alloc_n<cplx>(HB);
    cplx* s = ctx.arena.alloc_n<cplx>(1);
    unsigned g = (unsigned)std::max<long long>(1, std::min<long long>((m + 255) / 256, 148 * 16));
    std::vector<cplx> tau(k);
    for (int i = 0; i < k; ++i) {
        // pivot: the remaining column with the largest norm over rows i..m-1 (zgeqp3/zlaqp2)
        int piv = i;
        double best = -1;
        for (int j = i; j < n; ++j) {
            double v = dev_colnorm2(ctx, m, i, A + (size_t)j * m, part, s);
            if (v > best) { best = v; piv = j; }
        }
        if (piv != i) {
            swap_cols<<<g, 256, 0, ctx.stream>>>(m, A + (size_t)i * m, A + (size_t)piv * m);
            NC_CHECK_LAUNCH();
            ctx.launches++;
        }
        cplx* col = A + (size_t)i * m;
        // zlarfg: alpha = A(i,i), xnorm = ||A(i+1:m,i)||
        cplx alpha;
        read_scalars(ctx, col + i, sizeof(cplx), &alpha);
        double xnorm = (i + 1 < m) ? std::sqrt(dev_colnorm2(ctx, m, i + 1, col, part, s)) : 0.0;
        cplx t;
        if (xnorm == 0.0 && alpha.y == 0.0) {
            t = cmake(0, 0);
        } else {
            double beta = -std::copysign(std::sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm * xnorm), alpha.x);
            t = cmake((beta - alpha.x) / beta, -alpha.y / beta);
            // scale x by 1/(alpha - beta)
            cplx den = cmake(alpha.x - beta, alpha.y);
            double dd = den.x * den.x + den.y * den.y;
            cplx inv = cmake(den.x / dd, -den.y / dd);
            if (i + 1 < m) {
                scale_from<<<g, 256, 0, ctx.stream>>>(m, i + 1, inv, col);
                NC_CHECK_LAUNCH();
                ctx.launches++;
            }
            set_value<<<1, 1, 0, ctx.stream>>>(col + i, cmake(beta, 0));
            NC_CHECK_LAUNCH();
            ctx.launches++;
        }
        tau[i] = t;
        // apply H^H = I - conj(tau) v v^H to the remaining columns (zlarf 'Left')
        if (t.x != 0.0 || t.y != 0.0) {
            for (int j = i + 1; j < n; ++j) {
                cplx* a = A + (size_t)j * m;
                house_dotc_partial<<<HB, HT, 0, ctx.stream>>>(m, i, col, a, part);
                NC_CHECK_LAUNCH();
                reduce_to<<<1, HT, 0, ctx.stream>>>(HB, part, s);
                NC_CHECK_LAUNCH();
                house_left_update<<<g, 256, 0, ctx.stream>>>(m, i, cconj(t), s, col, a);
                NC_CHECK_LAUNCH();
                ctx.launches += 3;
            }
        }
    }
    NC_CUDA(cudaMemcpyAsync(tau_dev, tau.data(), k * sizeof(cplx), cudaMemcpyHostToDevice, ctx.stream));
    // rank rule of core.f95:1410-1433 on norms(i) = ||R(i, i:n)||
    std::vector<cplx> R((size_t)k * n);
    for (int c = 0; c < n; ++c)
        NC_CUDA(cudaMemcpyAsync(R.data() + (size_t)c * k, A + (size_t)c * m, k * sizeof(cplx),
                                cudaMemcpyDeviceToHost, ctx.stream));
    NC_CUDA(cudaStreamSynchronize(ctx.stream));
    std::vector<double> norms(k);
    for (int i = 0; i < k; ++i) {
        double a = 0;
        for (int c = i; c < n; ++c) {
            cplx v = R[(size_t)c * k + i];
            a += v.x * v.x + v.y * v.y;
        }
        norms[i] = std::sqrt(a);
    }
    swaps.resize(k);
    for (int i = 0; i < k; ++i) swaps[i] = (uint32_t)(i + 1);
    int i = 0;
    bool stopped = false;
    for (; i < k; ++i) {
        if (norms[i] < 1e-12) {
            int j = i;
            for (;;) {
                ++j;
                if (j == k || norms[j] > 1e-12) break;
            }
            if (j == k) { stopped = true; break; }
            std::swap(norms[i], norms[j]);
            swaps[i] = (uint32_t)(j + 1);
        }
    }
    return stopped ? i : k;
}

}  // namespace nc
