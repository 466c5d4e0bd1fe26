// Precision form of the site products: the effective-Hamiltonian product
// with its two contractions as complex FP32 on the tensor cores (3xTF32 with
// FP32 accumulation, tc32.cu) and FP64 everywhere else (input, output, the
// sparse-MPO mix accumulation).
//
// Stage A  T_a = psi_a [L_1 .. L_cl]     D = X_op L_op^T,  X_op(r, i) = psi(r,i,a)
// mix      U(r,k2,j,b) = sum_{n: to=k2} sum_a W(a,b,n) T(r,j,k1(n),a)
// Stage C  out_b = [R_1 .. R_cr] U_b     D = U_op R_op^T,  U_op(j, (r,k2)) = U(r,k2,j,b)
// The environment operands L_op, R_op are expanded to the (conjugate,
// swapped) row pairs of the real formulation once per site; psi and U are
// converted on every product.  Layouts are chosen so that every operand is
// K-major for TMA: see tc32.cu for the real formulation.
#include <algorithm>

#include "nc_common.cuh"
#include "nc_kernels.h"

namespace nc {

namespace {

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// x = big + small with both halves TF32 (the residual is taken in FP64).
__device__ __forceinline__ void split_tf32(double x, float& big, float& small) {
    big = tf32_rna((float)x);
    small = tf32_rna((float)(x - (double)big));
}

long long round4(long long x) { return (x + 3) & ~3LL; }
size_t align64(size_t x) { return (x + 63) & ~(size_t)63; }

// Row m, K index k of the complex input X[z*sxz + m*sxm + k*sxk] to TF32
// pairs, 32 x 32 tiles through shared memory (loads run along whichever of
// m, k is contiguous; stores run along k).
//   EXPAND = false: out[z*soz + m*ld + 2k + {0,1}] = (Re, Im)
//   EXPAND = true : out rows 2m = (Re, -Im), 2m+1 = (Im, Re)
// CONJ conjugates the input first.  soz may also be a column offset (a
// batch of inputs written side by side along K).
template <bool EXPAND, bool CONJ = false>
__global__ void split_rows_kernel(int rows, int K, const cplx* __restrict__ X, long long sxm, long long sxk,
                                  long long sxz, float* __restrict__ ob, float* __restrict__ os, long long ld,
                                  long long soz) {
    __shared__ cplx tile[32][33];
    const int k0 = blockIdx.x * 32, m0 = blockIdx.y * 32, z = blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const bool mcontig = (sxm == 1);
    const cplx* Xz = X + (long long)z * sxz;
    for (int yy = ty; yy < 32; yy += 8) {
        const int ml = mcontig ? tx : yy, kl = mcontig ? yy : tx;
        const int m = m0 + ml, k = k0 + kl;
        tile[ml][kl] = (m < rows && k < K) ? Xz[(long long)m * sxm + (long long)k * sxk] : cmake(0, 0);
    }
    __syncthreads();
    float* bz = ob + (long long)z * soz;
    float* sz = os + (long long)z * soz;
    for (int yy = ty; yy < 32; yy += 8) {
        const int m = m0 + yy, k = k0 + tx;
        if (m >= rows || k >= K) continue;
        cplx v = tile[yy][tx];
        if (CONJ) v.y = -v.y;
        float br, bi, sr, si;
        if (!EXPAND) {
            split_tf32(v.x, br, sr);
            split_tf32(v.y, bi, si);
            const long long o = (long long)m * ld + 2 * k;
            *reinterpret_cast<float2*>(bz + o) = make_float2(br, bi);
            *reinterpret_cast<float2*>(sz + o) = make_float2(sr, si);
        } else {
            split_tf32(v.x, br, sr);
            split_tf32(v.y, bi, si);
            const long long o0 = (long long)(2 * m) * ld + 2 * k, o1 = o0 + ld;
            *reinterpret_cast<float2*>(bz + o0) = make_float2(br, -bi);
            *reinterpret_cast<float2*>(sz + o0) = make_float2(sr, -si);
            *reinterpret_cast<float2*>(bz + o1) = make_float2(bi, br);
            *reinterpret_cast<float2*>(sz + o1) = make_float2(si, sr);
        }
    }
}

template <bool EXPAND, bool CONJ = false>
void split_rows(Context& ctx, int rows, int K, int batch, const cplx* X, long long sxm, long long sxk,
                long long sxz, float* ob, float* os, long long ld, long long soz) {
    dim3 grid((K + 31) / 32, (rows + 31) / 32, batch), block(32, 8);
    split_rows_kernel<EXPAND, CONJ><<<grid, block, 0, ctx.stream>>>(rows, K, X, sxm, sxk, sxz, ob, os, ld, soz);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

constexpr int MIXM_MAX_NNZ = 64;
constexpr int MIXM_MAX_D = 4;

// Output strides (complex units) of a mixed-precision operand element.
struct Out4 {
    long long s0, s1, s2, s3;
};

// U(r,k2,j,b) = sum_{n: to(n)=k2} sum_a W(a,b,n) T(r, j + bl*(k1(n) + cl*a))
// (T complex64 from stage A), accumulated in FP64 and written as a TF32
// pair at complex offset r*o.s0 + k2*o.s1 + j*o.s2 + b*o.s3.
__global__ void mix_left_tf32_kernel(int br, int bl, int cl, int cr, int d, int nnz, const uint32_t* __restrict__ idx,
                                     const cplx* __restrict__ W, const float2* __restrict__ T,
                                     float* __restrict__ Ub, float* __restrict__ Us, Out4 o) {
    __shared__ cplx Ws[MIXM_MAX_NNZ * MIXM_MAX_D * MIXM_MAX_D];
    __shared__ int k1s[MIXM_MAX_NNZ], k2s[MIXM_MAX_NNZ];
    for (int i = threadIdx.x; i < nnz * d * d; i += blockDim.x) Ws[i] = W[i];
    for (int i = threadIdx.x; i < nnz; i += blockDim.x) {
        k1s[i] = (int)idx[2 * i] - 1;
        k2s[i] = (int)idx[2 * i + 1] - 1;
    }
    __syncthreads();
    const long long total = (long long)br * cr * bl * d;
    const long long sT_j = br, sT_k = (long long)br * bl, sT_a = (long long)br * bl * cl;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long q = e;
        const int r = (int)(q % br); q /= br;
        const int k2 = (int)(q % cr); q /= cr;
        const int j = (int)(q % bl); q /= bl;
        const int b = (int)q;
        double ar = 0, ai = 0;
        const float2* Tb = T + r + j * sT_j;
        for (int n = 0; n < nnz; ++n) {
            if (k2s[n] != k2) continue;
            const float2* Tk = Tb + k1s[n] * sT_k;
            for (int a = 0; a < d; ++a) {
                const cplx w = Ws[(n * d + b) * d + a];
                const float2 t = Tk[a * sT_a];
                ar += w.x * (double)t.x - w.y * (double)t.y;
                ai += w.x * (double)t.y + w.y * (double)t.x;
            }
        }
        float brr, bii, srr, sii;
        split_tf32(ar, brr, srr);
        split_tf32(ai, bii, sii);
        const long long off = 2 * (r * o.s0 + k2 * o.s1 + j * o.s2 + b * o.s3);
        *reinterpret_cast<float2*>(Ub + off) = make_float2(brr, bii);
        *reinterpret_cast<float2*>(Us + off) = make_float2(srr, sii);
    }
}

// Z(x,r,a,k1) = sum_{n: from(n)=k1} sum_b W(a,b,n) Y(x, b, r, k2(n))
// (Y complex64 (bl,d,br,cr)), FP64 accumulation, written as a TF32 pair at
// complex offset x*o.s0 + r*o.s1 + a*o.s2 + k1*o.s3.
__global__ void mix_right_tf32_kernel(int br, int bl, int cl, int cr, int d, int nnz, const uint32_t* __restrict__ idx,
                                      const cplx* __restrict__ W, const float2* __restrict__ Y,
                                      float* __restrict__ Zb, float* __restrict__ Zs, Out4 o) {
    __shared__ cplx Ws[MIXM_MAX_NNZ * MIXM_MAX_D * MIXM_MAX_D];
    __shared__ int k1s[MIXM_MAX_NNZ], k2s[MIXM_MAX_NNZ];
    for (int i = threadIdx.x; i < nnz * d * d; i += blockDim.x) Ws[i] = W[i];
    for (int i = threadIdx.x; i < nnz; i += blockDim.x) {
        k1s[i] = (int)idx[2 * i] - 1;
        k2s[i] = (int)idx[2 * i + 1] - 1;
    }
    __syncthreads();
    const long long total = (long long)bl * br * d * cl;
    const long long sY_b = bl, sY_r = (long long)bl * d, sY_k = (long long)bl * d * br;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long q = e;
        const int x = (int)(q % bl); q /= bl;
        const int r = (int)(q % br); q /= br;
        const int a = (int)(q % d); q /= d;
        const int k1 = (int)q;
        double ar = 0, ai = 0;
        const float2* Yb = Y + x + r * sY_r;
        for (int n = 0; n < nnz; ++n) {
            if (k1s[n] != k1) continue;
            const float2* Yk = Yb + k2s[n] * sY_k;
            for (int b = 0; b < d; ++b) {
                const cplx w = Ws[(n * d + b) * d + a];
                const float2 t = Yk[b * sY_b];
                ar += w.x * (double)t.x - w.y * (double)t.y;
                ai += w.x * (double)t.y + w.y * (double)t.x;
            }
        }
        float brr, bii, srr, sii;
        split_tf32(ar, brr, srr);
        split_tf32(ai, bii, sii);
        const long long off = 2 * (x * o.s0 + r * o.s1 + a * o.s2 + k1 * o.s3);
        *reinterpret_cast<float2*>(Zb + off) = make_float2(brr, bii);
        *reinterpret_cast<float2*>(Zs + off) = make_float2(srr, sii);
    }
}

unsigned grid_for(long long total, int threads) {
    long long g = (total + threads - 1) / threads;
    return (unsigned)std::max<long long>(1, std::min<long long>(g, 148 * 32));
}

}  // namespace

// ---- layout of one MixedHeff buffer ----------------------------------------
namespace {
struct MixedLayout {
    long long ldL, ldR, ldX, ldU;
    size_t oLb, oLs, oRb, oRs, oXb, oXs, oT, oUb, oUs, total;
};
MixedLayout mixed_layout(int bl, int br, const MpoSite& op) {
    MixedLayout s;
    const int d = op.d, cl = op.cl, cr = op.cr;
    s.ldL = round4(2LL * bl);
    s.ldR = round4(2LL * br * cr);
    s.ldX = round4(2LL * bl);
    s.ldU = round4(2LL * br * cr);
    size_t o = 0;
    auto take = [&](size_t n) { size_t r = o; o += align64(n); return r; };
    s.oLb = take((size_t)2 * bl * cl * s.ldL);
    s.oLs = take((size_t)2 * bl * cl * s.ldL);
    s.oRb = take((size_t)2 * br * s.ldR);
    s.oRs = take((size_t)2 * br * s.ldR);
    s.oXb = take((size_t)d * br * s.ldX);
    s.oXs = take((size_t)d * br * s.ldX);
    s.oT = take((size_t)2 * br * bl * cl * d);
    s.oUb = take((size_t)d * bl * s.ldU);
    s.oUs = take((size_t)d * bl * s.ldU);
    s.total = o;
    return s;
}
}  // namespace

size_t mixed_heff_floats(int bl, int br, const MpoSite& op) { return mixed_layout(bl, br, op).total; }

void mixed_heff_prepare(Context& ctx, int bl, int br, const MpoSite& op, const cplx* L, const cplx* R,
                        float* buf, MixedHeff* h) {
    NC_ARG(op.nnz >= 1 && op.nnz <= MIXM_MAX_NNZ && op.d >= 1 && op.d <= MIXM_MAX_D,
           "mixed H_eff: nnz must be in [1,64] and d in [1,4]");
    const MixedLayout s = mixed_layout(bl, br, op);
    h->bl = bl; h->br = br; h->op = op;
    h->ldL = s.ldL; h->ldR = s.ldR; h->ldX = s.ldX; h->ldU = s.ldU;
    h->Lb = buf + s.oLb; h->Ls = buf + s.oLs;
    h->Rb = buf + s.oRb; h->Rs = buf + s.oRs;
    h->Xb = buf + s.oXb; h->Xs = buf + s.oXs;
    h->T = reinterpret_cast<float2*>(buf + s.oT);
    h->Ub = buf + s.oUb; h->Us = buf + s.oUs;
    // L_op: row n = j + bl*k1, K index i: L[i + bl*n]
    split_rows<true>(ctx, bl * op.cl, bl, 1, L, bl, 1, 0, h->Lb, h->Ls, s.ldL, 0);
    // R_op: row n = r', K index k = r + br*k2: R[r' + br*k]
    split_rows<true>(ctx, br, br * op.cr, 1, R, 1, br, 0, h->Rb, h->Rs, s.ldR, 0);
}

void heff_apply_mixed(Context& ctx, const MixedHeff& h, const cplx* x, cplx* y) {
    const int bl = h.bl, br = h.br, d = h.op.d, cl = h.op.cl, cr = h.op.cr;
    // X_op (per a): row r, K index i: x[r + br*i + br*bl*a]
    split_rows<false>(ctx, br, bl, d, x, 1, br, (long long)br * bl, h.Xb, h.Xs, h.ldX, (long long)br * h.ldX);
    TcGemm ga;
    ga.A.big = h.Xb; ga.A.small = h.Xs; ga.A.ld = h.ldX; ga.A.sbatch = (long long)br * h.ldX;
    ga.B.big = h.Lb; ga.B.small = h.Ls; ga.B.ld = h.ldL; ga.B.sbatch = 0;
    ga.M = br; ga.Nr = 2 * bl * cl; ga.Kr = 2 * bl; ga.batch = d;
    ga.C = h.T; ga.sm = 1; ga.sn = br; ga.sz = (long long)br * bl * cl; ga.c_fp64 = false;
    tc_gemm(ctx, ga);
    const long long total = (long long)br * cr * bl * d;
    const Out4 o = {1, br, h.ldU / 2, (long long)bl * (h.ldU / 2)};   // row (b, j), K index r + br*k2
    mix_left_tf32_kernel<<<grid_for(total, 256), 256, 0, ctx.stream>>>(br, bl, cl, cr, d, h.op.nnz, h.op.idx,
                                                                       h.op.W, h.T, h.Ub, h.Us, o);
    NC_CHECK_LAUNCH();
    ctx.launches++;
    TcGemm gc;
    gc.A.big = h.Ub; gc.A.small = h.Us; gc.A.ld = h.ldU; gc.A.sbatch = (long long)bl * h.ldU;
    gc.B.big = h.Rb; gc.B.small = h.Rs; gc.B.ld = h.ldR; gc.B.sbatch = 0;
    gc.M = bl; gc.Nr = 2 * br; gc.Kr = 2 * br * cr; gc.batch = d;
    gc.C = y; gc.sm = br; gc.sn = 1; gc.sz = (long long)br * bl; gc.c_fp64 = true;
    tc_gemm(ctx, gc);
}

void expectation_mixed(Context& ctx, const MixedHeff& h, const cplx* psi, cplx* result) {
    ArenaFrame f(ctx.arena);
    const long long n = (long long)h.br * h.bl * h.op.d;
    cplx* y = ctx.arena.alloc_n<cplx>(n);
    heff_apply_mixed(ctx, h, psi, y);
    zdotc(ctx, n, psi, y, result);
}

// contract_sos_left (core.f95:623-677) in the precision form:
// L'_{k2}(r,r'') = sum_{(j,b)} U(r,k2,j,b) conj(psi(r'',j,b)), U = mix(psi_a L).
void sos_left_mixed(Context& ctx, int bl, int br, const MpoSite& op, const cplx* L, const cplx* psi, cplx* Lnew) {
    NC_ARG(op.nnz >= 1 && op.nnz <= MIXM_MAX_NNZ && op.d >= 1 && op.d <= MIXM_MAX_D,
           "mixed environment: nnz must be in [1,64] and d in [1,4]");
    const int d = op.d, cl = op.cl, cr = op.cr;
    ArenaFrame f(ctx.arena);
    const long long ldL = round4(2LL * bl), ldX = round4(2LL * bl), ldS = round4(2LL * bl * d);
    float* Lb = ctx.arena.alloc_n<float>(align64((size_t)2 * bl * cl * ldL));
    float* Ls = ctx.arena.alloc_n<float>(align64((size_t)2 * bl * cl * ldL));
    float* Xb = ctx.arena.alloc_n<float>(align64((size_t)d * br * ldX));
    float* Xs = ctx.arena.alloc_n<float>(align64((size_t)d * br * ldX));
    float2* T = ctx.arena.alloc_n<float2>(align64((size_t)br * bl * cl * d));
    float* Ub = ctx.arena.alloc_n<float>(align64((size_t)cr * br * ldS));
    float* Us = ctx.arena.alloc_n<float>(align64((size_t)cr * br * ldS));
    float* Pb = ctx.arena.alloc_n<float>(align64((size_t)2 * br * ldS));
    float* Ps = ctx.arena.alloc_n<float>(align64((size_t)2 * br * ldS));
    split_rows<true>(ctx, bl * cl, bl, 1, L, bl, 1, 0, Lb, Ls, ldL, 0);
    split_rows<false>(ctx, br, bl, d, psi, 1, br, (long long)br * bl, Xb, Xs, ldX, (long long)br * ldX);
    TcGemm ga;
    ga.A.big = Xb; ga.A.small = Xs; ga.A.ld = ldX; ga.A.sbatch = (long long)br * ldX;
    ga.B.big = Lb; ga.B.small = Ls; ga.B.ld = ldL; ga.B.sbatch = 0;
    ga.M = br; ga.Nr = 2 * bl * cl; ga.Kr = 2 * bl; ga.batch = d;
    ga.C = T; ga.sm = 1; ga.sn = br; ga.sz = (long long)br * bl * cl; ga.c_fp64 = false;
    tc_gemm(ctx, ga);
    // U_op[k2][r][(j + bl*b)]
    const Out4 o = {ldS / 2, (long long)br * (ldS / 2), 1, bl};
    const long long total = (long long)br * cr * bl * d;
    mix_left_tf32_kernel<<<grid_for(total, 256), 256, 0, ctx.stream>>>(br, bl, cl, cr, d, op.nnz, op.idx, op.W, T,
                                                                       Ub, Us, o);
    NC_CHECK_LAUNCH();
    ctx.launches++;
    // B(k = j + bl*b, r'') = conj(psi[r'' + br*k]): expanded rows r''
    split_rows<true, true>(ctx, br, bl * d, 1, psi, 1, br, 0, Pb, Ps, ldS, 0);
    TcGemm gc;
    gc.A.big = Ub; gc.A.small = Us; gc.A.ld = ldS; gc.A.sbatch = (long long)br * ldS;
    gc.B.big = Pb; gc.B.small = Ps; gc.B.ld = ldS; gc.B.sbatch = 0;
    gc.M = br; gc.Nr = 2 * br; gc.Kr = 2 * bl * d; gc.batch = cr;
    gc.C = Lnew; gc.sm = 1; gc.sn = br; gc.sz = (long long)br * br; gc.c_fp64 = true;
    tc_gemm(ctx, gc);
}

// contract_sos_right (core.f95:679-848) in the precision form:
// Y = Psi^H R, Z = mix_right(Y), R'_{k1}(x,x') = sum_{(r,a)} Z(x,r,a,k1) psi(r,x',a).
void sos_right_mixed(Context& ctx, int bl, int br, const MpoSite& op, const cplx* R, const cplx* psi, cplx* Rnew) {
    NC_ARG(op.nnz >= 1 && op.nnz <= MIXM_MAX_NNZ && op.d >= 1 && op.d <= MIXM_MAX_D,
           "mixed environment: nnz must be in [1,64] and d in [1,4]");
    const int d = op.d, cl = op.cl, cr = op.cr;
    ArenaFrame f(ctx.arena);
    const long long ldA = round4(2LL * br), ldZ = round4(2LL * br * d);
    float* Ab = ctx.arena.alloc_n<float>(align64((size_t)bl * d * ldA));
    float* As = ctx.arena.alloc_n<float>(align64((size_t)bl * d * ldA));
    float* Rb = ctx.arena.alloc_n<float>(align64((size_t)2 * br * cr * ldA));
    float* Rs = ctx.arena.alloc_n<float>(align64((size_t)2 * br * cr * ldA));
    float2* Y = ctx.arena.alloc_n<float2>(align64((size_t)bl * d * br * cr));
    float* Zb = ctx.arena.alloc_n<float>(align64((size_t)cl * bl * ldZ));
    float* Zs = ctx.arena.alloc_n<float>(align64((size_t)cl * bl * ldZ));
    float* Pb = ctx.arena.alloc_n<float>(align64((size_t)2 * bl * ldZ));
    float* Ps = ctx.arena.alloc_n<float>(align64((size_t)2 * bl * ldZ));
    // A(m = x + bl*b, k = r'') = conj(psi[k + br*m]);  B(k = r'', n = r + br*k2) = R[k + br*n]
    split_rows<false, true>(ctx, bl * d, br, 1, psi, br, 1, 0, Ab, As, ldA, 0);
    split_rows<true>(ctx, br * cr, br, 1, R, br, 1, 0, Rb, Rs, ldA, 0);
    TcGemm gy;
    gy.A.big = Ab; gy.A.small = As; gy.A.ld = ldA; gy.A.sbatch = 0;
    gy.B.big = Rb; gy.B.small = Rs; gy.B.ld = ldA; gy.B.sbatch = 0;
    gy.M = bl * d; gy.Nr = 2 * br * cr; gy.Kr = 2 * br; gy.batch = 1;
    gy.C = Y; gy.sm = 1; gy.sn = (long long)bl * d; gy.sz = 0; gy.c_fp64 = false;
    tc_gemm(ctx, gy);
    // Z_op[k1][x][(r + br*a)]
    const Out4 o = {ldZ / 2, 1, br, (long long)bl * (ldZ / 2)};
    const long long total = (long long)bl * br * d * cl;
    mix_right_tf32_kernel<<<grid_for(total, 256), 256, 0, ctx.stream>>>(br, bl, cl, cr, d, op.nnz, op.idx, op.W, Y,
                                                                        Zb, Zs, o);
    NC_CHECK_LAUNCH();
    ctx.launches++;
    // B(k = r + br*a, x') = psi[r + br*x' + br*bl*a]: expanded rows x', one K block of 2*br floats per a
    split_rows<true>(ctx, bl, br, d, psi, br, 1, (long long)br * bl, Pb, Ps, ldZ, 2LL * br);
    TcGemm gr;
    gr.A.big = Zb; gr.A.small = Zs; gr.A.ld = ldZ; gr.A.sbatch = (long long)bl * ldZ;
    gr.B.big = Pb; gr.B.small = Ps; gr.B.ld = ldZ; gr.B.sbatch = 0;
    gr.M = bl; gr.Nr = 2 * bl; gr.Kr = 2 * br * d; gr.batch = cl;
    gr.C = Rnew; gr.sm = 1; gr.sn = bl; gr.sz = (long long)bl * bl; gr.c_fp64 = true;
    tc_gemm(ctx, gr);
}

void tc_zgemm(Context& ctx, int M, int N, int K, const cplx* A, const cplx* B, cplx* C, bool three) {
    NC_ARG(M >= 1 && N >= 1 && K >= 1, "tc_zgemm: empty product");
    ArenaFrame f(ctx.arena);
    const long long lda = round4(2LL * K);
    float* Ab = ctx.arena.alloc_n<float>(align64((size_t)M * lda));
    float* As = ctx.arena.alloc_n<float>(align64((size_t)M * lda));
    float* Bb = ctx.arena.alloc_n<float>(align64((size_t)2 * N * lda));
    float* Bs = ctx.arena.alloc_n<float>(align64((size_t)2 * N * lda));
    split_rows<false>(ctx, M, K, 1, A, 1, M, 0, Ab, As, lda, 0);       // A[m + M*k]
    split_rows<true>(ctx, N, K, 1, B, K, 1, 0, Bb, Bs, lda, 0);        // B[k + K*n]
    TcGemm g;
    g.A.big = Ab; g.A.small = As; g.A.ld = lda;
    g.B.big = Bb; g.B.small = Bs; g.B.ld = lda;
    g.M = M; g.Nr = 2 * N; g.Kr = 2 * K; g.batch = 1;
    g.C = C; g.sm = 1; g.sn = M; g.sz = 0; g.c_fp64 = true; g.three = three;
    tc_gemm(ctx, g);
    tc_check(ctx);
}

}  // namespace nc
