// Sparse-MPO contractions: the effective-Hamiltonian product and the
// environment updates, as grouped complex GEMMs plus an HBM-bound sparse mix.
//
// Notation (all column-major, reference layouts):
//   L (bl,bl,cl)  left environment, L(i=ket, j=bra, k)
//   R (br,br,cr)  right environment, R(r'=bra, r=ket, k)
//   psi (br,bl,d) site, psi_a = psi(:,:,a) is a br x bl matrix
//   W (d,d,nnz)   MPO blocks, idx(1,n)=k1 (from), idx(2,n)=k2 (to)
//
// H_eff psi (core.f95:2529-2556 restated):
//   out_b = sum_n W_n(a,b) R_{k2} psi_a L_{k1}
// is evaluated as
//   A: T_a   = psi_a * [L_1 | ... | L_cl]          (GEMM br x bl*cl x bl, batch d)
//   B: U_k2b = sum_{n: to=k2} sum_a W_n(a,b) T_{k1 a} (sparse mix, HBM-bound)
//   C: out_b = [R_1 | ... | R_cr] * [U_1b; ...]    (GEMM br x bl x br*cr, batch d)
// so the reference's dense (bl,d,cr,bl,d) stage-1 tensor is never formed.
// contract_sos_left shares A and B and ends with L'_{k2} = U_{k2} Psi^H;
// contract_sos_right runs Psi^H R, a mix over (from) indices, and a batched
// GEMM against a (r,a,l)-permuted copy of psi.
#include "nc_common.cuh"
#include "nc_kernels.h"

namespace nc {

namespace {

constexpr int MIX_MAX_NNZ = 64;
constexpr int MIX_MAX_D = 4;

// U(r,k2,j,b) = sum_{n: to(n)=k2} sum_a W(a,b,n) T(r,j,k1(n),a)
__global__ void mix_left_kernel(int br, int bl, int cl, int cr, int d, int nnz,
                                const uint32_t* __restrict__ idx, const cplx* __restrict__ W,
                                const cplx* __restrict__ T, cplx* __restrict__ U) {
    __shared__ cplx Ws[MIX_MAX_NNZ * MIX_MAX_D * MIX_MAX_D];
    __shared__ int k1s[MIX_MAX_NNZ], k2s[MIX_MAX_NNZ];
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
        int r = (int)(q % br); q /= br;
        int k2 = (int)(q % cr); q /= cr;
        int j = (int)(q % bl); q /= bl;
        int b = (int)q;
        cplx acc = cmake(0, 0);
        const cplx* Tb = T + r + j * sT_j;
        for (int n = 0; n < nnz; ++n) {
            if (k2s[n] != k2) continue;
            const cplx* Tk = Tb + k1s[n] * sT_k;
            for (int a = 0; a < d; ++a) {
                cplx w = Ws[(n * d + b) * d + a];
                cplx tv = Tk[a * sT_a];
                acc = cadd(acc, cmul(w, tv));
            }
        }
        U[e] = acc;
    }
}

// Z(x,r,a,k1) = sum_{n: from(n)=k1} sum_b W(a,b,n) Y(x,b,r,k2(n)),
// Y (bl,d,br,cr), Z (bl,br,d,cl).
__global__ void mix_right_kernel(int br, int bl, int cl, int cr, int d, int nnz,
                                 const uint32_t* __restrict__ idx, const cplx* __restrict__ W,
                                 const cplx* __restrict__ Y, cplx* __restrict__ Z) {
    __shared__ cplx Ws[MIX_MAX_NNZ * MIX_MAX_D * MIX_MAX_D];
    __shared__ int k1s[MIX_MAX_NNZ], k2s[MIX_MAX_NNZ];
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
        int x = (int)(q % bl); q /= bl;
        int r = (int)(q % br); q /= br;
        int a = (int)(q % d); q /= d;
        int k1 = (int)q;
        cplx acc = cmake(0, 0);
        const cplx* Yb = Y + x + r * sY_r;
        for (int n = 0; n < nnz; ++n) {
            if (k1s[n] != k1) continue;
            const cplx* Yk = Yb + k2s[n] * sY_k;
            for (int b = 0; b < d; ++b) {
                cplx w = Ws[(n * d + b) * d + a];
                acc = cadd(acc, cmul(w, Yk[b * sY_b]));
            }
        }
        Z[e] = acc;
    }
}

unsigned grid_for(long long total, int threads) {
    long long g = (total + threads - 1) / threads;
    if (g > 148 * 32) g = 148 * 32;
    if (g < 1) g = 1;
    return (unsigned)g;
}

void check_op(const MpoSite& op) {
    NC_ARG(op.nnz >= 1 && op.nnz <= MIX_MAX_NNZ, "MPO site: nnz must be in [1, 64]");
    NC_ARG(op.d >= 1 && op.d <= MIX_MAX_D, "MPO site: physical dimension must be in [1, 4]");
    NC_ARG(op.cl >= 1 && op.cr >= 1, "MPO site: bond dimensions must be >= 1");
}

void mix_left(Context& ctx, int bl, int br, const MpoSite& op, const cplx* T, cplx* U) {
    long long total = (long long)br * op.cr * bl * op.d;
    mix_left_kernel<<<grid_for(total, 256), 256, 0, ctx.stream>>>(br, bl, op.cl, op.cr, op.d, op.nnz,
                                                                   op.idx, op.W, T, U);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

// Step A of H_eff / sos_left: T(r,j,k1,a) = sum_i psi(r,i,a) L(i,j,k1)
void stage_a(Context& ctx, int bl, int br, const MpoSite& op, const cplx* L, const cplx* psi,
             cplx* T) {
    ZGemmParams p = zgemm_params(OP_N, OP_N, br, bl * op.cl, bl, psi, br, L, bl, T, br);
    p.batch = op.d;
    p.sA0 = (long long)br * bl; p.sB0 = 0; p.sC0 = (long long)br * bl * op.cl;
    zgemm(p, ctx);
}

}  // namespace

size_t heff_workspace_elems(int bl, int br, const MpoSite& op) {
    return (size_t)br * bl * op.cl * op.d + (size_t)br * op.cr * bl * op.d;
}

void heff_apply(Context& ctx, int bl, int br, const MpoSite& op, const cplx* L, const cplx* R,
                const cplx* x, cplx* y, cplx* ws) {
    check_op(op);
    cplx* T = ws;
    cplx* U = ws + (size_t)br * bl * op.cl * op.d;
    stage_a(ctx, bl, br, op, L, x, T);
    mix_left(ctx, bl, br, op, T, U);
    // out_b = Rhat (br x br*cr) * Uhat_b (br*cr x bl)
    ZGemmParams p = zgemm_params(OP_N, OP_N, br, bl, br * op.cr, R, br, U, (long long)br * op.cr, y, br);
    p.batch = op.d;
    p.sA0 = 0; p.sB0 = (long long)br * op.cr * bl; p.sC0 = (long long)br * bl;
    zgemm(p, ctx);
}

void heff_apply_stream(cudaStream_t s, int bl, int br, const MpoSite& op, const cplx* L, const cplx* R,
                       const cplx* x, cplx* y, cplx* ws) {
    // Same three steps as heff_apply, launched directly on `s` with the
    // caller's scratch `ws` and no split-K (nothing is allocated).
    check_op(op);
    cplx* T = ws;
    cplx* U = ws + (size_t)br * bl * op.cl * op.d;
    ZGemmParams a = zgemm_params(OP_N, OP_N, br, bl * op.cl, bl, x, br, L, bl, T, br);
    a.batch = op.d;
    a.sA0 = (long long)br * bl; a.sB0 = 0; a.sC0 = (long long)br * bl * op.cl;
    zgemm(a, s);
    long long total = (long long)br * op.cr * bl * op.d;
    mix_left_kernel<<<grid_for(total, 256), 256, 0, s>>>(br, bl, op.cl, op.cr, op.d, op.nnz, op.idx, op.W, T, U);
    NC_CHECK_LAUNCH();
    ZGemmParams c = zgemm_params(OP_N, OP_N, br, bl, br * op.cr, R, br, U, (long long)br * op.cr, y, br);
    c.batch = op.d;
    c.sA0 = 0; c.sB0 = (long long)br * op.cr * bl; c.sC0 = (long long)br * bl;
    zgemm(c, s);
}

void sos_left(Context& ctx, int bl, int br, const MpoSite& op, const cplx* L, const cplx* psi,
              cplx* Lnew) {
    check_op(op);
    ArenaFrame f(ctx.arena);
    cplx* ws = ctx.arena.alloc_n<cplx>(heff_workspace_elems(bl, br, op));
    cplx* T = ws;
    cplx* U = ws + (size_t)br * bl * op.cl * op.d;
    stage_a(ctx, bl, br, op, L, psi, T);
    mix_left(ctx, bl, br, op, T, U);
    // L'_{k2}(r,r'') = sum_{(j,b)} U(r,k2,j,b) conj(psi(r'',j,b))
    ZGemmParams p = zgemm_params(OP_N, OP_C, br, br, bl * op.d, U, (long long)br * op.cr, psi, br, Lnew, br);
    p.batch = op.cr;
    p.sA0 = br; p.sB0 = 0; p.sC0 = (long long)br * br;
    zgemm(p, ctx);
}

void sos_right(Context& ctx, int bl, int br, const MpoSite& op, const cplx* R, const cplx* psi,
               cplx* Rnew) {
    check_op(op);
    const int d = op.d;
    ArenaFrame f(ctx.arena);
    cplx* Y = ctx.arena.alloc_n<cplx>((size_t)bl * d * br * op.cr);
    cplx* Z = ctx.arena.alloc_n<cplx>((size_t)bl * br * d * op.cl);
    cplx* Pp = ctx.arena.alloc_n<cplx>((size_t)br * d * bl);
    // Y(x,b,r,k2) = sum_r'' conj(psi(r'',x,b)) R(r'',r,k2)
    ZGemmParams p = zgemm_params(OP_C, OP_N, bl * d, br * op.cr, br, psi, br, R, br, Y, (long long)bl * d);
    zgemm(p, ctx);
    long long total = (long long)bl * br * d * op.cl;
    mix_right_kernel<<<grid_for(total, 256), 256, 0, ctx.stream>>>(br, bl, op.cl, op.cr, d, op.nnz,
                                                                    op.idx, op.W, Y, Z);
    NC_CHECK_LAUNCH();
    ctx.launches++;
    // Pp(r,a,y) = psi(r,y,a)
    const int perm[3] = {0, 2, 1};
    permute3(ctx, psi, br, bl, d, perm, false, Pp);
    // R'_{k1} = Z_{k1} (bl x br*d) * Pp (br*d x bl)
    ZGemmParams q = zgemm_params(OP_N, OP_N, bl, bl, br * d, Z, bl, Pp, (long long)br * d, Rnew, bl);
    q.batch = op.cl;
    q.sA0 = (long long)bl * br * d; q.sB0 = 0; q.sC0 = (long long)bl * bl;
    zgemm(q, ctx);
}

void vs_left(Context& ctx, int blo, int bro, int bln, int brn, int d, const cplx* Lov,
             const cplx* P, const cplx* S, cplx* out) {
    // core.f95:850-896
    ArenaFrame f(ctx.arena);
    cplx* I = ctx.arena.alloc_n<cplx>((size_t)bln * d * bro);
    zgemm(zgemm_params(OP_N, OP_N, bln, d * bro, blo, Lov, bln, P, blo, I, bln), ctx);
    zgemm(zgemm_params(OP_N, OP_N, brn, bro, bln * d, S, brn, I, (long long)bln * d, out, brn), ctx);
}

void vs_right(Context& ctx, int blo, int bro, int bln, int brn, int d, const cplx* Rov,
              const cplx* P, const cplx* S, cplx* out) {
    // core.f95:898-952
    ArenaFrame f(ctx.arena);
    cplx* I = ctx.arena.alloc_n<cplx>((size_t)blo * d * brn);
    cplx* Ts = ctx.arena.alloc_n<cplx>((size_t)d * brn * bln);
    zgemm(zgemm_params(OP_N, OP_N, blo * d, brn, bro, P, (long long)blo * d, Rov, bro, I, (long long)blo * d),
          ctx);
    const int perm[3] = {2, 0, 1};  // Ts(s,r,l) = S(r,l,s)
    permute3(ctx, S, brn, bln, d, perm, false, Ts);
    zgemm(zgemm_params(OP_N, OP_N, blo, bln, d * brn, I, blo, Ts, (long long)d * brn, out, blo), ctx);
}

void overlap_vector(Context& ctx, int blo, int bro, int bln, int brn, int d, const cplx* Lov,
                    const cplx* Rov, const cplx* P, cplx* out) {
    // core.f95:954-1005
    ArenaFrame f(ctx.arena);
    cplx* I = ctx.arena.alloc_n<cplx>((size_t)blo * d * brn);
    cplx* T = ctx.arena.alloc_n<cplx>((size_t)bln * d * brn);
    zgemm(zgemm_params(OP_N, OP_N, blo * d, brn, bro, P, (long long)blo * d, Rov, bro, I, (long long)blo * d),
          ctx);
    zgemm(zgemm_params(OP_N, OP_N, bln, d * brn, blo, Lov, bln, I, blo, T, bln), ctx);
    const int perm[3] = {2, 0, 1};  // out(r,l,s) = T(l,s,r)
    permute3(ctx, T, bln, d, brn, perm, false, out);
}

void overlap_site_from_state(Context& ctx, int br, int bl, int d, const cplx* S, cplx* out) {
    // core.f95:3299-3313: out(l,s,r) = conj(S(r,l,s))
    const int perm[3] = {1, 2, 0};
    permute3(ctx, S, br, bl, d, perm, true, out);
}

namespace {
__global__ void exp_boundaries_partial(int b, int c, const cplx* __restrict__ L,
                                       const cplx* __restrict__ R, cplx* __restrict__ part) {
    __shared__ double sr[256], si[256];
    const long long total = (long long)b * b * c;
    double ar = 0, ai = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long q = e;
        int i = (int)(q % b); q /= b;
        int j = (int)(q % b); q /= b;
        int k = (int)q;
        cplx v = cmul(L[j + (long long)b * (i + (long long)b * k)], R[e]);
        ar += v.x; ai += v.y;
    }
    sr[threadIdx.x] = ar; si[threadIdx.x] = ai;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) { sr[threadIdx.x] += sr[threadIdx.x + s]; si[threadIdx.x] += si[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = cmake(sr[0], si[0]);
}
__global__ void sum_partials(int n, const cplx* __restrict__ part, cplx* __restrict__ out) {
    __shared__ double sr[256], si[256];
    double ar = 0, ai = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) { ar += part[i].x; ai += part[i].y; }
    sr[threadIdx.x] = ar; si[threadIdx.x] = ai;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) { sr[threadIdx.x] += sr[threadIdx.x + s]; si[threadIdx.x] += si[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = cmake(sr[0], si[0]);
}
}  // namespace

void contract_exp_boundaries(Context& ctx, int b, int c, const cplx* L, const cplx* R, cplx* result) {
    ArenaFrame f(ctx.arena);
    const int blocks = 256;
    cplx* part = ctx.arena.alloc_n<cplx>(blocks);
    exp_boundaries_partial<<<blocks, 256, 0, ctx.stream>>>(b, c, L, R, part);
    NC_CHECK_LAUNCH();
    sum_partials<<<1, 256, 0, ctx.stream>>>(blocks, part, result);
    NC_CHECK_LAUNCH();
    ctx.launches += 2;
}

}  // namespace nc
