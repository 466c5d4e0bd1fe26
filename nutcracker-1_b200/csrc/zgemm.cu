// Complex128 GEMM on the FP64 tensor pipe (sm_100a).
//
// C[b] = alpha * op(A[b]) * op(B[b]) + beta * C[b], column-major, with a
// two-level batch index b = b0 + nb0 * b1 (independent strides per level),
// op in {N, T, C}.  Blackwell's tcgen05 MMA has no f64 kind, so the FP64
// product runs as warp-level DMMA (mma.sync.m8n8k4.f64): each complex
// multiply-add is four real DMMAs on planar fragments read from
// interleaved (re, im) shared-memory tiles.  Tiles are staged global ->
// shared with 16-byte cp.async (one complex element per copy, zero-filled
// past the matrix edge) through a multi-stage pipeline.
//
// Shared-memory layouts are chosen per operand orientation so that both the
// cp.async stores and the 128-bit fragment loads are bank-conflict free:
//   A, op N : As[k][m] (pitch BM+2)   A, op T/C : As[m][k] (pitch BK+4)
//   B, op N : Bs[n][k] (pitch BK+4)   B, op T/C : Bs[k][n] (pitch BN+2)
#include "nc_common.cuh"
#include "nc_kernels.h"

namespace nc {

namespace {

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int sz = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

template <int BM, int BN, int BK, int WM, int WN, int STAGES, int OPA, int OPB>
struct ZTile {
    static constexpr int NWARPS = (BM / WM) * (BN / WN);
    static constexpr int THREADS = NWARPS * 32;
    static constexpr int MT = WM / 8, NT = WN / 8;
    static constexpr bool A_KM = (OPA == OP_N);
    static constexpr bool B_NK = (OPB == OP_N);
    static constexpr int A_PITCH = A_KM ? (BM + 2) : (BK + 4);
    static constexpr int B_PITCH = B_NK ? (BK + 4) : (BN + 2);
    static constexpr int A_ELEMS = A_KM ? BK * A_PITCH : BM * A_PITCH;
    static constexpr int B_ELEMS = B_NK ? BN * B_PITCH : BK * B_PITCH;
    static constexpr int STAGE_ELEMS = A_ELEMS + B_ELEMS;
    static constexpr size_t SMEM = (size_t)STAGES * STAGE_ELEMS * sizeof(cplx);
    static_assert((BM * BK) % THREADS == 0 && (BN * BK) % THREADS == 0, "tile/threads");
    static_assert(BK % 4 == 0 && WM % 8 == 0 && WN % 8 == 0, "shape");
};

template <int BM, int BN, int BK, int WM, int WN, int STAGES, int OPA, int OPB>
__global__ void __launch_bounds__(ZTile<BM, BN, BK, WM, WN, STAGES, OPA, OPB>::THREADS)
    zgemm_dmma_kernel(ZGemmParams p) {
    typedef ZTile<BM, BN, BK, WM, WN, STAGES, OPA, OPB> T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx* smem = reinterpret_cast<cplx*>(smem_raw);

    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm0 = (warp % (BM / WM)) * WM;
    const int wn0 = (warp / (BM / WM)) * WN;
    const int bm0 = blockIdx.y * BM;
    const int bn0 = blockIdx.x * BN;

    // blockIdx.z = b + batch * ks: batch entry b, K slice ks (split-K)
    const long long b = blockIdx.z % p.batch;
    const int ks = blockIdx.z / p.batch;
    const long long b0 = b % p.nb0, b1 = b / p.nb0;
    const cplx* __restrict__ A = p.A + b0 * p.sA0 + b1 * p.sA1;
    const cplx* __restrict__ B = p.B + b0 * p.sB0 + b1 * p.sB1;
    cplx* __restrict__ C = p.C + b0 * p.sC0 + b1 * p.sC1;
    const int M = p.M, N = p.N;
    int K = p.K;
    long long lda = p.lda, ldb = p.ldb, ldc = p.ldc;
    if (p.kchunk > 0) {
        const long long k0 = (long long)ks * p.kchunk;
        K = (int)min((long long)p.kchunk, (long long)p.K - k0);
        A += k0 * (T::A_KM ? lda : 1);
        B += k0 * (T::B_NK ? 1 : ldb);
        C = p.ws + ((long long)ks * p.batch + b) * (long long)M * N;  // raw partial, ld = M
        ldc = M;
    }
    const bool raw = (p.kchunk > 0);

    auto load_tile = [&](int stage, int kt) {
        cplx* As = smem + stage * T::STAGE_ELEMS;
        cplx* Bs = As + T::A_ELEMS;
        const int k0 = kt * BK;
#pragma unroll
        for (int i = 0; i < (BM * BK) / T::THREADS; ++i) {
            int idx = tid + i * T::THREADS;
            int m, k;
            if (T::A_KM) { m = idx % BM; k = idx / BM; }
            else { k = idx % BK; m = idx / BK; }
            int gm = bm0 + m, gk = k0 + k;
            bool ok = (gm < M) && (gk < K);
            const cplx* src = ok ? (T::A_KM ? A + gm + gk * lda : A + gk + gm * lda) : A;
            cplx* dst = T::A_KM ? As + k * T::A_PITCH + m : As + m * T::A_PITCH + k;
            cp_async16(dst, src, ok);
        }
#pragma unroll
        for (int i = 0; i < (BN * BK) / T::THREADS; ++i) {
            int idx = tid + i * T::THREADS;
            int n, k;
            if (T::B_NK) { k = idx % BK; n = idx / BK; }
            else { n = idx % BN; k = idx / BN; }
            int gn = bn0 + n, gk = k0 + k;
            bool ok = (gn < N) && (gk < K);
            const cplx* src = ok ? (T::B_NK ? B + gk + gn * ldb : B + gn + gk * ldb) : B;
            cplx* dst = T::B_NK ? Bs + n * T::B_PITCH + k : Bs + k * T::B_PITCH + n;
            cp_async16(dst, src, ok);
        }
    };

    double accr[T::MT][T::NT][2], acci[T::MT][T::NT][2];
#pragma unroll
    for (int i = 0; i < T::MT; ++i)
#pragma unroll
        for (int j = 0; j < T::NT; ++j) accr[i][j][0] = accr[i][j][1] = acci[i][j][0] = acci[i][j][1] = 0.0;

    const int ktiles = (K + BK - 1) / BK;
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < ktiles) load_tile(s, s);
        cp_async_commit();
    }

    for (int kt = 0; kt < ktiles; ++kt) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        {
            int nk = kt + STAGES - 1;
            if (nk < ktiles) load_tile(nk % STAGES, nk);
            cp_async_commit();
        }
        const cplx* As = smem + (kt % STAGES) * T::STAGE_ELEMS;
        const cplx* Bs = As + T::A_ELEMS;
#pragma unroll
        for (int kk = 0; kk < BK / 4; ++kk) {
            double ar[T::MT], ai[T::MT], nai[T::MT], br[T::NT], bi[T::NT];
#pragma unroll
            for (int i = 0; i < T::MT; ++i) {
                int m = wm0 + 8 * i + g, k = 4 * kk + t;
                cplx a = T::A_KM ? As[k * T::A_PITCH + m] : As[m * T::A_PITCH + k];
                ar[i] = a.x;
                ai[i] = (OPA == OP_C) ? -a.y : a.y;
                nai[i] = -ai[i];
            }
#pragma unroll
            for (int j = 0; j < T::NT; ++j) {
                int n = wn0 + 8 * j + g, k = 4 * kk + t;
                cplx v = T::B_NK ? Bs[n * T::B_PITCH + k] : Bs[k * T::B_PITCH + n];
                br[j] = v.x;
                bi[j] = (OPB == OP_C) ? -v.y : v.y;
            }
#pragma unroll
            for (int i = 0; i < T::MT; ++i)
#pragma unroll
                for (int j = 0; j < T::NT; ++j) {
                    dmma(accr[i][j], ar[i], br[j]);
                    dmma(accr[i][j], nai[i], bi[j]);
                    dmma(acci[i][j], ar[i], bi[j]);
                    dmma(acci[i][j], ai[i], br[j]);
                }
        }
    }
    cp_async_wait<0>();

    const cplx alpha = raw ? cmake(1, 0) : p.alpha, beta = p.beta;
    const bool use_beta = !raw && (beta.x != 0.0 || beta.y != 0.0);
#pragma unroll
    for (int i = 0; i < T::MT; ++i) {
        int m = bm0 + wm0 + 8 * i + g;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < T::NT; ++j) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                int n = bn0 + wn0 + 8 * j + 2 * t + q;
                if (n >= N) continue;
                cplx v = cmul(alpha, cmake(accr[i][j][q], acci[i][j][q]));
                cplx* dst = C + m + (long long)n * ldc;
                if (use_beta) v = cadd(v, cmul(beta, *dst));
                *dst = v;
            }
        }
    }
}

template <int BM, int BN, int BK, int WM, int WN, int STAGES, int OPA, int OPB>
void launch_cfg(const ZGemmParams& p, cudaStream_t s) {
    typedef ZTile<BM, BN, BK, WM, WN, STAGES, OPA, OPB> T;
    auto kern = zgemm_dmma_kernel<BM, BN, BK, WM, WN, STAGES, OPA, OPB>;
    NC_SET_SMEM_ONCE(kern, T::SMEM);
    dim3 grid(ceil_div(p.N, BN), ceil_div(p.M, BM), p.batch * p.nsplit);
    NC_ARG((long long)p.batch * p.nsplit <= 65535, "zgemm: batch too large");
    kern<<<grid, T::THREADS, T::SMEM, s>>>(p);
    NC_CHECK_LAUNCH();
}

template <int OPA, int OPB>
void launch_ops(const ZGemmParams& p, cudaStream_t s) {
    // Large problems: 128x64 tiles, 8 warps; small ones: 64x64, 4 warps.
    long long tiles128 = (long long)ceil_div(p.M, 128) * ceil_div(p.N, 64) * p.batch * p.nsplit;
    if (p.M >= 128 && tiles128 >= 148)
        launch_cfg<128, 64, 16, 32, 32, 3, OPA, OPB>(p, s);
    else
        launch_cfg<64, 64, 16, 32, 32, 3, OPA, OPB>(p, s);
}

// C[b] = alpha * sum_ks ws[ks][b] + beta * C[b]
__global__ void splitk_reduce_kernel(ZGemmParams p) {
    const long long b = blockIdx.z;
    cplx* C = p.C + (b % p.nb0) * p.sC0 + (b / p.nb0) * p.sC1;
    const long long mn = (long long)p.M * p.N;
    const bool use_beta = (p.beta.x != 0.0 || p.beta.y != 0.0);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < mn;
         e += (long long)gridDim.x * blockDim.x) {
        cplx acc = cmake(0, 0);
        for (int ks = 0; ks < p.nsplit; ++ks) acc = cadd(acc, p.ws[((long long)ks * p.batch + b) * mn + e]);
        int m = (int)(e % p.M), n = (int)(e / p.M);
        cplx* d = C + m + (long long)n * p.ldc;
        cplx v = cmul(p.alpha, acc);
        if (use_beta) v = cadd(v, cmul(p.beta, *d));
        *d = v;
    }
}

}  // namespace

namespace {
void zgemm_ctx(const ZGemmParams& p_in, Context& ctx);
}

void zgemm(const ZGemmParams& p, Context& ctx) {
    const double flops = 8.0 * p.M * (double)p.N * p.K * p.batch;
    profile_launch(ctx, flops, 0, [&] { zgemm_ctx(p, ctx); });
}

namespace {
void zgemm_ctx(const ZGemmParams& p_in, Context& ctx) {
    ZGemmParams p = p_in;
    if (p.M <= 0 || p.N <= 0 || p.batch <= 0) return;
    if (p.nb0 <= 0) p.nb0 = p.batch;
    // Split K when the tile grid cannot fill the 148 SMs and K is long.
    const long long tiles = (long long)ceil_div(p.M, 64) * ceil_div(p.N, 64) * p.batch;
    int nsplit = 1;
    if (p.K >= 256 && tiles < 2 * 148) {
        nsplit = (int)std::min<long long>((2 * 148 + tiles - 1) / tiles, p.K / 128);
        nsplit = std::max(1, std::min(nsplit, 32));
    }
    if (nsplit <= 1) {
        zgemm(p, ctx.stream);
        ctx.launches++;
        return;
    }
    int kchunk = (int)(((p.K + nsplit - 1) / nsplit + 15) / 16 * 16);
    nsplit = (p.K + kchunk - 1) / kchunk;
    ArenaFrame f(ctx.scratch());
    const long long mn = (long long)p.M * p.N;
    cplx* ws = ctx.scratch().alloc_n<cplx>((size_t)mn * p.batch * nsplit);
    ZGemmParams q = p;
    q.kchunk = kchunk;
    q.nsplit = nsplit;
    q.ws = ws;
    zgemm(q, ctx.stream);
    ZGemmParams r = p;
    r.nsplit = nsplit;
    r.ws = ws;
    dim3 grid(std::min<unsigned>(ceil_div((size_t)mn, 256), 1024), 1, p.batch);
    splitk_reduce_kernel<<<grid, 256, 0, ctx.stream>>>(r);
    NC_CHECK_LAUNCH();
    ctx.launches += 2;
}
}  // namespace

void zgemm(const ZGemmParams& p_in, cudaStream_t s) {
    ZGemmParams p = p_in;
    if (p.M <= 0 || p.N <= 0 || p.batch <= 0) return;
    if (p.nb0 <= 0) p.nb0 = p.batch;  // single-level batch: every index on level 0
    if (p.nsplit <= 0 || p.kchunk <= 0) { p.nsplit = 1; p.kchunk = 0; }
    if (p.K <= 0) {
        // C = beta * C
        scale_strided(p, s);
        return;
    }
#define NC_OPS(a, b) \
    if (p.opA == a && p.opB == b) { launch_ops<a, b>(p, s); return; }
    NC_OPS(OP_N, OP_N) NC_OPS(OP_N, OP_T) NC_OPS(OP_N, OP_C)
    NC_OPS(OP_T, OP_N) NC_OPS(OP_T, OP_T) NC_OPS(OP_T, OP_C)
    NC_OPS(OP_C, OP_N) NC_OPS(OP_C, OP_T) NC_OPS(OP_C, OP_C)
#undef NC_OPS
    throw Error(NC_ERR_ARG, "zgemm: bad op");
}

namespace {
__global__ void scale_strided_kernel(ZGemmParams p) {
    const long long b = blockIdx.z;
    cplx* C = p.C + (b % p.nb0) * p.sC0 + (b / p.nb0) * p.sC1;
    long long total = (long long)p.M * p.N;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int m = (int)(e % p.M), n = (int)(e / p.M);
        cplx* d = C + m + (long long)n * p.ldc;
        *d = (p.beta.x == 0.0 && p.beta.y == 0.0) ? cmake(0, 0) : cmul(p.beta, *d);
    }
}
}  // namespace

void scale_strided(const ZGemmParams& p_in, cudaStream_t s) {
    ZGemmParams p = p_in;
    if (p.nb0 <= 0) p.nb0 = p.batch;
    dim3 grid(std::min<unsigned>(ceil_div((size_t)p.M * p.N, 256), 4096), 1, p.batch);
    scale_strided_kernel<<<grid, 256, 0, s>>>(p);
    NC_CHECK_LAUNCH();
}

ZGemmParams zgemm_params(int opA, int opB, int M, int N, int K, const cplx* A, long long lda,
                         const cplx* B, long long ldb, cplx* C, long long ldc) {
    ZGemmParams p;
    p.opA = opA; p.opB = opB;
    p.M = M; p.N = N; p.K = K;
    p.A = A; p.lda = lda; p.sA0 = 0; p.sA1 = 0;
    p.B = B; p.ldb = ldb; p.sB0 = 0; p.sB1 = 0;
    p.C = C; p.ldc = ldc; p.sC0 = 0; p.sC1 = 0;
    p.nb0 = 0; p.batch = 1;  // nb0 = 0: single-level batch over the *0 strides
    p.alpha = cmake(1, 0); p.beta = cmake(0, 0);
    p.kchunk = 0; p.nsplit = 1; p.ws = nullptr;
    return p;
}

}  // namespace nc
