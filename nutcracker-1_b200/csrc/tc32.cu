// Complex GEMM on the 5th-generation tensor cores in 3xTF32 (sm_100a).
//
// The precision form of the H_eff product and the environment updates runs
// its complex contractions here.  A complex product C = A B (K complex terms)
// is one real GEMM with K_r = 2K:
//   A_r(m, 2k + {0,1}) = (Re, Im) A(m,k)              (interleaved complex64)
//   B_r(2n,   2k + {0,1}) = (Re, -Im) B(k,n)          (conjugate row)
//   B_r(2n+1, 2k + {0,1}) = (Im,  Re) B(k,n)          (swapped row)
//   D(m, 2n) = Re C(m,n),  D(m, 2n+1) = Im C(m,n)
// so D = A_r B_r^T with both operands K-major.  Every operand is held as a
// TF32 pair x = big + small (big = rna_tf32(x), small = rna_tf32(x - big))
// and the product runs as three K-segments (A_big, B_big), (A_big, B_small),
// (A_small, B_big) accumulating in FP32 in tensor memory: the 3xTF32
// scheme, which keeps roughly FP32 accuracy while every multiply is TF32.
//
// Kernel: one CTA per 128 x 256 tile of D (tcgen05.mma.cta_group::1,
// kind::tf32, M=128, N=256, K=8 per instruction), K staged 32 floats at a
// time through a 4-deep TMA ring (128-byte swizzle, one mbarrier pair per
// stage).  The tensor core's FP32 accumulation error grows linearly with the
// number of terms (measured on B200: ~2e-8 relative per complex term), so K
// is accumulated in chunks of CHUNK_KB stages per segment (the three
// segments interleaved inside a chunk) in two alternating 256-column TMEM
// buffers; while the MMAs fill one buffer, eight epilogue warps drain the
// other (tcgen05.ld 32x32b, two warps per 32-lane quadrant, 128 columns
// each) and add it into FP32 registers with round-to-nearest adds.  Warp 0
// issues the TMA loads, warp 1 owns TMEM and issues the MMAs from one
// thread.  The epilogue stores complex64 or complex128 to any strided
// layout.  No multicast; every mbarrier wait is bounded by the global timer
// and reports through g_tc_error.
#include <cuda.h>

#include <cstring>
#include <string>

#include "nc_common.cuh"
#include "nc_kernels.h"

namespace nc {

namespace {

constexpr int TM = 128;              // D rows per tile
constexpr int TN = 256;              // D real columns per tile (128 complex)
constexpr int TK = 32;               // floats of K per stage (128 bytes: one swizzle row)
constexpr int STAGES = 4;
constexpr int A_STAGE = TM * TK * 4;  // 16 KiB
constexpr int B_STAGE = TN * TK * 4;  // 32 KiB
constexpr int STAGE_BYTES = A_STAGE + B_STAGE;
constexpr int EPI_WARPS = 8;
constexpr int TC_THREADS = 64 + 32 * EPI_WARPS;
constexpr int TMEM_COLS = 512;       // two accumulator buffers of TN columns
constexpr int CHUNK_KB = 2;          // K stages (per segment) per accumulator chunk
constexpr size_t TC_SMEM = (size_t)STAGES * STAGE_BYTES + 1024 + 256;

__device__ int g_tc_error = 0;
// Limit of every mbarrier wait (2 s by default), and a test switch under
// which tile (0,0,0) leaves its first K stage unloaded, so that its MMA
// issuer's wait for that stage runs out and the failure path (g_tc_error,
// NC_ERR_TIMEOUT on the host) can be exercised without a fault: every other
// wait is bounded as well, no MMA has been issued, and the loads that were
// issued complete long before the waits expire.  Both are set only by
// tc_test_fault (nc_test_tc32_wait).
__device__ unsigned long long g_tc_wait_ns = 2000000000ull;
__device__ int g_tc_skip_first_load = 0;

struct TcParams {
    int M, Nr, Kr, nkb;      // nkb: K stages per segment
    int nseg;                // 3 (3xTF32) or 1 (big x big)
    int shareA, shareB;      // operand shared across the batch (TMA batch coordinate 0)
    void* C;
    long long sm, sn, sz;
    int c_fp64;
};

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false (and g_tc_error set) when the phase did not complete in `limit` ns.
__device__ __noinline__ bool mbar_wait(uint32_t bar, uint32_t parity, unsigned long long limit) {
    if (mbar_test(bar, parity)) return true;
    const unsigned long long t0 = gtimer();
    while (!mbar_test(bar, parity)) {
        if (gtimer() - t0 > limit) {
            atomicExch(&g_tc_error, 1);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

// K-major operand tile in the 128-byte-swizzled layout written by TMA:
// 8-row x 128-byte atoms, 1024 bytes apart (SBO); LBO unused for this layout.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// kind::tf32 instruction descriptor: D f32, A/B tf32, both K-major, M x N.
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TN >> 3) << 17) |
                           ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(IDESC), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
          "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
          "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__global__ void __launch_bounds__(TC_THREADS, 1)
tc32_gemm_kernel(const __grid_constant__ CUtensorMap mapAb, const __grid_constant__ CUtensorMap mapAs,
                 const __grid_constant__ CUtensorMap mapBb, const __grid_constant__ CUtensorMap mapBs,
                 TcParams P) {
    extern __shared__ unsigned char tc_smem_raw[];
    const uint32_t raw = su32(tc_smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;              // 1024-aligned for the 128B swizzle
    // full[S], empty[S], acc_full[2], acc_empty[2], TMEM slot
    const uint32_t bars = base + STAGES * STAGE_BYTES;
    const uint32_t full0 = bars, empty0 = bars + 8 * STAGES;
    const uint32_t accf0 = bars + 16 * STAGES, acce0 = accf0 + 16;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tc_smem_raw + (acce0 + 16 - raw));

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN, z = blockIdx.z;
    const unsigned long long limit = g_tc_wait_ns;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(accf0 + 8 * b, 1);
            mbar_init(acce0 + 8 * b, EPI_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem_d = *tmem_slot;
    // Stage sequence: chunk c covers K stages [c*CHUNK_KB, (c+1)*CHUNK_KB) of
    // every segment; step t of the flat sequence -> (chunk, segment, stage).
    const int nchunk = (P.nkb + CHUNK_KB - 1) / CHUNK_KB;

    if (warp == 0) {
        if (lane == 0) {
            const int zA = P.shareA ? 0 : z, zB = P.shareB ? 0 : z;
            const bool skip_first = g_tc_skip_first_load && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0;
            int t = 0;
            bool ok = true;
            for (int c = 0; c < nchunk && ok; ++c) {
                const int kb0 = c * CHUNK_KB, kb1 = min(P.nkb, kb0 + CHUNK_KB);
                for (int seg = 0; seg < P.nseg && ok; ++seg)
                    for (int kb = kb0; kb < kb1; ++kb, ++t) {
                        const int s = t % STAGES;
                        const uint32_t ph = (uint32_t)(t / STAGES) & 1u;
                        if (!mbar_wait(empty0 + 8 * s, ph ^ 1u, limit)) { ok = false; break; }
                        if (skip_first && t == 0) continue;   // test switch: stage 0 never arrives
                        const CUtensorMap* ma = (seg == 2) ? &mapAs : &mapAb;
                        const CUtensorMap* mb = (seg == 1) ? &mapBs : &mapBb;
                        mbar_expect_tx(full0 + 8 * s, STAGE_BYTES);
                        tma_load_3d(base + s * STAGE_BYTES, ma, kb * TK, m0, zA, full0 + 8 * s);
                        tma_load_3d(base + s * STAGE_BYTES + A_STAGE, mb, kb * TK, n0, zB, full0 + 8 * s);
                    }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int t = 0;
            bool ok = true;
            for (int c = 0; c < nchunk && ok; ++c) {
                const int b = c & 1;
                const uint32_t acc = tmem_d + (uint32_t)(b * TN);
                if (!mbar_wait(acce0 + 8 * b, ((uint32_t)(c >> 1) & 1u) ^ 1u, limit)) break;   // buffer drained
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const int kb0 = c * CHUNK_KB, kb1 = min(P.nkb, kb0 + CHUNK_KB);
                bool first = true;
                for (int seg = 0; seg < P.nseg && ok; ++seg)
                    for (int kb = kb0; kb < kb1; ++kb, ++t) {
                        const int s = t % STAGES;
                        const uint32_t ph = (uint32_t)(t / STAGES) & 1u;
                        if (!mbar_wait(full0 + 8 * s, ph, limit)) { ok = false; break; }
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        const uint64_t da = smem_desc(base + s * STAGE_BYTES);
                        const uint64_t db = smem_desc(base + s * STAGE_BYTES + A_STAGE);
#pragma unroll
                        for (int ks = 0; ks < TK / 8; ++ks) {   // 8 tf32 = 32 bytes per instruction
                            mma_tf32(acc, da + 2 * ks, db + 2 * ks, first ? 0u : 1u);
                            first = false;
                        }
                        mma_commit(empty0 + 8 * s);   // frees the stage once these MMAs have read it
                    }
                mma_commit(accf0 + 8 * b);   // chunk complete in buffer b
            }
        }
    } else {
        // epilogue: warp w drains TMEM lanes 32*(w%4) .. +31 (rows of D),
        // columns [128*h, 128*h + 128) of each buffer, h = (w-2)/4
        const int q = warp & 3, h = (warp - 2) >> 2;
        const int row = q * 32 + lane, m = m0 + row;
        float acc[TN / 2];
#pragma unroll
        for (int i = 0; i < TN / 2; ++i) acc[i] = 0.f;
        bool ok = true;
        for (int c = 0; c < nchunk; ++c) {
            const int b = c & 1;
            ok = __all_sync(0xffffffffu, mbar_wait(accf0 + 8 * b, (uint32_t)(c >> 1) & 1u, limit));   // warp-uniform
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int i = 0; i < TN / 64; ++i) {
                uint32_t v[32];
                tmem_ld32(tmem_d + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * TN + h * (TN / 2) + 32 * i), v);
#pragma unroll
                for (int e = 0; e < 32; ++e) acc[32 * i + e] += __uint_as_float(v[e]);
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(acce0 + 8 * b) : "memory");
        }
        if (ok && m < P.M) {
            const int nc0 = (n0 + h * (TN / 2)) / 2;   // complex column of acc[0], acc[1]
            const long long off = (long long)z * P.sz + (long long)m * P.sm;
#pragma unroll
            for (int e = 0; e < TN / 4; ++e) {
                const int n = nc0 + e;
                if (2 * n < P.Nr) {
                    const long long o = off + (long long)n * P.sn;
                    if (P.c_fp64) reinterpret_cast<double2*>(P.C)[o] = make_double2(acc[2 * e], acc[2 * e + 1]);
                    else reinterpret_cast<float2*>(P.C)[o] = make_float2(acc[2 * e], acc[2 * e + 1]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(TMEM_COLS)
                     : "memory");
    }
}

using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn() {
    static EncodeFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        NC_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (!p || q != cudaDriverEntryPointSuccess)
            throw Error(NC_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
        fn = reinterpret_cast<EncodeFn>(p);
    }
    return fn;
}

// rows x Kr floats (Kr contiguous, row stride ld floats), batch planes sbatch floats apart.
CUtensorMap make_map(const float* ptr, int Kr, int rows, long long ld, long long sbatch, int batch,
                     int box_rows) {
    NC_ARG(((uintptr_t)ptr & 15) == 0, "tc32: operand base must be 16-byte aligned");
    NC_ARG(ld % 4 == 0 && ld >= Kr, "tc32: operand row stride must be a multiple of 4 floats and >= Kr");
    NC_ARG(batch == 1 || sbatch % 4 == 0, "tc32: operand batch stride must be a multiple of 4 floats");
    CUtensorMap m;
    std::memset(&m, 0, sizeof(m));
    const cuuint64_t dims[3] = {(cuuint64_t)Kr, (cuuint64_t)rows, (cuuint64_t)batch};
    const cuuint64_t strides[2] = {(cuuint64_t)(ld * 4), (cuuint64_t)((batch > 1 ? sbatch : ld * rows) * 4)};
    const cuuint32_t box[3] = {(cuuint32_t)TK, (cuuint32_t)box_rows, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(ptr), dims, strides,
                             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        throw Error(NC_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}

}  // namespace

void tc_gemm(Context& ctx, const TcGemm& g) {
    NC_ARG(g.M >= 1 && g.Nr >= 2 && g.Kr >= 1 && g.batch >= 1, "tc32: empty GEMM");
    NC_ARG(g.Nr % 2 == 0, "tc32: Nr must be even (complex columns)");
    NC_SET_SMEM_ONCE(tc32_gemm_kernel, TC_SMEM);
    const int shareA = g.A.sbatch == 0, shareB = g.B.sbatch == 0;
    const int bA = shareA ? 1 : g.batch, bB = shareB ? 1 : g.batch;
    const CUtensorMap mAb = make_map(g.A.big, g.Kr, g.M, g.A.ld, g.A.sbatch, bA, TM);
    const CUtensorMap mAs = make_map(g.three ? g.A.small : g.A.big, g.Kr, g.M, g.A.ld, g.A.sbatch, bA, TM);
    const CUtensorMap mBb = make_map(g.B.big, g.Kr, g.Nr, g.B.ld, g.B.sbatch, bB, TN);
    const CUtensorMap mBs = make_map(g.three ? g.B.small : g.B.big, g.Kr, g.Nr, g.B.ld, g.B.sbatch, bB, TN);
    TcParams P;
    P.M = g.M; P.Nr = g.Nr; P.Kr = g.Kr;
    P.nkb = (g.Kr + TK - 1) / TK;
    P.nseg = g.three ? 3 : 1;
    P.shareA = shareA; P.shareB = shareB;
    P.C = g.C; P.sm = g.sm; P.sn = g.sn; P.sz = g.sz; P.c_fp64 = g.c_fp64 ? 1 : 0;
    dim3 grid((g.M + TM - 1) / TM, (g.Nr + TN - 1) / TN, g.batch);
    NC_ARG(grid.y <= 65535 && grid.z <= 65535, "tc32: grid too large");
    const double flops = 2.0 * g.M * (double)g.Nr * g.Kr * P.nseg * g.batch;
    profile_launch(ctx, flops, 1, [&] {
        tc32_gemm_kernel<<<grid, TC_THREADS, TC_SMEM, ctx.stream>>>(mAb, mAs, mBb, mBs, P);
        NC_CHECK_LAUNCH();
    });
    ctx.launches++;
}

void tc_test_fault(unsigned long long wait_ns, int skip_first_load) {
    NC_ARG(wait_ns >= 1000, "tc32 wait limit must be at least 1 microsecond");
    NC_CUDA(cudaMemcpyToSymbol(g_tc_wait_ns, &wait_ns, sizeof(wait_ns)));
    NC_CUDA(cudaMemcpyToSymbol(g_tc_skip_first_load, &skip_first_load, sizeof(int)));
}

void tc_check(Context& ctx) {
    NC_CUDA(cudaStreamSynchronize(ctx.stream));
    int flag = 0;
    NC_CUDA(cudaMemcpyFromSymbol(&flag, g_tc_error, sizeof(int)));
    if (flag) {
        const int zero = 0;
        NC_CUDA(cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(int)));
        throw Error(NC_ERR_TIMEOUT, "tc32 GEMM: a pipeline wait exceeded its time limit");
    }
}

}  // namespace nc
