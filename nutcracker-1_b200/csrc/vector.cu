// HBM-bound vector kernels (permutes, reductions, axpy) and the runtime
// (device arena, per-thread context).
#include <algorithm>

#include "nc_common.cuh"
#include "nc_kernels.h"

namespace nc {

// ---------------------------------------------------------------------------
// runtime
// ---------------------------------------------------------------------------

Arena::~Arena() {
    for (auto& b : blocks_) cudaFree(b.p);
    for (auto& b : spare_) cudaFree(b.p);
}

void* Arena::alloc(size_t bytes) {
    bytes = (bytes + 255) & ~size_t(255);
    if (bytes == 0) bytes = 256;
    if (!blocks_.empty()) {
        Block& b = blocks_.back();
        if (b.used + bytes <= b.size) {
            void* p = b.p + b.used;
            b.used += bytes;
            return p;
        }
    }
    // reuse a spare block large enough, else allocate a new one
    for (size_t i = 0; i < spare_.size(); ++i) {
        if (spare_[i].size >= bytes) {
            Block b = spare_[i];
            spare_.erase(spare_.begin() + i);
            b.used = bytes;
            blocks_.push_back(b);
            return b.p;
        }
    }
    size_t last = blocks_.empty() ? 0 : blocks_.back().size;
    size_t sz = std::max(bytes, std::max(last * 2, size_t(64) << 20));
    Block b;
    cudaError_t e = cudaMalloc(&b.p, sz);
    if (e != cudaSuccess) {
        // retry with the exact size before giving up
        cudaGetLastError();
        sz = bytes;
        e = cudaMalloc(&b.p, sz);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Error(NC_ERR_NOMEM, "device arena: cudaMalloc of " + std::to_string(sz) + " bytes failed");
        }
    }
    b.size = sz;
    b.used = bytes;
    blocks_.push_back(b);
    return b.p;
}

Arena::Mark Arena::mark() const {
    if (blocks_.empty()) return Mark{0, 0};
    return Mark{blocks_.size(), blocks_.back().used};
}

void Arena::release(Mark m) {
    while (blocks_.size() > m.block) {
        Block b = blocks_.back();
        blocks_.pop_back();
        b.used = 0;
        spare_.push_back(b);
    }
    if (!blocks_.empty() && m.block == blocks_.size()) blocks_.back().used = m.used;
}

size_t Arena::capacity() const {
    size_t c = 0;
    for (auto& b : blocks_) c += b.size;
    for (auto& b : spare_) c += b.size;
    return c;
}

Context::Context() {
    NC_CUDA(cudaGetDevice(&device));
    NC_CUDA(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
    stream = own_stream;
    pinned_bytes = 1 << 16;
    NC_CUDA(cudaMallocHost(&pinned, pinned_bytes));
}

unsigned* Context::reduction_counter() {
    if (!red_counter) {
        NC_CUDA(cudaMalloc(&red_counter, 64 * sizeof(unsigned)));
        NC_CUDA(cudaMemset(red_counter, 0, 64 * sizeof(unsigned)));
    }
    return red_counter;
}

void Context::sync() {
    if (!blocking_sync) {
        NC_CUDA(cudaStreamSynchronize(stream));
        return;
    }
    if (!sync_event)
        NC_CUDA(cudaEventCreateWithFlags(&sync_event, cudaEventBlockingSync | cudaEventDisableTiming));
    NC_CUDA(cudaEventRecord(sync_event, stream));
    NC_CUDA(cudaEventSynchronize(sync_event));
}

Context::~Context() {
    if (sync_event) cudaEventDestroy(sync_event);
    if (red_counter) cudaFree(red_counter);
    if (own_stream) cudaStreamDestroy(own_stream);
    if (pinned) cudaFreeHost(pinned);
}

Context& Context::get() {
    thread_local Context* ctx = nullptr;
    if (!ctx) ctx = new Context();  // lives until process exit (avoids teardown-order issues)
    return *ctx;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

namespace {

constexpr int RED_THREADS = 256;
constexpr int RED_BLOCKS = 592;  // 4 x 148 SMs

unsigned grid1(long long n, int threads) {
    long long g = (n + threads - 1) / threads;
    return (unsigned)std::max<long long>(1, std::min<long long>(g, 148LL * 16));
}

__global__ void permute3_kernel(const cplx* __restrict__ in, int o0, int o1, int o2, long long s0,
                                long long s1, long long s2, bool conj, cplx* __restrict__ out) {
    const long long total = (long long)o0 * o1 * o2;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long q = e;
        int i0 = (int)(q % o0); q /= o0;
        int i1 = (int)(q % o1); q /= o1;
        int i2 = (int)q;
        cplx v = in[i0 * s0 + i1 * s1 + i2 * s2];
        out[e] = conj ? cconj(v) : v;
    }
}

// <x,y> (or |x|^2) in one launch: every block stores its partial sum, and the
// last block to finish (by an atomic ticket after a fence) adds the partials
// in block order, so the result does not depend on block timing.
template <bool NORM>
__global__ void dot_fused(long long n, const cplx* __restrict__ x, const cplx* __restrict__ y,
                          cplx* __restrict__ part, unsigned* __restrict__ counter, cplx* __restrict__ out) {
    __shared__ double sr[RED_THREADS], si[RED_THREADS];
    __shared__ bool last;
    double ar = 0, ai = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        cplx a = x[e];
        if (NORM) {
            ar += a.x * a.x + a.y * a.y;
        } else {
            cplx b = y[e];
            ar += a.x * b.x + a.y * b.y;
            ai += a.x * b.y - a.y * b.x;
        }
    }
    sr[threadIdx.x] = ar; si[threadIdx.x] = ai;
    __syncthreads();
    for (int s = RED_THREADS / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) { sr[threadIdx.x] += sr[threadIdx.x + s]; si[threadIdx.x] += si[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[blockIdx.x] = cmake(sr[0], si[0]);
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    ar = 0; ai = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
        const cplx p = __ldcg(&part[i]);
        ar += p.x; ai += p.y;
    }
    sr[threadIdx.x] = ar; si[threadIdx.x] = ai;
    __syncthreads();
    for (int s = RED_THREADS / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) { sr[threadIdx.x] += sr[threadIdx.x + s]; si[threadIdx.x] += si[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = cmake(sr[0], si[0]);
        *counter = 0;
    }
}

__global__ void copy_kernel(long long n, const cplx* __restrict__ x, cplx* __restrict__ y) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x)
        y[e] = x[e];
}
__global__ void fill_kernel(long long n, cplx v, cplx* __restrict__ y) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x)
        y[e] = v;
}
__global__ void axpy_dev_kernel(long long n, const cplx* __restrict__ a_dev, double s,
                                const cplx* __restrict__ x, cplx* __restrict__ y) {
    cplx a = cscale(a_dev[0], s);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x)
        y[e] = cadd(y[e], cmul(a, x[e]));
}
__global__ void scal_kernel(long long n, cplx a, cplx* __restrict__ x) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x)
        x[e] = cmul(a, x[e]);
}
__global__ void normalize_kernel(long long n, const cplx* __restrict__ nrm2sq, cplx* __restrict__ x) {
    double s = 1.0 / sqrt(nrm2sq[0].x);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x)
        x[e] = cscale(x[e], s);
}

}  // namespace

void permute3(Context& ctx, const cplx* in, int n0, int n1, int n2, const int perm[3], bool conj,
              cplx* out) {
    const int nd[3] = {n0, n1, n2};
    const long long st[3] = {1, (long long)n0, (long long)n0 * n1};
    int o0 = nd[perm[0]], o1 = nd[perm[1]], o2 = nd[perm[2]];
    long long total = (long long)o0 * o1 * o2;
    if (total == 0) return;
    permute3_kernel<<<grid1(total, 256), 256, 0, ctx.stream>>>(in, o0, o1, o2, st[perm[0]], st[perm[1]],
                                                                st[perm[2]], conj, out);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

void zdotc(Context& ctx, long long n, const cplx* x, const cplx* y, cplx* result) {
    ArenaFrame f(ctx.arena);
    cplx* part = ctx.arena.alloc_n<cplx>(RED_BLOCKS);
    const unsigned nb = (unsigned)std::max<long long>(1, std::min<long long>(RED_BLOCKS, (n + RED_THREADS - 1) / RED_THREADS));
    dot_fused<false><<<nb, RED_THREADS, 0, ctx.stream>>>(n, x, y, part, ctx.reduction_counter(), result);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

void znrm2sq(Context& ctx, long long n, const cplx* x, cplx* result) {
    ArenaFrame f(ctx.arena);
    cplx* part = ctx.arena.alloc_n<cplx>(RED_BLOCKS);
    const unsigned nb = (unsigned)std::max<long long>(1, std::min<long long>(RED_BLOCKS, (n + RED_THREADS - 1) / RED_THREADS));
    dot_fused<true><<<nb, RED_THREADS, 0, ctx.stream>>>(n, x, x, part, ctx.reduction_counter(), result);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

void zcopy(Context& ctx, long long n, const cplx* x, cplx* y) {
    if (n <= 0) return;
    copy_kernel<<<grid1(n, 256), 256, 0, ctx.stream>>>(n, x, y);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

void zfill(Context& ctx, long long n, cplx v, cplx* y) {
    if (n <= 0) return;
    fill_kernel<<<grid1(n, 256), 256, 0, ctx.stream>>>(n, v, y);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

void zaxpy_dev(Context& ctx, long long n, const cplx* a_dev, double s, const cplx* x, cplx* y) {
    if (n <= 0) return;
    axpy_dev_kernel<<<grid1(n, 256), 256, 0, ctx.stream>>>(n, a_dev, s, x, y);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

void zscal_host(Context& ctx, long long n, cplx a, cplx* x) {
    if (n <= 0) return;
    scal_kernel<<<grid1(n, 256), 256, 0, ctx.stream>>>(n, a, x);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

void znormalize_dev(Context& ctx, long long n, const cplx* nrm2sq_dev, cplx* x) {
    if (n <= 0) return;
    normalize_kernel<<<grid1(n, 256), 256, 0, ctx.stream>>>(n, nrm2sq_dev, x);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

void read_scalars(Context& ctx, const void* dev, size_t bytes, void* host) {
    NC_ARG(bytes <= ctx.pinned_bytes, "read_scalars: too many bytes");
    NC_CUDA(cudaMemcpyAsync(ctx.pinned, dev, bytes, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    memcpy(host, ctx.pinned, bytes);
}

cplx read_scalar(Context& ctx, const cplx* dev) {
    cplx v;
    read_scalars(ctx, dev, sizeof(cplx), &v);
    return v;
}

}  // namespace nc
