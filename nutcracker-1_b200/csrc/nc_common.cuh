// Shared definitions for the B200 variational-MPS sweep library.
//
// Storage conventions follow the reference's Fortran core
// (sources/common/core.f95): every tensor is column-major complex128 stored
// as interleaved (re, im) doubles, i.e. layout-compatible with
// std::complex<double> / double _Complex.  MPO link indices are uint32
// (from, to) pairs, 1-based.
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

namespace nc {

typedef double2 cplx;

// Error type carried across the C-ABI as a status code plus message.
struct Error : public std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

enum Status : int {
    NC_OK = 0,
    NC_ERR_CUDA = 1001,
    NC_ERR_ARG = 1002,
    NC_ERR_NOMEM = 1003,
    NC_ERR_TIMEOUT = 1004,
    NC_ERR_NUMERIC = 1005,
};

#define NC_CUDA(expr)                                                                   \
    do {                                                                                \
        cudaError_t _e = (expr);                                                        \
        if (_e != cudaSuccess)                                                          \
            throw ::nc::Error(::nc::NC_ERR_CUDA, std::string(#expr) + ": " +            \
                                                     cudaGetErrorString(_e));           \
    } while (0)

#define NC_CHECK_LAUNCH() NC_CUDA(cudaGetLastError())

#define NC_ARG(cond, msg)                                                               \
    do {                                                                                \
        if (!(cond)) throw ::nc::Error(::nc::NC_ERR_ARG, msg);                          \
    } while (0)

__host__ __device__ inline cplx cmake(double r, double i) { return make_double2(r, i); }
__host__ __device__ inline cplx cadd(cplx a, cplx b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ inline cplx csub(cplx a, cplx b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ inline cplx cmul(cplx a, cplx b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ inline cplx cconj(cplx a) { return make_double2(a.x, -a.y); }
__host__ __device__ inline cplx cscale(cplx a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ inline double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }

// Device memory arena: a grow-only stack of cudaMalloc'd blocks reused across
// calls so that the hot path never calls cudaMalloc once warm.
class Arena {
   public:
    Arena() {}
    ~Arena();
    // Bump-allocate `bytes` (256-byte aligned) from the current frame.
    void* alloc(size_t bytes);
    template <class T>
    T* alloc_n(size_t n) { return static_cast<T*>(alloc(n * sizeof(T))); }
    struct Mark { size_t block, used; };
    Mark mark() const;
    void release(Mark m);
    size_t capacity() const;

   private:
    struct Block { char* p; size_t size; size_t used; };
    std::vector<Block> blocks_;   // live blocks, last one is the bump target
    std::vector<Block> spare_;    // released blocks kept for reuse (never freed while live)
};

// RAII frame over an Arena.
struct ArenaFrame {
    Arena& a;
    Arena::Mark m;
    explicit ArenaFrame(Arena& ar) : a(ar), m(ar.mark()) {}
    ~ArenaFrame() { a.release(m); }
};

// Per-host-thread execution context: stream, arena and small pinned buffers.
struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;      // stream all work is enqueued on
    cudaStream_t own_stream = nullptr;  // the context's own non-blocking stream
    Arena arena;
    void* pinned = nullptr;  // small pinned host staging buffer for scalars
    size_t pinned_bytes = 0;
    uint64_t launches = 0;   // kernels launched by this library on this context
    int krylov_dim = 24;     // Lanczos basis size before a restart
    // Gauge of the Level-0 norm_denorm_* / norm_for_* entry points: true
    // (default) = the reference's exact polar factor, false = the faster
    // Householder-QR gauge (the same state, a different site tensor).
    bool level0_polar = true;
    // Workspace arena for GEMM split-K partials and QR scratch: the context
    // arena, or a captured graph's private arena while it is being recorded.
    Arena* ws_override = nullptr;
    Arena& scratch() { return ws_override ? *ws_override : arena; }
    // Completion counter of single-kernel reductions (the last block to finish
    // combines the partial sums in a fixed order and resets it to zero); one
    // per context, used in stream order only.
    unsigned* red_counter = nullptr;
    unsigned* reduction_counter();
    // Kernel timing (nc_profile_begin/end): CUDA events around every complex
    // GEMM of at least profile_min_flops, on the launching stream.
    bool profile = false;
    double profile_min_flops = 1e9;
    std::vector<cudaEvent_t> prof_start, prof_stop;
    std::vector<double> prof_flops;
    std::vector<int> prof_kind;   // 0: FP64 DMMA complex GEMM, 1: tcgen05 3xTF32 GEMM
    size_t prof_used = 0;
    // Host waits on this context's stream: spin (cudaStreamSynchronize, the
    // lowest latency) by default; a blocking-sync event when many threads
    // share the host's cores (the serving engine's workers), so that waiting
    // threads leave the cores to the ones launching work.
    bool blocking_sync = false;
    cudaEvent_t sync_event = nullptr;
    void sync();
    Context();
    ~Context();
    static Context& get();   // thread-local default context
};

inline unsigned ceil_div(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

// Runs a set-up step (a kernel attribute, which belongs to the device context
// current when it is set) once per device.  One object per call site; safe
// for concurrent callers (the step may run twice, so it must be idempotent).
// Devices beyond the 64 tracked ones run the step on every call.
class PerDeviceOnce {
   public:
    template <class F>
    void operator()(F&& step) {
        int dev = 0;
        NC_CUDA(cudaGetDevice(&dev));
        const uint64_t bit = (dev >= 0 && dev < 64) ? (1ull << dev) : 0ull;
        if (bit && (done_.load(std::memory_order_acquire) & bit)) return;
        step();
        if (bit) done_.fetch_or(bit, std::memory_order_acq_rel);
    }

   private:
    std::atomic<uint64_t> done_{0};
};

// The largest dynamic shared memory of `kernel`, set once per device.
#define NC_SET_SMEM_ONCE(kernel, bytes)                                                             \
    do {                                                                                            \
        static ::nc::PerDeviceOnce _once;                                                           \
        _once([&] {                                                                                 \
            NC_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                         (int)(bytes)));                                            \
        });                                                                                         \
    } while (0)

}  // namespace nc
