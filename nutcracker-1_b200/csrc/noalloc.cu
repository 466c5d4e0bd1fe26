// H_eff product that allocates nothing.
//
// Some callers cannot let the library call cudaMalloc: a serving loop that
// runs under a fixed device-memory budget, or latency-critical code where a
// first-time cudaMalloc (or the cudaFree that would pair with it, which
// synchronises the whole device) would stall other work.  For them this
// entry point takes its scratch from one file-scope device array of a fixed
// size instead of the library's growable arena.
//
// * Capacity: kScratchBytes = 64 MiB.  A call needs
//   16 * (br*bl*cl*d + br*cr*bl*d) bytes (the step-A product T and the mixed
//   operand U); larger calls are rejected with an error, nothing is launched.
// * Every GPU that loads the library holds the 64 MiB array until the
//   process exits.
// * The array's host-side name is not a device address.  The first call on
//   each device looks the address up with cudaGetSymbolAddress (with that
//   device current) and caches it; make that first call before any stream
//   capture.
// * All calls share the array.  Nothing in it has to start at zero: each call
//   writes T and U completely before reading them.  Calls whose kernels
//   overlap on the GPU (different streams, or different host threads on one
//   device without ordering) race on the array; order them on one stream.
// * The MPO indices live in device memory and are not read back (that would
//   synchronise), so they are not range-checked: every (from, to) pair must
//   satisfy 1 <= from <= cl and 1 <= to <= cr, or the mix kernel reads
//   outside T.  The host-buffer entry points (optimize_ and friends) do
//   check them.
#include <climits>
#include <mutex>

#include "nc_abi_util.h"
#include "nc_common.cuh"
#include "nc_kernels.h"

using namespace nc;

namespace {

constexpr size_t kScratchBytes = 64ull << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_heff_scratch[kScratchBytes];

std::mutex g_scratch_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

cplx* scratch_for_current_device() {
    int dev = 0;
    NC_CUDA(cudaGetDevice(&dev));
    NC_ARG(dev >= 0 && dev < kMaxDevices, "device index out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_heff_scratch);
        if (e != cudaSuccess || !p)
            throw Error(NC_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = p;
    }
    return static_cast<cplx*>(g_scratch_ptr[dev]);
}

}  // namespace

extern "C" int nc_heff_apply_dev_noalloc(uint32_t bl, uint32_t br, uint32_t cl, uint32_t cr, uint32_t d,
                                         uint32_t nnz, const uint32_t* idx_dev, const void* W_dev,
                                         const void* L_dev, const void* R_dev, const void* x_dev, void* y_dev,
                                         void* stream) {
    NC_ABI_BEGIN
    // Sizes are checked as unsigned 64-bit products before anything is cast
    // to int, so no wrapped product can slip under the capacity check.
    NC_ARG(bl >= 1 && br >= 1 && cl >= 1 && cr >= 1 && d >= 1 && nnz >= 1,
           "nc_heff_apply_dev_noalloc: every dimension must be at least 1");
    NC_ARG(bl <= INT_MAX && br <= INT_MAX && cl <= INT_MAX && cr <= INT_MAX && d <= INT_MAX && nnz <= INT_MAX,
           "nc_heff_apply_dev_noalloc: dimension too large");
    uint64_t need = 0;
    {
        uint64_t brbld = 0, elems = 0;
        const bool wrap = __builtin_mul_overflow((uint64_t)br, (uint64_t)bl, &brbld) ||
                          __builtin_mul_overflow(brbld, (uint64_t)d, &brbld) ||
                          __builtin_mul_overflow(brbld, (uint64_t)cl + (uint64_t)cr, &elems) ||
                          __builtin_mul_overflow(elems, (uint64_t)sizeof(cplx), &need);
        if (wrap) need = UINT64_MAX;
    }
    if (need > kScratchBytes)
        throw Error(NC_ERR_ARG, "nc_heff_apply_dev_noalloc: needs " +
                                    (need == UINT64_MAX ? std::string("more than 2^64") : std::to_string(need)) +
                                    " bytes of scratch, more than the fixed 67108864-byte (64 MiB) maximum");
    MpoSite op;
    op.d = (int)d; op.cl = (int)cl; op.cr = (int)cr; op.nnz = (int)nnz;
    op.idx = idx_dev; op.W = static_cast<const cplx*>(W_dev);
    cplx* ws = scratch_for_current_device();
    heff_apply_stream(static_cast<cudaStream_t>(stream), (int)bl, (int)br, op, static_cast<const cplx*>(L_dev),
                      static_cast<const cplx*>(R_dev), static_cast<const cplx*>(x_dev), static_cast<cplx*>(y_dev),
                      ws);
    NC_ABI_END
    return g_status;
}
