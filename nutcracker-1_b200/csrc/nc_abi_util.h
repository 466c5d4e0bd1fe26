// Helpers for the host-buffer C-ABI entry points.
#pragma once

#include <cuda_runtime.h>

#include <exception>

#include "nc_common.cuh"
#include "nc_kernels.h"
#include "nutcracker_b200.h"

namespace nc {

void set_status(int code, const char* msg);
extern thread_local int g_status;

// Stages host inputs into the thread's device arena and copies results back.
struct HostStage {
    Context& ctx;
    ArenaFrame frame;
    HostStage() : ctx(Context::get()), frame(ctx.arena) {}

    template <class T>
    const cplx* in(const T* host, size_t n) {
        if (n == 0) return nullptr;
        cplx* d = ctx.arena.alloc_n<cplx>(n);
        NC_CUDA(cudaMemcpyAsync(d, host, n * sizeof(cplx), cudaMemcpyHostToDevice, ctx.stream));
        return d;
    }
    const uint32_t* in_u32(const uint32_t* host, size_t n) {
        if (n == 0) return nullptr;
        uint32_t* d = ctx.arena.alloc_n<uint32_t>(n);
        NC_CUDA(cudaMemcpyAsync(d, host, n * sizeof(uint32_t), cudaMemcpyHostToDevice, ctx.stream));
        return d;
    }
    cplx* out(size_t n) { return ctx.arena.alloc_n<cplx>(n ? n : 1); }
    template <class T>
    void back(T* host, const cplx* dev, size_t n) {
        if (n == 0) return;
        NC_CUDA(cudaMemcpyAsync(host, dev, n * sizeof(cplx), cudaMemcpyDeviceToHost, ctx.stream));
    }
    void back_u32(uint32_t* host, const uint32_t* dev, size_t n) {
        if (n == 0) return;
        NC_CUDA(cudaMemcpyAsync(host, dev, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx.stream));
    }
    void sync() { NC_CUDA(cudaStreamSynchronize(ctx.stream)); }

    MpoSite mpo(uint32_t d, uint32_t cl, uint32_t cr, uint32_t nnz, const uint32_t* idx,
                const nc_complex* W) {
        NC_ARG(nnz >= 1, "operator site needs at least one matrix");
        for (uint32_t i = 0; i < nnz; ++i) {
            NC_ARG(idx[2 * i] >= 1 && idx[2 * i] <= cl, "operator index 'from' out of range");
            NC_ARG(idx[2 * i + 1] >= 1 && idx[2 * i + 1] <= cr, "operator index 'to' out of range");
        }
        MpoSite op;
        op.d = (int)d; op.cl = (int)cl; op.cr = (int)cr; op.nnz = (int)nnz;
        op.idx = in_u32(idx, 2 * (size_t)nnz);
        op.W = in(W, (size_t)d * d * nnz);
        return op;
    }
};

}  // namespace nc

#define NC_ABI_BEGIN        \
    ::nc::set_status(0, ""); \
    try {
#define NC_ABI_END                                                 \
    }                                                              \
    catch (const ::nc::Error& e) {                                 \
        ::nc::set_status(e.code, e.what());                        \
    }                                                              \
    catch (const std::exception& e) {                              \
        ::nc::set_status(::nc::NC_ERR_ARG, e.what());              \
    }
