// Level-0 C-ABI: the Fortran-named numeric kernels of the reference
// (sources/common/core.cpp) re-implemented on the GPU.  Host buffers in,
// host buffers out; every call stages through the calling thread's device
// arena and stream.
#include <cstring>
#include <string>

#include "nc_abi_util.h"
#include "nc_common.cuh"
#include "nc_kernels.h"

using namespace nc;

namespace nc {

thread_local int g_status = 0;
thread_local std::string g_message;

void set_status(int code, const char* msg) {
    g_status = code;
    g_message = msg ? msg : "";
}

namespace {

__global__ void opt_matrix_kernel(int bl, int br, int cl, int cr, int d, int nnz,
                                  const cplx* __restrict__ L, const uint32_t* __restrict__ idx,
                                  const cplx* __restrict__ W, const cplx* __restrict__ R,
                                  cplx* __restrict__ H) {
    // H(r1,l2,o2 ; r2,l1,o1) = sum_n L(l1,l2,k1) W(o1,o2,n) R(r1,r2,k2)   (core.f95:1090-1140)
    const long long n = (long long)br * bl * d;
    const long long total = n * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long row = e % n, col = e / n;
        int r1 = (int)(row % br), l2 = (int)((row / br) % bl), o2 = (int)(row / ((long long)br * bl));
        int r2 = (int)(col % br), l1 = (int)((col / br) % bl), o1 = (int)(col / ((long long)br * bl));
        cplx acc = cmake(0, 0);
        for (int q = 0; q < nnz; ++q) {
            int k1 = (int)idx[2 * q] - 1, k2 = (int)idx[2 * q + 1] - 1;
            cplx lv = L[l1 + (long long)bl * (l2 + (long long)bl * k1)];
            cplx wv = W[o1 + d * (o2 + d * q)];
            cplx rv = R[r1 + (long long)br * (r2 + (long long)br * k2)];
            acc = cadd(acc, cmul(cmul(lv, wv), rv));
        }
        H[e] = acc;
    }
}

__global__ void exp_boundary_kernel(int b, int c, const cplx* __restrict__ sb,
                                    const cplx* __restrict__ ob, bool right, cplx* __restrict__ out) {
    // left:  L(i,j,k) = sb(i) conj(sb(j)) ob(k)   (core.f95:3401-3417)
    // right: R(i,j,k) = conj(sb(i)) sb(j) ob(k)   (core.f95:3419-3435)
    const long long total = (long long)b * b * c;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int i = (int)(e % b), j = (int)((e / b) % b), k = (int)(e / ((long long)b * b));
        cplx si = sb[i], sj = sb[j];
        cplx v = right ? cmul(cconj(si), sj) : cmul(si, cconj(sj));
        out[e] = cmul(v, ob[k]);
    }
}

}  // namespace

void expectation_dev(Context& ctx, int bl, int br, const MpoSite& op, const cplx* L, const cplx* psi,
                     const cplx* R, cplx* result) {
    ArenaFrame f(ctx.arena);
    const long long n = (long long)br * bl * op.d;
    cplx* y = ctx.arena.alloc_n<cplx>(n);
    cplx* ws = ctx.arena.alloc_n<cplx>(heff_workspace_elems(bl, br, op));
    heff_apply(ctx, bl, br, op, L, R, psi, y, ws);
    zdotc(ctx, n, psi, y, result);
}

void optimization_matrix_dev(Context& ctx, int bl, int br, const MpoSite& op, const cplx* L,
                             const cplx* R, cplx* H) {
    const long long n = (long long)br * bl * op.d;
    long long total = n * n;
    unsigned grid = (unsigned)std::min<long long>((total + 255) / 256, 148 * 16);
    opt_matrix_kernel<<<grid, 256, 0, ctx.stream>>>(bl, br, op.cl, op.cr, op.d, op.nnz, L, op.idx,
                                                    op.W, R, H);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

void exp_boundary_dev(Context& ctx, int b, int c, const cplx* sb, const cplx* ob, bool right, cplx* out) {
    long long total = (long long)b * b * c;
    unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148 * 16));
    exp_boundary_kernel<<<grid, 256, 0, ctx.stream>>>(b, c, sb, ob, right, out);
    NC_CHECK_LAUNCH();
    ctx.launches++;
}

}  // namespace nc

// ---------------------------------------------------------------------------
// extern "C"
// ---------------------------------------------------------------------------

extern "C" {

int nc_last_status(void) { return g_status; }
const char* nc_last_error(void) { return g_message.c_str(); }
uint64_t nc_launch_count(void) {
    try { return Context::get().launches; } catch (...) { return 0; }
}
const char* nc_version(void) { return "nutcracker-b200 0.1 (sm_100a)"; }

int nc_set_stream(void* stream) {
    NC_ABI_BEGIN
    Context::get().stream = (cudaStream_t)stream;
    NC_ABI_END
    return g_status;
}

int nc_use_own_stream(void) {
    NC_ABI_BEGIN
    Context& ctx = Context::get();
    ctx.stream = ctx.own_stream;
    NC_ABI_END
    return g_status;
}

int nc_profile_begin(double min_flops) {
    NC_ABI_BEGIN
    Context& ctx = Context::get();
    ctx.profile = true;
    ctx.profile_min_flops = min_flops;
    ctx.prof_used = 0;
    NC_ABI_END
    return g_status;
}

int nc_profile_end(uint64_t* launches, double* total_ms, double* total_flops) {
    NC_ABI_BEGIN
    Context& ctx = Context::get();
    NC_CUDA(cudaStreamSynchronize(ctx.stream));
    double ms = 0, fl = 0;
    uint64_t n = 0;
    for (size_t i = 0; i < ctx.prof_used; ++i) {
        if (ctx.prof_kind[i] != 0) continue;
        ++n;
        float t = 0;
        NC_CUDA(cudaEventElapsedTime(&t, ctx.prof_start[i], ctx.prof_stop[i]));
        ms += t;
        fl += ctx.prof_flops[i];
    }
    *launches = n;
    *total_ms = ms;
    *total_flops = fl;
    ctx.profile = false;
    ctx.prof_used = 0;
    NC_ABI_END
    return g_status;
}

int nc_profile_query(int kind, uint64_t* launches, double* total_ms, double* total_flops) {
    NC_ABI_BEGIN
    Context& ctx = Context::get();
    NC_CUDA(cudaStreamSynchronize(ctx.stream));
    double ms = 0, fl = 0;
    uint64_t n = 0;
    for (size_t i = 0; i < ctx.prof_used; ++i) {
        if (ctx.prof_kind[i] != kind) continue;
        ++n;
        float t = 0;
        NC_CUDA(cudaEventElapsedTime(&t, ctx.prof_start[i], ctx.prof_stop[i]));
        ms += t;
        fl += ctx.prof_flops[i];
    }
    *launches = n;
    *total_ms = ms;
    *total_flops = fl;
    NC_ABI_END
    return g_status;
}

int nc_synchronize(void) {
    NC_ABI_BEGIN
    NC_CUDA(cudaStreamSynchronize(Context::get().stream));
    NC_ABI_END
    return g_status;
}

int nc_heff_apply_dev(uint32_t bl, uint32_t br, uint32_t cl, uint32_t cr, uint32_t d, uint32_t nnz,
                      const uint32_t* idx_dev, const void* W_dev, const void* L_dev, const void* R_dev,
                      const void* x_dev, void* y_dev) {
    NC_ABI_BEGIN
    Context& ctx = Context::get();
    MpoSite op;
    op.d = (int)d; op.cl = (int)cl; op.cr = (int)cr; op.nnz = (int)nnz;
    op.idx = idx_dev; op.W = (const cplx*)W_dev;
    ArenaFrame f(ctx.arena);
    cplx* ws = ctx.arena.alloc_n<cplx>(heff_workspace_elems(bl, br, op));
    heff_apply(ctx, bl, br, op, (const cplx*)L_dev, (const cplx*)R_dev, (const cplx*)x_dev, (cplx*)y_dev, ws);
    NC_ABI_END
    return g_status;
}

int nc_heff_apply_mixed_dev(uint32_t bl, uint32_t br, uint32_t cl, uint32_t cr, uint32_t d, uint32_t nnz,
                            const uint32_t* idx_dev, const void* W_dev, const void* L_dev, const void* R_dev,
                            const void* x_dev, void* y_dev) {
    NC_ABI_BEGIN
    Context& ctx = Context::get();
    MpoSite op;
    op.d = (int)d; op.cl = (int)cl; op.cr = (int)cr; op.nnz = (int)nnz;
    op.idx = idx_dev; op.W = (const cplx*)W_dev;
    ArenaFrame f(ctx.arena);
    float* buf = ctx.arena.alloc_n<float>(mixed_heff_floats(bl, br, op));
    MixedHeff h;
    mixed_heff_prepare(ctx, bl, br, op, (const cplx*)L_dev, (const cplx*)R_dev, buf, &h);
    heff_apply_mixed(ctx, h, (const cplx*)x_dev, (cplx*)y_dev);
    tc_check(ctx);
    NC_ABI_END
    return g_status;
}

int nc_env_update_dev(int side, int mixed, uint32_t bl, uint32_t br, uint32_t cl, uint32_t cr, uint32_t d,
                      uint32_t nnz, const uint32_t* idx_dev, const void* W_dev, const void* env_dev,
                      const void* psi_dev, void* out_dev) {
    NC_ABI_BEGIN
    NC_ARG(side == 0 || side == 1, "side must be 0 (left) or 1 (right)");
    Context& ctx = Context::get();
    MpoSite op;
    op.d = (int)d; op.cl = (int)cl; op.cr = (int)cr; op.nnz = (int)nnz;
    op.idx = idx_dev; op.W = (const cplx*)W_dev;
    const cplx* env = (const cplx*)env_dev;
    const cplx* psi = (const cplx*)psi_dev;
    cplx* out = (cplx*)out_dev;
    if (side == 0) {
        if (mixed) sos_left_mixed(ctx, bl, br, op, env, psi, out);
        else sos_left(ctx, bl, br, op, env, psi, out);
    } else {
        if (mixed) sos_right_mixed(ctx, bl, br, op, env, psi, out);
        else sos_right(ctx, bl, br, op, env, psi, out);
    }
    if (mixed) tc_check(ctx);
    NC_ABI_END
    return g_status;
}

int nc_tc_zgemm_dev(uint32_t M, uint32_t N, uint32_t K, const void* A_dev, const void* B_dev, void* C_dev,
                    int three) {
    NC_ABI_BEGIN
    tc_zgemm(Context::get(), (int)M, (int)N, (int)K, (const cplx*)A_dev, (const cplx*)B_dev, (cplx*)C_dev,
             three != 0);
    NC_ABI_END
    return g_status;
}

int nc_test_tc32_wait(uint64_t wait_ns, int skip_first_load) {
    NC_ABI_BEGIN
    tc_test_fault((unsigned long long)wait_ns, skip_first_load);
    NC_ABI_END
    return g_status;
}

void compute_expectation_(const uint32_t* bl, const uint32_t* br, const uint32_t* cl, const uint32_t* cr,
                          const uint32_t* d, const nc_complex* L, const nc_complex* S,
                          const uint32_t* nnz, const uint32_t* idx, const nc_complex* W,
                          const nc_complex* R, nc_complex* expectation) {
    NC_ABI_BEGIN
    HostStage h;
    MpoSite op = h.mpo(*d, *cl, *cr, *nnz, idx, W);
    const cplx* dL = h.in(L, (size_t)*bl * *bl * *cl);
    const cplx* dS = h.in(S, (size_t)*br * *bl * *d);
    const cplx* dR = h.in(R, (size_t)*br * *br * *cr);
    cplx* res = h.out(1);
    expectation_dev(h.ctx, *bl, *br, op, dL, dS, dR, res);
    h.back(expectation, res, 1);
    h.sync();
    NC_ABI_END
}

void compute_optimization_matrix_(const uint32_t* bl, const uint32_t* br, const uint32_t* cl,
                                  const uint32_t* cr, const uint32_t* d, const nc_complex* L,
                                  const uint32_t* nnz, const uint32_t* idx, const nc_complex* W,
                                  const nc_complex* R, nc_complex* H) {
    NC_ABI_BEGIN
    HostStage h;
    MpoSite op = h.mpo(*d, *cl, *cr, *nnz, idx, W);
    const cplx* dL = h.in(L, (size_t)*bl * *bl * *cl);
    const cplx* dR = h.in(R, (size_t)*br * *br * *cr);
    size_t n = (size_t)*br * *bl * *d;
    cplx* dH = h.out(n * n);
    optimization_matrix_dev(h.ctx, *bl, *br, op, dL, dR, dH);
    h.back(H, dH, n * n);
    h.sync();
    NC_ABI_END
}

void construct_left_exp_boundary_(const uint32_t* b, const uint32_t* c, const nc_complex* sb,
                                  const nc_complex* ob, nc_complex* out) {
    NC_ABI_BEGIN
    HostStage h;
    const cplx* dsb = h.in(sb, *b);
    const cplx* dob = h.in(ob, *c);
    cplx* o = h.out((size_t)*b * *b * *c);
    exp_boundary_dev(h.ctx, *b, *c, dsb, dob, false, o);
    h.back(out, o, (size_t)*b * *b * *c);
    h.sync();
    NC_ABI_END
}

void construct_right_exp_boundary_(const uint32_t* b, const uint32_t* c, const nc_complex* sb,
                                   const nc_complex* ob, nc_complex* out) {
    NC_ABI_BEGIN
    HostStage h;
    const cplx* dsb = h.in(sb, *b);
    const cplx* dob = h.in(ob, *c);
    cplx* o = h.out((size_t)*b * *b * *c);
    exp_boundary_dev(h.ctx, *b, *c, dsb, dob, true, o);
    h.back(out, o, (size_t)*b * *b * *c);
    h.sync();
    NC_ABI_END
}

void contract_expectation_boundaries_(const uint32_t* b, const uint32_t* c, const nc_complex* L,
                                      const nc_complex* R, nc_complex* expectation) {
    NC_ABI_BEGIN
    HostStage h;
    size_t n = (size_t)*b * *b * *c;
    const cplx* dL = h.in(L, n);
    const cplx* dR = h.in(R, n);
    cplx* res = h.out(1);
    contract_exp_boundaries(h.ctx, *b, *c, dL, dR, res);
    h.back(expectation, res, 1);
    h.sync();
    NC_ABI_END
}

void contract_sos_left_(const uint32_t* bl, const uint32_t* br, const uint32_t* cl, const uint32_t* cr,
                        const uint32_t* d, const nc_complex* L, const uint32_t* nnz, const uint32_t* idx,
                        const nc_complex* W, const nc_complex* S, nc_complex* Lnew) {
    NC_ABI_BEGIN
    HostStage h;
    MpoSite op = h.mpo(*d, *cl, *cr, *nnz, idx, W);
    const cplx* dL = h.in(L, (size_t)*bl * *bl * *cl);
    const cplx* dS = h.in(S, (size_t)*br * *bl * *d);
    size_t no = (size_t)*br * *br * *cr;
    cplx* o = h.out(no);
    sos_left(h.ctx, *bl, *br, op, dL, dS, o);
    h.back(Lnew, o, no);
    h.sync();
    NC_ABI_END
}

void contract_sos_right_(const uint32_t* bl, const uint32_t* br, const uint32_t* cl, const uint32_t* cr,
                         const uint32_t* d, const nc_complex* R, const uint32_t* nnz, const uint32_t* idx,
                         const nc_complex* W, const nc_complex* S, nc_complex* Rnew) {
    NC_ABI_BEGIN
    HostStage h;
    MpoSite op = h.mpo(*d, *cl, *cr, *nnz, idx, W);
    const cplx* dR = h.in(R, (size_t)*br * *br * *cr);
    const cplx* dS = h.in(S, (size_t)*br * *bl * *d);
    size_t no = (size_t)*bl * *bl * *cl;
    cplx* o = h.out(no);
    sos_right(h.ctx, *bl, *br, op, dR, dS, o);
    h.back(Rnew, o, no);
    h.sync();
    NC_ABI_END
}

void contract_vs_left_(const uint32_t* blo, const uint32_t* bro, const uint32_t* bln, const uint32_t* brn,
                       const uint32_t* d, const nc_complex* Lov, const nc_complex* P, const nc_complex* S,
                       nc_complex* out) {
    NC_ABI_BEGIN
    HostStage h;
    const cplx* dL = h.in(Lov, (size_t)*bln * *blo);
    const cplx* dP = h.in(P, (size_t)*blo * *d * *bro);
    const cplx* dS = h.in(S, (size_t)*brn * *bln * *d);
    size_t no = (size_t)*brn * *bro;
    cplx* o = h.out(no);
    vs_left(h.ctx, *blo, *bro, *bln, *brn, *d, dL, dP, dS, o);
    h.back(out, o, no);
    h.sync();
    NC_ABI_END
}

void contract_vs_right_(const uint32_t* blo, const uint32_t* bro, const uint32_t* bln, const uint32_t* brn,
                        const uint32_t* d, const nc_complex* Rov, const nc_complex* P, const nc_complex* S,
                        nc_complex* out) {
    NC_ABI_BEGIN
    HostStage h;
    const cplx* dR = h.in(Rov, (size_t)*bro * *brn);
    const cplx* dP = h.in(P, (size_t)*blo * *d * *bro);
    const cplx* dS = h.in(S, (size_t)*brn * *bln * *d);
    size_t no = (size_t)*blo * *bln;
    cplx* o = h.out(no);
    vs_right(h.ctx, *blo, *bro, *bln, *brn, *d, dR, dP, dS, o);
    h.back(out, o, no);
    h.sync();
    NC_ABI_END
}

void form_overlap_vector_(const uint32_t* blo, const uint32_t* bro, const uint32_t* bln, const uint32_t* brn,
                          const uint32_t* d, const nc_complex* Lov, const nc_complex* Rov,
                          const nc_complex* P, nc_complex* out) {
    NC_ABI_BEGIN
    HostStage h;
    const cplx* dL = h.in(Lov, (size_t)*bln * *blo);
    const cplx* dR = h.in(Rov, (size_t)*bro * *brn);
    const cplx* dP = h.in(P, (size_t)*blo * *d * *bro);
    size_t no = (size_t)*brn * *bln * *d;
    cplx* o = h.out(no);
    overlap_vector(h.ctx, *blo, *bro, *bln, *brn, *d, dL, dR, dP, o);
    h.back(out, o, no);
    h.sync();
    NC_ABI_END
}

void form_overlap_site_tensor_(const uint32_t* br, const uint32_t* bl, const uint32_t* d,
                               const nc_complex* S, nc_complex* out) {
    NC_ABI_BEGIN
    HostStage h;
    size_t n = (size_t)*br * *bl * *d;
    const cplx* dS = h.in(S, n);
    cplx* o = h.out(n);
    overlap_site_from_state(h.ctx, *br, *bl, *d, dS, o);
    h.back(out, o, n);
    h.sync();
    NC_ABI_END
}

// core.f95:1195-1234 (contract_matrix_left): L' (br,br) = M L M^H for
// M (br,bl), L (bl,bl).
void contract_matrix_left_(const uint32_t* bl, const uint32_t* br, const nc_complex* left_environment,
                           const nc_complex* matrix, nc_complex* new_left_environment) {
    NC_ABI_BEGIN
    HostStage h;
    const int l = (int)*bl, r = (int)*br;
    const cplx* dL = h.in(left_environment, (size_t)l * l);
    const cplx* dM = h.in(matrix, (size_t)r * l);
    cplx* T = h.out((size_t)r * l);
    cplx* o = h.out((size_t)r * r);
    zgemm(zgemm_params(OP_N, OP_N, r, l, l, dM, r, dL, l, T, r), h.ctx);
    zgemm(zgemm_params(OP_N, OP_C, r, r, l, T, r, dM, r, o, r), h.ctx);
    h.back(new_left_environment, o, (size_t)r * r);
    h.sync();
    NC_ABI_END
}

// core.f95:1163-1193 (extend_state_vector_fragment): new (br,dr,dl) =
// site (br,bm,dr) permuted to (br,dr,bm) times old (bm,dl).
void extend_state_vector_fragment_(const uint32_t* bm, const uint32_t* br, const uint32_t* dl, const uint32_t* dr,
                                   const nc_complex* old_state_vector_fragment, const nc_complex* site_tensor,
                                   nc_complex* new_state_vector_fragment) {
    NC_ABI_BEGIN
    HostStage h;
    const int m = (int)*bm, r = (int)*br, a = (int)*dl, b = (int)*dr;
    const cplx* dOld = h.in(old_state_vector_fragment, (size_t)m * a);
    const cplx* dS = h.in(site_tensor, (size_t)r * m * b);
    cplx* T = h.out((size_t)r * b * m);
    cplx* o = h.out((size_t)r * b * a);
    const int p_rs[3] = {0, 2, 1};
    permute3(h.ctx, dS, r, m, b, p_rs, false, T);
    zgemm(zgemm_params(OP_N, OP_N, r * b, a, m, T, r * b, dOld, m, o, r * b), h.ctx);
    h.back(new_state_vector_fragment, o, (size_t)r * b * a);
    h.sync();
    NC_ABI_END
}

// core.f95:3246-3297 (increase_bandwidth_with_environment) belongs to the
// infinite-chain path, which this library does not implement: the symbol is
// exported so that a build of the reference's C++ layer links, and a call
// reports NC_ERR_ARG through nc_last_status() and leaves its outputs untouched.
void increase_bandwidth_with_environment_(const uint32_t*, const uint32_t*, const uint32_t*, const uint32_t*,
                                          const nc_complex*, const nc_complex*, const nc_complex*, nc_complex*,
                                          nc_complex*, nc_complex*) {
    NC_ABI_BEGIN
    throw nc::Error(nc::NC_ERR_ARG, "increase_bandwidth_with_environment_: the infinite chain is not supported");
    NC_ABI_END
}

}  // extern "C"
