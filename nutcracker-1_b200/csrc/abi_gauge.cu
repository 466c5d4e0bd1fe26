// Level-0 C-ABI: gauge moves, bandwidth growth, random sites and projector
// site formation (sources/common/core.cpp:463-765) on the GPU.
#include "nc_abi_util.h"
#include "nc_common.cuh"
#include "nc_kernels.h"

using namespace nc;

namespace {
uint64_t abi_seed() {
    static thread_local uint64_t counter = 0;
    return 0x243F6A8885A308D3ull ^ (++counter * 0x9E3779B97F4A7C15ull);
}
}  // namespace

extern "C" {

int32_t norm_denorm_going_left_(const uint32_t* bl, const uint32_t* bm, const uint32_t* br, const uint32_t* dl,
                                const uint32_t* dr, const nc_complex* A, const nc_complex* B, nc_complex* denormA,
                                nc_complex* normB) {
    NC_ABI_BEGIN
    HostStage h;
    const size_t na = (size_t)*bm * *bl * *dl, nbb = (size_t)*br * *bm * *dr;
    const cplx* dA = h.in(A, na);
    const cplx* dB = h.in(B, nbb);
    cplx* oA = h.out(na);
    cplx* oB = h.out(nbb);
    if (h.ctx.level0_polar) gauge_left_polar(h.ctx, *bl, *bm, *br, *dl, *dr, dA, dB, oA, oB);
    else gauge_left(h.ctx, *bl, *bm, *br, *dl, *dr, dA, dB, oA, oB);
    h.back(denormA, oA, na);
    h.back(normB, oB, nbb);
    h.sync();
    NC_ABI_END
    return g_status;
}

int32_t norm_denorm_going_right_(const uint32_t* bl, const uint32_t* bm, const uint32_t* br, const uint32_t* dl,
                                 const uint32_t* dr, const nc_complex* A, const nc_complex* B, nc_complex* normA,
                                 nc_complex* denormB) {
    NC_ABI_BEGIN
    HostStage h;
    const size_t na = (size_t)*bm * *bl * *dl, nbb = (size_t)*br * *bm * *dr;
    const cplx* dA = h.in(A, na);
    const cplx* dB = h.in(B, nbb);
    cplx* oA = h.out(na);
    cplx* oB = h.out(nbb);
    if (h.ctx.level0_polar) gauge_right_polar(h.ctx, *bl, *bm, *br, *dl, *dr, dA, dB, oA, oB);
    else gauge_right(h.ctx, *bl, *bm, *br, *dl, *dr, dA, dB, oA, oB);
    h.back(normA, oA, na);
    h.back(denormB, oB, nbb);
    h.sync();
    NC_ABI_END
    return g_status;
}

int nc_set_level0_gauge(int exact_polar) {
    NC_ABI_BEGIN
    Context::get().level0_polar = exact_polar != 0;
    NC_ABI_END
    return g_status;
}

int nc_gauge_move_dev(int direction, uint32_t bl, uint32_t bm, uint32_t br, uint32_t dl, uint32_t dr,
                      const void* A_dev, const void* B_dev, void* out_A_dev, void* out_B_dev) {
    NC_ABI_BEGIN
    NC_ARG(direction != 0 && A_dev && B_dev && out_A_dev && out_B_dev, "nc_gauge_move_dev: bad arguments");
    Context& ctx = Context::get();
    if (direction > 0)
        gauge_right(ctx, bl, bm, br, dl, dr, (const cplx*)A_dev, (const cplx*)B_dev, (cplx*)out_A_dev,
                    (cplx*)out_B_dev);
    else
        gauge_left(ctx, bl, bm, br, dl, dr, (const cplx*)A_dev, (const cplx*)B_dev, (cplx*)out_A_dev,
                   (cplx*)out_B_dev);
    NC_ABI_END
    return g_status;
}

int32_t norm_for_left_(const uint32_t* br, const uint32_t* bl, const uint32_t* d, const nc_complex* S,
                       nc_complex* out) {
    NC_ABI_BEGIN
    HostStage h;
    const size_t n = (size_t)*br * *bl * *d;
    const cplx* dS = h.in(S, n);
    cplx* o = h.out(n);
    if (h.ctx.level0_polar) gauge_right_polar(h.ctx, *bl, *br, 1, *d, 1, dS, nullptr, o, nullptr);
    else gauge_right(h.ctx, *bl, *br, 1, *d, 1, dS, nullptr, o, nullptr);
    h.back(out, o, n);
    h.sync();
    NC_ABI_END
    return g_status;
}

int32_t norm_for_right_(const uint32_t* br, const uint32_t* bl, const uint32_t* d, const nc_complex* S,
                        nc_complex* out) {
    NC_ABI_BEGIN
    HostStage h;
    const size_t n = (size_t)*br * *bl * *d;
    const cplx* dS = h.in(S, n);
    cplx* o = h.out(n);
    if (h.ctx.level0_polar) gauge_left_polar(h.ctx, 1, *bl, *br, 1, *d, nullptr, dS, nullptr, o);
    else gauge_left(h.ctx, 1, *bl, *br, 1, *d, nullptr, dS, nullptr, o);
    h.back(out, o, n);
    h.sync();
    NC_ABI_END
    return g_status;
}

int32_t increase_bandwidth_between_(const uint32_t* bl, const uint32_t* bm, const uint32_t* br, const uint32_t* dl,
                                    const uint32_t* dr, const uint32_t* new_bm, const nc_complex* A,
                                    const nc_complex* B, nc_complex* outA, nc_complex* outB) {
    NC_ABI_BEGIN
    HostStage h;
    NC_ARG(*new_bm >= *bm, "new bond dimension must not shrink");
    const size_t na = (size_t)*bm * *bl * *dl, nbb = (size_t)*br * *bm * *dr;
    const size_t oa = (size_t)*new_bm * *bl * *dl, ob = (size_t)*br * *new_bm * *dr;
    const cplx* dA = h.in(A, na);
    const cplx* dB = h.in(B, nbb);
    cplx* o1 = h.out(oa);
    cplx* o2 = h.out(ob);
    if (*new_bm > *bm)
        increase_bandwidth(h.ctx, *bl, *bm, *br, *dl, *dr, *new_bm, abi_seed(), dA, dB, o1, o2);
    else
        gauge_left(h.ctx, *bl, *bm, *br, *dl, *dr, dA, dB, o1, o2);
    h.back(outA, o1, oa);
    h.back(outB, o2, ob);
    h.sync();
    NC_ABI_END
    return g_status;
}

void rand_norm_state_site_tensor_(const uint32_t* br, const uint32_t* bl, const uint32_t* d, nc_complex* out) {
    NC_ABI_BEGIN
    HostStage h;
    const size_t n = (size_t)*br * *bl * *d;
    cplx* o = h.out(n);
    rand_norm_site(h.ctx, *br, *bl, *d, abi_seed(), o);
    h.back(out, o, n);
    h.sync();
    NC_ABI_END
}

void rand_unnorm_state_site_tensor_(const uint32_t* br, const uint32_t* bl, const uint32_t* d, nc_complex* out) {
    NC_ABI_BEGIN
    HostStage h;
    const size_t n = (size_t)*br * *bl * *d;
    cplx* o = h.out(n);
    rand_unnorm_site(h.ctx, *br, *bl, *d, abi_seed(), o);
    h.back(out, o, n);
    h.sync();
    NC_ABI_END
}

void form_norm_overlap_tensors_(const uint32_t* bl, const uint32_t* bm, const uint32_t* br, const uint32_t* dl,
                                const uint32_t* dr, const nc_complex* S1, const nc_complex* S2, nc_complex* lno,
                                nc_complex* uno, nc_complex* dS2, nc_complex* rno) {
    // core.f95:3315-3373
    NC_ABI_BEGIN
    HostStage h;
    const size_t n1 = (size_t)*bm * *bl * *dl, n2 = (size_t)*br * *bm * *dr;
    const cplx* d1 = h.in(S1, n1);
    const cplx* d2 = h.in(S2, n2);
    cplx* nS1 = h.out(n1);
    cplx* o_d2 = h.out(n2);
    cplx* o_l = h.out(n1);
    cplx* o_u = h.out(n1);
    cplx* o_r = h.out(n2);
    if (h.ctx.level0_polar) gauge_right_polar(h.ctx, *bl, *bm, *br, *dl, *dr, d1, d2, nS1, o_d2);
    else gauge_right(h.ctx, *bl, *bm, *br, *dl, *dr, d1, d2, nS1, o_d2);
    overlap_site_from_state(h.ctx, *bm, *bl, *dl, d1, o_u);
    overlap_site_from_state(h.ctx, *bm, *bl, *dl, nS1, o_l);
    overlap_site_from_state(h.ctx, *br, *bm, *dr, d2, o_r);
    h.back(lno, o_l, n1);
    h.back(uno, o_u, n1);
    h.back(dS2, o_d2, n2);
    h.back(rno, o_r, n2);
    h.sync();
    NC_ABI_END
}

}  // extern "C"
