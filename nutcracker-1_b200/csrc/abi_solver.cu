// Level-0 C-ABI: the site eigen-solve and the projector algebra
// (sources/common/core.cpp:420-760) on the GPU.
#include <cstring>
#include <vector>

#include "nc_abi_util.h"
#include "nc_common.cuh"
#include "nc_kernels.h"

using namespace nc;

namespace {

DevProjector stage_projector(HostStage& h, long long n, uint32_t nproj, uint32_t nrefl, uint32_t orth_dim,
                             const nc_complex* reflectors, const nc_complex* coefficients,
                             const uint32_t* swaps) {
    DevProjector P;
    P.n = n;
    P.nproj = (int)nproj;
    P.nrefl = (int)nrefl;
    P.orth_dim = orth_dim;
    if (nproj == 0) return P;
    NC_ARG(reflectors && coefficients && swaps, "projector data missing");
    NC_ARG(nrefl <= nproj && (long long)nrefl <= n, "bad number of reflectors");
    NC_ARG(nrefl <= (uint32_t)kMaxProjectors, "too many projectors");
    P.refl = h.in(reflectors, (size_t)n * nproj);
    P.tau = h.in(coefficients, nrefl);
    P.swaps.assign(swaps, swaps + nrefl);
    for (uint32_t s : P.swaps) NC_ARG(s >= 1 && s <= nrefl, "swap index out of range");
    return P;
}

}  // namespace

extern "C" {

uint32_t optimize_(const uint32_t* bl, const uint32_t* br, const uint32_t* cl, const uint32_t* cr,
                   const uint32_t* d, const nc_complex* L, const uint32_t* nnz, const uint32_t* idx,
                   const nc_complex* W, const nc_complex* R, const uint32_t* nproj, const uint32_t* nrefl,
                   const uint32_t* orth_dim, const nc_complex* reflectors, const nc_complex* coefficients,
                   const uint32_t* swaps, const char* which, const double* tol, uint32_t* iterations,
                   const nc_complex* guess, nc_complex* result, nc_complex* eigenvalue, double* normal) {
    int info = 0;
    NC_ABI_BEGIN
    HostStage h;
    MpoSite op = h.mpo(*d, *cl, *cr, *nnz, idx, W);
    const long long n = (long long)*br * *bl * *d;
    const cplx* dL = h.in(L, (size_t)*bl * *bl * *cl);
    const cplx* dR = h.in(R, (size_t)*br * *br * *cr);
    const cplx* dG = h.in(guess, n);
    DevProjector P = stage_projector(h, n, *nproj, *nrefl, *orth_dim, reflectors, coefficients, swaps);
    if (*nproj == 0) P.orth_dim = *orth_dim;
    cplx* res = h.out(n);
    double ev = 0, nrm = 0;
    EigenStats st;
    info = optimize_site(h.ctx, *bl, *br, op, dL, dR, P, parse_which(which), *tol, (int)*iterations, dG, res,
                         &ev, &nrm, &st);
    if (info == 0 || info < 0) {
        h.back(result, res, n);
        h.sync();
    }
    eigenvalue->re = ev;
    eigenvalue->im = 0;
    *normal = nrm;
    // strategy 1 reports no iterations (core.f95:2127); otherwise H_eff products
    const long long od = *nproj ? (long long)*orth_dim : n;
    *iterations = od <= 4 ? 0u : (uint32_t)st.matvecs;
    NC_ABI_END
    if (g_status != 0) return 0xFFFFFFFFu;
    return (uint32_t)info;
}

void convert_vectors_to_reflectors_(const uint32_t* n, const uint32_t* m, nc_complex* vectors, uint32_t* rank,
                                    nc_complex* coefficients, uint32_t* swaps) {
    NC_ABI_BEGIN
    HostStage h;
    const long long len = *n;
    const int cnt = (int)*m;
    if (cnt == 0) { *rank = 0; return; }
    cplx* A = const_cast<cplx*>(h.in(vectors, (size_t)len * cnt));
    const int k = (int)std::min<long long>(len, cnt);
    cplx* tau = h.out(k);
    std::vector<uint32_t> sw;
    int r = convert_vectors_to_reflectors_dev(h.ctx, len, cnt, A, tau, sw);
    h.back(vectors, A, (size_t)len * cnt);
    h.back(coefficients, tau, k);
    h.sync();
    std::memcpy(swaps, sw.data(), sw.size() * sizeof(uint32_t));
    *rank = (uint32_t)r;
    NC_ABI_END
}

void filter_components_outside_orthog_(const uint32_t* n, const uint32_t* nproj, const uint32_t* nrefl,
                                       const uint32_t* orth_dim, const nc_complex* reflectors,
                                       const nc_complex* coefficients, const uint32_t* swaps,
                                       const nc_complex* input, nc_complex* output) {
    NC_ABI_BEGIN
    HostStage h;
    DevProjector P = stage_projector(h, *n, *nproj, *nrefl, *orth_dim, reflectors, coefficients, swaps);
    const cplx* x = h.in(input, *n);
    cplx* y = h.out(*n);
    filter_outside(h.ctx, P, x, y);
    h.back(output, y, *n);
    h.sync();
    NC_ABI_END
}

void compute_overlap_with_projectors_(const uint32_t* nproj, const uint32_t* nrefl, const nc_complex* reflectors,
                                      const nc_complex* coefficients, const uint32_t* swaps,
                                      const uint32_t* vector_size, const nc_complex* vector,
                                      nc_complex* overlap) {
    NC_ABI_BEGIN
    HostStage h;
    DevProjector P = stage_projector(h, *vector_size, *nproj, *nrefl, *vector_size, reflectors, coefficients,
                                     swaps);
    const cplx* x = h.in(vector, *vector_size);
    double v = overlap_with_projectors(h.ctx, P, x);
    overlap->re = v;  // the Fortran routine writes a real; the imaginary part is zeroed
    overlap->im = 0;
    NC_ABI_END
}

void random_projector_matrix_(const uint32_t* projector_length, const uint32_t* number_of_projectors,
                              uint32_t* rank, nc_complex* reflectors, nc_complex* coefficients,
                              uint32_t* swaps) {
    NC_ABI_BEGIN
    HostStage h;
    const long long len = *projector_length;
    const int cnt = (int)*number_of_projectors;
    if (cnt == 0) { *rank = 0; return; }
    cplx* A = h.out((size_t)len * cnt);
    static thread_local uint64_t counter = 0;
    zrandom(h.ctx, len * cnt, 0xA5A5ull + 1315423911ull * (++counter), A);
    const int k = (int)std::min<long long>(len, cnt);
    cplx* tau = h.out(k);
    std::vector<uint32_t> sw;
    int r = convert_vectors_to_reflectors_dev(h.ctx, len, cnt, A, tau, sw);
    h.back(reflectors, A, (size_t)len * cnt);
    h.back(coefficients, tau, k);
    h.sync();
    std::memcpy(swaps, sw.data(), sw.size() * sizeof(uint32_t));
    *rank = (uint32_t)r;
    NC_ABI_END
}

int nc_set_krylov_dimension(int m) {
    NC_ABI_BEGIN
    NC_ARG(m >= 2 && m <= 128, "Krylov dimension must be in [2, 128]");
    Context::get().krylov_dim = m;
    NC_ABI_END
    return g_status;
}

}  // extern "C"
