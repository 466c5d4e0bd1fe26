// Device-resident chain: the sweep driver of the reference
// (sources/common/chain.cpp, base_chain.cpp, includes/nutcracker/chain.hpp)
// with every site tensor, expectation environment, overlap environment and
// projector site kept in HBM across sweeps.  The host runs only the control
// flow of the reference (cursor moves, acceptance rule, convergence tests)
// and reads back a handful of scalars per site.
//
// Storage: site[i] (br,bl,d); Lenv[i] = environment left of site i
// (bl,bl,cl), valid for i <= cursor; Renv[i] = environment right of site i
// (br,br,cr), valid for i >= cursor; likewise Lov/Rov per projector.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "nc_abi_util.h"
#include "nc_common.cuh"
#include "nc_kernels.h"
#include "nc_chain.h"

namespace nc {

namespace {

// Device buffer in stream-ordered memory (cudaMallocAsync / cudaFreeAsync on
// the allocating thread's stream): freeing a chain never synchronises the
// whole device, so chains run by other threads (the serving loop) keep going.
void keep_pool_memory() {
    static PerDeviceOnce once;   // the pool attribute belongs to each device's default pool
    once([] {
        int dev = 0;
        cudaMemPool_t pool;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;   // freed blocks stay in this process's pool
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
    });
}

struct DevBuf {
    cplx* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    DevBuf() {}
    explicit DevBuf(size_t count) { alloc(count); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; s = o.s; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t count) {
        release();
        keep_pool_memory();
        if (count == 0) count = 1;
        s = Context::get().stream;
        cudaError_t e = cudaMallocAsync(&p, count * sizeof(cplx), s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);   // usable from any stream and the host from here on
        if (e != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            throw Error(NC_ERR_NOMEM, "chain: allocation of " + std::to_string(count * sizeof(cplx)) + " bytes failed");
        }
        n = count;
    }
    void ensure(size_t count) { if (n < count) alloc(count); }
    void release() { if (p) cudaFreeAsync(p, s); p = nullptr; n = 0; }
};

// Second stream (and its two events) on which a move's neighbour absorbs the
// gauge factor while the environment update runs on the chain's stream.
struct SideStream {
    AbsorbAsync a{nullptr, nullptr, nullptr};
    SideStream() {
        cudaError_t e = cudaStreamCreateWithFlags(&a.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&a.ready, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&a.done, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            cudaGetLastError();
            destroy();
            throw Error(NC_ERR_CUDA, std::string("chain: side stream: ") + cudaGetErrorString(e));
        }
    }
    SideStream(const SideStream&) = delete;
    SideStream& operator=(const SideStream&) = delete;
    ~SideStream() { destroy(); }
    void destroy() {
        if (a.stream) { cudaStreamSynchronize(a.stream); cudaStreamDestroy(a.stream); }
        if (a.ready) cudaEventDestroy(a.ready);
        if (a.done) cudaEventDestroy(a.done);
        a = AbsorbAsync{nullptr, nullptr, nullptr};
    }
};

struct OpSite {
    MpoSite dev;
    DevBuf W;
    DevBuf idxbuf;   // (2,nnz) uint32 indices
    uint32_t* idx = nullptr;
};

struct ProjSite {
    DevBuf left, middle, right;    // overlap sites (bl,d,br) of the left-normalised, centre and right-normalised state
    int bl = 0, br = 0, d = 0;
};

// Diagnostic phase timer: synchronises the stream on entry and exit and adds
// the wall time to `acc` (only when the chain's time_phases option is set).
struct PhaseTimer {
    cudaStream_t s;
    double* acc;
    std::chrono::steady_clock::time_point t0;
    PhaseTimer(bool on, cudaStream_t st, double* a) : s(st), acc(on ? a : nullptr) {
        if (acc) {
            cudaStreamSynchronize(s);
            t0 = std::chrono::steady_clock::now();
        }
    }
    ~PhaseTimer() {
        if (acc) {
            cudaStreamSynchronize(s);
            *acc += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        }
    }
};

inline bool outside_tolerance(double a, double b, double tol) {
    // utilities.hpp:418-420
    return (std::fabs(a) + std::fabs(b)) / 2 > tol && std::fabs(a - b) / (std::fabs(a) + std::fabs(b) + tol) > tol;
}

}  // namespace

struct Chain {
    Context& ctx;
    ChainOptions opt;
    int N = 0;
    std::vector<int> phys;
    std::vector<std::unique_ptr<OpSite>> ops;
    std::vector<int> bonds;               // bond dimensions, size N+1
    std::vector<DevBuf> site, Lenv, Renv;
    std::vector<std::vector<DevBuf>> Lov, Rov;   // [projector][site]
    std::vector<std::vector<ProjSite>> projectors;
    DevBuf spare_a, spare_b;
    SideStream side;
    // projector matrix of the current site
    DevBuf pm_refl, pm_tau;
    DevProjector pm;
    int cur = 0;
    int bandwidth = 1;
    int max_bandwidth = 1;
    double energy = 0;
    bool optimized = false;
    uint64_t seed_counter = 0;
    ChainStats stats;
    // Signals (base_chain.hpp:54-60, chain.hpp:151): host callbacks run on the
    // calling thread, in connection order, when the event happens.
    struct Slot {
        int64_t id;
        int signal;
        nc_chain_signal_fn fn;
        void* user;
    };
    std::vector<Slot> slots;
    int64_t next_slot = 1;
    nc_chain* handle = nullptr;
    int last_matvecs = 0;
    void emit(int signal, int64_t value) {
        const std::vector<Slot> now = slots;   // callbacks may connect or disconnect
        for (const Slot& s : now)
            if (s.signal == signal) s.fn(handle, signal, value, s.user);
    }
    // precision form: 0 = FP64 sweeps, 1 = 3xTF32 tensor-core products
    int prec = 0;
    int free_sweeps = 0;   // sweeps still exempt from the regression check (after a precision hand-over)
    DevBuf mixbuf;       // MixedHeff operands of the current site (float storage)
    MixedHeff mh;

    // Work on this chain's stream finishes before its buffers return to the pool.
    ~Chain() { cudaStreamSynchronize(ctx.stream); }

    Chain(Context& c, int n, const OperatorSiteDesc* sites, const ChainOptions& o) : ctx(c), opt(o), N(n) {
        NC_ARG(N >= 1, "chain needs at least one site");
        for (int i = 0; i < N; ++i) {
            const OperatorSiteDesc& s = sites[i];
            NC_ARG(s.nnz >= 1 && s.d >= 1 && s.cl >= 1 && s.cr >= 1, "bad operator site");
            for (uint32_t q = 0; q < s.nnz; ++q) {
                NC_ARG(s.idx[2 * q] >= 1 && s.idx[2 * q] <= s.cl, "operator index 'from' out of range");
                NC_ARG(s.idx[2 * q + 1] >= 1 && s.idx[2 * q + 1] <= s.cr, "operator index 'to' out of range");
            }
            if (i > 0) NC_ARG(sites[i - 1].cr == s.cl, "operator bond dimensions do not connect");
            auto op = std::make_unique<OpSite>();
            op->W.alloc((size_t)s.d * s.d * s.nnz);
            op->idxbuf.alloc((2 * s.nnz * sizeof(uint32_t) + sizeof(cplx) - 1) / sizeof(cplx));
            op->idx = reinterpret_cast<uint32_t*>(op->idxbuf.p);
            NC_CUDA(cudaMemcpy(op->W.p, s.W, (size_t)s.d * s.d * s.nnz * sizeof(cplx), cudaMemcpyHostToDevice));
            NC_CUDA(cudaMemcpy(op->idx, s.idx, 2 * s.nnz * sizeof(uint32_t), cudaMemcpyHostToDevice));
            op->dev.d = (int)s.d; op->dev.cl = (int)s.cl; op->dev.cr = (int)s.cr; op->dev.nnz = (int)s.nnz;
            op->dev.idx = op->idx; op->dev.W = op->W.p;
            ops.push_back(std::move(op));
            phys.push_back((int)s.d);
        }
        NC_ARG(ops.front()->dev.cl == 1 && ops.back()->dev.cr == 1, "operator boundary dimensions must be 1");
        NC_ARG(opt.precision == 0 || opt.precision == 1, "precision must be 0 (FP64) or 1 (mixed)");
        prec = opt.precision;
        max_bandwidth = maximum_bandwidth_dimension(phys);
        ctx.krylov_dim = opt.krylov_dim;
        reset();
    }

    // ---- bond dimensions (utilities.cpp:32-91, utilities.hpp:264-283) ----------
    static int maximum_bandwidth_dimension(const std::vector<int>& p) {
        if (p.size() == 1) return 1;
        size_t mid = (p.size() + 1) / 2;
        long long a = 1, b = 1;
        for (size_t i = 0; i < mid; ++i) { a = std::min<long long>(a * p[i], 1LL << 40); }
        for (size_t i = 0; i < mid; ++i) { b = std::min<long long>(b * p[p.size() - 1 - i], 1LL << 40); }
        return (int)std::min<long long>(std::min(a, b), 1 << 30);
    }

    static std::vector<int> bandwidth_sequence(int requested, const std::vector<int>& p) {
        if (requested == 0) throw Error(NC_ERR_ARG, "requested bandwidth must be > 0");
        const size_t mid = (p.size() + 1) / 2;
        auto side = [&](bool rev) {
            std::vector<int> out{1};
            long long prod = 1;
            for (size_t i = 0; i < mid; ++i) {
                prod *= p[rev ? p.size() - 1 - i : i];
                if (prod >= requested) break;
                out.push_back((int)prod);
            }
            return out;
        };
        std::vector<int> fwd = side(false), rev = side(true);
        if (fwd.size() == mid + 1 || rev.size() == mid + 1)
            throw Error(NC_ERR_ARG, "requested bandwidth dimension too large: " + std::to_string(requested));
        std::vector<int> seq = fwd;
        for (size_t i = 0; i < p.size() + 1 - fwd.size() - rev.size(); ++i) seq.push_back(requested);
        for (auto it = rev.rbegin(); it != rev.rend(); ++it) seq.push_back(*it);
        return seq;
    }

    int minimum_bandwidth_for_projectors(int nproj) const {
        // projectors.cpp:108-133
        if (nproj == 0) return 1;
        for (int b = 1;; ++b) {
            std::vector<int> seq = bandwidth_sequence(b, phys);
            for (int i = 0; i < N; ++i)
                if ((long long)phys[i] * seq[i] * seq[i + 1] > nproj) return b;
        }
    }

    // ---- sizes ------------------------------------------------------------------
    int bl(int i) const { return bonds[i]; }
    int br(int i) const { return bonds[i + 1]; }
    size_t site_elems(int i) const { return (size_t)bonds[i + 1] * bonds[i] * phys[i]; }
    const MpoSite& op(int i) const { return ops[i]->dev; }

    void allocate_for_bonds() {
        site.resize(N); Lenv.resize(N); Renv.resize(N);
        size_t maxs = 1;
        for (int i = 0; i < N; ++i) maxs = std::max(maxs, site_elems(i));
        for (int i = 0; i < N; ++i) {
            // every site buffer gets the largest site's capacity: moves and
            // accepted solves swap site buffers with the spares
            site[i].ensure(maxs);
            Lenv[i].ensure((size_t)bl(i) * bl(i) * op(i).cl);
            Renv[i].ensure((size_t)br(i) * br(i) * op(i).cr);
        }
        spare_a.ensure(maxs);
        spare_b.ensure(maxs);
        const size_t np = projectors.size();
        Lov.resize(np); Rov.resize(np);
        for (size_t p = 0; p < np; ++p) {
            Lov[p].resize(N); Rov[p].resize(N);
            for (int i = 0; i < N; ++i) {
                Lov[p][i].ensure((size_t)bl(i) * projectors[p][i].bl);
                Rov[p][i].ensure((size_t)projectors[p][i].br * br(i));
            }
        }
    }

    void set_trivial(cplx* p) { zfill(ctx, 1, cmake(1, 0), p); }

    void reset_boundaries() {
        set_trivial(Lenv[0].p);
        set_trivial(Renv[N - 1].p);
        for (size_t p = 0; p < projectors.size(); ++p) {
            set_trivial(Lov[p][0].p);
            set_trivial(Rov[p][N - 1].p);
        }
    }

    // Right environments (and overlap environments) of site i-1 from site i.
    void absorb_right(int i) {
        if (prec) sos_right_mixed(ctx, bl(i), br(i), op(i), Renv[i].p, site[i].p, Renv[i - 1].p);
        else sos_right(ctx, bl(i), br(i), op(i), Renv[i].p, site[i].p, Renv[i - 1].p);
        for (size_t p = 0; p < projectors.size(); ++p) {
            const ProjSite& ps = projectors[p][i];
            vs_right(ctx, ps.bl, ps.br, bl(i), br(i), phys[i], Rov[p][i].p, ps.right.p, site[i].p, Rov[p][i - 1].p);
        }
    }
    void absorb_left(int i) {
        if (prec) sos_left_mixed(ctx, bl(i), br(i), op(i), Lenv[i].p, site[i].p, Lenv[i + 1].p);
        else sos_left(ctx, bl(i), br(i), op(i), Lenv[i].p, site[i].p, Lenv[i + 1].p);
        for (size_t p = 0; p < projectors.size(); ++p) {
            const ProjSite& ps = projectors[p][i];
            vs_left(ctx, ps.bl, ps.br, bl(i), br(i), phys[i], Lov[p][i].p, ps.left.p, site[i].p, Lov[p][i + 1].p);
        }
    }

    // ---- projector matrix (projectors.hpp:406-485) ------------------------------
    void reset_projector_matrix() {
        const int np = (int)projectors.size();
        pm = DevProjector();
        if (np == 0) return;
        const long long n = (long long)site_elems(cur);
        pm_refl.ensure((size_t)n * np);
        pm_tau.ensure(np);
        for (int p = 0; p < np; ++p) {
            const ProjSite& ps = projectors[p][cur];
            overlap_vector(ctx, ps.bl, ps.br, bl(cur), br(cur), phys[cur], Lov[p][cur].p, Rov[p][cur].p, ps.middle.p,
                           pm_refl.p + (size_t)p * n);
        }
        std::vector<uint32_t> sw;
        int rank = convert_vectors_to_reflectors_dev(ctx, n, np, pm_refl.p, pm_tau.p, sw);
        pm.nproj = np;
        pm.nrefl = (int)std::min<long long>(n, np);
        pm.n = n;
        pm.orth_dim = n - rank;
        pm.refl = pm_refl.p;
        pm.tau = pm_tau.p;
        pm.swaps = sw;
    }

    // ---- energies ---------------------------------------------------------------
    double expectation_value() {
        ArenaFrame f(ctx.arena);
        cplx* r = ctx.arena.alloc_n<cplx>(1);
        expectation_dev(ctx, bl(cur), br(cur), op(cur), Lenv[cur].p, site[cur].p, Renv[cur].p, r);
        cplx v = read_scalar(ctx, r);
        last_expectation = v;
        return v.x;
    }
    cplx last_expectation = cmake(0, 0);

    double norm_of(const cplx* x, long long n) {
        ArenaFrame f(ctx.arena);
        cplx* r = ctx.arena.alloc_n<cplx>(1);
        znrm2sq(ctx, n, x, r);
        return std::sqrt(read_scalar(ctx, r).x);
    }

    void normalize(cplx* x, long long n) {
        ArenaFrame f(ctx.arena);
        cplx* r = ctx.arena.alloc_n<cplx>(1);
        znrm2sq(ctx, n, x, r);
        znormalize_dev(ctx, n, r, x);
    }

    // ---- reset (chain.cpp:175-237) ------------------------------------------------
    void reset(const std::vector<int>* given_bonds = nullptr, const std::vector<const cplx*>* given_sites = nullptr) {
        optimized = false;
        if (given_bonds) {
            bonds = *given_bonds;
            bandwidth = *std::max_element(bonds.begin(), bonds.end());
        } else {
            bandwidth = std::min(max_bandwidth, std::max<int>((int)opt.initial_bandwidth_dimension,
                                                              minimum_bandwidth_for_projectors((int)projectors.size())));
            bonds = bandwidth_sequence(bandwidth, phys);
        }
        allocate_for_bonds();
        cur = 0;
        reset_boundaries();
        for (int i = N - 1; i >= 1; --i) {
            if (given_sites) {
                NC_CUDA(cudaMemcpyAsync(site[i].p, (*given_sites)[i], site_elems(i) * sizeof(cplx),
                                        cudaMemcpyHostToDevice, ctx.stream));
            } else {
                rand_norm_site(ctx, br(i), bl(i), phys[i], next_seed(), site[i].p);
            }
            absorb_right(i);
        }
        if (given_sites) {
            NC_CUDA(cudaMemcpyAsync(site[0].p, (*given_sites)[0], site_elems(0) * sizeof(cplx), cudaMemcpyHostToDevice,
                                    ctx.stream));
        } else {
            rand_unnorm_site(ctx, br(0), bl(0), phys[0], next_seed(), site[0].p);
        }
        reset_projector_matrix();
        if (!projectors.empty()) {
            while (pm.orth_dim == 0) move(+1);
            // applyProjectorMatrix (projectors.cpp:18-38)
            filter_outside(ctx, pm, site[cur].p, site[cur].p);
            double nrm = norm_of(site[cur].p, (long long)site_elems(cur));
            if (!(nrm > 1e-7)) throw Error(NC_ERR_NUMERIC, "projected initial site vanished");
            normalize(site[cur].p, (long long)site_elems(cur));
            move_to(0);
        }
        double e = expectation_value();
        // The precision form's products carry ~1e-6 relative error, so its
        // imaginary part is measured against an energy scale that cannot
        // vanish (a random initial state can have an energy near zero).
        const double mag = std::hypot(last_expectation.x, last_expectation.y);
        const double scale = prec ? std::max(mag, (double)N) : mag;
        const double imag_tol = prec ? kMixedSanity : 1e-10;
        if (std::fabs(last_expectation.y) / scale > imag_tol)
            throw Error(NC_ERR_NUMERIC, "initial chain energy is not real");
        energy = e;
        emit(NC_SIGNAL_CHAIN_RESET, 0);   // chain.cpp:236
    }

    uint64_t next_seed() { return opt.seed * 0x9E3779B97F4A7C15ull + (++seed_counter) * 0xD1B54A32D192ED03ull; }

    // ---- cursor moves (chain.hpp:287-315, states.cpp:94-164) ---------------------
    void move(int dir) {
        optimized = false;
        const int c = cur;
        if (dir > 0) {
            NC_ARG(c + 1 < N, "cannot move right from the last site");
            {
                // site c -> left-normalised, site c+1 absorbs the factor and becomes the centre
                PhaseTimer t(opt.time_phases, ctx.stream, &stats.t_gauge);
                gauge_right(ctx, bl(c), br(c), br(c + 1), phys[c], phys[c + 1], site[c].p, site[c + 1].p,
                            spare_a.p, spare_b.p, &side.a);
                std::swap(site[c], spare_a);
                std::swap(site[c + 1], spare_b);
            }
            {
                // the environment update needs only the normalised site c, so it
                // overlaps the absorption GEMM running on the side stream
                PhaseTimer t(opt.time_phases, ctx.stream, &stats.t_env);
                absorb_left(c);
            }
            {
                PhaseTimer t(opt.time_phases, ctx.stream, &stats.t_gauge);
                NC_CUDA(cudaStreamWaitEvent(ctx.stream, side.a.done, 0));
                normalize(site[c + 1].p, (long long)site_elems(c + 1));
            }
            cur = c + 1;
        } else {
            NC_ARG(c > 0, "cannot move left from the first site");
            {
                PhaseTimer t(opt.time_phases, ctx.stream, &stats.t_gauge);
                gauge_left(ctx, bl(c - 1), br(c - 1), br(c), phys[c - 1], phys[c], site[c - 1].p, site[c].p,
                           spare_a.p, spare_b.p, &side.a);
                std::swap(site[c - 1], spare_a);
                std::swap(site[c], spare_b);
            }
            {
                PhaseTimer t(opt.time_phases, ctx.stream, &stats.t_env);
                absorb_right(c);
            }
            {
                PhaseTimer t(opt.time_phases, ctx.stream, &stats.t_gauge);
                NC_CUDA(cudaStreamWaitEvent(ctx.stream, side.a.done, 0));
                normalize(site[c - 1].p, (long long)site_elems(c - 1));
            }
            cur = c - 1;
        }
        stats.moves++;
        PhaseTimer t(opt.time_phases, ctx.stream, &stats.t_proj);
        reset_projector_matrix();
    }

    void move_to(int n) {
        while (cur > n) move(-1);
        while (cur < n) move(+1);
    }

    // ---- optimisation (base_chain.cpp:81-110, optimizer.cpp:201-315) ------------
    bool regression(double from, double to, double tol) const {
        if (opt.mode == WHICH_SR) return to > from && outside_tolerance(from, to, tol);
        if (opt.mode == WHICH_LR) return to < from && outside_tolerance(from, to, tol);
        return std::fabs(to) < std::fabs(from) && outside_tolerance(std::fabs(from), std::fabs(to), tol);
    }

    int optimize_site_once() {
        PhaseTimer timer(opt.time_phases, ctx.stream, &stats.t_solve);
        const long long n = (long long)site_elems(cur);
        double ev = 0, normal = 0;
        EigenStats es;
        DevProjector P = pm;
        if (P.nproj == 0) { P.n = n; P.orth_dim = n; }
        const MixedHeff* mixed = nullptr;
        if (prec) {
            const size_t floats = mixed_heff_floats(bl(cur), br(cur), op(cur));
            mixbuf.ensure((floats + 3) / 4);
            mixed_heff_prepare(ctx, bl(cur), br(cur), op(cur), Lenv[cur].p, Renv[cur].p,
                               reinterpret_cast<float*>(mixbuf.p), &mh);
            mixed = &mh;
        }
        const double site_tol = prec ? std::max(opt.site_convergence_threshold, kMixedSiteTol)
                                     : opt.site_convergence_threshold;
        int info = nc::optimize_site(ctx, bl(cur), br(cur), op(cur), Lenv[cur].p, Renv[cur].p, P, opt.mode, site_tol,
                                     (int)opt.maximum_number_of_iterations, site[cur].p, spare_a.p, &ev, &normal, &es,
                                     mixed);
        stats.matvecs += es.matvecs;
        last_matvecs = es.matvecs;
        stats.site_solves++;
        const double sanity = prec ? std::max(opt.sanity_check_threshold, kMixedSanity) : opt.sanity_check_threshold;
        int failure = 0;
        if (info == -14) failure = NC_FAIL_UNABLE_TO_CONVERGE;
        else if (info == 10) failure = NC_FAIL_TOO_MANY_PROJECTORS;
        else if (info == 11) failure = NC_FAIL_GUESS_IN_PROJECTOR_SPACE;
        else if (info != 0) failure = NC_FAIL_UNKNOWN;
        if (!failure) {
            // sanity checks of optimizer.cpp:266-309 on the new site
            ArenaFrame f(ctx.arena);
            cplx* r = ctx.arena.alloc_n<cplx>(1);
            if (prec) expectation_mixed(ctx, mh, spare_a.p, r);
            else expectation_dev(ctx, bl(cur), br(cur), op(cur), Lenv[cur].p, spare_a.p, Renv[cur].p, r);
            cplx ex = read_scalar(ctx, r);
            double overlap = (pm.nproj > 0) ? overlap_with_projectors(ctx, pm, spare_a.p) : 0.0;
            // outsideTolerance on complex numbers (utilities.hpp:418-420 with |.| = modulus)
            const double aa = std::fabs(ev), bb = std::hypot(ex.x, ex.y), dd = std::hypot(ev - ex.x, ex.y);
            if ((aa + bb) / 2 > sanity && dd / (aa + bb + sanity) > sanity)
                failure = NC_FAIL_EIGENVALUE_NOT_EXPECTATION;
            else if (normal < 1 - sanity)
                failure = NC_FAIL_VANISHING_EIGENVECTOR;
            else if (overlap > sanity)
                failure = NC_FAIL_EIGENVECTOR_IN_PROJECTOR_SPACE;
            else if (free_sweeps == 0 && regression(energy, ev, sanity))
                failure = NC_FAIL_REGRESSIVE_EIGENVALUE;
        }
        if (failure) {
            stats.failures++;
            stats.last_failure = failure;
            return failure;
        }
        // acceptance rule (base_chain.cpp:97-103)
        if ((energy >= 0 && ev >= 0) || (energy <= 0 && ev <= 0) ||
            outside_tolerance(std::fabs(energy), std::fabs(ev), sanity)) {
            energy = ev;
            std::swap(site[cur], spare_a);
        }
        optimized = true;
        return 0;
    }

    int optimize_site() {
        last_matvecs = 0;
        int f = optimize_site_once();
        // base_chain.cpp:104-109: success carries the solver's iteration count
        // (here its H_eff products), failure the failure kind
        if (f) emit(NC_SIGNAL_OPTIMIZE_SITE_FAILURE, f);
        else emit(NC_SIGNAL_OPTIMIZE_SITE_SUCCESS, last_matvecs);
        if (f && opt.strict) throw Error(NC_ERR_NUMERIC, "site optimisation failed (code " + std::to_string(f) + ")");
        return f;
    }

    void perform_optimization_sweep() {
        // chain.cpp:147-163
        const int start = cur;
        if (!optimized) optimize_site();
        while (cur + 1 < N) { move(+1); optimize_site(); }
        while (cur > 0) { move(-1); optimize_site(); }
        while (cur < start) { move(+1); optimize_site(); }
        if (prec) {
            tc_check(ctx);
            stats.mixed_sweeps++;
        }
        if (free_sweeps > 0) --free_sweeps;
        stats.sweeps++;
        emit(NC_SIGNAL_SWEEP_PERFORMED, (int64_t)stats.sweeps);   // chain.cpp:162
    }

    void sweep_until_converged() {
        if (prec) {
            // precision form: mixed sweeps to kMixedSweepTol, then FP64
            // sweeps (the refinement) to the options' threshold
            double prev = energy;
            perform_optimization_sweep();
            double now = energy;
            for (int count = 1; count < kMixedMaxSweeps && outside_tolerance(prev, now, kMixedSweepTol); ++count) {
                perform_optimization_sweep();
                prev = now;
                now = energy;
            }
            prec = 0;
            try {
                refresh_environments();
                sweep_until_converged_fp64();
            } catch (...) {
                prec = 1;
                throw;
            }
            prec = 1;
            return;
        }
        sweep_until_converged_fp64();
    }

    // Rebuild every environment for the current state at the current
    // precision and take the current site's expectation value as the energy
    // reference (used when the mixed sweeps hand over to the FP64 ones, whose
    // regression checks must not compare against mixed-precision energies).
    //
    // The first sweep after the hand-over is exempt from the regression
    // check: with projectors, the mixed sweeps' orthogonality to the lower
    // levels holds only to ~1e-6, and restoring it in FP64 legitimately
    // raises the energy.
    void refresh_environments() {
        for (int i = 0; i < cur; ++i) absorb_left(i);
        for (int i = N - 1; i > cur; --i) absorb_right(i);
        energy = expectation_value();
        optimized = false;
        free_sweeps = 1;
    }

    void sweep_until_converged_fp64() {
        // base_chain.cpp:112-123
        double prev = energy;
        perform_optimization_sweep();
        double now = energy;
        uint64_t count = 1;
        while (outside_tolerance(prev, now, opt.sweep_convergence_threshold)) {
            // the reference loops without bound (slow linear convergence of a
            // level at a small bond dimension can take ~1000 sweeps at the
            // 1e-12 default); maximum_sweeps, when set, turns that into an error
            if (opt.maximum_sweeps && ++count > opt.maximum_sweeps)
                throw Error(NC_ERR_NUMERIC, "sweeps did not converge");
            perform_optimization_sweep();
            prev = now;
            now = energy;
        }
        emit(NC_SIGNAL_SWEEPS_CONVERGED, 0);   // base_chain.cpp:122
    }

    void increase_bandwidth_dimension(int new_b) {
        // chain.cpp:75-122
        optimized = false;
        if (new_b == bandwidth) return;
        NC_ARG(new_b > bandwidth && new_b <= max_bandwidth, "bad new bandwidth dimension");
        NC_ARG(cur == 0, "chain must be at the first site");
        std::vector<int> nb = bandwidth_sequence(new_b, phys);
        // grow bond by bond from the right end (pairs (i-1, i), i = N-1 .. 1); the
        // left site of each pair carries the weight into the next pair
        std::vector<DevBuf> cur_site(N);
        for (int i = 0; i < N; ++i) {
            cur_site[i].alloc(site_elems(i));
            NC_CUDA(cudaMemcpyAsync(cur_site[i].p, site[i].p, site_elems(i) * sizeof(cplx), cudaMemcpyDeviceToDevice,
                                    ctx.stream));
        }
        std::vector<int> dims = bonds;
        for (int i = N - 1; i >= 1; --i) {
            const int blp = dims[i - 1], bm = dims[i], brr = dims[i + 1];
            const int nbm = nb[i];
            DevBuf a((size_t)nbm * blp * phys[i - 1]), b((size_t)brr * nbm * phys[i]);
            if (nbm > bm) {
                increase_bandwidth(ctx, blp, bm, brr, phys[i - 1], phys[i], nbm, next_seed(), cur_site[i - 1].p,
                                   cur_site[i].p, a.p, b.p);
            } else {
                gauge_left(ctx, blp, bm, brr, phys[i - 1], phys[i], cur_site[i - 1].p, cur_site[i].p, a.p, b.p);
            }
            dims[i] = nbm;
            cur_site[i - 1] = std::move(a);
            cur_site[i] = std::move(b);
        }
        bonds = nb;
        bandwidth = new_b;
        // re-allocate environments for the new bonds and rebuild them from the right
        site.clear(); Lenv.clear(); Renv.clear();
        for (auto& v : Lov) v.clear();
        for (auto& v : Rov) v.clear();
        allocate_for_bonds();
        for (int i = 0; i < N; ++i)
            NC_CUDA(cudaMemcpyAsync(site[i].p, cur_site[i].p, site_elems(i) * sizeof(cplx), cudaMemcpyDeviceToDevice,
                                    ctx.stream));
        reset_boundaries();
        for (int i = N - 1; i >= 1; --i) absorb_right(i);
        cur = 0;
        reset_projector_matrix();
        NC_CUDA(cudaStreamSynchronize(ctx.stream));
    }

    void optimize_chain() {
        // base_chain.cpp:64-79
        sweep_until_converged();
        double prev = energy;
        increase_bandwidth_dimension(std::min<int>(bandwidth + (int)opt.bandwidth_increment, max_bandwidth));
        sweep_until_converged();
        double now = energy;
        while (outside_tolerance(prev, now, opt.chain_convergence_threshold) && bandwidth < max_bandwidth) {
            increase_bandwidth_dimension(std::min<int>(bandwidth + (int)opt.bandwidth_increment, max_bandwidth));
            sweep_until_converged();
            prev = now;
            now = energy;
        }
        emit(NC_SIGNAL_CHAIN_OPTIMIZED, 0);   // base_chain.cpp:78
    }

    void construct_and_add_projector_from_state() {
        // chain.cpp:63-73 + projectors.hpp:324-359 + core.f95:3315-3373
        optimized = false;
        NC_ARG(cur == 0, "chain must be at the first site");
        std::vector<ProjSite> proj(N);
        DevBuf centre(site_elems(0));
        NC_CUDA(cudaMemcpyAsync(centre.p, site[0].p, site_elems(0) * sizeof(cplx), cudaMemcpyDeviceToDevice,
                                ctx.stream));
        for (int i = 0; i < N; ++i) {
            ProjSite& ps = proj[i];
            ps.bl = bl(i); ps.br = br(i); ps.d = phys[i];
            const size_t ne = site_elems(i);
            ps.middle.alloc(ne);
            overlap_site_from_state(ctx, br(i), bl(i), phys[i], centre.p, ps.middle.p);
            if (i + 1 < N) {
                DevBuf normc(ne), next(site_elems(i + 1));
                gauge_right(ctx, bl(i), br(i), br(i + 1), phys[i], phys[i + 1], centre.p, site[i + 1].p, normc.p,
                            next.p);
                ps.left.alloc(ne);
                overlap_site_from_state(ctx, br(i), bl(i), phys[i], normc.p, ps.left.p);
                proj[i + 1].right.alloc(site_elems(i + 1));
                overlap_site_from_state(ctx, br(i + 1), bl(i + 1), phys[i + 1], site[i + 1].p, proj[i + 1].right.p);
                centre = std::move(next);
            }
        }
        if (!proj[0].right.p) proj[0].right.alloc(1);
        if (!proj[N - 1].left.p) proj[N - 1].left.alloc(1);
        NC_CUDA(cudaStreamSynchronize(ctx.stream));
        projectors.push_back(std::move(proj));
    }

    void solve_for_multiple_levels(int n, double* energies) {
        // chain.cpp:301-310
        for (int k = 0; k < n - 1; ++k) {
            optimize_chain();
            if (energies) energies[k] = energy;
            construct_and_add_projector_from_state();
            reset();
        }
        optimize_chain();
        if (energies) energies[n - 1] = energy;
    }

    // n levels at the current bond dimension: sweepUntilConverged per level
    // (solve_for_multiple_levels with optimize_chain replaced; no chi growth).
    void solve_levels_at_bandwidth(int n, double* energies) {
        for (int k = 0; k < n; ++k) {
            if (k > 0) {
                construct_and_add_projector_from_state();
                reset();
            }
            sweep_until_converged();
            if (energies) energies[k] = energy;
        }
    }

    // Device bytes a chain of this operator needs at bond dimension
    // `bandwidth` for `levels` levels: the buffers allocate_for_bonds and the
    // projector sites hold, plus the solver's arena peak (Lanczos basis,
    // H_eff scratch, the precision form's tensor-core operands) and the gauge
    // moves' QR plans, with a 25% margin.
    static uint64_t footprint_bytes(const std::vector<int>& d, const std::vector<int>& cl, const std::vector<int>& cr,
                                    int bandwidth, int levels, int krylov, int precision) {
        const int n = (int)d.size();
        const int b = std::min(bandwidth, maximum_bandwidth_dimension(d));
        const std::vector<int> bonds = bandwidth_sequence(std::max(1, b), d);
        double elems = 0, maxs = 1, maxenv = 1;
        for (int i = 0; i < n; ++i) {
            const double site = (double)bonds[i] * bonds[i + 1] * d[i];
            maxs = std::max(maxs, site);
            const double env = (double)bonds[i] * bonds[i] * cl[i] + (double)bonds[i + 1] * bonds[i + 1] * cr[i];
            maxenv = std::max(maxenv, env);
            elems += env;
        }
        elems += (n + 2) * maxs;                                   // sites and spares
        const int np = std::max(0, levels - 1);
        for (int i = 0; i < n; ++i)                                // projector sites and overlap environments
            elems += np * (3.0 * bonds[i] * bonds[i + 1] * d[i] + (double)bonds[i] * bonds[i] +
                           (double)bonds[i + 1] * bonds[i + 1]);
        elems += (krylov + 1 + std::max(4, krylov / 3) + 4) * maxs;   // Lanczos basis, restart vectors
        elems += 2.0 * maxs * 8 + maxenv;                         // H_eff / environment-update scratch
        double qr = 0;
        for (int i = 0; i + 1 < n; ++i) {                          // largest gauge QR plan (m x n, Q accumulated m x m)
            const double m = (double)bonds[i] * d[i], k = bonds[i + 1];
            qr = std::max(qr, 4.0 * m * k + m * m + 2.0 * k * k);
        }
        elems += 2 * qr;
        if (precision) elems += 3.0 * maxenv + 4.0 * maxs;       // TF32 pairs of environments and sites (float = elems/4)
        return (uint64_t)(1.25 * elems * sizeof(cplx)) + (64ull << 20);
    }
};

}  // namespace nc

// ---------------------------------------------------------------------------
// extern "C" (Level 1)
// ---------------------------------------------------------------------------
using namespace nc;

struct nc_chain {
    std::unique_ptr<Chain> impl;
};

namespace {
ChainOptions to_options(const nc_chain_options* o) {
    ChainOptions c;
    if (!o) return c;
    c.maximum_number_of_iterations = o->maximum_number_of_iterations;
    c.sanity_check_threshold = o->sanity_check_threshold;
    c.site_convergence_threshold = o->site_convergence_threshold;
    c.sweep_convergence_threshold = o->sweep_convergence_threshold;
    c.chain_convergence_threshold = o->chain_convergence_threshold;
    c.initial_bandwidth_dimension = o->initial_bandwidth_dimension;
    c.bandwidth_increment = o->bandwidth_increment ? o->bandwidth_increment : 1;
    const char* m = o->optimizer_mode;
    if (m[0] == '<' && m[1] == 'v') c.mode = WHICH_SR;
    else if (m[0] == '>' && m[1] == 'v') c.mode = WHICH_LR;
    else if (m[0] == '>' && m[1] == 'm') c.mode = WHICH_LM;
    else throw Error(NC_ERR_ARG, "optimizer mode must be one of <v, >v, >m");
    c.krylov_dim = o->krylov_dimension ? (int)o->krylov_dimension : 24;
    c.seed = o->seed;
    c.strict = o->strict != 0;
    c.time_phases = o->time_phases != 0;
    c.precision = (int)o->precision;
    c.maximum_sweeps = o->maximum_sweeps;
    return c;
}
}  // namespace

extern "C" {

void nc_chain_options_init(nc_chain_options* o) {
    // chain_options.cpp:21-30
    std::memset(o, 0, sizeof(*o));
    o->maximum_number_of_iterations = 10000;
    o->sanity_check_threshold = 1e-12;
    o->site_convergence_threshold = 1e-12;
    o->sweep_convergence_threshold = 1e-12;
    o->chain_convergence_threshold = 1e-12;
    o->initial_bandwidth_dimension = 1;
    o->bandwidth_increment = 1;
    o->optimizer_mode[0] = '<';
    o->optimizer_mode[1] = 'v';
    o->krylov_dimension = 24;
    o->seed = 1;
    o->strict = 0;
}

nc_chain* nc_chain_create(uint32_t number_of_sites, const nc_operator_site* sites, const nc_chain_options* options) {
    NC_ABI_BEGIN
    std::vector<OperatorSiteDesc> d(number_of_sites);
    for (uint32_t i = 0; i < number_of_sites; ++i) {
        d[i].d = sites[i].physical_dimension;
        d[i].cl = sites[i].left_dimension;
        d[i].cr = sites[i].right_dimension;
        d[i].nnz = sites[i].number_of_matrices;
        d[i].idx = sites[i].indices;
        d[i].W = reinterpret_cast<const cplx*>(sites[i].matrices);
    }
    auto h = new nc_chain;
    try {
        h->impl = std::make_unique<Chain>(Context::get(), (int)number_of_sites, d.data(), to_options(options));
        h->impl->handle = h;
    } catch (...) {
        delete h;
        throw;
    }
    return h;
    NC_ABI_END
    return nullptr;
}

void nc_chain_free(nc_chain* c) { delete c; }

#define NC_CHAIN_CALL(body)          \
    NC_ABI_BEGIN                     \
    NC_ARG(c && c->impl, "null chain"); \
    Chain& ch = *c->impl;            \
    (void)ch;                        \
    body;                            \
    NC_ABI_END                       \
    return g_status;

int nc_chain_reset(nc_chain* c) { NC_CHAIN_CALL(ch.reset()) }

int64_t nc_chain_connect(nc_chain* c, int signal, nc_chain_signal_fn fn, void* user) {
    NC_ABI_BEGIN
    NC_ARG(c && c->impl, "null chain");
    NC_ARG(fn != nullptr, "null callback");
    NC_ARG(signal >= NC_SIGNAL_OPTIMIZE_SITE_SUCCESS && signal <= NC_SIGNAL_CHAIN_RESET, "unknown signal");
    Chain& ch = *c->impl;
    const int64_t id = ch.next_slot++;
    ch.slots.push_back(Chain::Slot{id, signal, fn, user});
    return id;
    NC_ABI_END
    return -1;
}

int nc_chain_disconnect(nc_chain* c, int64_t id) {
    NC_CHAIN_CALL({
        auto it = std::find_if(ch.slots.begin(), ch.slots.end(), [&](const Chain::Slot& s) { return s.id == id; });
        NC_ARG(it != ch.slots.end(), "no such connection");
        ch.slots.erase(it);
    })
}

int nc_chain_set_state(nc_chain* c, const uint32_t* bond_dimensions, const nc_complex* const* sites) {
    NC_CHAIN_CALL({
        std::vector<int> b(ch.N + 1);
        for (int i = 0; i <= ch.N; ++i) b[i] = (int)bond_dimensions[i];
        NC_ARG(b[0] == 1 && b[ch.N] == 1, "boundary bond dimensions must be 1");
        std::vector<const cplx*> s(ch.N);
        for (int i = 0; i < ch.N; ++i) s[i] = reinterpret_cast<const cplx*>(sites[i]);
        ch.reset(&b, &s);
    })
}

int nc_chain_perform_optimization_sweep(nc_chain* c) { NC_CHAIN_CALL(ch.perform_optimization_sweep()) }
int nc_chain_sweep_until_converged(nc_chain* c) { NC_CHAIN_CALL(ch.sweep_until_converged()) }
int nc_chain_optimize_chain(nc_chain* c) { NC_CHAIN_CALL(ch.optimize_chain()) }
int nc_chain_optimize_site(nc_chain* c) { NC_CHAIN_CALL(ch.optimize_site()) }
int nc_chain_move_to(nc_chain* c, uint32_t s) {
    NC_CHAIN_CALL({
        NC_ARG((int)s < ch.N, "site out of range");
        ch.move_to((int)s);
    })
}
int nc_chain_increase_bandwidth_dimension(nc_chain* c, uint32_t b) { NC_CHAIN_CALL(ch.increase_bandwidth_dimension((int)b)) }
int nc_chain_construct_and_add_projector_from_state(nc_chain* c) {
    NC_CHAIN_CALL(ch.construct_and_add_projector_from_state())
}
int nc_chain_solve_for_eigenvalues(nc_chain* c, uint32_t n, double* eigenvalues) {
    NC_CHAIN_CALL({
        NC_ARG(n >= 1, "need at least one level");
        ch.solve_for_multiple_levels((int)n, eigenvalues);
    })
}
int nc_chain_get_energy(nc_chain* c, double* energy) { NC_CHAIN_CALL(*energy = ch.energy) }
int nc_chain_solve_levels_at_bandwidth(nc_chain* c, uint32_t n, double* energies) {
    NC_CHAIN_CALL({
        NC_ARG(n >= 1, "need at least one level");
        ch.solve_levels_at_bandwidth((int)n, energies);
    })
}

int nc_chain_footprint_bytes(uint32_t number_of_sites, const nc_operator_site* sites, const nc_chain_options* options,
                             uint32_t levels, uint64_t* bytes) {
    NC_ABI_BEGIN
    NC_ARG(number_of_sites >= 1 && sites && bytes, "bad arguments");
    std::vector<int> d(number_of_sites), cl(number_of_sites), cr(number_of_sites);
    for (uint32_t i = 0; i < number_of_sites; ++i) {
        d[i] = (int)sites[i].physical_dimension;
        cl[i] = (int)sites[i].left_dimension;
        cr[i] = (int)sites[i].right_dimension;
        NC_ARG(d[i] >= 1 && cl[i] >= 1 && cr[i] >= 1, "bad operator site");
    }
    const ChainOptions o = to_options(options);
    *bytes = Chain::footprint_bytes(d, cl, cr, (int)std::max<uint32_t>(1, o.initial_bandwidth_dimension),
                                    (int)std::max<uint32_t>(1, levels), o.krylov_dim, o.precision);
    NC_ABI_END
    return g_status;
}
int nc_chain_set_precision(nc_chain* c, uint32_t precision) {
    NC_CHAIN_CALL({
        NC_ARG(precision <= 1, "precision must be 0 (FP64) or 1 (mixed)");
        const int was = ch.prec;
        ch.prec = (int)precision;
        if (was == 1 && ch.prec == 0) ch.refresh_environments();
    })
}
int nc_chain_compute_expectation_value(nc_chain* c, double* value) { NC_CHAIN_CALL(*value = ch.expectation_value()) }

int nc_chain_get_info(nc_chain* c, nc_chain_info* info) {
    NC_CHAIN_CALL({
        info->number_of_sites = (uint32_t)ch.N;
        info->current_site = (uint32_t)ch.cur;
        info->bandwidth_dimension = (uint32_t)ch.bandwidth;
        info->maximum_bandwidth_dimension = (uint32_t)ch.max_bandwidth;
        info->number_of_projectors = (uint32_t)ch.projectors.size();
        info->sweeps = ch.stats.sweeps;
        info->site_solves = ch.stats.site_solves;
        info->matvecs = ch.stats.matvecs;
        info->moves = ch.stats.moves;
        info->failures = ch.stats.failures;
        info->last_failure = ch.stats.last_failure;
        info->energy = ch.energy;
        info->seconds_solve = ch.stats.t_solve;
        info->seconds_gauge = ch.stats.t_gauge;
        info->seconds_environment = ch.stats.t_env;
        info->seconds_projector = ch.stats.t_proj;
        info->mixed_sweeps = ch.stats.mixed_sweeps;
        info->precision = (uint32_t)ch.prec;
    })
}

int nc_chain_get_site(nc_chain* c, uint32_t i, nc_complex* out, uint32_t* dims) {
    NC_CHAIN_CALL({
        NC_ARG((int)i < ch.N, "site out of range");
        dims[0] = (uint32_t)ch.br(i); dims[1] = (uint32_t)ch.bl(i); dims[2] = (uint32_t)ch.phys[i];
        if (out) {
            NC_CUDA(cudaMemcpyAsync(out, ch.site[i].p, ch.site_elems(i) * sizeof(cplx), cudaMemcpyDeviceToHost,
                                    ch.ctx.stream));
            NC_CUDA(cudaStreamSynchronize(ch.ctx.stream));
        }
    })
}

}  // extern "C"
