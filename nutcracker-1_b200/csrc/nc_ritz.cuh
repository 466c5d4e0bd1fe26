// Projected (Rayleigh-Ritz) problem of the restarted Lanczos solvers, shared
// by the single-chain solver (lanczos.cu) and the batched one (batched.cu).
//
// T = V^H H V grows by one column per Lanczos step (real symmetric: a
// tridiagonal block plus, after a thick restart, an arrow of couplings to the
// kept Ritz vectors; both come out of the reorthogonalisation coefficients,
// T(i, m-1) = Re(h1_i + h2_i)).  Its eigen-decomposition T = Z Theta Z^T is
// kept between steps (the rotated matrix A ~ Theta and the accumulated
// rotations Z, row-major [row][col], MAXT x MAXT each): a new column t is
// taken into the current eigenbasis (z = Z^T t), which leaves a diagonal
// matrix bordered by one row and column, and one warp finishes it with
// cyclic Jacobi (round-robin pairing, which keeps clustered Ritz values such
// as near-degenerate doublets orthogonal).  Started from an almost diagonal
// matrix, Jacobi needs a few sweeps instead of the 6-10 of a cold start; a
// rotation is skipped when its off-diagonal element is below the rounding
// level of its diagonal pair, and the sweeps stop when a whole sweep skips
// every rotation.
#pragma once

#include "nc_common.cuh"

namespace nc {

enum RitzWhich { RITZ_SR = 0, RITZ_LR = 1, RITZ_LM = 2 };

struct RitzResult {
    double theta, res, beta, tnorm;
    int sweeps;
};

// Shared-memory work area of one warp's update.
template <int MAXT>
struct RitzSmem {
    double A[MAXT][MAXT + 1], Z[MAXT][MAXT + 1];
    double tcol[MAXT];
    double cs[MAXT / 2], sn[MAXT / 2];
    int pa[MAXT / 2], pb[MAXT / 2];
    int perm[MAXT];
    int rotated;
};

// After a thick restart: A = diag(theta_0 .. theta_{k-1}), Z = I.  Any
// number of threads of one block.
template <int MAXT>
__device__ __forceinline__ void ritz_restart_state(int k, const double* theta, double* state) {
    double* A = state;
    double* Z = state + MAXT * MAXT;
    for (int e = threadIdx.x; e < MAXT * MAXT; e += blockDim.x) {
        const int r = e / MAXT, c = e % MAXT;
        A[e] = (r == c && r < k) ? theta[r] : 0.0;
        Z[e] = (r == c) ? 1.0 : 0.0;
    }
}

// One warp (lanes 0..31, MAXT <= 32): adds column m-1 of T (tcol(i) =
// Re(h1_i + h2_i), i < m) to the kept decomposition of the leading
// (m-1) x (m-1) block in `state` and diagonalises.  The Ritz values, ordered
// by `which` (SR ascending, LR descending, LM by decreasing magnitude), go to
// theta[], the matching eigenvectors of T to S (column r at S[ldS * r], m
// entries; complex with zero imaginary part when S_complex, else real).  The
// wanted pair's value and Ritz estimate beta |z_{m-1,0}| (beta =
// sqrt(nrm2)) are returned to lane 0.
template <int MAXT, bool S_complex>
__device__ RitzResult ritz_update_warp(RitzSmem<MAXT>& w, int m, double* __restrict__ state,
                                       const cplx* __restrict__ h1, const cplx* __restrict__ h2, double nrm2,
                                       int which, void* __restrict__ S_out, int ldS, double* __restrict__ theta) {
    const int lane = threadIdx.x & 31;
    const int mp = m + (m & 1);
    const double* gA = state;
    const double* gZ = state + MAXT * MAXT;
    // load the kept (m-1) x (m-1) decomposition, pad to mp
    for (int r = 0; r < mp; ++r) {
        if (lane < MAXT) {
            const bool in = lane < m - 1 && r < m - 1;
            w.A[r][lane] = in ? gA[r * MAXT + lane] : 0.0;
            w.Z[r][lane] = in ? gZ[r * MAXT + lane] : (r == lane ? 1.0 : 0.0);
        }
    }
    if (lane < m) w.tcol[lane] = h1[lane].x + h2[lane].x;
    __syncwarp();
    // border: z = Z^T t over the old rows, diagonal t_{m-1}
    if (lane < m - 1) {
        double z = 0.0;
        for (int i = 0; i < m - 1; ++i) z += w.Z[i][lane] * w.tcol[i];
        w.A[lane][m - 1] = z;
        w.A[m - 1][lane] = z;
    }
    if (lane == 0) w.A[m - 1][m - 1] = w.tcol[m - 1];
    __syncwarp();
    int sweep = 0;
    for (; sweep < 30; ++sweep) {
        if (lane == 0) w.rotated = 0;
        __syncwarp();
        for (int s = 0; s < mp - 1; ++s) {
            if (lane < mp / 2) {
                int a, b;
                if (lane == 0) { a = mp - 1; b = s % (mp - 1); }
                else { a = (s + lane) % (mp - 1); b = (s - lane + mp - 1) % (mp - 1); }
                const double apq = w.A[a][b], app = w.A[a][a], aqq = w.A[b][b];
                double c = 1.0, sv = 0.0;
                const double small = 1.1102230246251565e-16 * sqrt(fabs(app) * fabs(aqq));
                if (fabs(apq) > small && fabs(apq) > 1e-300) {
                    const double tau = (aqq - app) / (2.0 * apq);
                    const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                    c = 1.0 / sqrt(1.0 + t * t);
                    sv = t * c;
                    w.rotated = 1;
                }
                w.pa[lane] = a; w.pb[lane] = b; w.cs[lane] = c; w.sn[lane] = sv;
            }
            __syncwarp();
            if (lane < mp) {
                for (int r = 0; r < mp / 2; ++r) {   // rows a, b of A
                    const double sv = w.sn[r];
                    if (sv == 0.0) continue;
                    const int a = w.pa[r], b = w.pb[r];
                    const double c = w.cs[r];
                    const double xa = w.A[a][lane], xb = w.A[b][lane];
                    w.A[a][lane] = c * xa - sv * xb;
                    w.A[b][lane] = sv * xa + c * xb;
                }
            }
            __syncwarp();
            if (lane < mp) {
                for (int r = 0; r < mp / 2; ++r) {   // columns a, b of A and Z
                    const double sv = w.sn[r];
                    if (sv == 0.0) continue;
                    const int a = w.pa[r], b = w.pb[r];
                    const double c = w.cs[r];
                    const double xa = w.A[lane][a], xb = w.A[lane][b];
                    w.A[lane][a] = c * xa - sv * xb;
                    w.A[lane][b] = sv * xa + c * xb;
                    const double va = w.Z[lane][a], vb = w.Z[lane][b];
                    w.Z[lane][a] = c * va - sv * vb;
                    w.Z[lane][b] = sv * va + c * vb;
                }
            }
            __syncwarp();
        }
        if (!w.rotated) break;
    }
    // keep the decomposition of the m x m block for the next step
    double* wA = state;
    double* wZ = state + MAXT * MAXT;
    for (int r = 0; r < m; ++r) {
        if (lane < m) {
            wA[r * MAXT + lane] = w.A[r][lane];
            wZ[r * MAXT + lane] = w.Z[r][lane];
        }
    }
    RitzResult out{};
    if (lane == 0) {
        // order the m genuine Ritz values (a padding direction, if any, is index m)
        for (int i = 0; i < m; ++i) w.perm[i] = i;
        for (int i = 0; i < m; ++i) {
            int best = i;
            for (int q = i + 1; q < m; ++q) {
                const double x = w.A[w.perm[q]][w.perm[q]], y = w.A[w.perm[best]][w.perm[best]];
                const bool better = (which == RITZ_SR) ? (x < y) : (which == RITZ_LR) ? (x > y) : (fabs(x) > fabs(y));
                if (better) best = q;
            }
            const int t = w.perm[i]; w.perm[i] = w.perm[best]; w.perm[best] = t;
        }
        double tn = 0;
        for (int i = 0; i < m; ++i) tn = fmax(tn, fabs(w.A[i][i]));
        const double beta = sqrt(nrm2);
        out.theta = w.A[w.perm[0]][w.perm[0]];
        out.res = beta * fabs(w.Z[m - 1][w.perm[0]]);
        out.beta = beta;
        out.tnorm = tn;
        out.sweeps = sweep;
    }
    __syncwarp();
    for (int r = 0; r < m; ++r) {
        const int p = w.perm[r];
        if (lane < m) {
            if (S_complex) reinterpret_cast<cplx*>(S_out)[lane + (size_t)ldS * r] = cmake(w.Z[lane][p], 0.0);
            else reinterpret_cast<double*>(S_out)[lane + (size_t)ldS * r] = w.Z[lane][p];
        }
        if (lane == 0) theta[r] = w.A[p][p];
    }
    return out;
}

}  // namespace nc
