// warp_eig.cuh — one warp projects a small symmetric matrix (n <= 12) held
// in shared memory onto the PSD cone: V max(L, 0) V^T.
//
// Parallel cyclic Jacobi with round-robin ("tournament") pair ordering:
// each round rotates n/2 disjoint index pairs at once, so for a product R of
// disjoint Givens rotations every entry of R^T A R depends on at most four
// entries of A and every lane updates its share of the entries
// independently.  n - 1 rounds (n even; odd n gets a dummy index) make one
// sweep.  A rotation is skipped when |a_pq| is at rounding level against its
// diagonal pair (1e-15 of their geometric mean) or against the whole matrix
// (1e-14 of its Frobenius norm: rotations leave fill of about the rounding
// unit times the norm, so a tighter floor would never be met on the barrier
// Hessians' wide spectra, and rank-deficient Hessians drive some diagonals to
// zero); sweeps stop when none was applied, the same
// criterion the serial oracle uses.  The entry a rotation annihilates is set
// to zero (not left at rounding level), so the sweeps end once the
// off-diagonal mass has decayed.  A matrix whose Cholesky factorization
// succeeds is left as it is (it is its own projection).
#pragma once
#include "common.cuh"

struct WarpEigSmem {
    double A[144];       // matrix, row-major n x n (ld 12)
    double T[144];       // scratch
    double V[144];       // eigenvectors
    double c[6], s[6];   // rotation of each pair this round
    int partner[12];     // partner of each index this round (-1 none)
    int role[12];        // 0: index is p of its pair, 1: index is q
    int pair_of[12];
    int flag;
    double red[4];       // per-warp partial sums of a team of up to 128 threads
};

// pairs of round r in a tournament of m players (m even): player m-1 fixed,
// the others rotate
DV void tournament_pair(int m, int r, int k, int& p, int& q) {
    if (k == 0) { p = m - 1; q = r % (m - 1); }
    else {
        p = (r + k) % (m - 1);
        q = (r - k + (m - 1)) % (m - 1);
    }
    if (p > q) { int t = p; p = q; q = t; }
}

template <int NT> DV void team_sync() { if (NT > 32) __syncthreads(); else __syncwarp(); }

// Cholesky of S.A into S.T (threads own rows): true when every pivot is
// positive, i.e. S.A is positive definite and its own PSD projection.  A team
// is one warp (NT = 32) or a whole block of NT threads.
template <int NT>
DV bool team_is_pd(WarpEigSmem& S, int n) {
    const int t = threadIdx.x % NT;
    for (int e = t; e < 144; e += NT) S.T[e] = S.A[e];
    team_sync<NT>();
    bool ok = true;
    for (int k = 0; k < n; k++) {
        double d = S.T[k*12+k];                 // same value in every thread
        if (!(d > 0.0)) { ok = false; break; }
        d = sqrt(d);
        if (t > k && t < n) S.T[t*12+k] /= d;
        team_sync<NT>();
        if (t > k && t < n) {
            double lik = S.T[t*12+k];
            for (int j = k + 1; j <= t; j++) S.T[t*12+j] -= lik * S.T[j*12+k];
        }
        team_sync<NT>();
    }
    team_sync<NT>();
    return ok;
}

// Project S.A (n x n, ld 12) in place.  All NT threads of the team call it.
// A positive definite matrix is returned unchanged.
template <int NT>
DV void team_psd_project(WarpEigSmem& S, int n) {
    const int t = threadIdx.x % NT, lane = threadIdx.x & 31;
    const int m = (n & 1) ? n + 1 : n;      // players, index n is a dummy when n is odd
    for (int e = t; e < 144; e += NT) { int i = e / 12, j = e % 12; S.V[e] = (i == j) ? 1.0 : 0.0; }
    // scale for the all-zero test and the rotation floor
    double fro = 0;
    for (int e = t; e < n * n; e += NT) { int i = e / n, j = e % n; fro += S.A[i*12+j] * S.A[i*12+j]; }
    for (int o = 16; o > 0; o >>= 1) fro += __shfl_xor_sync(0xffffffffu, fro, o);
    if (NT > 32) {
        if (lane == 0) S.red[t >> 5] = fro;
        team_sync<NT>();
        fro = 0;
        for (int w = 0; w < NT / 32; w++) fro += S.red[w];
    }
    if (fro == 0.0) return;
    team_sync<NT>();
    if (team_is_pd<NT>(S, n)) return;
    for (int sweep = 0; sweep < 50; sweep++) {
        if (t == 0) S.flag = 0;
        team_sync<NT>();
        for (int r = 0; r < m - 1; r++) {
            // rotation angles of this round's pairs
            if (t < m / 2) {
                int p, q; tournament_pair(m, r, t, p, q);
                double c = 1.0, s = 0.0;
                if (q < n) {
                    double apq = S.A[p*12+q], app = S.A[p*12+p], aqq = S.A[q*12+q];
                    if (fabs(apq) > fmax(1e-15 * sqrt(fabs(app * aqq)), 1e-14 * sqrt(fro))) {
                        double theta = (aqq - app) / (2 * apq);
                        double tt = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
                        c = rsqrt(tt * tt + 1); s = tt * c;
                        S.flag = 1;
                    }
                    S.partner[p] = q; S.partner[q] = p; S.role[p] = 0; S.role[q] = 1;
                    S.pair_of[p] = t; S.pair_of[q] = t;
                } else if (p < n) {
                    S.partner[p] = -1;
                }
                S.c[t] = c; S.s[t] = s;
            }
            team_sync<NT>();
            // column j of R: R[j][j] = c, R[partner][j] = -s if j is p, +s if j is q.
            // pass 1: T = R^T A R; every entry reads at most four entries of A
            for (int e = t; e < n * n; e += NT) {
                int i = e / n, j = e % n;
                int pi = S.partner[i], pj = S.partner[j];
                double ci = 1, si = 0, cj = 1, sj = 0;
                if (pi >= 0) { ci = S.c[S.pair_of[i]]; si = S.role[i] == 0 ? -S.s[S.pair_of[i]] : S.s[S.pair_of[i]]; }
                if (pj >= 0) { cj = S.c[S.pair_of[j]]; sj = S.role[j] == 0 ? -S.s[S.pair_of[j]] : S.s[S.pair_of[j]]; }
                double v = ci * cj * S.A[i*12+j];
                if (pj >= 0) v += ci * sj * S.A[i*12+pj];
                if (pi >= 0) v += si * cj * S.A[pi*12+j];
                if (pi >= 0 && pj >= 0) v += si * sj * S.A[pi*12+pj];
                // the entry of a rotated pair is annihilated
                if (pj == i && S.s[S.pair_of[i]] != 0.0) v = 0.0;
                S.T[i*12+j] = v;
            }
            team_sync<NT>();
            // pass 2: V R into A (free now that T holds the rotated matrix)
            for (int e = t; e < n * n; e += NT) {
                int i = e / n, j = e % n;
                int pj = S.partner[j];
                double cj = 1, sj = 0;
                if (pj >= 0) { cj = S.c[S.pair_of[j]]; sj = S.role[j] == 0 ? -S.s[S.pair_of[j]] : S.s[S.pair_of[j]]; }
                double w = cj * S.V[i*12+j];
                if (pj >= 0) w += sj * S.V[i*12+pj];
                S.A[i*12+j] = w;
            }
            team_sync<NT>();
            // pass 3: swap back
            for (int e = t; e < n * n; e += NT) {
                int i = e / n, j = e % n;
                double a = S.T[i*12+j], v = S.A[i*12+j];
                S.V[i*12+j] = v;
                S.A[i*12+j] = a;
            }
            team_sync<NT>();
            if (t < 12) { S.partner[t] = -1; }
            team_sync<NT>();
        }
        if (!S.flag) break;
        team_sync<NT>();
    }
    team_sync<NT>();
    // H = V max(L,0) V^T into T, then back into A
    for (int e = t; e < n * n; e += NT) {
        int i = e / n, j = e % n;
        double acc = 0;
        for (int k = 0; k < n; k++) { double l = S.A[k*12+k]; if (l > 0) acc += S.V[i*12+k] * l * S.V[j*12+k]; }
        S.T[i*12+j] = acc;
    }
    team_sync<NT>();
    for (int e = t; e < n * n; e += NT) { int i = e / n, j = e % n; S.A[i*12+j] = S.T[i*12+j]; }
    team_sync<NT>();
}

DV bool warp_is_pd(WarpEigSmem& S, int n) { return team_is_pd<32>(S, n); }
DV void warp_psd_project(WarpEigSmem& S, int n) { team_psd_project<32>(S, n); }

// ---------------------------------------------------------------------------
// Register-resident projection by one warp for n = N (6, 9 or 12).  Lane x
// holds row x of A and row x of V in registers (M = N rounded up to even;
// an odd N gets a zero row and column, which no rotation touches).  Every
// round rotates the fixed pairs (0, 1), (2, 3), ... and then moves the
// indices one step of the round-robin "circle": index 0 stays, the others
// advance along 2 -> 4 -> ... -> M-2 -> M-1 -> M-3 -> ... -> 1 -> 2, the
// same permutation in every round, so M - 1 rounds pair every two indices
// once and bring them back to their places (one sweep).  The pairing and the
// permutation being the same in every round, every register index is a
// constant without unrolling the rounds: the column rotations and the column
// permutation are moves within a lane, the row rotation is a shuffle with
// lane x ^ 1 and the row permutation one more shuffle, and the whole round
// stays a short loop body that the instruction cache holds.  The skip
// thresholds, the annihilated entry, the stopping rule, the
// positive-definite early exit and the reconstruction V max(L, 0) V^T are
// those of team_psd_project; the rotation annihilates a_pq as there, with
// its tangent t = sgn(d) e / (|d| + sqrt(d^2 + e^2)) (d = a_qq - a_pp,
// e = 2 a_pq) taken through three double-precision reciprocal square roots.
template <int N>
DV bool warp_rows_pd(const double (&a)[N]) {
    const int lane = threadIdx.x & 31;
    double l[N];
#pragma unroll
    for (int c = 0; c < N; c++) l[c] = a[c];
#pragma unroll
    for (int k = 0; k < N; k++) {
        const double d = __shfl_sync(0xffffffffu, l[k], k);     // pivot, the same in every lane
        if (!(d > 0.0)) return false;
        const double sd = sqrt(d);
        const double lik = l[k] / sd;                           // L[lane][k] for lanes > k
        if (lane > k) l[k] = lik;
#pragma unroll
        for (int j = k + 1; j < N; j++) {
            const double ljk = __shfl_sync(0xffffffffu, lik, j);
            if (lane > k && j <= lane) l[j] -= lik * ljk;
        }
    }
    return true;
}

// index whose entry moves to position y in one step of the circle (M even)
HD constexpr int circle_from(int M, int y) {
    return y == 0 ? 0 : y == 2 ? 1 : y == M - 1 ? M - 2 : (y & 1) ? y + 2 : y - 2;
}

template <int N>
DV void warp_psd_project_rows(WarpEigSmem& S) {
    constexpr int M = (N & 1) ? N + 1 : N;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    double a[M], v[M];
#pragma unroll
    for (int c = 0; c < M; c++) {
        a[c] = (lane < N && c < N) ? S.A[lane * 12 + c] : 0.0;
        v[c] = (c == lane) ? 1.0 : 0.0;
    }
    double fro = 0.0;
#pragma unroll
    for (int c = 0; c < M; c++) fro += a[c] * a[c];
    for (int o = 16; o > 0; o >>= 1) fro += __shfl_xor_sync(full, fro, o);
    if (fro == 0.0) return;
    {
        double an[N];
#pragma unroll
        for (int c = 0; c < N; c++) an[c] = a[c];
        if (warp_rows_pd<N>(an)) return;
    }
    const double floor2 = 1e-28 * fro;          // (1e-14 of the Frobenius norm)^2
    const int partner = lane < M ? (lane ^ 1) : lane;
    const int from = lane < M ? circle_from(M, lane) : lane;
    for (int sweep = 0; sweep < 50; sweep++) {
        bool rotated = false;
#pragma unroll 1
        for (int r = 0; r < M - 1; r++) {
            double aii = 0.0, aip = 0.0;
#pragma unroll
            for (int c = 0; c < M; c++) { if (c == lane) aii = a[c]; if (c == partner) aip = a[c]; }
            const double aqq = __shfl_sync(full, aii, partner);
            // the even lane of a pair computes its rotation
            double cs = 1.0, sn = 0.0;
            if (!(lane & 1) && lane < M && aip * aip > fmax(1e-30 * fabs(aii * aqq), floor2)) {
                const double d = aqq - aii, e = 2.0 * aip;
                const double h2 = fma(d, d, e * e);
                const double q = fabs(d) + h2 * rsqrt(h2);
                const double t = (d >= 0.0 ? e : -e) * rsqrt(q * q);
                cs = rsqrt(fma(t, t, 1.0)); sn = t * cs;
            }
            rotated |= sn != 0.0;
            // A R and V R: column 2k -> c col_2k - s col_2k+1, column 2k+1 -> s col_2k + c col_2k+1
#pragma unroll
            for (int k = 0; k < M / 2; k++) {
                const double ck = __shfl_sync(full, cs, 2 * k), sk = __shfl_sync(full, sn, 2 * k);
                const double ap = a[2 * k], aq = a[2 * k + 1], vp = v[2 * k], vq = v[2 * k + 1];
                a[2 * k] = ck * ap - sk * aq; a[2 * k + 1] = sk * ap + ck * aq;
                v[2 * k] = ck * vp - sk * vq; v[2 * k + 1] = sk * vp + ck * vq;
            }
            // R^T (A R): the even row of a pair -> c row_p - s row_q, the odd one -> s row_p + c row_q
            const double cm = __shfl_sync(full, cs, lane & ~1), sm = __shfl_sync(full, sn, lane & ~1);
            const bool even = !(lane & 1);
#pragma unroll
            for (int c = 0; c < M; c++) {
                const double o = __shfl_sync(full, a[c], partner);
                a[c] = even ? cm * a[c] - sm * o : sm * o + cm * a[c];
            }
            // the entry the rotation annihilates is zero, not rounding residue
            if (sm != 0.0) {
#pragma unroll
                for (int c = 0; c < M; c++) if (c == partner) a[c] = 0.0;
            }
            // one step of the circle: rows by shuffle, columns (of A and V) by moves
#pragma unroll
            for (int c = 0; c < M; c++) a[c] = __shfl_sync(full, a[c], from);
            double na[M], nv[M];
#pragma unroll
            for (int y = 0; y < M; y++) { na[y] = a[circle_from(M, y)]; nv[y] = v[circle_from(M, y)]; }
#pragma unroll
            for (int y = 0; y < M; y++) { a[y] = na[y]; v[y] = nv[y]; }
        }
        if (!__any_sync(full, rotated)) break;
    }
    // H = V max(L, 0) V^T: rows of V and the clamped eigenvalues through shared memory
    double lam = 0.0;
#pragma unroll
    for (int c = 0; c < M; c++) if (c == lane) lam = a[c];
    if (lane < M) {
#pragma unroll
        for (int c = 0; c < M; c++) S.V[lane * 12 + c] = v[c];
        S.T[lane] = lam > 0 ? lam : 0.0;
    }
    __syncwarp();
    if (lane < N) {
#pragma unroll
        for (int j = 0; j < N; j++) {
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < M; k++) acc += v[k] * S.T[k] * S.V[j * 12 + k];
            S.A[lane * 12 + j] = acc;
        }
    }
    __syncwarp();
}

// All NT threads of a team call it: for n = 6, 9 or 12 the team's first warp
// projects in registers while the others wait; other sizes take the
// shared-memory team version.
template <int NT>
DV void team_psd_project_fast(WarpEigSmem& S, int n) {
    if (n == 12 || n == 9 || n == 6) {
        if ((int)(threadIdx.x % NT) < 32) {
            if (n == 12) warp_psd_project_rows<12>(S);
            else if (n == 9) warp_psd_project_rows<9>(S);
            else warp_psd_project_rows<6>(S);
        }
        team_sync<NT>();
    } else {
        team_psd_project<NT>(S, n);
    }
}
