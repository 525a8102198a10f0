// Driver for tests/test_psd_project_cpu.py: runs the register-resident PSD
// projection (warp_psd_project_rows<N>, colb_b200/csrc/warp_eig.cuh) and the
// shared-memory one (team_psd_project<32>) on the same symmetric matrices
// under the host emulation of simt.h, one warp, and compares them.  The
// matrices are of the kinds the contact Hessians produce: indefinite,
// rank-deficient (a low-rank positive part minus a low-rank negative part,
// which leaves zero eigenvalues), positive definite (left unchanged), and
// zero, for n = 6, 9 and 12.  Exit status 0 when every pair agrees to 1e-12
// of the matrix scale and every result is symmetric to 1e-12 of the scale
// with no eigenvalue below -1e-12 of it (a Cholesky of the result plus that
// shift succeeds).
#include "simt.h"
#include "warp_eig.inc"  // written by tests/test_psd_project_cpu.py
#include <random>

static WarpEigSmem S1, S2;

template <int N>
static double run_case(const std::vector<double>& A, double& asym, bool& psd) {
    for (int e = 0; e < 144; e++) { S1.A[e] = 0; S2.A[e] = 0; }
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) S1.A[i * 12 + j] = S2.A[i * 12 + j] = A[i * N + j];
    launch(1, 32, 0, [&] {
        team_psd_project<32>(S1, N);
        warp_psd_project_rows<N>(S2);
    });
    double scale = 0, diff = 0;
    for (int i = 0; i < N * N; i++) scale = std::max(scale, std::fabs(A[i]));
    if (scale == 0) scale = 1;
    asym = 0;
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            diff = std::max(diff, std::fabs(S1.A[i * 12 + j] - S2.A[i * 12 + j]));
            asym = std::max(asym, std::fabs(S2.A[i * 12 + j] - S2.A[j * 12 + i]));
        }
    // positive semidefinite up to 1e-12 of the scale: Cholesky of H + shift I
    std::vector<double> L(N * N);
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) L[i * N + j] = 0.5 * (S2.A[i * 12 + j] + S2.A[j * 12 + i]) + (i == j ? 1e-12 * scale : 0.0);
    psd = true;
    for (int k = 0; k < N && psd; k++) {
        double d = L[k * N + k];
        for (int s = 0; s < k; s++) d -= L[k * N + s] * L[k * N + s];
        if (!(d > 0)) { psd = false; break; }
        d = std::sqrt(d); L[k * N + k] = d;
        for (int i = k + 1; i < N; i++) {
            double v = L[i * N + k];
            for (int s = 0; s < k; s++) v -= L[i * N + s] * L[k * N + s];
            L[i * N + k] = v / d;
        }
    }
    asym /= scale;
    return diff / scale;
}

template <int N>
static double run_kind(std::mt19937_64& rng, int kind, bool& ok) {
    std::normal_distribution<double> nd(0.0, 1.0);
    std::vector<double> A(N * N, 0.0);
    if (kind == 0) {                      // indefinite, entries of mixed size
        for (int i = 0; i < N; i++)
            for (int j = 0; j <= i; j++) A[i * N + j] = A[j * N + i] = nd(rng) * std::pow(10.0, 3 * nd(rng) / 2);
    } else if (kind == 1 || kind == 2) {  // rank-deficient: rp positive and rn negative directions
        const int rp = kind == 1 ? 3 : N - 2, rn = kind == 1 ? 2 : 1;
        for (int t = 0; t < rp + rn; t++) {
            std::vector<double> u(N);
            for (auto& x : u) x = nd(rng);
            const double w = (t < rp ? 1.0 : -1.0) * std::pow(10.0, 4 * std::fabs(nd(rng)));
            for (int i = 0; i < N; i++)
                for (int j = 0; j < N; j++) A[i * N + j] += w * u[i] * u[j];
        }
    } else if (kind == 3) {               // positive definite: returned unchanged by both
        for (int i = 0; i < N; i++)
            for (int j = 0; j <= i; j++) A[i * N + j] = A[j * N + i] = 0.1 * nd(rng);
        for (int i = 0; i < N; i++) A[i * N + i] += N;
    }                                     // kind 4: zero
    double asym; bool psd;
    const double d = run_case<N>(A, asym, psd);
    if (!(d < 1e-12) || !(asym < 1e-12) || !psd) {
        ok = false;
        printf("n %d kind %d: difference %.3e, asymmetry %.3e, psd %d\n", N, kind, d, asym, (int)psd);
    }
    return d;
}

int main() {
    setvbuf(stdout, nullptr, _IONBF, 0);
    std::mt19937_64 rng(11);
    bool ok = true;
    double worst = 0;
    for (int rep = 0; rep < 2; rep++)
        for (int kind = 0; kind < 5; kind++) {
            worst = std::max(worst, run_kind<12>(rng, kind, ok));
            worst = std::max(worst, run_kind<9>(rng, kind, ok));
            worst = std::max(worst, run_kind<6>(rng, kind, ok));
        }
    printf("cases %d worst difference %.3e of the scale: %s\n", 2 * 5 * 3, worst, ok ? "ok" : "FAILED");
    return ok ? 0 : 1;
}
