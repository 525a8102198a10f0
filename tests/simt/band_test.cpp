// Driver for tests/test_band_kernel_cpu.py: builds random SPD block-band
// matrices in the band kernel's input layout (block A(i, i - d) row-major at
// i * BAND_W + d), splits each component between the two CTAs of a cluster
// the way the solver does (band_split_point: bodies [0, m + wb) forward,
// [m, n) reversed), runs k_band_solve on all of them in one launch under the
// host emulation of simt.h (fewer clusters than jobs, so clusters take
// several jobs), and compares every solution with a dense Cholesky solve.
// Exit status 0 when every component is within 1e-12 relative.
#include "simt.h"
#include "band_kernel.inc"  // written by tests/test_band_kernel_cpu.py
#include <random>
// dense SPD solve by Cholesky (reference)
static std::vector<double> dense_solve(std::vector<double> A, std::vector<double> b, int n) {
    for (int j = 0; j < n; j++) {
        double d = A[j * n + j];
        for (int k = 0; k < j; k++) d -= A[j * n + k] * A[j * n + k];
        d = std::sqrt(d); A[j * n + j] = d;
        for (int i = j + 1; i < n; i++) {
            double s = A[i * n + j];
            for (int k = 0; k < j; k++) s -= A[i * n + k] * A[j * n + k];
            A[i * n + j] = s / d;
        }
    }
    for (int i = 0; i < n; i++) { double s = b[i]; for (int k = 0; k < i; k++) s -= A[i * n + k] * b[k]; b[i] = s / A[i * n + i]; }
    for (int i = n - 1; i >= 0; i--) { double s = b[i]; for (int k = i + 1; k < n; k++) s -= A[k * n + i] * b[k]; b[i] = s / A[i * n + i]; }
    return b;
}
int main(int argc, char** argv) {
    setvbuf(stdout, nullptr, _IONBF, 0);
    const int cases[][2] = {{2, 1}, {5, 4}, {9, 8}, {11, 8}, {17, 5}, {30, 8}, {40, 1}, {23, 3}, {46, 5}, {29, 8}, {13, 1}};
    const int ncase = sizeof(cases) / sizeof(cases[0]);
    std::mt19937_64 rng(7);
    std::normal_distribution<double> nd(0.0, 1.0);
    // bodies of all components in one global numbering, like the solver's
    std::vector<int> base(ncase + 1, 0);
    for (int c = 0; c < ncase; c++) base[c + 1] = base[c] + cases[c][0];
    const int nb = base[ncase];
    std::vector<std::vector<double>> Ms(ncase);
    std::vector<double> g(12 * (size_t)nb);
    for (auto& v : g) v = nd(rng);
    std::vector<int> cptr(1, 0), order, cbw, jobs;
    std::vector<long long> loff;
    long long ltot = 0;
    std::vector<std::vector<int>> sub_bodies;
    auto add_sub = [&](std::vector<int> bodies, int wb) {
        loff.push_back(ltot);
        ltot += (long long)bodies.size() * BAND_W;
        order.insert(order.end(), bodies.begin(), bodies.end());
        cptr.push_back((int)order.size());
        cbw.push_back(wb);
        sub_bodies.push_back(bodies);
        return (int)cbw.size() - 1;
    };
    int nsplit = 0;
    for (int c = 0; c < ncase; c++) {
        const int N = cases[c][0], wb = cases[c][1], n = 12 * N;
        std::vector<double>& M = Ms[c];
        M.assign((size_t)n * n, 0.0);
        for (int i = 0; i < N; i++)
            for (int j = std::max(0, i - wb); j <= i; j++)
                for (int r = 0; r < 12; r++)
                    for (int cc = 0; cc < 12; cc++) {
                        double v = 0.3 * nd(rng);
                        M[(12 * i + r) * n + 12 * j + cc] = v;
                        M[(12 * j + cc) * n + 12 * i + r] = v;
                    }
        for (int i = 0; i < n; i++) M[i * n + i] = 0.0;
        for (int i = 0; i < n; i++) { double s = 0; for (int j = 0; j < n; j++) s += std::fabs(M[i * n + j]); M[i * n + i] = s + 1.0; }
        std::vector<int> bodies(N);
        for (int i = 0; i < N; i++) bodies[i] = base[c] + i;
        const int m = band_split_point(N, wb);
        if (m > 0) {
            const int ct = add_sub(std::vector<int>(bodies.begin(), bodies.begin() + m + wb), wb);
            const int cb = add_sub(std::vector<int>(bodies.rbegin(), bodies.rend() - m), wb);
            jobs.insert(jobs.end(), {ct, cb, m});
            nsplit++;
        } else {
            const int ct = add_sub(bodies, wb);
            jobs.insert(jobs.end(), {ct, -1, N});
        }
    }
    // gather: block A(i, i - d) of each sub-component in its own order
    std::vector<double> Ab((size_t)ltot * 144, 0.0);
    for (size_t s = 0; s < sub_bodies.size(); s++) {
        const auto& bo = sub_bodies[s];
        int c = 0;
        while (base[c + 1] <= bo[0]) c++;
        const int n = 12 * cases[c][0], wb = cbw[s];
        for (int i = 0; i < (int)bo.size(); i++)
            for (int d = 0; d <= std::min(wb, i); d++) {
                const int bi = bo[i] - base[c], bj = bo[i - d] - base[c];
                for (int r = 0; r < 12; r++)
                    for (int cc = 0; cc < 12; cc++)
                        Ab[((size_t)loff[s] + (size_t)i * BAND_W + d) * 144 + r * 12 + cc] = Ms[c][(12 * bi + r) * n + 12 * bj + cc];
            }
    }
    std::vector<double> Lg((size_t)ltot * 144 + 12 * order.size(), 0.0), du(12 * (size_t)nb, 0.0);
    int status = 0;
    const size_t smem = (size_t)band_smem_doubles() * 8;
    const int njobs = (int)jobs.size() / 3, clusters = std::max(1, njobs / 3);
    launch(2 * clusters, BAND_THREADS, smem, [&] {
        k_band_solve(njobs, jobs.data(), cptr.data(), order.data(), cbw.data(), loff.data(), Ab.data(), ltot, g.data(),
                     Lg.data(), du.data(), &status);
    }, 2);
    double worst = 0;
    for (int c = 0; c < ncase; c++) {
        const int N = cases[c][0], n = 12 * N;
        std::vector<double> gc(g.begin() + 12 * base[c], g.begin() + 12 * base[c + 1]);
        auto ref = dense_solve(Ms[c], gc, n);
        double err = 0, sc = 0;
        for (int i = 0; i < n; i++) { err = std::max(err, std::fabs(du[12 * base[c] + i] - ref[i])); sc = std::max(sc, std::fabs(ref[i])); }
        printf("N %2d wb %d%s: rel err %.3e\n", N, cases[c][1], band_split_point(N, cases[c][1]) > 0 ? " (split)" : "", err / sc);
        worst = std::max(worst, err / sc);
    }
    printf("jobs %d split %d clusters %d status %d\nworst %.3e\n", njobs, nsplit, clusters, status, worst);
    return worst < 1e-12 && status == 0 ? 0 : 1;
}
