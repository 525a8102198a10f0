// Driver for tests/test_band_kernel_cpu.py: builds random SPD block-band
// matrices in the band kernel's input layout (block A(i, i - d) row-major at
// i * BAND_W + d), runs k_band_solve on one component under the host
// emulation of simt.h, and compares its solution with a dense Cholesky
// solve.  Exit status 0 when every case is within 1e-12 relative.
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
    int cases[][2] = {{2, 1}, {5, 4}, {9, 8}, {11, 8}, {17, 5}, {30, 8}, {40, 1}, {23, 3}};
    std::mt19937_64 rng(7);
    std::normal_distribution<double> nd(0.0, 1.0);
    double worst = 0;
    for (auto& cs : cases) {
        int N = cs[0], wb = cs[1], n = 12 * N;
        std::vector<double> M((size_t)n * n, 0.0);
        for (int i = 0; i < N; i++)
            for (int j = std::max(0, i - wb); j <= i; j++)
                for (int r = 0; r < 12; r++)
                    for (int c = 0; c < 12; c++) {
                        double v = 0.3 * nd(rng);
                        M[(12 * i + r) * n + 12 * j + c] = v;
                        M[(12 * j + c) * n + 12 * i + r] = v;
                    }
        for (int i = 0; i < n; i++) M[i * n + i] = 0.0;
        for (int i = 0; i < n; i++) { double s = 0; for (int j = 0; j < n; j++) s += std::fabs(M[i * n + j]); M[i * n + i] = s + 1.0; }
        std::vector<double> g(n); for (auto& v : g) v = nd(rng);
        std::vector<double> Ab((size_t)N * BAND_W * 144, 0.0);
        for (int i = 0; i < N; i++)
            for (int d = 0; d <= std::min(wb, i); d++)
                for (int r = 0; r < 12; r++) for (int c = 0; c < 12; c++)
                    Ab[((size_t)i * BAND_W + d) * 144 + r * 12 + c] = M[(12 * i + r) * n + 12 * (i - d) + c];
        std::vector<int> order(N); for (int i = 0; i < N; i++) order[i] = i;
        int cptr[2] = {0, N}, cbw[1] = {wb}; long long loff[1] = {0};
        std::vector<double> Lg((size_t)N * BAND_W * 144 + 12 * N, 0.0), du(n, 0.0);
        int status = 0;
        // the kernel's shared-memory size, as the solver launches it
        size_t smem = (size_t)band_smem_doubles() * 8;
        const long long ltot = (long long)N * BAND_W;
        launch(1, BAND_THREADS, smem, [&] { k_band_solve(1, cptr, order.data(), cbw, loff, Ab.data(), ltot, g.data(), Lg.data(), du.data(), &status); });
        auto ref = dense_solve(M, g, n);
        double err = 0, sc = 0;
        for (int i = 0; i < n; i++) { err = std::max(err, std::fabs(du[i] - ref[i])); sc = std::max(sc, std::fabs(ref[i])); }
        printf("N %2d wb %d: rel err %.3e status %d\n", N, wb, err / sc, status);
        worst = std::max(worst, err / sc);
    }
    printf("worst %.3e\n", worst);
    return worst < 1e-12 ? 0 : 1;
}
