// Host build of the engine's grid searches (agama_b200/csrc/common.cuh): binSearchScaled (the
// device form: a multiplied first guess and a short walk to the neighbouring segment before the
// bisection) must return the segment of binSearch (the restatement of math::binSearch) for every
// point.  Grids: uniform, geometric, irregular (random spacing), the Multipole tau grids of lmax
// 2..16, and one- and two-node grids; points: every node, its two floating-point neighbours,
// random points over and around the grid, NaN and the infinities.  Prints "checked N mismatches M".
#include "common.cuh"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

using namespace agb;

namespace {

/// the Multipole tau grid of order lmax: Gauss-Legendre nodes of lmax+1 points in cos(theta)
/// mapped to tau = cos / (1 + sin), the end points -1 and 1, every interval cut in three
std::vector<double> tauGrid(int lmax)
{
    const int n = lmax + 1;
    std::vector<double> t(n + 2);
    for(int i = 0; i < n; i++) {     // nodes by Newton on the Legendre polynomial
        double x = std::cos(M_PI * (i + 0.75) / (n + 0.5));
        for(int it = 0; it < 100; it++) {
            double p0 = 1, p1 = x;
            for(int k = 2; k <= n; k++) { const double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
            const double dp = n * (x * p1 - p0) / (x * x - 1);
            x -= p1 / dp;
        }
        t[1 + i] = -x;
    }
    std::sort(t.begin() + 1, t.end() - 1);
    for(int i = 1; i <= n; i++) t[i] /= 1 + std::sqrt(1 - t[i] * t[i]);
    t.front() = -1;
    t.back() = 1;
    std::vector<double> g;
    for(int i = 0; i <= n; i++)
        for(int k = 0; k < 3; k++) g.push_back((t[i] * (3 - k) + t[i + 1] * k) / 3);
    g.push_back(1);
    return g;
}

}  // namespace

int main()
{
    std::mt19937_64 rng(5);
    std::uniform_real_distribution<double> U(0, 1);
    std::vector<std::vector<double>> grids;
    for(int lmax = 2; lmax <= 16; lmax++) grids.push_back(tauGrid(lmax));
    grids.push_back({ 0.5 });
    grids.push_back({ -1, 1 });
    for(int g = 0; g < 3000; g++) {
        const int n = 2 + static_cast<int>(rng() % 90);
        std::vector<double> a(n);
        double acc = -1;
        for(int i = 0; i < n; i++) {
            if(g % 3 == 0) a[i] = -1 + 2.0 * i / (n - 1);
            else if(g % 3 == 1) { acc += 0.05 + U(rng); a[i] = acc; }
            else a[i] = std::log(1e-3) + std::log(1e6) * i / (n - 1);
        }
        grids.push_back(a);
    }
    long total = 0, bad = 0;
    for(const std::vector<double>& a : grids) {
        const int n = static_cast<int>(a.size());
        const double scale = n > 1 ? (n - 1) / (a[n - 1] - a[0]) : 0;
        std::vector<double> xs = { NAN, INFINITY, -INFINITY };
        for(int i = 0; i < n; i++) {
            xs.push_back(a[i]);
            xs.push_back(std::nextafter(a[i], -INFINITY));
            xs.push_back(std::nextafter(a[i], INFINITY));
        }
        const double span = n > 1 ? a[n - 1] - a[0] : 1;
        for(int k = 0; k < 400; k++) xs.push_back(a[0] - 0.1 * span + 1.2 * span * U(rng));
        for(double x : xs) {
            total++;
            const int want = binSearch(x, a.data(), n), got = binSearchScaled(x, a.data(), n, scale);
            if(want != got) {
                if(bad < 10) std::printf("n=%d x=%.17g binSearch %d binSearchScaled %d\n", n, x, want, got);
                bad++;
            }
        }
    }
    std::printf("checked %ld mismatches %ld\n", total, bad);
    return bad != 0;
}
