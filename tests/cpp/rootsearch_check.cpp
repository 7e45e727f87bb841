// The engine's root finders compiled for the host (agama_b200/csrc/common.cuh): the function
// form findRoot (used by the radius routines and the shell-orbit search) and the resumable
// RootSearch state machine (used by the action kernels), plain and seeded with a guess.
// Input lines: n c[0..n-1] lo hi reltol guess; output per line: findRoot, RootSearch (plain),
// RootSearch (seeded with guess; the plain result when the guess is refused), as %.17g.
#include "common.cuh"
#include <cstdio>
#include <vector>

using namespace agb;

struct Poly {
    static constexpr bool hasDeriv = true;
    const double* c;
    int n;
    void operator()(double x, double* val, double* der) const {
        double v = 0, d = 0;
        for(int k = n - 1; k >= 0; k--) { d = d * x + v; v = v * x + c[k]; }
        if(val) *val = v;
        if(der) *der = d;
    }
};

static double runSearch(const Poly& f, double lo, double hi, double reltol, const double* guess)
{
    RootSearch s;
    double x = s.start(lo, hi, reltol), v, d;
    while(true) {
        f(x, &v, &d);
        if(s.feed(v, d, &x)) return s.result;
        if(guess && s.phase == 2 && s.iter == 0) {
            s.seed(*guess, &x);
            guess = nullptr;
        }
    }
}

int main()
{
    int n;
    while(std::scanf("%d", &n) == 1) {
        std::vector<double> c(n);
        bool ok = true;
        for(int k = 0; k < n; k++) ok &= std::scanf("%lf", &c[k]) == 1;
        double lo, hi, reltol, guess;
        ok &= std::scanf("%lf %lf %lf %lf", &lo, &hi, &reltol, &guess) == 4;
        if(!ok) { std::fprintf(stderr, "rootsearch_check: malformed input\n"); return 2; }
        const Poly f{ c.data(), n };
        std::printf("%.17g %.17g %.17g\n", findRoot(f, lo, hi, reltol), runSearch(f, lo, hi, reltol, nullptr),
                    runSearch(f, lo, hi, reltol, &guess));
    }
    return 0;
}
