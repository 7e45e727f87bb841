// Host build of the engine's restated numerics (agama_b200/csrc/sphharm.cuh, common.cuh): the
// normalised Legendre functions with derivatives, the multiple-angle recurrence and the interval
// scalings.  Input lines (output one line each, %.17g):
//   L lmax m tau        -> P[0..lmax-m], dP[...], d2P[...]
//   T phi m needSine    -> cos(k phi) k=1..m [, sin(k phi)]
//   U kind a b s        -> u, du/ds  (kind 0: (-inf, inf); 1: [a, inf); 2: cubic stretch of [a, b])
//   S a b u             -> s of the cubic stretch of [a, b]
#include "sphharm.cuh"
#include <cstdio>

using namespace agb;

int main()
{
    char mode;
    while(std::scanf(" %c", &mode) == 1) {
        if(mode == 'L') {
            int lmax, m; double tau;
            if(std::scanf("%d %d %lf", &lmax, &m, &tau) != 3) return 2;
            double P[LMAX_MAX + 1], dP[LMAX_MAX + 1], d2P[LMAX_MAX + 1];
            legendreArray(lmax, m, tau, P, dP, d2P);
            for(int k = 0; k <= lmax - m; k++) std::printf("%.17g %.17g %.17g ", P[k], dP[k], d2P[k]);
        } else if(mode == 'T') {
            double phi; int m, ns;
            if(std::scanf("%lf %d %d", &phi, &m, &ns) != 3) return 2;
            double out[2 * LMAX_MAX];
            trigMultiAngle(phi, m, ns != 0, out);
            for(int k = 0; k < (ns ? 2 * m : m); k++) std::printf("%.17g ", out[k]);
        } else if(mode == 'U') {
            int kind; double a, b, s, duds = 0, u;
            if(std::scanf("%d %lf %lf %lf", &kind, &a, &b, &s) != 4) return 2;
            u = kind == 0 ? unscaleInf(s, &duds) : kind == 1 ? unscaleSemiInf(a, s, &duds) : unscaleCub(a, b, s, &duds);
            std::printf("%.17g %.17g ", u, duds);
        } else if(mode == 'S') {
            double a, b, u;
            if(std::scanf("%lf %lf %lf", &a, &b, &u) != 3) return 2;
            std::printf("%.17g ", scaleCub(a, b, u));
        } else
            return 2;
        std::printf("\n");
    }
    return 0;
}
