// Drives the C++ mirror of the reference API (include/agama_b200.hpp) the way a reference C++
// caller would: reads points from text files, writes the engine's results as text.
//   cpp_api_check <coef file> <points n x 3> <phase-space points n x 6> <out prefix>
// Writes <prefix>_pot.txt (Phi, dPhi/dx, dPhi/dy, dPhi/dz per point), <prefix>_act.txt
// (Jr, Jz, Jphi per point through ActionFinderAxisymFudge::evalmany; the first point also through
// actions() on cylindrical input, printed to stderr) and
// <prefix>_orb.txt (final point after T = 1 of each phase-space point, Omega = 0) and
// <prefix>_traj.txt (time and point of 11 samples of the first orbit over T = 1).
// Exit status 3 when the engine refuses to run (no CUDA device), with the message on stderr.
#include "agama_b200.hpp"
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <vector>

using namespace agama_b200;

static std::vector<double> readAll(const char* file)
{
    std::ifstream f(file);
    std::vector<double> v;
    double x;
    while(f >> x) v.push_back(x);
    return v;
}

int main(int argc, char** argv)
{
    if(argc != 5) { std::cerr << "usage: cpp_api_check coef pos3 posvel6 outprefix\n"; return 2; }
    try {
        potential::PtrPotential pot(new potential::Multipole(argv[1]));
        const std::vector<double> p3 = readAll(argv[2]), p6 = readAll(argv[3]);
        const std::string prefix = argv[4];
        FILE* f = std::fopen((prefix + "_pot.txt").c_str(), "w");
        for(size_t i = 0; i + 2 < p3.size(); i += 3) {
            double phi;
            coord::GradCar g;
            pot->eval(coord::PosCar(p3[i], p3[i + 1], p3[i + 2]), &phi, &g);
            std::fprintf(f, "%.17g %.17g %.17g %.17g\n", phi, g.dx, g.dy, g.dz);
        }
        std::fclose(f);
        actions::ActionFinderAxisymFudge af(pot);
        const size_t n6 = p6.size() / 6;
        std::vector<coord::PosVelCar> pv(n6);
        for(size_t i = 0; i < n6; i++)
            pv[i] = coord::PosVelCar(p6[6 * i], p6[6 * i + 1], p6[6 * i + 2], p6[6 * i + 3], p6[6 * i + 4], p6[6 * i + 5]);
        std::vector<actions::Actions> act(n6);
        af.evalmany(n6, pv.data(), act.data());
        f = std::fopen((prefix + "_act.txt").c_str(), "w");
        for(size_t i = 0; i < n6; i++) std::fprintf(f, "%.17g %.17g %.17g\n", act[i].Jr, act[i].Jz, act[i].Jphi);
        std::fclose(f);
        if(n6 > 0) {       // the reference's own call form: one cylindrical point
            const double x = p6[0], y = p6[1], R = std::sqrt(x * x + y * y), phi = std::atan2(y, x);
            const double c = R > 0 ? x / R : 1, s = R > 0 ? y / R : 0;
            const actions::Actions a = af.actions(coord::PosVelCyl(R, p6[2], phi, p6[3] * c + p6[4] * s, p6[5],
                                                                   -p6[3] * s + p6[4] * c));
            std::fprintf(stderr, "actions of the first point (cylindrical input): %.17g %.17g %.17g\n", a.Jr, a.Jz, a.Jphi);
        }
        std::vector<double> T(n6, 1.0);
        std::vector<coord::PosVelCar> fin(n6);
        orbit::integratemany(n6, pv.data(), T.data(), *pot, 0, orbit::OrbitIntParams(), fin.data());
        f = std::fopen((prefix + "_orb.txt").c_str(), "w");
        for(size_t i = 0; i < n6; i++)
            std::fprintf(f, "%.17g %.17g %.17g %.17g %.17g %.17g\n", fin[i].x, fin[i].y, fin[i].z, fin[i].vx, fin[i].vy,
                         fin[i].vz);
        std::fclose(f);
        // a trajectory of the first phase-space point: 11 samples over T = 1
        if(p6.size() >= 6) {
            const orbit::Trajectory traj = orbit::integrateTraj(
                coord::PosVelCar(p6[0], p6[1], p6[2], p6[3], p6[4], p6[5]), 1.0, 0.1, *pot);
            f = std::fopen((prefix + "_traj.txt").c_str(), "w");
            for(size_t j = 0; j < traj.size(); j++)
                std::fprintf(f, "%.17g %.17g %.17g %.17g %.17g %.17g %.17g\n", traj[j].second, traj[j].first.x,
                             traj[j].first.y, traj[j].first.z, traj[j].first.vx, traj[j].first.vy, traj[j].first.vz);
            std::fclose(f);
        }
    } catch(std::exception& e) {
        std::cerr << "cpp_api_check: " << e.what() << "\n";
        return 3;
    }
    return 0;
}
