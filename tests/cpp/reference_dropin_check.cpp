// The engine's drop-in classes (include/agama_b200_reference.hpp) used by C++ code built against
// the reference library, the way its own callers hold a potential and an action finder:
//   * a potential::PtrPotential to the engine's MultipoleB200 and one to the reference's own
//     Multipole (potential::readPotential of the same coefficient file), evaluated through the
//     reference's eval front-ends in Cartesian, cylindrical and spherical coordinates, with
//     gradient and Hessian;
//   * the reference's own routines given the engine's potential: potential::R_circ, and the
//     standalone Staeckel fudge actions::evalAxisymFudge at a fixed focal distance;
//   * the batched density (BaseDensity::evalmanyDensityCar, overridden by the engine);
//   * the engine's ActionFinderB200 through actions::BaseActionFinder (eval / actions) against
//     the reference's golden actions (compared by the test that runs this program).
// usage: reference_dropin_check coef.coef points3.txt points6.txt fd.txt outprefix
// Writes outprefix_{pot,cyl,sph,hess,rc,fud,rho,act}.txt with the engine's and the reference's
// values side by side; exit code 3 when the engine has no CUDA device (no CPU fallback).
#include "agama_b200_reference.hpp"
#include "potential_factory.h"
#include "potential_utils.h"
#include "actions_staeckel.h"
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>

namespace {

std::vector<std::vector<double> > readRows(const char* file, size_t ncol)
{
    std::ifstream in(file);
    std::vector<std::vector<double> > rows;
    std::string line;
    while(std::getline(in, line)) {
        std::istringstream ss(line);
        std::vector<double> r(ncol);
        for(size_t k = 0; k < ncol; k++) ss >> r[k];
        if(ss) rows.push_back(r);
    }
    return rows;
}

}  // namespace

int main(int argc, char** argv)
{
    if(argc < 6) {
        std::cerr << "usage: reference_dropin_check coef points3 points6 fd outprefix\n";
        return 2;
    }
    const std::string coef = argv[1], out = argv[5];
    shared_ptr<const agama_b200::MultipoleB200> engine;
    try {
        engine.reset(new agama_b200::MultipoleB200(coef));
    } catch(std::exception& e) {
        std::cerr << "engine: " << e.what() << "\n";
        return 3;
    }
    const potential::PtrPotential gpu = engine;
    const potential::PtrPotential cpu = potential::readPotential(coef);
    const std::vector<std::vector<double> > p3 = readRows(argv[2], 3), p6 = readRows(argv[3], 6),
        fd = readRows(argv[4], 1);
    std::cout << "potentials: " << gpu->name() << " (engine) / " << cpu->name() << " (reference), symmetry "
              << gpu->symmetry() << " / " << cpu->symmetry() << "\n";

    // Phi and gradient at Cartesian points, through BasePotential::eval(PosCar)
    {
        FILE* f = std::fopen((out + "_pot.txt").c_str(), "w");
        FILE* fh = std::fopen((out + "_hess.txt").c_str(), "w");
        for(size_t i = 0; i < p3.size(); i++) {
            const coord::PosCar x(p3[i][0], p3[i][1], p3[i][2]);
            double pg, pc;
            coord::GradCar gg, gc;
            coord::HessCar hg, hc;
            gpu->eval(x, &pg, &gg, &hg);
            cpu->eval(x, &pc, &gc, &hc);
            std::fprintf(f, "%.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n", pg, gg.dx, gg.dy, gg.dz,
                pc, gc.dx, gc.dy, gc.dz);
            std::fprintf(fh, "%.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n",
                hg.dx2, hg.dy2, hg.dz2, hg.dxdy, hg.dydz, hg.dxdz, hc.dx2, hc.dy2, hc.dz2, hc.dxdy, hc.dydz, hc.dxdz);
        }
        std::fclose(f);
        std::fclose(fh);
    }
    // cylindrical and spherical front-ends (value, gradient, Hessian)
    {
        FILE* f = std::fopen((out + "_cyl.txt").c_str(), "w");
        FILE* fs = std::fopen((out + "_sph.txt").c_str(), "w");
        for(size_t i = 0; i < p3.size(); i++) {
            const coord::PosCyl x = coord::toPosCyl(coord::PosCar(p3[i][0], p3[i][1], p3[i][2]));
            double pg, pc;
            coord::GradCyl gg, gc;
            coord::HessCyl hg, hc;
            gpu->eval(x, &pg, &gg, &hg);
            cpu->eval(x, &pc, &gc, &hc);
            std::fprintf(f, "%.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g "
                "%.17g %.17g %.17g %.17g %.17g %.17g\n", pg, gg.dR, gg.dz, gg.dphi, hg.dR2, hg.dz2, hg.dphi2,
                hg.dRdz, hg.dzdphi, hg.dRdphi, pc, gc.dR, gc.dz, gc.dphi, hc.dR2, hc.dz2, hc.dphi2, hc.dRdz,
                hc.dzdphi, hc.dRdphi);
            const coord::PosSph s = coord::toPosSph(coord::PosCar(p3[i][0], p3[i][1], p3[i][2]));
            coord::GradSph sg, sc;
            gpu->eval(s, &pg, &sg);
            cpu->eval(s, &pc, &sc);
            std::fprintf(fs, "%.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n", pg, sg.dr, sg.dtheta, sg.dphi,
                pc, sc.dr, sc.dtheta, sc.dphi);
        }
        std::fclose(f);
        std::fclose(fs);
    }
    // the reference's own routines given the engine's potential
    {
        FILE* f = std::fopen((out + "_rc.txt").c_str(), "w");
        const double Phi0 = gpu->value(coord::PosCyl(0, 0, 0));
        for(int k = 1; k <= 8; k++) {
            const double E = Phi0 * (1 - 0.11 * k);
            std::fprintf(f, "%.17g %.17g %.17g\n", E, potential::R_circ(*gpu, E), potential::R_circ(*cpu, E));
        }
        std::fclose(f);
        FILE* fa = std::fopen((out + "_fud.txt").c_str(), "w");
        for(size_t i = 0; i < p6.size() && i < 12; i++) {
            const coord::PosVelCyl w = coord::toPosVelCyl(coord::PosVelCar(p6[i][0], p6[i][1], p6[i][2],
                p6[i][3], p6[i][4], p6[i][5]));
            actions::Actions ag, ac;
            actions::evalAxisymFudge(*gpu, w, &ag, NULL, NULL, fd[i][0]);
            actions::evalAxisymFudge(*cpu, w, &ac, NULL, NULL, fd[i][0]);
            std::fprintf(fa, "%.17g %.17g %.17g %.17g %.17g %.17g\n", ag.Jr, ag.Jz, ag.Jphi, ac.Jr, ac.Jz, ac.Jphi);
        }
        std::fclose(fa);
    }
    // batched density, overridden by the engine (one call for the array)
    {
        std::vector<coord::PosCar> pos(p3.size());
        for(size_t i = 0; i < p3.size(); i++) pos[i] = coord::PosCar(p3[i][0], p3[i][1], p3[i][2]);
        std::vector<double> rg(pos.size()), rc(pos.size());
        gpu->evalmanyDensityCar(pos.size(), &pos[0], &rg[0]);
        cpu->evalmanyDensityCar(pos.size(), &pos[0], &rc[0]);
        FILE* f = std::fopen((out + "_rho.txt").c_str(), "w");
        for(size_t i = 0; i < pos.size(); i++) std::fprintf(f, "%.17g %.17g\n", rg[i], rc[i]);
        std::fclose(f);
    }
    // the engine's action finder through the reference's abstract interface
    {
        const actions::PtrActionFinder af(new agama_b200::ActionFinderB200(engine));
        std::cout << "action finder: " << af->name() << "\n";
        FILE* f = std::fopen((out + "_act.txt").c_str(), "w");
        std::vector<coord::PosVelCyl> pts;
        for(size_t i = 0; i < p6.size(); i++)
            pts.push_back(coord::toPosVelCyl(coord::PosVelCar(p6[i][0], p6[i][1], p6[i][2], p6[i][3], p6[i][4],
                p6[i][5])));
        std::vector<actions::Actions> many(pts.size());
        static_cast<const agama_b200::ActionFinderB200&>(*af).evalmany(pts.size(), &pts[0], &many[0]);
        for(size_t i = 0; i < pts.size(); i++) {
            const actions::Actions one = i < 16 ? af->actions(pts[i]) : many[i];     // the single-point path too
            std::fprintf(f, "%.17g %.17g %.17g %.17g %.17g %.17g\n", one.Jr, one.Jz, one.Jphi, many[i].Jr, many[i].Jz,
                many[i].Jphi);
        }
        std::fclose(f);
    }
    std::cout << "done\n";
    return 0;
}
