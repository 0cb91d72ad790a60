// A C++ caller written against goss's ODESystemSolver API, built with g++
// against include/goss_b200.hpp and libgoss_b200.so by tests/test_cpp_dropin.py.
//
//   dropin_main <model library> <variant> <case> <N> <in.bin> <out.bin>
//
// in.bin holds the initial states [N][n] (then, for case "fields", the field
// parameters [N][nfp]); out.bin receives what the case computes.
//   grl1   : GRL1, internal step 0.01 ms, forward(k, 1 ms) for k < 10; the
//            final states [N][n]
//   fields : the same with set_field_parameters, then solve() over 5 more
//            1 ms steps with V as the field state; the final states [N][n],
//            the field parameters read back [N][nfp] and the solve trajectory
//            [6][N][1]
//   theta  : ThetaSolver (theta = 0.5, internal step 0.1 ms), 10 x forward(0.1 ms)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "goss_b200.hpp"

namespace goss = goss_b200;

static std::vector<double> read_all(const char* path)
{
    std::vector<double> v;
    FILE* f = std::fopen(path, "rb");
    if (!f)
        return v;
    double x;
    while (std::fread(&x, sizeof(double), 1, f) == 1)
        v.push_back(x);
    std::fclose(f);
    return v;
}

int main(int argc, char** argv)
{
    if (argc != 7) {
        std::fprintf(stderr, "usage: %s <lib> <variant> <case> <N> <in.bin> <out.bin>\n", argv[0]);
        return 2;
    }
    const std::string kase = argv[3];
    const goss::uint N = (goss::uint)std::strtoul(argv[4], nullptr, 10);
    try {
        auto ode = goss::ParameterizedODE::load(argv[1], argv[2]);
        const goss::uint n = ode->num_states(), nfp = ode->num_field_parameters();
        std::vector<double> in = read_all(argv[5]);
        if (in.size() < (size_t)N * n)
            throw std::runtime_error("short input");
        std::vector<double> out;
        if (kase == "theta") {
            auto solver = std::make_shared<goss::ThetaSolver>();
            solver->set_internal_time_step(0.1);
            solver->theta = 0.5;
            goss::ODESystemSolver system(N, solver, ode);
            system.set_states(in.data());
            for (int k = 0; k < 10; ++k)
                system.forward(0.1 * k, 0.1);
            out.assign(system.states(), system.states() + (size_t)N * n);
        } else {
            if (kase == "fields")
                ode->set_field_states({"V"});
            auto solver = std::make_shared<goss::GRL1>(ode);
            solver->set_internal_time_step(0.01);
            goss::ODESystemSolver system(N, solver, ode);
            if (system.num_nodes() != N || solver->get_ode() != ode)
                throw std::runtime_error("accessors");
            system.set_states(in.data());
            if (kase == "fields") {
                if (in.size() < (size_t)N * (n + nfp))
                    throw std::runtime_error("short input");
                system.set_field_parameters(in.data() + (size_t)N * n);
            }
            for (int k = 0; k < 10; ++k)
                system.forward(1.0 * k, 1.0);
            if (kase == "fields") {
                std::vector<double> t = {10.0, 11.0, 12.0, 13.0, 14.0, 15.0};
                std::vector<double> traj(t.size() * N, 0.0);
                system.solve(traj.data(), t.data(), t.size());
                out.assign(system.states(), system.states() + (size_t)N * n);
                std::vector<double> fp((size_t)N * nfp);
                system.get_field_parameters(fp.data());
                out.insert(out.end(), fp.begin(), fp.end());
                out.insert(out.end(), traj.begin(), traj.end());
            } else {
                out.assign(system.states(), system.states() + (size_t)N * n);
            }
        }
        FILE* f = std::fopen(argv[6], "wb");
        if (!f || std::fwrite(out.data(), sizeof(double), out.size(), f) != out.size())
            throw std::runtime_error("cannot write output");
        std::fclose(f);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
