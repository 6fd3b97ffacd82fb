// The reference's C++ call sequence (interfaces/python/sodecl.cpp:56-94) on
// the CUDA engine: oculomotor RK4, dt 1e-6, tspan 0.1, ksteps 400, 2 orbits.
// argv[1] = system file, argv[2] = where to write m_output (raw doubles).
// A second manager with output_Type::File writes sodecloutput.bin in the CWD.
#include <cstdio>
#include <fstream>
#include <vector>

#include "sodeclmgr.hpp"

int main(int argc, char **argv)
{
    if (argc < 3) return 2;
    std::vector<double> t0(2, 0.0), y0, params;
    for (int o = 0; o < 2; ++o) {
        double y[6] = {0, 0, 0, 0, 0, 2.0};
        double p[6] = {120, 1.5, 0.0045, 0.05, 600, 9};
        y0.insert(y0.end(), y, y + 6);
        params.insert(params.end(), p, p + 6);
    }
    for (int pass = 0; pass < 2; ++pass) {
        const auto kind = pass == 0 ? sodecl::output_Type::Array : sodecl::output_Type::File;
        sodecl::sodeclmgr mgr("kernels", argv[1], sodecl::solver_Type::RungeKutta, 1e-6, 0.1, 400, 6, 6, 0, 2, kind);
        if (mgr.choose_device(0, sodecl::device_Type::ALL, 0) == 0) return 3;
        mgr.set_t0(t0.data());
        mgr.set_y0(y0.data());
        mgr.set_params(params.data());
        mgr.set_local_group_size(0);
        if (mgr.setup_sode_solver() == 0) return 4;
        if (mgr.run_sode_solver() == 0) return 5;
        if (pass == 0) {
            if (mgr.m_output.size() != 12u * 252u) return 6;
            std::ofstream out(argv[2], std::ios::binary);
            out.write(reinterpret_cast<const char *>(mgr.m_output.data()), mgr.m_output.size() * sizeof(double));
        }
    }
    return 0;
}
