// Python module `sodecl_interface`: the reference's pybind11 binding
// (interfaces/python/sodecl.cpp:16-101) over the CUDA engine.
//
// sodeclcall(...) keeps the reference's signature and return value -- a flat
// list of doubles in [record][equation][orbit] order, empty on failure -- so
// the reference's sodecl.py runs on top unchanged.  sodeclcall_array(...)
// returns the same values as a numpy array without the list round trip and
// takes this library's options as keywords.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "sodeclmgr.hpp"

namespace py = pybind11;

namespace {

struct CallOptions {
    int precision = SODECL_FP64;
    int fmad = 1;
    double newton_tol = 1e-7;
    int newton_max_iter = 1000;
    const std::vector<double> *counters = nullptr;
};

bool run_call(std::vector<double> &a_t0, std::vector<double> &a_y0, std::vector<double> &a_params, int a_platform,
              int a_device, const std::string &a_system, int a_solver_type, int a_orbits, int a_equats, int a_nparams,
              int a_nnoi, double a_dt, double a_tspan, int a_ksteps, int a_local_group_size, const CallOptions &opt,
              std::vector<double> &out)
{
    if (a_solver_type < 0 || a_solver_type > 4) {
        std::cout << "Unknown SODE solver selection." << std::endl;
        return false;
    }
    const size_t n = a_orbits > 0 ? static_cast<size_t>(a_orbits) : 0;
    if (a_t0.size() < n || a_y0.size() < n * static_cast<size_t>(std::max(0, a_equats)) ||
        a_params.size() < n * static_cast<size_t>(std::max(0, a_nparams)) ||
        (opt.counters && opt.counters->size() < n)) {
        std::cout << "Input arrays are shorter than orbits x sizes." << std::endl;
        return false;
    }
    std::string path = a_system;
    sodecl::sodeclmgr mgr("kernels", &path[0], static_cast<sodecl::solver_Type>(a_solver_type), a_dt, a_tspan, a_ksteps,
                          a_equats, a_nparams, a_nnoi, a_orbits, sodecl::output_Type::Array);
    if (mgr.choose_device(a_platform, sodecl::device_Type::ALL, a_device) == 0)
        std::cerr << "Error selecting CUDA device!" << std::endl;
    mgr.set_t0(a_t0.data());
    mgr.set_y0(a_y0.data());
    mgr.set_params(a_params.data());
    mgr.set_local_group_size(a_local_group_size);
    mgr.set_precision(opt.precision);
    mgr.set_fmad(opt.fmad != 0);
    mgr.set_newton(opt.newton_tol, opt.newton_max_iter);
    if (opt.counters) mgr.set_noise_counters(opt.counters->data());
    if (mgr.setup_sode_solver() == 0) return false;
    if (mgr.run_sode_solver() == 0) return false;
    out.swap(mgr.m_output);
    return true;
}

std::vector<double> sodeclcall(std::vector<double> &a_t0, std::vector<double> &a_y0, std::vector<double> &a_params,
                               int a_platform, int a_device, std::string a_system, int a_solver_type, int a_orbits,
                               int a_equats, int a_nparams, int a_nnoi, double a_dt, double a_tspan, int a_ksteps,
                               int a_local_group_size)
{
    std::vector<double> out;
    py::gil_scoped_release release;
    if (!run_call(a_t0, a_y0, a_params, a_platform, a_device, a_system, a_solver_type, a_orbits, a_equats, a_nparams,
                  a_nnoi, a_dt, a_tspan, a_ksteps, a_local_group_size, CallOptions(), out))
        out.clear();
    return out;
}

using InArray = py::array_t<double, py::array::c_style | py::array::forcecast>;

// sodeclcall with numpy arrays in and out: the inputs are read in place (no
// per-element conversion to lists) and the records are written by the
// library straight into a new, uninitialised numpy array -- the device's
// record stream staged through pinned memory by the library's copy threads
// while the launches still run.  Returns an empty array on failure.
py::array_t<double> sodeclcall_array(InArray a_t0, InArray a_y0, InArray a_params, int a_platform, int a_device,
                                     std::string a_system, int a_solver_type, int a_orbits, int a_equats,
                                     int a_nparams, int a_nnoi, double a_dt, double a_tspan, int a_ksteps,
                                     int a_local_group_size, int precision, int fmad, double newton_tol,
                                     int newton_max_iter, py::object counters)
{
    if (a_solver_type < 0 || a_solver_type > 4) {
        std::cout << "Unknown SODE solver selection." << std::endl;
        return py::array_t<double>(0);
    }
    const py::ssize_t n = a_orbits > 0 ? a_orbits : 0;
    const bool have_counters = !counters.is_none();
    InArray cnt;
    if (have_counters) cnt = InArray::ensure(counters);
    if (a_t0.size() < n || a_y0.size() < n * std::max(0, a_equats) || a_params.size() < n * std::max(0, a_nparams) ||
        (have_counters && (!cnt || cnt.size() < n))) {
        std::cout << "Input arrays are shorter than orbits x sizes." << std::endl;
        return py::array_t<double>(0);
    }
    std::string path = a_system;
    sodecl::sodeclmgr mgr("kernels", &path[0], static_cast<sodecl::solver_Type>(a_solver_type), a_dt, a_tspan,
                          a_ksteps, a_equats, a_nparams, a_nnoi, a_orbits, sodecl::output_Type::Array);
    if (mgr.choose_device(a_platform, sodecl::device_Type::ALL, a_device) == 0)
        std::cerr << "Error selecting CUDA device!" << std::endl;
    mgr.set_t0(const_cast<double *>(a_t0.data()));
    mgr.set_y0(const_cast<double *>(a_y0.data()));
    mgr.set_params(const_cast<double *>(a_params.data()));
    mgr.set_local_group_size(a_local_group_size);
    mgr.set_precision(precision);
    mgr.set_fmad(fmad != 0);
    mgr.set_newton(newton_tol, newton_max_iter);
    if (have_counters) mgr.set_noise_counters(cnt.data());
    bool ok;
    {
        py::gil_scoped_release release;
        ok = mgr.setup_sode_solver() != 0;
    }
    if (!ok) return py::array_t<double>(0);
    py::array_t<double> out(static_cast<py::ssize_t>(mgr.output_length()));
    double *dst = out.mutable_data();
    const int64_t len = out.size();
    {
        py::gil_scoped_release release;
        ok = mgr.run_sode_solver_into(dst, len) != 0;
    }
    return ok ? out : py::array_t<double>(0);
}

}  // namespace

PYBIND11_MODULE(sodecl_interface, m)
{
    m.doc() = "sodecl plugin (CUDA engine for B200)";
    m.def("sodeclcall", &sodeclcall, "A function that integrates a SDE/ODE system.");
    m.def("sodeclcall_array", &sodeclcall_array, "sodeclcall returning a numpy array, with extra options.",
          py::arg("t0"), py::arg("y0"), py::arg("params"), py::arg("platform"), py::arg("device"), py::arg("system"),
          py::arg("solver_type"), py::arg("orbits"), py::arg("equats"), py::arg("nparams"), py::arg("nnoi"),
          py::arg("dt"), py::arg("tspan"), py::arg("ksteps"), py::arg("local_group_size"),
          py::arg("precision") = 0, py::arg("fmad") = 1, py::arg("newton_tol") = 1e-7,
          py::arg("newton_max_iter") = 1000, py::arg("counters") = py::none());
}
