// sodeclmgr.hpp -- drop-in C++ manager for the CUDA engine.
//
// Same public surface as the reference's sodecl::sodeclmgr
// (include/sodeclmgr.hpp:27-369 of the reference): constructor, choose_device,
// set_local_group_size, set_t0/set_y0/set_params, setup_sode_solver,
// run_sode_solver, m_output.  The OpenCL types become plain C++ types
// (cl_uint -> unsigned, cl_double -> double); the enums keep their names and
// values.  Everything below the public methods is the C ABI of sodecl_cuda.h.
#ifndef SODECL_B200_SODECLMGR_HPP
#define SODECL_B200_SODECLMGR_HPP

#include <cstdint>
#include <sstream>
#include <string>
#include <vector>

#include "sodecl_cuda.h"

namespace sodecl {

// include/solver_Type.hpp:14-20 of the reference
// DormandPrince (adaptive steps) has no counterpart in the reference
enum class solver_Type {
    StochasticEuler = 0, Euler = 1, RungeKutta = 2, ImplicitEuler = 3, ImplicitMidpoint = 4, DormandPrince = 5
};

// include/output_Type.hpp:14-18 of the reference
enum class output_Type { None = 0, Array = 1, File = 2 };

// include/device_Type.hpp:14-19 of the reference (OpenCL device-type bits);
// accepted for source compatibility, CUDA devices are chosen by ordinal.
enum class device_Type : uint64_t { ALL = 0xFFFFFFFFull, CPU = 1ull << 1, GPU = 1ull << 2, ACCELERATOR = 1ull << 3 };

class sodeclmgr {
  public:
    std::vector<double> m_output;  // records, [record][equation][orbit]
    // Number of doubles in m_output after a run.  The reference declares this
    // member as int (and never sets it); 64 bits here, because the records
    // of large runs pass 2^31 doubles (2^20 orbits x 6 equations x 400
    // records).
    int64_t m_output_size = 0;

    // kernel_path_str is accepted and ignored (the solvers are built in);
    // sode_system_str is the path of the system file, read at setup.  As the
    // reference's manager does, construction starts sodecllog.txt and
    // sodeclexitstatus.txt empty in the working directory, each run appends
    // its log lines to the first, and destruction appends "1 Normal." to the
    // second.
    sodeclmgr(std::string kernel_path_str, char *sode_system_str, solver_Type solver, double dt, double int_time,
              int kernel_steps, int num_equat, int num_params, int num_noi, int list_size, output_Type output_type);
    ~sodeclmgr();
    sodeclmgr(const sodeclmgr &) = delete;
    sodeclmgr &operator=(const sodeclmgr &) = delete;

    // platform_num and device_type are ignored; device_num is the CUDA ordinal.
    // Returns 1 if the device exists, 0 otherwise.
    int choose_device(unsigned platform_num, device_Type device_type, unsigned device_num);

    // Threads per CUDA block (0 = library default).
    void set_local_group_size(int local_group_size);

    // Non-owning: the arrays must stay valid until setup_sode_solver returns.
    void set_t0(double *t0);
    void set_y0(double *y0);
    void set_params(double *params);

    // Reads a whitespace-separated text file / raw doubles into `data`.
    int read_binary_data_from_file(char *filename, double *data);
    int read_data_from_file(char *filename, double *data);

    // 1 = success, 0 = failure, as the reference.
    int setup_sode_solver();
    int run_sode_solver();

    // ---- additions (no counterpart in the reference) ----
    // Noise draw counters, list_size doubles (non-owning, read at setup);
    // without them the counters are drawn as the reference draws them.
    void set_noise_counters(const double *counters);
    void set_newton(double tol, int max_iter);
    void set_tolerances(double rtol, double atol, int max_steps);  // solver_Type::DormandPrince
    void set_precision(int precision);  // SODECL_FP64 or SODECL_FP32
    void set_fmad(bool on);
    // Doubles one run writes (records x equations x orbits); valid after
    // setup_sode_solver.
    int64_t output_length() const;
    // run_sode_solver with the records written to `out` (host or device
    // memory of at least output_length() doubles) instead of m_output; the
    // output type is not consulted.  1 = success, 0 = failure.
    int run_sode_solver_into(double *out, int64_t out_len);
    sodecl_ctx *context() const { return m_ctx; }
    const std::string &last_error() const { return m_error; }

  private:
    sodecl_cfg m_cfg{};
    std::string m_system_path;
    output_Type m_output_type;
    std::string m_outputfile_str = "sodecloutput.bin";
    double *m_t0 = nullptr;
    double *m_y0 = nullptr;
    double *m_params = nullptr;
    const double *m_counters = nullptr;
    sodecl_ctx *m_ctx = nullptr;
    std::string m_error;
    // What the reference's log singleton collects (src/clog.cpp): appended
    // to sodecllog.txt in the working directory after each run.
    std::ostringstream m_log;
    void flush_log();
};

}  // namespace sodecl

#endif
