// sodecl::sodeclmgr over the C ABI: the reference's manager
// (src/sodeclmgr.cpp) with the OpenCL discovery, program build and buffer
// code replaced by libsodecl_cuda calls.
#include "sodeclmgr.hpp"

#include <chrono>
#include <fstream>
#include <iostream>
#include <iterator>
#include <sstream>

namespace sodecl {

namespace {
std::string ctx_error(const sodecl_ctx *ctx)
{
    std::string s(sodecl_cuda_last_error(ctx, nullptr, 0) + 1, '\0');
    sodecl_cuda_last_error(ctx, &s[0], s.size());
    s.resize(s.size() - 1);
    return s;
}
}  // namespace

sodeclmgr::sodeclmgr(std::string kernel_path_str, char *sode_system_str, solver_Type solver, double dt, double int_time,
                     int kernel_steps, int num_equat, int num_params, int num_noi, int list_size, output_Type output_type)
    : m_output_type(output_type)
{
    (void)kernel_path_str;
    sodecl_cfg_init(&m_cfg);
    m_system_path = sode_system_str ? sode_system_str : "";
    m_cfg.solver = static_cast<int>(solver);
    m_cfg.dt = dt;
    m_cfg.int_time = int_time;
    m_cfg.kernel_steps = kernel_steps;
    m_cfg.num_equat = num_equat;
    m_cfg.num_params = num_params;
    m_cfg.num_noi = num_noi;
    m_cfg.list_size = list_size;
    // the log files start empty (src/clog.cpp:22-28)
    std::ofstream("sodecllog.txt", std::ios::binary | std::ios::out);
    std::ofstream("sodeclexitstatus.txt", std::ios::binary | std::ios::out);
}

sodeclmgr::~sodeclmgr()
{
    sodecl_cuda_destroy(m_ctx);
    // a normal exit (src/sodeclmgr.cpp:146-147, src/clog.cpp:76-92)
    std::ofstream f("sodeclexitstatus.txt", std::ios::binary | std::ios::app | std::ios::out);
    f << "1 Normal.";
}

void sodeclmgr::flush_log()
{
    std::ofstream f("sodecllog.txt", std::ios::binary | std::ios::app | std::ios::out);
    f << m_log.str();
    m_log.str(std::string());
}

int sodeclmgr::choose_device(unsigned platform_num, device_Type device_type, unsigned device_num)
{
    (void)platform_num;
    (void)device_type;
    int count = 0;
    if (sodecl_cuda_device_count(&count) != SODECL_OK || static_cast<int>(device_num) >= count) {
        m_error = "CUDA device " + std::to_string(device_num) + " not available";
        return 0;
    }
    m_cfg.device = static_cast<int>(device_num);
    // the selected device, as src/sodeclmgr.cpp:195-205 logs its OpenCL device
    char name[256] = {0};
    int major = 0, minor = 0;
    if (sodecl_cuda_device_describe(m_cfg.device, name, sizeof name, &major, &minor) == SODECL_OK) {
        m_log << "Selected platform name: NVIDIA CUDA\n";
        m_log << "Selected device name: " << name << "\n";
        m_log << "Selected device compute capability: " << major << "." << minor << "\n";
    }
    return 1;
}

void sodeclmgr::set_local_group_size(int local_group_size) { m_cfg.local_group_size = local_group_size; }
void sodeclmgr::set_t0(double *t0) { m_t0 = t0; }
void sodeclmgr::set_y0(double *y0) { m_y0 = y0; }
void sodeclmgr::set_params(double *params) { m_params = params; }
void sodeclmgr::set_noise_counters(const double *counters) { m_counters = counters; }
void sodeclmgr::set_newton(double tol, int max_iter)
{
    m_cfg.newton_tol = tol;
    m_cfg.newton_max_iter = max_iter;
}
void sodeclmgr::set_tolerances(double rtol, double atol, int max_steps)
{
    m_cfg.rtol = rtol;
    m_cfg.atol = atol;
    m_cfg.max_steps = max_steps;
}
void sodeclmgr::set_precision(int precision) { m_cfg.precision = precision; }
void sodeclmgr::set_fmad(bool on) { m_cfg.fmad = on ? 1 : 0; }

int sodeclmgr::read_binary_data_from_file(char *filename, double *data)
{
    std::ifstream ifs(filename, std::ios::in | std::ios::binary | std::ios::ate);
    if (!ifs.good()) {
        std::cout << "ERROR: can't open " << filename << " file." << std::endl;
        return 0;
    }
    const std::streamoff size = ifs.tellg();
    ifs.seekg(0, std::ios::beg);
    ifs.read(reinterpret_cast<char *>(data), (size / 8) * 8);
    return 1;
}

int sodeclmgr::read_data_from_file(char *filename, double *data)
{
    std::ifstream ifs(filename);
    if (!ifs.good()) {
        std::cout << "ERROR: can't open " << filename << " file." << std::endl;
        return 0;
    }
    size_t j = 0;
    std::string word;
    while (ifs >> word) data[j++] = std::atof(word.c_str());
    return 1;
}

int sodeclmgr::setup_sode_solver()
{
    std::ifstream f(m_system_path, std::ios::in | std::ios::binary);
    if (!f.good()) {
        m_error = "cannot read the system file " + m_system_path;
        std::cout << "Kernel code creation failed." << std::endl;
        return 0;
    }
    const std::string src((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    sodecl_cuda_destroy(m_ctx);
    m_ctx = nullptr;
    int rc = sodecl_cuda_create(&m_cfg, &m_ctx);
    if (rc != SODECL_OK) {
        m_error = std::string("invalid configuration: ") + sodecl_cuda_strerror(rc);
        std::cout << "Kernel code creation failed." << std::endl;
        return 0;
    }
    rc = sodecl_cuda_compile(m_ctx, src.data(), src.size());
    if (rc != SODECL_OK) {
        m_error = ctx_error(m_ctx);
        std::cout << "Failed to build kernel." << std::endl << m_error << std::endl;
        return 0;
    }
    {
        // the assembled program, written to the working directory as the
        // reference writes its OpenCL source (src/sodeclmgr.cpp:497-500)
        std::string program(sodecl_cuda_program_source(m_ctx, nullptr, 0) + 1, '\0');
        sodecl_cuda_program_source(m_ctx, &program[0], program.size());
        program.resize(program.size() - 1);
        std::ofstream dump("Generated_kernel.cl");
        dump << program;
    }
    // the files the program was built from and how (src/sodeclmgr.cpp:459-460, :579-581)
    m_log << m_system_path << "\n";
    m_log << "Build options string: NVRTC --gpu-architecture=sm_100a --fmad=" << (m_cfg.fmad ? "true" : "false")
          << "\n";
    rc = sodecl_cuda_upload(m_ctx, m_t0, m_y0, m_params, m_counters);
    if (rc != SODECL_OK) {
        m_error = ctx_error(m_ctx);
        std::cout << "Failed to write the data to the device buffers." << std::endl << m_error << std::endl;
        return 0;
    }
    return 1;
}

int sodeclmgr::run_sode_solver()
{
    if (!m_ctx) return 0;
    const int64_t per_run = sodecl_cuda_num_records(m_ctx) * m_cfg.num_equat * m_cfg.list_size;
    m_log << "The local group size is: " << static_cast<double>(m_cfg.local_group_size) << "\n";
    const auto start = std::chrono::steady_clock::now();
    int rc;
    if (m_output_type == output_Type::None) {
        rc = sodecl_cuda_run(m_ctx, nullptr, 0);
    } else {
        // a second run appends, as the reference's push_back does
        const size_t base = (m_output_type == output_Type::Array) ? m_output.size() : 0;
        std::vector<double> file_buf;
        std::vector<double> &dst = (m_output_type == output_Type::Array) ? m_output : file_buf;
        dst.resize(base + static_cast<size_t>(per_run));
        rc = sodecl_cuda_run(m_ctx, dst.data() + base, per_run);
        if (rc == SODECL_OK && m_output_type == output_Type::File) {
            // raw doubles appended, same order (src/sodeclmgr.cpp:926-927, :987-988)
            std::ofstream out(m_outputfile_str, std::ios::binary | std::ios::app | std::ios::out);
            out.write(reinterpret_cast<const char *>(file_buf.data()), static_cast<std::streamsize>(file_buf.size() * sizeof(double)));
        }
        if (rc != SODECL_OK && m_output_type == output_Type::Array) m_output.resize(base);
    }
    if (rc != SODECL_OK) {
        m_error = ctx_error(m_ctx);
        std::cout << "Error: failed to run the solver: " << m_error << std::endl;
        m_log << "Error: Failed to execute kernel!" << m_error;
        flush_log();
        return 0;
    }
    m_output_size = static_cast<int64_t>(m_output.size());
    const double walltime = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    std::cout << "Compute results runtime: " << walltime << " sec.\n";
    m_log << "Compute results runtime: " << walltime << "sec.\n";  // src/sodeclmgr.cpp:1019-1029
    flush_log();
    return 1;
}

int64_t sodeclmgr::output_length() const
{
    return m_ctx ? sodecl_cuda_num_records(m_ctx) * m_cfg.num_equat * m_cfg.list_size : 0;
}

int sodeclmgr::run_sode_solver_into(double *out, int64_t out_len)
{
    if (!m_ctx) return 0;
    m_log << "The local group size is: " << static_cast<double>(m_cfg.local_group_size) << "\n";
    const auto start = std::chrono::steady_clock::now();
    if (sodecl_cuda_run(m_ctx, out, out_len) != SODECL_OK) {
        m_error = ctx_error(m_ctx);
        std::cout << "Error: failed to run the solver: " << m_error << std::endl;
        m_log << "Error: Failed to execute kernel!" << m_error;
        flush_log();
        return 0;
    }
    const double walltime = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    std::cout << "Compute results runtime: " << walltime << " sec.\n";
    m_log << "Compute results runtime: " << walltime << "sec.\n";
    flush_log();
    return 1;
}

}  // namespace sodecl
