// NVRTC front end: turns a SODECL system file into an sm_100a cubin.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace sodecl_b200 {

struct ProgramSpec {
    int solver = 1;          // solver_Type numbering
    int num_equat = 0;
    int num_params = 0;
    int num_noi = 0;
    int64_t list_size = 0;
    int kernel_steps = 1;
    double dt = 0.0;         // user dt; printed like the reference
    bool fp32 = false;
    bool fmad = true;
    bool record_f32 = false;
    bool fast_div = false;   // FP64 through sodecl_f64 (exact reciprocal quotients)
    double newton_tol = 1e-7;
    int newton_max_iter = 1000;
    int block_max = 256;
    int min_blocks = 0;
    int lanes = 1;           // lanes per orbit (1, or a power of two up to 32)
    bool pair_stores = false;  // one thread per orbit: records two orbits per vector store
    double rtol = 1e-6;      // adaptive solver (solver 5): error tolerances and
    double atol = 1e-9;      // step attempts per record interval
    int max_steps = 100000;
};

struct Program {
    std::string source;      // full program text handed to NVRTC
    std::string log;         // NVRTC log (with ptxas resource usage)
    std::vector<char> cubin;
    std::string kernel_name = "sodecl_orbits";
    bool fast_div = false;   // built with the reciprocal-division wrapper
};

// What the system file provides.
struct SystemTraits {
    bool has_system = false;
    bool has_jacobian = false;
    bool has_stoch = false;
    bool has_pjacobian = false;  // calc_jacobian_params (df/dp), used by the adjoint
    bool has_row = false;        // sode_system_row (one equation's right-hand side)
    bool has_stoch_row = false;  // sode_system_stoch_row
    bool has_jac_band = false;   // calc_jacobian_band (row i's entries in columns i-1, i, i+1)
    bool has_row_band = false;   // sode_system_row_band (a row's right-hand side and band together)
    bool has_vjp = false;        // calc_vjp (v^T df/dy and v^T df/dp), used by the adjoint
    bool uses_listsize = false;
};

SystemTraits inspect_system(const std::string &src);

// `dt` exactly as the reference writes it into `#define _m_dt_`: a default
// std::ostream, i.e. %g with 6 significant digits (src/sodeclmgr.cpp:356-367).
std::string print_like_reference(double x);
// "#define SODECL_L2_BOUND <t>\n": the exact bound for the implicit midpoint's
// stop test sqrt(norm) < tol (norm < t), or "" where it is not a normal number.
std::string l2_bound_define(double newton_tol, bool fp32);

// Every unsuffixed floating literal outside comments, strings and character
// constants gets an `f` suffix (fp32 programs).
std::string suffix_float_literals(const std::string &src);

// Shared memory words (real_t) of one orbit in the lanes-per-orbit kernel;
// must match SODECL_SLOT in device/solvers.cuh.
int lanes_slot_words(const ProgramSpec &spec);

// Assembles the program text.
std::string assemble(const ProgramSpec &spec, const std::string &system_src, const SystemTraits &traits);

// Compiles (or returns from the process-wide cache) the program.  Throws
// std::runtime_error with the NVRTC log on failure.
std::shared_ptr<const Program> build(const ProgramSpec &spec, const std::string &system_src);

// The discrete-adjoint program (kernel `sodecl_adjoint`) for the Euler or RK4
// solver: the system file twice, plain and with `double` recording on a tape
// of `tape_cap` entries per right-hand-side evaluation.  mode: where the
// vector-Jacobian products come from -- 2 the file's calc_vjp, 1 its
// calc_jacobian and calc_jacobian_params, 0 the tape.  gradient = false
// builds the loss-only kernel (the forward sweep alone).
std::shared_ptr<const Program> build_adjoint(const ProgramSpec &spec, const std::string &system_src, int tape_cap,
                                             int mode, bool gradient = true);

// One class of a heterogeneous batch: a system file with a solver, sizes,
// step and Newton settings (kernel_steps/list_size unused).
struct BatchClass {
    ProgramSpec spec;
    std::string system_src;
};

// Doubles of dynamic shared memory each warp of the batch kernel needs: the
// largest (32 / lanes) x slot of the classes with lanes per orbit, else 0.
int batch_warp_words(const std::vector<BatchClass> &classes);

// All classes in one program with the persistent kernel `sodecl_batch`,
// for blocks of at most block_max threads; min_blocks > 0 asks the compiler
// for that many resident blocks of block_max threads (a register cap of
// 65536 / (min_blocks x block_max) per thread).
std::shared_ptr<const Program> build_batch(const std::vector<BatchClass> &classes, bool fmad, bool fast_div,
                                           int block_max, int min_blocks = 0);

}  // namespace sodecl_b200
