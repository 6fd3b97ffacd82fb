// NVRTC front end: the CUDA counterpart of the reference's
// create_kernel_string + build_program (src/sodeclmgr.cpp:374-622).
//
// The reference concatenates size #defines, the user's system file, one
// solver file and one caller kernel into an OpenCL program.  Here the
// program is: config macros, the OpenCL-compatibility prelude, the noise
// generator, the same size #defines with the same names and values, the
// user's system file verbatim, and this library's solver kernels -- compiled
// by NVRTC straight to an sm_100a cubin.
#include "program.hpp"

#include <nvrtc.h>

#include <dlfcn.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <limits>
#include <mutex>
#include <regex>
#include <sstream>
#include <stdexcept>
#include <unordered_map>

namespace sodecl_b200 {

namespace {
#include "embedded_sources.inc"  // kFastDivSrc kPreludeSrc kThreefrySrc kSolversSrc kBatchSrc kAdjointSrc (build.py)

// Splits `src` into code / comment / literal runs and passes the code runs
// through `on_code`; comments are kept (or blanked), literals kept.
template <class F>
std::string scan_code(const std::string &src, F on_code, bool keep_comments)
{
    std::string out, code;
    out.reserve(src.size() + 64);
    auto flush = [&]() {
        if (!code.empty()) {
            out += on_code(code);
            code.clear();
        }
    };
    const size_t n = src.size();
    size_t i = 0;
    while (i < n) {
        const char c = src[i];
        if (c == '/' && i + 1 < n && src[i + 1] == '/') {
            size_t j = src.find('\n', i);
            if (j == std::string::npos) j = n;
            flush();
            out += keep_comments ? src.substr(i, j - i) : std::string(j - i, ' ');
            i = j;
        } else if (c == '/' && i + 1 < n && src[i + 1] == '*') {
            size_t j = src.find("*/", i + 2);
            j = (j == std::string::npos) ? n : j + 2;
            flush();
            if (keep_comments) {
                out += src.substr(i, j - i);
            } else {
                for (size_t k = i; k < j; ++k) out += (src[k] == '\n') ? '\n' : ' ';
            }
            i = j;
        } else if (c == '"' || c == '\'') {
            size_t j = i + 1;
            while (j < n && src[j] != c) j += (src[j] == '\\') ? 2 : 1;
            j = std::min(j + 1, n);
            flush();
            out += src.substr(i, j - i);
            i = j;
        } else {
            code += c;
            ++i;
        }
    }
    flush();
    return out;
}

bool ident_char(char c) { return std::isalnum(static_cast<unsigned char>(c)) || c == '_'; }

std::string suffix_in_code(const std::string &code)
{
    std::string out;
    out.reserve(code.size() + 16);
    const size_t n = code.size();
    size_t i = 0;
    while (i < n) {
        const char c = code[i];
        const bool starts_number = std::isdigit(static_cast<unsigned char>(c)) ||
                                   (c == '.' && i + 1 < n && std::isdigit(static_cast<unsigned char>(code[i + 1])));
        const bool glued = i > 0 && (ident_char(code[i - 1]) || code[i - 1] == '.');
        if (!starts_number || glued) {
            out += c;
            ++i;
            continue;
        }
        // a preprocessing number: digits, letters, '.', and exponent signs
        size_t j = i;
        while (j < n) {
            const char d = code[j];
            if (ident_char(d) || d == '.') {
                ++j;
            } else if ((d == '+' || d == '-') && j > i &&
                       (code[j - 1] == 'e' || code[j - 1] == 'E' || code[j - 1] == 'p' || code[j - 1] == 'P')) {
                ++j;
            } else {
                break;
            }
        }
        std::string num = code.substr(i, j - i);
        const bool hex = num.size() > 1 && num[0] == '0' && (num[1] == 'x' || num[1] == 'X');
        bool floating;
        if (hex) {
            floating = num.find_first_of("pP") != std::string::npos;
        } else {
            floating = num.find('.') != std::string::npos || num.find_first_of("eE") != std::string::npos;
        }
        const char last = num.back();
        const bool suffixed = last == 'f' || last == 'F' || last == 'l' || last == 'L';
        out += num;
        if (floating && !suffixed) out += 'f';
        i = j;
    }
    return out;
}

// Inside the parameter lists of file-scope function declarators, empties
// the first array bound of every parameter: `double noise[_numnoi_]` ->
// `double noise[]`.  C and C++ ignore that bound (the parameter is a
// pointer), but C++ rejects it when it is zero -- which the reference's
// system files produce for ODE runs, where _numnoi_ is 0 -- while OpenCL C
// compilers accept it.  Inner bounds (`jac[][_numeq_]`) are kept.
std::string relax_parameter_bounds(const std::string &src)
{
    std::string out = src;
    const size_t n = src.size();
    int brace = 0;
    bool line_start = true;
    size_t i = 0;
    auto skip_trivia = [&](size_t k) {
        while (k < n) {
            if (std::isspace(static_cast<unsigned char>(src[k]))) {
                ++k;
            } else if (src.compare(k, 2, "//") == 0) {
                k = src.find('\n', k);
                if (k == std::string::npos) return n;
            } else if (src.compare(k, 2, "/*") == 0) {
                k = src.find("*/", k + 2);
                if (k == std::string::npos) return n;
                k += 2;
            } else {
                break;
            }
        }
        return k;
    };
    while (i < n) {
        const char c = src[i];
        if (c == '\n') { line_start = true; ++i; continue; }
        if (std::isspace(static_cast<unsigned char>(c))) { ++i; continue; }
        if (src.compare(i, 2, "//") == 0) { i = src.find('\n', i); if (i == std::string::npos) break; continue; }
        if (src.compare(i, 2, "/*") == 0) { i = src.find("*/", i + 2); if (i == std::string::npos) break; i += 2; continue; }
        if (line_start && c == '#') {  // preprocessor line, with continuations
            while (i < n && !(src[i] == '\n' && src[i - 1] != '\\')) ++i;
            continue;
        }
        line_start = false;
        if (c == '"' || c == '\'') {
            size_t j = i + 1;
            while (j < n && src[j] != c) j += (src[j] == '\\') ? 2 : 1;
            i = j + 1;
            continue;
        }
        if (c == '{') { ++brace; ++i; continue; }
        if (c == '}') { --brace; ++i; continue; }
        if (c != '(' || brace != 0) { ++i; continue; }
        // candidate parameter list at file scope: find the matching ')'
        size_t j = i + 1;
        int depth = 1;
        while (j < n && depth > 0) {
            if (src.compare(j, 2, "//") == 0 || src.compare(j, 2, "/*") == 0) { j = skip_trivia(j); continue; }
            if (src[j] == '(') ++depth;
            else if (src[j] == ')') --depth;
            if (depth > 0) ++j;
        }
        if (j >= n) break;
        const size_t after = skip_trivia(j + 1);
        if (after < n && (src[after] == '{' || src[after] == ';')) {
            // blank the first [...] of each top-level parameter
            bool first_bracket_done = false;
            int pdepth = 0;
            for (size_t k = i + 1; k < j; ++k) {
                const char d = src[k];
                if (d == '(') ++pdepth;
                else if (d == ')') --pdepth;
                else if (d == ',' && pdepth == 0) first_bracket_done = false;
                else if (d == '[' && pdepth == 0 && !first_bracket_done) {
                    size_t e = k + 1;
                    int bdepth = 1;
                    while (e < j && bdepth > 0) {
                        if (src[e] == '[') ++bdepth;
                        else if (src[e] == ']') --bdepth;
                        if (bdepth > 0) ++e;
                    }
                    for (size_t q = k + 1; q < e; ++q)
                        if (out[q] != '\n') out[q] = ' ';
                    first_bracket_done = true;
                    k = e;
                }
            }
        }
        i = j + 1;
    }
    return out;
}

bool defines_function(const std::string &stripped, const char *name)
{
    const std::regex def(std::string("\\b") + name + "\\s*\\([^;{}]*\\)\\s*\\{");
    return std::regex_search(stripped, def);
}

std::string compile_options_key(const std::vector<std::string> &opts)
{
    std::string k;
    for (const auto &o : opts) {
        k += o;
        k += '\x1f';
    }
    return k;
}

std::mutex g_cache_mutex;
std::unordered_map<std::string, std::shared_ptr<const Program>> g_cache;

// ---- on-disk cubin cache --------------------------------------------------
// Directory: $SODECL_B200_CACHE_DIR, else `_cache` next to this library
// (so programs built once travel with the package); disabled when the
// variable is set to an empty string or the directory cannot be made.
// Entry name = two 64-bit FNV-1a hashes of the full key (options + source);
// each entry stores the key and is used only when it matches byte for byte.

std::string cache_dir()
{
    const char *env = std::getenv("SODECL_B200_CACHE_DIR");
    if (env) return env;
    Dl_info info{};
    if (dladdr(reinterpret_cast<void *>(&cache_dir), &info) && info.dli_fname) {
        std::string path(info.dli_fname);
        const size_t slash = path.rfind('/');
        return (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) + "/_cache";
    }
    return std::string();
}

uint64_t fnv1a(const std::string &s, uint64_t h)
{
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ULL;
    }
    return h;
}

std::string cache_path(const std::string &key)
{
    const std::string dir = cache_dir();
    if (dir.empty()) return std::string();
    mkdir(dir.c_str(), 0755);
    char name[64];
    std::snprintf(name, sizeof(name), "/%016llx%016llx.cubin", (unsigned long long)fnv1a(key, 1469598103934665603ULL),
                  (unsigned long long)fnv1a(key, 0x9E3779B97F4A7C15ULL));
    return dir + name;
}

bool cache_load(const std::string &key, Program &prog)
{
    const std::string path = cache_path(key);
    if (path.empty()) return false;
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    uint64_t sizes[3];
    if (!f.read(reinterpret_cast<char *>(sizes), sizeof(sizes))) return false;
    if (sizes[0] != key.size() || sizes[1] > (1ull << 30) || sizes[2] > (1ull << 26)) return false;
    std::string stored(sizes[0], '\0');
    if (!f.read(&stored[0], sizes[0]) || stored != key) return false;
    prog.cubin.resize(sizes[1]);
    prog.log.resize(sizes[2]);
    if (!f.read(prog.cubin.data(), sizes[1])) return false;
    if (sizes[2] && !f.read(&prog.log[0], sizes[2])) return false;
    return true;
}

void cache_store(const std::string &key, const Program &prog)
{
    const std::string path = cache_path(key);
    if (path.empty()) return;
    const std::string tmp = path + ".tmp" + std::to_string(getpid());
    {
        std::ofstream f(tmp, std::ios::binary);
        if (!f) return;
        const uint64_t sizes[3] = {key.size(), prog.cubin.size(), prog.log.size()};
        f.write(reinterpret_cast<const char *>(sizes), sizeof(sizes));
        f.write(key.data(), key.size());
        f.write(prog.cubin.data(), prog.cubin.size());
        f.write(prog.log.data(), prog.log.size());
        if (!f) {
            std::remove(tmp.c_str());
            return;
        }
    }
    std::rename(tmp.c_str(), path.c_str());
}

}  // namespace

std::string print_like_reference(double x)
{
    std::ostringstream ss;
    ss << x;
    return ss.str();
}

namespace {

// The least t >= 0 whose correctly rounded square root (in T, double or float)
// reaches eps, as an exact hexadecimal literal: sqrt(norm) < eps holds exactly
// when norm < t, the root being monotone.  Empty when eps is not positive and
// finite or t is not a normal number (the solvers then keep the root).
template <typename T>
std::string l2_bound_literal(T eps)
{
    if (!(eps > 0) || !std::isfinite(eps)) return "";
    T t = eps * eps;
    if (!std::isfinite(t) || t < std::numeric_limits<T>::min()) return "";
    while (t > 0 && std::sqrt(t) >= eps) t = std::nextafter(t, T(0));
    while (std::sqrt(t) < eps) t = std::nextafter(t, std::numeric_limits<T>::infinity());
    if (!std::isfinite(t) || t < std::numeric_limits<T>::min()) return "";
    char buf[64];
    std::snprintf(buf, sizeof buf, "%a", static_cast<double>(t));
    return std::string(buf) + (sizeof(T) == sizeof(float) ? "f" : "");
}

}  // namespace

std::string l2_bound_define(double newton_tol, bool fp32)
{
    // the tolerance as the program's _epsilon1_ text reads it
    const std::string text = print_like_reference(newton_tol);
    const std::string lit = fp32 ? l2_bound_literal(std::strtof(text.c_str(), nullptr))
                                 : l2_bound_literal(std::strtod(text.c_str(), nullptr));
    return lit.empty() ? std::string() : "#define SODECL_L2_BOUND " + lit + "\n";
}

std::string suffix_float_literals(const std::string &src)
{
    return scan_code(src, suffix_in_code, true);
}

SystemTraits inspect_system(const std::string &src)
{
    const std::string stripped = scan_code(src, [](const std::string &s) { return s; }, false);
    SystemTraits t;
    t.has_system = defines_function(stripped, "sode_system");
    t.has_jacobian = defines_function(stripped, "calc_jacobian");
    t.has_stoch = defines_function(stripped, "sode_system_stoch");
    t.has_pjacobian = defines_function(stripped, "calc_jacobian_params");
    t.has_row = defines_function(stripped, "sode_system_row");
    t.has_stoch_row = defines_function(stripped, "sode_system_stoch_row");
    t.has_jac_band = defines_function(stripped, "calc_jacobian_band");
    t.has_row_band = defines_function(stripped, "sode_system_row_band");
    t.has_vjp = defines_function(stripped, "calc_vjp");
    t.uses_listsize = std::regex_search(stripped, std::regex("\\b_listsize_\\b"));
    return t;
}

int lanes_slot_words(const ProgramSpec &spec)
{
    const int nvec = spec.solver == 2 ? 3 : (spec.solver == 3 || spec.solver == 4) ? 8 : 1;
    return (nvec * spec.num_equat + spec.num_params + spec.num_noi) | 1;
}

std::string assemble(const ProgramSpec &spec, const std::string &system_src, const SystemTraits &traits)
{
    std::ostringstream s;
    s << "// SODECL program generated by libsodecl_cuda (sm_100a)\n";
    s << "#define SODECL_SOLVER " << spec.solver << "\n";
    s << "#define SODECL_FP32 " << (spec.fp32 ? 1 : 0) << "\n";
    s << "#define SODECL_RECORD_F32 " << (spec.record_f32 ? 1 : 0) << "\n";
    s << "#define SODECL_FAST_DIV " << (spec.fast_div ? 1 : 0) << "\n";
    s << "#define SODECL_HAS_JACOBIAN " << (traits.has_jacobian ? 1 : 0) << "\n";
    s << "#define SODECL_HAS_STOCH " << (traits.has_stoch ? 1 : 0) << "\n";
    s << "#define SODECL_NEWTON_MAX " << spec.newton_max_iter << "\n";
    s << "#define SODECL_BLOCK_MAX " << spec.block_max << "\n";
    if (spec.min_blocks > 0) s << "#define SODECL_MIN_BLOCKS " << spec.min_blocks << "\n";
    s << "#define SODECL_LANES " << spec.lanes << "\n";
    if (spec.pair_stores) s << "#define SODECL_PAIR_STORES 1\n";
    s << "#define SODECL_HAS_ROW " << (traits.has_row ? 1 : 0) << "\n";
    s << "#define SODECL_HAS_STOCH_ROW " << (traits.has_stoch_row ? 1 : 0) << "\n";
    s << "#define SODECL_HAS_JAC_BAND " << (traits.has_jac_band ? 1 : 0) << "\n";
    s << "#define SODECL_HAS_ROW_BAND " << (traits.has_row_band ? 1 : 0) << "\n";
    s << kFastDivSrc << "\n" << kPreludeSrc << "\n" << kThreefrySrc << "\n";
    // the reference's program defines (src/sodeclmgr.cpp:379-430); _listsize_
    // only when the system file names it, so one program serves every size
    s << "#define _numnoi_ " << spec.num_noi << "\n";
    if (traits.uses_listsize) s << "#define _listsize_ " << spec.list_size << "\n";
    s << "#define _numsteps_ " << spec.kernel_steps << "\n";
    std::string dt = print_like_reference(spec.dt);
    if (spec.fp32) dt = suffix_in_code(dt);
    s << "#define _m_dt_ " << dt << "\n";
    s << "#define _numeq_ " << spec.num_equat << "\n";
    s << "#define _numpar_ " << spec.num_params << "\n";
    // the Newton bound, printed the same way (src/sodeclmgr.cpp:423-428)
    std::string eps = print_like_reference(spec.newton_tol);
    if (spec.fp32) eps = suffix_in_code(eps);
    s << "#define _epsilon1_ " << eps << "\n";
    s << l2_bound_define(spec.newton_tol, spec.fp32);
    if (spec.solver == 5) {
        char buf[96];
        std::snprintf(buf, sizeof buf, "#define SODECL_RTOL %a\n#define SODECL_ATOL %a\n", spec.rtol, spec.atol);
        s << buf << "#define SODECL_MAX_STEPS " << spec.max_steps << "\n";
    }
    if (spec.fast_div) s << "#define double sodecl_num\n";
    else if (spec.fp32) s << "#define double float\n";
    s << "#line 1 \"system.cl\"\n";
    const std::string user = relax_parameter_bounds(system_src);
    s << (spec.fp32 ? suffix_float_literals(user) : user) << "\n";
    if (spec.fp32 || spec.fast_div) s << "#undef double\n";
    s << "#line 1 \"solvers.cuh\"\n" << kSolversSrc << "\n";
    return s.str();
}

namespace {

std::shared_ptr<const Program> compile_text(std::string source, bool fmad, bool fast_div, const char *kernel)
{
    auto prog = std::make_shared<Program>();
    prog->source = std::move(source);
    prog->fast_div = fast_div;
    prog->kernel_name = kernel;

    std::vector<std::string> opts = {
        "--gpu-architecture=sm_100a",
        "--device-as-default-execution-space",
        "--std=c++17",
        fmad ? "--fmad=true" : "--fmad=false",
        "--generate-line-info",
        "--ptxas-options=-v",
    };
    const std::string key = compile_options_key(opts) + prog->source;
    {
        std::lock_guard<std::mutex> lock(g_cache_mutex);
        auto it = g_cache.find(key);
        if (it != g_cache.end()) return it->second;
    }

    if (cache_load(key, *prog)) {
        std::shared_ptr<const Program> done = prog;
        std::lock_guard<std::mutex> lock(g_cache_mutex);
        g_cache.emplace(key, done);
        return done;
    }

    nvrtcProgram p = nullptr;
    nvrtcResult rc = nvrtcCreateProgram(&p, prog->source.c_str(), "sodecl_program.cu", 0, nullptr, nullptr);
    if (rc != NVRTC_SUCCESS) throw std::runtime_error(std::string("nvrtcCreateProgram: ") + nvrtcGetErrorString(rc));
    std::vector<const char *> argv;
    for (const auto &o : opts) argv.push_back(o.c_str());
    rc = nvrtcCompileProgram(p, static_cast<int>(argv.size()), argv.data());
    size_t log_size = 0;
    nvrtcGetProgramLogSize(p, &log_size);
    if (log_size > 1) {
        prog->log.resize(log_size);
        nvrtcGetProgramLog(p, &prog->log[0]);
        while (!prog->log.empty() && prog->log.back() == '\0') prog->log.pop_back();
    }
    if (rc != NVRTC_SUCCESS) {
        std::string msg = std::string("NVRTC compilation failed: ") + nvrtcGetErrorString(rc) + "\n" + prog->log;
        nvrtcDestroyProgram(&p);
        throw std::runtime_error(msg);
    }
    size_t cubin_size = 0;
    nvrtcGetCUBINSize(p, &cubin_size);
    prog->cubin.resize(cubin_size);
    nvrtcGetCUBIN(p, prog->cubin.data());
    nvrtcDestroyProgram(&p);
    cache_store(key, *prog);

    std::shared_ptr<const Program> done = prog;
    std::lock_guard<std::mutex> lock(g_cache_mutex);
    g_cache.emplace(key, done);
    return done;
}

std::shared_ptr<const Program> compile_one(const ProgramSpec &spec, const std::string &system_src,
                                           const SystemTraits &traits)
{
    return compile_text(assemble(spec, system_src, traits), spec.fmad, spec.fast_div, "sodecl_orbits");
}

// Names of the object-like and function-like macros a source #defines, so a
// batch program can #undef them after each class.
std::vector<std::string> defined_macros(const std::string &src)
{
    std::vector<std::string> names;
    const std::regex def("^[ \\t]*#[ \\t]*define[ \\t]+([A-Za-z_][A-Za-z0-9_]*)");
    const std::string stripped = scan_code(src, [](const std::string &x) { return x; }, false);
    for (std::sregex_iterator it(stripped.begin(), stripped.end(), def), end; it != end; ++it)
        names.push_back((*it)[1].str());
    return names;
}

}  // namespace

int batch_warp_words(const std::vector<BatchClass> &classes)
{
    int words = 0;
    for (const auto &c : classes)
        if (c.spec.lanes > 1) words = std::max(words, (32 / c.spec.lanes) * lanes_slot_words(c.spec));
    return words;
}

namespace {

std::string assemble_batch(const std::vector<BatchClass> &classes, bool fast_div, int block_max, int min_blocks)
{
    std::ostringstream s;
    s << "// SODECL batch program generated by libsodecl_cuda (sm_100a)\n";
    s << "#define SODECL_STEPS_ONLY 1\n#define SODECL_FP32 0\n#define SODECL_RECORD_F32 0\n";
    s << "#define SODECL_FAST_DIV " << (fast_div ? 1 : 0) << "\n";
    s << "#define SODECL_BLOCK_MAX " << block_max << "\n";
    s << "#define SODECL_BATCH_MIN_BLOCKS " << std::max(1, min_blocks) << "\n";
    s << kFastDivSrc << "\n" << kPreludeSrc << "\n" << kThreefrySrc << "\n" << kBatchSrc << "\n";
    static const char *per_class[] = {"SODECL_SOLVER", "SODECL_HAS_JACOBIAN", "SODECL_HAS_STOCH", "SODECL_NEWTON_MAX",
                                      "_numnoi_", "_numsteps_", "_m_dt_", "_numeq_", "_numpar_", "_epsilon1_",
                                      "SODECL_L2_BOUND", "_listsize_", "SODECL_BATCH_CLASS_BODY", "SODECL_LANES",
                                      "SODECL_HAS_ROW", "SODECL_HAS_STOCH_ROW", "SODECL_HAS_JAC_BAND",
                                      "SODECL_HAS_ROW_BAND"};
    for (size_t k = 0; k < classes.size(); ++k) {
        const ProgramSpec &sp = classes[k].spec;
        const std::string &src = classes[k].system_src;
        const SystemTraits tr = inspect_system(src);
        s << "\n// ---- class " << k << "\n";
        for (const char *m : per_class) s << "#undef " << m << "\n";
        s << "#define SODECL_SOLVER " << sp.solver << "\n";
        s << "#define SODECL_HAS_JACOBIAN " << (tr.has_jacobian ? 1 : 0) << "\n";
        s << "#define SODECL_HAS_STOCH " << (tr.has_stoch ? 1 : 0) << "\n";
        s << "#define SODECL_NEWTON_MAX " << sp.newton_max_iter << "\n";
        s << "#define SODECL_LANES " << sp.lanes << "\n";
        s << "#define SODECL_HAS_ROW " << (tr.has_row ? 1 : 0) << "\n";
        s << "#define SODECL_HAS_STOCH_ROW " << (tr.has_stoch_row ? 1 : 0) << "\n";
        s << "#define SODECL_HAS_JAC_BAND " << (tr.has_jac_band ? 1 : 0) << "\n";
        s << "#define SODECL_HAS_ROW_BAND " << (tr.has_row_band ? 1 : 0) << "\n";
        s << "#define _numnoi_ " << sp.num_noi << "\n";
        s << "#define _listsize_ " << sp.list_size << "\n";
        s << "#define _numsteps_ 1\n";
        s << "#define _m_dt_ " << print_like_reference(sp.dt) << "\n";
        s << "#define _numeq_ " << sp.num_equat << "\n";
        s << "#define _numpar_ " << sp.num_params << "\n";
        s << "#define _epsilon1_ " << print_like_reference(sp.newton_tol) << "\n";
        s << l2_bound_define(sp.newton_tol, false);
        s << "namespace sodecl_cls_" << k << " {\n";
        if (fast_div) s << "#define double sodecl_num\n";
        s << "#line 1 \"class" << k << ".cl\"\n" << relax_parameter_bounds(src) << "\n";
        if (fast_div) s << "#undef double\n";
        for (const auto &m : defined_macros(src)) s << "#undef " << m << "\n";
        s << "#line 1 \"solvers.cuh\"\n" << kSolversSrc << "\n";
        s << "#define SODECL_BATCH_CLASS_BODY 1\n#line 1 \"batch.cuh\"\n" << kBatchSrc << "\n";
        s << "}  // namespace sodecl_cls_" << k << "\n";
    }
    const int warp_words = batch_warp_words(classes);
    s << "\n#define SODECL_BATCH_WARP_WORDS " << warp_words << "\n";
    s << "extern \"C\" __global__ void __launch_bounds__(SODECL_BLOCK_MAX, SODECL_BATCH_MIN_BLOCKS) "
         "sodecl_batch(const sodecl_batch_args a)\n{\n";
    if (warp_words > 0) {
        s << "    extern __shared__ __align__(16) unsigned char sodecl_smem[];\n";
        s << "    double *warp_smem = reinterpret_cast<double *>(sodecl_smem) + (threadIdx.x / 32) * "
             "SODECL_BATCH_WARP_WORDS;\n";
    } else {
        s << "    double *warp_smem = nullptr;\n";
    }
    s << "    for (int k = 0; k < a.nclasses; ++k) {\n        switch (a.order[k]) {\n";
    for (size_t k = 0; k < classes.size(); ++k)
        s << "        case " << k << ": sodecl_cls_" << k << "::sodecl_class_run(a, " << k << ", warp_smem); break;\n";
    s << "        default: break;\n        }\n        __syncwarp();\n    }\n}\n";
    return s.str();
}

std::string assemble_adjoint(const ProgramSpec &spec, const std::string &src, int tape_cap, int mode,
                             bool fast_div, bool gradient)
{
    const SystemTraits tr = inspect_system(src);
    std::ostringstream s;
    s << "// SODECL adjoint program generated by libsodecl_cuda (sm_100a)\n";
    s << "#define SODECL_STEPS_ONLY 1\n#define SODECL_FP32 0\n#define SODECL_RECORD_F32 0\n";
    s << "#define SODECL_FAST_DIV " << (fast_div ? 1 : 0) << "\n";
    s << "#define SODECL_SOLVER " << spec.solver << "\n";
    s << "#define SODECL_HAS_JACOBIAN " << (tr.has_jacobian ? 1 : 0) << "\n";
    s << "#define SODECL_HAS_STOCH " << (tr.has_stoch ? 1 : 0) << "\n";
    s << "#define SODECL_NEWTON_MAX " << spec.newton_max_iter << "\n";
    s << "#define SODECL_BLOCK_MAX " << spec.block_max << "\n";
    if (spec.min_blocks > 0) s << "#define SODECL_MIN_BLOCKS " << spec.min_blocks << "\n";
    s << "#define SODECL_TAPE_CAP " << tape_cap << "\n";
    s << "#define SODECL_ADJ_MODE " << mode << "\n";
    s << "#define SODECL_ADJ_GRADIENT " << (gradient ? 1 : 0) << "\n";
    s << kFastDivSrc << "\n" << kPreludeSrc << "\n" << kThreefrySrc << "\n" << kAdjointSrc << "\n";
    s << "#define _numnoi_ " << spec.num_noi << "\n";
    s << "#define _listsize_ " << spec.list_size << "\n";
    s << "#define _numsteps_ " << spec.kernel_steps << "\n";
    s << "#define _m_dt_ " << print_like_reference(spec.dt) << "\n";
    s << "#define _numeq_ " << spec.num_equat << "\n";
    s << "#define _numpar_ " << spec.num_params << "\n";
    s << "#define _epsilon1_ " << print_like_reference(spec.newton_tol) << "\n";
    s << l2_bound_define(spec.newton_tol, false);
    const std::string user = relax_parameter_bounds(src);
    const std::vector<std::string> macros = defined_macros(src);
    if (fast_div) s << "#define double sodecl_num\n";
    s << "#line 1 \"system.cl\"\n" << user << "\n";
    if (fast_div) s << "#undef double\n";
    for (const auto &m : macros) s << "#undef " << m << "\n";
    // the recording copy: every double of the system file is a sodecl_ad
    s << "namespace sodecl_adsys {\n#define double sodecl_ad\n#line 1 \"system.cl\"\n" << user
      << "\n#undef double\n}  // namespace sodecl_adsys\n";
    for (const auto &m : macros) s << "#undef " << m << "\n";
    s << "#line 1 \"solvers.cuh\"\n" << kSolversSrc << "\n";
    s << "#define SODECL_ADJOINT_KERNEL 1\n#line 1 \"adjoint.cuh\"\n" << kAdjointSrc << "\n";
    return s.str();
}

}  // namespace

std::shared_ptr<const Program> build_adjoint(const ProgramSpec &spec, const std::string &system_src, int tape_cap,
                                             int mode, bool gradient)
{
    // the reciprocal quotients only where the system file is plain arithmetic
    if (spec.fast_div && system_src.find("printf") == std::string::npos) {
        try {
            return compile_text(assemble_adjoint(spec, system_src, tape_cap, mode, true, gradient), spec.fmad, true,
                                "sodecl_adjoint");
        } catch (const std::exception &) {
        }
    }
    return compile_text(assemble_adjoint(spec, system_src, tape_cap, mode, false, gradient), spec.fmad, false,
                        "sodecl_adjoint");
}

std::shared_ptr<const Program> build_batch(const std::vector<BatchClass> &classes, bool fmad, bool fast_div,
                                           int block_max, int min_blocks)
{
    if (classes.empty()) throw std::runtime_error("a batch needs at least one class");
    bool fd = fast_div;
    for (const auto &c : classes)
        if (c.system_src.find("printf") != std::string::npos) fd = false;
    if (fd) {
        try {
            return compile_text(assemble_batch(classes, true, block_max, min_blocks), fmad, true, "sodecl_batch");
        } catch (const std::exception &) {
        }
    }
    return compile_text(assemble_batch(classes, false, block_max, min_blocks), fmad, false, "sodecl_batch");
}

std::shared_ptr<const Program> build(const ProgramSpec &spec, const std::string &system_src)
{
    const SystemTraits traits = inspect_system(system_src);
    ProgramSpec s = spec;
    // the wrapper type would hand a struct to printf's varargs
    if (s.fast_div && system_src.find("printf") != std::string::npos) s.fast_div = false;
    if (!s.fast_div) return compile_one(s, system_src, traits);
    try {
        return compile_one(s, system_src, traits);
    } catch (const std::exception &) {
        // the system file needs plain `double` (an implicit conversion, say)
        s.fast_div = false;
        return compile_one(s, system_src, traits);
    }
}

}  // namespace sodecl_b200
