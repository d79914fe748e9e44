// single_dev_expt_main — drop-in replacement for the reference's CLI driver
// (src/single_dev_expt_main.cpp + Simulator::Data::Data / Simulator::run of
// src/simulator/single_dev_expt/simulator_expt_platform.cu), written as host
// C++ over the C ABI of include/culbm.h.
//
// Same flags, defaults, vector syntax ([a,b,c], a,b,c or three values), stdout
// lines ("Init ... successfully", "speed = X (MLUPS)"), dump files
// <dumpFolder>/<field>_<step>.dat and exit codes (0; 1 with the message on
// stderr for a runtime failure; the CLI11 parse-error codes for bad argv).
// Additions: --storage fp32|fp16|bf16|fp64, --persistL2 (--noPersistL2, the
// default, is accepted), --noCacheHints, --noGraphs.
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "culbm.h"

namespace {

// Exit codes of CLI11 2.x (CLI::ExitCodes), which the reference's parser
// returns through app.exit(e) (simulator_expt_platform.cu:356-363).
constexpr int kConversionError = 104;
constexpr int kExtrasError = 109;
constexpr int kArgumentMismatch = 114;

struct ParseError {
    int code;
    std::string msg;
};

struct Options {
    culbm_config cfg{};
    uint32_t dstep = 100;
    uint32_t nstep = 1000;
    std::string init_folder;
    std::string dump_folder = "data/left_inlet_right_outlet_256_256_256_output";
    bool dump[4] = {false, false, false, false};
    bool help = false;
    bool auto_block = false;   // --blockDim auto
};

void usage(std::ostream& os)
{
    os << "Single Device Expt Fluid Solver\n"
          "Usage: single_dev_expt_main [OPTIONS]\n\n"
          "Options:\n"
          "  -h,--help                 Print this help message and exit\n"
          "  --devId INT [0]           Device index of the GPU\n"
          "  --dstep UINT [100]        Delta time steps of the simulation.\n"
          "  --nstep UINT [1000]       Total time steps of the simulation.\n"
          "  --invTau FLOAT [0.5]      Reciprocal of Tau.\n"
          "  --blockDim UINT x 3 [[32,16,2]]   Dimension of blocks per grid; `auto`: the whole domain\n"
          "                            without blocking, else the tile and innerLoop of the largest\n"
          "                            modelled speed-up (culbm_select_tile).\n"
          "  --gridDim UINT x 3 [[2,3,19]]     Dimension of grids per kernel.\n"
          "  --domainDim UINT x 3 [[256,256,256]] Dimension of the domain.\n"
          "  --streamPolicy INT [0]    {[0]:PULL_STREAM, [1]:INPLACE_STREAM}.\n"
          "  --optPolicy INT [0]       {[0]:NONE, [1]:HALO_BLOCKING_STATIC_L2, [2]:HALO_BLOCKING_L1L2, "
          "[3]:HALO_BLOCKING_DYNAMIC_L2}.\n"
          "  --velSet INT [0]          The velocity set of the solver ([0]:D3Q27).\n"
          "  --initStateFolder TEXT    The folder contains initial state of the simulation.\n"
          "  --dumpFolder TEXT [data/left_inlet_right_outlet_256_256_256_output]\n"
          "                            The folder contains final output.\n"
          "  --dumpRho, --dumpVx, --dumpVy, --dumpVz\n"
          "                            Dump the field every `dstep` time steps.\n"
          "  --useRingDDFBuf           One global DDF ring buffer for in-place dynamic L2 blocking.\n"
          "  --innerLoop INT [5]       # of iterations in halo-blocking.\n"
          "  --storage TEXT [fp32]     Population storage: fp32, fp16, bf16, fp64, fp16sr or bf16sr.\n"
          "  --persistL2               Persisting-L2 window over tile buffers (off by default: slower on B200).\n"
          "  --noPersistL2             No persisting-L2 window (the default).\n"
          "  --noCacheHints            No evict-first/evict-last cache hints.\n"
          "  --noGraphs                Launch tile sequences directly instead of CUDA graphs.\n";
}

long long parse_int(const std::string& opt, const std::string& s, long long lo, long long hi)
{
    if (s.empty()) throw ParseError{kConversionError, "Could not convert: " + opt + " = " + s};
    char* end = nullptr;
    errno = 0;
    const long long v = std::strtoll(s.c_str(), &end, 10);
    if (*end != '\0' || errno != 0 || v < lo || v > hi)
        throw ParseError{kConversionError, "Could not convert: " + opt + " = " + s};
    return v;
}

float parse_float(const std::string& opt, const std::string& s)
{
    char* end = nullptr;
    const float v = std::strtof(s.c_str(), &end);
    if (s.empty() || *end != '\0' || !std::isfinite(v))
        throw ParseError{kConversionError, "Could not convert: " + opt + " = " + s};
    return v;
}

// Collects the values of a 3-vector option: "[a,b,c]", "a,b,c" or "a b c".
void parse_vec3(const std::string& opt, std::vector<std::string>& args, size_t& k, const std::string* inline_val,
                uint32_t out[3])
{
    std::vector<std::string> toks;
    auto split = [&](std::string s) {
        std::string cur;
        for (char ch : s) {
            if (ch == '[' || ch == ']' || ch == ' ') continue;
            if (ch == ',') {
                toks.push_back(cur);
                cur.clear();
            } else {
                cur += ch;
            }
        }
        if (!cur.empty()) toks.push_back(cur);
    };
    if (inline_val) {
        split(*inline_val);
    } else {
        while (k + 1 < args.size() && toks.size() < 3 && args[k + 1].rfind("--", 0) != 0) split(args[++k]);
    }
    if (toks.size() != 3)
        throw ParseError{kArgumentMismatch, opt + ": 3 required UINT:UINT in [0 - 4294967295] missing"};
    for (int j = 0; j < 3; ++j) out[j] = static_cast<uint32_t>(parse_int(opt, toks[j], 0, 4294967295ll));
}

Options parse(int argc, char** argv)
{
    Options o;
    culbm_config_init(&o.cfg);
    std::vector<std::string> args(argv + 1, argv + argc);
    for (size_t k = 0; k < args.size(); ++k) {
        std::string a = args[k];
        std::string name = a, val;
        bool has_inline = false;
        const size_t eq = a.find('=');
        if (a.rfind("--", 0) == 0 && eq != std::string::npos) {
            name = a.substr(0, eq);
            val = a.substr(eq + 1);
            has_inline = true;
        }
        auto value = [&]() -> std::string {
            if (has_inline) return val;
            if (k + 1 >= args.size()) throw ParseError{kArgumentMismatch, name + ": 1 required argument missing"};
            return args[++k];
        };
        auto flag = [&]() {
            if (has_inline) throw ParseError{kArgumentMismatch, name + ": flag takes no value"};
        };
        if (name == "-h" || name == "--help") {
            o.help = true;
        } else if (name == "--devId") {
            o.cfg.dev_id = static_cast<int32_t>(parse_int(name, value(), -2147483648ll, 2147483647ll));
        } else if (name == "--dstep") {
            o.dstep = static_cast<uint32_t>(parse_int(name, value(), 0, 4294967295ll));
        } else if (name == "--nstep") {
            o.nstep = static_cast<uint32_t>(parse_int(name, value(), 0, 4294967295ll));
        } else if (name == "--invTau") {
            o.cfg.inv_tau = parse_float(name, value());
        } else if (name == "--blockDim") {
            const std::string next = has_inline ? val : (k + 1 < args.size() ? args[k + 1] : std::string());
            if (next == "auto") {
                if (!has_inline) ++k;
                o.auto_block = true;
            } else {
                parse_vec3(name, args, k, has_inline ? &val : nullptr, o.cfg.block_dim);
            }
        } else if (name == "--gridDim") {
            parse_vec3(name, args, k, has_inline ? &val : nullptr, o.cfg.grid_dim);
        } else if (name == "--domainDim") {
            parse_vec3(name, args, k, has_inline ? &val : nullptr, o.cfg.domain_dim);
        } else if (name == "--streamPolicy") {
            o.cfg.stream_policy = static_cast<int32_t>(parse_int(name, value(), -2147483648ll, 2147483647ll));
        } else if (name == "--optPolicy") {
            o.cfg.opt_policy = static_cast<int32_t>(parse_int(name, value(), -2147483648ll, 2147483647ll));
        } else if (name == "--velSet") {
            o.cfg.vel_set = static_cast<int32_t>(parse_int(name, value(), -2147483648ll, 2147483647ll));
        } else if (name == "--initStateFolder") {
            o.init_folder = value();
        } else if (name == "--dumpFolder") {
            o.dump_folder = value();
        } else if (name == "--dumpRho") {
            flag();
            o.dump[0] = true;
        } else if (name == "--dumpVx") {
            flag();
            o.dump[1] = true;
        } else if (name == "--dumpVy") {
            flag();
            o.dump[2] = true;
        } else if (name == "--dumpVz") {
            flag();
            o.dump[3] = true;
        } else if (name == "--useRingDDFBuf") {
            flag();
            o.cfg.use_ring_ddf_buf = 1;
        } else if (name == "--innerLoop") {
            o.cfg.inner_loop = static_cast<int32_t>(parse_int(name, value(), -2147483648ll, 2147483647ll));
        } else if (name == "--storage") {
            const std::string v = value();
            if (v == "fp32") o.cfg.storage = CULBM_STORAGE_F32;
            else if (v == "fp16") o.cfg.storage = CULBM_STORAGE_F16;
            else if (v == "bf16") o.cfg.storage = CULBM_STORAGE_BF16;
            else if (v == "fp64") o.cfg.storage = CULBM_STORAGE_F64;
            else if (v == "fp16sr") o.cfg.storage = CULBM_STORAGE_F16_SR;
            else if (v == "bf16sr") o.cfg.storage = CULBM_STORAGE_BF16_SR;
            else throw ParseError{kConversionError, "Could not convert: --storage = " + v};
        } else if (name == "--noPersistL2") {
            flag();
            o.cfg.persist_l2 = 0;
        } else if (name == "--persistL2") {
            flag();
            o.cfg.persist_l2 = 1;
        } else if (name == "--noCacheHints") {
            flag();
            o.cfg.cache_hints = 0;
        } else if (name == "--noGraphs") {
            flag();
            o.cfg.use_graphs = 0;
        } else {
            throw ParseError{kExtrasError, "The following arguments were not expected: " + a};
        }
    }
    return o;
}

void check(culbm_status s)
{
    if (s != CULBM_OK) throw std::runtime_error(std::string(culbm_status_string(s)) + ": " + culbm_last_error());
}

std::string fmt_default(float v)
{
    char buf[32];
    std::snprintf(buf, sizeof(buf), "%g", v);
    return buf;
}

int run(Options o)
{
    if (o.auto_block) {
        if (o.cfg.opt_policy == CULBM_OPT_NONE) {
            for (int k = 0; k < 3; ++k) {
                o.cfg.block_dim[k] = o.cfg.domain_dim[k];
                o.cfg.grid_dim[k] = 1;
            }
        } else {
            culbm_tile_choice t;
            check(culbm_select_tile(o.cfg.domain_dim, o.cfg.storage, 0.0, 0.0, 0, 0, &t));
            for (int k = 0; k < 3; ++k) {
                o.cfg.block_dim[k] = t.tile[k];
                o.cfg.grid_dim[k] = 1;
            }
            o.cfg.inner_loop = t.inner_loop;
            std::cout << "Auto tile: blockDim [" << t.tile[0] << "," << t.tile[1] << "," << t.tile[2]
                      << "] gridDim [1,1,1] innerLoop " << t.inner_loop << " (modelled speed-up "
                      << t.predicted_speedup << " over plain streaming, " << t.predicted_speedup_b200
                      << " with B200's measured step costs)" << std::endl;
        }
    }
    if (o.dstep == 0) throw std::invalid_argument("--dstep must be positive");
    culbm_sim* sim = nullptr;
    check(culbm_create(&o.cfg, &sim));
    struct Guard {
        culbm_sim* s;
        ~Guard() { culbm_destroy(s); }
    } guard{sim};

    const bool blocked = o.cfg.opt_policy != CULBM_OPT_NONE;
    uint32_t mask = 0;
    check(culbm_load_state_folder(sim, o.init_folder.c_str(), &mask));
    if (!o.init_folder.empty() || blocked)
        std::cout << "Init flag successfully, from file: " << o.init_folder << "/flag.dat." << std::endl;
    const char* names[4] = {"rho", "vx", "vy", "vz"};
    const float dflt[4] = {1.0f, 0.0f, 0.0f, 0.0f};
    for (int k = 0; k < 4; ++k) {
        if (mask & (1u << (k + 1)))
            std::cout << "Init " << names[k] << " successfully, from file: " << o.init_folder << "/" << names[k]
                      << ".dat." << std::endl;
        else
            std::cout << "Init " << names[k] << " successfully, default init with value " << fmt_default(dflt[k])
                      << "." << std::endl;
    }
    std::cout << (o.cfg.use_ring_ddf_buf ? "Init ring ddf buffer successfully." : "Init double ddf buffer successfully.")
              << std::endl;

    // Steps per dump period: blocked policies advance whole innerLoop rounds,
    // like the reference's `locStep += innerLoop` loops (simulator_expt_platform.cu:785).
    uint32_t chunk = o.dstep;
    if (blocked) {
        const uint32_t I = static_cast<uint32_t>(o.cfg.inner_loop);
        chunk = (o.dstep + I - 1) / I * I;
    }
    const uint32_t field_mask = (o.dump[0] ? 1u : 0u) | (o.dump[1] ? 2u : 0u) | (o.dump[2] ? 4u : 0u) |
                                (o.dump[3] ? 8u : 0u);
    uint64_t step = 0;
    while (step < o.nstep) {
        float ms = 0.0f;
        check(culbm_step_timed(sim, chunk, &ms));
        const uint32_t cells = o.cfg.domain_dim[0] * o.cfg.domain_dim[1] * o.cfg.domain_dim[2];
        const float mlups = static_cast<float>(cells) * 1e-6f / (ms / 1000) * static_cast<float>(chunk);
        char line[64];
        std::snprintf(line, sizeof(line), "speed = %.4f (MLUPS)", mlups);
        std::cout << line << std::endl;
        step += chunk;
        check(culbm_moments(sim));
        check(culbm_dump(sim, o.dump_folder.c_str(), field_mask));
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv)
{
    Options o;
    try {
        o = parse(argc, argv);
    } catch (const ParseError& e) {
        std::cerr << e.msg << "\nRun with --help for more information." << std::endl;
        return e.code;
    }
    if (o.help) {
        usage(std::cout);
        return 0;
    }
    try {
        return run(o);
    } catch (const std::exception& e) {
        std::cerr << e.what() << std::endl;
        return 1;
    }
}
