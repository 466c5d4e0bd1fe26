// nutcracker_b200: the reference's command-line program (programs/nutcracker,
// sources/programs/nutcracker.cpp:178-256; options of configuration.cpp:11-180)
// on the B200 library.
//
// Reads an operator in the YAML format (file or standard input, optionally at
// a location inside the document), solves for the requested number of levels
// (Chain::solveForMultipleLevels: optimizeChain per level, each converged
// level becoming a projector) and writes the YAML result
// (yaml.cpp:106-143):
//
//   Configuration:
//     site convergence tolerance: 1e-12
//     ...
//   Energy levels:
//     - -10.022510957077
//
// one energy per level as soon as it is found, with ceil(-log10(chain
// tolerance)) significant digits.  Options come from the command line and
// from `nutcracker.cfg` (or --config-file) lines "name = value"; the command
// line wins.  As in the reference, option errors exit with status 255 and
// the format errors of main() print their message and exit 255, while other
// failures print their message and exit 0 (nutcracker.cpp:253-256).
//
// B200 additions: --precision 1 (3xTF32 tensor-core sweeps closed by FP64
// refinement), --seed, --initial-bandwidth (first chi of optimizeChain's
// growth schedule).
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "nutcracker_b200.h"

namespace {

struct OptionError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct FormatError : std::runtime_error {   // caught by main with exit status 255
    using std::runtime_error::runtime_error;
};

struct OptionSpec {
    const char* name;
    char shortcut;
    bool flag;
    const char* help;
};

const OptionSpec kOptions[] = {
    {"help", 0, true, "print help message and exit"},
    {"help-formats", 0, true, "print the supported input and output formats and exit"},
    {"help-modes", 0, true, "print the supported optimizer modes"},
    {"config-file", 'C', false, "configuration file (default: nutcracker.cfg)"},
    {"number-of-levels", 'n', false, "number of energy levels to find, including the ground state (default 1)"},
    {"optimizer-mode", 0, false, "'<v' least value (default), '>v' greatest value, '>m' largest magnitude"},
    {"input-file", 'f', false, "file with the hamiltonian (default: standard input)"},
    {"input-format", 0, false, "format of the input (default: from the file extension, else yaml)"},
    {"input-location", 0, false, "slash-separated location of the hamiltonian inside the input document"},
    {"output-file", 'o', false, "file for the results (default: standard output)"},
    {"output-format", 0, false, "format of the output (default: from the file extension, else yaml)"},
    {"output-location", 0, false, "location of the results inside the output file"},
    {"output-states", 0, true, "also output the states"},
    {"output-overwrite", 0, true, "overwrite an existing output file"},
    {"site-tolerance", 0, false, "site convergence tolerance"},
    {"sweep-tolerance", 0, false, "sweep convergence tolerance"},
    {"chain-tolerance", 0, false, "chain convergence tolerance"},
    {"sanity-tolerance", 0, false, "sanity check tolerance"},
    {"precision", 0, false, "0: FP64 sweeps (default); 1: 3xTF32 tensor-core sweeps closed by FP64 refinement"},
    {"seed", 0, false, "seed of the random initial states"},
    {"initial-bandwidth", 0, false, "initial bond dimension of the chain"},
};

const OptionSpec* find_option(const std::string& name) {
    for (const OptionSpec& o : kOptions)
        if (name == o.name) return &o;
    return nullptr;
}
const OptionSpec* find_short(char c) {
    for (const OptionSpec& o : kOptions)
        if (o.shortcut && o.shortcut == c) return &o;
    return nullptr;
}

std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

// The first value stored for an option wins (boost::program_options::store):
// the command line is stored before the configuration file.
using Values = std::map<std::string, std::string>;

void store(Values& v, const OptionSpec* o, const std::string& value) {
    if (v.count(o->name)) return;
    v[o->name] = value;
}

void parse_command_line(int argc, char** argv, Values& v) {
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        const OptionSpec* o = nullptr;
        std::string value;
        bool has_value = false;
        if (a.rfind("--", 0) == 0) {
            std::string name = a.substr(2);
            const size_t eq = name.find('=');
            if (eq != std::string::npos) {
                value = name.substr(eq + 1);
                name = name.substr(0, eq);
                has_value = true;
            }
            o = find_option(name);
            if (!o) throw OptionError("unrecognised option '--" + name + "'");
        } else if (a.size() >= 2 && a[0] == '-' && a[1] != '-') {
            o = find_short(a[1]);
            if (!o) throw OptionError(std::string("unrecognised option '-") + a[1] + "'");
            if (a.size() > 2) {
                value = a.substr(2);
                has_value = true;
            }
        } else {
            throw OptionError("unexpected argument '" + a + "'");
        }
        if (o->flag) {
            store(v, o, has_value ? value : "true");
            continue;
        }
        if (!has_value) {
            if (i + 1 >= argc) throw OptionError(std::string("the required argument for option '--") + o->name +
                                                 "' is missing");
            value = argv[++i];
        }
        store(v, o, value);
    }
}

void parse_config_file(const std::string& path, Values& v) {
    std::ifstream in(path);
    if (!in) return;   // a missing configuration file is not an error (nutcracker.cpp:190-198)
    std::string line;
    while (std::getline(in, line)) {
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        line = trim(line);
        if (line.empty()) continue;
        const size_t eq = line.find('=');
        if (eq == std::string::npos) throw OptionError("the configuration line '" + line + "' is not 'name = value'");
        const std::string name = trim(line.substr(0, eq));
        const OptionSpec* o = find_option(name);
        if (!o) throw OptionError("unrecognised option '" + name + "' in the configuration file");
        store(v, o, trim(line.substr(eq + 1)));
    }
}

double to_double(const Values& v, const char* name) {
    const std::string& s = v.at(name);
    char* end = nullptr;
    const double x = std::strtod(s.c_str(), &end);
    if (end == s.c_str() || *end) throw OptionError(std::string("the argument ('") + s + "') for option '--" +
                                                     name + "' is invalid");
    return x;
}

// An unsigned option value no larger than `max` (the 32-bit options of the
// reference by default); anything else is invalid, as a failed conversion is.
unsigned long long to_unsigned(const Values& v, const char* name, unsigned long long max = UINT32_MAX) {
    const std::string& s = v.at(name);
    char* end = nullptr;
    errno = 0;
    const unsigned long long x = std::strtoull(s.c_str(), &end, 10);
    if (end == s.c_str() || *end || s[0] == '-' || errno == ERANGE || x > max)
        throw OptionError(std::string("the argument ('") + s + "') for option '--" + name + "' is invalid");
    return x;
}

bool to_flag(const Values& v, const char* name) {
    auto it = v.find(name);
    if (it == v.end()) return false;
    return it->second == "true" || it->second == "1" || it->second == "yes" || it->second == "on";
}

}  // namespace

namespace {

void print_help_and_exit() {
    std::cerr << "All options:\n";
    for (const OptionSpec& o : kOptions) {
        std::string head = std::string("  --") + o.name;
        if (o.shortcut) head += std::string(" [ -") + o.shortcut + " ]";
        if (!o.flag) head += " arg";
        std::cerr << std::left << std::setw(40) << head << o.help << "\n";
    }
    std::cerr << "\nOptions may also be specified in 'nutcracker.cfg' (or in an alternative configuration file "
                 "specified via --config-file) in the format option=value.  For example, the line\n\n"
                 "\tsite-tolerance = 1e-10\n\nis equivalence to specifying --site-tolerance 1e-10 on the command "
                 "line.\n";
    std::exit(1);
}

void print_formats_and_exit() {
    std::cerr << "The recognized input format types are:\n  - protobuf: Google Protocol Buffers format\n"
                 "  - yaml: YAML format\n\n"
                 "The recognized output format types are:\n  - protobuf: Google Protocol Buffers format\n"
                 "  - yaml: YAML format\n\n";
    std::exit(1);
}

void print_modes_and_exit() {
    std::cerr << "The recognized optimizer modes are:\n  '<v' - least value\n  '>m' - largest magnitude\n"
                 "  '>v' - greatest value\n\n";
    std::exit(1);
}

// resolveAndCheckFormat (io.hpp:389-418) over the two formats (yaml.cpp:145-148,
// protobuf.cpp:191-194): both read and write pipes, the named format wins,
// else the file extension (.yaml, .prb), else yaml; only the YAML input
// supports locations.
std::string resolve_format(const Values& v, const char* type, const char* format_key, const char* file_key,
                           const char* location_key) {
    std::string format = "yaml";
    auto f = v.find(format_key);
    if (f != v.end()) {
        if (f->second != "yaml" && f->second != "protobuf")
            throw FormatError(f->second + " is not a recognized/supported " + type + " format type.\n\nThe "
                              "recognized " + type + " format types are:\n  - protobuf\n  - yaml\n\nRun Nutcracker "
                              "with the --help-formats option for more informaton about supported formats.");
        format = f->second;
    } else if (v.count(file_key)) {
        const std::string& name = v.at(file_key);
        const size_t dot = name.rfind('.'), slash = name.rfind('/');
        if (dot != std::string::npos && (slash == std::string::npos || dot > slash) && name.substr(dot + 1) == "prb")
            format = "protobuf";
    }
    const bool locations = std::string(type) == "input" && format == "yaml";
    if (v.count(location_key) && !locations)
        throw FormatError("The " + std::string(type) + " format type " + format + " does not support locations.");
    return format;
}

std::string read_all(std::istream& in) {
    std::ostringstream ss;
    ss << in.rdbuf();
    return ss.str();
}

struct Library {
    [[noreturn]] static void fail() { throw std::runtime_error(nc_last_error()); }
};

unsigned digits_of_precision(double tolerance) {   // utilities.cpp:92-95
    const double estimated = std::ceil(-std::log10(tolerance));
    return estimated > 0 ? (unsigned)estimated : 1;
}

// ---- protobuf output: SimulationResultsBuffer of nutcracker.proto ----
void pb_varint(std::string& o, uint64_t v) {
    while (v >= 0x80) {
        o.push_back((char)(v | 0x80));
        v >>= 7;
    }
    o.push_back((char)v);
}
void pb_uint(std::string& o, unsigned field, uint64_t v) {
    pb_varint(o, (uint64_t)field << 3);
    pb_varint(o, v);
}
void pb_double(std::string& o, unsigned field, double x) {
    pb_varint(o, ((uint64_t)field << 3) | 1);
    char b[8];
    std::memcpy(b, &x, 8);
    o.append(b, 8);
}
void pb_bytes(std::string& o, unsigned field, const std::string& b) {
    pb_varint(o, ((uint64_t)field << 3) | 2);
    pb_varint(o, b.size());
    o += b;
}

// StateBuffer of the chain's state with its centre on site 0 (protobuf.cpp:86-104).
std::string state_buffer(nc_chain* chain, uint32_t n) {
    if (nc_chain_move_to(chain, 0) != 0) Library::fail();
    std::string out;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t dims[3];
        if (nc_chain_get_site(chain, i, nullptr, dims) != 0) Library::fail();
        std::vector<nc_complex> w((size_t)dims[0] * dims[1] * dims[2]);
        if (nc_chain_get_site(chain, i, w.data(), dims) != 0) Library::fail();
        std::string m;
        pb_uint(m, 1, i == 0 ? 0 : 2);   // MIDDLE, then RIGHT
        pb_uint(m, 2, dims[2]);
        pb_uint(m, 3, dims[1]);
        pb_uint(m, 4, dims[0]);
        pb_bytes(m, 5, std::string(reinterpret_cast<const char*>(w.data()), w.size() * sizeof(nc_complex)));
        pb_bytes(out, 1, m);
    }
    return out;
}

int run(const Values& v) {
    const std::string in_format = resolve_format(v, "input", "input-format", "input-file", "input-location");
    const std::string out_format = resolve_format(v, "output", "output-format", "output-file", "output-location");
    if (to_flag(v, "output-states") && out_format == "yaml")
        throw FormatError("Output format yaml does not support outputing states.");

    nc_chain_options o;
    nc_chain_options_init(&o);
    if (v.count("site-tolerance")) o.site_convergence_threshold = to_double(v, "site-tolerance");
    if (v.count("sweep-tolerance")) o.sweep_convergence_threshold = to_double(v, "sweep-tolerance");
    if (v.count("chain-tolerance")) o.chain_convergence_threshold = to_double(v, "chain-tolerance");
    if (v.count("sanity-tolerance")) o.sanity_check_threshold = to_double(v, "sanity-tolerance");
    if (v.count("precision")) o.precision = (uint32_t)to_unsigned(v, "precision");
    if (v.count("seed")) o.seed = to_unsigned(v, "seed", UINT64_MAX);
    if (v.count("initial-bandwidth")) o.initial_bandwidth_dimension = (uint32_t)to_unsigned(v, "initial-bandwidth");
    const std::string mode = v.count("optimizer-mode") ? v.at("optimizer-mode") : std::string("<v");
    std::snprintf(o.optimizer_mode, sizeof o.optimizer_mode, "%s", mode.c_str());
    const unsigned levels = v.count("number-of-levels") ? (unsigned)to_unsigned(v, "number-of-levels") : 1u;

    // the operator
    std::string text;
    if (v.count("input-file")) {
        std::ifstream in(v.at("input-file"), std::ios::binary);
        if (!in) throw std::runtime_error("cannot open the input file " + v.at("input-file"));
        text = read_all(in);
    } else {
        text = read_all(std::cin);
    }
    nc_parsed_operator* op;
    if (in_format == "protobuf") {
        op = nc_protobuf_read_operator(text.data(), text.size());
    } else {
        const char* location = v.count("input-location") ? v.at("input-location").c_str() : nullptr;
        op = nc_yaml_read_operator(text.data(), text.size(), location);
    }
    if (!op) Library::fail();
    const uint32_t n_sites = nc_parsed_operator_number_of_sites(op);
    nc_chain* chain = nc_chain_create(n_sites, nc_parsed_operator_sites(op), &o);
    nc_parsed_operator_free(op);
    if (!chain) Library::fail();
    std::unique_ptr<nc_chain, void (*)(nc_chain*)> guard(chain, nc_chain_free);

    // the outputters (yaml.cpp:106-143; protobuf.cpp:132-170, which checks no
    // existing file and writes everything at the end)
    const bool yaml = out_format == "yaml";
    std::ofstream file;
    if (v.count("output-file")) {
        const std::string& name = v.at("output-file");
        if (yaml && !to_flag(v, "output-overwrite") && std::ifstream(name).good())
            throw std::runtime_error("The output filename " + name + " already exists.");
        file.open(name, std::ios::binary);
        if (!file) throw std::runtime_error("cannot open the output file " + name);
    }
    std::ostream& out = v.count("output-file") ? static_cast<std::ostream&>(file) : std::cout;
    if (yaml) {
        out << "Configuration:\n"
            << "  site convergence tolerance: " << o.site_convergence_threshold << "\n"
            << "  sweep convergence tolerance: " << o.sweep_convergence_threshold << "\n"
            << "  chain convergence tolerance: " << o.chain_convergence_threshold << "\n"
            << "  sanity check threshold: " << o.sanity_check_threshold << "\n"
            << "Energy levels:\n";
        out.flush();
    }
    const unsigned digits = digits_of_precision(o.chain_convergence_threshold);
    std::string results;

    // solveForMultipleLevels (chain.cpp:301-310), one result per optimised level
    for (unsigned k = 0; k < levels; ++k) {
        if (k > 0 && (nc_chain_construct_and_add_projector_from_state(chain) != 0 || nc_chain_reset(chain) != 0))
            Library::fail();
        double e = 0;
        if (nc_chain_optimize_chain(chain) != 0 || nc_chain_get_energy(chain, &e) != 0) Library::fail();
        if (yaml) {
            out << "  - " << std::setprecision(digits) << e << "\n";
            out.flush();
        } else {
            std::string solution;
            pb_double(solution, 1, e);
            pb_bytes(solution, 2, state_buffer(chain, n_sites));   // states are always written, as the reference does
            pb_bytes(results, 1, solution);
        }
    }
    if (!yaml) {
        pb_double(results, 2, o.sanity_check_threshold);
        pb_double(results, 3, o.site_convergence_threshold);
        pb_double(results, 4, o.sweep_convergence_threshold);
        pb_double(results, 5, o.chain_convergence_threshold);
        out.write(results.data(), (std::streamsize)results.size());
        out.flush();
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    Values v;
    try {
        parse_command_line(argc, argv, v);
        parse_config_file(v.count("config-file") ? v.at("config-file") : std::string("nutcracker.cfg"), v);
        if (to_flag(v, "help")) print_help_and_exit();
        if (to_flag(v, "help-formats")) print_formats_and_exit();
        if (to_flag(v, "help-modes")) print_modes_and_exit();
        if (v.count("optimizer-mode")) {
            const std::string& m = v.at("optimizer-mode");
            if (m != "<v" && m != ">v" && m != ">m") throw OptionError("There is no such optimizer mode '" + m + "'.");
        }
    } catch (const std::exception& e) {
        std::cerr << "An error was encounted while parsing the options:\n\n"
                  << e.what() << "\n\nRun Nutcracker with the --help option for a description of the available "
                                  "options.\n";
        return -1;
    }
    try {
        return run(v);
    } catch (const FormatError& e) {
        std::cerr << e.what() << "\n";
        return -1;
    } catch (const OptionError& e) {
        std::cerr << "An error was encounted while parsing the options:\n\n"
                  << e.what() << "\n\nRun Nutcracker with the --help option for a description of the available "
                                  "options.\n";
        return -1;
    } catch (const std::exception& e) {
        std::cerr << e.what() << "\n";
    }
    return 0;
}
