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
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
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

unsigned long long to_unsigned(const Values& v, const char* name) {
    const std::string& s = v.at(name);
    char* end = nullptr;
    const unsigned long long x = std::strtoull(s.c_str(), &end, 10);
    if (end == s.c_str() || *end || s[0] == '-')
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
    std::cerr << "The recognized input format types are:\n  - yaml: YAML format\n\n"
                 "The recognized output format types are:\n  - yaml: YAML format\n\n";
    std::exit(1);
}

void print_modes_and_exit() {
    std::cerr << "The recognized optimizer modes are:\n  '<v' - least value\n  '>m' - largest magnitude\n"
                 "  '>v' - greatest value\n\n";
    std::exit(1);
}

// resolveAndCheckFormat (io.hpp:389-418) with yaml as the only (and default)
// format: it reads and writes pipes; only the input supports locations; the
// output supports no states.
void resolve_format(const Values& v, const char* type, const char* format_key, const char* location_key) {
    auto f = v.find(format_key);
    if (f != v.end() && f->second != "yaml")
        throw FormatError(f->second + " is not a recognized/supported " + type + " format type.\n\nThe recognized " +
                          type + " format types are:\n  - yaml\n\nRun Nutcracker with the --help-formats option for "
                          "more informaton about supported formats.");
    if (std::string(type) == "output" && v.count(location_key))
        throw FormatError("The output format type yaml does not support locations.");
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

int run(const Values& v) {
    resolve_format(v, "input", "input-format", "input-location");
    resolve_format(v, "output", "output-format", "output-location");
    if (to_flag(v, "output-states")) throw FormatError("Output format yaml does not support outputing states.");

    nc_chain_options o;
    nc_chain_options_init(&o);
    if (v.count("site-tolerance")) o.site_convergence_threshold = to_double(v, "site-tolerance");
    if (v.count("sweep-tolerance")) o.sweep_convergence_threshold = to_double(v, "sweep-tolerance");
    if (v.count("chain-tolerance")) o.chain_convergence_threshold = to_double(v, "chain-tolerance");
    if (v.count("sanity-tolerance")) o.sanity_check_threshold = to_double(v, "sanity-tolerance");
    if (v.count("precision")) o.precision = (uint32_t)to_unsigned(v, "precision");
    if (v.count("seed")) o.seed = to_unsigned(v, "seed");
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
    const char* location = v.count("input-location") ? v.at("input-location").c_str() : nullptr;
    nc_yaml_operator* op = nc_yaml_read_operator(text.data(), text.size(), location);
    if (!op) Library::fail();
    nc_chain* chain = nc_chain_create(nc_yaml_operator_number_of_sites(op), nc_yaml_operator_sites(op), &o);
    nc_yaml_operator_free(op);
    if (!chain) Library::fail();

    // the YAML outputter (yaml.cpp:106-143)
    std::ofstream file;
    if (v.count("output-file")) {
        const std::string& name = v.at("output-file");
        if (!to_flag(v, "output-overwrite") && std::ifstream(name).good()) {
            nc_chain_free(chain);
            throw std::runtime_error("The output filename " + name + " already exists.");
        }
        file.open(name);
        if (!file) {
            nc_chain_free(chain);
            throw std::runtime_error("cannot open the output file " + name);
        }
    }
    std::ostream& out = v.count("output-file") ? static_cast<std::ostream&>(file) : std::cout;
    out << "Configuration:\n"
        << "  site convergence tolerance: " << o.site_convergence_threshold << "\n"
        << "  sweep convergence tolerance: " << o.sweep_convergence_threshold << "\n"
        << "  chain convergence tolerance: " << o.chain_convergence_threshold << "\n"
        << "  sanity check threshold: " << o.sanity_check_threshold << "\n"
        << "Energy levels:\n";
    out.flush();
    const unsigned digits = digits_of_precision(o.chain_convergence_threshold);

    // solveForMultipleLevels (chain.cpp:301-310), one line per optimised level
    for (unsigned k = 0; k < levels; ++k) {
        if (k > 0 && (nc_chain_construct_and_add_projector_from_state(chain) != 0 || nc_chain_reset(chain) != 0)) {
            nc_chain_free(chain);
            Library::fail();
        }
        double e = 0;
        if (nc_chain_optimize_chain(chain) != 0 || nc_chain_get_energy(chain, &e) != 0) {
            const std::string msg = nc_last_error();
            nc_chain_free(chain);
            throw std::runtime_error(msg);
        }
        out << "  - " << std::setprecision(digits) << e << "\n";
        out.flush();
    }
    nc_chain_free(chain);
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
