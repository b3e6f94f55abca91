// cfd-bench for the B200 engine: the reference benchmark CLI's interface
// (apps/cfd-bench.cpp: option names, the in-place D3Q19/D3Q27 Taylor-Green
// case, the cfd_solvers.benchmark.v1 record keys) with the `--backend cuda`
// branch its dispatch_backend (apps/cfd-bench.cpp:236-261) would gain,
// written against the C++20 front end include/cfd/solvers/lbm/esoteric_pull_cuda.hpp.
//
// Structure: one table of options drives parsing, validation and --help; one
// ordered record of (key, value) fields is built per run and printed by one
// of three writers (text, --csv, --json).  Timing: `--warmup` untimed steps,
// then `--steps` steps timed on the host steady clock around step() + wait(),
// as the reference's SYCL branch does.  Keys beyond the reference's: glups,
// algorithmic_bytes_per_update, roofline_fraction (with --hbm-peak-gbs),
// storage_precision, collision, case, checksum.  Extensions: --storage
// fp32|fp16s|fp64, --collision bgk|trt, --les, --case taylor-green|cavity.
#include "cfd/solvers/lbm/esoteric_pull_cuda.hpp"

#include <algorithm>
#include <array>
#include <charconv>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <iostream>
#include <optional>
#include <stdexcept>
#include <string>
#include <string_view>
#include <type_traits>
#include <variant>
#include <vector>

namespace {

struct Settings {
    std::string lattice = "d3q19";
    std::string storage = "fp32";
    std::string collision = "bgk";
    std::string case_name = "taylor-green";
    std::size_t extent[3] = {64, 64, 64};
    std::size_t warmup = 10;
    std::size_t steps = 100;
    float tau = 0.6F;
    bool les = false;
    double hbm_peak_gbs = 0.0;
    enum class Format { text, csv, json } format = Format::text;
};

[[noreturn]] void reject(std::string_view option, std::string_view why) {
    throw std::invalid_argument(std::string(option) + " " + std::string(why));
}

std::size_t positive_count(std::string_view option, std::string_view text) {
    unsigned long long v = 0;
    const auto [end, ec] = std::from_chars(text.data(), text.data() + text.size(), v);
    if (ec != std::errc{} || end != text.data() + text.size() || v == 0) reject(option, "must be > 0");
    return static_cast<std::size_t>(v);
}

double real_value(std::string_view option, std::string_view text) {
    // strtod: from_chars for floating point is not in every libstdc++ this header meets
    const std::string copy(text);
    char* end = nullptr;
    const double v = std::strtod(copy.c_str(), &end);
    if (end == copy.c_str() || *end != '\0') reject(option, "needs a number");
    return v;
}

std::string one_of(std::string_view option, std::string_view text, std::initializer_list<std::string_view> allowed) {
    for (const auto a : allowed)
        if (a == text) return std::string(text);
    std::string list;
    for (const auto a : allowed) list += (list.empty() ? "" : "|") + std::string(a);
    reject(option, "must be " + list);
}

// One command-line option: `value` names its argument (empty for a switch).
struct OptionSpec {
    std::string_view name;
    std::string_view value;
    std::string_view help;
    void (*apply)(Settings&, std::string_view name, std::string_view arg);
};

constexpr std::array<OptionSpec, 17> kOptions{{
    {"--lattice", "d3q19|d3q27", "velocity set",
     [](Settings& s, std::string_view n, std::string_view v) { s.lattice = one_of(n, v, {"d3q19", "d3q27"}); }},
    {"--backend", "cuda", "execution backend (this build: cuda)",
     [](Settings&, std::string_view, std::string_view v) {
         if (v != "cuda") throw std::invalid_argument("this build provides --backend cuda");
     }},
    {"--streaming", "in-place", "streaming scheme (the CUDA backend runs in-place Esoteric-Pull)",
     [](Settings&, std::string_view, std::string_view v) {
         if (v != "in-place") throw std::invalid_argument("the CUDA backend runs --streaming in-place");
     }},
    {"--nx", "N", "cells in x", [](Settings& s, std::string_view n, std::string_view v) { s.extent[0] = positive_count(n, v); }},
    {"--ny", "N", "cells in y", [](Settings& s, std::string_view n, std::string_view v) { s.extent[1] = positive_count(n, v); }},
    {"--nz", "N", "cells in z", [](Settings& s, std::string_view n, std::string_view v) { s.extent[2] = positive_count(n, v); }},
    {"--warmup", "N", "untimed steps", [](Settings& s, std::string_view n, std::string_view v) { s.warmup = positive_count(n, v); }},
    {"--steps", "N", "timed steps", [](Settings& s, std::string_view n, std::string_view v) { s.steps = positive_count(n, v); }},
    {"--tau", "T", "relaxation time (> 0.5)",
     [](Settings& s, std::string_view n, std::string_view v) {
         const double t = real_value(n, v);
         if (!(t > 0.5)) reject(n, "must be > 0.5");
         s.tau = static_cast<float>(t);
     }},
    {"--storage", "fp32|fp16s|fp64", "population storage",
     [](Settings& s, std::string_view n, std::string_view v) { s.storage = one_of(n, v, {"fp32", "fp16s", "fp64"}); }},
    {"--collision", "bgk|trt", "collision operator",
     [](Settings& s, std::string_view n, std::string_view v) { s.collision = one_of(n, v, {"bgk", "trt"}); }},
    {"--case", "taylor-green|cavity", "start: Taylor-Green vortex (periodic) or lid-driven cavity",
     [](Settings& s, std::string_view n, std::string_view v) { s.case_name = one_of(n, v, {"taylor-green", "cavity"}); }},
    {"--les", "", "Smagorinsky closure with Cs = 0.1", [](Settings& s, std::string_view, std::string_view) { s.les = true; }},
    {"--hbm-peak-gbs", "G", "HBM bandwidth for roofline_fraction",
     [](Settings& s, std::string_view n, std::string_view v) { s.hbm_peak_gbs = real_value(n, v); }},
    {"--csv", "", "CSV record", [](Settings& s, std::string_view, std::string_view) { s.format = Settings::Format::csv; }},
    {"--json", "", "JSON record", [](Settings& s, std::string_view, std::string_view) { s.format = Settings::Format::json; }},
    {"--help", "", "this text", nullptr},
}};

void print_help() {
    std::cout << "usage: cfd-bench-cuda [options]   (in-place Esoteric-Pull LBM on the CUDA engine)\n";
    for (const auto& o : kOptions) {
        std::string head = "  " + std::string(o.name) + (o.value.empty() ? "" : " " + std::string(o.value));
        head.resize(std::max<std::size_t>(head.size() + 1, 34), ' ');
        std::cout << head << o.help << '\n';
    }
}

// nullopt: --help was printed.
std::optional<Settings> parse(int argc, char** argv) {
    Settings s;
    for (int i = 1; i < argc; ++i) {
        const std::string_view arg = argv[i];
        if (arg == "-h") {
            print_help();
            return std::nullopt;
        }
        const OptionSpec* spec = nullptr;
        for (const auto& o : kOptions)
            if (o.name == arg) spec = &o;
        if (!spec) throw std::invalid_argument("unknown option " + std::string(arg));
        if (!spec->apply) {
            print_help();
            return std::nullopt;
        }
        std::string_view value;
        if (!spec->value.empty()) {
            if (i + 1 >= argc) reject(arg, "requires a value");
            value = argv[++i];
        }
        spec->apply(s, arg, value);
    }
    return s;
}

// ------------------------------------------------------------------ records
struct Field {
    std::string key;
    std::variant<std::string, std::uint64_t, double, std::nullptr_t> value;
    int digits = 12; // significant digits of a double
};

using Record = std::vector<Field>;

std::string number(double v, int digits) {
    char buf[64];
    const auto [end, ec] = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::general, digits);
    return ec == std::errc{} ? std::string(buf, end) : std::string("nan");
}

std::string plain(const Field& f) {
    return std::visit(
        [&](const auto& v) -> std::string {
            using T = std::decay_t<decltype(v)>;
            if constexpr (std::is_same_v<T, std::string>) return v;
            else if constexpr (std::is_same_v<T, std::uint64_t>) return std::to_string(v);
            else if constexpr (std::is_same_v<T, double>) return number(v, f.digits);
            else return "null";
        },
        f.value);
}

std::string quote_text(std::string_view text) {
    std::string out = "\"";
    for (const char c : text) {
        if (c == '"' || c == '\\') out.push_back('\\');
        out.push_back(c);
    }
    return out + "\"";
}

void write_json(const Record& r) {
    std::string out = "{";
    for (const auto& f : r) {
        if (out.size() > 1) out += ",";
        out += quote_text(f.key) + ":" + (std::holds_alternative<std::string>(f.value) ? quote_text(plain(f)) : plain(f));
    }
    std::cout << out << "}\n";
}

void write_csv(const Record& r) {
    std::string keys, values;
    for (const auto& f : r) {
        const bool first = keys.empty();
        keys += (first ? "" : ",") + f.key;
        std::string v = plain(f);
        if (v.find_first_of(",\" ") != std::string::npos) v = quote_text(v);
        values += (first ? "" : ",") + v;
    }
    std::cout << keys << '\n' << values << '\n';
}

void write_text(const Record& r) {
    // key=value, a few fields per line
    std::size_t on_line = 0;
    for (const auto& f : r) {
        std::string v = plain(f);
        if (v.find(' ') != std::string::npos) v = quote_text(v);
        std::cout << (on_line ? " " : "") << f.key << '=' << v;
        if (++on_line == 6) {
            std::cout << '\n';
            on_line = 0;
        }
    }
    if (on_line) std::cout << '\n';
}

// Walls on x = 0, nx-1, y = 0, z = 0, nz-1; the lid (moving wall id 2) on y = ny-1.
std::vector<std::uint8_t> cavity(const std::size_t (&e)[3]) {
    std::vector<std::uint8_t> flags(e[0] * e[1] * e[2], 0);
    std::size_t n = 0;
    for (std::size_t z = 0; z < e[2]; ++z)
        for (std::size_t y = 0; y < e[1]; ++y)
            for (std::size_t x = 0; x < e[0]; ++x, ++n) {
                const bool side = x == 0 || x + 1 == e[0] || z == 0 || z + 1 == e[2];
                flags[n] = (side || y == 0) ? 1 : (y + 1 == e[1] ? 2 : 0);
            }
    return flags;
}

template <class Descriptor> Record run(const Settings& s) {
    namespace cu = cfd::lbm::cuda;
    cu::InPlaceLbmConfig config;
    config.nx = s.extent[0];
    config.ny = s.extent[1];
    config.nz = s.extent[2];
    config.tau = s.tau;
    config.smagorinsky_les = s.les;
    config.smagorinsky_cs = s.les ? 0.1F : 0.0F;
    config.collision = s.collision == "trt" ? cu::Collision::trt : cu::Collision::bgk;
    config.storage = s.storage == "fp16s" ? cu::Storage::fp16s : (s.storage == "fp64" ? cu::Storage::fp64 : cu::Storage::fp32);

    cfd::lbm::EsotericPullCudaSolver<Descriptor> solver(config);
    const std::size_t cells = solver.cells();
    std::size_t fluid = cells;
    if (s.case_name == "cavity") {
        const auto flags = cavity(s.extent);
        solver.set_flags(flags);
        solver.set_wall_velocity(2, 0.1F, 0.0F, 0.0F);
        solver.initialize_uniform();
        fluid = 0;
        for (const auto f : flags) fluid += f == 0 ? 1U : 0U;
    } else {
        solver.initialize_taylor_green(0.02F);
    }
    const double mass0 = solver.total_mass();
    solver.step(s.warmup);
    solver.wait();
    const auto t0 = std::chrono::steady_clock::now();
    solver.step(s.steps);
    solver.wait();
    const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const double mass1 = solver.total_mass();

    const double q = Descriptor::q;
    const double mlups = static_cast<double>(cells) * static_cast<double>(s.steps) / seconds * 1e-6;
    const double value_bytes = s.storage == "fp16s" ? 2.0 : (s.storage == "fp64" ? 8.0 : 4.0);
    // every fluid cell reads and writes its q populations once; with flags every cell's byte is read
    const double bytes_per_update =
        (2.0 * q * value_bytes * static_cast<double>(fluid) + (fluid == cells ? 0.0 : static_cast<double>(cells))) /
        static_cast<double>(cells);
    const double mib = 1.0 / (1024.0 * 1024.0);
    const double mass_abs = std::abs(mass1 - mass0);
    const std::string collision = s.collision + (s.les ? "+les" : "");
    Record r;
    r.push_back({"schema", std::string("cfd_solvers.benchmark.v1")});
    r.push_back({"lattice", s.lattice});
    r.push_back({"backend", std::string("cuda")});
    r.push_back({"streaming", std::string("in-place")});
    r.push_back({"device", solver.device_name()});
    r.push_back({"nx", std::uint64_t{s.extent[0]}});
    r.push_back({"ny", std::uint64_t{s.extent[1]}});
    r.push_back({"nz", std::uint64_t{s.extent[2]}});
    r.push_back({"q", std::uint64_t{Descriptor::q}});
    r.push_back({"steps", std::uint64_t{s.steps}});
    r.push_back({"seconds", seconds});
    r.push_back({"mlups", mlups});
    // the reference's estimate: 2 q FP32 values per update
    r.push_back({"estimated_ddf_gbps", mlups * 2.0 * q * 4.0 * 1e-3});
    r.push_back({"allocated_ddf_mib", static_cast<double>(solver.population_bytes()) * mib});
    r.push_back({"single_grid_ddf_mib", q * static_cast<double>(cells) * 4.0 * mib});
    r.push_back({"mass_error_abs", mass_abs});
    r.push_back({"mass_error_rel", mass0 != 0.0 ? mass_abs / std::abs(mass0) : 0.0});
    r.push_back({"glups", mlups * 1e-3});
    r.push_back({"algorithmic_bytes_per_update", bytes_per_update});
    if (s.hbm_peak_gbs > 0.0)
        r.push_back({"roofline_fraction", mlups * bytes_per_update * 1e-3 / s.hbm_peak_gbs});
    else
        r.push_back({"roofline_fraction", nullptr});
    r.push_back({"storage_precision", s.storage});
    r.push_back({"collision", collision});
    r.push_back({"case", s.case_name});
    r.push_back({"checksum", solver.checksum(), 17});
    return r;
}

} // namespace

int main(int argc, char** argv) {
    try {
        const auto settings = parse(argc, argv);
        if (!settings) return 0;
        const Settings& s = *settings;
        const Record record = s.lattice == "d3q27" ? run<cfd::lbm::cuda::D3Q27>(s) : run<cfd::lbm::cuda::D3Q19>(s);
        switch (s.format) {
        case Settings::Format::json: write_json(record); break;
        case Settings::Format::csv: write_csv(record); break;
        case Settings::Format::text: write_text(record); break;
        }
        return 0;
    } catch (const std::exception& error) {
        std::cerr << "cfd-bench: " << error.what() << '\n';
        return 1;
    }
}
