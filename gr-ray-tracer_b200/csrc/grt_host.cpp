// Host-side formats of the hot path's boundary: the reference's NumPy .npy
// grid inputs and its uncompressed .npz output archives, plus the defaults
// and validity checks of grt_params.
//
//   grt_params_default fills the reference's compiled-in defaults
//     (src/utils.cpp:4-37, src/simulation_options.hpp:13-32,
//     src/radiative_transfer/photon_generation.hpp:18-50);
//   grt_params_validate checks what the kernels need of a grt_params;
//   npy_load_f64 reads what load_numpy_field_bundle accepts
//     (src/input/load_python_arrays.hpp:115-193: '<f8'/'=f8', C order);
//   NpzOut writes the byte layout of cnpy::NpzWriter (src/cnpy.h:146-300):
//     NPY 1.0 members, 16-byte padded headers, STORED ZIP with zero timestamps,
//     so archives are byte-for-byte the ones the reference writes.
// The reference's TOML config is read by the reference's own loader; its
// parsed structs reach the ABI through include/grt_reference_adapter.hpp.
#include "grt_host.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "grt.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

void set_err(char* err, size_t len, const std::string& msg) {
    if (err && len > 0) {
        std::snprintf(err, len, "%s", msg.c_str());
    }
}

std::string strip(const std::string& s) {
    const auto b = s.find_first_not_of(" \t\r\n");
    if (b == std::string::npos) return "";
    const auto e = s.find_last_not_of(" \t\r\n");
    return s.substr(b, e - b + 1);
}

// One condition of grt_params_validate and what it says when it fails.
struct Rule {
    bool ok;
    const char* message;
};

bool finite_positive(double v) { return std::isfinite(v) && v > 0.0; }
bool finite_nonnegative(double v) { return std::isfinite(v) && v >= 0.0; }

}  // namespace

extern "C" {

void grt_params_default(grt_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->mode = GRT_MODE_IMAGE;
    p->integrator = GRT_RK45;
    p->precision = GRT_PREC_FP64;
    p->generator = GRT_GEN_BLACKBODY;
    p->mass = 1.0;
    p->spin = 1.0;
    const double horizon = p->mass + std::sqrt(std::fmax(0.0, p->mass * p->mass - p->spin * p->spin));
    p->camera_theta = kPi / 4.0;
    p->camera_phi = kPi / 4.0;
    p->camera_width = 20.0;
    p->camera_height = 20.0;
    p->camera_distance = 10000.0;
    p->r_term_min = horizon;
    p->r_term_max = 1.5 * p->camera_distance;
    p->atol = 1e-8;
    p->rtol = 1e-8;
    p->min_step_scale = 0.01;
    p->max_step_scale = 10.0;
    p->safety = 0.9;
    p->max_steps = 10000;
    p->termination_percent = 0.9;
    p->output_interval = 1;
    p->nphotons = 20;
    p->initial_step = 0.1;
    p->scattering_albedo = 1.0;
    p->scattering_seed = 12345u;
    p->superphoton_count_normalization = 1.0;
    p->energy_per_cell_erg = 1.0;
    p->power_law_slope = 2.0;
    p->nu_min_hz = 1.0e9;
    p->nu_max_hz = 1.0e20;
    p->custom_frequency_hz = 2.30e11;
    p->length_cm_per_code = p->time_s_per_code = p->density_g_cm3_per_code = 1.0;
    p->temperature_k_per_code = p->four_velocity_cm_s_per_code = p->magnetic_gauss_per_code = 1.0;
    p->image_nx = p->image_ny = 256;
    p->spectrum_bins = 128;
    p->spectrum_min_hz = 1.0e8;
    p->spectrum_max_hz = 1.0e22;
}

grt_status grt_params_validate(const grt_params* p, char* err, size_t err_len) {
    if (!p) {
        set_err(err, err_len, "null params");
        return GRT_EINVAL;
    }
    const bool gen_ok = p->generator == GRT_GEN_BLACKBODY || p->generator == GRT_GEN_POWER_LAW ||
                        p->generator == GRT_GEN_CUSTOM;
    const bool power_law_ok = p->generator != GRT_GEN_POWER_LAW ||
                              (std::isfinite(p->power_law_slope) && finite_positive(p->nu_min_hz) &&
                               std::isfinite(p->nu_max_hz) && p->nu_max_hz > p->nu_min_hz);
    const bool units_ok = finite_positive(p->length_cm_per_code) && finite_positive(p->time_s_per_code) &&
                          finite_positive(p->density_g_cm3_per_code) && finite_positive(p->temperature_k_per_code) &&
                          finite_positive(p->four_velocity_cm_s_per_code) &&
                          finite_positive(p->magnetic_gauss_per_code);
    const Rule rules[] = {
        {p->mode == GRT_MODE_IMAGE || p->mode == GRT_MODE_DISK, "grt_params.mode: GRT_MODE_IMAGE or GRT_MODE_DISK"},
        {p->integrator == GRT_RK4 || p->integrator == GRT_RK45, "grt_params.integrator: GRT_RK4 or GRT_RK45"},
        {p->precision == GRT_PREC_FP64 || p->precision == GRT_PREC_MIXED || p->precision == GRT_PREC_MIXED_GRID,
         "grt_params.precision: GRT_PREC_FP64, GRT_PREC_MIXED or GRT_PREC_MIXED_GRID"},
        {gen_ok, "grt_params.generator: GRT_GEN_BLACKBODY, GRT_GEN_POWER_LAW or GRT_GEN_CUSTOM"},
        {finite_positive(p->mass), "grt_params.mass: finite and positive"},
        {std::isfinite(p->spin) && std::fabs(p->spin) <= p->mass,
         "grt_params.spin: |spin| <= mass (a Kerr black hole, not a naked singularity)"},
        {finite_nonnegative(p->r_term_min) && p->r_term_max > p->r_term_min,
         "grt_params termination radii: 0 <= r_term_min < r_term_max"},
        {finite_positive(p->atol) && finite_positive(p->rtol), "grt_params.atol, rtol: finite and positive"},
        {finite_positive(p->min_step_scale) && p->min_step_scale <= 1.0 && std::isfinite(p->max_step_scale) &&
             p->max_step_scale >= 1.0 && finite_positive(p->safety),
         "grt_params step-size controller: 0 < min_step_scale <= 1 <= max_step_scale, safety > 0"},
        {p->max_steps > 0, "grt_params.max_steps: positive"},
        {p->termination_percent > 0.0 && p->termination_percent <= 1.0,
         "grt_params.termination_percent: in (0, 1]"},
        {p->output_interval > 0, "grt_params.output_interval: positive"},
        {p->nphotons > 0, "grt_params.nphotons: positive (the count the terminated fraction is taken of)"},
        {finite_positive(p->initial_step), "grt_params.initial_step: finite and positive"},
        {finite_positive(p->camera_distance) && finite_positive(p->camera_width) &&
             finite_positive(p->camera_height) && std::isfinite(p->camera_theta) && std::isfinite(p->camera_phi),
         "grt_params camera: distance, width and height finite and positive, angles finite"},
        {finite_nonnegative(p->absorption_coefficient) && finite_nonnegative(p->emission_coefficient),
         "grt_params transfer coefficients: finite and non-negative"},
        {finite_nonnegative(p->scattering_albedo) && p->scattering_albedo <= 1.0,
         "grt_params.scattering_albedo: in [0, 1]"},
        {finite_positive(p->superphoton_count_normalization),
         "grt_params.superphoton_count_normalization: finite and positive"},
        {finite_nonnegative(p->energy_per_cell_erg), "grt_params.energy_per_cell_erg: finite and non-negative"},
        {power_law_ok, "grt_params power-law generator: finite slope and 0 < nu_min_hz < nu_max_hz"},
        {p->generator != GRT_GEN_CUSTOM || finite_positive(p->custom_frequency_hz),
         "grt_params.custom_frequency_hz: finite and positive for the custom generator"},
        {units_ok, "grt_params unit scales: every *_per_code factor finite and positive"},
        {p->image_nx > 0 && p->image_ny > 0 && p->spectrum_bins > 0,
         "grt_params image_nx, image_ny, spectrum_bins: positive"},
        {finite_positive(p->spectrum_min_hz) && std::isfinite(p->spectrum_max_hz) &&
             p->spectrum_max_hz > p->spectrum_min_hz,
         "grt_params spectrum range: 0 < spectrum_min_hz < spectrum_max_hz"},
    };
    for (const Rule& r : rules) {
        if (!r.ok) {
            set_err(err, err_len, r.message);
            return GRT_EINVAL;
        }
    }
    return GRT_OK;
}

grt_status grt_parse_output_variables(const char* spec, int32_t* fields, size_t* count, char* err, size_t err_len) {
    if (!spec || !count) {
        set_err(err, err_len, "null argument");
        return GRT_EINVAL;
    }
    std::vector<int> f;
    std::string msg;
    if (!grt::parse_output_variables(spec, f, msg)) {
        set_err(err, err_len, msg);
        return GRT_EINVAL;
    }
    if (fields)
        for (size_t k = 0; k < f.size(); ++k) fields[k] = f[k];
    *count = f.size();
    return GRT_OK;
}

}  // extern "C"

namespace grt {

// Reads a little-endian float64, C-order .npy file.
bool npy_load_f64(const std::string& path, std::vector<size_t>& shape, std::vector<double>& data,
                  std::string& err) {
    std::ifstream in(path, std::ios::binary);
    if (!in) {
        err = "Failed to open numpy file: " + path;
        return false;
    }
    char magic[6];
    in.read(magic, 6);
    if (!in || std::memcmp(magic, "\x93NUMPY", 6) != 0) {
        err = "Invalid .npy magic: " + path;
        return false;
    }
    unsigned char ver[2];
    in.read(reinterpret_cast<char*>(ver), 2);
    size_t hlen = 0;
    if (ver[0] == 1) {
        unsigned char b[2];
        in.read(reinterpret_cast<char*>(b), 2);
        hlen = b[0] | (static_cast<size_t>(b[1]) << 8);
    } else {
        unsigned char b[4];
        in.read(reinterpret_cast<char*>(b), 4);
        hlen = b[0] | (static_cast<size_t>(b[1]) << 8) | (static_cast<size_t>(b[2]) << 16) |
               (static_cast<size_t>(b[3]) << 24);
    }
    std::string header(hlen, '\0');
    in.read(&header[0], static_cast<std::streamsize>(hlen));
    if (!in) {
        err = "Truncated .npy header: " + path;
        return false;
    }
    const auto dpos = header.find("'descr'");
    const auto q1 = header.find('\'', header.find(':', dpos) + 1);
    const auto q2 = header.find('\'', q1 + 1);
    const std::string descr = (dpos == std::string::npos || q1 == std::string::npos) ? "" : header.substr(q1 + 1, q2 - q1 - 1);
    if (descr != "<f8" && descr != "=f8") {
        err = "Grid arrays must use native/little-endian float64 values: " + path;
        return false;
    }
    if (header.find("'fortran_order': True") != std::string::npos) {
        err = "Fortran-ordered arrays are not supported: " + path;
        return false;
    }
    const auto open = header.find('(');
    const auto close = header.find(')', open);
    if (open == std::string::npos || close == std::string::npos) {
        err = "Invalid .npy header: missing shape";
        return false;
    }
    shape.clear();
    std::stringstream ss(header.substr(open + 1, close - open - 1));
    std::string item;
    size_t total = 1;
    while (std::getline(ss, item, ',')) {
        item = strip(item);
        if (!item.empty()) {
            shape.push_back(static_cast<size_t>(std::stoll(item)));
            total *= shape.back();
        }
    }
    data.resize(total);
    in.read(reinterpret_cast<char*>(data.data()), static_cast<std::streamsize>(total * sizeof(double)));
    if (!in) {
        err = "Unexpected EOF while reading numpy data: " + path;
        return false;
    }
    return true;
}

namespace {
void put16(std::vector<char>& b, uint16_t v) {
    b.push_back(static_cast<char>(v & 0xff));
    b.push_back(static_cast<char>(v >> 8));
}
void put32(std::vector<char>& b, uint32_t v) {
    for (int i = 0; i < 4; ++i) b.push_back(static_cast<char>((v >> (8 * i)) & 0xff));
}
uint32_t crc32_of(const std::vector<char>& bytes) {
    uint32_t crc = 0xffffffffu;
    for (const unsigned char byte : bytes) {
        crc ^= byte;
        for (int bit = 0; bit < 8; ++bit) crc = (crc >> 1) ^ (0xedb88320u & (0u - (crc & 1u)));
    }
    return ~crc;
}
}  // namespace

std::vector<char> npy_bytes(const char* descr, const std::vector<size_t>& shape, const void* data,
                            size_t item_size) {
    std::ostringstream h;
    h << "{'descr': '" << descr << "', 'fortran_order': False, 'shape': (";
    size_t total = 1;
    for (size_t i = 0; i < shape.size(); ++i) {
        h << shape[i];
        total *= shape[i];
        if (shape.size() == 1 || i + 1 < shape.size()) h << ", ";
    }
    h << "), }";
    std::string header = h.str();
    while ((10 + header.size()) % 16 != 0) header.push_back(' ');
    header.push_back('\n');
    std::vector<char> b;
    b.reserve(10 + header.size() + total * item_size);
    const char magic[] = "\x93NUMPY";
    b.insert(b.end(), magic, magic + 6);
    b.push_back(1);
    b.push_back(0);
    put16(b, static_cast<uint16_t>(header.size()));
    b.insert(b.end(), header.begin(), header.end());
    const char* raw = static_cast<const char*>(data);
    b.insert(b.end(), raw, raw + total * item_size);
    return b;
}

const char* const kOutputFields[kOutputFieldCount] = {
    "id", "frequency", "emission_frame_energy", "x0", "x1", "x2", "x3", "k0", "k1", "k2", "k3",
    "I", "Q", "U", "V", "dlambda", "terminate", "phase", "theta_disp", "phi_disp"};

namespace {
std::string trim_spaces(const std::string& v) {
    size_t a = 0, b = v.size();
    while (a < b && std::isspace(static_cast<unsigned char>(v[a]))) ++a;
    while (b > a && std::isspace(static_cast<unsigned char>(v[b - 1]))) --b;
    return v.substr(a, b - a);
}
}  // namespace

bool parse_output_variables(const std::string& spec_in, std::vector<int>& fields, std::string& err) {
    fields.clear();
    std::string spec = trim_spaces(spec_in);
    if (spec.empty()) {
        err = "output variables cannot be empty";
        return false;
    }
    if (spec.size() >= 2 && spec.front() == '[' && spec.back() == ']') spec = spec.substr(1, spec.size() - 2);
    size_t begin = 0;
    while (begin <= spec.size()) {
        const size_t comma = spec.find(',', begin);
        std::string name = trim_spaces(spec.substr(begin, comma == std::string::npos ? std::string::npos : comma - begin));
        if (name.size() >= 2 && ((name.front() == '"' && name.back() == '"') ||
                                 (name.front() == '\'' && name.back() == '\'')))
            name = trim_spaces(name.substr(1, name.size() - 2));
        if (name == "all") {
            // appended to what came before, as the reference does (so "I,all"
            // writes I twice)
            for (int k = 0; k < kOutputFieldCount; ++k) fields.push_back(k);
            return true;
        }
        if (!name.empty()) {
            int k = 0;
            while (k < kOutputFieldCount && name != kOutputFields[k]) ++k;
            if (k == kOutputFieldCount) {
                err = "unknown output variable: " + name;
                fields.clear();
                return false;
            }
            if (std::find(fields.begin(), fields.end(), k) == fields.end()) fields.push_back(k);
        }
        if (comma == std::string::npos) break;
        begin = comma + 1;
    }
    if (fields.empty()) {
        err = "output variables cannot be empty";
        return false;
    }
    return true;
}

bool NpzOut::open(const std::string& path) {
    out_.open(path, std::ios::binary | std::ios::trunc);
    offset_ = 0;
    entries_.clear();
    error_.clear();
    if (!out_) error_ = "Failed to open output NumPy archive: " + path;
    return static_cast<bool>(out_);
}

// The archive is a stored (uncompressed) ZIP without the ZIP64 extension, as
// the reference writes it (cnpy.h:176-181, 220-248): sizes and offsets are
// 32-bit fields, so an archive that outgrows them is refused, not wrapped.
bool NpzOut::add(const std::string& name, const std::vector<char>& payload) {
    const std::string member = name + ".npy";
    if (member.size() > 0xffffu || payload.size() > limit_ || offset_ > limit_) {
        error_ = "NumPy archive exceeds the non-ZIP64 size limit";
        return false;
    }
    Entry e{member, crc32_of(payload), static_cast<uint32_t>(payload.size()), static_cast<uint32_t>(offset_)};
    std::vector<char> h;
    put32(h, 0x04034b50u);
    put16(h, 20); put16(h, 0); put16(h, 0); put16(h, 0); put16(h, 0);
    put32(h, e.crc); put32(h, e.size); put32(h, e.size);
    put16(h, static_cast<uint16_t>(member.size()));
    put16(h, 0);
    out_.write(h.data(), static_cast<std::streamsize>(h.size()));
    out_.write(member.data(), static_cast<std::streamsize>(member.size()));
    out_.write(payload.data(), static_cast<std::streamsize>(payload.size()));
    offset_ += h.size() + member.size() + payload.size();
    entries_.push_back(e);
    if (!out_) error_ = "Failed while writing NumPy archive";
    return static_cast<bool>(out_);
}

bool NpzOut::close() {
    if (entries_.size() > 0xffffu) {
        error_ = "NumPy archive contains too many arrays";
        out_.close();
        return false;
    }
    const uint64_t cd_offset = offset_;
    for (const Entry& e : entries_) {
        std::vector<char> h;
        put32(h, 0x02014b50u);
        put16(h, 20); put16(h, 20); put16(h, 0); put16(h, 0); put16(h, 0); put16(h, 0);
        put32(h, e.crc); put32(h, e.size); put32(h, e.size);
        put16(h, static_cast<uint16_t>(e.name.size()));
        put16(h, 0); put16(h, 0); put16(h, 0); put16(h, 0);
        put32(h, 0);
        put32(h, e.offset);
        out_.write(h.data(), static_cast<std::streamsize>(h.size()));
        out_.write(e.name.data(), static_cast<std::streamsize>(e.name.size()));
        offset_ += h.size() + e.name.size();
    }
    if (cd_offset > limit_ || offset_ - cd_offset > limit_) {
        error_ = "NumPy archive exceeds the non-ZIP64 size limit";
        out_.close();
        return false;
    }
    std::vector<char> end;
    put32(end, 0x06054b50u);
    put16(end, 0); put16(end, 0);
    put16(end, static_cast<uint16_t>(entries_.size()));
    put16(end, static_cast<uint16_t>(entries_.size()));
    put32(end, static_cast<uint32_t>(offset_ - cd_offset));
    put32(end, static_cast<uint32_t>(cd_offset));
    put16(end, 0);
    out_.write(end.data(), static_cast<std::streamsize>(end.size()));
    out_.close();
    if (!out_ && error_.empty()) error_ = "Failed while writing NumPy archive";
    return static_cast<bool>(out_);
}

}  // namespace grt
