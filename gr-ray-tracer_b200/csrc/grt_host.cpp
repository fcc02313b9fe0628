// Host-side formats of the hot path's boundary: the reference's flat TOML
// config, its NumPy .npy grid inputs and its uncompressed .npz output archives.
//
//   grt_params_default / grt_params_from_toml / grt_params_validate mirror
//     toml_config::parse_flat_toml + load_and_apply_toml_config
//     (src/input/toml_config.hpp:40-77, 129-278) with defaults from
//     src/utils.cpp:4-37, src/simulation_options.hpp:13-32 and
//     src/radiative_transfer/photon_generation.hpp:18-50;
//   npy_load_f64 reads what load_numpy_field_bundle accepts
//     (src/input/load_python_arrays.hpp:115-193: '<f8'/'=f8', C order);
//   NpzOut writes the byte layout of cnpy::NpzWriter (src/cnpy.h:146-300):
//     NPY 1.0 members, 16-byte padded headers, STORED ZIP with zero timestamps,
//     so archives are byte-for-byte the ones the reference writes.
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

void set_str(char* dst, size_t len, const std::string& s) {
    if (dst && len > 0) std::snprintf(dst, len, "%s", s.c_str());
}

std::string strip(const std::string& s) {
    const auto b = s.find_first_not_of(" \t\r\n");
    if (b == std::string::npos) return "";
    const auto e = s.find_last_not_of(" \t\r\n");
    return s.substr(b, e - b + 1);
}

using Raw = std::map<std::string, std::string>;

// toml_config.hpp:40-77
Raw parse_flat(const std::string& path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("Failed to open config file: " + path);
    Raw values;
    std::string section, line;
    while (std::getline(in, line)) {
        bool quoted = false;
        for (size_t i = 0; i < line.size(); ++i) {
            if (line[i] == '"') quoted = !quoted;
            else if (line[i] == '#' && !quoted) {
                line = line.substr(0, i);
                break;
            }
        }
        const std::string t = strip(line);
        if (t.empty()) continue;
        if (t.front() == '[' && t.back() == ']') {
            section = strip(t.substr(1, t.size() - 2));
            continue;
        }
        const auto eq = t.find('=');
        if (eq == std::string::npos)
            throw std::runtime_error("Malformed config line (expected 'key = value'): " + line);
        const std::string key = strip(t.substr(0, eq));
        std::string value = strip(t.substr(eq + 1));
        if (value.size() >= 2 && value.front() == '"' && value.back() == '"') value = value.substr(1, value.size() - 2);
        values[section.empty() ? key : section + "." + key] = value;
    }
    return values;
}

double get_real(const Raw& c, const std::string& k, double fb) {
    const auto it = c.find(k);
    return it == c.end() ? fb : std::stod(it->second);
}
int get_int(const Raw& c, const std::string& k, int fb) {
    const auto it = c.find(k);
    return it == c.end() ? fb : std::stoi(it->second);
}
uint64_t get_u64(const Raw& c, const std::string& k, uint64_t fb) {
    const auto it = c.find(k);
    if (it == c.end()) return fb;
    if (!it->second.empty() && it->second.front() == '-') throw std::runtime_error(k + " must not be negative");
    return std::stoull(it->second);
}
bool get_bool(const Raw& c, const std::string& k, bool fb) {
    const auto it = c.find(k);
    if (it == c.end()) return fb;
    if (it->second == "true") return true;
    if (it->second == "false") return false;
    throw std::runtime_error(k + " must be true or false");
}
std::string get_str(const Raw& c, const std::string& k, const std::string& fb) {
    const auto it = c.find(k);
    return it == c.end() ? fb : it->second;
}

// photon_generation.hpp:77-85
int parse_generator(const std::string& name) {
    if (name == "blackbody") return GRT_GEN_BLACKBODY;
    if (name == "power-law" || name == "power_law" || name == "powerlaw") return GRT_GEN_POWER_LAW;
    if (name == "custom") return GRT_GEN_CUSTOM;
    throw std::runtime_error("photons.generator must be 'blackbody', 'power-law', or 'custom' (got '" + name + "')");
}

// The reference's validate() checks (toml_config.hpp:238-276,
// photon_generation.hpp:26-74) as one function.
void validate_or_throw(const grt_params& p) {
    if (p.nphotons == 0 || p.nphotons > 100000000000ULL)
        throw std::runtime_error("photons.count must be in [1, 100000000000]");
    if (p.max_steps <= 0) throw std::runtime_error("integration.max_steps must be positive");
    if (p.output_interval == 0) throw std::runtime_error("output.interval must be positive");
    if (p.image_nx == 0 || p.image_ny == 0 || p.spectrum_bins == 0)
        throw std::runtime_error("output image dimensions and spectrum_bins must be positive");
    if (!(p.spectrum_min_hz > 0.0) || !(p.spectrum_max_hz > p.spectrum_min_hz))
        throw std::runtime_error("output requires 0 < spectrum_min_hz < spectrum_max_hz");
    if (!(p.camera_distance > 0.0) || !(p.camera_width > 0.0) || !(p.camera_height > 0.0))
        throw std::runtime_error("camera distance, width, and height must be positive");
    if (!std::isfinite(p.scattering_albedo) || p.scattering_albedo < 0.0 || p.scattering_albedo > 1.0)
        throw std::runtime_error("scattering.albedo must be finite and in [0, 1]");
    if (!std::isfinite(p.absorption_coefficient) || p.absorption_coefficient < 0.0)
        throw std::runtime_error("radiative_transfer.absorption_coefficient must be finite and non-negative");
    if (!std::isfinite(p.emission_coefficient) || p.emission_coefficient < 0.0)
        throw std::runtime_error("radiative_transfer.emission_coefficient must be finite and non-negative");
    if (p.termination_percent <= 0.0 || p.termination_percent > 1.0)
        throw std::runtime_error("integration.termination_percent must be in (0, 1]");
    if (!(p.superphoton_count_normalization > 0.0) || !std::isfinite(p.superphoton_count_normalization))
        throw std::runtime_error("photons.superphoton_count_normalization must be finite and positive");
    if (!(p.energy_per_cell_erg >= 0.0) || !std::isfinite(p.energy_per_cell_erg))
        throw std::runtime_error("photons.energy_per_cell_erg must be finite and non-negative");
    if (p.generator == GRT_GEN_POWER_LAW) {
        if (!std::isfinite(p.power_law_slope)) throw std::runtime_error("photons.power_law_slope must be finite");
        if (!(p.nu_min_hz > 0.0) || !(p.nu_max_hz > p.nu_min_hz) || !std::isfinite(p.nu_min_hz) ||
            !std::isfinite(p.nu_max_hz))
            throw std::runtime_error("power-law generation requires 0 < photons.nu_min_hz < photons.nu_max_hz");
    }
    if (p.generator == GRT_GEN_CUSTOM && (!(p.custom_frequency_hz > 0.0) || !std::isfinite(p.custom_frequency_hz)))
        throw std::runtime_error("photons.custom_frequency_hz must be finite and positive");
    const double units[6] = {p.length_cm_per_code, p.time_s_per_code, p.density_g_cm3_per_code,
                             p.temperature_k_per_code, p.four_velocity_cm_s_per_code, p.magnetic_gauss_per_code};
    for (double u : units)
        if (!(u > 0.0) || !std::isfinite(u))
            throw std::runtime_error("all [units] conversion factors must be finite and positive");
    if (!(p.mass > 0.0)) throw std::runtime_error("black_hole.mass must be positive");
    if (std::fabs(p.spin) > p.mass) throw std::runtime_error("black_hole.spin must satisfy |spin| <= mass");
    if (p.mode != GRT_MODE_IMAGE && p.mode != GRT_MODE_DISK) throw std::runtime_error("simulation.mode must be 'image' or 'disk'");
    if (p.integrator != GRT_RK4 && p.integrator != GRT_RK45)
        throw std::runtime_error("integration.integrator must be \"rk4\" or \"rk45\"");
    if (p.precision != GRT_PREC_FP64 && p.precision != GRT_PREC_MIXED)
        throw std::runtime_error("precision must be GRT_PREC_FP64 or GRT_PREC_MIXED");
}

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
    try {
        validate_or_throw(*p);
    } catch (const std::exception& e) {
        set_err(err, err_len, e.what());
        return GRT_EINVAL;
    }
    return GRT_OK;
}

grt_status grt_params_from_toml(const char* path, grt_params* p, char* numpy_dir, size_t numpy_dir_len,
                                char* output_dir, size_t output_dir_len, char* name, size_t name_len,
                                char* err, size_t err_len) {
    if (!path || !p) {
        set_err(err, err_len, "null argument");
        return GRT_EINVAL;
    }
    grt_params q;
    grt_params_default(&q);
    try {
        const Raw c = parse_flat(path);
        const std::string mode = get_str(c, "simulation.mode", "image");
        if (mode == "image") q.mode = GRT_MODE_IMAGE;
        else if (mode == "disk") q.mode = GRT_MODE_DISK;
        else throw std::runtime_error("simulation.mode must be 'image' or 'disk'");
        const std::string sim_name = get_str(c, "simulation.name", "output");
        const std::string npdir = get_str(c, "input.numpy_dir", ".");
        q.scattering_enabled = get_bool(c, "scattering.enabled", false);
        q.scattering_albedo = get_real(c, "scattering.albedo", q.scattering_albedo);
        q.scattering_seed = get_u64(c, "scattering.seed", q.scattering_seed);
        q.absorption_enabled = get_bool(c, "radiative_transfer.absorption_enabled", false);
        q.emission_enabled = get_bool(c, "radiative_transfer.emission_enabled", false);
        q.absorption_coefficient = get_real(c, "radiative_transfer.absorption_coefficient", 0.0);
        q.emission_coefficient = get_real(c, "radiative_transfer.emission_coefficient", 0.0);
        const std::string integ = get_str(c, "integration.integrator", "rk45");
        if (integ == "rk4") q.integrator = GRT_RK4;
        else if (integ == "rk45") q.integrator = GRT_RK45;
        else throw std::runtime_error("integration.integrator must be \"rk4\" or \"rk45\"");
        q.mass = get_real(c, "black_hole.mass", q.mass);
        q.spin = get_real(c, "black_hole.spin", q.spin);
        if (q.mass <= 0.0) throw std::runtime_error("black_hole.mass must be positive (got " + std::to_string(q.mass) + ")");
        if (std::fabs(q.spin) > q.mass)
            throw std::runtime_error("black_hole.spin must satisfy |spin| <= mass, i.e. dimensionless spin a/M in [-1, 1] (got spin=" +
                                     std::to_string(q.spin) + ", mass=" + std::to_string(q.mass) +
                                     "); |spin| > mass is a naked singularity.");
        const double horizon = q.mass + std::sqrt(std::fmax(0.0, q.mass * q.mass - q.spin * q.spin));
        q.camera_theta = get_real(c, "camera.theta", q.camera_theta);
        q.camera_phi = get_real(c, "camera.phi", q.camera_phi);
        q.camera_width = get_real(c, "camera.width", q.camera_width);
        q.camera_height = get_real(c, "camera.height", q.camera_height);
        q.camera_distance = get_real(c, "camera.distance", q.camera_distance);
        q.nphotons = get_u64(c, "photons.count", q.nphotons);
        q.generator = parse_generator(get_str(c, "photons.generator", "blackbody"));
        q.superphoton_count_normalization = get_real(c, "photons.superphoton_count_normalization", q.superphoton_count_normalization);
        q.energy_per_cell_erg = get_real(c, "photons.energy_per_cell_erg", q.energy_per_cell_erg);
        q.power_law_slope = get_real(c, "photons.power_law_slope", q.power_law_slope);
        q.nu_min_hz = get_real(c, "photons.nu_min_hz", q.nu_min_hz);
        q.nu_max_hz = get_real(c, "photons.nu_max_hz", q.nu_max_hz);
        q.custom_frequency_hz = get_real(c, "photons.custom_frequency_hz", q.custom_frequency_hz);
        q.length_cm_per_code = get_real(c, "units.length_cm_per_code", q.length_cm_per_code);
        q.time_s_per_code = get_real(c, "units.time_s_per_code", q.time_s_per_code);
        q.density_g_cm3_per_code = get_real(c, "units.density_g_cm3_per_code", q.density_g_cm3_per_code);
        q.temperature_k_per_code = get_real(c, "units.temperature_k_per_code", q.temperature_k_per_code);
        q.four_velocity_cm_s_per_code = get_real(c, "units.four_velocity_cm_s_per_code", q.four_velocity_cm_s_per_code);
        q.magnetic_gauss_per_code = get_real(c, "units.magnetic_gauss_per_code", q.magnetic_gauss_per_code);
        q.max_steps = get_int(c, "integration.max_steps", static_cast<int>(q.max_steps));
        q.termination_percent = get_real(c, "integration.termination_percent", q.termination_percent);
        q.initial_step = get_real(c, "integration.initial_step", q.initial_step);
        q.atol = get_real(c, "integration.atol", q.atol);
        q.rtol = get_real(c, "integration.rtol", q.rtol);
        q.r_term_min = get_real(c, "termination.r_min", horizon);
        q.r_term_max = get_real(c, "termination.r_max", 1.5 * q.camera_distance);
        q.output_interval = get_u64(c, "output.interval", q.output_interval);
        const std::string outdir = get_str(c, "output.directory", "./output");
        q.image_nx = get_u64(c, "output.image_nx", q.image_nx);
        q.image_ny = get_u64(c, "output.image_ny", q.image_ny);
        q.spectrum_bins = get_u64(c, "output.spectrum_bins", q.spectrum_bins);
        q.spectrum_min_hz = get_real(c, "output.spectrum_min_hz", q.spectrum_min_hz);
        q.spectrum_max_hz = get_real(c, "output.spectrum_max_hz", q.spectrum_max_hz);
        if (npdir.empty()) throw std::runtime_error("input.numpy_dir must not be empty");
        if (outdir.empty()) throw std::runtime_error("output.directory must not be empty");
        if (sim_name.empty()) throw std::runtime_error("simulation.name must not be empty");
        validate_or_throw(q);
        set_str(numpy_dir, numpy_dir_len, npdir);
        set_str(output_dir, output_dir_len, outdir);
        set_str(name, name_len, sim_name);
    } catch (const std::runtime_error& e) {
        set_err(err, err_len, e.what());
        return std::string(e.what()).rfind("Failed to open config file", 0) == 0 ? GRT_EIO : GRT_EINVAL;
    } catch (const std::exception& e) {
        set_err(err, err_len, std::string("invalid config value: ") + e.what());
        return GRT_EINVAL;
    }
    *p = q;
    return GRT_OK;
}

grt_status grt_output_options_from_toml(const char* path, char* variables, size_t variables_len, uint64_t* stride,
                                        char* err, size_t err_len) {
    if (!path) {
        set_err(err, err_len, "null argument");
        return GRT_EINVAL;
    }
    try {
        const Raw c = parse_flat(path);
        const std::string spec = get_str(c, "output.variables", "id,frequency,x0,x1,x2,x3,k0,k1,k2,k3,I,Q,U,V,phase");
        const uint64_t st = get_u64(c, "output.stride", 1);
        if (st == 0) throw std::runtime_error("output.stride must be positive");
        std::vector<int> fields;
        std::string msg;
        if (!grt::parse_output_variables(spec, fields, msg)) throw std::runtime_error(msg);
        if (variables && variables_len) {
            if (spec.size() + 1 > variables_len) throw std::runtime_error("output.variables longer than the buffer");
            set_str(variables, variables_len, spec);
        }
        if (stride) *stride = st;
    } catch (const std::runtime_error& e) {
        set_err(err, err_len, e.what());
        return std::string(e.what()).rfind("Failed to open config file", 0) == 0 ? GRT_EIO : GRT_EINVAL;
    } catch (const std::exception& e) {
        set_err(err, err_len, std::string("invalid config value: ") + e.what());
        return GRT_EINVAL;
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
