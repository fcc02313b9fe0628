// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// Drives the reference GR-ray-tracer's own, unmodified code (compiled from the
// reference source tree against oracle/shim) through a C entry point, so the
// tests and the CPU baseline can run the reference's step loop on the same
// inputs as the sm_100a kernels:
//   * the reference's TOML loader      src/input/toml_config.hpp:129-278
//   * the reference's NumPy loader     src/input/load_python_arrays.hpp:195-223
//   * the reference's step loop        src/geodesic_integrate/integrate_cart_ks.hpp:423-535
//   * the reference's image products   src/radiative_transfer/observation.hpp:31-84
// The only project-written physics here is the deterministic pixel-grid camera
// initialisation, which follows initialize_photons_image
// (src/radiative_transfer/initialize_photons.hpp:82-170) with the random screen
// draw replaced by pixel centres, calling the reference's own
// null_covariant_momentum_from_spatial_direction.

#include "utils.hpp"
#include "simulation_options.hpp"
#include "input/load_python_arrays.hpp"
#include "input/toml_config.hpp"
#include "radiative_transfer/initialize_photons.hpp"
#include "geodesic_integrate/integrate_cart_ks.hpp"
#include "analysis/geodesic_observables.hpp"
#include "output/write_output.hpp"

#include <chrono>
#include <cstring>
#include <iostream>
#include <sstream>

#include "grt.h"
#include "grt_reference_adapter.hpp"  // the product's drop-in mapping, checked below

namespace {

struct GlobalDefaults {
    real M, a, RH, cth, cph, w, h, D;
    std::uint64_t n;
    int steps;
    real pct, rmin, rmax, dl, atol, rtol;
    size_t interval, stride;
    std::string outdir, name;
};

// Snapshot of the reference's compiled-in globals (src/utils.cpp:4-37), taken
// before any config is applied, so every call starts from the same defaults
// (the reference's loader only overwrites keys present in the file).
GlobalDefaults& defaults() {
    static GlobalDefaults d{M_BH, a_BH, R_HORIZON, camera_theta, camera_phi, plane_dim1, plane_dim2,
                            camera_distance, nphotons, max_steps, termination_percent,
                            termination_r_min, termination_r_max, dlambda, atol_default,
                            rtol_default, output_interval, output_stride, output_directory,
                            simulation_name};
    return d;
}

void restore_defaults() {
    const GlobalDefaults& d = defaults();
    M_BH = d.M; a_BH = d.a; R_HORIZON = d.RH;
    camera_theta = d.cth; camera_phi = d.cph; plane_dim1 = d.w; plane_dim2 = d.h;
    camera_distance = d.D; nphotons = d.n; max_steps = d.steps;
    termination_percent = d.pct; termination_r_min = d.rmin; termination_r_max = d.rmax;
    dlambda = d.dl; atol_default = d.atol; rtol_default = d.rtol;
    output_interval = d.interval; output_stride = d.stride;
    output_directory = d.outdir; simulation_name = d.name;
}

struct Loaded {
    SimulationOptions options;
    std::string output_variables{default_output_variables};
    PhotonGenerationConfig generation;
    UnitConversions units;
    DomainDecompositionSpec decomposition;
};

std::string g_error;

bool load_config(const char* toml_path, Loaded& cfg) {
    try {
        (void)defaults();
        restore_defaults();
        toml_config::load_and_apply_toml_config(toml_path, cfg.options, cfg.output_variables,
                                                cfg.generation, cfg.units, cfg.decomposition);
        output_directory = cfg.options.output_dir;
        cfg.generation.validate();
        cfg.units.validate();
        return true;
    } catch (const std::exception& e) {
        g_error = e.what();
        return false;
    }
}

void to_soa(Photons& photons, grt_photon_soa* out) {
    const std::size_t n = photons.x0.extent(0);
    for (std::size_t i = 0; i < n; ++i) {
        out->id[i] = photons.id(i);
        out->frequency[i] = photons.frequency(i);
        out->emission_frame_energy[i] = photons.emission_frame_energy(i);
        out->x0[i] = photons.x0(i); out->x1[i] = photons.x1(i);
        out->x2[i] = photons.x2(i); out->x3[i] = photons.x3(i);
        out->k0[i] = photons.k0(i); out->k1[i] = photons.k1(i);
        out->k2[i] = photons.k2(i); out->k3[i] = photons.k3(i);
        out->I[i] = photons.I(i); out->Q[i] = photons.Q(i);
        out->U[i] = photons.U(i); out->V[i] = photons.V(i);
        out->dlambda[i] = photons.dlambda(i);
        out->theta_disp[i] = photons.theta_disp(i);
        out->phi_disp[i] = photons.phi_disp(i);
        out->terminate[i] = photons.terminate(i) ? 1 : 0;
        out->phase[i] = photons.phase(i);
    }
}

void from_soa(const grt_photon_soa* in, Photons& photons) {
    const std::size_t n = photons.x0.extent(0);
    for (std::size_t i = 0; i < n; ++i) {
        photons.id(i) = in->id[i];
        photons.frequency(i) = in->frequency[i];
        photons.emission_frame_energy(i) = in->emission_frame_energy[i];
        photons.x0(i) = in->x0[i]; photons.x1(i) = in->x1[i];
        photons.x2(i) = in->x2[i]; photons.x3(i) = in->x3[i];
        photons.k0(i) = in->k0[i]; photons.k1(i) = in->k1[i];
        photons.k2(i) = in->k2[i]; photons.k3(i) = in->k3[i];
        photons.I(i) = in->I[i]; photons.Q(i) = in->Q[i];
        photons.U(i) = in->U[i]; photons.V(i) = in->V[i];
        photons.dlambda(i) = in->dlambda[i];
        photons.theta_disp(i) = in->theta_disp[i];
        photons.phi_disp(i) = in->phi_disp[i];
        photons.terminate(i) = in->terminate[i] != 0;
        photons.phase(i) = in->phase[i];
    }
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_error.c_str(); }

// Fill p from the reference's own TOML loader (the globals it mutates and the
// structs it fills), so tests can check the product's TOML mirror against it.
int ref_params_from_toml(const char* toml_path, grt_params* p) {
    Loaded cfg;
    if (!load_config(toml_path, cfg)) return 1;
    std::memset(p, 0, sizeof(*p));
    p->mode = cfg.options.mode == SimulationMode::Image ? GRT_MODE_IMAGE : GRT_MODE_DISK;
    p->integrator = cfg.options.integrator == IntegratorType::RK4 ? GRT_RK4 : GRT_RK45;
    p->precision = GRT_PREC_FP64;
    p->generator = static_cast<int32_t>(cfg.generation.generator);
    p->mass = M_BH; p->spin = a_BH;
    p->r_term_min = termination_r_min; p->r_term_max = termination_r_max;
    p->atol = atol_default; p->rtol = rtol_default;
    p->min_step_scale = min_scale; p->max_step_scale = max_scale; p->safety = safety;
    p->max_steps = max_steps;
    p->termination_percent = termination_percent;
    p->output_interval = output_interval;
    p->nphotons = nphotons;
    p->initial_step = dlambda;
    p->camera_distance = camera_distance; p->camera_theta = camera_theta;
    p->camera_phi = camera_phi; p->camera_width = plane_dim1; p->camera_height = plane_dim2;
    p->absorption_enabled = cfg.options.enable_absorption;
    p->emission_enabled = cfg.options.enable_emission;
    p->absorption_coefficient = cfg.options.absorption_coefficient;
    p->emission_coefficient = cfg.options.emission_coefficient;
    p->scattering_enabled = cfg.options.enable_scattering;
    p->scattering_albedo = cfg.options.scattering_albedo;
    p->scattering_seed = cfg.options.scattering_seed;
    p->superphoton_count_normalization = cfg.generation.superphoton_count_normalization;
    p->energy_per_cell_erg = cfg.generation.energy_per_cell_erg;
    p->power_law_slope = cfg.generation.power_law_slope;
    p->nu_min_hz = cfg.generation.nu_min_hz; p->nu_max_hz = cfg.generation.nu_max_hz;
    p->custom_frequency_hz = cfg.generation.custom_frequency_hz;
    p->length_cm_per_code = cfg.units.length_cm_per_code;
    p->time_s_per_code = cfg.units.time_s_per_code;
    p->density_g_cm3_per_code = cfg.units.density_g_cm3_per_code;
    p->temperature_k_per_code = cfg.units.temperature_k_per_code;
    p->four_velocity_cm_s_per_code = cfg.units.four_velocity_cm_s_per_code;
    p->magnetic_gauss_per_code = cfg.units.magnetic_gauss_per_code;
    p->image_nx = cfg.options.image_nx; p->image_ny = cfg.options.image_ny;
    p->spectrum_bins = cfg.options.spectrum_bins;
    p->spectrum_min_hz = cfg.options.spectrum_min_hz;
    p->spectrum_max_hz = cfg.options.spectrum_max_hz;
    return 0;
}

// The product's drop-in mapping (grt_adapter::params_from_reference in
// include/grt_reference_adapter.hpp) of what the reference's loader fills,
// with the models main() builds from it (src/main.cpp:246-266), to compare
// with ref_params_from_toml.
int ref_adapter_params_from_toml(const char* toml_path, grt_params* p) {
    Loaded cfg;
    if (!load_config(toml_path, cfg)) return 1;
    *p = grt_adapter::params_from_reference(
        cfg.options, cfg.generation, cfg.units,
        ScatteringModel{cfg.options.enable_scattering, cfg.options.scattering_albedo, cfg.options.scattering_seed},
        RadiativeTransferModel{cfg.options.enable_absorption, cfg.options.enable_emission,
                               cfg.options.absorption_coefficient, cfg.options.emission_coefficient},
        cfg.options.integrator, 0);
    return 0;
}

// Pixel-grid camera rays through the reference's formulas
// (initialize_photons.hpp:94-168, screen (u,v) at pixel centres).
int ref_init_image_photons(const char* toml_path, std::uint64_t nx, std::uint64_t ny,
                           std::uint64_t id_offset, grt_photon_soa* out) {
    Loaded cfg;
    if (!load_config(toml_path, cfg)) return 1;
    const real cx = camera_distance * Kokkos::sin(camera_theta) * Kokkos::cos(camera_phi);
    const real cy = camera_distance * Kokkos::sin(camera_theta) * Kokkos::sin(camera_phi);
    const real cz = camera_distance * Kokkos::cos(camera_theta);
    const real theta_hat[3] = {Kokkos::cos(camera_theta) * Kokkos::cos(camera_phi),
                               Kokkos::cos(camera_theta) * Kokkos::sin(camera_phi),
                               -Kokkos::sin(camera_theta)};
    const real phi_hat[3] = {-Kokkos::sin(camera_phi), Kokkos::cos(camera_phi), 0.0};
    for (std::uint64_t iy = 0; iy < ny; ++iy) {
        for (std::uint64_t ix = 0; ix < nx; ++ix) {
            const std::uint64_t i = iy * nx + ix;
            const real screen_u = -0.5 * plane_dim1 + (static_cast<real>(ix) + 0.5) * plane_dim1 / static_cast<real>(nx);
            const real screen_v = -0.5 * plane_dim2 + (static_cast<real>(iy) + 0.5) * plane_dim2 / static_cast<real>(ny);
            const real x = cx + screen_u * theta_hat[0] + screen_v * phi_hat[0];
            const real y = cy + screen_u * theta_hat[1] + screen_v * phi_hat[1];
            const real z = cz + screen_u * theta_hat[2] + screen_v * phi_hat[2];
            real kx = -cx, ky = -cy, kz = -cz;
            const real k_norm = Kokkos::sqrt(kx * kx + ky * ky + kz * kz);
            kx /= k_norm; ky /= k_norm; kz /= k_norm;
            const real X[4] = {0.0, x, y, z};
            const real K[3] = {kx, ky, kz};
            real p_cov[4] = {0.0, 0.0, 0.0, 0.0};
            kerr_schild::null_covariant_momentum_from_spatial_direction(X, K, a_BH, M_BH, p_cov);
            out->id[i] = id_offset + i;
            out->frequency[i] = 0.0;
            out->emission_frame_energy[i] = 1.0;
            out->x0[i] = 0.0; out->x1[i] = x; out->x2[i] = y; out->x3[i] = z;
            out->k0[i] = p_cov[0]; out->k1[i] = p_cov[1]; out->k2[i] = p_cov[2]; out->k3[i] = p_cov[3];
            out->I[i] = out->Q[i] = out->U[i] = out->V[i] = 0.0;
            out->dlambda[i] = dlambda * camera_distance;
            out->terminate[i] = 0;
            out->phase[i] = static_cast<std::uint8_t>(PhotonPhase::ImageBackward);
            out->theta_disp[i] = screen_u;
            out->phi_disp[i] = screen_v;
        }
    }
    return 0;
}

// The reference's own initialize_photons_image
// (src/radiative_transfer/initialize_photons.hpp:82-170) with its random
// screen draw, on rank 0 of 1, through the shim's random pool (its own
// XorShift streams, not Kokkos's): n photons with ids id_offset + i.
int ref_init_image_photons_random(const char* toml_path, std::uint64_t n, std::uint64_t id_offset,
                                  grt_photon_soa* out) {
    Loaded cfg;
    if (!load_config(toml_path, cfg)) return 1;
    try {
        Photons photons(static_cast<int>(n), "photons_");
        initialize_photons_image(static_cast<int>(n), camera_distance, camera_theta, camera_phi, 0, 1, id_offset,
                                 photons);
        to_soa(photons, out);
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 2;
    }
}

// Run the reference's integrate_geodesics on n caller-provided photons (in
// place), with the grid from the config's input.numpy_dir (numpy_dir_override
// replaces it when non-NULL) and output archives under output_dir.  When
// products is non-NULL, fills it with build_observation_products of the final
// photons.  elapsed_s = wall time of integrate_geodesics; stepped = functor
// invocations that advanced a photon.
int ref_run_photons(const char* toml_path, const char* numpy_dir_override, const char* output_dir,
                    grt_photon_soa* soa, std::uint64_t n, grt_image_products* products,
                    double* elapsed_s, std::uint64_t* stepped, std::uint64_t* live_calls) {
    Loaded cfg;
    if (!load_config(toml_path, cfg)) return 1;
    try {
        if (numpy_dir_override) cfg.options.numpy_dir = numpy_dir_override;
        if (output_dir) {
            cfg.options.output_dir = output_dir;
            output_directory = output_dir;
        }
        const NumpyFieldPaths paths = discover_numpy_field_paths(cfg.options.numpy_dir);
        NumpyFieldViews fields = load_numpy_field_bundle(paths, cfg.decomposition, 0, 1);
        nphotons = n;
        Photons photons(static_cast<int>(n), "photons_");
        from_soa(soa, photons);
        Timers timers(output_interval);
        const OutputSelection selection = OutputSelection::parse(cfg.output_variables);
        Kokkos::shim_detail::stats() = {};
        std::streambuf* saved = std::cout.rdbuf();
        std::ostringstream sink;
        std::cout.rdbuf(sink.rdbuf());
        const auto t0 = std::chrono::steady_clock::now();
        integrate_geodesics(photons, fields, cfg.units, 0, timers, selection, cfg.options,
                            cfg.generation,
                            ScatteringModel{cfg.options.enable_scattering, cfg.options.scattering_albedo,
                                            cfg.options.scattering_seed},
                            RadiativeTransferModel{cfg.options.enable_absorption, cfg.options.enable_emission,
                                                   cfg.options.absorption_coefficient,
                                                   cfg.options.emission_coefficient},
                            cfg.options.integrator);
        const auto t1 = std::chrono::steady_clock::now();
        std::cout.rdbuf(saved);
        if (elapsed_s) *elapsed_s = std::chrono::duration<double>(t1 - t0).count();
        if (stepped) *stepped = Kokkos::shim_detail::stats().stepped_invocations;
        if (live_calls) *live_calls = Kokkos::shim_detail::stats().live_invocations;
        to_soa(photons, soa);
        if (products) {
            photons.copy_observation_to_host();
            const ObservationProducts obs = build_observation_products(
                photons, cfg.options.image_nx, cfg.options.image_ny, cfg.options.spectrum_bins,
                cfg.options.spectrum_min_hz, cfg.options.spectrum_max_hz, plane_dim1, plane_dim2);
            std::memcpy(products->image_I, obs.image_I.data(), obs.image_I.size() * sizeof(double));
            std::memcpy(products->image_Q, obs.image_Q.data(), obs.image_Q.size() * sizeof(double));
            std::memcpy(products->image_U, obs.image_U.data(), obs.image_U.size() * sizeof(double));
            std::memcpy(products->image_V, obs.image_V.data(), obs.image_V.size() * sizeof(double));
            std::memcpy(products->spectrum_frequency_hz, obs.spectrum_frequency_hz.data(),
                        obs.spectrum_frequency_hz.size() * sizeof(double));
            std::memcpy(products->spectrum_I, obs.spectrum_I.data(), obs.spectrum_I.size() * sizeof(double));
            products->arrived_count[0] = obs.arrived_count;
        }
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 2;
    }
}

// The reference's own disk-mode emission: build_superphoton_cell_offsets +
// initialize_photons_disk (src/radiative_transfer/initialize_photons.hpp:
// 32-64,173-327) on the config's grid, with the shim's random pool (its own
// XorShift streams, not Kokkos's).  out == NULL only counts the packets.
int ref_init_disk_photons(const char* toml_path, const char* numpy_dir_override, std::uint64_t id_offset,
                          grt_photon_soa* out, std::uint64_t* n_out) {
    Loaded cfg;
    if (!load_config(toml_path, cfg)) return 1;
    try {
        if (numpy_dir_override) cfg.options.numpy_dir = numpy_dir_override;
        const NumpyFieldPaths paths = discover_numpy_field_paths(cfg.options.numpy_dir);
        NumpyFieldViews fields = load_numpy_field_bundle(paths, cfg.decomposition, 0, 1);
        const SuperphotonCellOffsets offsets =
            build_superphoton_cell_offsets(fields.density, cfg.generation.superphoton_count_normalization);
        if (n_out) *n_out = offsets.total_photons;
        if (!out) return 0;
        Photons photons(static_cast<int>(offsets.total_photons), "photons_");
        initialize_photons_disk(static_cast<int>(offsets.total_photons), 0, id_offset, fields.r, fields.theta,
                                fields.phi, fields.density, fields.temperature, fields.velocity, fields.magnetic,
                                cfg.generation, cfg.units, offsets.offsets, photons);
        to_soa(photons, out);
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 2;
    }
}

// ---- reference functions exposed for known-answer checks ----
void ref_hamiltonian_rhs(const double X[4], const double p[4], double a, double M, double rhs[8]) {
    kerr_schild::compute_hamiltonian_rhs(X, p, a, M, rhs);
}
int ref_null_momentum(const double X[4], const double K[3], double a, double M, double p[4]) {
    return kerr_schild::null_covariant_momentum_from_spatial_direction(X, K, a, M, p) ? 1 : 0;
}
void ref_inverse_metric_deriv(const double X[4], double a, double M, double d[64]) {
    kerr_schild::compute_inverse_metric_deriv(X, a, M, reinterpret_cast<double(*)[4][4]>(d));
}
// Geodesic observables (src/analysis/geodesic_observables.hpp:7-35): norm, E, Lz, Carter.
void ref_geodesic_observables(const double state[8], double a, double M, double out[4]) {
    const GeodesicObservables o = compute_geodesic_observables(state, a, M);
    out[0] = o.norm; out[1] = o.energy; out[2] = o.angular_momentum_z; out[3] = o.carter;
}
int ref_locate_cell(std::size_t nr, std::size_t nth, std::size_t nph, const double* r,
                    const double* th, const double* ph, double radius, double polar, double azimuth,
                    int ijk[3]) {
    Kokkos::View<real***> R("r", nr, nth, nph), TH("t", nr, nth, nph), PH("p", nr, nth, nph);
    std::memcpy(R.data(), r, nr * nth * nph * sizeof(double));
    std::memcpy(TH.data(), th, nr * nth * nph * sizeof(double));
    std::memcpy(PH.data(), ph, nr * nth * nph * sizeof(double));
    int i = -1, j = -1, k = -1;
    const bool ok = locate_structured_grid_cell(R, TH, PH, radius, polar, azimuth, i, j, k);
    ijk[0] = i; ijk[1] = j; ijk[2] = k;
    return ok ? 1 : 0;
}

// OutputSelection::parse of the reference (src/output/output_variables.hpp:
// 27-70): the selected fields as indices into available_output_variables, in
// the order the reference writes them (fields has room for 40).  Returns 0, or
// 1 with the message.
int ref_parse_output_variables(const char* spec, int32_t* fields, size_t* count) {
    try {
        const OutputSelection sel = OutputSelection::parse(spec);
        size_t k = 0;
        if (sel.names().size() > 40) throw std::runtime_error("more than 40 selected fields");
        for (const std::string& name : sel.names()) {
            int idx = 0;
            while (available_output_variables[idx] != name) ++idx;
            fields[k++] = idx;
        }
        *count = k;
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

}  // extern "C"
