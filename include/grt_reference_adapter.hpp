/*
 * Drop-in for the reference's integrate_geodesics
 * (src/geodesic_integrate/integrate_cart_ks.hpp:423-535), for the reference's
 * own C++ build.  Include it after the reference's headers (utils.hpp,
 * simulation_options.hpp, input/load_python_arrays.hpp, output/write_output.hpp,
 * radiative_transfer/ *.hpp) and call integrate_geodesics_b200 where main()
 * calls integrate_geodesics (src/main.cpp:246-266); link libgrt_b200.so.
 *
 * It takes exactly what the reference's step loop takes -- the parsed
 * SimulationOptions / PhotonGenerationConfig / UnitConversions, the models,
 * the reference's runtime globals (src/utils.cpp:4-37), the loaded
 * NumpyFieldViews and the Photons views -- and maps them onto the C ABI of
 * grt.h: grt_params, the seven grid arrays in C order, the photon
 * structure-of-arrays.  The step loop then runs on the GPU through
 * grt_run_with_output, which writes the same output-step archives and image
 * products the reference writes, and the final photon state is copied back
 * into the caller's Photons views.  No TOML is parsed here: the reference's
 * own loader stays in charge of the config.
 *
 * One rank: the B200 path holds the whole grid on one GPU, so a run over
 * several MPI ranks is refused with std::runtime_error (split the photons over
 * GPUs instead: grt_init_image_rows and a reduce of the image products, the
 * analogue of write_output.hpp:116-127).
 */
#pragma once

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "grt.h"

namespace grt_adapter {

/* grt_params from the reference's globals and parsed structs -- the values the
 * step functor receives (integrate_cart_ks.hpp:63-94, 471-476). */
inline grt_params params_from_reference(const SimulationOptions& options, const PhotonGenerationConfig& generation,
                                        const UnitConversions& units, const ScatteringModel& scattering,
                                        const RadiativeTransferModel& transfer, IntegratorType integrator, int rank) {
    grt_params p;
    std::memset(&p, 0, sizeof(p));  // every field is set below
    p.mode = options.mode == SimulationMode::Image ? GRT_MODE_IMAGE : GRT_MODE_DISK;
    p.integrator = integrator == IntegratorType::RK4 ? GRT_RK4 : GRT_RK45;
    p.precision = GRT_PREC_FP64;
    switch (generation.generator) {
        case PhotonGeneratorType::PowerLaw: p.generator = GRT_GEN_POWER_LAW; break;
        case PhotonGeneratorType::Custom: p.generator = GRT_GEN_CUSTOM; break;
        default: p.generator = GRT_GEN_BLACKBODY; break;
    }
    p.mass = M_BH;
    p.spin = a_BH;
    p.r_term_min = termination_r_min;
    p.r_term_max = termination_r_max;
    p.atol = atol_default;
    p.rtol = rtol_default;
    p.min_step_scale = min_scale;
    p.max_step_scale = max_scale;
    p.safety = safety;
    p.max_steps = max_steps;
    p.termination_percent = termination_percent;
    p.output_interval = output_interval;
    p.nphotons = nphotons;
    p.initial_step = dlambda;
    p.camera_distance = camera_distance;
    p.camera_theta = camera_theta;
    p.camera_phi = camera_phi;
    p.camera_width = plane_dim1;
    p.camera_height = plane_dim2;
    p.absorption_enabled = transfer.absorption_enabled ? 1 : 0;
    p.emission_enabled = transfer.emission_enabled ? 1 : 0;
    p.absorption_coefficient = transfer.absorption_coefficient;
    p.emission_coefficient = transfer.emission_coefficient;
    p.scattering_enabled = scattering.enabled ? 1 : 0;
    p.scattering_albedo = scattering.albedo;
    p.scattering_seed = scattering.seed;
    p.rank = rank;
    p.superphoton_count_normalization = generation.superphoton_count_normalization;
    p.energy_per_cell_erg = generation.energy_per_cell_erg;
    p.power_law_slope = generation.power_law_slope;
    p.nu_min_hz = generation.nu_min_hz;
    p.nu_max_hz = generation.nu_max_hz;
    p.custom_frequency_hz = generation.custom_frequency_hz;
    p.length_cm_per_code = units.length_cm_per_code;
    p.time_s_per_code = units.time_s_per_code;
    p.density_g_cm3_per_code = units.density_g_cm3_per_code;
    p.temperature_k_per_code = units.temperature_k_per_code;
    p.four_velocity_cm_s_per_code = units.four_velocity_cm_s_per_code;
    p.magnetic_gauss_per_code = units.magnetic_gauss_per_code;
    p.image_nx = options.image_nx;
    p.image_ny = options.image_ny;
    p.spectrum_bins = options.spectrum_bins;
    p.spectrum_min_hz = options.spectrum_min_hz;
    p.spectrum_max_hz = options.spectrum_max_hz;
    return p;
}

/* A (n0, n1, n2) or (n0, n1, n2, n3) view as one C-order float64 array (the
 * reference reads its grid layout-agnostically through host mirrors,
 * load_python_arrays.hpp:126-144). */
template <int Rank, class View>
std::vector<double> c_order(const View& v) {
    auto h = Kokkos::create_mirror_view(v);
    Kokkos::deep_copy(h, v);
    const std::size_t n0 = v.extent(0), n1 = v.extent(1), n2 = v.extent(2);
    const std::size_t n3 = Rank == 4 ? v.extent(3) : 1;
    std::vector<double> out(n0 * n1 * n2 * n3);
    std::size_t q = 0;
    for (std::size_t i = 0; i < n0; ++i)
        for (std::size_t j = 0; j < n1; ++j)
            for (std::size_t k = 0; k < n2; ++k)
                for (std::size_t c = 0; c < n3; ++c) {
                    if constexpr (Rank == 4) out[q++] = h(i, j, k, c);
                    else out[q++] = h(i, j, k);
                }
    return out;
}

/* Host staging of the 20 photon views (struct Photons, utils.hpp:40-133). */
struct PhotonStage {
    std::vector<std::uint64_t> id;
    std::vector<double> f[17];  // frequency .. phi_disp in grt_photon_soa order
    std::vector<std::uint8_t> terminate, phase;
    grt_photon_soa soa{};

    explicit PhotonStage(std::size_t n) : id(n), terminate(n), phase(n) {
        for (auto& v : f) v.resize(n);
        soa.id = id.data();
        double** d[17] = {&soa.frequency, &soa.emission_frame_energy, &soa.x0, &soa.x1, &soa.x2, &soa.x3,
                          &soa.k0,        &soa.k1, &soa.k2, &soa.k3, &soa.I,  &soa.Q,  &soa.U,
                          &soa.V,         &soa.dlambda, &soa.theta_disp, &soa.phi_disp};
        for (int k = 0; k < 17; ++k) *d[k] = f[k].data();
        soa.terminate = terminate.data();
        soa.phase = phase.data();
    }
};

template <class F>
void for_each_real_view(Photons& ph, F&& fn) {
    fn(0, ph.frequency); fn(1, ph.emission_frame_energy);
    fn(2, ph.x0); fn(3, ph.x1); fn(4, ph.x2); fn(5, ph.x3);
    fn(6, ph.k0); fn(7, ph.k1); fn(8, ph.k2); fn(9, ph.k3);
    fn(10, ph.I); fn(11, ph.Q); fn(12, ph.U); fn(13, ph.V);
    fn(14, ph.dlambda); fn(15, ph.theta_disp); fn(16, ph.phi_disp);
}

inline void photons_to_stage(Photons& ph, PhotonStage& s) {
    const std::size_t n = ph.x0.extent(0);
    {
        auto h = Kokkos::create_mirror_view(ph.id);
        Kokkos::deep_copy(h, ph.id);
        for (std::size_t i = 0; i < n; ++i) s.id[i] = h(i);
    }
    for_each_real_view(ph, [&](int k, auto& v) {
        auto h = Kokkos::create_mirror_view(v);
        Kokkos::deep_copy(h, v);
        for (std::size_t i = 0; i < n; ++i) s.f[k][i] = h(i);
    });
    auto ht = Kokkos::create_mirror_view(ph.terminate);
    auto hp = Kokkos::create_mirror_view(ph.phase);
    Kokkos::deep_copy(ht, ph.terminate);
    Kokkos::deep_copy(hp, ph.phase);
    for (std::size_t i = 0; i < n; ++i) {
        s.terminate[i] = ht(i) ? 1 : 0;
        s.phase[i] = hp(i);
    }
}

inline void stage_to_photons(const PhotonStage& s, Photons& ph) {
    const std::size_t n = ph.x0.extent(0);
    {
        auto h = Kokkos::create_mirror_view(ph.id);
        for (std::size_t i = 0; i < n; ++i) h(i) = s.id[i];
        Kokkos::deep_copy(ph.id, h);
    }
    for_each_real_view(ph, [&](int k, auto& v) {
        auto h = Kokkos::create_mirror_view(v);
        for (std::size_t i = 0; i < n; ++i) h(i) = s.f[k][i];
        Kokkos::deep_copy(v, h);
    });
    auto ht = Kokkos::create_mirror_view(ph.terminate);
    auto hp = Kokkos::create_mirror_view(ph.phase);
    for (std::size_t i = 0; i < n; ++i) {
        ht(i) = s.terminate[i] != 0;
        hp(i) = s.phase[i];
    }
    Kokkos::deep_copy(ph.terminate, ht);
    Kokkos::deep_copy(ph.phase, hp);
}

/* Throw with the library's message (and release the context) on failure. */
inline void check(grt_ctx*& ctx, grt_status st, const char* what) {
    if (st == GRT_OK) return;
    const std::string msg = std::string(what) + ": " + (ctx ? grt_last_error(ctx) : "could not create a context");
    if (ctx) grt_destroy(ctx);
    ctx = nullptr;
    throw std::runtime_error(msg);
}

}  // namespace grt_adapter

/* The reference's integrate_geodesics, same arguments, on the GPU. */
inline void integrate_geodesics_b200(Photons& photons, const NumpyFieldViews& fields, const UnitConversions& units,
                                     const int rank, Timers& timers, const OutputSelection& output_selection,
                                     const SimulationOptions& options, const PhotonGenerationConfig& photon_generation,
                                     const ScatteringModel& scattering_model = ScatteringModel{},
                                     const RadiativeTransferModel& radiative_transfer_model = RadiativeTransferModel{},
                                     IntegratorType integrator = IntegratorType::RK45) {
    int mpi_size = 1;
    MPI_Comm_size(MPI_COMM_WORLD, &mpi_size);
    if (mpi_size > 1)
        throw std::runtime_error("integrate_geodesics_b200 runs on one rank: the B200 path holds the whole grid "
                                 "on one GPU (split photons over GPUs instead)");
    const grt_params p = grt_adapter::params_from_reference(options, photon_generation, units, scattering_model,
                                                            radiative_transfer_model, integrator, rank);
    grt_ctx* ctx = nullptr;
    grt_adapter::check(ctx, grt_create(&p, &ctx), "grt_create");
    // the grid, unless it is empty (vacuum): the library gates transfer and
    // scattering on its presence, as the reference gates them on fluid_available
    const std::size_t nr = fields.r.extent(0), nth = fields.r.extent(1), nph = fields.r.extent(2);
    if (nr * nth * nph > 0 && fields.density.extent(0) > 0) {
        const auto r = grt_adapter::c_order<3>(fields.r), th = grt_adapter::c_order<3>(fields.theta);
        const auto ph = grt_adapter::c_order<3>(fields.phi), rho = grt_adapter::c_order<3>(fields.density);
        const auto T = grt_adapter::c_order<3>(fields.temperature);
        const auto vel = grt_adapter::c_order<4>(fields.velocity), mag = grt_adapter::c_order<4>(fields.magnetic);
        grt_adapter::check(ctx, grt_upload_grid(ctx, nr, nth, nph, r.data(), th.data(), ph.data(), rho.data(),
                                                T.data(), vel.data(), mag.data()), "grt_upload_grid");
    } else {
        grt_adapter::check(ctx, grt_upload_grid(ctx, 0, 0, 0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                                nullptr), "grt_upload_grid");
    }
    const std::size_t n = photons.x0.extent(0);
    grt_adapter::PhotonStage stage(n);
    grt_adapter::photons_to_stage(photons, stage);
    grt_adapter::check(ctx, grt_upload_photons(ctx, &stage.soa, n), "grt_upload_photons");
    std::string variables;
    for (const std::string& name : output_selection.names()) variables += (variables.empty() ? "" : ",") + name;
    timers.AddTimer("Geodesic Integration");
    timers.BeginTimer("Geodesic Integration");
    grt_run_stats st;
    grt_adapter::check(ctx, grt_run_with_output(ctx, output_directory.c_str(), simulation_name.c_str(),
                                                variables.c_str(), output_stride, &st), "grt_run_with_output");
    timers.EndTimer("Geodesic Integration");
    grt_adapter::check(ctx, grt_download_photons(ctx, &stage.soa), "grt_download_photons");
    grt_destroy(ctx);
    grt_adapter::stage_to_photons(stage, photons);
}
