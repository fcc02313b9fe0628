/*
 * User-editable physics extension points of the per-photon hot path.
 *
 * These are the reference's user-editable device functions, with the same
 * names, argument lists and default bodies:
 *   ComputeOpticalDepthIncrement  src/radiative_transfer/radiative_transfer.hpp:61-67
 *   ComputeEmissivityIncrement    src/radiative_transfer/radiative_transfer.hpp:69-75
 *   GeneratePhotonsCustom         src/radiative_transfer/photon_generation.hpp:147-155
 *   ComputeSuperphotonsPerCell    src/radiative_transfer/initialize_photons.hpp:16-19
 * and the FluidCellCGS record they receive (photon_generation.hpp:87-97).
 *
 * Edit the bodies here exactly as you would in the reference.  This one header
 * is compiled __host__ __device__: the same body is built into the sm_100a trace
 * kernels and into the CPU oracle used by the parity tests, so a custom model
 * stays checkable.  The bodies must be pure functions of their arguments.
 *
 * RandomGenerator is any type with `double drand()` returning a uniform draw
 * in [0,1) (a counter-based Philox stream in this build).
 */
#ifndef GRT_USER_PHYSICS_H
#define GRT_USER_PHYSICS_H

#include <math.h>

#if defined(__CUDACC__)
#define GRT_HD __host__ __device__ __forceinline__
#else
#define GRT_HD inline
#endif

namespace grt {

typedef double real;

/* Fluid sample handed to the extension points (CGS units). */
struct FluidCellCGS {
    real position_cm[3] = {0.0, 0.0, 0.0};
    real coordinate_time_s = 0.0;
    real density_g_cm3 = 0.0;
    real temperature_k = 0.0;
    /* Orthonormal components in the fluid tetrad. */
    real magnetic_gauss[4] = {0.0, 0.0, 0.0, 0.0};
    /* Cartesian Kerr-Schild coordinate components, cm/s. */
    real coordinate_four_velocity_cm_s[4] = {1.0, 0.0, 0.0, 0.0};
};

/* Optical depth dtau >= 0 accumulated over one step (absorption only). */
GRT_HD real ComputeOpticalDepthIncrement(const FluidCellCGS& fluid, real frequency_hz,
                                         real path_length_step, real absorption_coefficient) {
    (void)frequency_hz;
    return fmax(real(0.0),
                absorption_coefficient * fluid.density_g_cm3 * fabs(path_length_step));
}

/* Intensity added to Stokes I over one step (emission only). */
GRT_HD real ComputeEmissivityIncrement(const FluidCellCGS& fluid, real frequency_hz,
                                       real path_length_step, real emission_coefficient) {
    (void)frequency_hz;
    return fmax(real(0.0), emission_coefficient * fluid.density_g_cm3 *
                               fluid.temperature_k * fabs(path_length_step));
}

/* Superphotons emitted from a cell with the given code-unit density. */
GRT_HD int ComputeSuperphotonsPerCell(real density_code_units, real normalization) {
    return static_cast<int>(density_code_units * normalization);
}

/* Application-specific packet generator used when photons.generator = "custom". */
template <typename RandomGenerator>
GRT_HD bool GeneratePhotonsCustom(const FluidCellCGS&, RandomGenerator&,
                                  int packets_per_cell, real configured_frequency_hz,
                                  real energy_per_cell_erg, real& sampled_frequency_hz,
                                  real& packet_energy_erg) {
    sampled_frequency_hz = configured_frequency_hz;
    packet_energy_erg = energy_per_cell_erg / static_cast<real>(packets_per_cell);
    return true;
}

}  // namespace grt

#endif  /* GRT_USER_PHYSICS_H */
