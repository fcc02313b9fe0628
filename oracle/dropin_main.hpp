// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// Forced include (g++ -include) that builds the reference's own src/main.cpp
// with its integrate_geodesics call (src/main.cpp:246-266) routed to the
// product's drop-in, integrate_geodesics_b200 (include/grt_reference_adapter.hpp).
// A maintainer makes that one-line change in main.cpp; the tests make it this
// way so the reference tree stays untouched.  The reference's headers are
// included first (they are include-guarded, so main.cpp's own includes are
// no-ops), then the adapter, then the call is renamed.
#pragma once

#include "utils.hpp"
#include "simulation_options.hpp"
#include "input/load_python_arrays.hpp"
#include "input/toml_config.hpp"
#include "radiative_transfer/initialize_photons.hpp"
#include "geodesic_integrate/integrate_cart_ks.hpp"
#include "output/write_output.hpp"
#include "output/display.hpp"

#include "grt_reference_adapter.hpp"

#define integrate_geodesics integrate_geodesics_b200
