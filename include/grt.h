/*
 * grt.h -- C ABI of the B200-native GR-ray-tracer per-photon hot path.
 *
 * This library replaces the body of the reference's host step loop in
 * integrate_geodesics (src/geodesic_integrate/integrate_cart_ks.hpp:468-527):
 *   - the per-step Kokkos::parallel_for over Geodesic_cartesian_kerr_schild
 *     (integrate_cart_ks.hpp:470-481, functor operator() :230-419),
 *   - the "Count Terminated Photons" parallel_reduce (:496-503),
 *   - and, in image mode, the host build_observation_products pass
 *     (src/radiative_transfer/observation.hpp:31-84) behind write_image_products
 *     (src/output/write_output.hpp:107-142).
 *
 * Ownership: a context owns every device buffer.  Callers pass host pointers
 * that stay caller-owned; the library copies in and out.  No function throws
 * across this boundary; each returns a grt_status and grt_last_error() holds a
 * message.  A context is not re-entrant: use one context per host thread.
 *
 * Plain C types only (no CUDA or torch types); compiled for sm_100a.
 */
#ifndef GRT_H
#define GRT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GRT_ABI_VERSION 5

typedef enum grt_status {
    GRT_OK = 0,
    GRT_EINVAL = 1,     /* invalid argument or configuration value */
    GRT_ECUDA = 2,      /* a CUDA runtime call failed */
    GRT_ENOMEM = 3,     /* device allocation failed */
    GRT_ESTATE = 4,     /* call out of order (e.g. run before upload) */
    GRT_ETIMEOUT = 5,   /* device work hit its iteration limit and returned */
    GRT_EIO = 6,        /* file could not be read or written */
    GRT_ENODEV = 7      /* no usable sm_100 device */
} grt_status;

/* SimulationMode (src/simulation_options.hpp:11) */
enum { GRT_MODE_IMAGE = 0, GRT_MODE_DISK = 1 };
/* IntegratorType (src/utils.hpp:169) */
enum { GRT_RK4 = 0, GRT_RK45 = 1 };
/* PhotonGeneratorType (src/radiative_transfer/photon_generation.hpp:12-16) */
enum { GRT_GEN_BLACKBODY = 0, GRT_GEN_POWER_LAW = 1, GRT_GEN_CUSTOM = 2 };
/* PhotonPhase (src/utils.hpp:135-141) */
enum { GRT_PHASE_DISK = 0, GRT_PHASE_IMAGE_BACKWARD = 1, GRT_PHASE_IMAGE_FORWARD = 2,
       GRT_PHASE_IMAGE_ARRIVED = 3, GRT_PHASE_REJECTED = 4 };
/* Arithmetic form of the trace kernel. */
enum { GRT_PREC_FP64 = 0,        /* all-FP64, operation order of the reference (parity form) */
       GRT_PREC_MIXED = 1,       /* FP32 right-hand side after emission outside the fluid grid (and in RK4
                                    steps); FP64 state, stage sums and controller */
       GRT_PREC_MIXED_GRID = 2   /* as GRT_PREC_MIXED, and the FP32 right-hand side after emission inside
                                    the grid too (r > 4M, away from the polar axis) */ };

/*
 * Every runtime parameter the reference's step functor and step loop read.
 * Field meanings and defaults are those of the reference's TOML keys
 * (src/input/toml_config.hpp:129-278, defaults src/utils.cpp:4-37 and
 * src/simulation_options.hpp:13-32); grt_params_default() fills them.
 */
typedef struct grt_params {
    int32_t mode;                 /* simulation.mode */
    int32_t integrator;           /* integration.integrator */
    int32_t precision;            /* GRT_PREC_* (not a reference key) */
    int32_t generator;            /* photons.generator */
    double mass;                  /* black_hole.mass   (M_BH) */
    double spin;                  /* black_hole.spin   (a_BH) */
    double r_term_min;            /* termination.r_min (default R_HORIZON) */
    double r_term_max;            /* termination.r_max (default 1.5*camera.distance) */
    double atol;                  /* integration.atol */
    double rtol;                  /* integration.rtol */
    double min_step_scale;        /* 0.01 (utils.hpp:179) */
    double max_step_scale;        /* 10.0 (utils.hpp:180) */
    double safety;                /* 0.9  (utils.hpp:178) */
    int64_t max_steps;            /* integration.max_steps */
    double termination_percent;   /* integration.termination_percent */
    uint64_t output_interval;     /* output.interval: termination is checked on these steps */
    uint64_t nphotons;            /* global photon count the termination fraction divides by */
    double initial_step;          /* integration.initial_step (dlambda) */
    double camera_distance;       /* camera.distance */
    double camera_theta;          /* camera.theta */
    double camera_phi;            /* camera.phi */
    double camera_width;          /* camera.width  (plane_dim1) */
    double camera_height;         /* camera.height (plane_dim2) */
    int32_t absorption_enabled;   /* radiative_transfer.absorption_enabled */
    int32_t emission_enabled;     /* radiative_transfer.emission_enabled */
    double absorption_coefficient;/* radiative_transfer.absorption_coefficient */
    double emission_coefficient;  /* radiative_transfer.emission_coefficient */
    int32_t scattering_enabled;   /* scattering.enabled */
    int32_t rank;                 /* rank offset added to the scattering seed */
    double scattering_albedo;     /* scattering.albedo */
    uint64_t scattering_seed;     /* scattering.seed */
    double superphoton_count_normalization; /* photons.superphoton_count_normalization */
    double energy_per_cell_erg;   /* photons.energy_per_cell_erg */
    double power_law_slope;       /* photons.power_law_slope */
    double nu_min_hz;             /* photons.nu_min_hz */
    double nu_max_hz;             /* photons.nu_max_hz */
    double custom_frequency_hz;   /* photons.custom_frequency_hz */
    double length_cm_per_code;    /* units.* (photon_generation.hpp:18-38) */
    double time_s_per_code;
    double density_g_cm3_per_code;
    double temperature_k_per_code;
    double four_velocity_cm_s_per_code;
    double magnetic_gauss_per_code;
    uint64_t image_nx;            /* output.image_nx */
    uint64_t image_ny;            /* output.image_ny */
    uint64_t spectrum_bins;       /* output.spectrum_bins */
    double spectrum_min_hz;       /* output.spectrum_min_hz */
    double spectrum_max_hz;       /* output.spectrum_max_hz */
} grt_params;

/*
 * Host structure-of-arrays photon state, one pointer per field of the
 * reference's struct Photons (src/utils.hpp:40-133).  k0..k3 are the covariant
 * momentum p_mu.  terminate is one byte per photon (0/1).  Any pointer may be
 * NULL in grt_download_photons to skip that field.
 */
typedef struct grt_photon_soa {
    uint64_t* id;
    double* frequency;
    double* emission_frame_energy;
    double* x0; double* x1; double* x2; double* x3;
    double* k0; double* k1; double* k2; double* k3;
    double* I; double* Q; double* U; double* V;
    double* dlambda;
    double* theta_disp;
    double* phi_disp;
    uint8_t* terminate;
    uint8_t* phase;
} grt_photon_soa;

/* What one grt_run call did. */
typedef struct grt_run_stats {
    int64_t steps_done;         /* host-loop steps covered (index of last step + 1) */
    uint64_t n_terminated;      /* photons with terminate set after the run */
    uint64_t accepted_steps;    /* ray-steps that advanced a photon */
    uint64_t rejected_attempts; /* RK45 attempts rejected by the controller */
    uint64_t photon_calls;      /* functor invocations on live photons */
    uint64_t launches;          /* trace-kernel launches issued */
    double trace_ms;            /* device time of the trace launches (CUDA events) */
    int32_t timed_out;          /* 1 if a launch hit its iteration limit */
    int32_t pad;
} grt_run_stats;

/* Image products of write_image_products (write_output.hpp:130-141). */
typedef struct grt_image_products {
    double* image_I;              /* [image_ny][image_nx] */
    double* image_Q;
    double* image_U;
    double* image_V;
    double* spectrum_frequency_hz;/* [spectrum_bins] */
    double* spectrum_I;           /* [spectrum_bins] */
    uint64_t* arrived_count;      /* [1] */
} grt_image_products;

/* Launch shape of the trace kernel: the library's default is {128, 0, 8, 32, 1, 0, 0};
 * grt/autotune.py times the candidates on a workload and picks one. */
typedef struct grt_launch_config {
    int32_t threads_per_block;    /* 128 (the trace kernels' block size) */
    int32_t blocks_per_sm;        /* 2, 3 or 4 resident blocks per SM: register caps 255 / 170 / 128;
                                     0 = automatic: the fewest that keep every geodesic resident */
    int32_t refill_threshold;     /* idle lanes in a warp before it pulls new photons (1..32) */
    int32_t photons_per_grab;     /* photons a warp claims per access to the global queue; an
                                     image-mode queue is laid out in 8 x 4 pixel tiles, so 32 is
                                     one tile.  When every claim fits in the resident warps, the
                                     first claims are spread evenly over the SMs. */
    int32_t split_legs;           /* image mode: 1 = the backward legs, the packet generation at first
                                     fluid contact and the rest as three launches (same results, smaller
                                     loop bodies); 0 = one launch for whole rays */
    int32_t pad;
    int64_t max_iterations;       /* per-warp loop iterations a trace launch may take before it stops,
                                     writes every photon back at its last call boundary and the run
                                     returns GRT_ETIMEOUT (stats.timed_out = 1); 0 = automatic (a bound
                                     well above any launch that makes progress).  A later grt_run
                                     continues the photons from where they were left. */
} grt_launch_config;

typedef struct grt_ctx grt_ctx;

/* Library / build identification. */
int32_t grt_abi_version(void);
const char* grt_build_info(void);

/* Fill p with the reference's compiled-in defaults (src/utils.cpp:4-37). */
void grt_params_default(grt_params* p);

/* Check that p describes a run the kernels can trace (every mode, integrator and generator
 * field known; masses, tolerances, radii, camera, scales and ranges finite and ordered);
 * GRT_EINVAL and a message naming the field on failure.  grt_create and grt_set_params
 * call it.  The reference's TOML config is read by the reference's own loader: its parsed
 * structs reach grt_params through include/grt_reference_adapter.hpp. */
grt_status grt_params_validate(const grt_params* p, char* err, size_t err_len);

/* Create a context on the current CUDA device. */
grt_status grt_create(const grt_params* p, grt_ctx** out);
void grt_destroy(grt_ctx* ctx);
const char* grt_last_error(const grt_ctx* ctx);
grt_status grt_set_params(grt_ctx* ctx, const grt_params* p);

/* Use the caller's CUDA stream (a cudaStream_t passed as void*); NULL = the context's own. */
grt_status grt_set_stream(grt_ctx* ctx, void* stream);
grt_status grt_synchronize(grt_ctx* ctx);

/*
 * Upload the fluid grid: C-order float64 host arrays of shape
 * (nr, ntheta, nphi) for r/theta/phi/rho/T and (nr, ntheta, nphi, 4) for
 * vel/mag, exactly the seven NumPy inputs of load_numpy_field_bundle
 * (src/input/load_python_arrays.hpp:195-223).  Replaces ScatteringFluidGrid
 * (src/radiative_transfer/scattering.hpp:22-39).  Passing nr*ntheta*nphi == 0
 * uploads "no fluid" (fluid_available false, integrate_cart_ks.hpp:436-452).
 */
grt_status grt_upload_grid(grt_ctx* ctx, size_t nr, size_t ntheta, size_t nphi,
                           const double* r, const double* theta, const double* phi,
                           const double* rho, const double* temperature,
                           const double* vel4, const double* mag4);

/* Load the seven .npy files of a reference input directory and upload them. */
grt_status grt_upload_grid_numpy_dir(grt_ctx* ctx, const char* numpy_dir);

/*
 * Copy n photons from host SoA into the context (replaces the Photons views).
 * After an image initialisation with the same photon count the slots keep
 * their images (a saved batch state can be restored); otherwise the image set
 * is dropped and every photon uses the camera of grt_params.
 */
grt_status grt_upload_photons(grt_ctx* ctx, const grt_photon_soa* soa, size_t n);

/*
 * Initialise nx*ny image-plane photons on the device, one per pixel centre
 * u = -W/2 + (ix+1/2) W/nx, v = -H/2 + (iy+1/2) H/ny, photon id = id_offset +
 * iy*nx + ix.  Same construction as initialize_photons_image
 * (src/radiative_transfer/initialize_photons.hpp:82-170) with the random
 * screen draw replaced by the deterministic pixel grid.
 */
grt_status grt_init_image_photons(grt_ctx* ctx, uint64_t nx, uint64_t ny, uint64_t id_offset);

/*
 * Initialise n image-plane photons on the device with the reference's random
 * screen: replaces initialize_photons_image
 * (src/radiative_transfer/initialize_photons.hpp:82-170) as it stands, whose
 * screen position is (u, v) = (drand(-W/2, W/2), drand(-H/2, H/2)) from a
 * random pool seeded 12345 + rank (:115-126).  Here each photon's two draws
 * come from Philox4x32-10 keyed by (12345 + params.rank, photon id), so they
 * do not depend on scheduling: u = -W/2 + W d1, v = -H/2 + H d2 with d in
 * [0, 1), photon id = id_offset + i.  The rays are binned into the
 * output.image_nx x image_ny image of grt_get_image_products, as there.
 */
grt_status grt_init_image_photons_random(grt_ctx* ctx, uint64_t n, uint64_t id_offset);

/*
 * The pixel rows [row0, row0 + nrows) of the nx*ny screen of
 * grt_init_image_photons (same rays, same ids id_offset + iy*nx + ix): one
 * image split across GPUs, each rank tracing its rows; every rank's
 * grt_get_image_products covers the full image, so summing them over the
 * ranks gives the single-GPU products.
 */
grt_status grt_init_image_rows(grt_ctx* ctx, uint64_t nx, uint64_t ny, uint64_t row0, uint64_t nrows,
                               uint64_t id_offset);

/*
 * Line-of-sight forward rays (no counterpart in the reference's initialisers;
 * its functor handles them as ImageForward photons): one per pixel centre
 * (u, v) of the camera window, starting at -back_distance * n + u th + v ph
 * behind the scene and aimed along the camera normal n, with I = 0,
 * frequency = custom_frequency_hz, emission_frame_energy = -p_t and
 * dlambda = initial_step * back_distance.  They cross the fluid, accumulating
 * emission and absorption on the way, and are binned where they cross the
 * camera plane -- the volumetric image the adjoint differentiates (the
 * reference's image mode emits at the first fluid contact and retraces its
 * path outward, sampling no fluid on its forward leg).
 */
grt_status grt_init_image_forward_photons(grt_ctx* ctx, uint64_t nx, uint64_t ny, double back_distance,
                                          uint64_t id_offset);

/*
 * Advance the photons: equivalent to the reference's step loop for
 * step in [0, p.max_steps), stopping after the first output step
 * (step % output_interval == 0 or the last step) at which the terminated
 * fraction reaches termination_percent.  stats may be NULL.
 */
grt_status grt_run(grt_ctx* ctx, grt_run_stats* stats);

/* Copy the photon state back to host SoA (NULL fields are skipped). */
grt_status grt_download_photons(grt_ctx* ctx, grt_photon_soa* soa);
size_t grt_photon_count(const grt_ctx* ctx);
/* Geodesics a run traces (no counterpart in the reference): the photon count,
 * or, for a batch whose frequency channels share their geodesic
 * (grt_set_channel_sharing, scattering off), one per channel group and pixel. */
uint64_t grt_geodesic_count(const grt_ctx* ctx);

/*
 * Host photon block (no counterpart in the reference, whose Photons are 20
 * separate Kokkos views): the device keeps the SoA in one block, the 20
 * fields back to back in grt_photon_soa order (id, the 17 doubles, terminate,
 * phase; 146 bytes per photon).  grt_host_photon_layout points soa's fields
 * into a caller-owned host block of grt_photon_block_bytes(n) bytes
 * (8-byte aligned; pinned memory for asynchronous copies) in that layout;
 * grt_upload_photons / grt_download_photons given such a SoA move it with
 * one transfer instead of 20.
 */
size_t grt_photon_block_bytes(size_t n);
grt_status grt_host_photon_layout(void* block, size_t n, grt_photon_soa* soa);

/*
 * Image products of the ImageArrived photons, accumulated on the device
 * (build_observation_products, observation.hpp:31-84): every output array is
 * a caller-owned host buffer sized from p.image_nx/ny/spectrum_bins.
 */
grt_status grt_get_image_products(grt_ctx* ctx, grt_image_products* out);

/* Write <output_dir>/<name>_image_products.npz like write_image_products. */
grt_status grt_write_image_products_npz(grt_ctx* ctx, const char* output_dir, const char* name);

/*
 * Output-step archives (the reference's checkpoints).  The photon fields an
 * output step can write, in the reference's order (available_output_variables,
 * src/output/output_variables.hpp:12-18):
 *   0 id, 1 frequency, 2 emission_frame_energy, 3-6 x0..x3, 7-10 k0..k3,
 *   11-14 I Q U V, 15 dlambda, 16 terminate, 17 phase, 18 theta_disp, 19 phi_disp.
 *
 * grt_parse_output_variables is OutputSelection::parse (output_variables.hpp:
 * 27-70): a comma list, optionally in [ ] with quoted names, duplicates
 * dropped; "all" appends every field to the names before it and ends the list
 * (as in the reference, a name before "all" is then written twice).  fields
 * (may be NULL; room for 40) receives the indices in the order written,
 * *count their number.  GRT_EINVAL with the
 * reference's message ("unknown output variable: X", "output variables cannot
 * be empty") otherwise.
 */
grt_status grt_parse_output_variables(const char* spec, int32_t* fields, size_t* count, char* err, size_t err_len);
/*
 * write_output_step (write_output.hpp:90-103): <output_dir>/<name>_step_<step>_rank<rank>.npz
 * holding the selected fields of photons 0, stride, 2*stride, ... (each a 1-D
 * array: id <u8, terminate and phase |u1, the rest <f8), written under a
 * temporary name and renamed into place.  The fields are gathered on the
 * device and copied back in one transfer.
 */
grt_status grt_write_output_step_npz(grt_ctx* ctx, const char* output_dir, const char* name, int64_t step,
                                     int32_t rank, const char* variables, uint64_t stride);

/*
 * The reference's whole step loop with its output (integrate_geodesics,
 * integrate_cart_ks.hpp:468-532): trace launches end on every output step
 * (step % output_interval == 0, and the last step); after each, the
 * terminated fraction is evaluated and the output-step archive written (rank
 * p.rank); the loop stops once the fraction reaches termination_percent.  In
 * image mode the image-products archive follows (grt_write_image_products_npz,
 * or grt_write_batch_products_npz for a batch).  Per-photon results equal
 * grt_run's.
 */
grt_status grt_run_with_output(grt_ctx* ctx, const char* output_dir, const char* name, const char* variables,
                               uint64_t stride, grt_run_stats* stats);

/*
 * Disk-mode emission, as initialize_photons_disk (initialize_photons.hpp:
 * 173-327) after build_superphoton_cell_offsets (:32-64): every grid cell
 * emits ComputeSuperphotonsPerCell(rho, superphoton_count_normalization)
 * packets from its centre, with the generator's frequency and energy and an
 * isotropic fluid-frame direction; packets whose cell has no valid fluid tetrad
 * or whose generator fails start Rejected.  Random draws use Philox keyed by
 * (scattering_seed + rank, photon id).  Replaces the context's photons;
 * *n_photons (may be NULL) receives the packet count.
 */
grt_status grt_init_disk_photons(grt_ctx* ctx, uint64_t id_offset, uint64_t* n_photons);

/*
 * Batched image mode (no counterpart in the reference, which renders one
 * camera per run): several images, each with its own camera and radiative
 * coefficients (inclinations, resolutions, frequency channels), traced by ONE
 * persistent launch whose work queue spans every image's rays, so long and
 * short rays of all images balance across the GPU.  Each image follows
 * grt_init_image_photons for its own camera; the other parameters come from
 * the context's grt_params.
 */
typedef struct grt_image_spec {
    double camera_theta;            /* camera.theta / camera.phi / distance / width / height of this image */
    double camera_phi;
    double camera_distance;
    double camera_width;
    double camera_height;
    uint64_t nx, ny;                /* pixels = rays of this image */
    double custom_frequency_hz;     /* photon_generation.custom_frequency_hz (custom generator) */
    double absorption_coefficient;  /* radiative_transfer.absorption_coefficient */
    double emission_coefficient;    /* radiative_transfer.emission_coefficient */
} grt_image_spec;

/*
 * Initialise the rays of nimages images on the device: image k occupies the
 * photon slots [start_k, start_k + nx_k*ny_k) with start_0 = 0 and ids
 * id_offset + start_k + iy*nx_k + ix.  Replaces any earlier photons.
 */
grt_status grt_init_image_batch(grt_ctx* ctx, const grt_image_spec* specs, size_t nimages, uint64_t id_offset);
size_t grt_batch_image_count(const grt_ctx* ctx);

/*
 * Frequency channels: images of a batch with identical camera and screen
 * (theta, phi, distance, width, height, nx, ny) differ only in frequency and
 * coefficients, which change Stokes vectors but never a geodesic.  With
 * scattering off they share one traced geodesic per pixel (up to 32 channels
 * per group); each channel keeps its own id, random draws, frequency and
 * Stokes vector, and its photons end bit for bit as if traced alone.  On by
 * default; enable = 0 traces every image separately.
 */
grt_status grt_set_channel_sharing(grt_ctx* ctx, int enable);

/* Products of image k of the batch (buffers sized nx_k*ny_k and p.spectrum_bins). */
grt_status grt_get_batch_image_products(grt_ctx* ctx, size_t image, grt_image_products* out);
/* Every image's products of the batch at once, outs[k] for image k (nimages
 * = grt_batch_image_count): the copies of all images and one synchronisation. */
grt_status grt_get_all_batch_image_products(grt_ctx* ctx, grt_image_products* outs, size_t nimages);

/*
 * The image products of the current image set (single image or batch) as one
 * block, for collectives and device-side consumers (no counterpart in the
 * reference, whose products go through host vectors and MPI_Reduce,
 * write_output.hpp:109-127): every image's image_I, image_Q, image_U, image_V
 * ([ny_k][nx_k] float64 each) in image order, then every image's spectrum_I
 * ([spectrum_bins] float64), then every image's arrived count (uint64).  The
 * products of the last render are used, or built first.  dst may be device or
 * host memory; the copies are enqueued on the context's stream and the
 * caller synchronises with it.
 */
size_t grt_products_block_bytes(const grt_ctx* ctx);
grt_status grt_copy_products_block(grt_ctx* ctx, void* dst, size_t bytes);

/* Write <output_dir>/<name>_image<k>_image_products.npz for every image k. */
grt_status grt_write_batch_products_npz(grt_ctx* ctx, const char* output_dir, const char* name);

/*
 * Render through a CUDA graph: re-initialise the rays of the last
 * grt_init_image_photons / grt_init_image_batch call, trace them and build
 * every image's products on the device.  The graph is captured on the first
 * call and replayed afterwards (re-captured after a change of parameters,
 * grid, images, stream or launch shape).  Needs termination_percent >= 1 (one
 * trace launch, no host decision inside the loop), else GRT_EINVAL.
 * stats->trace_ms is the trace kernel's time (event-record nodes inside the
 * graph).  Products are then read with grt_get_image_products /
 * grt_get_batch_image_products.
 */
grt_status grt_render_graph(grt_ctx* ctx, grt_run_stats* stats);

/*
 * Asynchronous render of host photons (no counterpart in the reference, whose
 * step loop is synchronous; integrate_cart_ks.hpp:468-527 with the products
 * of observation.hpp:31-84).  grt_render_async enqueues, without waiting:
 * the copy of `photons` (a host photon block of grt_photon_count photons,
 * grt_host_photon_layout; pinned for the copy to overlap) into the batch's
 * slots on the context's copy stream; the trace and every image's products on
 * the context's stream once the copy has landed; and the copy of the products
 * into outs[k] (as grt_get_all_batch_image_products) on the copy stream.
 * The batch keeps its images, as grt_upload_photons with the batch's count
 * does.  Needs an image batch and termination_percent >= 1.  The host buffers
 * must stay untouched until grt_render_wait returns; one render is in flight
 * per context, and until its grt_render_wait every other call on the context
 * that sets it up, enqueues work or reads results returns GRT_ESTATE.  Two contexts given the same stream
 * (grt_set_stream) and used in turn keep their traces in order on it while
 * one's copies overlap the other's trace.  grt_render_wait blocks until the
 * render's products are on the host and fills stats as grt_run does.
 */
grt_status grt_render_async(grt_ctx* ctx, const grt_photon_soa* photons, grt_image_products* outs, size_t nimages);
grt_status grt_render_wait(grt_ctx* ctx, grt_run_stats* stats);

/*
 * Differentiable radiative transfer (no counterpart in the reference).
 * Per-cell multipliers scale the values the user extension points return:
 * dtau = m_abs[cell] * ComputeOpticalDepthIncrement(...) and
 * dI = m_emis[cell] * ComputeEmissivityIncrement(...)
 * (radiative_transfer.hpp:61-96), so the gradient below is exact for any
 * user body.  Arrays are host float64 of length nr*ntheta*nphi (C order of
 * the grid); NULL switches that multiplier off (all ones).  Applies to every
 * later trace (grt_run, grt_render_graph, the checkpointed forward).
 */
grt_status grt_set_cell_multipliers(grt_ctx* ctx, const double* m_abs, const double* m_emis);

/*
 * Trace the context's photons like grt_run (termination_percent >= 1, FP64
 * form) and keep, per ray, its state right after the emission call and every
 * checkpoint_interval calls after it, for grt_adjoint_image_I.
 */
grt_status grt_forward_checkpointed(grt_ctx* ctx, int64_t checkpoint_interval, grt_run_stats* stats);

/*
 * Adjoint of the last grt_forward_checkpointed: given dL/d(image_I) (host,
 * [image_ny][image_nx], the binning of grt_get_image_products), write
 * dL/dm_abs and dL/dm_emis (host, [nr*ntheta*nphi]; either may be NULL).
 * Each ray's segments are recomputed from its checkpoints (bit-identical to
 * the forward pass) and its radiative-transfer updates swept backwards.
 */
grt_status grt_adjoint_image_I(grt_ctx* ctx, const double* dL_dimage_I, double* dL_dm_abs, double* dL_dm_emis);

/* Launch shape of the trace kernel. */
grt_status grt_get_launch_config(const grt_ctx* ctx, grt_launch_config* cfg);
grt_status grt_set_launch_config(grt_ctx* ctx, const grt_launch_config* cfg);

/*
 * Fluid grid already in caller-owned device memory, in the reference's own
 * layout: the seven NumPy inputs as C-order float64 arrays of shape
 * (nr, ntheta, nphi) for r/theta/phi/rho/temperature and (nr, ntheta, nphi, 4)
 * for vel4/mag4.  nr*ntheta*nphi == 0 means no fluid.
 */
typedef struct grt_device_grid {
    uint64_t nr, ntheta, nphi;
    const double* r;
    const double* theta;
    const double* phi;
    const double* rho;
    const double* temperature;
    const double* vel4;
    const double* mag4;
} grt_device_grid;

/*
 * Allocation-free tracing (no counterpart in the reference).  For callers
 * that cannot call cudaMalloc where they trace -- hosts whose device memory is
 * owned by their own pool or a fixed budget, or latency-critical loops that
 * must not allocate (cudaMalloc can synchronise the device) -- this traces
 * n photons that already live in caller-owned device memory (`photons` holds
 * DEVICE pointers here) against a grid in caller-owned device memory, in
 * place, with the same step-loop semantics as grt_run and the FP64 parity
 * kernel, on `stream` (a cudaStream_t, NULL = legacy default stream).
 * It creates no context, allocates nothing and frees nothing.  Its scratch
 * (work-queue head, counters, staged grid axes) is a 128 KiB array in the
 * library that each GPU loading the library holds until exit, shared by all
 * calls: serialise calls per device, because calls that overlap on the GPU
 * race on it.  Limits: nr + ntheta + nphi <= 8160 (larger grids are rejected
 * with GRT_EINVAL and a message), FP64 precision only.  Each call checks the
 * grid's separability on the device (one pass over the coordinate arrays),
 * then reads the axes back and derives the lookup's acceptance bounds on the
 * host with the routine grt_upload_grid uses, so the lookup accepts and
 * rejects exactly what the context entry point's does, cell edges included.
 * The grid stays in the reference's raw layout, so each sample's spherical
 * four-velocity and field are turned Cartesian with the GPU's sin/cos (the
 * context entry point precomputes them with the host's): results equal the
 * context entry point's bit for bit without scattering, and in distribution
 * with it, where an ulp in the fluid frame changes a scattered direction.
 * The call waits for the read-back and for the trace on `stream` before it
 * returns.  The first call
 * on a device looks up the scratch address (cudaGetSymbolAddress) with that
 * device current; make it before any stream capture.  err receives a message
 * on failure (may be NULL).  When a launch runs out of iterations the call
 * returns GRT_ETIMEOUT with stats filled as grt_run fills them.
 */
grt_status grt_trace_device_noalloc(const grt_params* p, const grt_device_grid* grid,
                                    const grt_photon_soa* photons, uint64_t n, grt_run_stats* stats,
                                    void* stream, char* err, size_t err_len);

/*
 * Roofline denominators (no counterpart in the reference): FP64 and FP32 FMA
 * throughput of the current device in TFLOP/s (2 flops per FMA), measured
 * with CUDA events over long independent FMA chains.
 */
grt_status grt_measure_fma_peaks(double* fp64_tflops, double* fp32_tflops);

#ifdef __cplusplus
}
#endif

#endif /* GRT_H */
