/*
 * icp_b200.h -- C ABI of the B200-native phase-function generation path.
 *
 * Plain pointers, sizes and POD structs only.  Every function returns an int
 * status (ICP_OK = 0) and records a message retrievable with icp_last_error().
 * Calls are synchronous with respect to the context's stream unless stated;
 * device pointers are borrowed only for the duration of a call.
 *
 * Reference interfaces replaced (Somatic-Cell/ice-crystal-phase):
 *   icp_context_*         rainbow::CudaContext            include/rainbow/cuda_driver.hpp, src/cuda_driver.cpp:148-215
 *   icp_abi_version       ABI marker kernels              hex_trace/device/hex_trace.cu:6-11,
 *                                                         hex_phase/device/phase_accumulate.cu:9,
 *                                                         device/phase_cdf.cu:65
 *   icp_hex_trace_bin     HexPrismTracer::trace +         hex_trace/include/ice_crystal/hex_trace_cuda.hpp:26-27
 *                         PhaseMassAccumulatorCuda::add   hex_phase/include/ice_crystal/phase_cuda.hpp:25
 *   icp_phase_cdf_build   PhaseMassAccumulatorCuda::finish hex_phase/include/ice_crystal/phase_cuda.hpp:26
 *                         + rainbow::PhaseCdf::build       include/rainbow/phase_cdf.hpp:63-65
 *   icp_hex_generate      the CUDA branch of ice_generate_phase's record loop
 *                                                         hex_phase/apps/generate_hex_phase.cpp:92-134
 *   icp_drop_trace_bin    RaindropTracer::trace_unpolarized + patch/query/optics stages
 *                                                         include/rainbow/raindrop_tracer.hpp, apps/generate_phase.cpp:431-439
 *   icp_drop_generate     rainbow_generate's record path   apps/generate_phase.cpp:395-453
 *   icp_patch_build       PatchAccel::build's kernels    device/patch_build.cu:13-77
 *   icp_patch_query       PatchQuery::query_grid          src/patch_query.cpp, shaders/entry/patch_query.cu
 *   icp_patch_optics      evaluate_patch_optics / evaluate_focal_optics  device/patch_optics.cu:7-24
 *   icp_stage_density     density() + phase_check_density device/phase_cdf.cu:40-56, 93-108
 *   icp_rainbow_*         RainbowDiffraction + PatchOptics::run_diffraction
 *                                                         include/rainbow/rainbow_diffraction.hpp,
 *                                                         src/patch_optics.cpp:334-348
 */
#ifndef ICP_B200_H
#define ICP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ICP_ABI_VERSION 0x49435001u /* "ICP" v1 */

enum icp_status {
    ICP_OK = 0,
    ICP_ERR_INVALID_ARGUMENT = 1, /* rejected input (reference: std::invalid_argument)        */
    ICP_ERR_AUDIT = 2,            /* numerical/quality audit failed (reference: runtime_error) */
    ICP_ERR_CAPACITY = 3,         /* an explicit capacity/size limit was exceeded              */
    ICP_ERR_DEVICE = 4,           /* CUDA error                                                */
    ICP_ERR_TIMEOUT = 5,          /* a bounded device-side wait gave up                        */
    ICP_ERR_STATE = 6             /* call sequence error (reference: std::logic_error)         */
};

/* Trace arithmetic: FP32 (default fast path) or FP64 (reference-exact tolerances). */
enum icp_precision { ICP_FP32 = 0, ICP_FP64 = 1 };

/* Ray status codes, identical to the reference TraceStatus (hex_trace_core.hpp:97-102). */
enum icp_ray_status {
    ICP_RAY_EXHAUSTED = 0, ICP_RAY_TAIL = 1, ICP_RAY_LIMIT = 2, ICP_RAY_AMBIGUOUS = 3,
    ICP_RAY_INVALID = 4, ICP_RAY_NUMERICAL = 5, ICP_RAY_OVERFLOW = 6, ICP_RAY_REPLAY = 7
};

typedef struct icp_context icp_context;

/* ------------------------------------------------------------------ context */
uint32_t icp_abi_version(void);
/* Number of CUDA kernels this library has launched in this process (all contexts). */
unsigned long long icp_kernel_launches(void);
/* Copies the calling thread's last error message (NUL-terminated, truncated to n). */
size_t icp_last_error(char* buffer, size_t n);
/* Creates a context on CUDA device `device` with one non-blocking stream. */
int icp_context_create(int device, icp_context** out);
int icp_context_destroy(icp_context* ctx);
/* Synchronises the context stream. */
int icp_context_synchronize(icp_context* ctx);
/* Iteration limit of the CDF kernels' grid-barrier waits and of the tensor-core pipeline waits
 * of icp_mlp_gemm_bf16 on this context (0 = the library's default, about four million polls).
 * A wait that runs out ends the call with ICP_ERR_TIMEOUT and leaves the context usable.  No
 * reference counterpart: the reference's stages have no bounded device waits; this lets a host
 * shorten them (and tests make them run out). */
int icp_context_set_wait_limit(icp_context* ctx, uint32_t limit);
/* The context's cudaStream_t, for callers that enqueue their own work. */
void* icp_context_stream(icp_context* ctx);
/* Device memory owned by the context's caller (thin wrappers for FFI users). */
int icp_device_alloc(icp_context* ctx, size_t bytes, void** out);
int icp_device_free(icp_context* ctx, void* ptr);
int icp_memcpy_h2d(icp_context* ctx, void* dst, const void* src, size_t bytes);
int icp_memcpy_d2h(icp_context* ctx, void* dst, const void* src, size_t bytes);
int icp_memset_d(icp_context* ctx, void* dst, int value, size_t bytes);

/* -------------------------------------------------------------- (u,phi) grid */
/* Ensemble-frame sampling grid: u = (1-cos theta)/2 rows, phi columns.
 * ki, e0, e1: unit incident axis and its transverse frame (sampling_frame_columns). */
typedef struct {
    uint32_t nt, np;
    double ki[3], e0[3], e1[3];
} icp_grid;

/* Writes the nt+1 saved u edges (bit-identical to make_phase_u_edges,
 * include/rainbow/phase_cdf_math.hpp:16-32). Host function, no device use. */
int icp_u_edges(uint32_t nt, double* edges_out);

/* Refractive index of ice Ih at a vacuum wavelength (replaces evaluate_ice_wb2008,
 * hex_atlas/src/ice_optics.cpp:13-30): the Warren & Brandt (2008) table, real index linear and
 * imaginary index log-linear in log(wavelength) between its rows; 200..1100 nm, no
 * extrapolation (ICP_ERR_INVALID_ARGUMENT outside).  The tracer uses n; kappa is reported, not
 * applied.  Host function, no device use. */
typedef struct {
    double wavelength_nm;
    double n, kappa;
    double lower_nm, upper_nm;      /* bracketing table wavelengths (equal at a table row)     */
    double log_wavelength_fraction; /* ln(lambda / lower) / ln(upper / lower), 0 at a row      */
} icp_ice_state;
int icp_ice_index(double wavelength_nm, icp_ice_state* out);

/* Statistics of one trace+bin call (raw sums in units of incident power per ray;
 * multiply by the per-ray area weight to obtain mm^2). */
typedef struct {
    double escaped;          /* sum over rays of escaped power                              */
    double unresolved;       /* sum over rays of residual power left when a ray stopped     */
    double point_axial;      /* sum of power * cos(scattering angle) over binned exits      */
    double forward_pole;     /* power within the forward pole cap                           */
    double backward_pole;    /* power within the backward pole cap                          */
    double max_ray_balance;  /* max |escaped + residual - 1| over rays                      */
    double max_interface_balance; /* max relative Fresnel power imbalance at one interface   */
    uint64_t rays;
    uint64_t outputs;
    uint64_t status_counts[8];
    uint64_t rejected_rays;  /* rays failing the acceptance predicate (status/balance)      */
    uint64_t snapped;        /* exits assigned to a cell edge by the roundoff snap rule     */
    uint64_t near_edge;      /* FP32: interactions within rounding distance of a prism edge */
    uint64_t fallback_adds;  /* exits that bypassed the shared-memory privatised table      */
    uint64_t max_batch_outputs; /* largest number of exits produced by one batch of rays    */
    uint64_t invalid;        /* exits that could not be binned (non-finite direction)       */
    uint64_t encounters;     /* internal boundary interactions traced                       */
    uint64_t missed;         /* sampled rays that miss the particle (drops; never prisms)   */
    uint64_t gauge_evals;    /* Newton evaluations of the drop surface (non-spherical drops) */
} icp_trace_stats;

/* Histogram privatisation / launch tuning (all zero = autotuned defaults). */
typedef struct {
    uint32_t block_threads;  /* 0 = the kernel's size (FP32 drop 128, others 256), else 64 up
                              * to that size, a multiple of 32                               */
    uint32_t blocks_per_sm;  /* resident blocks per SM requested                              */
    uint32_t hash_slots;     /* shared-memory table slots (power of two; 0 = default; 1 = off) */
    uint32_t reserved;
} icp_tuning;

/* ----------------------------------------------------------------- hex prism */
/* One orientation node of a hexagonal prism (hex_trace/include/ice_crystal/hex_prism.hpp:6-12:
 * circumradius R and FULL length L in mm, long axis body +y). */
typedef struct {
    double circumradius_mm, length_mm;
    double rotation[9];       /* column-major body->ensemble rotation (active quaternion)  */
    double exterior_index, interior_index;
    double tail_tolerance;    /* per-ray residual power at which tracing stops              */
    double balance_tolerance; /* per-ray |escaped+residual-1| acceptance bound              */
    double area_weight;       /* mm^2 added to the histogram per unit exit power            */
    uint64_t seed, total_samples, first_sample, sample_count;
    uint32_t max_internal_hits;
    uint32_t batch_size;      /* audit batch size (capacity check granularity)              */
    uint32_t precision;       /* icp_precision                                              */
    uint32_t reserved;
} icp_hex_node;

/* Projected area (mm^2) of the prism along the node's body-frame incident direction,
 * rotation^T * grid.ki (hex_prism.hpp:37-43). Host function. */
int icp_hex_node_area(const icp_hex_node* node, const icp_grid* grid, double* area_mm2);

/* Traces sample_count rays of one node and adds area_weight * exit power into
 * d_cell_mass[nt*np] (FP64, theta-major), pole caps into the stats.
 * d_edges: nt+1 u edges on the device. d_stats: one icp_trace_stats on the device
 * (accumulated into, caller zeroes). d_batch_outputs may be NULL or hold
 * ceil(total_samples/batch_size) uint32 counters (accumulated into). */
int icp_hex_trace_bin(icp_context* ctx, const icp_hex_node* node, const icp_grid* grid,
                      const double* d_edges, double* d_cell_mass, icp_trace_stats* d_stats,
                      uint32_t* d_batch_outputs, const icp_tuning* tuning);

/* --------------------------------------------------------------------- CDF */
typedef struct {
    double max_l1_error;      /* 1e-10 */
    double max_lost_mass;     /* 1e-12 */
    double max_coarsening_tv; /* 1     */
} icp_cdf_policy;

typedef struct {
    double g_source, g_stored, coarsening_tv, cdf_mass;
    double l1_error, lost_mass, maximum_cell_error, aggregation_relative_error;
    double fine_mass, fine_axial;
    uint64_t lost_cells;
    uint64_t malformed;
    uint32_t status;          /* icp_status of the audit                                     */
    uint32_t reserved;
} icp_cdf_report;

/* Input kinds for icp_phase_cdf_build. */
enum icp_cdf_input { ICP_CDF_MASS = 0, ICP_CDF_DENSITY = 1 };

/* Builds the stored CDF from a fine theta-major grid d_values[nt*np] (cell masses, or
 * densities per steradian when input_kind == ICP_CDF_DENSITY).  forward_pole /
 * backward_pole masses are spread uniformly over the first / last fine row
 * (hex_phase/src/phase_table.cpp:63-76).  Aggregates conservatively to ct x cp
 * (ct | nt, cp | np), scans each phi column in ascending theta with ordered binary64
 * additions, scans the marginal in ascending phi, normalises and audits.
 * Outputs (device): d_phi[cp+1], d_theta[cp*(ct+1)] (phi-major); the stored u edges are
 * every (nt/ct)-th fine edge.  The report is written to host memory. */
int icp_phase_cdf_build(icp_context* ctx, const double* d_values, uint32_t input_kind, uint32_t nt,
                        uint32_t np, double forward_pole, double backward_pole, uint32_t ct, uint32_t cp,
                        const icp_cdf_policy* policy, double* d_phi, double* d_theta, icp_cdf_report* report);
/* icp_phase_cdf_build in two halves, for device-resident callers that keep the build on the
 * context's stream with other work (the reference's PhaseCdf::build waits before returning,
 * src/phase_cdf.cpp:211-223): icp_phase_cdf_enqueue checks the arguments and enqueues the build
 * (one cooperative kernel once the grid's u edges are on the device) without waiting;
 * icp_phase_cdf_result waits for the stream, applies the quality gates and fills the report.
 * One build in flight per context. */
int icp_phase_cdf_enqueue(icp_context* ctx, const double* d_values, uint32_t input_kind, uint32_t nt, uint32_t np,
                          double forward_pole, double backward_pole, uint32_t ct, uint32_t cp, double* d_phi,
                          double* d_theta);
int icp_phase_cdf_result(icp_context* ctx, const icp_cdf_policy* policy, icp_cdf_report* report);
/* The same for `count` histograms of one shape (mass input, no pole caps) at d_values +
 * r*nt*np, built in few cooperative launches (no reference counterpart; the reference builds one
 * record per process): phi / theta of record r at d_phi + r*(cp+1), d_theta + r*cp*(ct+1), equal
 * to icp_phase_cdf_build's; reports[count] on the host (status = the record's audit). */
int icp_phase_cdf_build_batch(icp_context* ctx, const double* d_values, uint32_t count, uint32_t nt, uint32_t np,
                              uint32_t ct, uint32_t cp, const icp_cdf_policy* policy, double* d_phi, double* d_theta,
                              icp_cdf_report* reports);

/* Static-scratch CDF builder: no counterpart in the reference.  For callers that cannot
 * allocate device memory themselves or through this library -- an embedding application
 * whose own allocator already owns the device, or a callback context where allocating is
 * not allowed.  Same inputs, outputs, gates and report as icp_phase_cdf_build, on the given
 * cudaStream_t (NULL = legacy default stream of the current device; a stream must belong to
 * the current device and context, else ICP_ERR_INVALID_ARGUMENT), but every scratch buffer
 * (u edges, block partials, column sums, barrier counters, audit record) lives in one
 * file-scope device array of ICP_STATIC_SCRATCH_BYTES (216.75 KiB) that each GPU holds until
 * the process exits.  Limits: nt <= ICP_STATIC_MAX_THETA, cp <= ICP_STATIC_MAX_PHI
 * (ICP_ERR_CAPACITY beyond).  The first call in a CUDA context looks the array's address up in
 * that context (make it before any stream capture); the entry copies host memory and waits
 * for the stream, so it is never called inside a stream capture.  All calls share the array,
 * so calls that overlap on the GPU race on it. */
#define ICP_STATIC_MAX_THETA 4096u
#define ICP_STATIC_MAX_PHI 8192u
#define ICP_STATIC_MAX_BLOCKS 1024u
#define ICP_STATIC_SCRATCH_BYTES 221952u
int icp_phase_cdf_build_static(void* stream, const double* d_values, uint32_t input_kind, uint32_t nt, uint32_t np,
                               double forward_pole, double backward_pole, uint32_t ct, uint32_t cp,
                               const icp_cdf_policy* policy, double* d_phi, double* d_theta, icp_cdf_report* report);

/* ----------------------------------------------------- whole hex record (e2e) */
typedef struct {
    double circumradius_mm, length_mm;
    double ki[3];             /* ensemble incident direction (normalised internally)          */
    double exterior_index, interior_index;
    double tail_tolerance, balance_tolerance;
    uint32_t nt, np, ct, cp;  /* histogram and stored CDF dimensions                          */
    uint32_t max_internal_hits, batch_size;
    uint64_t max_output_records; /* per batch; 0 = unlimited                                  */
    uint32_t precision, reserved;
    icp_cdf_policy policy;
    icp_tuning tuning;
} icp_hex_record;

typedef struct {
    double quaternion[4];     /* w, x, y, z (active Hamilton, body -> ensemble)              */
    double weight;            /* normalised number probability                               */
    uint64_t samples, seed;
} icp_orientation;

typedef struct {
    icp_trace_stats trace;    /* raw sums over all nodes (escaped/unresolved unweighted)     */
    double expected_area_mm2, escaped_area_mm2, unresolved_area_mm2;
    double histogram_mass_mm2, histogram_axial_mm2; /* fine grid (incl. poles), area units  */
    double point_mass_mm2, point_axial_mm2, forward_mass_mm2, backward_mass_mm2;
    double histogram_relative_error;
    icp_cdf_report cdf;
    double seconds_trace, seconds_cdf;
} icp_record_report;

/* Host-buffer entry point used by the ice_generate_phase drop-in: traces every node,
 * bins, builds and audits the CDF, and copies phi[cp+1], theta[cp*(ct+1)], u[ct+1]
 * to the caller's host arrays. Quality gates are NOT applied here (report only);
 * the CLI applies them with the reference's tolerances. */
int icp_hex_generate(icp_context* ctx, const icp_hex_record* record, const icp_orientation* nodes,
                     uint32_t node_count, double* h_phi, double* h_theta, double* h_u,
                     icp_record_report* report);

/* ------------------------------------------------------------ water drops */
/* Host helpers for the drop record inputs (all binary64, CPU):
 *  icp_water_index      IAPWS R9-97 index at the drop's wavelength / temperature / pressure
 *                       (replaces evaluate_water_optics, src/water_refractive_index.cpp:157-187;
 *                       liquid density by bisection of the IAPWS-95 pressure equation, all 56
 *                       residual terms, in [970, 1060] kg m^-3)
 *  icp_water_state      the same with the state, the density's pressure residual and the final
 *                       bracket width (rainbow::WaterOptics, the fields metadata.json reports)
 *  icp_drop_shape       Table-I coefficients for an equal-volume radius
 *                       (RaindropShape::try_make, include/rainbow/raindrop_shape.hpp:22-67)
 *  icp_drop_projected_area  convex-surface projected area (compute_projected_area,
 *                       src/projected_area.cpp:163-229)
 *  icp_drop_frame       ki = (cos a, -sin a, 0) and its transverse frame (RaindropSettings,
 *                       include/rainbow/raindrop_settings.hpp:123-147) */
int icp_water_index(double wavelength_nm, double temperature_c, double pressure_pa, double* index, double* density);
typedef struct {
    double temperature_kelvin, pressure_pascal, density_kg_m3;
    double density_pressure_residual_pascal, density_bracket_width_kg_m3;
    double refractive_index;
} icp_water_optics;
int icp_water_state(double wavelength_nm, double temperature_c, double pressure_pa, icp_water_optics* out);
int icp_drop_shape(double radius_mm, int sphere, double coefficients[8], double* inner_radius, double* outer_radius);
int icp_drop_projected_area(const double coefficients[8], double radius_mm, const double k[3], double* area_mm2);
int icp_drop_frame(double inclination_deg, double k[3], double e0[3], double e1[3]);
/* Analytic diffraction stage (no reference counterpart; the reference's "diffraction" stage is
 * a Table-II blur at rainbow transitions, include/rainbow/rainbow_diffraction.hpp:16-28):
 * Fraunhofer diffraction of the circle of equal projected area, rows[i] = power (mm^2) between
 * u_edges[i] and u_edges[i+1] from Rayleigh's encircled energy 1 - J0(x)^2 - J1(x)^2,
 * x = (2 pi a_eq / lambda) sin(theta), over the forward hemisphere, summing to area_mm2. */
int icp_drop_diffraction_rows(const double* u_edges, uint32_t nt, double area_mm2, double wavelength_nm, double* rows);

/* One drop record (particle frame: gravity along -y, shape polar axis -y).
 * r/a = 1 + sum_n coefficients[n] T_n(mu), mu = cos(angle from -y); a = radius_mm. */
typedef struct {
    double radius_mm;
    double coefficients[8];
    double inclination_deg;    /* ki = (cos a, -sin a, 0)                                     */
    double exterior_index, interior_index, wavelength_nm;
    double tail_tolerance, balance_tolerance;
    uint32_t nt, np, ct, cp;
    uint32_t max_internal_hits, precision;
    uint64_t rays, seed;       /* rays sampled uniformly over the bounding disk (counter RNG) */
    uint32_t diffraction;      /* 1: add the analytic Fraunhofer stage (equal power to Aproj) */
    uint32_t reserved;
    icp_cdf_policy policy;
    icp_tuning tuning;
} icp_drop_record;

typedef struct {
    icp_trace_stats trace;
    double projected_area_mm2;  /* CPU binary64 integral                                        */
    double sampled_area_mm2;    /* area of the sampling disk                                    */
    double incident_area_mm2;   /* hit fraction x disk area (Monte Carlo estimate of Aproj)     */
    double escaped_area_mm2, unresolved_area_mm2, diffraction_area_mm2;
    double forward_mass_mm2, backward_mass_mm2, histogram_mass_mm2, point_axial_mm2;
    double histogram_relative_error;
    double ki[3], e0[3], e1[3]; /* ensemble frame of the stored CDF (sampling_frame_columns)   */
    icp_cdf_report cdf;
    double seconds_trace, seconds_cdf;
} icp_drop_report;

/* Area (mm^2) of the disk the drop's rays are sampled on: radius 1 + c0 for a sphere, else the
 * conservative outer radius (1 + c0 + sum|c_n|)(1 + 1e-6) + 1e-6, times radius_mm.  A record of
 * N rays weighs each unit of exit power sampled_area / N. */
int icp_drop_sampling_area(const double coefficients[8], double radius_mm, double* area_mm2);
/* Traces rays [first, first+count) of a drop record into d_cell_mass (FP64, theta-major);
 * area_weight mm^2 per unit exit power.  Stats accumulate into *stats (host). */
int icp_drop_trace_bin(icp_context* ctx, const icp_drop_record* record, uint64_t first, uint64_t count,
                       double area_weight, const icp_grid* grid, const double* d_edges, double* d_cell_mass,
                       icp_trace_stats* stats);
/* Host-buffer entry used by the rainbow_generate drop-in: trace + bin (+ diffraction) + CDF. */
int icp_drop_generate(icp_context* ctx, const icp_drop_record* record, double* h_phi, double* h_theta, double* h_u,
                      icp_drop_report* report);
/* The same record with the stored CDF left in caller device arrays d_phi[cp+1],
 * d_theta[cp*(ct+1)] and (unless NULL) d_u[ct+1]: no host copy of the outputs. */
int icp_drop_generate_device(icp_context* ctx, const icp_drop_record* record, double* d_phi, double* d_theta,
                             double* d_u, icp_drop_report* report);

/* ------------------------------------------------------------ batched drop records */
/* Many drop records in one persistent launch fed from a device work queue (no reference
 * counterpart: the reference runs one rainbow_generate process per record, driven by
 * tools/generate_phase_dataset.py:296-311).  Every record keeps its own seed and ray ids,
 * so its result equals the single-record entry's up to FP64 summation order. */
typedef struct {
    double radius_mm;
    double coefficients[8];
    double inclination_deg;
    double interior_index;
    double wavelength_nm;     /* used by the diffraction stage                              */
    uint64_t rays, seed;
    uint32_t diffraction;     /* 1: add the analytic Fraunhofer stage                       */
    uint32_t reserved;
} icp_drop_item;

typedef struct {
    uint32_t nt, np, ct, cp;  /* one (u, phi) grid and storage grid for the whole batch      */
    uint32_t max_internal_hits, precision;
    double exterior_index, tail_tolerance, balance_tolerance;
    icp_cdf_policy policy;
    uint32_t block_threads;   /* 0: autotuned or 256                                        */
    uint32_t blocks_per_sm;   /* 0: as many as fit                                          */
    uint32_t chunk_rays;      /* ray ids per work-queue chunk, 0: autotuned or 8192         */
    uint32_t use_graph;       /* 1: launch the batch as a captured CUDA graph (replayed when
                                 the next batch has the same shape)                         */
} icp_batch_settings;

/* Traces, bins and stores `count` records; phi/theta of record r at d_phi + r*(cp+1) and
 * d_theta + r*cp*(ct+1) (device arrays).  reports[count] on the host. */
int icp_drop_batch_generate_device(icp_context* ctx, const icp_drop_item* items, uint32_t count,
                                   const icp_batch_settings* settings, double* d_phi, double* d_theta,
                                   icp_drop_report* reports);
/* The same with host output arrays (phi, theta as above; u[ct+1] shared by all records). */
int icp_drop_batch_generate(icp_context* ctx, const icp_drop_item* items, uint32_t count,
                            const icp_batch_settings* settings, double* h_phi, double* h_theta, double* h_u,
                            icp_drop_report* reports);
/* Autotuner: times the batch kernel on a bounded sample of `items` for each candidate block
 * size and chunk size and returns the fastest in settings->block_threads / chunk_rays
 * (cached in the context per precision and grid, and used when those fields are 0). */
int icp_drop_batch_autotune(icp_context* ctx, const icp_drop_item* items, uint32_t count,
                            icp_batch_settings* settings, double* best_rays_per_second);

/* ------------------------------------------------------------ surrogate */
/* Building block of the learned surrogate's dense layers (no reference counterpart): BF16
 * C[m x n] = A[m x k] * B[n x k]^T on the 5th-generation tensor cores with FP32 accumulation in
 * tensor memory (tcgen05.mma, TMA-fed).  A and B row-major (K contiguous), 16-byte aligned;
 * m % 128 == 0, n in {64, 128, 256}, k % 64 == 0, m and k at most 2^31.  accumulate = 0: C is written (split_k must
 * be 1); accumulate = 1: C += A B^T with the K range split over split_k CTAs per row tile. */
int icp_mlp_gemm_bf16(icp_context* ctx, const void* d_a, const void* d_b, uint32_t m, uint32_t n, uint32_t k,
                      uint32_t split_k, float* d_c, int accumulate);

/* A small MLP conditioned on a drop record's parameters that predicts the log cell mass of its
 * record on an (nt x np) cell grid: input row = 16 record features + cell features (theta,
 * phi harmonics; the phi harmonics are even about phi = pi/2, the mirror symmetry of a drop
 * record), three SiLU layers of `hidden` units (BF16 weights and activations, FP32
 * accumulation on the tensor cores), a linear head to one value y per cell.  Cell probability =
 * softmax of y over the record's cells.  Trained by the mean per-record KL divergence of the
 * tracer's cell probabilities (records traced without the diffraction stage, which
 * icp_surrogate_generate adds analytically) from the prediction. */
typedef struct icp_surrogate icp_surrogate;

typedef struct {
    uint32_t nt, np;               /* cell grid: theta rows x phi columns, nt * np % 256 == 0   */
    uint32_t hidden;               /* 128 or 256                                                */
    uint32_t input_width;          /* 64 or 128: 16 record features, then the cell features     */
    uint32_t theta_frequencies;    /* sin / cos (k theta), k = 1..F                             */
    uint32_t phi_frequencies;      /* cos (l (phi - pi/2)), l = 1..G                            */
    uint32_t max_records;          /* records per call (sizes the activation buffers);          */
                                   /* max_records * nt * np <= 2^31                             */
    uint32_t axis_harmonics;       /* P: T_k(cos psi), k = 1..P, in the last P input columns;   */
                                   /* psi = angle of the cell's direction to the drop's axis,   */
                                   /* P % 8 == 0, 4 + 2F + G + P <= width - 16                  */
    double log_radius_mm[2];       /* ranges mapped onto [-1, 1] by the record features         */
    double wavelength_nm[2];
    double log_wavelength_over_radius[2]; /* ln(lambda / radius), both in mm                    */
    double index_center, index_scale;     /* (n - center) / scale                               */
    double coefficient_scale[8];          /* shape coefficient c_n enters as c_n * scale_n     */
} icp_surrogate_config;

typedef struct {
    float lr, beta1, beta2, eps, weight_decay;
    uint32_t step;                 /* 1-based step number (bias correction)                     */
} icp_adam;

/* Defaults for the batched-record distribution: 256 x 512 cells, 256 hidden, width 128,
 * F = 40, G = 12, P = 16, radius 0.1-3 mm, wavelength 400-700 nm, 16 records per call. */
int icp_surrogate_default_config(icp_surrogate_config* cfg);
/* FP32 parameters, in this order: W1[H][K0], b1[H], W2[H][H], b2[H], W3[H][H], b3[H], w4[H],
 * head bias (1): H*K0 + 2H^2 + 4H + 1. */
uint64_t icp_surrogate_parameter_count(const icp_surrogate_config* cfg);
/* Host-side feature rows (no GPU): 16 BF16 values per record, and the cell table of
 * nt*np rows x (input_width - 16) BF16 values (theta-major cells, as the histogram). */
int icp_surrogate_record_features(const icp_surrogate_config* cfg, const icp_drop_item* items, uint32_t count,
                                  uint16_t* out);
int icp_surrogate_cell_features(const icp_surrogate_config* cfg, uint16_t* out);
/* The input rows the device builds for `count` records (count * nt*np rows x input_width BF16
 * bits, record-major): record features, cell features and the axis harmonics, which depend on
 * both (cos psi = -sin(a) cos(theta) - cos(a) sin(theta) sin(phi), a = inclination, phi the
 * column's azimuth in [-pi, pi), each T_k by the Chebyshev recurrence in FP64, then rounded to
 * FP32 and BF16). */
int icp_surrogate_inputs(icp_surrogate* s, const icp_drop_item* items, uint32_t count, uint16_t* h_out);
int icp_surrogate_create(icp_context* ctx, const icp_surrogate_config* cfg, icp_surrogate** out);
void icp_surrogate_destroy(icp_surrogate* s);
/* Loads the parameters (and their BF16 copies); resets the Adam moments. */
int icp_surrogate_set_parameters(icp_surrogate* s, const float* h_params, uint64_t count);
int icp_surrogate_get_parameters(icp_surrogate* s, float* h_params, uint64_t count);
/* Mean per-record KL divergence of d_target[count][nt*np] (FP32 cell probabilities, device,
 * each record summing to 1) from the prediction, and (h_grad not NULL) its gradient in the
 * parameter layout. */
int icp_surrogate_gradient(icp_surrogate* s, const icp_drop_item* items, uint32_t count, const float* d_target,
                           float* h_grad, double* loss);
/* One training step: the gradient above, then Adam on the device. loss may be NULL. */
int icp_surrogate_train_step(icp_surrogate* s, const icp_drop_item* items, uint32_t count, const float* d_target,
                             const icp_adam* opt, double* loss);
/* y of every cell: d_logits[count][nt*np] (device FP32), log cell mass up to a per-record constant. */
int icp_surrogate_predict(icp_surrogate* s, const icp_drop_item* items, uint32_t count, float* d_logits);
/* Records from the prediction: the network gives the geometric-optics cell mass exp(y); an item
 * with diffraction = 1 also gets the analytic Fraunhofer rows of the circle of its projected area
 * (CPU FP64, on host threads while the device runs the network) carrying the same total power,
 * as in a traced record.  Then the CDF build at storage grid (ct, cp); phi / theta of record r
 * at d_phi + r*(cp+1), d_theta + r*cp*(ct+1) (device), one CDF report per record (host; status
 * = the record's audit result). */
int icp_surrogate_generate(icp_surrogate* s, const icp_drop_item* items, uint32_t count, uint32_t ct, uint32_t cp,
                           const icp_cdf_policy* policy, double* d_phi, double* d_theta, icp_cdf_report* reports);
/* Training targets: cell probabilities of `count` stored records at the surrogate's grid
 * (ct = nt, cp = np), d_target[count][nt*np] (device FP32). */
int icp_surrogate_targets(icp_surrogate* s, const double* d_phi, const double* d_theta, uint32_t count,
                          float* d_target);

/* --------------------------------------------------------------------- deterministic atlas
 * Fixed-incidence responses of one hexagonal prism on a grid of incident directions in the
 * symmetry domain (theta in [0, pi/2] from the body +y axis, phi in [0, pi/6]), then reused by
 * a deterministic orientation composition.  No random numbers anywhere: entry points come
 * from a projected-area quadrature, orientations from a fixed product rule. */

/* One quadrature ray: entry face, entry point in units of the circumradius (body frame), and
 * its projected-area weight in mm^2.  40 bytes. */
typedef struct {
    uint32_t face;
    uint32_t reserved;
    double x, y, z;
    double weight_mm2;
} icp_atlas_ray;

/* Projected-area quadrature of the prism lit from direction ki (used as given when it is a unit
 * vector to 128 ulp, as make_area_rule requires; otherwise normalised first): S x S equal-area cells per lit side face and per end-cap sector, 2 x 3
 * Gauss-Legendre points per cell; replaces atlas::make_area_rule
 * (hex_atlas/include/ice_crystal/atlas.hpp:17, hex_atlas/src/atlas.cpp:11-51).  rays == NULL
 * returns the count only; otherwise capacity must hold it (ICP_ERR_CAPACITY).  Invalid
 * geometry or S (S*S > 10^6) -> ICP_ERR_INVALID_ARGUMENT; a point on an ambiguous boundary or
 * a failed area audit (1e-12) -> ICP_ERR_AUDIT. */
int icp_atlas_area_rule(double circumradius_mm, double length_mm, const double ki[3], uint32_t subdivisions,
                        icp_atlas_ray* rays, uint64_t capacity, uint64_t* count);

typedef struct {
    double theta, phi;  /* node angles (rad) */
    double ki[3];       /* incident propagation direction of the trace */
    double e0[3], e1[3];/* its spherical frame: e0 = (cos t cos p, -sin t, cos t sin p), e1 = ki x e0 */
    double rule_ki[3];  /* the direction the area quadrature is built for (ki before its second
                           normalisation, as atlas::make_node passes it to make_area_rule) */
} icp_atlas_incident;

/* Incident node (i, j) of theta_intervals x phi_intervals (end points included); replaces the
 * frame part of atlas::make_node (hex_atlas/src/atlas.cpp:76-97). */
int icp_atlas_incident_node(uint32_t theta_intervals, uint32_t phi_intervals, uint32_t i, uint32_t j,
                            icp_atlas_incident* out);

typedef struct {
    double circumradius_mm, length_mm;
    double interior_index, exterior_index;
    uint32_t theta_intervals, phi_intervals; /* incident grid, <= 4096 each */
    uint32_t nt, np;                         /* outgoing cell grid, nt*np <= 10^8 */
    uint32_t subdivisions;                   /* area quadrature S, S*S <= 10^6 */
    uint32_t max_internal_hits;              /* 2048 */
    double tail_tolerance;                   /* 1e-12 */
    double max_unresolved_fraction;          /* 1e-10 */
    double max_balance_error;                /* 1e-10 */
} icp_atlas_settings;

typedef struct {
    double projected_area_mm2;   /* analytic projected area at the node */
    double escaped_mm2;          /* sum over rays of weight x escaped power (ray order, Kahan) */
    double unresolved_mm2;       /* the same for the power left in the chain */
    double histogram_mass_mm2;   /* sum of the node's cell masses */
    double histogram_relative_error;
    double max_balance_error, max_interface_balance_error;
    uint64_t rays, outputs, invalid_bins;
    uint64_t status[8];          /* rays per icp_ray_status */
    int64_t first_rejected;      /* quadrature index of the first rejected ray, -1 if none */
} icp_atlas_node_report;

/* Traces every quadrature ray of incident node (i, j) on the device (FP64, each ray's linear
 * R/T chain as the prism tracer) and writes the node's cell masses in mm^2 to
 * d_mass[nt*np] (device, theta-major; pole exits spread uniformly over the end rows).  The
 * histogram is accumulated in exact 64-bit fixed point (2^-62 of the node's projected
 * area), so the result does not depend on thread scheduling; no floating-point atomics.
 * Replaces atlas::CudaTracer::trace (hex_atlas/include/ice_crystal/atlas_cuda.hpp:15,
 * hex_atlas/src/atlas_cuda.cpp:30-58) and atlas::trace_cpu (atlas.cpp:140-153), with the
 * same gates: every ray accepted with interface balance <= max_balance_error
 * (ICP_ERR_AUDIT naming the first rejected ray), histogram / escaped and
 * (escaped + unresolved) / area within max_balance_error, unresolved / area <=
 * max_unresolved_fraction. */
int icp_atlas_trace_node(icp_context* ctx, const icp_atlas_settings* settings, uint32_t i, uint32_t j,
                         double* d_mass, icp_atlas_node_report* report);

/* Orientation coupling of one incident direction: for every rotation r (d_rotations[n][9],
 * row-major body -> ensemble, device) with number weight d_weights[n] (device), the body
 * direction r^T ki is folded into the symmetry domain by one of the 24 operations of D6h
 * (reflections included), the node response is interpolated bilinearly in (theta, phi) after
 * division by the node areas h_node_area[(T+1)*(P+1)] (host), weighted by the exact
 * projected area at the query and shifted in phi by the (fractional) cell offset of the
 * folded frame.  Adds fraction x weights into d_coupling[(T+1)(P+1)][2][np] (device,
 * [node][parity][shift]; parity 1 = phi reflected), after replacing each [node][parity]
 * row by its mean when orbit_average != 0 (exact average over a uniform world azimuth, used
 * at vertical incidence).  Accumulation is exact fixed point (order-independent).  Replaces
 * coupling / coupling_for_rule (hex_atlas/python/atlas_math.py:272-428).  *expected_area =
 * sum of weight x projected area (mm^2, before the fraction).  A fold outside the domain or
 * an inconsistent unfolding -> ICP_ERR_AUDIT. */
int icp_atlas_coupling(icp_context* ctx, uint32_t theta_intervals, uint32_t phi_intervals, uint32_t np,
                       double circumradius_mm, double length_mm, const double* h_node_area,
                       const double* d_rotations, const double* d_weights, uint64_t count, const double ki[3],
                       double fraction, int orbit_average, double* d_coupling, double* expected_area);

/* Composed cell mass d_out[nt*np] (device) = sum over nodes n, parities q and shifts s of
 * d_coupling[n][q][s] x (the node's cell masses d_mass[n][nt][np], phi-reflected when q = 1,
 * rolled by s cells in phi): a non-negative direct cyclic convolution in FP64 with a fixed
 * summation order per cell.  Replaces compose_mass (atlas_math.py:431-447). */
int icp_atlas_compose(icp_context* ctx, uint32_t nodes, uint32_t nt, uint32_t np, const double* d_mass,
                      const double* d_coupling, double* d_out);

/* -------------------------------------------------- Table-II rainbow diffraction */
/* Local diffraction at the rainbows on a (theta, phi) query grid of the drop's focal stage:
 * the reference's Sadeghi-2012 Table-II model (include/rainbow/rainbow_diffraction.hpp) run by
 * PatchOptics::run_diffraction (src/patch_optics.cpp:334-348).  The query grid has nt theta
 * rows (centre theta = (row + 1/2) pi / nt, theta = angle between the incident and outgoing
 * propagation directions) of np phi cells, direction index = row * np + column.
 *
 * One direction of the focal stage, laid out as rainbow::FocalOpticalResult
 * (include/rainbow/wave_optics_data.hpp:27-40, 144 bytes), so that the reference's
 * focal-results buffer is passed unchanged.  The pass reads intensity_s, intensity_p,
 * family_incoherent[2..3], family_hits[2..3] (families R, TT, TRT, TRRT) and flags
 * (0 = valid). */
typedef struct {
    double field[4];                 /* column-0 field: s re, s im, p re, p im (unused)      */
    double intensity_s, intensity_p; /* unpolarized focal intensities                         */
    double family_incoherent[4];
    uint32_t family_hits[4];
    uint32_t corrected_hits, extra_quarter_turn_hits;
    uint32_t flags, first_problem_patch_id;
    double field_second[4];          /* column-1 field (unused)                               */
} icp_focal_sample;

/* rainbow::DiffractionConfig (wave_optics_data.hpp:48-54). */
typedef struct {
    double primary_sigma_rad;   /* Gaussian width at the primary bow; the secondary uses 2x   */
    double support_sigma;       /* stencil radius in sigmas (4)                               */
    double transition_contrast; /* minimum relative jump of the total intensity (0.25)        */
    double inner_blend_sigma;   /* full blend inside, smoothstep taper to the support (3)     */
} icp_diffraction_config;

/* rainbow::DiffractionResult (wave_optics_data.hpp:66-78, 40 bytes). */
typedef struct {
    double intensity_s, intensity_p; /* NaN when unavailable                                  */
    double sigma_rad, blend;
    uint32_t flags, transition_kind;
} icp_diffraction_result;

/* Transition flags of the edge between row r and row r + 1 at one phi (RainbowTransitionFlags),
 * and result flags (DiffractionFlags). */
enum icp_transition_flags { ICP_TRANSITION_PRIMARY = 1, ICP_TRANSITION_SECONDARY = 2, ICP_TRANSITION_UNKNOWN = 4 };
enum icp_diffraction_flags {
    ICP_DIFFRACTION_FILTERED = 1,
    ICP_DIFFRACTION_UNDERRESOLVED = 2,
    ICP_DIFFRACTION_INPUT_UNAVAILABLE = 4,
    ICP_DIFFRACTION_STENCIL_UNAVAILABLE = 8,
    ICP_DIFFRACTION_DETECTION_UNAVAILABLE = 16,
    ICP_DIFFRACTION_INVALID_DATA = 32
};

/* The diffraction counters of rainbow::WaveOpticsStatistics (src/patch_optics.cpp:224-229). */
typedef struct {
    uint32_t primary_transitions, secondary_transitions, unknown_transitions;
    uint32_t filtered_directions, unavailable_directions, underresolved_directions;
} icp_diffraction_stats;

/* Table-II primary width in degrees for a drop radius in mm (0.1 .. 1.0 mm, linear between
 * the table's radii; RainbowDiffraction::table_sigma_degrees, rainbow_diffraction.hpp:16-28).
 * Host function.  Outside the table -> ICP_ERR_INVALID_ARGUMENT, *primary_sigma_deg untouched. */
int icp_rainbow_table_sigma(float radius_mm, double* primary_sigma_deg);

/* Transition labels d_transitions[nt*np] (device) of the focal grid d_focal[nt*np] (device):
 * kernel detect_rainbow_transitions (device/patch_optics.cu:26-32).  An invalid configuration
 * (RainbowDiffraction::valid_config) -> ICP_ERR_INVALID_ARGUMENT, as PatchOptics::evaluate
 * rejects it (src/patch_optics.cpp:92-95). */
int icp_rainbow_detect(icp_context* ctx, const icp_focal_sample* d_focal, uint32_t nt, uint32_t np,
                       const icp_diffraction_config* config, uint32_t* d_transitions);

/* Filtered directions d_results[nt*np] (device) from the focal grid and the given labels:
 * kernel filter_rainbow_diffraction (device/patch_optics.cu:34-40).  d_density (device, may
 * be NULL) receives intensity_s + intensity_p of every result, the density the reference's
 * CDF builder reads for the diffraction stage (device/phase_cdf.cu:53-55), ready for
 * icp_phase_cdf_build(ICP_CDF_DENSITY).  stats (host, may be NULL): the result counters
 * (transition counters zero). */
int icp_rainbow_filter(icp_context* ctx, const icp_focal_sample* d_focal, const uint32_t* d_transitions, uint32_t nt,
                       uint32_t np, const icp_diffraction_config* config, icp_diffraction_result* d_results,
                       double* d_density, icp_diffraction_stats* stats);

/* Both passes and all counters, as PatchOptics::run_diffraction plus its statistics loop. */
int icp_rainbow_diffraction(icp_context* ctx, const icp_focal_sample* d_focal, uint32_t nt, uint32_t np,
                            const icp_diffraction_config* config, uint32_t* d_transitions,
                            icp_diffraction_result* d_results, double* d_density, icp_diffraction_stats* stats);

/* ----------------------------------------- patch optics (incoherent, path, focal stages) */
/* Per-direction optics of the drop's wave stages from the outgoing-ray lattice, its patches
 * and the query hits: the reference's PatchOpticalEvaluator
 * (include/rainbow/patch_optical_evaluator.hpp) as launched by evaluate_patch_optics /
 * evaluate_focal_optics (device/patch_optics.cu:7-24; src/patch_optics.cpp:150-175).  The
 * records below have the reference's layouts (raindrop_trace_data.hpp, outgoing_patch.hpp,
 * patch_query_data.hpp, patch_optics_data.hpp), so its device buffers pass unchanged.
 * Folded-branch records are not taken: a hit on a NeedsRefinement patch is reported as
 * refinement-pending, as the reference does without its folded view. */
typedef struct { float x, y, z; } icp_vec3f;
typedef struct { float real, imag; } icp_complex32;
typedef struct { icp_complex32 x, y; } icp_field32;          /* Jones vector in a transverse frame */
typedef struct { int32_t turns; float fraction; } icp_phase_cycles; /* optical path in cycles  */

typedef struct {                                             /* rainbow::OutgoingVertex, 68 B     */
    icp_vec3f position_drop, direction_drop, basis_x;
    icp_field32 field;
    icp_phase_cycles optical_cycles;
    uint32_t status;                                         /* 1 = valid                         */
    uint32_t diagnostics;
} icp_outgoing_vertex;

typedef struct {                                             /* rainbow::OutgoingPatch, 32 B      */
    uint32_t vertex_indices[4];
    uint32_t patch_id;                                       /* family x cells + iy (W-1) + ix    */
    uint32_t status;                                         /* 1 / 2 regular, 3 needs refinement */
    float signed_solid_angle_sr, incident_area_drop2;
} icp_outgoing_patch;

typedef struct {                                             /* rainbow::PatchQueryHit, 32 B      */
    uint32_t compact_index, patch_id, root_index, flags;     /* flags: 1 boundary, 2 singular, 4 fp64 */
    float u, v, t, residual;
} icp_query_hit;

typedef struct {                                             /* rainbow::PatchQuerySummary, 32 B  */
    uint32_t candidate_count, hit_count, regular_hits, refinement_hits, boundary_hits, flags;
    uint32_t first_problem_patch_id, reserved;
} icp_query_summary;

typedef struct { double s_real, s_imag, p_real, p_imag; } icp_field64;

typedef struct {                                             /* rainbow::PatchOpticalResult, 136 B */
    icp_field64 path_field;                                  /* input column 0                    */
    double incoherent_s, incoherent_p, path_s, path_p;
    uint32_t hit_count, evaluated_hits, rejected_hits, refinement_hits, boundary_hits, singular_hits;
    uint32_t flags, query_flags, first_problem_patch_id, folded_hits;
    icp_field64 path_field_second;                           /* input column 1 (unpolarized)      */
} icp_optical_result;

typedef struct {                                             /* rainbow::PatchOpticsParams        */
    const icp_outgoing_vertex* vertices;                     /* device arrays                     */
    const icp_outgoing_patch* patches;
    const icp_vec3f* directions;                             /* direction_count query directions  */
    const uint64_t* offsets;                                 /* direction_count + 1 hit offsets   */
    const icp_query_summary* summaries;
    const icp_query_hit* hits;
    const icp_field32* second_input_fields;                  /* vertex_count, or NULL             */
    uint64_t hit_storage_count;
    uint32_t vertex_count, patch_count, direction_count, second_input_count;
    icp_vec3f incident_direction, incident_basis_x;
    uint32_t input_polarization;                             /* 0 single Jones, 1 unpolarized     */
    uint32_t reserved;
} icp_optics_input;

typedef struct {                                             /* rainbow::FocalPhaseConfig, 32 B   */
    uint32_t grid_width, grid_height;
    float grid_half_extent;
    uint32_t reserved;
    uint32_t quarter_turn_offsets[4];                        /* per family, 0 .. 3                */
} icp_focal_config;

/* ------------------------------------------------------- lattice trace (drop wave stages) */
/* rainbow::RaindropTraceConfig, 116 B (include/rainbow/raindrop_trace_data.hpp:61-96): the drop
 * shape (r/a = 1 + sum c_n cos(n chi), chi from -y, with conservative inner / outer radii), the
 * incident direction and its transverse basis e0, the single-input field, the radius, vacuum
 * wavelength and indices, and the incident lattice (grid_width x grid_height vertices spanning
 * [-grid_half_extent, grid_half_extent]^2 about the drop, reference_distance before it). */
typedef struct {
    float coefficients[8];
    float inner_radius, outer_radius;
    icp_vec3f incident_direction, incident_basis_x;
    icp_field32 incident_field;
    float radius_mm, wavelength_nm, exterior_index, interior_index;
    float grid_half_extent, reference_distance, outgoing_reference_distance;
    uint32_t grid_width, grid_height;
} icp_raindrop_config;

/* RaindropSettings::make_config (include/rainbow/raindrop_settings.hpp:19-43) for an
 * unpolarised trace: the Table-I shape of radius_mm (RaindropShape::try_make; sphere != 0 forces
 * the sphere) or, with coefficients != NULL, those 8 coefficients with the same bounding radii;
 * incident_direction normalised in binary32 and e0 from TransverseFrame::from_direction;
 * exterior index 1, half extent 1.01 r_out, reference distances 2 r_out.  The reference's range
 * checks and messages (radius (0,3], wavelength [380,830] nm, interior index [1,2], grid >= 2 with
 * 4 W H < 2^32, finite nonzero direction) -> ICP_ERR_INVALID_ARGUMENT.  Host function. */
int icp_raindrop_config_make(float radius_mm, int sphere, const float* coefficients, float wavelength_nm,
                             float interior_index, const float incident_direction[3], uint32_t grid_width,
                             uint32_t grid_height, icp_raindrop_config* out);

/* Per-family vertex statuses of a lattice trace and the trace validation of
 * PhaseCdf::validate_trace (src/phase_cdf.cpp:238-253). */
typedef struct {
    uint64_t status_counts[4][8];   /* [family R, TT, TRT, TRRT][VertexStatus 0..7]                 */
    uint64_t intersection_fallbacks; /* records whose diagnostics carry IntersectionFallback (1)    */
    uint64_t snell_fallbacks;        /* ... SnellFallback (2)                                        */
    uint64_t incomplete;             /* records neither Valid, Miss nor TIR, or Valid with a
                                        non-finite value or an invalid optical path                  */
    uint64_t first_problem;          /* smallest such record index, or UINT64_MAX                    */
} icp_lattice_stats;

/* The four-family outgoing-ray lattice of one drop: per vertex (row-major, index iy W + ix) one
 * incident ray traced through R, TT, TRT and TRRT into d_vertices[4 W H] (device, family-major:
 * record f W H + index), exactly RaindropPathTracer::trace_vertex_unpolarized
 * (include/rainbow/raindrop_paths.hpp:27-107) with the reference's intersector and interface,
 * every record bit-identical to the reference's.  d_second_fields[4 W H] (device) receives the
 * second response column (unpolarised trace: unit input states, RaindropTracer::
 * trace_unpolarized); with d_second_fields == NULL the single-input trace of
 * config->incident_field (RaindropTracer::trace).  stats (host, may be NULL) gets the status
 * histogram and the trace validation.  Replaces RaindropTracer::trace_unpolarized's OptiX launch
 * (src/raindrop_tracer.cpp:144-177, shaders/entry/raindrop_trace.cu:49-83) and
 * PhaseCdf::validate_trace. */
int icp_lattice_trace(icp_context* ctx, const icp_raindrop_config* config, icp_outgoing_vertex* d_vertices,
                      icp_field32* d_second_fields, icp_lattice_stats* stats);

/* Padded bounding box of a patch's four corner directions (rainbow::PatchAabb, 24 B). */
typedef struct { float min_x, min_y, min_z, max_x, max_y, max_z; } icp_patch_aabb;

/* Patches of a four-family outgoing-ray lattice d_vertices[4 * W * H] (device; family-major,
 * row-major within a family, the layout of RaindropTracer's vertex buffer): every cell with
 * four outgoing corner rays, certified regular (status 1 / 2, signed solid angle) or needing
 * refinement (3), stored compactly in patch_id order in d_patches (device, capacity
 * 4 (W-1)(H-1)) with its padded box in d_aabbs (device, may be NULL); each cell's status
 * (0..7) in d_statuses[4 (W-1)(H-1)] (device, may be NULL).  *patch_count and histogram[8]
 * (per status, may be NULL) on the host.  Replaces PatchAccel::build's kernels
 * classify_outgoing_patches / compact_outgoing_patches (device/patch_build.cu:13-77) and their
 * host-side scan; an invalid layout (PatchBuildLayout::try_make) -> ICP_ERR_INVALID_ARGUMENT. */
int icp_patch_build(icp_context* ctx, const icp_outgoing_vertex* d_vertices, uint32_t grid_width, uint32_t grid_height,
                    float grid_half_extent, icp_outgoing_patch* d_patches, icp_patch_aabb* d_aabbs, uint32_t* d_statuses,
                    uint32_t* patch_count, uint64_t histogram[8]);

/* The reference's query directions (QueryDirectionGrid, include/rainbow/query_direction_grid.hpp
 * :14-58): theta_count x phi_count cell centres about `axis` (theta from the axis, phi from -pi
 * at e0 toward axis x e0), normalised binary32, row-major, into directions[3 * nt * np] (host).
 * A frame that is not orthonormal to 1e-5 -> ICP_ERR_INVALID_ARGUMENT.  Host function. */
int icp_query_directions(uint32_t theta_count, uint32_t phi_count, const float axis[3], const float e0[3],
                         float* directions);

/* All-hit query of the patches (device arrays from icp_patch_build) for every direction:
 * each patch whose padded box the ray t d (0 <= t <= 4) meets is intersected (binary32, and
 * binary64 where binary32 is not conclusive: BilinearPatchIntersector, include/rainbow/
 * bilinear_patch_intersection.hpp), and each direction's hits are stored sorted by
 * (patch_id, compact index, root) with duplicates removed, as the reference's OptiX query and
 * PatchHitCollector produce them (shaders/entry/patch_query.cu, include/rainbow/
 * patch_query_data.hpp:43-128).  d_offsets[direction_count + 1] (device) always; *hit_count
 * (host) = d_offsets[direction_count].  With d_hits == NULL or d_summaries == NULL the call only
 * sizes; otherwise d_hits needs hit_capacity >= *hit_count (else ICP_ERR_CAPACITY) and
 * d_summaries[direction_count] receives the summaries.  Replaces PatchQuery::query_grid's two
 * OptiX launches (src/patch_query.cpp). */
int icp_patch_query(icp_context* ctx, const icp_outgoing_vertex* d_vertices, uint32_t vertex_count,
                    const icp_outgoing_patch* d_patches, const icp_patch_aabb* d_aabbs, uint32_t patch_count,
                    const icp_vec3f* d_directions, uint32_t direction_count, uint64_t* d_offsets,
                    icp_query_summary* d_summaries, icp_query_hit* d_hits, uint64_t hit_capacity, uint64_t* hit_count);

/* Optics of every query direction: d_results[direction_count] (device).  With focal != NULL
 * also the focal stage d_focal[direction_count] (device; the input of icp_rainbow_diffraction).
 * Malformed inputs are reported per direction in the result flags, as the reference does;
 * only null pointers and sizes that overflow are rejected here.  Without folded records: a hit
 * on a NeedsRefinement patch is refinement-pending. */
int icp_patch_optics(icp_context* ctx, const icp_optics_input* input, icp_optical_result* d_results,
                     const icp_focal_config* focal, icp_focal_sample* d_focal);

/* --------------------------------------------------------------------- folded patches */
/* A NeedsRefinement patch's direction map folds (its Jacobian changes sign inside the cell);
 * the reference then evaluates each hit with the connected sign component ("branch") that
 * contains it (include/rainbow/folded_patch_data.hpp, folded_patch_geometry.hpp,
 * folded_patch_builder.hpp). */
typedef struct {                                             /* rainbow::FoldedPatchConfig, 16 B */
    double relative_tolerance;                               /* 1e-8 (1e-12 .. 1e-3)             */
    uint32_t maximum_panels;                                 /* 2048 (1 .. 65536)                */
    uint32_t maximum_depth;                                  /* 20 (1 .. 24)                     */
} icp_folded_config;

typedef struct {                                             /* rainbow::FoldedBranch, 64 B      */
    double u0, u1;                                           /* u extent of the component        */
    double area_fraction, solid_angle_sr;                    /* share of the cell, unsigned sr   */
    double representative_u, representative_v;
    int32_t sign;                                            /* sign of J on the component       */
    uint32_t focal_flags, quarter_turns, extra_quarter_turn; /* focal estimate at the point      */
} icp_folded_branch;

typedef struct {                                             /* rainbow::FoldedPatchRecord, 320 B */
    uint32_t compact_index, patch_id;
    uint32_t flags;                                          /* 0 ready; FoldedPatchFlags bits   */
    uint32_t branch_count;
    double jacobian[4];                                      /* corners 00 10 01 11, scaled      */
    icp_folded_branch branches[4];
    double largest_estimated_relative_error;
    uint32_t panels, reserved;
} icp_folded_record;

typedef struct {                                             /* rainbow::FoldedPatchView, 24 B   */
    const uint32_t* record_indices;                          /* by compact patch index (device)  */
    const icp_folded_record* records;                        /* device                           */
    uint32_t patch_count, record_count;
} icp_folded_view;

typedef struct {                                             /* FoldedPatchStatistics (records)  */
    uint32_t candidates, prepared, unresolved, branch_count, focal_pending_branches, reserved;
    double largest_estimated_relative_error;
} icp_folded_stats;

/* The folded-patch record of every NeedsRefinement patch of d_patches[patch_count] (device,
 * from icp_patch_build) over the lattice d_vertices[vertex_count] (device): records in
 * compact-index order in d_records (device, capacity), d_record_indices[patch_count] (device)
 * the record of each patch or 0xffffffff.  FoldedPatchBuilder::prepare per record (the
 * reference's prepare_folded_patches, device/patch_optics.cu:46-60, which takes slots in
 * completion order); with focal != NULL each ready branch also gets its focal quarter turns
 * (FocalPhase::estimate_at).  config NULL = the reference's defaults.  *record_count (host)
 * always; with d_records == NULL or capacity < count -> ICP_ERR_CAPACITY after the count.
 * stats (host, may be NULL): PatchOptics::collect_folded_statistics. */
int icp_folded_prepare(icp_context* ctx, const icp_outgoing_vertex* d_vertices, uint32_t vertex_count,
                       const icp_outgoing_patch* d_patches, uint32_t patch_count, const float incident[3],
                       const icp_focal_config* focal, const icp_folded_config* config, uint32_t* d_record_indices,
                       icp_folded_record* d_records, uint32_t capacity, uint32_t* record_count,
                       icp_folded_stats* stats);

/* icp_patch_optics with folded records (folded may be NULL): the reference's
 * evaluate_folded_optics (device/patch_optics.cu:62-68) -- a hit on a folded patch takes the
 * area and solid angle of its branch and, for the focal stage, the branch's quarter turns; a
 * direction whose refinement hits are not all accounted for by records stays pending or is
 * flagged invalid (PatchOpticalEvaluator::evaluate_direction). */
int icp_patch_optics_folded(icp_context* ctx, const icp_optics_input* input, icp_optical_result* d_results,
                            const icp_focal_config* focal, icp_focal_sample* d_focal, const icp_folded_view* folded);

/* ------------------------------------------------------- wave-stage CDF input */
/* The density a wave stage hands to the CDF builder and the builder's input audit
 * (device/phase_cdf.cu:40-56, 93-108: density() and phase_check_density).  Per direction:
 *   incoherent   incoherent_s + incoherent_p of d_optical
 *   path         path_s + path_p of d_optical
 *   focal        intensity_s + intensity_p of d_focal
 *   diffraction  intensity_s + intensity_p of d_diffraction (underresolved when flagged)
 * incomplete: the optical result's known hits are not complete (flags with an error or pending
 * bit, a rejected hit, or evaluated != hit_count), and for focal / diffraction also an invalid
 * focal or an unavailable diffraction result.  The reference rejects a record whose input has
 * an invalid value (non-finite or negative), an incomplete direction, no positive density, or an
 * underresolved direction unless allowed (src/phase_cdf.cpp:325-328); the report carries the
 * counts, the host applies that gate.  d_density[count] (device) feeds icp_phase_cdf_build with
 * ICP_CDF_DENSITY. */
enum icp_wave_stage { ICP_STAGE_INCOHERENT = 1, ICP_STAGE_PATH = 2, ICP_STAGE_FOCAL = 3, ICP_STAGE_DIFFRACTION = 4 };
typedef struct {
    double maximum;            /* largest valid density                                      */
    uint64_t invalid_values, incomplete, underresolved;
    uint64_t first_problem;    /* first direction that is invalid, incomplete or underresolved;
                                  UINT64_MAX when none                                        */
} icp_density_report;
int icp_stage_density(icp_context* ctx, uint32_t stage, const icp_optical_result* d_optical,
                      const icp_focal_sample* d_focal, const icp_diffraction_result* d_diffraction, uint64_t count,
                      double* d_density, icp_density_report* report);

#ifdef __cplusplus
}
#endif
#endif /* ICP_B200_H */
