/* coffee_b200.h -- C ABI of the B200 force-free field-update library.
 *
 * The library replaces one hot path of COFFEE (fizban007/CoffeeGPU): the
 * field update of the EZ force-free solver, i.e.
 *   Coffee::field_solver_EZ::evolve_fields(Scalar time)
 *     (src/algorithms/field_solver_EZ.h:6-33; CPU build
 *      src/algorithms/field_solver_EZ.cpp:1007-1073; GPU build
 *      src/algorithms/field_solver_EZ.cu:656-707)
 * together with the single-rank guard-cell fill it calls after every stage
 *   Coffee::sim_environment::send_guard_cells(sim_data&)
 *     (src/sim_env_impl.hpp:179-228).
 * The objects the reference passes around map to opaque handles:
 *   sim_environment  (src/sim_env.h:17-87)      -> coffee_env
 *   sim_data         (src/data/sim_data.h:11-24) -> coffee_fields
 *   field_solver_EZ  (src/algorithms/field_solver_EZ.h:6-33) -> coffee_solver
 * The reference's staggered RK3 solver, Coffee::field_solver::evolve_fields
 * (src/algorithms/field_solver.h:8-35, src/algorithms/field_solver.cu:690-726),
 * is the variant COFFEE_VARIANT_YEE of the same handle, and its Kerr-Schild
 * counterpart Coffee::field_solver_gr::evolve_fields_gr
 * (src/algorithms/field_solver_gr.cu:810-861) the variant COFFEE_VARIANT_GRYEE.
 * include/coffee_b200.hpp re-creates the reference's C++ classes on top of
 * these calls.
 *
 * Conventions: every call returns COFFEE_OK (0) or a negative status and
 * never exits or throws; coffee_last_error_string() describes the last
 * failure of the calling thread.  Arrays use the reference layout: one array
 * per component, dims = N + 2*guard points per axis (guards included), index
 * i + j*dims[0] + k*dims[0]*dims[1] (src/data/multi_array_impl.hpp:81-91).
 * Real parameters are passed as double and used in the field precision.
 */
#ifndef COFFEE_B200_H
#define COFFEE_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define COFFEE_API __attribute__((visibility("default")))
#else
#define COFFEE_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  COFFEE_OK = 0,
  COFFEE_E_INVALID = -1,   /* bad argument or unsupported configuration */
  COFFEE_E_CONFIG = -2,    /* inconsistent simulation parameters */
  COFFEE_E_CUDA = -3,      /* a CUDA runtime call failed */
  COFFEE_E_NOMEM = -4,     /* device or host allocation failed */
  COFFEE_E_NONFINITE = -5, /* a field holds NaN or Inf */
  COFFEE_E_TIMEOUT = -6,   /* a bounded device wait ran out */
  COFFEE_E_IO = -7         /* file could not be read or written */
};

/* ---- identifiers ------------------------------------------------------- */
enum { /* field ids for coffee_fields_ptr / upload / download */
  COFFEE_EX = 0, COFFEE_EY, COFFEE_EZ, COFFEE_BX, COFFEE_BY, COFFEE_BZ, COFFEE_P,
  COFFEE_JX, COFFEE_JY, COFFEE_JZ, COFFEE_DIVE, COFFEE_DIVB,
  /* background field sim_data::B0, read by the staggered solver (allocated
   * on first use; zero until written) */
  COFFEE_B0X, COFFEE_B0Y, COFFEE_B0Z,
  /* the CPU build's energy-change diagnostics, sim_data::dU_* (sim_data.h:
   * 15-16), written by the flat solver with coffee_solver_set_energy_diag
   * (allocated on first use, zero until written) */
  COFFEE_DU_EGTB, COFFEE_DU_EPAR, COFFEE_DU_KO,
  COFFEE_DU_EGTB_CUM, COFFEE_DU_EPAR_CUM, COFFEE_DU_KO_CUM,
  COFFEE_NUM_FIELDS
};
enum { /* solver variants */
  COFFEE_VARIANT_FLAT = 0,   /* Cartesian EZ, field_solver_EZ */
  COFFEE_VARIANT_LOGSPH = 1, /* 2D log-spherical EZ, field_solver_EZ_spherical (GPU build) */
  COFFEE_VARIANT_CYL = 2,    /* 2D cylindrical EZ, field_solver_EZ_cylindrical (GPU build) */
  COFFEE_VARIANT_GR = 3,     /* Kerr-Schild GR EZ, field_solver_gr_EZ (GPU build); E holds D */
  COFFEE_VARIANT_YEE = 4,    /* staggered (Yee) RK3, field_solver (GPU build only): E and B on
                              * the staggered positions of sim_data.cpp:19-25, B0 subtracted
                              * in curl B; the rotating star with problem 1 (any
                              * other problem: none), shift_ghost 0 */
  COFFEE_VARIANT_GRYEE = 5   /* staggered RK3 in Kerr-Schild coordinates, field_solver_gr
                              * (GPU build only; evolve_fields_gr): E holds D, staggered as
                              * above; no periodic axis, shift_ghost 0; the time argument of
                              * coffee_solver_step is not used */
};
enum { /* which reference build the flat solver reproduces */
  COFFEE_SEM_CPU_REF = 0, /* field_solver_EZ.cpp (the parity oracle build) */
  COFFEE_SEM_GPU_REF = 1  /* field_solver_EZ.cu */
};
enum { /* coffee_diag_reduce quantities, accumulated in FP64 */
  COFFEE_DIAG_ENERGY_E = 0, /* sum E^2 over the region of total_energy() */
  COFFEE_DIAG_ENERGY_B = 1, /* sum B^2 over the same region */
  COFFEE_DIAG_DIVB_L2 = 2,  /* sqrt(sum divB^2) over the interior */
  COFFEE_DIAG_MAX_EDOTB = 3,/* max |E.B| / B^2 over the interior */
  COFFEE_DIAG_MAX_EOVERB = 4/* max |E|/|B| over the interior */
};

/* ---- simulation parameters ---------------------------------------------
 * Same fields, order and defaults as Coffee::sim_params
 * (src/sim_params.h:15-124); coffee_params_default() fills the defaults,
 * coffee_params_parse_toml() reads the keys of parse_config
 * (src/sim_params.cpp:7-146). */
typedef struct coffee_params {
  double dt;
  uint64_t max_steps;
  int data_interval;
  int snapshot_interval;
  int periodic_boundary[3];
  int downsample;
  int slice_x; double slice_x_pos;
  int slice_y; double slice_y_pos;
  int slice_z; double slice_z_pos;
  int slice_xy;
  int slice_interval;
  int downsample_2d;
  int N[3];
  int guard[3];
  double lower[3];
  double size[3];
  int nodes[3];
  int shift_ghost;
  int kn[3];
  double a;
  int calc_current;
  int clean_ep;
  int check_egb;
  int pml[3];
  int pmllen;
  double sigpml;
  int divB_clean;
  double ch2;
  double tau;
  double KOeps;
  int KO_geometry;
  int use_edotb_damping;
  double damp_gamma;
  int problem;
  double radius, omega, b0;
  double p1, p2, p3;
  double q11, q12, q13, q22, q23;
  double q_offset_x, q_offset_y, q_offset_z;
  double tp_start, tp_end, rpert1, rpert2, thp1, thp2, dw0, nT, shear, ph1, ph2, dph,
      theta0, drpert;
  double tp_start1, tp_end1, rpert11, rpert21, thp11, thp21, dw1, nT1, shear1, ph11,
      ph21, dph1;
  int pert_type;
  int skymap_Nth, skymap_Nph;
} coffee_params;

/* Coffee::Grid of one rank (src/data/grid.h:11-266). */
typedef struct coffee_grid {
  int dims[3];
  int guard[3];
  double delta[3];
  double inv_delta[3];
  double lower[3];
  double sizes[3];
  int offset[3];
} coffee_grid;

typedef struct coffee_env coffee_env;
typedef struct coffee_fields coffee_fields;
typedef struct coffee_solver coffee_solver;

/* ---- errors ------------------------------------------------------------ */
/* Message of the last failing call on this thread ("" if none). */
COFFEE_API const char* coffee_last_error_string(void);
/* Library version string. */
COFFEE_API const char* coffee_version(void);

/* ---- parameters -------------------------------------------------------- */
/* sim_params defaults (src/sim_params.h:15-124). */
COFFEE_API void coffee_params_default(coffee_params* p);
/* parse_config (src/sim_params.cpp:7-146): keys missing from the TOML text
 * keep their defaults.  Accepts the TOML subset the reference's config files
 * use (key = value, arrays, # comments). */
COFFEE_API int coffee_params_parse_toml(const char* text, coffee_params* p);

/* ---- environment: sim_environment::sim_environment (src/sim_env_impl.hpp:12-86)
 * for one rank on one GPU: dims = N + 2 guard, delta = size / N. */
COFFEE_API int coffee_env_create(const coffee_params* p, int device, coffee_env** env);
COFFEE_API int coffee_env_destroy(coffee_env* env);
COFFEE_API int coffee_env_grid(const coffee_env* env, coffee_grid* grid);
COFFEE_API int coffee_env_params(const coffee_env* env, coffee_params* p);

/* ---- fields: sim_data (src/data/sim_data.cpp:6-26) on the device -------
 * elem_size 4 (float, the reference's default Scalar) or 8 (USE_DOUBLE). */
COFFEE_API int coffee_fields_create(coffee_env* env, int elem_size, coffee_fields** f);
COFFEE_API int coffee_fields_destroy(coffee_fields* f);
/* Device pointer of one field array (multi_array::dev_ptr). */
COFFEE_API int coffee_fields_ptr(coffee_fields* f, int id, void** dev_ptr);
/* Copy one field (id >= 0) or E,B,P (id == -1, 7 arrays back to back) from
 * host memory in the reference layout (multi_array::sync_to_device). */
COFFEE_API int coffee_fields_upload(coffee_fields* f, int id, const void* host);
/* Copy to host memory (multi_array::sync_to_host); synchronises. */
COFFEE_API int coffee_fields_download(coffee_fields* f, int id, void* host);
/* Fill E, B, P with the periodic guard images of the interior
 * (sim_environment::send_guard_cells for one rank). */
COFFEE_API int coffee_fields_fill_guards(coffee_fields* f);

/* ---- solver: field_solver_EZ (src/algorithms/field_solver_EZ.h:6-33) --- */
/* stream: a cudaStream_t (NULL = the legacy default stream).  The solver
 * owns its scratch (LSRK accumulators, the second field buffer, the
 * start-of-step copy) as the reference's solver owns dE, dB, dP, Etmp,
 * Btmp, Ptmp. */
COFFEE_API int coffee_solver_create(coffee_env* env, coffee_fields* f, int variant, int semantics,
                         void* stream, coffee_solver** s);
COFFEE_API int coffee_solver_destroy(coffee_solver* s);
/* evolve_fields(time) called nsteps times, time advancing by dt after each
 * call (src/main-alfven3d.cpp:117-119).  Asynchronous on the solver's
 * stream. */
COFFEE_API int coffee_solver_step(coffee_solver* s, double time, int nsteps);
/* Request J, divE, divB (the reference stores them on every stage) to be
 * written by the last stage of the following steps (1) or not (0, the
 * default: they cost 20 bytes per cell per stage).  The staggered solver
 * has no such outputs (COFFEE_E_INVALID). */
COFFEE_API int coffee_solver_set_aux(coffee_solver* s, int enable);
enum { /* arithmetic of the flat EZ solver (coffee_solver_set_arithmetic) */
  COFFEE_ARITH_REFERENCE = 0, /* the default.  CPU semantics: every operation of the
                               * reference CPU build's rk_step, Kreiss_Oliger and
                               * clean_epar_check_eGTb (field_solver_EZ.cpp:105-634) in
                               * its order and rounding, including the fused
                               * multiply-adds its compiler forms and its vector
                               * library's tanh, so that FP32 runs give the float
                               * build's fields bit for bit (the star and absorbing
                               * boundaries agree to rounding).  GPU semantics: as
                               * COFFEE_ARITH_FAST. */
  COFFEE_ARITH_FAST = 1       /* the same algorithm with the derivatives and the current
                               * regrouped for fewer instructions (reciprocal-based
                               * division, one exponential in the taper); agrees with
                               * COFFEE_ARITH_REFERENCE to rounding */
};
/* Select the arithmetic of a flat solver's following steps (no counterpart
 * in the reference, which has one arithmetic per build).  The other
 * variants have only COFFEE_ARITH_REFERENCE. */
COFFEE_API int coffee_solver_set_arithmetic(coffee_solver* s, int mode);
/* Keep the CPU build's per-point energy-change diagnostics (1) or not (0,
 * the default) in the following steps: the change of |E|^2 made by the E.B
 * cleaning (COFFEE_DU_EPAR) and by both clamps (COFFEE_DU_EGTB), summed over
 * the stages and the closing KO pass of a step, and the change of
 * |E|^2 + |B|^2 made by the KO pass (COFFEE_DU_KO), each zeroed at the start
 * of every step as evolve_fields does (field_solver_EZ.cpp:1019-1021), and
 * their sums over steps (COFFEE_DU_*_CUM), which keep accumulating until the
 * caller resets them (the reference's exporter does after each output,
 * data_exporter.cpp:633-638).  Computed in the CPU build's own arithmetic:
 * flat solver, CPU semantics, COFFEE_ARITH_REFERENCE only. */
COFFEE_API int coffee_solver_set_energy_diag(coffee_solver* s, int enable);
/* The SIMD width by which the CPU build's P-gradient taper offsets a point's
 * x, y and z (field_solver_EZ.cpp:222-224): 16 in its float build, 8 in its
 * double build (AVX-512), so the two builds differ in more than rounding.
 * 0 (the default) takes the width of the field precision; another value
 * (1..64) runs a precision with the other build's width, e.g. FP64 with 16
 * lanes as the exact counterpart of an FP32 run.  Flat solver only. */
COFFEE_API int coffee_solver_set_taper_lanes(coffee_solver* s, int lanes);
/* Bracket every kernel launch of the following coffee_solver_step calls with
 * CUDA events on the solver's stream (1) or not (0, the default). */
COFFEE_API int coffee_solver_set_timing(coffee_solver* s, int enable);
enum { /* kernel kinds reported by coffee_solver_last_timing */
  COFFEE_KERNEL_STAGE_FIRST = 0, /* first LSRK stage (As = 0: dU is not read);
                                  * staggered solver: update pass of substep 1 */
  COFFEE_KERNEL_STAGE = 1,       /* LSRK stages 2-5; staggered: update passes 2-3 */
  COFFEE_KERNEL_KO = 2           /* Kreiss-Oliger + clamps + boundary pass;
                                  * staggered: the clamp passes */
};
/* Device time of the last coffee_solver_step call in timing mode: summed
 * milliseconds ms[kind] and launch counts launches[kind] per kernel kind,
 * and the whole call.  Waits for the call to finish. */
COFFEE_API int coffee_solver_last_timing(coffee_solver* s, double ms[3], int launches[3],
                                         double* total_ms);
/* Number of kernel launches one coffee_solver_step(s, t, 1) issues. */
COFFEE_API int coffee_solver_launches_per_step(coffee_solver* s);
/* Problem set-up on the device (the role of the reference's user_*.hpp
 * initial conditions): at every grid point x, guards included,
 *   B = b0 + sum_m bamp[m] sin(kb[m].x + phib[m]),
 *   v = sum_n vamp[n] sin(kv[n].x + phiv[n]),  E = -v x B,  P = 0,
 * evaluated in FP64 and stored in the field precision.  kb, bamp, kv, vamp
 * hold 3 doubles per mode. */
COFFEE_API int coffee_fields_init_fourier(coffee_fields* f, const double b0[3], int nb,
                                          const double* kb, const double* bamp,
                                          const double* phib, int nv, const double* kv,
                                          const double* vamp, const double* phiv);

/* FP64 reduction of a diagnostic (Coffee::field_solver_EZ::total_energy,
 * src/algorithms/field_solver_EZ.cu:755-795, and the checks listed with
 * COFFEE_DIAG_*).  Synchronises. */
COFFEE_API int coffee_diag_reduce(coffee_solver* s, int what, double* out);
/* FP64 Poynting luminosity of the flat solver's fields through the sphere
 * |x| = r: the flux of S = E x B averaged over a shell around r,
 * sum over interior points of (S . x/|x|) w(|x| - r) dx dy dz with the tent
 * w(s) = max(0, 1 - |s|/h) / h, h the largest grid spacing.  No reference
 * counterpart (the reference reports total_energy only); the spindown
 * luminosity of a rotator.  Synchronises. */
COFFEE_API int coffee_diag_luminosity(coffee_solver* s, double r, double* out);
/* Check every field for NaN/Inf: COFFEE_OK or COFFEE_E_NONFINITE. */
COFFEE_API int coffee_solver_check_finite(coffee_solver* s);

/* ---- snapshots (replacing the reference's HDF5 save/load_snapshot,
 * src/utils/data_exporter.cpp:134-259): E, B, P plus the LSRK accumulators,
 * time and step, CRC-checked, in the format of include/coffee_fld.h. */
COFFEE_API int coffee_solver_save_snapshot(coffee_solver* s, const char* path, double time,
                                int64_t step);
COFFEE_API int coffee_solver_load_snapshot(coffee_solver* s, const char* path, double* time,
                                int64_t* step);

/* ---- batches of log-spherical runs -------------------------------------
 * No counterpart in the reference (which runs one grid per process).  Many
 * independent log-spherical runs (COFFEE_VARIANT_LOGSPH solvers on the same
 * device, each with its own grid, parameters and fields) advanced together:
 * one kernel launch per phase covers every run, so small grids do not pay a
 * launch each.  Results are those of coffee_solver_step on each solver.  At
 * most 128 runs, all of one precision; the solvers must outlive the batch.
 * coffee_batch_create autotunes the batch: it times the first-stage kernel
 * (which writes only the solvers' scratch) for four 256-thread tile shapes
 * and two run orders and keeps the fastest.  coffee_batch_step advances
 * every run by nsteps evolve_fields calls from times[m] and writes the new
 * times back (advanced in field precision); one step of the batch is a
 * captured CUDA graph, made on the first call and replayed for every step. */
typedef struct coffee_batch coffee_batch;
COFFEE_API int coffee_batch_create(coffee_solver* const* solvers, int n, void* stream,
                                   coffee_batch** out);
COFFEE_API int coffee_batch_step(coffee_batch* b, double* times, int nsteps);
/* The autotuner's choice: tile shape, run order (0 as given, 1 largest
 * first) and the first stage's time with it in ms. */
COFFEE_API int coffee_batch_info(coffee_batch* b, int* tile_x, int* tile_y, int* order,
                                 double* tuned_ms);
COFFEE_API int coffee_batch_destroy(coffee_batch* b);
/* The persistent mode (on != 0): every coffee_batch_step call runs all of
 * its steps in one cooperative launch (all CTAs resident) that separates the
 * phases by grid-wide barriers instead of launch boundaries; results are
 * bitwise those of the default mode.  Each barrier wait is bounded (2 s by
 * default): a wait that runs out ends the launch, and coffee_batch_step
 * returns COFFEE_E_TIMEOUT with the barrier and CTA in the error string; the
 * fields are then partly advanced.  In this mode coffee_batch_step
 * synchronises its stream before it returns (it reads the barrier status). */
COFFEE_API int coffee_batch_set_persistent(coffee_batch* b, int on);
/* Limit of one barrier wait of the persistent mode, in ns (> 0).
 * stall_block >= 0 is a test hook: that CTA leaves out its arrival at the
 * first barrier, so the other CTAs' waits run out; -1 turns it off. */
COFFEE_API int coffee_batch_set_wait_limit(coffee_batch* b, long long limit_ns, int stall_block);

/* ---- one step loop that allocates nothing ------------------------------
 * No counterpart in the reference.  For callers that must not allocate
 * device memory: hosts whose device memory is all handed out by their own
 * allocator or pool, and hosts that cannot afford the device-wide
 * synchronisation that cudaMalloc/cudaFree can cause in the middle of their
 * own pipeline.  It runs the same kernels as coffee_solver_step on the 7 FP32
 * field arrays the caller owns (Ex Ey Ez Bx By Bz P on the current device,
 * the reference layout, dims = N + 2*guard), in place, nsteps evolve_fields
 * calls from `time`, on `stream`.  Its scratch -- the second field buffer,
 * the LSRK accumulators and the start-of-step copy -- lives in one static
 * 32 MiB device array that every GPU loading the library holds until the
 * process exits, so grids are limited to 399,457 points per array (e.g. a
 * 64^3 interior with 3 guards, 70^3 = 343,000 points); larger grids are
 * rejected with COFFEE_E_INVALID.  It calls no cudaMalloc or cudaFree.  The
 * first call on a device looks up the array's device address for that
 * device and keeps it for the life of the process: it belongs to the
 * device's primary context, so it is stale after cudaDeviceReset (do not
 * call this after resetting the device).  The first call also loads the
 * kernels' code, which may allocate and synchronise inside the driver:
 * make it once outside the caller's critical pipeline, and before any
 * stream capture.  All calls share the one array, which keeps the last
 * call's contents: calls that overlap on the GPU (other streams, other host
 * threads) race.  J, divE and divB are not produced. */
COFFEE_API int coffee_evolve_noalloc(const coffee_params* p, int semantics,
                                     float* const fields[7], double time, int nsteps,
                                     void* stream);

#ifdef __cplusplus
}
#endif
#endif /* COFFEE_B200_H */
