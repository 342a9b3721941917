/* ffe_oracle.h -- CPU restatement of the reference's flat EZ solver step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg; the library never
 * links or calls it.
 *
 * It restates, in plain C and in scalar loops, one call of
 * Coffee::field_solver_EZ::evolve_fields (reference
 * src/algorithms/field_solver_EZ.cpp:1007-1073 for the CPU build,
 * src/algorithms/field_solver_EZ.cu:656-707 for the GPU build) including the
 * single-rank periodic guard fill of sim_environment::send_guard_cells
 * (src/sim_env_impl.hpp:179-228).  Both builds of the reference are
 * restated, selected by `semantics`, because they compute different things
 * (the P-gradient taper, KO on P, the clamp flags, the absorbing-layer target
 * and scale, the pulsar blend radius).
 *
 * Parity pin: tests/test_oracle.py checks this restatement against the
 * output of the reference's own CPU build (oracle/_ref, built by
 * oracle/Makefile from the reference sources) through the fixtures in
 * tests/golden/.  The GPU-build semantics have no CPU reference to pin
 * against; for them this restatement is the checker only.
 */
#ifndef COFFEE_FFE_ORACLE_H
#define COFFEE_FFE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_SEM_CPU_REF = 0, ORACLE_SEM_GPU_REF = 1 };

typedef struct oracle_params {
  /* grid (sim_environment, src/sim_env_impl.hpp:52-60) */
  int N[3];
  int guard[3];
  double lower[3];
  double size[3];
  int periodic[3];
  int shift_ghost;
  /* scheme (src/sim_params.h:15-124) */
  double dt;
  int divB_clean;
  double ch2, tau, KOeps;
  int use_edotb_damping;
  double damp_gamma;
  int clean_ep, check_egb; /* consulted by the GPU-build semantics only */
  int pml[3];
  int pmllen;
  double sigpml;
  int problem;
  /* pulsar */
  double radius, omega, b0;
  double p1, p2, p3, q11, q12, q13, q22, q23, q_offset_x, q_offset_y, q_offset_z;
  /* Alfven perturbation (problem 2, CPU build only) */
  double tp_start, tp_end, rpert1, rpert2, dw0, nT, ph1, ph2, dph, theta0, drpert;
  double tp_start1, tp_end1, rpert11, rpert21, dw1, nT1, ph11, ph21, dph1;
  int pert_type;
  /* which reference build to restate */
  int semantics;
  /* CPU build only: SIMD width of the reference's vector loop (16 float /
   * 8 double with AVX-512).  The P-gradient taper offsets y and z by
   * lane*delta (field_solver_EZ.cpp:222-224). */
  int taper_lanes;
} oracle_params;

/* Advance E, B, P by `nsteps` full steps starting at `time0`.  `fields` holds
 * 7 arrays (Ex Ey Ez Bx By Bz P) of dims = N + 2*guard each, guards
 * included.  Optional `aux` (may be NULL) receives J (3 arrays), divE, divB
 * of the last stage.  Optional `diag` (may be NULL; CPU-build semantics
 * only) holds the 6 energy-change arrays dU_EgtB, dU_Epar, dU_KO,
 * dU_EgtB_cum, dU_Epar_cum, dU_KO_cum (sim_data.h:15-16): the first three are
 * rewritten every step, the _cum ones accumulated from their values on
 * entry.  Returns 0, or a negative code on bad input / OOM. */
int oracle_evolve_f32(const oracle_params* p, float* const* fields, float* const* aux,
                      float* const* diag, int nsteps, double time0);
int oracle_evolve_f64(const oracle_params* p, double* const* fields, double* const* aux,
                      double* const* diag, int nsteps, double time0);

#ifdef __cplusplus
}
#endif
#endif
