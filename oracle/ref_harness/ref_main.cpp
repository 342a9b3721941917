// Driver for the reference's own CPU EZ solver (test infrastructure only).
//
// Usage:  coffee_ref_{float,double} IN.fld OUT.fld NSTEPS [--aux] [--diag] [--warmup W]
//
// The TOML config is read by the reference's parse_config through the
// single-rank sim_environment double (ref_env.cpp): $COFFEE_ORACLE_CONFIG or
// ./config.toml.  IN.fld holds E, B, P with guard cells (the layout of
// src/data/multi_array_impl.hpp:81-91: i fastest, then j, then k) in the
// precision of this build.  The driver:
//   1. builds sim_data and sets every component to the collocated EZ stagger
//      0b111 (as src/user_alfven.hpp:34-39 does before the solver exists);
//   2. loads E, B, P from IN.fld;
//   3. constructs the reference field_solver_EZ and calls evolve_fields
//      NSTEPS times, advancing time by dt as src/main-alfven3d.cpp:117-119;
//   4. writes E, B, P (and with --aux also J = the B0 arrays, divE, divB,
//      src/algorithms/field_solver_EZ.cpp:149-200; with --diag also the
//      energy-change arrays dU_EgtB, dU_Epar, dU_KO, dU_EgtB_cum,
//      dU_Epar_cum, dU_KO_cum of src/data/sim_data.h:15-16, the _cum ones
//      set to zero before the first step, as the reference's exporter leaves
//      them after an output, src/utils/data_exporter.cpp:633-638) to OUT.fld;
//   5. prints one JSON line with the wall time of step 3; with --warmup W,
//      W further evolve_fields calls run first, untimed.
// The reference prints a timer line per phase per stage to stdout; those are
// sent to /dev/null while it runs so they do not perturb the timing.
#include <fcntl.h>
#include <unistd.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "algorithms/field_solver_EZ.h"
#include "data/sim_data.h"
#include "sim_env.h"
#include "coffee_fld.h"

using namespace Coffee;

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s IN.fld OUT.fld NSTEPS [--aux] [--diag] [--warmup W]\n",
                 argv[0]);
    return 2;
  }
  const std::string in_path = argv[1], out_path = argv[2];
  const long nsteps = std::atol(argv[3]);
  bool aux = false, diag = false;
  long warmup = 0;
  for (int a = 4; a < argc; ++a) {
    const std::string opt = argv[a];
    if (opt == "--aux") aux = true;
    else if (opt == "--diag") diag = true;
    else if (opt == "--warmup" && a + 1 < argc) warmup = std::atol(argv[++a]);
    else {
      std::fprintf(stderr, "unknown option %s\n", opt.c_str());
      return 2;
    }
  }

  sim_environment env(nullptr, nullptr);
  const Grid& grid = env.grid();
  sim_data data(env);
  Stagger st[3] = {Stagger(0b111), Stagger(0b111), Stagger(0b111)};
  data.E.set_stagger(st);
  data.B.set_stagger(st);
  data.B0.set_stagger(st);
  data.B0.initialize();

  fld_header hin;
  std::vector<char> payload;
  if (!fld_read(in_path.c_str(), &hin, &payload)) {
    std::fprintf(stderr, "cannot read %s\n", in_path.c_str());
    return 3;
  }
  const size_t n = (size_t)grid.dims[0] * grid.dims[1] * grid.dims[2];
  if (hin.elem_size != (int)sizeof(Scalar) || hin.nfields < 7 ||
      hin.dims[0] != grid.dims[0] || hin.dims[1] != grid.dims[1] ||
      hin.dims[2] != grid.dims[2]) {
    std::fprintf(stderr,
                 "input mismatch: elem %d (want %d), dims %d %d %d (want %d %d %d)\n",
                 hin.elem_size, (int)sizeof(Scalar), hin.dims[0], hin.dims[1],
                 hin.dims[2], grid.dims[0], grid.dims[1], grid.dims[2]);
    return 4;
  }
  Scalar* dst[7] = {data.E.host_ptr(0), data.E.host_ptr(1), data.E.host_ptr(2),
                    data.B.host_ptr(0), data.B.host_ptr(1), data.B.host_ptr(2),
                    data.P.host_ptr()};
  for (int f = 0; f < 7; ++f)
    std::memcpy(dst[f], payload.data() + f * n * sizeof(Scalar),
                n * sizeof(Scalar));
  payload.clear();
  payload.shrink_to_fit();

  field_solver_EZ solver(data, env);
  data.dU_EgtB_cum.assign(0.0);
  data.dU_Epar_cum.assign(0.0);
  data.dU_KO_cum.assign(0.0);

  // Silence the reference's per-phase timer prints while it runs.
  std::fflush(stdout);
  const int saved_stdout = dup(1);
  const int devnull = open("/dev/null", O_WRONLY);
  dup2(devnull, 1);

  Scalar time = (Scalar)hin.time;  // Scalar, as src/main-alfven3d.cpp:61
  for (long s = 0; s < warmup; ++s) {
    solver.evolve_fields(time);
    time += env.params().dt;
  }
  const auto t0 = std::chrono::steady_clock::now();
  for (long s = 0; s < nsteps; ++s) {
    solver.evolve_fields(time);
    time += env.params().dt;
  }
  const auto t1 = std::chrono::steady_clock::now();

  std::fflush(stdout);
  dup2(saved_stdout, 1);
  close(devnull);
  close(saved_stdout);

  std::vector<const Scalar*> out = {
      data.E.host_ptr(0), data.E.host_ptr(1), data.E.host_ptr(2),
      data.B.host_ptr(0), data.B.host_ptr(1), data.B.host_ptr(2),
      data.P.host_ptr()};
  if (aux) {
    out.push_back(data.B0.host_ptr(0));
    out.push_back(data.B0.host_ptr(1));
    out.push_back(data.B0.host_ptr(2));
    out.push_back(data.divE.host_ptr());
    out.push_back(data.divB.host_ptr());
  }
  if (diag) {
    out.push_back(data.dU_EgtB.host_ptr());
    out.push_back(data.dU_Epar.host_ptr());
    out.push_back(data.dU_KO.host_ptr());
    out.push_back(data.dU_EgtB_cum.host_ptr());
    out.push_back(data.dU_Epar_cum.host_ptr());
    out.push_back(data.dU_KO_cum.host_ptr());
  }
  fld_header hout = hin;
  hout.nfields = (int)out.size();
  hout.time = time;
  hout.step = hin.step + warmup + nsteps;
  if (!fld_write(out_path.c_str(), &hout, (const void* const*)out.data(), n)) {
    std::fprintf(stderr, "cannot write %s\n", out_path.c_str());
    return 5;
  }
  const double secs = std::chrono::duration<double>(t1 - t0).count();
  const long long interior =
      (long long)(grid.dims[0] - 2 * grid.guard[0]) *
      (grid.dims[1] - 2 * grid.guard[1]) * (grid.dims[2] - 2 * grid.guard[2]);
  std::printf(
      "{\"impl\": \"reference-cpu\", \"scalar_bytes\": %d, \"steps\": %ld, "
      "\"seconds\": %.6f, \"interior_cells\": %lld, \"cell_updates_per_s\": %.6e}\n",
      (int)sizeof(Scalar), nsteps, secs, interior,
      secs > 0 ? (double)interior * nsteps / secs : 0.0);
  return 0;
}
