// A COFFEE-style driver (shape of the reference's src/main-alfven3d.cpp with
// the initial condition of src/user_alfven.hpp replaced by the 3D Alfven
// packet of the benchmark) written against include/coffee_b200.hpp.
//
//   alfven_driver            reads ./config.toml, runs max_steps steps,
//                            writes in.fld (initial E, B, P) and out.fld
#include <cmath>
#include <cstdio>
#include <vector>

#include "coffee_b200.hpp"
#include "coffee_fld.h"

using namespace Coffee;

static void dump(const char* path, sim_data& data, const Grid& g, double time, long step) {
  data.sync_to_host();
  const void* arrays[7] = {data.E.host_ptr(0), data.E.host_ptr(1), data.E.host_ptr(2),
                           data.B.host_ptr(0), data.B.host_ptr(1), data.B.host_ptr(2),
                           data.P.host_ptr()};
  fld_header h;
  fld_header_init(&h, (int)sizeof(Scalar), 7, g.dims, g.guard);
  h.time = time;
  h.step = step;
  if (!fld_write(path, &h, arrays, g.size())) throw std::runtime_error("cannot write output");
}

int main(int argc, char* argv[]) {
  sim_environment env(&argc, &argv);
  sim_data data(env);

  Stagger st[3] = {Stagger(0b111), Stagger(0b111), Stagger(0b111)};
  data.E.set_stagger(st);
  data.B.set_stagger(st);
  const Scalar vz = 0.1, amp = 0.1;
  auto by = [&](Scalar x, Scalar y, Scalar z) {
    return amp * std::sin(2 * M_PI * x) *
           std::exp(-((y - 0.5) * (y - 0.5) + (z - 0.5) * (z - 0.5)) / 0.02);
  };
  data.B.initialize(0, [](Scalar, Scalar, Scalar) { return (Scalar)1; });
  data.B.initialize(1, [&](Scalar x, Scalar y, Scalar z) { return (Scalar)by(x, y, z); });
  data.B.initialize(2, [](Scalar, Scalar, Scalar) { return (Scalar)0; });
  data.E.initialize(0, [&](Scalar x, Scalar y, Scalar z) { return (Scalar)(vz * by(x, y, z)); });
  data.E.initialize(1, [&](Scalar, Scalar, Scalar) { return (Scalar)(-vz); });
  data.E.initialize(2, [](Scalar, Scalar, Scalar) { return (Scalar)0; });
  data.P.assign(0);
  data.P.sync_to_device();

  field_solver_EZ solver(data, env);
  dump("in.fld", data, env.grid(), 0.0, 0);

  Scalar time = 0;
  const long steps = (long)env.params().max_steps;
  for (long step = 0; step < steps; ++step) {
    solver.evolve_fields(time);
    time += env.params().dt;
  }
  Scalar wb = solver.total_energy(data.B);
  dump("out.fld", data, env.grid(), time, steps);
  std::printf("steps %ld time %.6f energy_B %.9e\n", steps, (double)time, (double)wb);
  return 0;
}
