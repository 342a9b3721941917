// coffee_b200.hpp -- the reference's C++ objects of the field-update path,
// re-created over the C ABI of libcoffee_b200 (include/coffee_b200.h).
//
// A COFFEE driver such as src/main-alfven3d.cpp builds, in order,
//   sim_environment env(&argc, &argv);      (src/sim_env.h:17-87)
//   sim_data data(env);                     (src/data/sim_data.h:11-24)
//   data.E.initialize(n, f); ...            (src/data/fields.h:11-132)
//   field_solver_EZ solver(data, env);      (src/algorithms/field_solver_EZ.h:6-33)
//   solver.evolve_fields(time);             once per step
// The classes below keep those names, constructors and member functions, so
// such a driver compiles against this header instead of the reference's
// src/ tree and links with -lcoffee_b200.  Fields live on the GPU; host
// copies exist for initialisation and output (sync_to_host/sync_to_device),
// exactly as in the reference's GPU build.  Every C-ABI failure becomes a
// std::runtime_error carrying coffee_last_error_string(); the reference
// instead prints and exits (src/cuda/cuda_utility.h:20-58).
//
// Scalar is float, or double with USE_DOUBLE (src/data/typedefs.h:6-12).
#ifndef COFFEE_B200_HPP
#define COFFEE_B200_HPP

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "coffee_b200.h"

namespace Coffee {

#ifndef USE_DOUBLE
typedef float Scalar;
#else
typedef double Scalar;
#endif

inline void coffee_check(int rc, const char* what) {
  if (rc != COFFEE_OK)
    throw std::runtime_error(std::string(what) + ": " + coffee_last_error_string());
}

// ---------------------------------------------------------------- sim_params
// Same members and defaults as src/sim_params.h:15-124 (it is coffee_params).
struct sim_params : coffee_params {
  sim_params() { coffee_params_default(this); }
};

// parse_config (src/sim_params.cpp:7-146): read a TOML file.
inline sim_params parse_config(const std::string& filename) {
  std::ifstream in(filename);
  if (!in) throw std::runtime_error("cannot open config file " + filename);
  std::stringstream ss;
  ss << in.rdbuf();
  sim_params p;
  coffee_check(coffee_params_parse_toml(ss.str().c_str(), &p), "parse_config");
  return p;
}

// ---------------------------------------------------------------------- Grid
// src/data/grid.h:11-266 (the members a field-update driver uses).
struct Grid {
  int dims[3] = {1, 1, 1};
  int guard[3] = {0, 0, 0};
  Scalar delta[3] = {1, 1, 1};
  Scalar inv_delta[3] = {1, 1, 1};
  Scalar lower[3] = {0, 0, 0};
  Scalar sizes[3] = {0, 0, 0};
  int offset[3] = {0, 0, 0};

  int reduced_dim(int i) const { return dims[i] - 2 * guard[i]; }
  // coordinate of point n along axis i; stagger 1 is the vertex (EZ scheme)
  Scalar pos(int i, int n, int stagger) const {
    return lower[i] + delta[i] * (n - guard[i] + (Scalar)(stagger * -0.5 + 0.5));
  }
  int get_idx(int c1, int c2 = 0, int c3 = 0) const {
    return c1 + c2 * dims[0] + c3 * dims[0] * dims[1];
  }
  size_t size() const { return (size_t)dims[0] * dims[1] * dims[2]; }
};

class sim_data;

// ---------------------------------------------------------- sim_environment
// One rank on one GPU.  The (argc, argv) constructor reads ./config.toml like
// src/sim_env_impl.hpp:12-86; there is no MPI, so the guard exchange is the
// periodic fill of the one rank (send_guard_cells).
class sim_environment {
 public:
  sim_environment(int* argc, char*** argv) : sim_environment(parse_config("config.toml")) {
    (void)argc;
    (void)argv;
  }
  explicit sim_environment(const sim_params& p, int device = 0) : m_params(p) {
    coffee_check(coffee_env_create(&m_params, device, &m_env), "sim_environment");
    coffee_grid g;
    coffee_check(coffee_env_grid(m_env, &g), "sim_environment");
    for (int i = 0; i < 3; ++i) {
      m_grid.dims[i] = g.dims[i];
      m_grid.guard[i] = g.guard[i];
      m_grid.delta[i] = (Scalar)g.delta[i];
      m_grid.inv_delta[i] = (Scalar)g.inv_delta[i];
      m_grid.lower[i] = (Scalar)g.lower[i];
      m_grid.sizes[i] = (Scalar)g.sizes[i];
      m_grid.offset[i] = g.offset[i];
    }
  }
  ~sim_environment() { coffee_env_destroy(m_env); }
  sim_environment(const sim_environment&) = delete;
  sim_environment& operator=(const sim_environment&) = delete;

  inline void send_guard_cells(sim_data& data);

  const Grid& grid() const { return m_grid; }
  const sim_params& params() const { return m_params; }
  int size() const { return 1; }
  int rank() const { return 0; }
  bool is_periodic(int n) const { return m_params.periodic_boundary[n] != 0; }
  bool is_boundary(int n) const { return !is_periodic(n / 2); }
  coffee_env* handle() const { return m_env; }

 private:
  sim_params m_params;
  Grid m_grid;
  coffee_env* m_env = nullptr;
};

// ------------------------------------------------------------------- Stagger
// src/data/stagger.h:8-65: bit i set = the component sits on the vertex
// along axis i (0b111 is the collocated EZ arrangement).
struct Stagger {
  unsigned char s = 0;
  Stagger(unsigned char v = 0) : s(v) {}
  int operator[](int i) const { return (s >> i) & 1; }
};

// --------------------------------------------------------------- multi_array
// src/data/multi_array.h:14-116: a host array in the reference layout
// (i + j*width + k*width*height) mirrored by one device field of the
// library when it belongs to a sim_data.
template <typename T>
class multi_array {
 public:
  multi_array() = default;
  explicit multi_array(int width, int height = 1, int depth = 1)
      : m_w(width), m_h(height), m_d(depth), m_host((size_t)width * height * depth) {}

  T& operator()(int x, int y = 0, int z = 0) { return m_host[idx(x, y, z)]; }
  const T& operator()(int x, int y = 0, int z = 0) const { return m_host[idx(x, y, z)]; }
  T& operator[](size_t n) { return m_host[n]; }
  const T& operator[](size_t n) const { return m_host[n]; }

  void assign(const T& value) { std::fill(m_host.begin(), m_host.end(), value); }
  void copy_from(const multi_array& o) {
    if (o.size() != size()) throw std::range_error("multi_array::copy_from: size mismatch");
    m_host = o.m_host;
  }
  // Host -> device (multi_array::sync_to_device).
  void sync_to_device() {
    if (m_fields) coffee_check(coffee_fields_upload(m_fields, m_id, m_host.data()), "sync_to_device");
  }
  // Device -> host (multi_array::sync_to_host).
  void sync_to_host() {
    if (m_fields)
      coffee_check(coffee_fields_download(m_fields, m_id, m_host.data()), "sync_to_host");
  }
  T* host_ptr() { return m_host.data(); }
  const T* host_ptr() const { return m_host.data(); }
  // Device pointer of the bound field (nullptr for a host-only array).
  T* dev_ptr() {
    if (!m_fields) return nullptr;
    void* p = nullptr;
    coffee_check(coffee_fields_ptr(m_fields, m_id, &p), "dev_ptr");
    return static_cast<T*>(p);
  }
  int width() const { return m_w; }
  int height() const { return m_h; }
  int depth() const { return m_d; }
  size_t size() const { return m_host.size(); }

  void bind(coffee_fields* f, int id) {
    m_fields = f;
    m_id = id;
  }

 private:
  size_t idx(int x, int y, int z) const { return (size_t)x + ((size_t)y + (size_t)z * m_h) * m_w; }
  int m_w = 0, m_h = 1, m_d = 1;
  std::vector<T> m_host;
  coffee_fields* m_fields = nullptr;
  int m_id = -1;
};

// -------------------------------------------------------------- vector_field
// src/data/fields.h:11-132: three components, each with its stagger.
template <typename T>
class vector_field {
 public:
  vector_field() = default;
  explicit vector_field(const Grid& grid) : m_grid(&grid) {
    for (int i = 0; i < 3; ++i) m_data[i] = multi_array<T>(grid.dims[0], grid.dims[1], grid.dims[2]);
  }
  // All components to zero (vector_field::initialize()).
  void initialize() {
    for (int i = 0; i < 3; ++i) {
      m_data[i].assign(T(0));
      m_data[i].sync_to_device();
    }
  }
  // Component n from f(x, y, z) at every point, guards included, at the
  // coordinates given by the component's stagger (fields_impl.hpp:8-30).
  template <typename Func>
  void initialize(int n, const Func& f) {
    const Grid& g = *m_grid;
    for (int k = 0; k < g.dims[2]; ++k) {
      const Scalar x3 = g.pos(2, k, m_stagger[n][2]);
      for (int j = 0; j < g.dims[1]; ++j) {
        const Scalar x2 = g.pos(1, j, m_stagger[n][1]);
        for (int i = 0; i < g.dims[0]; ++i) {
          const Scalar x1 = g.pos(0, i, m_stagger[n][0]);
          m_data[n](i, j, k) = f(x1, x2, x3);
        }
      }
    }
    m_data[n].sync_to_device();
  }
  void assign(T value, int n) { m_data[n].assign(value); }
  void assign(T value) {
    for (int i = 0; i < 3; ++i) m_data[i].assign(value);
  }
  void copy_from(const vector_field& o) {
    for (int i = 0; i < 3; ++i) m_data[i].copy_from(o.m_data[i]);
  }
  void copy_stagger(const vector_field& o) {
    for (int i = 0; i < 3; ++i) m_stagger[i] = o.m_stagger[i];
  }
  void set_stagger(int n, Stagger s) { m_stagger[n] = s; }
  void set_stagger(const Stagger s[]) {
    for (int i = 0; i < 3; ++i) m_stagger[i] = s[i];
  }
  Stagger stagger(int n) const { return m_stagger[n]; }
  T& operator()(int n, int i, int j = 0, int k = 0) { return m_data[n](i, j, k); }
  const T& operator()(int n, int i, int j = 0, int k = 0) const { return m_data[n](i, j, k); }
  multi_array<T>& data(int n) { return m_data[n]; }
  const multi_array<T>& data(int n) const { return m_data[n]; }
  T* dev_ptr(int n) { return m_data[n].dev_ptr(); }
  T* host_ptr(int n) { return m_data[n].host_ptr(); }
  const T* host_ptr(int n) const { return m_data[n].host_ptr(); }
  void sync_to_host() {
    for (int i = 0; i < 3; ++i) m_data[i].sync_to_host();
  }
  void sync_to_host(int n) { m_data[n].sync_to_host(); }
  void sync_to_device() {
    for (int i = 0; i < 3; ++i) m_data[i].sync_to_device();
  }
  void sync_to_device(int n) { m_data[n].sync_to_device(); }
  const Grid& grid() const { return *m_grid; }

 private:
  const Grid* m_grid = nullptr;
  multi_array<T> m_data[3];
  Stagger m_stagger[3] = {Stagger(0b111), Stagger(0b111), Stagger(0b111)};
};

// ------------------------------------------------------------------ sim_data
// src/data/sim_data.h:11-24.  E, B, P are the evolved fields; B0 holds the
// force-free current J, as the reference's EZ solvers write it there
// (field_solver_EZ.cu:580-581); divE, divB are the last stage's divergences.
// dU_* are the CPU build's per-cell energy-change diagnostics, written when
// the solver's set_energy_diag(true) is on (their device arrays are made on
// first use; sync_to_host() leaves them out: call their own sync_to_host).
class sim_data {
 public:
  vector_field<Scalar> E, B, B0;
  multi_array<Scalar> P, divB, divE;
  multi_array<Scalar> dU_EgtB, dU_Epar, dU_KO;
  multi_array<Scalar> dU_EgtB_cum, dU_Epar_cum, dU_KO_cum;
  const sim_environment& env;

  explicit sim_data(const sim_environment& e) : E(e.grid()), B(e.grid()), B0(e.grid()), env(e) {
    const Grid& g = e.grid();
    P = multi_array<Scalar>(g.dims[0], g.dims[1], g.dims[2]);
    divB = multi_array<Scalar>(g.dims[0], g.dims[1], g.dims[2]);
    divE = multi_array<Scalar>(g.dims[0], g.dims[1], g.dims[2]);
    multi_array<Scalar>* du[6] = {&dU_EgtB, &dU_Epar, &dU_KO,
                                  &dU_EgtB_cum, &dU_Epar_cum, &dU_KO_cum};
    for (auto* a : du) *a = multi_array<Scalar>(g.dims[0], g.dims[1], g.dims[2]);
    coffee_check(coffee_fields_create(e.handle(), (int)sizeof(Scalar), &m_fields), "sim_data");
    for (int i = 0; i < 3; ++i) {
      E.data(i).bind(m_fields, COFFEE_EX + i);
      B.data(i).bind(m_fields, COFFEE_BX + i);
      B0.data(i).bind(m_fields, COFFEE_JX + i);
    }
    P.bind(m_fields, COFFEE_P);
    divE.bind(m_fields, COFFEE_DIVE);
    divB.bind(m_fields, COFFEE_DIVB);
    for (int i = 0; i < 6; ++i) du[i]->bind(m_fields, COFFEE_DU_EGTB + i);
  }
  ~sim_data() { coffee_fields_destroy(m_fields); }
  sim_data(const sim_data&) = delete;
  sim_data& operator=(const sim_data&) = delete;

  void sync_to_host() {
    E.sync_to_host();
    B.sync_to_host();
    B0.sync_to_host();
    P.sync_to_host();
    divB.sync_to_host();
    divE.sync_to_host();
  }
  void sync_to_device() {
    E.sync_to_device();
    B.sync_to_device();
    B0.sync_to_device();
    P.sync_to_device();
  }
  coffee_fields* handle() const { return m_fields; }

 private:
  coffee_fields* m_fields = nullptr;
};

inline void sim_environment::send_guard_cells(sim_data& data) {
  coffee_check(coffee_fields_fill_guards(data.handle()), "send_guard_cells");
}

// ----------------------------------------------------------- field_solver_EZ
// src/algorithms/field_solver_EZ.h:6-33.  semantics selects which reference
// build's arithmetic is reproduced: COFFEE_SEM_CPU_REF (field_solver_EZ.cpp,
// the default) or COFFEE_SEM_GPU_REF (field_solver_EZ.cu).  J, divE and divB
// are produced as in the reference unless set_aux(false).
class field_solver_EZ {
 public:
  field_solver_EZ(sim_data& mydata, sim_environment& env, int semantics = COFFEE_SEM_CPU_REF,
                  void* stream = nullptr)
      : m_data(mydata), m_env(env) {
    coffee_check(coffee_solver_create(env.handle(), mydata.handle(), COFFEE_VARIANT_FLAT,
                                      semantics, stream, &m_solver),
                 "field_solver_EZ");
    coffee_check(coffee_solver_set_aux(m_solver, 1), "field_solver_EZ");
  }
  ~field_solver_EZ() { coffee_solver_destroy(m_solver); }
  field_solver_EZ(const field_solver_EZ&) = delete;
  field_solver_EZ& operator=(const field_solver_EZ&) = delete;

  // Keep the CPU build's energy-change diagnostics in sim_data::dU_*
  // (coffee_solver_set_energy_diag).
  void set_energy_diag(bool enable) {
    coffee_check(coffee_solver_set_energy_diag(m_solver, enable ? 1 : 0), "set_energy_diag");
  }
  // One step: 5 LSRK stages + Kreiss-Oliger, clamps, boundaries, guards.
  void evolve_fields(Scalar time) {
    coffee_check(coffee_solver_step(m_solver, (double)time, 1), "evolve_fields");
  }
  // total_energy (field_solver_EZ.cu:755-795) of E or B, summed in FP64.
  Scalar total_energy(vector_field<Scalar>& f) {
    const int what = (&f == &m_data.E) ? COFFEE_DIAG_ENERGY_E : COFFEE_DIAG_ENERGY_B;
    double out = 0;
    coffee_check(coffee_diag_reduce(m_solver, what, &out), "total_energy");
    return (Scalar)out;
  }
  // FP64 Poynting luminosity through the sphere |x| = r (no reference
  // counterpart; coffee_diag_luminosity).
  double poynting_luminosity(double r) {
    double out = 0;
    coffee_check(coffee_diag_luminosity(m_solver, r, &out), "poynting_luminosity");
    return out;
  }
  void set_aux(bool enable) { coffee_check(coffee_solver_set_aux(m_solver, enable), "set_aux"); }
  coffee_solver* handle() const { return m_solver; }

 private:
  sim_data& m_data;
  sim_environment& m_env;
  coffee_solver* m_solver = nullptr;
};

// The solvers the reference has only in its GPU build share one shape:
// (sim_data&, sim_environment&) and evolve_fields(Scalar time).
class gpu_variant_solver {
 public:
  gpu_variant_solver(sim_data& mydata, sim_environment& env, int variant, const char* name,
                     void* stream) {
    coffee_check(coffee_solver_create(env.handle(), mydata.handle(), variant,
                                      COFFEE_SEM_GPU_REF, stream, &m_solver),
                 name);
  }
  ~gpu_variant_solver() { coffee_solver_destroy(m_solver); }
  gpu_variant_solver(const gpu_variant_solver&) = delete;
  gpu_variant_solver& operator=(const gpu_variant_solver&) = delete;

  void evolve_fields(Scalar time) {
    coffee_check(coffee_solver_step(m_solver, (double)time, 1), "evolve_fields");
  }
  void set_aux(bool enable) { coffee_check(coffee_solver_set_aux(m_solver, enable), "set_aux"); }
  coffee_solver* handle() const { return m_solver; }

 private:
  coffee_solver* m_solver = nullptr;
};

// field_solver_EZ_spherical (src/algorithms/field_solver_EZ_spherical.h:6-32):
// 2D, x = ln r, y = theta; N[2] = 1, guard[2] = 0, guard[1] >= 4.
class field_solver_EZ_spherical : public gpu_variant_solver {
 public:
  field_solver_EZ_spherical(sim_data& mydata, sim_environment& env, void* stream = nullptr)
      : gpu_variant_solver(mydata, env, COFFEE_VARIANT_LOGSPH, "field_solver_EZ_spherical",
                           stream) {}
};

// field_solver_EZ_cylindrical (src/algorithms/field_solver_EZ_cylindrical.h:6-30):
// 2D, x = R, y = z.  Evolves sim_data's P (the reference keeps its own).
class field_solver_EZ_cylindrical : public gpu_variant_solver {
 public:
  field_solver_EZ_cylindrical(sim_data& mydata, sim_environment& env, void* stream = nullptr)
      : gpu_variant_solver(mydata, env, COFFEE_VARIANT_CYL, "field_solver_EZ_cylindrical",
                           stream) {}
};

// field_solver_gr_EZ (src/algorithms/field_solver_gr_EZ.h:6-32): Kerr-Schild
// black hole of spin params().a; sim_data's E holds D.
class field_solver_gr_EZ : public gpu_variant_solver {
 public:
  field_solver_gr_EZ(sim_data& mydata, sim_environment& env, void* stream = nullptr)
      : gpu_variant_solver(mydata, env, COFFEE_VARIANT_GR, "field_solver_gr_EZ", stream) {}
};

// field_solver (src/algorithms/field_solver.h:8-35): the staggered (Yee)
// RK3 solver.  E and B sit on the staggered positions of
// src/data/sim_data.cpp:19-25, and sim_data's B0 is the background field
// subtracted in curl B (the EZ solvers keep J there instead), so this
// constructor binds data.B0 to the library's B0 arrays.
class field_solver : public gpu_variant_solver {
 public:
  field_solver(sim_data& mydata, sim_environment& env, void* stream = nullptr)
      : gpu_variant_solver((rebind_background(mydata), mydata), env, COFFEE_VARIANT_YEE,
                           "field_solver", stream),
        m_data(mydata) {}
  // total_energy (field_solver.cu:829-866): each component interpolated to
  // the vertex, summed in FP64 over the region outside the star and the
  // absorbing layer.
  Scalar total_energy(vector_field<Scalar>& f) {
    const int what = (&f == &m_data.E) ? COFFEE_DIAG_ENERGY_E : COFFEE_DIAG_ENERGY_B;
    double out = 0;
    coffee_check(coffee_diag_reduce(handle(), what, &out), "total_energy");
    return (Scalar)out;
  }

 private:
  static void rebind_background(sim_data& d) {
    for (int i = 0; i < 3; ++i) d.B0.data(i).bind(d.handle(), COFFEE_B0X + i);
  }
  sim_data& m_data;
};

// field_solver_gr (src/algorithms/field_solver_gr.h:6-29): the staggered
// solver in Kerr-Schild coordinates; sim_data's E holds D.
class field_solver_gr : public gpu_variant_solver {
 public:
  field_solver_gr(sim_data& mydata, sim_environment& env, void* stream = nullptr)
      : gpu_variant_solver(mydata, env, COFFEE_VARIANT_GRYEE, "field_solver_gr", stream) {}
  void evolve_fields_gr() { evolve_fields((Scalar)0); }
};

}  // namespace Coffee

#endif  // COFFEE_B200_HPP
