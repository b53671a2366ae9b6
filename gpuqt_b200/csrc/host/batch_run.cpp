// lsqt() over groups of random vectors (para.in `batch_vectors B`; the reference runs
// one vector at a time, src/lsqt.cu:65-116). A group of V vectors is one multi-vector
// state, so every Chebyshev step, evolution term and operator application of the
// group is one launch that reads the operator once for V vectors. The stages are those
// of src/sigma.cu (DOS, VAC0, VAC, MSD, spin) on V vectors at a time; each .out file
// receives the group's rows vector by vector, which is the order of the one-vector
// run, and the phases are drawn from the model's generator in the same order.
#include <fstream>
#include <iostream>
#include <vector>

#include "gpuqt.h"
#include "lsqt/hamiltonian.h"
#include "lsqt/model.h"
#include "lsqt/vector.h"
#include "stages.h"

namespace gqt_host {

namespace {

// Owner of a multi-vector state handle.
struct State {
  gqt_vec* v = nullptr;
  State(int n, int nvec) { check(gqt_vec_create(n, nvec, Vector::default_precision, &v), "batch state"); }
  explicit State(const State& o) { check(gqt_vec_clone(o.v, &v), "batch state"); }
  State& operator=(const State&) = delete;
  ~State() { gqt_vec_destroy(v); }
};

struct Group {
  Model& model;
  Hamiltonian& H;
  int V;
  int N;
  Vector mu;  // device moments, [m][vector] (M * V double2)

  Group(Model& m, Hamiltonian& h, int nvec)
      : model(m), H(h), V(nvec), N(m.number_of_atoms), mu(m.number_of_moments * nvec, GQT_FP64)
  {
  }

  // mu_m of every vector of the group; rows[v] gets one row of each.
  void moments(State& left, State& right, std::vector<std::vector<std::vector<real>>>& rows,
               std::vector<std::vector<std::vector<real>>>& rows_im)
  {
    const int M = model.number_of_moments;
    void* d = gqt_vec_data(mu.handle());
    if (model.kpm_doubling && left.v == right.v)
      check(gqt_moments_doubled_device(H.handle(), right.v, M, Vector::moment_precision, d),
            "find_moments_chebyshev");
    else
      check(gqt_moments_device_form(H.handle(), left.v, right.v, M, Vector::moment_precision, d),
            "find_moments_chebyshev");
    std::vector<real> re((size_t)M * V), im((size_t)M * V);
    mu.copy_to_host(re.data(), im.data());
    for (int v = 0; v < V; ++v) {
      std::vector<real> r(M), i(M);
      for (int m = 0; m < M; ++m) {
        r[m] = re[(size_t)m * V + v];
        i[m] = im[(size_t)m * V + v];
      }
      rows[v].push_back(std::move(r));
      rows_im[v].push_back(std::move(i));
    }
  }

  void write(const char* stem, std::vector<std::vector<std::vector<real>>>& re,
             std::vector<std::vector<std::vector<real>>>& im)
  {
    std::ofstream out = open_out(model, stem);
    for (int v = 0; v < V; ++v)
      for (size_t k = 0; k < re[v].size(); ++k)
        append_row(model, re[v][k].data(), im[v][k].data(), stem, out);
  }

  using Rows = std::vector<std::vector<std::vector<real>>>;

  void run(State& phi)
  {
    const int steps = model.number_of_steps_correlation;
    {  // DOS (src/sigma.cu:204-239)
      Rows re(V), im(V);
      moments(phi, phi, re, im);
      write("dos", re, im);
    }
    if (model.calculate_vac0) {  // src/sigma.cu:243-274
      Rows re(V), im(V);
      State s(N, V);
      check(gqt_apply_current(H.handle(), phi.v, s.v), "apply_current");
      moments(s, s, re, im);
      write("vac0", re, im);
    }
    if (model.calculate_vac) {  // src/sigma.cu:278-327
      Rows re(V), im(V);
      State left(phi), right(phi), left_copy(N, V);
      check(gqt_apply_current(H.handle(), left.v, right.v), "apply_current");
      for (int m = 0; m < steps; ++m) {
        check(gqt_apply_current(H.handle(), left.v, left_copy.v), "apply_current");
        moments(right, left_copy, re, im);
        if (m < steps - 1) {
          const real dt = model.time_step[m] * model.energy_max;
          check(gqt_evolve(H.handle(), -1, dt, left.v), "evolve");
          check(gqt_evolve(H.handle(), -1, dt, right.v), "evolve");
        }
      }
      write("vac", re, im);
    }
    if (model.calculate_msd) {  // src/sigma.cu:331-391
      Rows re(V), im(V);
      State state(phi), state_x(phi), copy(N, V);
      real dt = model.time_step[0] * model.energy_max;
      check(gqt_evolve(H.handle(), 1, dt, state.v), "evolve");
      check(gqt_evolvex(H.handle(), 1, dt, state_x.v), "evolvex");
      for (int m = 0; m < steps; ++m) {
        moments(state_x, state_x, re, im);
        if (m < steps - 1) {
          dt = model.time_step[m + 1] * model.energy_max;
          check(gqt_vec_copy(copy.v, state.v), "copy");
          check(gqt_evolvex(H.handle(), 1, dt, copy.v), "evolvex");
          check(gqt_evolve(H.handle(), 1, dt, state_x.v), "evolve");
          check(gqt_vec_add(state_x.v, copy.v), "add");
          check(gqt_evolve(H.handle(), 1, dt, state.v), "evolve");
        }
      }
      write("msd", re, im);
    }
    if (model.calculate_spin) {  // src/sigma.cu:395-442
      Rows re(V), im(V);
      State state(phi), sz(N, V);
      for (int m = 0; m < steps; ++m) {
        check(gqt_vec_apply_sz(sz.v, state.v), "apply_sz");
        moments(state, sz, re, im);
        if (m < steps - 1) {
          const real dt = model.time_step[m] * model.energy_max;
          check(gqt_evolve(H.handle(), 1, dt, state.v), "evolve");
        }
      }
      write("S", re, im);
    }
  }
};

// Vectors per launch the library offers for the FP64 states (and the FP32 form).
int group_size(int want, int left)
{
  const int cap = want < left ? want : left;
  for (int v : {16, 4})
    if (v <= cap)
      return v;
  return 1;
}

}  // namespace

void run_vector_groups(Model& model, Hamiltonian& H, int first, int count, int batch)
{
  const int N = model.number_of_atoms;
  int done = 0;
  while (done < count) {
    const int V = group_size(batch, count - done);
    if (model.verbose)
      std::cout << "\nStarted  simulation with random vectors " << first + done << " to "
                << first + done + V - 1 << std::endl;
    std::vector<real> re((size_t)V * N), im((size_t)V * N);
    for (int v = 0; v < V; ++v)
      model.initialize_state_host(re.data() + (size_t)v * N, im.data() + (size_t)v * N, -1);
    State phi(N, V);
    check(gqt_vec_upload(phi.v, re.data(), im.data()), "Vector::copy_from_host");
    Group g(model, H, V);
    g.run(phi);
    done += V;
  }
}

}  // namespace gqt_host
