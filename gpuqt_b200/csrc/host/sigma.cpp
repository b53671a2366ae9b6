// The LSQT algorithms of src/sigma.cu over the C ABI: the moment loop, Jackson
// damping and Chebyshev summation, Bessel time evolution, and the DOS / VAC0 / VAC /
// MSD / spin drivers with the reference's .out formats (one row per call, default
// ostream formatting, appended).
#include "lsqt/sigma.h"

#include <fstream>
#include <iostream>
#include <vector>

#include "gpuqt.h"
#include "lsqt/hamiltonian.h"
#include "lsqt/model.h"
#include "lsqt/vector.h"

using gqt_host::check;

void find_moments_chebyshev(Model& model, Hamiltonian& H, Vector& state_left,
                            Vector& state_right, Vector& output)
{
  // One fused step+moment kernel per moment, replayed as a CUDA graph, in the form
  // Vector::moment_precision; the moments land in `output` (FP64, number_of_moments
  // entries) on the device.
  check(gqt_moments_device_form(H.handle(), state_left.handle(), state_right.handle(),
                                model.number_of_moments, Vector::moment_precision,
                                gqt_vec_data(output.handle())),
        "find_moments_chebyshev");
}

void apply_damping(Model& model, real* re, real* im)
{
  const double PI = 3.141592653589793;
  const int M = model.number_of_moments;
  for (int k = 0; k < M; ++k) {
    const real factor = 1.0 / (M + 1);
    const real damping =
      (1 - k * factor) * cos(k * PI * factor) + sin(k * PI * factor) * factor / tan(PI * factor);
    re[k] *= damping;
    im[k] *= damping;
  }
}

void perform_chebyshev_summation(Model& model, real* re, real* im, real* out)
{
  // src/sigma.cu:89-110: the damped moments summed at each scaled energy.
  const double PI = 3.141592653589793;
  const int M = model.number_of_moments;
  if (M < 2)
    gqt_host::die("Error: the Chebyshev summation needs at least 2 moments");
  (void)im;
  for (int e = 0; e < model.number_of_energy_points; ++e) {
    const real es = model.energy[e] / model.energy_max;
    real c0 = 1.0, c1 = es, c2;
    real temp = re[1] * c1;
    for (int s = 2; s < M; ++s) {
      c2 = 2.0 * es * c1 - c0;
      c0 = c1;
      c1 = c2;
      temp += re[s] * c2;
    }
    temp *= 2.0;
    temp += re[0];
    temp *= 2.0 / (PI * model.volume);
    temp /= sqrt(1.0 - es * es);
    out[e] = temp / model.energy_max;
  }
}

void evolve(Model&, int direction, real time_step_scaled, Hamiltonian& H, Vector& state_in)
{
  check(gqt_evolve(H.handle(), direction, time_step_scaled, state_in.handle()), "evolve");
}

void evolvex(Model&, int direction, real time_step_scaled, Hamiltonian& H, Vector& state_in)
{
  check(gqt_evolvex(H.handle(), direction, time_step_scaled, state_in.handle()), "evolvex");
}

namespace {

// Moments -> damped Chebyshev sum -> one appended row of `file`.
void write_row(Model& model, Vector& moments, const std::string& file, std::ofstream& out)
{
  const int M = model.number_of_moments;
  std::vector<real> re(M), im(M), row(model.number_of_energy_points);
  moments.copy_to_host(re.data(), im.data());
  apply_damping(model, re.data(), im.data());
  perform_chebyshev_summation(model, re.data(), im.data(), row.data());
  for (int n = 0; n < model.number_of_energy_points; ++n)
    out << row[n] << " ";
  out << std::endl;
  if (!out)
    gqt_host::die("Error: cannot write " + file);
}

std::ofstream open_out(Model& model, const char* name)
{
  const std::string file = model.input_dir + name;
  std::ofstream out(file, std::ios::app);
  if (!out.is_open())
    gqt_host::die("Error: cannot open " + file);
  return out;
}

}  // namespace

// src/sigma.cu:204-239.
void find_dos(Model& model, Hamiltonian& H, Vector& random_state, int flag)
{
  Vector moments(model.number_of_moments, GQT_FP64);
  find_moments_chebyshev(model, H, random_state, random_state, moments);
  const char* name = flag == 0 ? "/dos.out" : "/ldos.out";
  std::ofstream out = open_out(model, name);
  write_row(model, moments, model.input_dir + name, out);
}

// src/sigma.cu:243-274.
void find_vac0(Model& model, Hamiltonian& H, Vector& random_state)
{
  Vector moments(model.number_of_moments, GQT_FP64);
  Vector state(model.number_of_atoms);
  H.apply_current(random_state, state);
  find_moments_chebyshev(model, H, state, state, moments);
  std::ofstream out = open_out(model, "/vac0.out");
  write_row(model, moments, model.input_dir + "/vac0.out", out);
}

// src/sigma.cu:278-327.
void find_vac(Model& model, Hamiltonian& H, Vector& random_state)
{
  Vector state_left(random_state);
  Vector state_left_copy(model.number_of_atoms);
  Vector state_right(random_state);
  Vector moments(model.number_of_moments, GQT_FP64);
  H.apply_current(state_left, state_right);
  std::ofstream out = open_out(model, "/vac.out");
  for (int m = 0; m < model.number_of_steps_correlation; ++m) {
    if (model.verbose)
      std::cout << "- calculating VAC step " << m << std::endl;
    H.apply_current(state_left, state_left_copy);
    find_moments_chebyshev(model, H, state_right, state_left_copy, moments);
    write_row(model, moments, model.input_dir + "/vac.out", out);
    if (m < model.number_of_steps_correlation - 1) {
      const real dt = model.time_step[m] * model.energy_max;
      evolve(model, -1, dt, H, state_left);
      evolve(model, -1, dt, H, state_right);
    }
  }
}

// src/sigma.cu:331-391 (note the time step index m + 1 inside the loop).
void find_msd(Model& model, Hamiltonian& H, Vector& random_state)
{
  Vector state(random_state);
  Vector state_x(random_state);
  Vector state_copy(model.number_of_atoms);
  Vector moments(model.number_of_moments, GQT_FP64);
  real dt = model.time_step[0] * model.energy_max;
  evolve(model, 1, dt, H, state);
  evolvex(model, 1, dt, H, state_x);
  std::ofstream out = open_out(model, "/msd.out");
  for (int m = 0; m < model.number_of_steps_correlation; ++m) {
    if (model.verbose)
      std::cout << "- calculating MSD step " << m << std::endl;
    find_moments_chebyshev(model, H, state_x, state_x, moments);
    write_row(model, moments, model.input_dir + "/msd.out", out);
    if (m < model.number_of_steps_correlation - 1) {
      dt = model.time_step[m + 1] * model.energy_max;
      state_copy.copy(state);
      evolvex(model, 1, dt, H, state_copy);
      evolve(model, 1, dt, H, state_x);
      state_x.add(state_copy);
      evolve(model, 1, dt, H, state);
    }
  }
}

// src/sigma.cu:395-442.
void find_spin_polarization(Model& model, Hamiltonian& H, Vector& random_state)
{
  Vector state(random_state);
  Vector state_sz(model.number_of_atoms);
  Vector moments(model.number_of_moments, GQT_FP64);
  std::ofstream out = open_out(model, "/S.out");
  for (int m = 0; m < model.number_of_steps_correlation; ++m) {
    if (model.verbose)
      std::cout << "- calculating spin step " << m << std::endl;
    state_sz.apply_sz(state);
    find_moments_chebyshev(model, H, state, state_sz, moments);
    write_row(model, moments, model.input_dir + "/S.out", out);
    if (m < model.number_of_steps_correlation - 1) {
      const real dt = model.time_step[m] * model.energy_max;
      evolve(model, 1, dt, H, state);
    }
  }
}
