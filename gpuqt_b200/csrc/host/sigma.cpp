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
#include "checkpoint.h"
#include "stages.h"

using gqt_host::check;

void find_moments_chebyshev(Model& model, Hamiltonian& H, Vector& state_left,
                            Vector& state_right, Vector& output)
{
  // One fused step+moment kernel per moment, replayed as a CUDA graph, in the form
  // Vector::moment_precision; the moments land in `output` (FP64, number_of_moments
  // entries) on the device.
  if (model.kpm_doubling && &state_left == &state_right) {
    // A symmetric set from half the steps (para.in kpm_doubling).
    check(gqt_moments_doubled_device(H.handle(), state_right.handle(), model.number_of_moments,
                                     Vector::moment_precision, gqt_vec_data(output.handle())),
          "find_moments_chebyshev");
    return;
  }
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

using gqt_host::open_out;

// Moments -> one appended row of <stem>.out (gqt_host::append_row).
void write_row(Model& model, Vector& moments, const char* stem, std::ofstream& out)
{
  const int M = model.number_of_moments;
  std::vector<real> re(M), im(M);
  moments.copy_to_host(re.data(), im.data());
  gqt_host::append_row(model, re.data(), im.data(), stem, out);
}

void restore(Vector& v, const std::vector<real>& s)
{
  const size_t n = (size_t)v.size();
  if (s.size() != 2 * n)
    gqt_host::die("Error: a checkpointed state does not match the model size", GQT_ERR_INPUT);
  std::vector<real> re(s.begin(), s.begin() + n), im(s.begin() + n, s.end());
  v.copy_from_host(re.data(), im.data());
}

void report(gqt_host::StageRun& run, int next, std::vector<Vector*> live)
{
  if (run.after_row)
    run.after_row(next, live);
}

}  // namespace

namespace gqt_host {

void append_row(Model& model, const real* mu_re, const real* mu_im, const char* stem,
                std::ofstream& out)
{
  const int M = model.number_of_moments;
  std::vector<real> re(mu_re, mu_re + M), im(mu_im, mu_im + M), row(model.number_of_energy_points);
  if (model.output_moments)
    append_moments(model.input_dir + "/" + stem + "_moments.bin", M, re.data(), im.data());
  apply_damping(model, re.data(), im.data());
  perform_chebyshev_summation(model, re.data(), im.data(), row.data());
  for (int n = 0; n < model.number_of_energy_points; ++n)
    out << row[n] << " ";
  out << std::endl;
  if (!out)
    die("Error: cannot write " + model.input_dir + "/" + stem + ".out");
}

std::ofstream open_out(Model& model, const char* stem)
{
  const std::string file = model.input_dir + "/" + stem + ".out";
  std::ofstream out(file, std::ios::app);
  if (!out.is_open())
    die("Error: cannot open " + file);
  return out;
}

// src/sigma.cu:204-239.
void dos_stage(Model& model, Hamiltonian& H, Vector& random_state, int flag, StageRun& run)
{
  Vector moments(model.number_of_moments, GQT_FP64);
  find_moments_chebyshev(model, H, random_state, random_state, moments);
  const char* stem = flag == 0 ? "dos" : "ldos";
  std::ofstream out = open_out(model, stem);
  write_row(model, moments, stem, out);
  report(run, 1, {});
}

// src/sigma.cu:243-274.
void vac0_stage(Model& model, Hamiltonian& H, Vector& random_state, StageRun& run)
{
  Vector moments(model.number_of_moments, GQT_FP64);
  Vector state(model.number_of_atoms);
  H.apply_current(random_state, state);
  find_moments_chebyshev(model, H, state, state, moments);
  std::ofstream out = open_out(model, "vac0");
  write_row(model, moments, "vac0", out);
  report(run, 1, {});
}

// src/sigma.cu:278-327.
void vac_stage(Model& model, Hamiltonian& H, Vector& random_state, StageRun& run)
{
  Vector state_left(random_state);
  Vector state_left_copy(model.number_of_atoms);
  Vector state_right(random_state);
  Vector moments(model.number_of_moments, GQT_FP64);
  if (run.start > 0) {
    restore(state_left, run.restore->at(0));
    restore(state_right, run.restore->at(1));
  } else {
    H.apply_current(state_left, state_right);
  }
  std::ofstream out = open_out(model, "vac");
  const int steps = model.number_of_steps_correlation;
  for (int m = run.start; m < steps; ++m) {
    if (model.verbose)
      std::cout << "- calculating VAC step " << m << std::endl;
    H.apply_current(state_left, state_left_copy);
    find_moments_chebyshev(model, H, state_right, state_left_copy, moments);
    write_row(model, moments, "vac", out);
    if (m < steps - 1) {
      const real dt = model.time_step[m] * model.energy_max;
      evolve(model, -1, dt, H, state_left);
      evolve(model, -1, dt, H, state_right);
      report(run, m + 1, {&state_left, &state_right});
    } else {
      report(run, steps, {});
    }
  }
}

// src/sigma.cu:331-391 (note the time step index m + 1 inside the loop).
void msd_stage(Model& model, Hamiltonian& H, Vector& random_state, StageRun& run)
{
  Vector state(random_state);
  Vector state_x(random_state);
  Vector state_copy(model.number_of_atoms);
  Vector moments(model.number_of_moments, GQT_FP64);
  if (run.start > 0) {
    restore(state, run.restore->at(0));
    restore(state_x, run.restore->at(1));
  } else {
    const real dt = model.time_step[0] * model.energy_max;
    evolve(model, 1, dt, H, state);
    evolvex(model, 1, dt, H, state_x);
  }
  std::ofstream out = open_out(model, "msd");
  const int steps = model.number_of_steps_correlation;
  for (int m = run.start; m < steps; ++m) {
    if (model.verbose)
      std::cout << "- calculating MSD step " << m << std::endl;
    find_moments_chebyshev(model, H, state_x, state_x, moments);
    write_row(model, moments, "msd", out);
    if (m < steps - 1) {
      const real dt = model.time_step[m + 1] * model.energy_max;
      state_copy.copy(state);
      evolvex(model, 1, dt, H, state_copy);
      evolve(model, 1, dt, H, state_x);
      state_x.add(state_copy);
      evolve(model, 1, dt, H, state);
      report(run, m + 1, {&state, &state_x});
    } else {
      report(run, steps, {});
    }
  }
}

// src/sigma.cu:395-442.
void spin_stage(Model& model, Hamiltonian& H, Vector& random_state, StageRun& run)
{
  Vector state(random_state);
  Vector state_sz(model.number_of_atoms);
  Vector moments(model.number_of_moments, GQT_FP64);
  if (run.start > 0)
    restore(state, run.restore->at(0));
  std::ofstream out = open_out(model, "S");
  const int steps = model.number_of_steps_correlation;
  for (int m = run.start; m < steps; ++m) {
    if (model.verbose)
      std::cout << "- calculating spin step " << m << std::endl;
    state_sz.apply_sz(state);
    find_moments_chebyshev(model, H, state, state_sz, moments);
    write_row(model, moments, "S", out);
    if (m < steps - 1) {
      const real dt = model.time_step[m] * model.energy_max;
      evolve(model, 1, dt, H, state);
      report(run, m + 1, {&state});
    } else {
      report(run, steps, {});
    }
  }
}

}  // namespace gqt_host

void find_dos(Model& model, Hamiltonian& H, Vector& random_state, int flag)
{
  gqt_host::StageRun run;
  gqt_host::dos_stage(model, H, random_state, flag, run);
}

void find_vac0(Model& model, Hamiltonian& H, Vector& random_state)
{
  gqt_host::StageRun run;
  gqt_host::vac0_stage(model, H, random_state, run);
}

void find_vac(Model& model, Hamiltonian& H, Vector& random_state)
{
  gqt_host::StageRun run;
  gqt_host::vac_stage(model, H, random_state, run);
}

void find_msd(Model& model, Hamiltonian& H, Vector& random_state)
{
  gqt_host::StageRun run;
  gqt_host::msd_stage(model, H, random_state, run);
}

void find_spin_polarization(Model& model, Hamiltonian& H, Vector& random_state)
{
  gqt_host::StageRun run;
  gqt_host::spin_stage(model, H, random_state, run);
}
