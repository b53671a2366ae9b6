// lsqt(): the run over one input directory (src/lsqt.cu:135-152), and the C-ABI
// model / driver entry points (gqt_model_*, gqt_lsqt).
#include "lsqt/lsqt.h"

#include <chrono>
#include <cstring>
#include <iostream>
#include <vector>

#include "gpuqt.h"
#include "lsqt/hamiltonian.h"
#include "lsqt/model.h"
#include "lsqt/sigma.h"
#include "lsqt/vector.h"

namespace {

template <class F>
void timed(bool verbose, const char* what, F&& f)
{
  const auto t0 = std::chrono::steady_clock::now();
  f();
  gqt_sync();
  const double s =
    std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (verbose)
    std::cout << "- Time used for finding " << what << " = " << s << " s" << std::endl;
}

void run(Model& model)
{
  Hamiltonian H(model);
  Vector random_state(model.number_of_atoms);
  const bool v = model.verbose;
  for (int i = 0; i < model.number_of_random_vectors; ++i) {
    if (v)
      std::cout << "\nStarted  simulation with random vector number " << i << std::endl;
    model.initialize_state(random_state, -1);
    timed(v, "DOS", [&] { find_dos(model, H, random_state, 0); });
    if (model.calculate_vac0)
      timed(v, "VAC0", [&] { find_vac0(model, H, random_state); });
    if (model.calculate_vac)
      timed(v, "VAC", [&] { find_vac(model, H, random_state); });
    if (model.calculate_msd)
      timed(v, "MSD", [&] { find_msd(model, H, random_state); });
    if (model.calculate_spin)
      timed(v, "spin polarization", [&] { find_spin_polarization(model, H, random_state); });
    if (v)
      std::cout << "Finished simulation with random vector number " << i << std::endl;
  }
  if (model.calculate_ldos) {
    timed(v, "LDOS", [&] {
      for (int i = 0; i < model.number_of_local_orbitals; ++i) {
        model.initialize_state(random_state, model.local_orbitals[i]);
        find_dos(model, H, random_state, 1);
      }
    });
  }
}

}  // namespace

void lsqt(std::string input_directory)
{
  Model model(input_directory);
  run(model);
}

// ------------------------------------------------------------------ C ABI
struct gqt_model {
  Model* m = nullptr;
};

extern "C" gqt_status gqt_model_load(const char* dir, int verbose, gqt_model** out)
{
  if (!dir || !out)
    return GQT_ERR_ARG;
  *out = nullptr;
  try {
    auto* gm = new gqt_model;
    gm->m = new Model(dir, Model::Quiet{});
    gm->m->verbose = verbose != 0;
    *out = gm;
    return GQT_OK;
  } catch (const std::exception& e) {
    gqt_host::set_error(e.what());
    return GQT_ERR_INPUT;
  }
}

extern "C" gqt_status gqt_model_destroy(gqt_model* gm)
{
  if (gm) {
    delete gm->m;
    delete gm;
  }
  return GQT_OK;
}

extern "C" gqt_status gqt_model_ell(const gqt_model* gm, gqt_ell_desc* d)
{
  if (!gm || !d)
    return GQT_ERR_ARG;
  const Model& m = *gm->m;
  d->n = m.number_of_atoms;
  d->max_neighbor = m.max_neighbor;
  d->energy_max = m.energy_max;
  d->neighbor_number = m.neighbor_number;
  d->neighbor_list = m.neighbor_list;
  d->potential = m.potential;
  d->hopping_real = m.hopping_real;
  d->hopping_imag = m.hopping_imag;
  d->xx = m.xx;
  return GQT_OK;
}

extern "C" gqt_status gqt_model_params(const gqt_model* gm, int* n_moments, int* n_energy,
                                       int* n_steps, int* n_random_vectors, double* volume)
{
  if (!gm)
    return GQT_ERR_ARG;
  const Model& m = *gm->m;
  if (n_moments)
    *n_moments = m.number_of_moments;
  if (n_energy)
    *n_energy = m.number_of_energy_points;
  if (n_steps)
    *n_steps = m.number_of_steps_correlation;
  if (n_random_vectors)
    *n_random_vectors = m.number_of_random_vectors;
  if (volume)
    *volume = m.volume;
  return GQT_OK;
}

extern "C" gqt_status gqt_model_energy(const gqt_model* gm, double* energy)
{
  if (!gm || !energy)
    return GQT_ERR_ARG;
  std::memcpy(energy, gm->m->energy, sizeof(double) * gm->m->number_of_energy_points);
  return GQT_OK;
}

extern "C" gqt_status gqt_model_time_step(const gqt_model* gm, double* time_step)
{
  if (!gm || !time_step)
    return GQT_ERR_ARG;
  if (gm->m->number_of_steps_correlation > 0 && gm->m->time_step)
    std::memcpy(time_step, gm->m->time_step, sizeof(double) * gm->m->number_of_steps_correlation);
  return GQT_OK;
}

extern "C" gqt_status gqt_model_initial_state(gqt_model* gm, int orbital, double* re,
                                              double* im)
{
  if (!gm || !re || !im)
    return GQT_ERR_ARG;
  if (orbital >= gm->m->number_of_atoms)
    return GQT_ERR_ARG;
  gm->m->initialize_state_host(re, im, orbital);
  return GQT_OK;
}

extern "C" gqt_status gqt_lsqt(const char* dir, int precision, int verbose)
{
  if (!dir)
    return GQT_ERR_ARG;
  if (precision != GQT_FP64 && precision != GQT_FP32)
    return GQT_ERR_ARG;
  const int saved = Vector::moment_precision;
  gqt_host::ThrowScope scope;
  Vector::moment_precision = precision;
  gqt_status st = GQT_OK;
  try {
    Model model(dir, Model::Quiet{});
    model.verbose = verbose != 0;
    run(model);
  } catch (const gqt_host::InputError& e) {
    gqt_host::set_error(e.what());
    st = GQT_ERR_INPUT;
  } catch (const gqt_host::RunError& e) {
    gqt_host::set_error(e.what());
    st = e.code;
  }
  Vector::moment_precision = saved;
  return st;
}
