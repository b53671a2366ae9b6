// lsqt(): the run over one input directory (src/lsqt.cu:135-152), and the C-ABI
// model / driver entry points (gqt_model_*, gqt_lsqt).
#include "lsqt/lsqt.h"

#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <vector>

#include "gpuqt.h"
#include "lsqt/hamiltonian.h"
#include "lsqt/model.h"
#include "lsqt/sigma.h"
#include "lsqt/vector.h"
#include "checkpoint.h"
#include "stages.h"

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

// The row budget of a bounded run is spent (a checkpoint has been written).
struct StopRun {};

using gqt_host::RunPosition;

bool stage_on(const Model& m, int stage)
{
  switch (stage) {
    case gqt_host::kStageDos:
      return true;
    case gqt_host::kStageVac0:
      return m.calculate_vac0;
    case gqt_host::kStageVac:
      return m.calculate_vac;
    case gqt_host::kStageMsd:
      return m.calculate_msd;
    case gqt_host::kStageSpin:
      return m.calculate_spin;
    case gqt_host::kStageLdos:
      return m.calculate_ldos;
    default:
      return false;
  }
}

int stage_rows(const Model& m, int stage)
{
  if (stage == gqt_host::kStageDos || stage == gqt_host::kStageVac0)
    return 1;
  if (stage == gqt_host::kStageLdos)
    return m.number_of_local_orbitals;
  return m.number_of_steps_correlation;
}

// Where the run continues after the row that left `stage` of `vector` at `next`.
RunPosition next_position(const Model& m, int vector, int stage, int next)
{
  if (next < stage_rows(m, stage))
    return {vector, stage, next};
  if (stage < gqt_host::kStageLdos) {
    for (int s = stage + 1; s < gqt_host::kStageLdos; ++s)
      if (stage_on(m, s))
        return {vector, s, 0};
    if (vector + 1 < m.number_of_random_vectors)
      return {vector + 1, gqt_host::kStageDos, 0};
  }
  const int v = m.number_of_random_vectors;
  if (stage < gqt_host::kStageLdos && stage_on(m, gqt_host::kStageLdos) &&
      m.number_of_local_orbitals > 0)
    return {v, gqt_host::kStageLdos, 0};
  return {v, gqt_host::kStageEnd, 0};
}

uint64_t file_size(const std::string& path)
{
  struct stat st;
  return stat(path.c_str(), &st) == 0 ? (uint64_t)st.st_size : 0;
}

// The run over one input directory. Checkpointing is on when para.in asks for it
// (checkpoint_every) or the run is bounded (max_rows > 0): an existing checkpoint is
// then resumed, one is written every checkpoint_every rows and when the row budget is
// spent (StopRun), and it is removed when the run completes. With checkpointing off
// this is the reference's run, row for row.
void run(Model& model, long long max_rows, int precision)
{
  using namespace gqt_host;
  const bool ckpt = model.checkpoint_every > 0 || max_rows > 0;
  const std::string path = checkpoint_path(model);
  Checkpoint ck;
  RunPosition start;
  bool resumed = false;
  uint64_t fingerprint = 0;
  if (ckpt) {
    fingerprint = run_fingerprint(model, precision);  // before the Hamiltonian takes the arrays
    if (load_checkpoint(path, ck)) {
      if (ck.fingerprint != fingerprint)
        throw InputError(path + " belongs to a different run (parameters, operator or precision changed)");
      for (size_t k = 0; k < ck.files.size(); ++k) {
        const std::string f = model.input_dir + "/" + ck.files[k];
        const uint64_t have = file_size(f);
        if (have < ck.sizes[k])
          throw InputError(f + " is shorter than at the checkpoint; cannot resume");
        if (have > ck.sizes[k] && truncate(f.c_str(), (off_t)ck.sizes[k]) != 0)
          die("Error: cannot truncate " + f, GQT_ERR_IO);
      }
      model.set_rng_state(ck.rng);
      start = ck.pos;
      resumed = true;
      if (model.verbose)
        std::cout << "Resuming from " << path << " at random vector " << start.vector
                  << ", stage " << start.stage << ", step " << start.step << std::endl;
    }
  }

  if (model.batch_vectors > 1 && ckpt)
    throw InputError("batch_vectors cannot be combined with checkpoints (checkpoint_every, "
                     "a bounded run): checkpoints are per row of one vector");
  // The FP32R moment form launches 4, 16 or 32 vectors at a time: every moment set must
  // come from a group of 16 or 4 (the LDOS runs one orbital vector at a time).
  if (precision == GQT_FP32R &&
      (model.batch_vectors < 4 || model.number_of_random_vectors % 4 != 0 ||
       model.calculate_ldos))
    throw InputError("the FP32R moment form runs groups of 4 or 16 vectors: set batch_vectors "
                     "4 or 16, a number_of_random_vectors divisible by 4, and no local "
                     "orbitals (the LDOS runs one vector at a time)");
  Hamiltonian H(model);
  Vector random_state(model.number_of_atoms);
  const bool v = model.verbose;
  long long rows = 0;
  int since = 0;
  std::string rng_before;  // the generator before the current vector's phase draw
  int current = -1;        // the vector being run
  auto save = [&](const RunPosition& pos, const std::vector<Vector*>& live) {
    Checkpoint c;
    c.fingerprint = fingerprint;
    c.pos = pos;
    c.rng = pos.vector == current ? rng_before : model.rng_state();
    c.files = output_files(model);
    for (const auto& f : c.files)
      c.sizes.push_back(file_size(model.input_dir + "/" + f));
    const size_t n = (size_t)model.number_of_atoms;
    for (Vector* s : live) {
      std::vector<real> buf(2 * n);
      s->copy_to_host(buf.data(), buf.data() + n);
      c.states.push_back(std::move(buf));
    }
    save_checkpoint(path, c);
    since = 0;
  };
  auto after_row = [&](const RunPosition& pos, const std::vector<Vector*>& live) {
    ++rows;
    ++since;
    if (!ckpt)
      return;
    const bool stop = max_rows > 0 && rows >= max_rows;
    if (stop || (model.checkpoint_every > 0 && since >= model.checkpoint_every))
      save(pos, live);
    if (stop)
      throw StopRun{};
  };
  auto stage_run = [&](int vector, int stage, StageRun& sr) {
    const bool first = resumed && vector == start.vector && stage == start.stage;
    sr.start = first ? start.step : 0;
    sr.restore = first ? &ck.states : nullptr;
    sr.after_row = [&, vector, stage](int next, const std::vector<Vector*>& live) {
      after_row(next_position(model, vector, stage, next), live);
    };
  };

  const int first_vector = resumed ? start.vector : 0;
  if (model.batch_vectors > 1) {
    timed(v, "random vectors in groups", [&] {
      run_vector_groups(model, H, 0, model.number_of_random_vectors, model.batch_vectors);
    });
  }
  for (int i = model.batch_vectors > 1 ? model.number_of_random_vectors : first_vector;
       i < model.number_of_random_vectors; ++i) {
    if (v)
      std::cout << "\nStarted  simulation with random vector number " << i << std::endl;
    current = i;
    rng_before = model.rng_state();
    model.initialize_state(random_state, -1);
    const int first_stage = (resumed && i == start.vector) ? start.stage : kStageDos;
    StageRun sr;
    if (first_stage <= kStageDos) {
      stage_run(i, kStageDos, sr);
      timed(v, "DOS", [&] { dos_stage(model, H, random_state, 0, sr); });
    }
    if (model.calculate_vac0 && first_stage <= kStageVac0) {
      stage_run(i, kStageVac0, sr);
      timed(v, "VAC0", [&] { vac0_stage(model, H, random_state, sr); });
    }
    if (model.calculate_vac && first_stage <= kStageVac) {
      stage_run(i, kStageVac, sr);
      timed(v, "VAC", [&] { vac_stage(model, H, random_state, sr); });
    }
    if (model.calculate_msd && first_stage <= kStageMsd) {
      stage_run(i, kStageMsd, sr);
      timed(v, "MSD", [&] { msd_stage(model, H, random_state, sr); });
    }
    if (model.calculate_spin && first_stage <= kStageSpin) {
      stage_run(i, kStageSpin, sr);
      timed(v, "spin polarization", [&] { spin_stage(model, H, random_state, sr); });
    }
    if (v)
      std::cout << "Finished simulation with random vector number " << i << std::endl;
  }
  current = -1;
  if (model.calculate_ldos && !(resumed && start.stage == kStageEnd)) {
    const int k0 = (resumed && start.stage == kStageLdos) ? start.step : 0;
    timed(v, "LDOS", [&] {
      for (int k = k0; k < model.number_of_local_orbitals; ++k) {
        model.initialize_state(random_state, model.local_orbitals[k]);
        StageRun sr;
        sr.after_row = [&, k](int, const std::vector<Vector*>&) {
          after_row(next_position(model, model.number_of_random_vectors, kStageLdos, k + 1), {});
        };
        dos_stage(model, H, random_state, 1, sr);
      }
    });
  }
  if (ckpt)
    std::remove(path.c_str());
}

}  // namespace

void lsqt(std::string input_directory)
{
  Model model(input_directory);
  try {
    run(model, 0, Vector::moment_precision);
  } catch (const gqt_host::InputError& e) {
    gqt_host::die(std::string("Error: ") + e.what());
  }
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

extern "C" gqt_status gqt_lsqt_run(const char* dir, int precision, int verbose,
                                   long long max_rows, int* finished)
{
  if (finished)
    *finished = 0;
  if (!dir)
    return GQT_ERR_ARG;
  if (precision != GQT_FP64 && precision != GQT_FP32 && precision != GQT_FP32R)
    return GQT_ERR_ARG;
  const int saved = Vector::moment_precision;
  gqt_host::ThrowScope scope;
  Vector::moment_precision = precision;
  gqt_status st = GQT_OK;
  try {
    Model model(dir, Model::Quiet{});
    model.verbose = verbose != 0;
    run(model, max_rows, precision);
    if (finished)
      *finished = 1;
  } catch (const StopRun&) {
    // the row budget is spent; the checkpoint holds the rest of the run
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

extern "C" gqt_status gqt_lsqt(const char* dir, int precision, int verbose)
{
  return gqt_lsqt_run(dir, precision, verbose, 0, nullptr);
}
