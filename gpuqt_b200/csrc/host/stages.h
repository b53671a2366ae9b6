// The find_* drivers of src/sigma.cu as resumable stages: a stage can start at a
// correlation step from saved states, and reports after every .out row where it
// would continue from. find_dos / find_vac0 / find_vac / find_msd /
// find_spin_polarization run their stage from the start with no report, as the
// reference does.
#pragma once

#include <fstream>
#include <functional>
#include <vector>

#include "lsqt/common.h"

class Model;
class Hamiltonian;
class Vector;

namespace gqt_host {

struct StageRun {
  int start = 0;  // first correlation step; > 0 needs `restore`
  // The states the stage continues from at `start`: re then im, number_of_atoms each
  // (VAC: left, right; MSD: state, state_x; spin: state).
  const std::vector<std::vector<real>>* restore = nullptr;
  // After each row: the step the stage would continue from and the states it would
  // continue with (none once the stage is complete).
  std::function<void(int next, const std::vector<Vector*>& live)> after_row;
};

// <stem>.out opened for appending (dies if it cannot be opened).
std::ofstream open_out(Model& model, const char* stem);
// One row from host moments: with output_moments the raw moments go to
// <stem>_moments.bin, then Jackson damping and the Chebyshev sum at the energy grid are
// appended to `out` in the reference's format (src/sigma.cu:204-239).
void append_row(Model& model, const real* mu_re, const real* mu_im, const char* stem,
                std::ofstream& out);
// Random vectors first .. first + count - 1 as groups of up to `batch` vectors per
// launch (para.in batch_vectors): every stage of a group runs on multi-vector states,
// and each .out file receives the group's rows vector by vector, as the one-vector
// run writes them. Draws the group's phases from the model's generator in order.
void run_vector_groups(Model& model, Hamiltonian& H, int first, int count, int batch);

void dos_stage(Model& model, Hamiltonian& H, Vector& random_state, int flag, StageRun& run);
void vac0_stage(Model& model, Hamiltonian& H, Vector& random_state, StageRun& run);
void vac_stage(Model& model, Hamiltonian& H, Vector& random_state, StageRun& run);
void msd_stage(Model& model, Hamiltonian& H, Vector& random_state, StageRun& run);
void spin_stage(Model& model, Hamiltonian& H, Vector& random_state, StageRun& run);

}  // namespace gqt_host
