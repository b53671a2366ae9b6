// The find_* drivers of src/sigma.cu as resumable stages: a stage can start at a
// correlation step from saved states, and reports after every .out row where it
// would continue from. find_dos / find_vac0 / find_vac / find_msd /
// find_spin_polarization run their stage from the start with no report, as the
// reference does.
#pragma once

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

void dos_stage(Model& model, Hamiltonian& H, Vector& random_state, int flag, StageRun& run);
void vac0_stage(Model& model, Hamiltonian& H, Vector& random_state, StageRun& run);
void vac_stage(Model& model, Hamiltonian& H, Vector& random_state, StageRun& run);
void msd_stage(Model& model, Hamiltonian& H, Vector& random_state, StageRun& run);
void spin_stage(Model& model, Hamiltonian& H, Vector& random_state, StageRun& run);

}  // namespace gqt_host
