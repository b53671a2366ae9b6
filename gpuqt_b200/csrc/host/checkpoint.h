// Checkpoint / resume of an lsqt() run and the raw moment output. The reference has
// neither (its run appends .out rows and, if stopped, must start over).
//
// A run is a sequence of .out rows: per random vector DOS, VAC0, VAC steps, MSD steps
// and spin steps, then the LDOS orbitals. A checkpoint records where the next row
// starts (vector, stage, step), the generator state before that vector's phase draw,
// the evolved states the stage continues from, and the size of every output file, so
// a resumed run truncates rows written after the checkpoint and continues. Moment
// sums are reduced in a fixed order, so a resumed run writes the same bytes as an
// uninterrupted one.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "lsqt/common.h"

class Model;

namespace gqt_host {

enum Stage { kStageDos = 0, kStageVac0, kStageVac, kStageMsd, kStageSpin, kStageLdos, kStageEnd };

struct RunPosition {
  int vector = 0;  // random vector (kStageLdos: unused)
  int stage = kStageDos;
  int step = 0;    // correlation step, or local orbital in kStageLdos
};

struct Checkpoint {
  RunPosition pos;
  std::string rng;                 // Model::rng_state() before pos.vector's phase draw
  std::vector<std::string> files;  // output files (names relative to the input dir)
  std::vector<uint64_t> sizes;     // their sizes at the checkpoint
  // States the stage continues from (pos.step > 0): re then im, number_of_atoms each.
  std::vector<std::vector<real>> states;
  uint64_t fingerprint = 0;
};

// File name of the checkpoint inside the input directory.
std::string checkpoint_path(const Model& model);
// The run's parameters and operator (sizes, flags, precision, a hash of the host ELL
// arrays): a checkpoint is only resumed by the run it came from.
uint64_t run_fingerprint(const Model& model, int precision);
// The output files a run of `model` may append to, relative to its input directory.
std::vector<std::string> output_files(const Model& model);

// Written to <path>.tmp, then renamed over <path>. Throws RunError on I/O failure.
void save_checkpoint(const std::string& path, const Checkpoint& ck);
// false when no checkpoint exists; throws InputError on a damaged file.
bool load_checkpoint(const std::string& path, Checkpoint& ck);

// Raw moments of one row appended to a `<name>_moments.bin` file: a 16-byte header
// ("GQTMOMv1", int32 number_of_moments, int32 0) when the file is new, then the
// moments as number_of_moments (re, im) double pairs, little-endian.
void append_moments(const std::string& file, int n_moments, const real* re, const real* im);

}  // namespace gqt_host
