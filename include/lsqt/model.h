// Replaces class Model (src/model.h:27-104): reads an input directory and builds
// the tight-binding model on the host, bit-for-bit as the reference does (same
// std::mt19937 stream and draw order: vacancies, Anderson disorder, charged
// impurities, then the random phases).
#pragma once

#include <random>
#include <string>
#include <vector>

#include "lsqt/common.h"

class Vector;

class Model
{
public:
  Model(std::string input_dir);
  ~Model();
  Model(const Model&) = delete;
  Model& operator=(const Model&) = delete;

  // The next random-phase vector (orbital < 0) or sqrt(N) e_orbital
  // (src/model.cu:77-109).
  void initialize_state(Vector& random_state, int orbital);
  // The same draw into host arrays of number_of_atoms doubles.
  void initialize_state_host(real* re, real* im, int orbital);

  bool calculate_vac0 = false;
  bool calculate_vac = false;
  bool calculate_msd = false;
  bool calculate_spin = false;
  bool calculate_ldos = false;
  int number_of_random_vectors = 1;
  int number_of_atoms = 0;
  int max_neighbor = 0;
  int number_of_pairs = 0;
  int number_of_energy_points = 0;
  int number_of_moments = 1000;
  int number_of_steps_correlation = 0;
  int number_of_local_orbitals = 0;
  std::string input_dir;
  real energy_max = 10;
  real* energy = nullptr;
  real* time_step = nullptr;
  std::vector<int> local_orbitals;
  // ELL arrays, row-major [i * max_neighbor + m]; the Hamiltonian frees them.
  int* neighbor_number = nullptr;
  int* neighbor_list = nullptr;
  real* xx = nullptr;
  real* potential = nullptr;
  real* hopping_real = nullptr;
  real* hopping_imag = nullptr;
  real volume = 0;

  // Seeds (para.in keywords `seed`, `disorder_seed`, `phase_seed`; the reference's
  // DEBUG build fixes the single stream at 12345678, src/model.cu:34). A disorder
  // seed reseeds the generator right before the Anderson draws; a phase seed right
  // before the first phase draw.
  unsigned seed = 12345678u;
  long disorder_seed = -1;
  long phase_seed = -1;
  bool verbose = true;

  // Extensions (para.in keywords; the reference has none of them): `output_moments`
  // appends each row's raw moments to <name>_moments.bin; `checkpoint_every K`
  // writes lsqt.checkpoint every K rows so that an interrupted run resumes.
  bool output_moments = false;
  int checkpoint_every = 0;
  // `kpm_doubling`: symmetric moment sets (DOS, VAC0, MSD, LDOS) from half the
  // Chebyshev steps (gqt_moments_doubled); equal to the direct moments up to rounding.
  bool kpm_doubling = false;
  // `batch_vectors B`: random vectors run B at a time (16 or 4 per launch) through the
  // multi-vector kernels; the .out files are those of the one-vector run.
  int batch_vectors = 1;
  // The generator's state (with the one-time phase reseed flag), as text.
  std::string rng_state() const;
  void set_rng_state(const std::string& state);

  // Builds without printing or exiting: failures raise gqt_host::InputError.
  struct Quiet {};
  Model(std::string input_dir, Quiet);

private:
  void build();
  void initialize_parameters();
  void verify_parameters();
  void initialize_energy();
  void initialize_time();
  void initialize_local_orbitals();
  void initialize_model_general();
  void initialize_neighbor();
  void initialize_positions();
  void initialize_potential();
  void initialize_hopping();
  void initialize_lattice_model();
  void add_vacancies();
  void add_anderson();
  void add_charged_impurities(const std::vector<real>& x, const std::vector<real>& y,
                              const std::vector<real>& z);
  std::vector<int> random_permutation_prefix(int max_value, int count);
  void say(const std::string& line) const;

  bool requires_time = false;
  bool use_lattice_model = false;
  bool has_anderson = false;
  real anderson_strength = 0;
  bool has_charge = false;
  int charge_number = 0;
  real charge_strength = 0;
  real charge_range = 0;
  bool has_vacancy_disorder = false;
  int number_of_vacancies = 0;
  bool phase_reseeded = false;
  int pbc[3] = {0, 0, 0};
  real box_length[3] = {0, 0, 0};
  std::mt19937 generator;
};
