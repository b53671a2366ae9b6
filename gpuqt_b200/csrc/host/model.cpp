// Model: input parsing and tight-binding model construction on the host.
//
// Follows the reference's Model (src/model.cu, src/model_lattice.cu,
// src/model_general.cu, src/anderson.cu, src/charge.cu): the same input files and
// keywords, the same validation errors, and the same random stream — one
// std::mt19937 drawn in the order vacancies -> Anderson -> charged impurities ->
// phases — so the ELL arrays, potentials and phase vectors are bit-identical.
#include "lsqt/model.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <thread>

#include "gpuqt.h"
#include "lsqt/vector.h"

namespace {
const double kPi = 3.141592653589793;  // src/model.cu:27

std::string dir_file(const std::string& dir, const char* name) { return dir + "/" + name; }

[[noreturn]] void bad(const std::string& m) { throw gqt_host::InputError(m); }
}  // namespace

namespace gqt_host {
namespace {
thread_local bool t_throw = false;
}

ThrowScope::ThrowScope() : saved(t_throw) { t_throw = true; }
ThrowScope::~ThrowScope() { t_throw = saved; }

void die(const std::string& message, int code)
{
  if (t_throw)
    throw RunError(message, code);
  std::cout << message << std::endl;
  std::exit(1);
}

void check(int status, const char* what)
{
  if (status != GQT_OK)
    die(std::string("Error in ") + what + ": " + gqt_last_error(), status);
}
}  // namespace gqt_host

Model::Model(std::string input_dir_) : input_dir(std::move(input_dir_))
{
  try {
    build();
  } catch (const gqt_host::InputError& e) {
    gqt_host::die(std::string("Error: ") + e.what());
  }
}

Model::Model(std::string input_dir_, Quiet) : input_dir(std::move(input_dir_))
{
  verbose = false;
  build();
}

Model::~Model()
{
  delete[] energy;
  delete[] time_step;
  delete[] neighbor_number;
  delete[] neighbor_list;
  delete[] xx;
  delete[] potential;
  delete[] hopping_real;
  delete[] hopping_imag;
}

void Model::say(const std::string& line) const
{
  if (verbose)
    std::cout << line << std::endl;
}

void Model::build()
{
  initialize_parameters();
  generator = std::mt19937(seed);
  if (use_lattice_model)
    initialize_lattice_model();
  else
    initialize_model_general();
  initialize_energy();
  if (requires_time)
    initialize_time();
  if (calculate_ldos)
    initialize_local_orbitals();
}

// ------------------------------------------------------------------ para.in
// Keywords of src/model.cu:260-305, plus `seed`, `disorder_seed`, `phase_seed`.
void Model::initialize_parameters()
{
  const std::string filename = dir_file(input_dir, "para.in");
  std::ifstream input(filename);
  if (!input.is_open())
    bad("cannot open " + filename);
  say("- reading " + filename);
  std::string line;
  while (std::getline(input, line)) {
    std::stringstream ss(line);
    std::string token;
    ss >> token;
    if (token.empty())
      continue;
    if (token == "model") {
      ss >> use_lattice_model;
    } else if (token == "anderson_disorder") {
      has_anderson = true;
      ss >> anderson_strength;
    } else if (token == "charged_impurity") {
      has_charge = true;
      ss >> charge_number >> charge_strength >> charge_range;
    } else if (token == "vacancy_disorder") {
      has_vacancy_disorder = true;
      ss >> number_of_vacancies;
    } else if (token == "calculate_vac0") {
      calculate_vac0 = true;
    } else if (token == "calculate_vac") {
      calculate_vac = true;
    } else if (token == "calculate_msd") {
      calculate_msd = true;
    } else if (token == "calculate_spin") {
      calculate_spin = true;
    } else if (token == "calculate_ldos") {
      calculate_ldos = true;
    } else if (token == "number_of_random_vectors") {
      ss >> number_of_random_vectors;
    } else if (token == "number_of_moments") {
      ss >> number_of_moments;
    } else if (token == "energy_max") {
      ss >> energy_max;
    } else if (token == "seed") {
      ss >> seed;
    } else if (token == "disorder_seed") {
      ss >> disorder_seed;
    } else if (token == "phase_seed") {
      ss >> phase_seed;
    } else if (token == "output_moments") {
      output_moments = true;
    } else if (token == "kpm_doubling") {
      kpm_doubling = true;
    } else if (token == "batch_vectors") {
      ss >> batch_vectors;
      if (!ss || batch_vectors < 1)
        bad("batch_vectors needs a number of vectors >= 1");
    } else if (token == "checkpoint_every") {
      ss >> checkpoint_every;
      if (!ss || checkpoint_every < 1)
        bad("checkpoint_every needs a number of rows >= 1");
    } else {
      bad("Unknown identifier in " + filename + ": " + line +
          "\nValid keywords include: model anderson_disorder charged_impurity "
          "vacancy_disorder calculate_vac0 calculate_vac calculate_msd calculate_spin "
          "calculate_ldos number_of_random_vectors number_of_moments energy_max seed "
          "disorder_seed phase_seed output_moments checkpoint_every kpm_doubling "
          "batch_vectors");
    }
  }
  verify_parameters();
}

// src/model.cu:128-241.
void Model::verify_parameters()
{
  requires_time = calculate_vac || calculate_msd || calculate_spin;
  if (use_lattice_model) {
    say("- Use lattice model");
    if (calculate_spin)
      bad("lattice model does not support spin calculations yet");
    if (has_vacancy_disorder && number_of_vacancies <= 0)
      bad("number of vacancies should > 0");
  } else {
    say("- Use general model");
    if (has_anderson)
      bad("General model does not allowed to add Anderson disorder");
    if (has_vacancy_disorder)
      bad("General model does not allowed to add vacancy disorder");
    if (has_charge)
      bad("General model does not allowed to add charged impurities");
  }
  if (calculate_spin && calculate_vac0)
    bad("spin and VAC0 cannot be calculated together");
  if (calculate_spin && calculate_vac)
    bad("spin and VAC cannot be calculated together");
  if (calculate_spin && calculate_msd)
    bad("spin and MSD cannot be calculated together");
  if (number_of_random_vectors <= 0)
    bad("Number of random vectors should > 0");
  if (number_of_moments <= 0)
    bad("Number of moments should > 0");
  if (energy_max <= 0)
    bad("Energy maximum should > 0");
  if (verbose) {
    std::cout << "- Number of random vectors is " << number_of_random_vectors << "\n"
              << "- Number of moments is " << number_of_moments << "\n"
              << "- Energy maximum is " << energy_max << std::endl;
  }
}

// ------------------------------------------------------------------ data files
void Model::initialize_energy()
{
  const std::string filename = dir_file(input_dir, "energy.in");
  std::ifstream input(filename);
  if (!input.is_open())
    bad("cannot open " + filename);
  input >> number_of_energy_points;
  if (!input || number_of_energy_points < 0)
    bad("cannot read the number of energy points in " + filename);
  energy = new real[number_of_energy_points > 0 ? number_of_energy_points : 1];
  for (int n = 0; n < number_of_energy_points; ++n)
    input >> energy[n];
  say("- number of energy points = " + std::to_string(number_of_energy_points));
}

void Model::initialize_time()
{
  const std::string filename = dir_file(input_dir, "time_step.in");
  std::ifstream input(filename);
  if (!input.is_open())
    bad("cannot open " + filename);
  input >> number_of_steps_correlation;
  if (!input || number_of_steps_correlation < 0)
    bad("cannot read the number of time steps in " + filename);
  time_step = new real[number_of_steps_correlation > 0 ? number_of_steps_correlation : 1];
  for (int n = 0; n < number_of_steps_correlation; ++n)
    input >> time_step[n];
  say("- number of time steps = " + std::to_string(number_of_steps_correlation));
}

void Model::initialize_local_orbitals()
{
  const std::string filename = dir_file(input_dir, "local_orbitals.in");
  std::ifstream input(filename);
  if (!input.is_open())
    bad("cannot open " + filename);
  input >> number_of_local_orbitals;
  if (!input || number_of_local_orbitals < 0)
    bad("cannot read the number of local orbitals in " + filename);
  local_orbitals.resize(number_of_local_orbitals);
  for (int n = 0; n < number_of_local_orbitals; ++n) {
    input >> local_orbitals[n];
    if (local_orbitals[n] < 0 || local_orbitals[n] >= number_of_atoms)
      bad("wrong local orbital index: " + std::to_string(local_orbitals[n]));
  }
}

// ------------------------------------------------------------------ general model
// src/model_general.cu:24-185.
void Model::initialize_model_general()
{
  initialize_neighbor();
  initialize_positions();
  initialize_potential();
  initialize_hopping();
}

void Model::initialize_neighbor()
{
  const std::string filename = dir_file(input_dir, "neighbor.in");
  std::ifstream input(filename);
  if (!input.is_open())
    bad("cannot open " + filename);
  input >> number_of_atoms >> max_neighbor;
  if (!input || number_of_atoms <= 0 || max_neighbor <= 0)
    bad("bad header in " + filename);
  number_of_pairs = number_of_atoms * max_neighbor;
  neighbor_number = new int[number_of_atoms];
  neighbor_list = new int[number_of_pairs]();
  for (int n = 0; n < number_of_atoms; ++n) {
    input >> neighbor_number[n];
    if (!input || neighbor_number[n] < 0 || neighbor_number[n] > max_neighbor)
      bad("bad neighbour count for orbital " + std::to_string(n) + " in " + filename);
    for (int m = 0; m < neighbor_number[n]; ++m)
      input >> neighbor_list[n * max_neighbor + m];
  }
  say("- Number of orbitals is " + std::to_string(number_of_atoms));
}

void Model::initialize_positions()
{
  const std::string filename = dir_file(input_dir, "position.in");
  std::ifstream input(filename);
  if (!input.is_open())
    bad("cannot open " + filename);
  real box;
  input >> box >> volume;
  std::vector<real> x(number_of_atoms);
  for (int i = 0; i < number_of_atoms; ++i)
    input >> x[i];
  // Minimum-image separation along the transport direction (src/model_general.cu:64-72).
  auto reduce = [box](real d) {
    if (d > box / 2.0)
      return d - box;
    if (d < -box / 2.0)
      return d + box;
    return d;
  };
  xx = new real[number_of_pairs]();
  for (int n = 0; n < number_of_atoms; ++n)
    for (int m = 0; m < neighbor_number[n]; ++m) {
      const int k = n * max_neighbor + m;
      const int j = neighbor_list[k];
      if (j < 0 || j >= number_of_atoms)
        bad("neighbour index " + std::to_string(j) + " of orbital " + std::to_string(n) +
            " out of range");
      xx[k] = reduce(x[j] - x[n]);
    }
}

void Model::initialize_potential()
{
  const std::string filename = dir_file(input_dir, "potential.in");
  std::ifstream input(filename);
  potential = new real[number_of_atoms];
  const bool given = input.is_open();
  say(given ? "- On-site potential will be read in" : "- Assuming zero on-site potential");
  for (int n = 0; n < number_of_atoms; ++n) {
    if (given)
      input >> potential[n];
    else
      potential[n] = 0.0;
  }
}

void Model::initialize_hopping()
{
  const std::string filename = dir_file(input_dir, "hopping.in");
  std::ifstream input(filename);
  int type = 3;  // 1 complex, 2 real, 3 uniform -1 (file absent)
  if (input.is_open()) {
    std::string kind;
    input >> kind;
    if (kind == "complex")
      type = 1;
    else if (kind == "real")
      type = 2;
    else
      bad("Hoppings can only be real or complex");
  }
  hopping_real = new real[number_of_pairs]();
  hopping_imag = new real[number_of_pairs]();
  for (int n = 0; n < number_of_atoms; ++n)
    for (int m = 0; m < neighbor_number[n]; ++m) {
      const int k = n * max_neighbor + m;
      if (type < 3)
        input >> hopping_real[k];
      else
        hopping_real[k] = -1.0;
      if (type == 1)
        input >> hopping_imag[k];
      else
        hopping_imag[k] = 0.0;
    }
}

// ------------------------------------------------------------------ lattice model
namespace {
int wrap_index(int nx, int ny, int nz, const int* N, int orbital, int n_orbital)
{
  // One periodic wrap per direction (src/model_lattice.cu:148-163).
  if (nx < 0)
    nx += N[0];
  if (nx >= N[0])
    nx -= N[0];
  if (ny < 0)
    ny += N[1];
  if (ny >= N[1])
    ny -= N[1];
  if (nz < 0)
    nz += N[2];
  if (nz >= N[2])
    nz -= N[2];
  return ((nx * N[1] + ny) * N[2] + nz) * n_orbital + orbital;
}
}  // namespace

// src/model_lattice.cu:165-402.
void Model::initialize_lattice_model()
{
  const std::string filename = dir_file(input_dir, "lattice.in");
  std::ifstream input(filename);
  if (!input.is_open())
    bad("Could not open " + filename);
  int N[3];
  input >> N[0] >> N[1] >> N[2];
  const char* axis = "xyz";
  for (int d = 0; d < 3; ++d)
    if (!input || N[d] <= 0)
      bad(std::string("Number of cells in the ") + axis[d] + " direction should > 0");
  int transport;
  input >> pbc[0] >> pbc[1] >> pbc[2] >> transport;
  for (int d = 0; d < 3; ++d)
    if (pbc[d] != 0 && pbc[d] != 1)
      bad(std::string(1, axis[d]) + " direction has wrong boundary");
  if (transport < 0 || transport > 2)
    bad("wrong transport direction");
  if (pbc[transport] != 1)
    bad("transport direction must be periodic");
  real a[3];
  input >> a[0] >> a[1] >> a[2];
  for (int d = 0; d < 3; ++d)
    if (!(a[d] > 0))
      bad(std::string("lattice constant in ") + axis[d] + " direction < 0");
  for (int d = 0; d < 3; ++d)
    box_length[d] = a[d] * N[d];
  volume = box_length[0] * box_length[1] * box_length[2];

  int n_orbital;
  input >> n_orbital >> max_neighbor;
  if (!input || n_orbital <= 0)
    bad("number of orbitals per cell should > 0");
  if (max_neighbor <= 0)
    bad("maximum number of hoppings per orbital should > 0");
  const long long sites = (long long)n_orbital * N[0] * N[1] * N[2];
  if (sites * max_neighbor > INT_MAX)
    bad("lattice too large for 32-bit ELL indices");
  number_of_atoms = (int)sites;
  number_of_pairs = number_of_atoms * max_neighbor;

  std::vector<real> xc(n_orbital), yc(n_orbital), zc(n_orbital);
  for (int m = 0; m < n_orbital; ++m)
    input >> xc[m] >> yc[m] >> zc[m];
  // Per orbital m, hopping i lives at slot m * max_neighbor + i.
  const int slots = n_orbital * max_neighbor;
  std::vector<int> hop_cell(3 * slots, 0), hop_orbital(slots, 0), n_hop(n_orbital, 0);
  std::vector<real> hop_re(slots, 0), hop_im(slots, 0);
  for (int m = 0; m < n_orbital; ++m) {
    input >> n_hop[m];
    if (!input || n_hop[m] < 0 || n_hop[m] > max_neighbor)
      bad("bad number of hoppings for orbital " + std::to_string(m));
    for (int i = 0; i < n_hop[m]; ++i) {
      const int k = m * max_neighbor + i;
      input >> hop_cell[3 * k] >> hop_cell[3 * k + 1] >> hop_cell[3 * k + 2] >> hop_orbital[k] >>
        hop_re[k] >> hop_im[k];
      if (!input || hop_orbital[k] < 0 || hop_orbital[k] >= n_orbital)
        bad("bad hopping " + std::to_string(i) + " of orbital " + std::to_string(m));
    }
  }
  say("- total number of orbitals = " + std::to_string(number_of_atoms));

  neighbor_number = new int[number_of_atoms];
  neighbor_list = new int[number_of_pairs]();
  hopping_real = new real[number_of_pairs]();
  hopping_imag = new real[number_of_pairs]();
  xx = new real[number_of_pairs]();
  potential = new real[number_of_atoms]();
  std::vector<real> px, py, pz;
  if (has_charge) {
    px.resize(number_of_atoms);
    py.resize(number_of_atoms);
    pz.resize(number_of_atoms);
  }

  for (int c0 = 0; c0 < N[0]; ++c0)
    for (int c1 = 0; c1 < N[1]; ++c1)
      for (int c2 = 0; c2 < N[2]; ++c2)
        for (int m = 0; m < n_orbital; ++m) {
          const int site = wrap_index(c0, c1, c2, N, m, n_orbital);
          if (has_charge) {
            px[site] = xc[m] + a[0] * c0;
            py[site] = yc[m] + a[1] * c1;
            pz[site] = zc[m] + a[2] * c2;
          }
          int count = 0;
          for (int i = 0; i < n_hop[m]; ++i) {
            const int k = m * max_neighbor + i;
            const int t0 = c0 + hop_cell[3 * k], t1 = c1 + hop_cell[3 * k + 1],
                      t2 = c2 + hop_cell[3 * k + 2];
            // Hoppings that leave an open boundary are dropped (rows become short).
            if ((!pbc[0] && (t0 < 0 || t0 >= N[0])) || (!pbc[1] && (t1 < 0 || t1 >= N[1])) ||
                (!pbc[2] && (t2 < 0 || t2 >= N[2])))
              continue;
            const int e = site * max_neighbor + count;
            neighbor_list[e] = wrap_index(t0, t1, t2, N, hop_orbital[k], n_orbital);
            // The orbital offset is taken from the x coordinates whatever the
            // transport direction (src/model_lattice.cu:373-376).
            real dx = a[transport] * hop_cell[3 * k + transport];
            dx += xc[hop_orbital[k]] - xc[m];
            xx[e] = dx;
            hopping_real[e] = hop_re[k];
            hopping_imag[e] = hop_im[k];
            ++count;
          }
          neighbor_number[site] = count;
        }

  if (has_vacancy_disorder)
    add_vacancies();
  if (has_anderson)
    add_anderson();
  if (has_charge)
    add_charged_impurities(px, py, pz);
}

// The first `count` entries of the permutation of 0..max_value-1 that the reference
// builds with j = U{0..INT_MAX} % (max_value - i) + i (src/model_lattice.cu:26-43,
// src/charge.cu:46-62).
std::vector<int> Model::random_permutation_prefix(int max_value, int count)
{
  std::vector<int> perm(max_value);
  for (int i = 0; i < max_value; ++i)
    perm[i] = i;
  std::uniform_int_distribution<int> pick(0, INT_MAX);
  for (int i = 0; i < max_value; ++i) {
    const int j = pick(generator) % (max_value - i) + i;
    std::swap(perm[i], perm[j]);
  }
  perm.resize(count < max_value ? count : max_value);
  return perm;
}

// src/model_lattice.cu:70-146: remove the vacancy sites and compact the ELL rows.
void Model::add_vacancies()
{
  if (number_of_vacancies > number_of_atoms)
    bad("more vacancies than orbitals");
  const int n0 = number_of_atoms, z = max_neighbor;
  std::vector<int> chosen = random_permutation_prefix(n0, number_of_vacancies);
  std::vector<char> gone(n0, 0);
  for (int k : chosen)
    gone[k] = 1;
  std::vector<int> new_index(n0, -1);
  int kept = 0;
  for (int i = 0; i < n0; ++i)
    if (!gone[i])
      new_index[i] = kept++;
  const int n1 = kept;
  int* nn = new int[n1];
  int* nl = new int[(size_t)n1 * z]();
  real* hr = new real[(size_t)n1 * z]();
  real* hi = new real[(size_t)n1 * z]();
  real* x1 = new real[(size_t)n1 * z]();
  for (int i = 0; i < n0; ++i) {
    if (gone[i])
      continue;
    const int r = new_index[i];
    int c = 0;
    for (int m = 0; m < neighbor_number[i]; ++m) {
      const int old = i * z + m;
      const int j = neighbor_list[old];
      if (gone[j])
        continue;
      const int e = r * z + c;
      nl[e] = new_index[j];
      hr[e] = hopping_real[old];
      hi[e] = hopping_imag[old];
      x1[e] = xx[old];
      ++c;
    }
    nn[r] = c;
  }
  delete[] neighbor_number;
  delete[] neighbor_list;
  delete[] hopping_real;
  delete[] hopping_imag;
  delete[] xx;
  delete[] potential;
  neighbor_number = nn;
  neighbor_list = nl;
  hopping_real = hr;
  hopping_imag = hi;
  xx = x1;
  potential = new real[n1]();
  number_of_atoms = n1;
  number_of_pairs = n1 * z;
  say("- removed " + std::to_string(number_of_vacancies) + " vacancies");
}

// Anderson::add_disorder (src/anderson.cu:22-29).
void Model::add_anderson()
{
  if (disorder_seed >= 0)
    generator.seed((unsigned)disorder_seed);
  const real half = anderson_strength * 0.5;
  std::uniform_real_distribution<real> draw(-half, half);
  for (int n = 0; n < number_of_atoms; ++n)
    potential[n] = draw(generator);
}

// Charge::add_impurities (src/charge.cu:25-44, :109-172): Gaussian impurity
// potentials summed through a periodic cell list of cell size 5 xi. The potential is
// reset first, as in the reference.
void Model::add_charged_impurities(const std::vector<real>& x, const std::vector<real>& y,
                                   const std::vector<real>& z)
{
  const int N = number_of_atoms, Ni = charge_number;
  if (Ni < 0 || Ni > N)
    bad("bad number of charged impurities");
  const real rc = 5.0 * charge_range, rc2 = rc * rc;
  std::vector<int> where = random_permutation_prefix(N, Ni);
  std::vector<real> strength(Ni);
  {
    const real half = charge_strength * 0.5;
    std::uniform_real_distribution<real> draw(-half, half);
    for (int i = 0; i < Ni; ++i)
      strength[i] = draw(generator);
  }
  int nc[3];
  for (int d = 0; d < 3; ++d)
    nc[d] = pbc[d] ? (int)std::floor(box_length[d] / rc) : 1;
  if (nc[0] <= 0 || nc[1] <= 0 || nc[2] <= 0)
    bad("charged-impurity range larger than the box");
  const int ncell = nc[0] * nc[1] * nc[2];
  auto cell_of = [&](real px, real py, real pz, int* c) {
    c[0] = (int)std::floor(px / rc);
    c[1] = (int)std::floor(py / rc);
    c[2] = (int)std::floor(pz / rc);
    for (int d = 0; d < 3; ++d) {
      while (c[d] < 0)
        c[d] += nc[d];
      while (c[d] >= nc[d])
        c[d] -= nc[d];
    }
    return c[0] + nc[0] * c[1] + nc[0] * nc[1] * c[2];
  };
  std::vector<int> count(ncell, 0), start(ncell, 0), members(N, 0);
  int c[3];
  for (int i = 0; i < N; ++i)
    ++count[cell_of(x[i], y[i], z[i], c)];
  for (int i = 1; i < ncell; ++i)
    start[i] = count[i - 1] + start[i - 1];
  std::fill(count.begin(), count.end(), 0);
  for (int i = 0; i < N; ++i) {
    const int id = cell_of(x[i], y[i], z[i], c);
    members[start[id] + count[id]] = i;
    ++count[id];
  }
  const real factor = -0.5 / (charge_range * charge_range);
  real half_box[3];
  for (int d = 0; d < 3; ++d)
    half_box[d] = box_length[d] * 0.5;
  for (int n = 0; n < N; ++n)
    potential[n] = 0.0;
  const int lim[3] = {pbc[0] ? 1 : 0, pbc[1] ? 1 : 0, pbc[2] ? 1 : 0};
  for (int q = 0; q < Ni; ++q) {
    const int n1 = where[q];
    const int id = cell_of(x[n1], y[n1], z[n1], c);
    for (int k = -lim[2]; k <= lim[2]; ++k)
      for (int j = -lim[1]; j <= lim[1]; ++j)
        for (int i = -lim[0]; i <= lim[0]; ++i) {
          int nb = id + k * nc[0] * nc[1] + j * nc[0] + i;
          if (c[0] + i < 0)
            nb += nc[0];
          if (c[0] + i >= nc[0])
            nb -= nc[0];
          if (c[1] + j < 0)
            nb += nc[1] * nc[0];
          if (c[1] + j >= nc[1])
            nb -= nc[1] * nc[0];
          if (c[2] + k < 0)
            nb += ncell;
          if (c[2] + k >= nc[2])
            nb -= ncell;
          for (int s = 0; s < count[nb]; ++s) {
            const int n2 = members[start[nb] + s];
            real r[3] = {x[n2] - x[n1], y[n2] - y[n1], z[n2] - z[n1]};
            real d2 = 0.0;
            for (int d = 0; d < 3; ++d) {
              r[d] = std::fabs(r[d]);
              if (pbc[d] == 1 && r[d] > half_box[d])
                r[d] = box_length[d] - r[d];
              d2 += r[d] * r[d];
            }
            if (d2 > rc2)
              continue;
            potential[n2] += strength[q] * std::exp(d2 * factor);
          }
        }
  }
}

// ------------------------------------------------------------------ states
void Model::initialize_state_host(real* re, real* im, int orbital)
{
  const int N = number_of_atoms;
  if (orbital >= 0) {
    for (int n = 0; n < N; ++n) {
      re[n] = 0.0;
      im[n] = 0.0;
    }
    re[orbital] = std::sqrt(1.0 * N);
    return;
  }
  if (phase_seed >= 0 && !phase_reseeded) {
    generator.seed((unsigned)phase_seed);
    phase_reseeded = true;
  }
  // The phases are drawn in the reference's order (one draw per phase-carrying
  // orbital; with spin only the even orbitals carry one, src/model.cu:77-109); cos and
  // sin of them, the bulk of the work, are evaluated over chunks in parallel threads,
  // which gives the same values as the serial loop.
  std::uniform_real_distribution<real> phase(0, 2 * kPi);
  const int step = calculate_spin ? 2 : 1;
  const int count = (N + step - 1) / step;
  std::vector<real> p(count);
  for (int k = 0; k < count; ++k)
    p[k] = phase(generator);
  auto fill = [&](int k0, int k1) {
    for (int k = k0; k < k1; ++k) {
      const int n = k * step;
      re[n] = std::cos(p[k]);
      im[n] = std::sin(p[k]);
      if (step == 2 && n + 1 < N) {
        re[n + 1] = 0.0;
        im[n + 1] = 0.0;
      }
    }
  };
  const unsigned hw = std::thread::hardware_concurrency();
  const int threads = count < (1 << 16) ? 1 : (int)std::min(16u, hw ? hw : 1u);
  if (threads <= 1) {
    fill(0, count);
    return;
  }
  std::vector<std::thread> pool;
  const int chunk = (count + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    const int k0 = t * chunk, k1 = std::min(count, k0 + chunk);
    if (k0 < k1)
      pool.emplace_back(fill, k0, k1);
  }
  for (auto& th : pool)
    th.join();
}

std::string Model::rng_state() const
{
  std::ostringstream os;
  os << (phase_reseeded ? 1 : 0) << ' ' << generator;
  return os.str();
}

void Model::set_rng_state(const std::string& state)
{
  std::istringstream is(state);
  int reseeded = 0;
  is >> reseeded >> generator;
  if (!is)
    bad("the checkpoint's generator state cannot be read");
  phase_reseeded = reseeded != 0;
}

void Model::initialize_state(Vector& random_state, int orbital)
{
  std::vector<real> re(number_of_atoms), im(number_of_atoms);
  initialize_state_host(re.data(), im.data(), orbital);
  random_state.copy_from_host(re.data(), im.data());
}
