/* Test infrastructure only: the CPU oracle the parity tests check the CUDA library
 * against. It is a plain-C restatement of the reference's CPU path (the
 * `#else`/CPU_ONLY twins in src/hamiltonian.cu, src/vector.cu, the algorithms in
 * src/sigma.cu and the builders in src/model*.cu, src/anderson.cu), pinned against
 * the reference's own build (oracle/_ref) and its shipped example outputs.
 * The product never links or calls it.
 *
 * Vectors are split real/imaginary double arrays and the ELL arrays are row-major
 * [i*max_neighbor + m], exactly the layout of the reference's CPU build. */
#ifndef LSQT_ORACLE_H
#define LSQT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- random numbers (libstdc++ std::mt19937 + its distributions) ---- */
typedef struct {
  uint32_t x[624];
  int i;
} orc_mt19937;

void orc_mt_seed(orc_mt19937* g, uint32_t seed);
uint32_t orc_mt_next(orc_mt19937* g);
void orc_mt_discard(orc_mt19937* g, uint64_t count);
double orc_uniform_real(orc_mt19937* g, double a, double b);
int orc_uniform_int_0_intmax(orc_mt19937* g);

/* ---- model construction ---- */
typedef struct {
  int n_cell[3];
  int pbc[3];
  int transport_direction;
  double lattice_constant[3];
  int n_orbital;
  int max_neighbor;
  const double* orbital_xyz; /* [n_orbital*3] */
  const int* n_hoppings;     /* [n_orbital] */
  const int* hop_index;      /* [n_orbital*max_neighbor*4]: dx, dy, dz, orbital */
  const double* hop_value;   /* [n_orbital*max_neighbor*2]: re, im */
} orc_lattice;

long orc_lattice_sites(const orc_lattice* lat);
/* Arrays are n*max_neighbor long; entries past neighbor_number[i] are zeroed. */
int orc_build_lattice(const orc_lattice* lat, int* neighbor_number, int* neighbor_list,
                      double* hopping_real, double* hopping_imag, double* xx,
                      double* potential, double* volume);
/* Vacancies (src/model_lattice.cu:26-146): compacts the arrays in place and returns
 * the new number of sites. */
int orc_add_vacancies(orc_mt19937* g, int n, int max_neighbor, int n_vacancies,
                      int* neighbor_number, int* neighbor_list, double* hopping_real,
                      double* hopping_imag, double* xx);
void orc_add_anderson(orc_mt19937* g, int n, double W, double* potential);
void orc_random_phase_state(orc_mt19937* g, int n, int spin, double* re, double* im);

/* ---- the operator ---- */
typedef struct {
  int n;
  int max_neighbor;
  double energy_max;
  const int* neighbor_number;
  const int* neighbor_list;
  const double* potential;
  const double* hopping_real;
  const double* hopping_imag;
  const double* xx;
} orc_ham;

void orc_apply(const orc_ham* h, const double* ir, const double* ii, double* orr, double* oi);
void orc_apply_commutator(const orc_ham* h, const double* ir, const double* ii, double* orr,
                          double* oi);
void orc_apply_current(const orc_ham* h, const double* ir, const double* ii, double* orr,
                       double* oi);
void orc_kernel_polynomial(const orc_ham* h, const double* s0r, const double* s0i,
                           const double* s1r, const double* s1i, double* s2r, double* s2i);
void orc_chebyshev_01(int n, const double* s0r, const double* s0i, const double* s1r,
                      const double* s1i, double* sr, double* si, double b0, double b1,
                      int direction);
void orc_chebyshev_2(const orc_ham* h, const double* s0r, const double* s0i, const double* s1r,
                     const double* s1i, double* s2r, double* s2i, double* sr, double* si,
                     double bessel_m, int label);
void orc_chebyshev_1x(int n, const double* s1xr, const double* s1xi, double* sr, double* si,
                      double b1);
void orc_chebyshev_2x(const orc_ham* h, const double* s0r, const double* s0i,
                      const double* s0xr, const double* s0xi, const double* s1r,
                      const double* s1i, const double* s1xr, const double* s1xi, double* s2r,
                      double* s2i, double* s2xr, double* s2xi, double* sr, double* si,
                      double bessel_m, int label);

/* <left|state> with the reference's two-stage order: sequential sums over blocks of
 * 512 sites, then a sequential sum of the block partials. */
void orc_inner_product(int n, const double* state_r, const double* state_i,
                       const double* left_r, const double* left_i, double* re, double* im);

/* ---- algorithms (src/sigma.cu) ---- */
void orc_find_moments(const orc_ham* h, int n_moments, const double* lr, const double* li,
                      const double* rr, const double* ri, double* mu_re, double* mu_im);
void orc_apply_damping(int n_moments, double* mu_re, double* mu_im);
void orc_chebyshev_summation(int n_moments, const double* mu_re, int n_energy,
                             const double* energy, double energy_max, double volume,
                             double* out);
/* Number of Bessel terms evolve/evolvex use (the |J_m| < 1e-15 cut), m = 2.. */
int orc_bessel_cut(double dt_scaled);
void orc_evolve(const orc_ham* h, int direction, double dt_scaled, double* re, double* im);
void orc_evolvex(const orc_ham* h, int direction, double dt_scaled, double* re, double* im);
/* Moment sets of find_vac / find_msd: out holds n_steps*n_moments (re, im) pairs. */
void orc_vac_moments(const orc_ham* h, int n_moments, int n_steps, const double* time_step,
                     const double* pr, const double* pi, double* mu_re, double* mu_im);
void orc_msd_moments(const orc_ham* h, int n_moments, int n_steps, const double* time_step,
                     const double* pr, const double* pi, double* mu_re, double* mu_im);

#ifdef __cplusplus
}
#endif
#endif
