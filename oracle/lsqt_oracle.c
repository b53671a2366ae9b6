/* Test infrastructure only — the CPU oracle for the parity tests; never part of the
 * product. A plain-C restatement of the reference's CPU path: each function cites
 * the reference lines it follows (paths relative to the reference checkout).
 *
 * Arithmetic is kept in the reference's exact operation order and compiled with
 * -ffp-contract=off, so every value matches the reference's own CPU build bit for
 * bit. OpenMP splits only loops whose iterations are independent (one site, or one
 * 512-site reduction block, per iteration); the serial order of every floating-point
 * sum is unchanged, so the threaded oracle is bit-identical to the serial reference.
 *
 * Pinning: tests/test_oracle.py checks this file against the reference built from
 * its sources (oracle/_ref) and against the reference's shipped example outputs
 * (tests/golden/). */
#define _GNU_SOURCE
#include "lsqt_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.141592653589793 /* src/sigma.cu:27, src/model.cu:27 */
#define ORC_BLOCK 512            /* BLOCK_SIZE, src/vector.cu:22 */

/* ------------------------------------------------------------------------------
 * Random numbers. The reference draws everything from one std::mt19937
 * (src/model.h:103). MT19937 is the published generator of Matsumoto & Nishimura
 * (1998); the two distributions follow libstdc++ 13 as the reference uses them.
 * ---------------------------------------------------------------------------- */
void orc_mt_seed(orc_mt19937* g, uint32_t seed)
{
  g->x[0] = seed;
  for (int i = 1; i < 624; ++i)
    g->x[i] = 1812433253u * (g->x[i - 1] ^ (g->x[i - 1] >> 30)) + (uint32_t)i;
  g->i = 624;
}

static void orc_mt_twist(orc_mt19937* g)
{
  for (int k = 0; k < 624; ++k) {
    uint32_t y = (g->x[k] & 0x80000000u) | (g->x[(k + 1) % 624] & 0x7fffffffu);
    uint32_t v = g->x[(k + 397) % 624] ^ (y >> 1);
    if (y & 1u)
      v ^= 0x9908b0dfu;
    g->x[k] = v;
  }
  g->i = 0;
}

uint32_t orc_mt_next(orc_mt19937* g)
{
  if (g->i >= 624)
    orc_mt_twist(g);
  uint32_t y = g->x[g->i++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

void orc_mt_discard(orc_mt19937* g, uint64_t count)
{
  for (uint64_t k = 0; k < count; ++k)
    (void)orc_mt_next(g);
}

/* std::uniform_real_distribution<double>(a, b): generate_canonical<double, 53> takes
 * two 32-bit draws, (x1 + x2 * 2^32) / 2^64, clamped below 1, then u * (b - a) + a. */
double orc_uniform_real(orc_mt19937* g, double a, double b)
{
  double x1 = (double)orc_mt_next(g);
  double x2 = (double)orc_mt_next(g);
  double sum = x1;
  sum = sum + x2 * 4294967296.0;
  double u = sum / 18446744073709551616.0;
  if (u >= 1.0)
    u = nextafter(1.0, 0.0);
  return u * (b - a) + a;
}

/* std::uniform_int_distribution<int>(0, INT_MAX) on a 32-bit engine: libstdc++
 * downscales with Lemire's multiply-shift (range 2^31, no rejection possible),
 * which reduces to the top 31 bits of one draw. Used by src/model_lattice.cu:33. */
int orc_uniform_int_0_intmax(orc_mt19937* g)
{
  uint64_t product = (uint64_t)orc_mt_next(g) * (uint64_t)2147483648u;
  return (int)(product >> 32);
}

/* ------------------------------------------------------------------------------
 * Model construction.
 * ---------------------------------------------------------------------------- */
long orc_lattice_sites(const orc_lattice* lat)
{
  return (long)lat->n_orbital * lat->n_cell[0] * lat->n_cell[1] * lat->n_cell[2];
}

/* find_index, src/model_lattice.cu:148-163: one periodic wrap per direction. */
static int orc_find_index(int nx, int ny, int nz, int Nx, int Ny, int Nz, int m, int No)
{
  if (nx < 0)
    nx += Nx;
  if (nx >= Nx)
    nx -= Nx;
  if (ny < 0)
    ny += Ny;
  if (ny >= Ny)
    ny -= Ny;
  if (nz < 0)
    nz += Nz;
  if (nz >= Nz)
    nz -= Nz;
  return ((nx * Ny + ny) * Nz + nz) * No + m;
}

/* Model::initialize_lattice_model, src/model_lattice.cu:165-387 (without the
 * printing and the optional disorder calls at :389-399). */
int orc_build_lattice(const orc_lattice* lat, int* neighbor_number, int* neighbor_list,
                      double* hopping_real, double* hopping_imag, double* xx,
                      double* potential, double* volume)
{
  const int* Nc = lat->n_cell;
  int No = lat->n_orbital, z = lat->max_neighbor, td = lat->transport_direction;
  long n = orc_lattice_sites(lat);
  double box[3];
  for (int d = 0; d < 3; ++d)
    box[d] = lat->lattice_constant[d] * Nc[d];
  *volume = box[0] * box[1] * box[2];
  memset(neighbor_list, 0, sizeof(int) * (size_t)n * z);
  memset(hopping_real, 0, sizeof(double) * (size_t)n * z);
  memset(hopping_imag, 0, sizeof(double) * (size_t)n * z);
  memset(xx, 0, sizeof(double) * (size_t)n * z);
  for (long i = 0; i < n; ++i)
    potential[i] = 0.0;

  for (int nx1 = 0; nx1 < Nc[0]; ++nx1)
    for (int ny1 = 0; ny1 < Nc[1]; ++ny1)
      for (int nz1 = 0; nz1 < Nc[2]; ++nz1)
        for (int m = 0; m < No; ++m) {
          int n1 = orc_find_index(nx1, ny1, nz1, Nc[0], Nc[1], Nc[2], m, No);
          int count = 0;
          for (int i = 0; i < lat->n_hoppings[m]; ++i) {
            int k = m * z + i;
            const int* hi = lat->hop_index + 4 * k;
            int nx2 = hi[0] + nx1, ny2 = hi[1] + ny1, nz2 = hi[2] + nz1;
            int skip_x = !lat->pbc[0] && (nx2 < 0 || nx2 >= Nc[0]);
            int skip_y = !lat->pbc[1] && (ny2 < 0 || ny2 >= Nc[1]);
            int skip_z = !lat->pbc[2] && (nz2 < 0 || nz2 >= Nc[2]);
            if (skip_x || skip_y || skip_z)
              continue;
            long e = (long)n1 * z + count;
            neighbor_list[e] = orc_find_index(nx2, ny2, nz2, Nc[0], Nc[1], Nc[2], hi[3], No);
            /* :373-376: the orbital offset is always taken from the x coordinate. */
            double x12 = lat->lattice_constant[td] * (double)hi[td];
            x12 += lat->orbital_xyz[3 * hi[3]] - lat->orbital_xyz[3 * m];
            xx[e] = x12;
            hopping_real[e] = lat->hop_value[2 * k];
            hopping_imag[e] = lat->hop_value[2 * k + 1];
            ++count;
          }
          neighbor_number[n1] = count;
        }
  return 0;
}

/* Model::add_vacancies with create_random_numbers / specify_vacancies /
 * find_new_atom_index, src/model_lattice.cu:26-146. */
int orc_add_vacancies(orc_mt19937* g, int n, int z, int n_vacancies, int* nn, int* nl,
                      double* hr, double* hi, double* xx)
{
  int* perm = (int*)malloc(sizeof(int) * n);
  for (int i = 0; i < n; ++i)
    perm[i] = i;
  for (int i = 0; i < n; ++i) {
    int j = orc_uniform_int_0_intmax(g) % (n - i) + i;
    int t = perm[i];
    perm[i] = perm[j];
    perm[j] = t;
  }
  int* is_vac = (int*)calloc(n, sizeof(int));
  for (int v = 0; v < n_vacancies; ++v)
    is_vac[perm[v]] = 1;
  int* new_index = (int*)malloc(sizeof(int) * n);
  int count = 0;
  for (int i = 0; i < n; ++i)
    if (!is_vac[i])
      new_index[i] = count++;
  size_t pairs = (size_t)n * z;
  int* nn0 = (int*)malloc(sizeof(int) * n);
  int* nl0 = (int*)malloc(sizeof(int) * pairs);
  double* hr0 = (double*)malloc(sizeof(double) * pairs);
  double* hi0 = (double*)malloc(sizeof(double) * pairs);
  double* xx0 = (double*)malloc(sizeof(double) * pairs);
  memcpy(nn0, nn, sizeof(int) * n);
  memcpy(nl0, nl, sizeof(int) * pairs);
  memcpy(hr0, hr, sizeof(double) * pairs);
  memcpy(hi0, hi, sizeof(double) * pairs);
  memcpy(xx0, xx, sizeof(double) * pairs);
  memset(nl, 0, sizeof(int) * pairs);
  memset(hr, 0, sizeof(double) * pairs);
  memset(hi, 0, sizeof(double) * pairs);
  memset(xx, 0, sizeof(double) * pairs);
  int atom = 0;
  for (int i = 0; i < n; ++i) {
    if (is_vac[i])
      continue;
    int c = 0;
    for (int m = 0; m < nn0[i]; ++m) {
      size_t old = (size_t)i * z + m;
      int k = nl0[old];
      if (!is_vac[k]) {
        size_t e = (size_t)atom * z + c;
        nl[e] = new_index[k];
        hr[e] = hr0[old];
        hi[e] = hi0[old];
        xx[e] = xx0[old];
        ++c;
      }
    }
    nn[atom] = c;
    ++atom;
  }
  free(perm);
  free(is_vac);
  free(new_index);
  free(nn0);
  free(nl0);
  free(hr0);
  free(hi0);
  free(xx0);
  return atom;
}

/* Anderson::add_disorder, src/anderson.cu:22-29. */
void orc_add_anderson(orc_mt19937* g, int n, double W, double* potential)
{
  double W2 = W * 0.5;
  for (int i = 0; i < n; ++i)
    potential[i] = orc_uniform_real(g, -W2, W2);
}

/* Model::initialize_state with orbital < 0, src/model.cu:77-109. */
void orc_random_phase_state(orc_mt19937* g, int n, int spin, double* re, double* im)
{
  if (spin) {
    for (int i = 0; i < n; i += 2) {
      double ph = orc_uniform_real(g, 0.0, 2 * ORC_PI);
      re[i] = cos(ph);
      im[i] = sin(ph);
      re[i + 1] = 0.0;
      im[i + 1] = 0.0;
    }
  } else {
    for (int i = 0; i < n; ++i) {
      double ph = orc_uniform_real(g, 0.0, 2 * ORC_PI);
      re[i] = cos(ph);
      im[i] = sin(ph);
    }
  }
}

/* ------------------------------------------------------------------------------
 * Operators: the CPU twins of src/hamiltonian.cu.
 * ---------------------------------------------------------------------------- */

/* cpu_apply_hamiltonian, src/hamiltonian.cu:188-221. */
void orc_apply(const orc_ham* h, const double* ir, const double* ii, double* orr, double* oi)
{
  int N = h->n, z = h->max_neighbor;
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    double tr = h->potential[n] * ir[n];
    double ti = h->potential[n] * ii[n];
    for (int m = 0; m < h->neighbor_number[n]; ++m) {
      long e = (long)n * z + m;
      int j = h->neighbor_list[e];
      double a = h->hopping_real[e], b = h->hopping_imag[e];
      double c = ir[j], d = ii[j];
      tr += a * c - b * d;
      ti += a * d + b * c;
    }
    tr /= h->energy_max;
    ti /= h->energy_max;
    orr[n] = tr;
    oi[n] = ti;
  }
}

/* cpu_apply_commutator, src/hamiltonian.cu:273-305. */
void orc_apply_commutator(const orc_ham* h, const double* ir, const double* ii, double* orr,
                          double* oi)
{
  int N = h->n, z = h->max_neighbor;
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    double tr = 0.0, ti = 0.0;
    for (int m = 0; m < h->neighbor_number[n]; ++m) {
      long e = (long)n * z + m;
      int j = h->neighbor_list[e];
      double a = h->hopping_real[e], b = h->hopping_imag[e];
      double c = ir[j], d = ii[j];
      double x = h->xx[e];
      tr -= (a * c - b * d) * x;
      ti -= (a * d + b * c) * x;
    }
    orr[n] = tr / h->energy_max;
    oi[n] = ti / h->energy_max;
  }
}

/* cpu_apply_current, src/hamiltonian.cu:354-384. */
void orc_apply_current(const orc_ham* h, const double* ir, const double* ii, double* orr,
                       double* oi)
{
  int N = h->n, z = h->max_neighbor;
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    double tr = 0.0, ti = 0.0;
    for (int m = 0; m < h->neighbor_number[n]; ++m) {
      long e = (long)n * z + m;
      int j = h->neighbor_list[e];
      double a = h->hopping_real[e], b = h->hopping_imag[e];
      double c = ir[j], d = ii[j];
      tr += (a * c - b * d) * h->xx[e];
      ti += (a * d + b * c) * h->xx[e];
    }
    orr[n] = +ti;
    oi[n] = -tr;
  }
}

/* cpu_kernel_polynomial, src/hamiltonian.cu:927-967. */
void orc_kernel_polynomial(const orc_ham* h, const double* s0r, const double* s0i,
                           const double* s1r, const double* s1i, double* s2r, double* s2i)
{
  int N = h->n, z = h->max_neighbor;
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    double tr = h->potential[n] * s1r[n];
    double ti = h->potential[n] * s1i[n];
    for (int m = 0; m < h->neighbor_number[n]; ++m) {
      long e = (long)n * z + m;
      int j = h->neighbor_list[e];
      double a = h->hopping_real[e], b = h->hopping_imag[e];
      double c = s1r[j], d = s1i[j];
      tr += a * c - b * d;
      ti += a * d + b * c;
    }
    tr /= h->energy_max;
    ti /= h->energy_max;
    tr = 2.0 * tr - s0r[n];
    ti = 2.0 * ti - s0i[n];
    s2r[n] = tr;
    s2i[n] = ti;
  }
}

/* cpu_chebyshev_01, src/hamiltonian.cu:425-444. */
void orc_chebyshev_01(int N, const double* s0r, const double* s0i, const double* s1r,
                      const double* s1i, double* sr, double* si, double b0, double b1,
                      int direction)
{
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    double bessel_0 = b0;
    double bessel_1 = b1 * direction;
    sr[n] = bessel_0 * s0r[n] + bessel_1 * s1i[n];
    si[n] = bessel_0 * s0i[n] - bessel_1 * s1r[n];
  }
}

/* The four accumulation labels shared by src/hamiltonian.cu:498-523 and :727-752. */
static inline void orc_accumulate(double* sr, double* si, double b, double tr, double ti,
                                  int label)
{
  switch (label) {
    case 1:
      *sr += b * tr;
      *si += b * ti;
      break;
    case 2:
      *sr -= b * tr;
      *si -= b * ti;
      break;
    case 3:
      *sr += b * ti;
      *si -= b * tr;
      break;
    case 4:
      *sr -= b * ti;
      *si += b * tr;
      break;
  }
}

/* cpu_chebyshev_2, src/hamiltonian.cu:531-596. */
void orc_chebyshev_2(const orc_ham* h, const double* s0r, const double* s0i, const double* s1r,
                     const double* s1i, double* s2r, double* s2i, double* sr, double* si,
                     double bessel_m, int label)
{
  int N = h->n, z = h->max_neighbor;
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    double tr = h->potential[n] * s1r[n];
    double ti = h->potential[n] * s1i[n];
    for (int m = 0; m < h->neighbor_number[n]; ++m) {
      long e = (long)n * z + m;
      int j = h->neighbor_list[e];
      double a = h->hopping_real[e], b = h->hopping_imag[e];
      double c = s1r[j], d = s1i[j];
      tr += a * c - b * d;
      ti += a * d + b * c;
    }
    tr /= h->energy_max;
    ti /= h->energy_max;
    tr = 2.0 * tr - s0r[n];
    ti = 2.0 * ti - s0i[n];
    orc_accumulate(&sr[n], &si[n], bessel_m, tr, ti, label);
    s2r[n] = tr;
    s2i[n] = ti;
  }
}

/* cpu_chebyshev_1x, src/hamiltonian.cu:635-649. */
void orc_chebyshev_1x(int N, const double* s1xr, const double* s1xi, double* sr, double* si,
                      double b1)
{
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    sr[n] = +b1 * s1xi[n];
    si[n] = -b1 * s1xr[n];
  }
}

/* cpu_chebyshev_2x, src/hamiltonian.cu:760-853. */
void orc_chebyshev_2x(const orc_ham* h, const double* s0r, const double* s0i,
                      const double* s0xr, const double* s0xi, const double* s1r,
                      const double* s1i, const double* s1xr, const double* s1xi, double* s2r,
                      double* s2i, double* s2xr, double* s2xi, double* sr, double* si,
                      double bessel_m, int label)
{
  int N = h->n, z = h->max_neighbor;
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; ++n) {
    double p = h->potential[n];
    double tr = p * s1r[n];
    double ti = p * s1i[n];
    double txr = p * s1xr[n];
    double txi = p * s1xi[n];
    for (int m = 0; m < h->neighbor_number[n]; ++m) {
      long e = (long)n * z + m;
      int j = h->neighbor_list[e];
      double a = h->hopping_real[e], b = h->hopping_imag[e];
      double c = s1r[j], d = s1i[j];
      tr += a * c - b * d;
      ti += a * d + b * c;
      double cx = s1xr[j], dx = s1xi[j];
      txr += a * cx - b * dx;
      txi += a * dx + b * cx;
      double x = h->xx[e];
      txr -= (a * c - b * d) * x;
      txi -= (a * d + b * c) * x;
    }
    tr /= h->energy_max;
    ti /= h->energy_max;
    tr = 2.0 * tr - s0r[n];
    ti = 2.0 * ti - s0i[n];
    s2r[n] = tr;
    s2i[n] = ti;
    txr /= h->energy_max;
    txi /= h->energy_max;
    txr = 2.0 * txr - s0xr[n];
    txi = 2.0 * txi - s0xi[n];
    s2xr[n] = txr;
    s2xi[n] = txi;
    orc_accumulate(&sr[n], &si[n], bessel_m, txr, txi, label);
  }
}

/* cpu_find_inner_product_1 + cpu_find_inner_product_2, src/vector.cu:300-329 and
 * :403-423, for one moment. */
void orc_inner_product(int N, const double* ar, const double* ai, const double* cr,
                       const double* ci, double* re, double* im)
{
  int grid = (N - 1) / ORC_BLOCK + 1;
  double* pr = (double*)malloc(sizeof(double) * grid);
  double* pi = (double*)malloc(sizeof(double) * grid);
#pragma omp parallel for schedule(static)
  for (int g = 0; g < grid; ++g) {
    double sr = 0.0, si = 0.0;
    for (int k = 0; k < ORC_BLOCK; ++k) {
      int n = g * ORC_BLOCK + k;
      if (n < N) {
        double a = ar[n], b = ai[n], c = cr[n], d = ci[n];
        sr += (a * c + b * d);
        si += (b * c - a * d);
      }
    }
    pr[g] = sr;
    pi[g] = si;
  }
  double sr = 0.0, si = 0.0;
  for (int g = 0; g < grid; ++g) {
    sr += pr[g];
    si += pi[g];
  }
  *re = sr;
  *im = si;
  free(pr);
  free(pi);
}

/* ------------------------------------------------------------------------------
 * Algorithms: src/sigma.cu.
 * ---------------------------------------------------------------------------- */

typedef struct {
  double* r;
  double* i;
} orc_vec;

static orc_vec orc_vec_new(int n)
{
  orc_vec v;
  v.r = (double*)calloc((size_t)n, sizeof(double));
  v.i = (double*)calloc((size_t)n, sizeof(double));
  return v;
}

static orc_vec orc_vec_copy(int n, const double* r, const double* i)
{
  orc_vec v = orc_vec_new(n);
  memcpy(v.r, r, sizeof(double) * n);
  memcpy(v.i, i, sizeof(double) * n);
  return v;
}

static void orc_vec_free(orc_vec v)
{
  free(v.r);
  free(v.i);
}

static void orc_vec_swap(orc_vec* a, orc_vec* b)
{
  orc_vec t = *a;
  *a = *b;
  *b = t;
}

/* find_moments_chebyshev, src/sigma.cu:33-61. */
void orc_find_moments(const orc_ham* h, int M, const double* lr, const double* li,
                      const double* rr, const double* ri, double* mu_re, double* mu_im)
{
  int n = h->n;
  orc_vec s0 = orc_vec_copy(n, rr, ri), s1 = orc_vec_new(n), s2 = orc_vec_new(n);
  orc_inner_product(n, s0.r, s0.i, lr, li, &mu_re[0], &mu_im[0]);
  if (M > 1) {
    orc_apply(h, s0.r, s0.i, s1.r, s1.i);
    orc_inner_product(n, s1.r, s1.i, lr, li, &mu_re[1], &mu_im[1]);
  }
  for (int m = 2; m < M; ++m) {
    orc_kernel_polynomial(h, s0.r, s0.i, s1.r, s1.i, s2.r, s2.i);
    orc_inner_product(n, s2.r, s2.i, lr, li, &mu_re[m], &mu_im[m]);
    orc_vec_swap(&s0, &s1);
    orc_vec_swap(&s1, &s2);
  }
  orc_vec_free(s0);
  orc_vec_free(s1);
  orc_vec_free(s2);
}

/* Jackson damping, src/sigma.cu:76-86. */
void orc_apply_damping(int M, double* mu_re, double* mu_im)
{
  for (int k = 0; k < M; ++k) {
    double factor = 1.0 / (M + 1);
    double damping = (1 - k * factor) * cos(k * ORC_PI * factor) +
                     sin(k * ORC_PI * factor) * factor / tan(ORC_PI * factor);
    mu_re[k] *= damping;
    mu_im[k] *= damping;
  }
}

/* perform_chebyshev_summation, src/sigma.cu:89-110. */
void orc_chebyshev_summation(int M, const double* mu, int n_energy, const double* energy,
                             double energy_max, double volume, double* out)
{
  for (int s1 = 0; s1 < n_energy; ++s1) {
    double es = energy[s1] / energy_max;
    double c0 = 1.0, c1 = es, c2;
    double temp = mu[1] * c1;
    for (int s2 = 2; s2 < M; ++s2) {
      c2 = 2.0 * es * c1 - c0;
      c0 = c1;
      c1 = c2;
      temp += mu[s2] * c2;
    }
    temp *= 2.0;
    temp += mu[0];
    temp *= 2.0 / (ORC_PI * volume);
    temp /= sqrt(1.0 - es * es);
    out[s1] = temp / energy_max;
  }
}

int orc_bessel_cut(double dt)
{
  int m = 2;
  for (; m < 1000000; ++m) {
    double b = jn(m, dt);
    if (b < 1.0e-15 && b > -1.0e-15)
      break;
  }
  return m;
}

/* evolve, src/sigma.cu:116-151. */
void orc_evolve(const orc_ham* h, int direction, double dt, double* re, double* im)
{
  int n = h->n;
  orc_vec s0 = orc_vec_copy(n, re, im), s1 = orc_vec_new(n), s2 = orc_vec_new(n);
  orc_apply(h, re, im, s1.r, s1.i);
  double b0 = j0(dt);
  double b1 = 2.0 * j1(dt);
  orc_chebyshev_01(n, s0.r, s0.i, s1.r, s1.i, re, im, b0, b1, direction);
  for (int m = 2; m < 1000000; ++m) {
    double bm = jn(m, dt);
    if (bm < 1.0e-15 && bm > -1.0e-15)
      break;
    bm *= 2.0;
    int label, r = m % 4;
    if (r == 0)
      label = 1;
    else if (r == 2)
      label = 2;
    else if ((r == 1 && direction == 1) || (r == 3 && direction == -1))
      label = 3;
    else
      label = 4;
    orc_chebyshev_2(h, s0.r, s0.i, s1.r, s1.i, s2.r, s2.i, re, im, bm, label);
    orc_vec_swap(&s0, &s1);
    orc_vec_swap(&s1, &s2);
  }
  orc_vec_free(s0);
  orc_vec_free(s1);
  orc_vec_free(s2);
}

/* evolvex, src/sigma.cu:157-200. */
void orc_evolvex(const orc_ham* h, int direction, double dt, double* re, double* im)
{
  int n = h->n;
  orc_vec s0 = orc_vec_copy(n, re, im), s0x = orc_vec_new(n);
  orc_vec s1 = orc_vec_new(n), s1x = orc_vec_new(n);
  orc_vec s2 = orc_vec_new(n), s2x = orc_vec_new(n);
  orc_apply(h, re, im, s1.r, s1.i);
  orc_apply_commutator(h, re, im, s1x.r, s1x.i);
  double b1 = 2.0 * j1(dt);
  orc_chebyshev_1x(n, s1x.r, s1x.i, re, im, b1);
  for (int m = 2; m <= 1000000; ++m) {
    double bm = jn(m, dt);
    if (bm < 1.0e-15 && bm > -1.0e-15)
      break;
    bm *= 2.0;
    int label, r = m % 4;
    if (r == 1)
      label = 3;
    else if (r == 3)
      label = 4;
    else if ((r == 0 && direction == 1) || (r == 2 && direction == -1))
      label = 1;
    else
      label = 2;
    orc_chebyshev_2x(h, s0.r, s0.i, s0x.r, s0x.i, s1.r, s1.i, s1x.r, s1x.i, s2.r, s2.i, s2x.r,
                     s2x.i, re, im, bm, label);
    orc_vec_swap(&s0, &s1);
    orc_vec_swap(&s1, &s2);
    orc_vec_swap(&s0x, &s1x);
    orc_vec_swap(&s1x, &s2x);
  }
  orc_vec_free(s0);
  orc_vec_free(s0x);
  orc_vec_free(s1);
  orc_vec_free(s1x);
  orc_vec_free(s2);
  orc_vec_free(s2x);
}

/* The moment sets of find_vac, src/sigma.cu:278-327 (the .out writing aside). */
void orc_vac_moments(const orc_ham* h, int M, int n_steps, const double* time_step,
                     const double* pr, const double* pi, double* mu_re, double* mu_im)
{
  int n = h->n;
  orc_vec left = orc_vec_copy(n, pr, pi), left_copy = orc_vec_new(n);
  orc_vec right = orc_vec_copy(n, pr, pi);
  orc_apply_current(h, left.r, left.i, right.r, right.i);
  for (int m = 0; m < n_steps; ++m) {
    orc_apply_current(h, left.r, left.i, left_copy.r, left_copy.i);
    orc_find_moments(h, M, right.r, right.i, left_copy.r, left_copy.i, mu_re + (size_t)m * M,
                     mu_im + (size_t)m * M);
    if (m < n_steps - 1) {
      double dts = time_step[m] * h->energy_max;
      orc_evolve(h, -1, dts, left.r, left.i);
      orc_evolve(h, -1, dts, right.r, right.i);
    }
  }
  orc_vec_free(left);
  orc_vec_free(left_copy);
  orc_vec_free(right);
}

/* The moment sets of find_msd, src/sigma.cu:331-391. */
void orc_msd_moments(const orc_ham* h, int M, int n_steps, const double* time_step,
                     const double* pr, const double* pi, double* mu_re, double* mu_im)
{
  int n = h->n;
  orc_vec state = orc_vec_copy(n, pr, pi), state_x = orc_vec_copy(n, pr, pi);
  orc_vec copy = orc_vec_new(n);
  double dts = time_step[0] * h->energy_max;
  orc_evolve(h, 1, dts, state.r, state.i);
  orc_evolvex(h, 1, dts, state_x.r, state_x.i);
  for (int m = 0; m < n_steps; ++m) {
    orc_find_moments(h, M, state_x.r, state_x.i, state_x.r, state_x.i, mu_re + (size_t)m * M,
                     mu_im + (size_t)m * M);
    if (m < n_steps - 1) {
      dts = time_step[m + 1] * h->energy_max;
      memcpy(copy.r, state.r, sizeof(double) * n);
      memcpy(copy.i, state.i, sizeof(double) * n);
      orc_evolvex(h, 1, dts, copy.r, copy.i);
      orc_evolve(h, 1, dts, state_x.r, state_x.i);
      for (int k = 0; k < n; ++k) {
        state_x.r[k] += copy.r[k];
        state_x.i[k] += copy.i[k];
      }
      orc_evolve(h, 1, dts, state.r, state.i);
    }
  }
  orc_vec_free(state);
  orc_vec_free(state_x);
  orc_vec_free(copy);
}
