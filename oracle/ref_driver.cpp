// Test infrastructure only (never linked into the product): a driver that links the
// reference's own CPU objects (src/*.cu built with -DCPU_ONLY -DDEBUG, see Makefile), or
// its GPU objects (target ref_gpu, the same source compiled by nvcc),
// and writes their raw results at full precision, so the parity tests can pin the
// C restatement (lsqt_oracle.c) and the CUDA library against the reference itself.
//
// Usage:
//   ref_driver ell     DIR OUT.bin [dseed pseed]  Model ELL arrays (src/model.h:51-60)
//   ref_driver ops     DIR OUT.bin DT [dseed pseed]  operator outputs on the phase vector
//   ref_driver moments DIR OUT.txt [dseed pseed]  mu_m of find_moments_chebyshev (%.17g)
//   ref_driver vacmom  DIR OUT.txt [dseed pseed]  per-step VAC moments (src/sigma.cu:278-327)
//   ref_driver msdmom  DIR OUT.txt [dseed pseed]  per-step MSD moments (src/sigma.cu:331-391)
//   ref_driver time    DIR NMOM REPS [dseed pseed]  seconds per find_moments_chebyshev call
//
// Seeds: without dseed/pseed the single reference stream (seed 12345678, src/model.cu:34)
// is used as is. With them, the Anderson potential is redrawn by the reference's own
// Anderson::add_disorder on a generator reseeded with dseed (valid when no vacancy or
// charged-impurity disorder is configured), and the phases are drawn by the reference's
// Model::initialize_state on a generator reseeded with pseed.

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#define private public  // reach Model::generator for the split-seed mode
#include "model.h"
#undef private
#include "hamiltonian.h"
#include "vector.h"

// Defined with external linkage in src/sigma.cu but not declared in src/sigma.h.
void find_moments_chebyshev(Model&, Hamiltonian&, Vector&, Vector&, Vector&);
void evolve(Model&, int, real, Hamiltonian&, Vector&);
void evolvex(Model&, int, real, Hamiltonian&, Vector&);

static void reseed_disorder(Model& model, long dseed)
{
  if (dseed < 0)
    return;
  if (model.has_vacancy_disorder || model.charge.has) {
    std::fprintf(stderr, "split seeds need a model without vacancies/charges\n");
    std::exit(2);
  }
  model.generator.seed((unsigned)dseed);
  if (model.anderson.has_disorder)
    model.anderson.add_disorder(model.number_of_atoms, model.generator, model.potential);
}

static void reseed_phase(Model& model, long pseed)
{
  if (pseed >= 0)
    model.generator.seed((unsigned)pseed);
}

static void write_vec(FILE* f, Vector& v, int n)
{
  std::vector<double> re(n), im(n);
  v.copy_to_host(re.data(), im.data());
  std::fwrite(re.data(), sizeof(double), n, f);
  std::fwrite(im.data(), sizeof(double), n, f);
}

static void write_moments(FILE* f, Vector& out, int M)
{
  std::vector<double> re(M), im(M);
  out.copy_to_host(re.data(), im.data());
  for (int m = 0; m < M; ++m)
    std::fprintf(f, "%.17g %.17g\n", re[m], im[m]);
}

int main(int argc, char** argv)
{
  if (argc < 4) {
    std::fprintf(stderr, "usage: ref_driver MODE DIR OUT [..]\n");
    return 2;
  }
  std::string mode = argv[1];
  std::string dir = argv[2];
  int extra = (mode == "ops" || mode == "time") ? 1 : 0;
  long dseed = -1, pseed = -1;
  if (argc >= 6 + extra) {
    dseed = std::atol(argv[4 + extra]);
    pseed = std::atol(argv[5 + extra]);
  }

  Model model(dir);
  reseed_disorder(model, dseed);
  int n = model.number_of_atoms;
  int z = model.max_neighbor;

  if (mode == "ell") {
    FILE* f = std::fopen(argv[3], "wb");
    int hdr[2] = {n, z};
    double meta[2] = {model.energy_max, model.volume};
    std::fwrite(hdr, sizeof(int), 2, f);
    std::fwrite(meta, sizeof(double), 2, f);
    std::vector<int> nl((size_t)n * z, 0);
    std::vector<double> hr((size_t)n * z, 0.0), hi((size_t)n * z, 0.0), xx((size_t)n * z, 0.0);
    for (int i = 0; i < n; ++i)
      for (int m = 0; m < model.neighbor_number[i]; ++m) {
        size_t k = (size_t)i * z + m;
        nl[k] = model.neighbor_list[k];
        hr[k] = model.hopping_real[k];
        hi[k] = model.hopping_imag[k];
        xx[k] = model.xx[k];
      }
    std::fwrite(model.neighbor_number, sizeof(int), n, f);
    std::fwrite(nl.data(), sizeof(int), nl.size(), f);
    std::fwrite(model.potential, sizeof(double), n, f);
    std::fwrite(hr.data(), sizeof(double), hr.size(), f);
    std::fwrite(hi.data(), sizeof(double), hi.size(), f);
    std::fwrite(xx.data(), sizeof(double), xx.size(), f);
    std::fclose(f);
    return 0;
  }

  Hamiltonian H(model);
  Vector phi(n);
  reseed_phase(model, pseed);
  model.initialize_state(phi, -1);

  if (mode == "ops") {
    real dt = std::atof(argv[4]);
    FILE* f = std::fopen(argv[3], "wb");
    write_vec(f, phi, n);
    Vector h1(n), cx(n), cur(n), t2(n);
    H.apply(phi, h1);
    write_vec(f, h1, n);
    H.apply_commutator(phi, cx);
    write_vec(f, cx, n);
    H.apply_current(phi, cur);
    write_vec(f, cur, n);
    H.kernel_polynomial(phi, h1, t2);
    write_vec(f, t2, n);
    for (int dir = 1; dir >= -1; dir -= 2) {
      Vector s(phi);
      evolve(model, dir, dt, H, s);
      write_vec(f, s, n);
    }
    for (int dir = 1; dir >= -1; dir -= 2) {
      Vector s(phi);
      evolvex(model, dir, dt, H, s);
      write_vec(f, s, n);
    }
    std::fclose(f);
    return 0;
  }

  int M = model.number_of_moments;
  if (mode == "moments") {
    Vector out(M);
    find_moments_chebyshev(model, H, phi, phi, out);
    FILE* f = std::fopen(argv[3], "w");
    write_moments(f, out, M);
    std::fclose(f);
    return 0;
  }

  if (mode == "vacmom") {
    // The moment sets of find_vac (src/sigma.cu:278-327), one block of M lines per step.
    FILE* f = std::fopen(argv[3], "w");
    Vector left(phi), left_copy(n), right(phi), out(M);
    H.apply_current(left, right);
    for (int m = 0; m < model.number_of_steps_correlation; ++m) {
      H.apply_current(left, left_copy);
      find_moments_chebyshev(model, H, right, left_copy, out);
      write_moments(f, out, M);
      if (m < model.number_of_steps_correlation - 1) {
        real dts = model.time_step[m] * model.energy_max;
        evolve(model, -1, dts, H, left);
        evolve(model, -1, dts, H, right);
      }
    }
    std::fclose(f);
    return 0;
  }

  if (mode == "msdmom") {
    // The moment sets of find_msd (src/sigma.cu:331-391).
    FILE* f = std::fopen(argv[3], "w");
    Vector state(phi), state_x(phi), state_copy(n), out(M);
    real dts = model.time_step[0] * model.energy_max;
    evolve(model, 1, dts, H, state);
    evolvex(model, 1, dts, H, state_x);
    for (int m = 0; m < model.number_of_steps_correlation; ++m) {
      find_moments_chebyshev(model, H, state_x, state_x, out);
      write_moments(f, out, M);
      if (m < model.number_of_steps_correlation - 1) {
        dts = model.time_step[m + 1] * model.energy_max;
        state_copy.copy(state);
        evolvex(model, 1, dts, H, state_copy);
        evolve(model, 1, dts, H, state_x);
        state_x.add(state_copy);
        evolve(model, 1, dts, H, state);
      }
    }
    std::fclose(f);
    return 0;
  }

  if (mode == "time") {
    // Seconds per call of the reference's moment loop at NMOM moments (wall clock).
    model.number_of_moments = std::atoi(argv[3]);
    int reps = std::atoi(argv[4]);
    Vector out(model.number_of_moments);
    std::printf("{\"n\": %d, \"moments\": %d, \"reps_s\": [", n, model.number_of_moments);
    for (int r = 0; r < reps; ++r) {
      auto t0 = std::chrono::steady_clock::now();
      find_moments_chebyshev(model, H, phi, phi, out);
#ifdef __CUDACC__
      cudaDeviceSynchronize();  // the GPU build's launches are asynchronous
#endif
      auto t1 = std::chrono::steady_clock::now();
      std::printf("%s%.6f", r ? ", " : "", std::chrono::duration<double>(t1 - t0).count());
      std::fflush(stdout);
    }
    std::printf("]}\n");
    return 0;
  }

  std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
  return 2;
}
