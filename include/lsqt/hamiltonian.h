// Replaces class Hamiltonian (src/hamiltonian.h:25-54): the ELL operator on the
// device. Each method issues one of the library's sm_100a kernels.
#pragma once

#include "gpuqt.h"
#include "lsqt/common.h"

class Vector;
class Model;

class Hamiltonian
{
public:
  // Uploads the model's ELL arrays and, like the reference, takes them over: the
  // Model's neighbor_number, neighbor_list, potential, hopping_real, hopping_imag
  // and xx host arrays are freed (and set to null) here.
  Hamiltonian(Model& model);
  ~Hamiltonian();
  Hamiltonian(const Hamiltonian&) = delete;
  Hamiltonian& operator=(const Hamiltonian&) = delete;
  void apply(Vector& input, Vector& output);
  void apply_commutator(Vector& input, Vector& output);
  void apply_current(Vector& input, Vector& output);
  void kernel_polynomial(Vector& state_0, Vector& state_1, Vector& state_2);
  void chebyshev_01(Vector& state_0, Vector& state_1, Vector& state, real bessel_0,
                    real bessel_1, int direction);
  void chebyshev_2(Vector& state_0, Vector& state_1, Vector& state_2, Vector& state,
                   real bessel_m, int label);
  void chebyshev_1x(Vector& input, Vector& output, real bessel_1);
  void chebyshev_2x(Vector& state_0, Vector& state_0x, Vector& state_1, Vector& state_1x,
                    Vector& state_2, Vector& state_2x, Vector& state, real bessel_m, int label);

  gqt_ham* handle() { return h; }

private:
  gqt_ham* h = nullptr;
};
