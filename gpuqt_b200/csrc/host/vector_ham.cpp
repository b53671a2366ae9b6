// Vector and Hamiltonian: the reference's device classes (src/vector.cu,
// src/hamiltonian.cu) as thin owners of C-ABI handles.
#include <vector>

#include "gpuqt.h"
#include "lsqt/hamiltonian.h"
#include "lsqt/model.h"
#include "lsqt/vector.h"

using gqt_host::check;

int Vector::default_precision = GQT_FP64;
int Vector::moment_precision = GQT_FP64;

Vector::Vector(int n_) : Vector(n_, default_precision) {}

Vector::Vector(int n_, int precision) : n(n_)
{
  check(gqt_vec_create(n_, 1, precision, &v), "Vector::Vector");
}

Vector::Vector(Vector& original) : n(original.n)
{
  check(gqt_vec_clone(original.v, &v), "Vector::Vector(Vector&)");
}

Vector::~Vector() { gqt_vec_destroy(v); }

void Vector::add(Vector& other) { check(gqt_vec_add(v, other.v), "Vector::add"); }

void Vector::copy(Vector& other) { check(gqt_vec_copy(v, other.v), "Vector::copy"); }

void Vector::apply_sz(Vector& other) { check(gqt_vec_apply_sz(v, other.v), "Vector::apply_sz"); }

void Vector::copy_from_host(real* re, real* im)
{
  check(gqt_vec_upload(v, re, im), "Vector::copy_from_host");
}

void Vector::copy_to_host(real* re, real* im)
{
  check(gqt_vec_download(v, re, im), "Vector::copy_to_host");
}

void Vector::swap(Vector& other) { check(gqt_vec_swap(v, other.v), "Vector::swap"); }

void Vector::inner_product_1(int, Vector& other, Vector& target, int offset)
{
  check(gqt_inner_product_into(v, other.v, target.v, offset), "Vector::inner_product_1");
}

void Vector::inner_product_2(int number_of_atoms, int number_of_moments, Vector& target)
{
  const int segment = (number_of_atoms - 1) / 512 + 1;  // grid size of src/vector.cu:333
  check(gqt_vec_segment_sum(v, segment, number_of_moments, target.v),
        "Vector::inner_product_2");
}

Hamiltonian::Hamiltonian(Model& model)
{
  gqt_ell_desc d;
  d.n = model.number_of_atoms;
  d.max_neighbor = model.max_neighbor;
  d.energy_max = model.energy_max;
  d.neighbor_number = model.neighbor_number;
  d.neighbor_list = model.neighbor_list;
  d.potential = model.potential;
  d.hopping_real = model.hopping_real;
  d.hopping_imag = model.hopping_imag;
  d.xx = model.xx;
  check(gqt_ham_create(&d, &h), "Hamiltonian::Hamiltonian");
  // The reference hands the host arrays over to the Hamiltonian, which frees them
  // (src/hamiltonian.cu:43-88).
  delete[] model.neighbor_number;
  delete[] model.neighbor_list;
  delete[] model.potential;
  delete[] model.hopping_real;
  delete[] model.hopping_imag;
  delete[] model.xx;
  model.neighbor_number = nullptr;
  model.neighbor_list = nullptr;
  model.potential = nullptr;
  model.hopping_real = nullptr;
  model.hopping_imag = nullptr;
  model.xx = nullptr;
}

Hamiltonian::~Hamiltonian() { gqt_ham_destroy(h); }

void Hamiltonian::apply(Vector& in, Vector& out)
{
  check(gqt_apply(h, in.handle(), out.handle()), "Hamiltonian::apply");
}

void Hamiltonian::apply_commutator(Vector& in, Vector& out)
{
  check(gqt_apply_commutator(h, in.handle(), out.handle()), "Hamiltonian::apply_commutator");
}

void Hamiltonian::apply_current(Vector& in, Vector& out)
{
  check(gqt_apply_current(h, in.handle(), out.handle()), "Hamiltonian::apply_current");
}

void Hamiltonian::kernel_polynomial(Vector& s0, Vector& s1, Vector& s2)
{
  check(gqt_kernel_polynomial(h, s0.handle(), s1.handle(), s2.handle()),
        "Hamiltonian::kernel_polynomial");
}

void Hamiltonian::chebyshev_01(Vector& s0, Vector& s1, Vector& s, real b0, real b1, int dir)
{
  check(gqt_chebyshev_01(h, s0.handle(), s1.handle(), s.handle(), b0, b1, dir),
        "Hamiltonian::chebyshev_01");
}

void Hamiltonian::chebyshev_2(Vector& s0, Vector& s1, Vector& s2, Vector& s, real b, int label)
{
  check(gqt_chebyshev_2(h, s0.handle(), s1.handle(), s2.handle(), s.handle(), b, label),
        "Hamiltonian::chebyshev_2");
}

void Hamiltonian::chebyshev_1x(Vector& in, Vector& out, real b1)
{
  check(gqt_chebyshev_1x(h, in.handle(), out.handle(), b1), "Hamiltonian::chebyshev_1x");
}

void Hamiltonian::chebyshev_2x(Vector& s0, Vector& s0x, Vector& s1, Vector& s1x, Vector& s2,
                               Vector& s2x, Vector& s, real b, int label)
{
  check(gqt_chebyshev_2x(h, s0.handle(), s0x.handle(), s1.handle(), s1x.handle(), s2.handle(),
                         s2x.handle(), s.handle(), b, label),
        "Hamiltonian::chebyshev_2x");
}
