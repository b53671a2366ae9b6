// Replaces class Vector (src/vector.h:23-47). The two device buffers real_part /
// imag_part of the reference become one interleaved complex buffer owned by a
// gqt_vec handle; swap exchanges buffers without copying, as in the reference.
#pragma once

#include "gpuqt.h"
#include "lsqt/common.h"

class Vector
{
public:
  Vector(int n);                     // zero vector of n sites (src/vector.cu:61-70)
  Vector(int n, int precision);      // explicit arithmetic form (GQT_FP64 / GQT_FP32)
  Vector(Vector& original);          // deep copy (src/vector.cu:92-105)
  ~Vector();
  Vector& operator=(const Vector&) = delete;
  void add(Vector& other);
  void copy(Vector& other);
  void apply_sz(Vector& other);
  void copy_from_host(real* other_real, real* other_imag);
  void copy_to_host(real* target_real, real* target_imag);
  void swap(Vector& other);
  // Stage 1 of <other|this>: writes the full FP64 sum to element `offset` of target
  // (the reference writes per-block partials from there on; their segment sum is
  // the same moment). Stage 2 sums each segment of ceil(n/512) elements of this
  // vector into target[m] (src/vector.cu:331-344, :425-436).
  void inner_product_1(int number_of_atoms, Vector& other, Vector& target, int offset);
  void inner_product_2(int number_of_atoms, int number_of_moments, Vector& target);

  gqt_vec* handle() { return v; }
  int size() const { return n; }
  // Arithmetic form of vectors built with Vector(int); GQT_FP64 unless changed.
  static int default_precision;
  // Arithmetic form of the Chebyshev recurrence in find_moments_chebyshev (GQT_FP32
  // for the FP32-storage form); the states themselves keep default_precision, so
  // time-evolved states stay FP64 across evolution steps.
  static int moment_precision;

private:
  gqt_vec* v = nullptr;
  int n = 0;
};
