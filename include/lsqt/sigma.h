// Replaces src/sigma.h and the non-header functions of src/sigma.cu.
#pragma once

#include "lsqt/common.h"

class Model;
class Hamiltonian;
class Vector;

void find_dos(Model&, Hamiltonian&, Vector&, int);
void find_vac0(Model&, Hamiltonian&, Vector&);
void find_vac(Model&, Hamiltonian&, Vector&);
void find_msd(Model&, Hamiltonian&, Vector&);
void find_spin_polarization(Model&, Hamiltonian&, Vector&);

// Defined with external linkage in the reference (src/sigma.cu:33, :65, :89, :116,
// :157) and declared here.
void find_moments_chebyshev(Model& model, Hamiltonian& H, Vector& state_left,
                            Vector& state_right, Vector& output);
void apply_damping(Model& model, real* inner_product_real, real* inner_product_imag);
void perform_chebyshev_summation(Model& model, real* inner_product_real,
                                 real* inner_product_imag, real* correlation_function);
void evolve(Model& model, int direction, real time_step_scaled, Hamiltonian& H,
            Vector& state_in);
void evolvex(Model& model, int direction, real time_step_scaled, Hamiltonian& H,
             Vector& state_in);
