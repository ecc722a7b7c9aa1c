// The wave-function record shared with Python: field-for-field the layout of
// nAPMO's `struct wf` (src/wavefunction/wavefunction.h:20-44), which the
// ctypes Structure PSIB mirrors (napmo/wavefunction/psi_base.py:18-45).
// Matrices are row-major ndim x ndim, owned by Python.
#pragma once

extern "C" {

struct wf {
  double *S;   // overlap
  double *X;   // transformation
  double *T;   // kinetic
  double *V;   // nuclear attraction
  double *H;   // one-particle Hamiltonian
  double *C;   // coefficients
  double *D;   // density
  double *L;   // previous density
  double *G;   // two-particle matrix
  double *J;   // coupling
  double *XC;  // exchange-correlation
  double *F;   // Fock
  double *O;   // orbital energies
  int nbasis;
  int ndim;
  int occupation;
  double eta;
  double kappa;
  double x_factor;
  double xc_energy;
  double energy;
  double rmsd;
};
typedef struct wf WaveFunction;

}  // extern "C"
