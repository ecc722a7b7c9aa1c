// Plain-old-data layouts shared by host code and CUDA kernels.
#pragma once

#include <vector>

namespace napmo {

// Radial transform parameters for device-side evaluation (t <-> r).
enum RTKind : int {
  kRTIdentity = 0,
  kRTLinear = 1,
  kRTExp = 2,
  kRTShiftedExp = 3,
  kRTPower = 4,
  kRTChebyshev = 5,
};

struct RTParams {
  int kind;
  int npoint;
  double p0, p1, p2;  // linear/exp: rmin, alpha; shifted: r0, rshift, alpha;
                      // power: rmin, power; chebyshev: radii, z
};

// Device mirror of a molecular grid.  Points are stored structure-of-arrays so
// that a warp reading 32 consecutive points issues 3 coalesced 256-byte loads.
struct DeviceGrid {
  int npoint = 0;
  int ncenter = 0;
  double *x = nullptr, *y = nullptr, *z = nullptr;
  double *w = nullptr;        // atomic quadrature weight w_ang * w_rad
  double *wb = nullptr;       // Becke partition weight
  double *origin = nullptr;   // [ncenter][3]
  double *radii = nullptr;    // [ncenter]
  int *atom_offset = nullptr; // [ncenter + 1]
};

// Cartesian GTO basis packed by shell.  A shell is a run of consecutive
// contracted functions sharing centre, exponents and total angular momentum;
// the primitive exponentials are evaluated once per shell and point.
//   shell_info[s*6 + {0..5}] = first function, #components, first primitive,
//                              #primitives, first coefficient, L
//   coef[first_coef + c*nprim + k] = coefficient of primitive k in component c
//                                    (contraction norm x primitive norm x c_k)
//   func_l[f*3 + {0,1,2}] = Cartesian exponents of function f
//   shell_center[s*4 + {0,1,2,3}] = centre x, y, z and the smallest exponent
struct HostBasisPack {
  int nfunc = 0, nshell = 0, max_nprim = 0, max_l = 0;
  std::vector<int> shell_info;
  std::vector<double> shell_center;
  std::vector<double> prim_zeta;
  std::vector<double> coef;
  std::vector<int> func_l;
};

struct DeviceBasis {
  int nfunc = 0, nshell = 0, max_nprim = 0, max_l = 0;
  int *shell_info = nullptr;
  double *shell_center = nullptr;
  double *prim_zeta = nullptr;
  double *coef = nullptr;
  int *func_l = nullptr;
};

}  // namespace napmo
