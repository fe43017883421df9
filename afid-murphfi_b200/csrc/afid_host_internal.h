// afid_host_internal.h — host-side pieces shared by the host-code translation units.
#pragma once
#include <stdint.h>

#include <map>
#include <new>
#include <string>
#include <vector>

#include "afid_host.h"

// Runs the body of a C entry point so that no C++ exception crosses the C ABI: a failed host
// allocation becomes AFID_E_ALLOC, anything else AFID_E_INVALID.
template <class F>
int afid_guard(F &&body) noexcept {
  try {
    return body();
  } catch (const std::bad_alloc &) {
    return AFID_E_ALLOC;
  } catch (...) {
    return AFID_E_INVALID;
  }
}

// The tables behind afid_tables_t (include/afid_host.h).
struct afid_tables {
  afid_input_t in;
  std::map<std::string, std::vector<double>> arr;
  std::vector<double> tempbp, temptp;
  afid_grid_t grid;
  afid_params_t params;
  double ren, pect, byct, pi, dx, dy, dz;
};

namespace afid_hostd {

// Philox4x32-10 uniform in [0, 1) for counter n and key seed.
double philox_u(uint64_t seed, uint64_t n);
// grid.F90:12-27: faces c[0..nm] and centres m[0..nm-1] of a uniform grid of length len.
void uniform_grid(std::vector<double> &c, std::vector<double> &m, int nm, double len);
// grid.F90:264-307: second-derivative coefficients at the n points x with Dirichlet (fix = 1)
// or Neumann (fix = 0) walls.
void second_derivative_coeff(std::vector<double> &ap3, std::vector<double> &ac3, std::vector<double> &am3,
                             const double *x, int n, double xlen, int fix_up, int fix_low);
// Wall-normal faces of grid type istr3 (0, 1, 2, 3, 4, 6, 7); AFID_E_INVALID otherwise.
int x_grid(int istr3, int nxm, double L, double s, double pi, double schmidt, std::vector<double> &xc);

// Hermite stencils of multires/HermiteInterpolations.F90 (afid_mgrd.cpp).
// :26-57: idx[io], io = 0 .. n_old+1 (Fortran values), the first new index at or past x_old(io).
std::vector<int> interpolation_indices(const std::vector<double> &x_old, const std::vector<double> &x_new,
                                       double x_len);
// :105-164: weights cx[4*(in-1) + a] of every new point; axis 'x' (walls, linear at the ends),
// 'y' or 'z' (periodic).
std::vector<double> construct_stencil(const std::vector<double> &x_old, const std::vector<double> &x_new,
                                      double x_len, const std::vector<int> &idx, char axis);
// Per-target form of the interval loops io = io_lo .. io_hi: the 0-based first source row of every
// new point (Fortran io - 1, less one).  False if a point is covered twice or not at all.
bool starts_from_intervals(const std::vector<int> &idx, int n_new, int io_lo, int io_hi, std::vector<int> &start);

}  // namespace afid_hostd
