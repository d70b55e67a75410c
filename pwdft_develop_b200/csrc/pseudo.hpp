// HGH pseudopotential tables and real-space projector / pseudocharge set-up.
#pragma once
#include <vector>

namespace pwb {

struct Spline {
  std::vector<double> x, y, b, c, d;
  void build(const std::vector<double>& xs, const std::vector<double>& ys);
  double eval(double u) const;
};

void spline_coef(int n, const double* x, const double* y, double* b, double* c, double* d);

struct Species {
  int znuc = 0;
  double zion = 0, mass = 0, eself = 0, rhocut = 0, wavcut = 0;
  Spline rho, drho;     // table columns PSEUDO_CHARGE (-rho0) and its derivative
  struct Proj {
    int l;
    double h;
    Spline val, der;
  };
  std::vector<Proj> proj;
};

// Cached HGH species (Si: 14, Al: 13); nullptr if unknown.
const Species* species(int znuc);

// One atom's vnlList: shared index set and, per projector, npts x 4 values
// (VAL, DX, DY, DZ interleaved per point) and the weight.
struct AtomNL {
  int npts = 0;
  std::vector<int> idx;
  std::vector<double> disp;   // 3 per point: Cartesian grid point - atom (unwrapped), for the Bloch phase
  std::vector<std::vector<double>> val;
  std::vector<double> wgt;
};

struct AtomRho {
  std::vector<int> idx;
  std::vector<double> val;   // 4 per point: VAL, DX, DY, DZ
};

int nonlocal_pp(const Species& sp, const double pos[3], const double L[3], const int nG[3], AtomNL& out);
int pseudo_charge(const Species& sp, const double pos[3], const double L[3], const int N[3], AtomRho& out);

}  // namespace pwb
