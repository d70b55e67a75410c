// Drives the C++ host mirror (include/pwdft_b200.hpp) the way a reference
// KohnSham would: reads a cell, atoms, a potential and a band block from a
// binary file, applies MultSpinor and AddTeterPrecond, runs LOBPCG, and
// writes the results back.  Used by tests/test_cpp_mirror*.py.
#include <cstdio>
#include <vector>

#include "pwdft_b200.hpp"

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
    return 2;
  }
  std::FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 3;
  pwdft_b200::Domain dm;
  int natom = 0, nband = 0;
  if (std::fread(dm.length, 8, 3, f) != 3 || std::fread(dm.numGrid, 4, 3, f) != 3 ||
      std::fread(dm.numGridFine, 4, 3, f) != 3 || std::fread(&natom, 4, 1, f) != 1 || std::fread(&nband, 4, 1, f) != 1)
    return 4;
  std::vector<int> z(natom);
  std::vector<double> pos(3 * natom), vtot(dm.NumGridTotalFine()), psi((size_t)nband * dm.NumGridTotal());
  if (std::fread(z.data(), 4, natom, f) != (size_t)natom || std::fread(pos.data(), 8, pos.size(), f) != pos.size() ||
      std::fread(vtot.data(), 8, vtot.size(), f) != vtot.size() || std::fread(psi.data(), 8, psi.size(), f) != psi.size())
    return 5;
  std::fclose(f);
  try {
    pwdft_b200::Hamiltonian ham(dm, PW_F64, 0);
    ham.SetAtoms(z, pos);
    ham.SetVtot(vtot.data());
    const int nt = (int)dm.NumGridTotal();
    std::vector<double> hpsi(psi.size()), prec(psi.size(), 0.0), x(psi);
    pwdft_b200::BandBlock bp{psi.data(), nt, nband}, bh{hpsi.data(), nt, nband}, bt{prec.data(), nt, nband};
    ham.MultSpinor(bp, bh);
    ham.AddTeterPrecond(bp, bt);
    pwdft_b200::EigenSolver es(ham);
    pwdft_b200::BandBlock bx{x.data(), nt, nband};
    std::vector<double> eig = es.Solve(bx, PW_SOLVER_LOBPCG, 200, 1e-9);
    std::FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 6;
    std::fwrite(hpsi.data(), 8, hpsi.size(), o);
    std::fwrite(prec.data(), 8, prec.size(), o);
    std::fwrite(eig.data(), 8, eig.size(), o);
    std::fclose(o);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
