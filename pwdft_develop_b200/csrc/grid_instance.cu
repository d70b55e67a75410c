// One coarse grid (PWB_N0 x PWB_N1 x PWB_N2, fine grid twice that) of the
// H*psi pipeline, FP64 and FP32.  Compiled once per line of grids.inc with
// -DPWB_N0=... -DPWB_N1=... -DPWB_N2=... (pwdft_develop_b200/build.py); the
// object registers its entry points when the library is loaded.
#include "pipeline.cuh"

#if !defined(PWB_N0) || !defined(PWB_N1) || !defined(PWB_N2)
#error "grid_instance.cu is compiled with -DPWB_N0 -DPWB_N1 -DPWB_N2"
#endif

namespace pwb {
namespace {
struct Registrar {
  Registrar() {
    const GridEntry e = PWB_GRID_ENTRY(PWB_N0, PWB_N1, PWB_N2);
    register_grid(e);
  }
};
Registrar registrar_instance;
}  // namespace
}  // namespace pwb
