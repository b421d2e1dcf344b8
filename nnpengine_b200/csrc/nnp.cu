// Network term (NNPOTENTIAL_TBL, pair_nnp.cpp:433-793, and the radial-embedding network).
#include "internal.cuh"

struct NnpModel {
  int dummy;
};

void nnp_free(nnpe_ctx* c) {
  delete c->nnp;
  c->nnp = nullptr;
}
int nnp_forces_enqueue(nnpe_ctx*, bool) { return 0; }
const double* nnp_atom_energy_ptr(nnpe_ctx*) { return nullptr; }
