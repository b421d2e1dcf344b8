// BF16 tensor-core (tcgen05) path of the embedding network.
#include "nnp.cuh"

struct NnpTc {
  int dummy = 0;
};

int nnp_tc_setup(nnpe_ctx*) { return 0; }
void nnp_tc_free(NnpModel* m) {
  delete m->tc;
  m->tc = nullptr;
}
int nnp_tc_forces_enqueue(nnpe_ctx* c, bool) { return nnpe_fail(c, NNPE_EARG, "BF16 path not built"); }
