// dct_tc.cu -- the four DCT GEMMs of dct.cu on the tcgen05 tensor cores.
#include "engine.h"

namespace ep {

int dct_tc_init(DctPlan &p, std::string &err) {
    err = "tensor-core DCT not built in this library";
    return EP_ERR_UNSUPPORTED;
}

void dct_tc_free(DctPlan &p) { p.tc = nullptr; }

int dct_tc_run(DctPlan &p, float2 *field, float *phi, const DevScalars *S, cudaStream_t st) {
    return EP_ERR_UNSUPPORTED;
}

void *dct_tc_rho_planes(DctPlan &p) { return nullptr; }

}  // namespace ep
