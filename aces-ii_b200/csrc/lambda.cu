// lambda.cu -- Lambda equations and the one-particle density.
#include "engine.cuh"

using namespace acesb200;

extern "C" int xlambda_run(aces_cc_config *cfg) {
  (void)cfg;
  set_error("xlambda_run: not available in this build");
  return ACES_ERR_UNSUPPORTED;
}

extern "C" int xdens_1pdm(aces_cc_config *cfg) {
  (void)cfg;
  set_error("xdens_1pdm: not available in this build");
  return ACES_ERR_UNSUPPORTED;
}
