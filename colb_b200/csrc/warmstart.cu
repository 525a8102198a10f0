// warmstart.cu — per-body features for the learned warm start.
#include "engine.cuh"

extern "C" int abd_get_features(AbdHandle* h, float* feat, int32_t n) {
    Engine* E = reinterpret_cast<Engine*>(h);
    if (!E) return ABD_ERR_INVALID_ARG;
    (void)feat; (void)n;
    return E->fail(ABD_ERR_NOT_BUILT, "abd_get_features: not available in this build");
}
