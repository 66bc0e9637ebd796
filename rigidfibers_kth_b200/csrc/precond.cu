// precond.cu - block preconditioners (filled in below).
#include "handle.h"

namespace rf {

rf_status build_preconditioner(rf_handle *h) {
    return fail(h, RF_ERR_INVALID_ARG, "preconditioner not available");
}

rf_status apply_mlp(rf_handle *h) { return fail(h, RF_ERR_INVALID_ARG, "MLP not available"); }

}  // namespace rf

extern "C" {
int64_t rf_mlp_num_params(void) {
    return (int64_t)RF_MLP_HIDDEN * RF_MLP_IN + RF_MLP_HIDDEN + (int64_t)RF_MLP_HIDDEN * RF_MLP_HIDDEN +
           RF_MLP_HIDDEN + (int64_t)RF_MLP_OUT * RF_MLP_HIDDEN + RF_MLP_OUT;
}
rf_status rf_set_mlp_weights(rf_handle *h, const float *, int64_t) { return rf::fail(h, RF_ERR_INVALID_ARG, "n/a"); }
rf_status rf_compute_features(rf_handle *h, float *) { return rf::fail(h, RF_ERR_INVALID_ARG, "n/a"); }
rf_status rf_compute_cluster_targets(rf_handle *h, float *) { return rf::fail(h, RF_ERR_INVALID_ARG, "n/a"); }
rf_status rf_trainer_create(int32_t, uint64_t, rf_trainer **) { return RF_ERR_INVALID_ARG; }
rf_status rf_trainer_destroy(rf_trainer *) { return RF_ERR_INVALID_ARG; }
rf_status rf_trainer_add_samples(rf_trainer *, const float *, const float *, int64_t) { return RF_ERR_INVALID_ARG; }
rf_status rf_trainer_train(rf_trainer *, int32_t, int32_t, float, float *) { return RF_ERR_INVALID_ARG; }
rf_status rf_trainer_get_weights(rf_trainer *, float *) { return RF_ERR_INVALID_ARG; }
rf_status rf_trainer_set_weights(rf_trainer *, const float *) { return RF_ERR_INVALID_ARG; }
rf_status rf_trainer_loss_grad(rf_trainer *, const float *, const float *, int64_t, float *, float *) {
    return RF_ERR_INVALID_ARG;
}
}
