// mlp.cu -- cooling-surrogate MLP (placeholder until the tensor-core kernels land)
#include "sph_internal.cuh"

int launch_cooling_mlp(sph_ctx *ctx) { (void)ctx; return SPH_ERR_STATE; }

extern "C" {
int sph_mlp_set(sph_ctx *, const float *, const float *, int32_t) { return SPH_ERR_STATE; }
int sph_mlp_get(sph_ctx *, float *, float *, int32_t) { return SPH_ERR_STATE; }
int sph_mlp_forward(sph_ctx *, int32_t, const float *, float *, int32_t) { return SPH_ERR_STATE; }
int sph_mlp_grad(sph_ctx *, int32_t, const float *, const float *, float *, float *, int32_t) { return SPH_ERR_STATE; }
int sph_mlp_train(sph_ctx *, int32_t, const float *, const float *, int32_t, int32_t, float, float *) { return SPH_ERR_STATE; }
}
