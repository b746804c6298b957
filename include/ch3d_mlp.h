/* ch3d_mlp.h -- the learned subgrid-stress closure of the LES step: a
   10 -> 64 -> 64 -> 64 -> 6 multilayer perceptron (GELU activations in their
   tanh form, BF16 tensor-core operands, FP32 accumulation) trained and
   evaluated on the GPU.
   No counterpart in the reference (its LES models are the eddy-viscosity
   closures of src/CFD_2nd/m_LESModels.f90); the LES step calls it in place
   of Clc_SGS_Vis when LES_type = CH3D_LES_MLP.

   All pointers are DEVICE pointers; `stream` is a cudaStream_t (NULL = the
   legacy default stream).  Functions return 0 on success, 1 for a bad
   argument, 2 for a CUDA launch error; a kernel that times out waiting for
   its tensor-core work sets *status to 1 (leave *status at 0 before the call).

   Parameter blob (FP32, CH3D_MLP_NPARAM values): W1 [64 x 10], b1 [64],
   W2 [64 x 64], b2 [64], W3 [64 x 64], b3 [64], W4 [6 x 64], b4 [6];
   each W is [out x in], row-major.  Inputs X are [batch x 10] and outputs /
   targets [batch x 6], row-major FP32 (normalised by the caller). */
#ifndef CH3D_MLP_H
#define CH3D_MLP_H
#include <stddef.h>

#if defined(__GNUC__)
#define CH3D_MLP_API __attribute__((visibility("default")))
#else
#define CH3D_MLP_API
#endif

#define CH3D_MLP_NPARAM 9414

#ifdef __cplusplus
extern "C" {
#endif

/* Inference: Y = MLP(X). */
CH3D_MLP_API int ch3d_mlp_forward(const float* X, int batch, const float* params, float* Y, int* status,
                                  void* stream);

/* Bytes of the device workspace ch3d_mlp_grad needs for `batch` points. */
CH3D_MLP_API size_t ch3d_mlp_workspace_bytes(int batch);

/* Gradient of the mean-squared loss sum((Y - T)^2) / (6 batch) with respect
   to the parameters (grad, CH3D_MLP_NPARAM FP32) and the summed squared error
   (*loss, device), forward and backward on the tensor cores. */
CH3D_MLP_API int ch3d_mlp_grad(const float* X, const float* T, int batch, const float* params, void* work,
                               float* grad, float* loss, int* status, void* stream);

/* One Adam step (Kingma & Ba 2015) on the FP32 parameters; step counts from 1. */
CH3D_MLP_API int ch3d_mlp_adam(float* params, const float* grad, float* m, float* v, float lr, float beta1,
                               float beta2, float eps, int step, void* stream);

/* Failure detection of the tensor-core kernels without a fault: runs their
   bounded mbarrier wait, `limit` polls long, on a barrier nothing completes
   (no MMA in flight, no tensor memory held) and sets *status to 1 when the
   wait gives up, as a kernel whose tensor-core work never completes does;
   the context stays usable. */
CH3D_MLP_API int ch3d_mlp_wait_check(unsigned limit, int* status, void* stream);

#ifdef __cplusplus
}
#endif
#endif
