// mlp_tc.cu -- the learned subgrid-stress closure: a 10 -> 64 -> 64 -> 64 -> 6
// MLP (GELU in its tanh form, BF16 operands, FP32 accumulation) on the
// 5th-generation tensor cores.  Forward (inference and training) and
// backward kernels issue tcgen05.mma from one thread of the CTA with operands
// in shared memory and the accumulator in tensor memory, read back with
// tcgen05.ld.  One CTA processes a tile of 128 points (M = 128, one TMEM
// lane per point).  The operand layout, the wrappers and the forward pass of
// a tile are in mlp_tc.cuh.
#include "mlp_tc.cuh"
#include "ch3d_common.cuh"

namespace ch3d_mlp {

// ---------------------------------------------------------------------------
// forward: X [B x 10] FP32 -> Y [B x 6] FP32.  Training mode also stores the
// pre-activations Z1..Z3 (FP32) and activations H1..H3 (BF16), [B x 64] each.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(TILE, 6) k_mlp_fwd(const float* __restrict__ X, int B,
                                                     const float* __restrict__ P, float* __restrict__ Y,
                                                     float* __restrict__ Z, __nv_bfloat16* __restrict__ H,
                                                     int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x;
  const long long pt = (long long)blockIdx.x * TILE + tid;
  const bool valid = pt < B;
  float x[NIN];
#pragma unroll
  for (int k = 0; k < NIN; ++k) x[k] = valid ? X[pt * NIN + k] : 0.f;
  fwd_prologue(smem, P, x);
  float y[NOUT];
  if (!fwd_layers(smem, y, Z, H, pt, valid, B)) {
    if (tid == 0) atomicExch(status, 1);
    return;
  }
  if (valid)
    for (int c = 0; c < NOUT; ++c) Y[pt * NOUT + c] = y[c];
}

// ---------------------------------------------------------------------------
// backward of the mean-squared loss L = sum (Y - T)^2 / (B*6) for one tile:
// per-CTA partial gradients part[blockIdx.x][NPARAM] and partial loss.
// Weight gradients are dW^T = dZ^T H_prev, computed as MMAs with M = 128
// (output features, zero-padded rows) and K = the tile's 128 points.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(TILE, 1) k_mlp_bwd(const float* __restrict__ X, const float* __restrict__ T,
                                                     int B, const float* __restrict__ P,
                                                     const float* __restrict__ Y, const float* __restrict__ Z,
                                                     const __nv_bfloat16* __restrict__ H, float* __restrict__ part,
                                                     float* __restrict__ lpart, int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char smem[];
  Smem* S = (Smem*)smem;
  unsigned char* DA = smem + 1024;                 // dZ (or dY) as A: 128 points x 64
  unsigned char* DT = DA + TILE * NH * 2;          // dZ^T as A: 128 (features, padded) x 128 points
  unsigned char* HT = DT + TILE * TILE * 2;        // H_prev^T as B: 64 features x 128 points
  unsigned char* WT = HT + NH * TILE * 2;          // W as B for dH = dZ W: 64 x 64
  float* red = (float*)(WT + NH * NH * 2);         // 4 warps x 64 column sums
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long p0 = (long long)blockIdx.x * TILE;
  const long long pt = p0 + tid;
  const bool valid = pt < B;
  float* G = part + (long long)blockIdx.x * NPARAM;

  if (tid == 0) { mbar_init(&S->bar, 1); S->err = 0; }
  if (warp == 0) { tmem_alloc(&S->tmem, 128); tmem_relinquish(); }
  const float invn = 1.0f / ((float)B * (float)NOUT);
  // dY and the loss partial
  float d[64];
  float lsum = 0.f;
  for (int c = 0; c < NOUTP; ++c) {
    float v = 0.f;
    if (valid && c < NOUT) {
      const float e = Y[pt * NOUT + c] - T[pt * NOUT + c];
      lsum += e * e;
      v = 2.0f * e * invn;
    }
    d[c] = v;
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if (lane == 0) red[warp] = lsum;
  __syncthreads();
  if (tid == 0) lpart[blockIdx.x] = red[0] + red[1] + red[2] + red[3];
  __syncthreads();
  const uint32_t tm = S->tmem;
  const uint32_t lane_addr = tm + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;
  bool ok = true;
  const float* Wl[4] = {P + OW1, P + OW2, P + OW3, P + OW4};
  const int oW[4] = {OW1, OW2, OW3, OW4}, oB[4] = {OB1, OB2, OB3, OB4};
  for (int l = 3; l >= 0 && ok; --l) {
    const int nout = l == 3 ? NOUT : NH;       // rows of W_l
    const int nin = l == 0 ? NIN : NH;         // cols of W_l
    const int KD = l == 3 ? NOUTP : NH;        // K of dH = dZ W (padded nout)
    const int NI = l == 0 ? NINP : NH;         // N of the weight-gradient MMA (padded nin)
    // bias gradient: column sums of dZ over the tile (FP32)
    for (int c = 0; c < nout; ++c) {
      float v = d[c];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp * 64 + c] = v;
    }
    // operands: dZ (A, points x KD), dZ^T (A, 128 padded features x points), H_prev^T (B), W (B)
    for (int c = 0; c < KD; ++c) st_bf16(DA, tid, c, TILE, d[c]);
    for (int c = 0; c < TILE; ++c) st_bf16(DT, c, tid, TILE, c < nout ? d[c] : 0.f);
    for (int c = 0; c < NI; ++c) {
      float h = 0.f;
      if (valid && c < nin) h = l == 0 ? X[pt * NIN + c] : __bfloat162float(H[(long long)(l - 1) * B * NH + pt * NH + c]);
      st_bf16(HT, c, tid, NI, h);
    }
    if (l > 0) stage_wt(WT, Wl[l], nout, nin, NH, KD);
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    if (tid < nout) G[oB[l] + tid] = red[tid] + red[64 + tid] + red[128 + tid] + red[192 + tid];
    if (tid == 0) {
      gemm_issue(tm, DT, HT, NI, TILE);                  // dW^T[o][i] in columns 0..NI-1
      if (l > 0) gemm_issue(tm + 64, DA, WT, NH, KD);   // dH[p][i] in columns 64..127
      mma_commit(&S->bar);
    }
    ok = __syncthreads_or(mbar_wait(&S->bar, phase) ? 0 : 1) == 0;  // uniform across the CTA
    phase ^= 1;
    if (!ok) { if (tid == 0) atomicExch(status, 1); break; }
    fence_after();
    float w[64];
    for (int c = 0; c < NI; c += 16) tmem_ld16(lane_addr + c, w + c);
    if (tid < nout)
      for (int i = 0; i < nin; ++i) G[oW[l] + tid * nin + i] = w[i];
    if (l > 0) {
      float dh[64];
      for (int c = 0; c < NH; c += 16) tmem_ld16(lane_addr + 64 + c, dh + c);
      for (int c = 0; c < NH; ++c) {
        const float z = valid ? Z[(long long)(l - 1) * B * NH + pt * NH + c] : 0.f;
        d[c] = valid ? dh[c] * gelu_d(z) : 0.f;
      }
    }
    fence_before();
    __syncthreads();  // TMEM reads and the smem operands done before they are reused
    fence_after();
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_dealloc(tm, 128);
}

// fixed-order sum of the per-CTA partials: grad[q] = sum_b part[b][q]
__global__ void k_mlp_reduce(const float* __restrict__ part, const float* __restrict__ lpart, int nb,
                             float* __restrict__ grad, float* __restrict__ loss) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < NPARAM) {
    float s = 0.f;
    for (int b = 0; b < nb; ++b) s += part[(long long)b * NPARAM + q];
    grad[q] = s;
  }
  if (q == 0) {
    float s = 0.f;
    for (int b = 0; b < nb; ++b) s += lpart[b];
    *loss = s;
  }
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters
__global__ void k_adam(float* __restrict__ P, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float bc1, float bc2) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= NPARAM) return;
  const float gq = g[q];
  const float mq = b1 * m[q] + (1.f - b1) * gq;
  const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
  m[q] = mq;
  v[q] = vq;
  P[q] -= lr * (mq / bc1) / (sqrtf(vq / bc2) + eps);
}

constexpr size_t SMEM_FWD = FwdSmem::BYTES;
constexpr size_t SMEM_BWD = 1024 + TILE * NH * 2 + TILE * TILE * 2 + NH * TILE * 2 + NH * NH * 2 + 4 * 64 * 4;

// The expiry path of the bounded waits: one thread waits on an mbarrier that
// nothing arrives at (no MMA issued, no tensor memory held) and, when the
// wait gives up after `limit` polls, records the expiry in *status as the
// MLP kernels do.
__global__ void k_mlp_wait_check(unsigned limit, int* __restrict__ status) {
  __shared__ uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  if (!mbar_wait(&bar, 0, limit)) atomicExch(status, 1);
}

}  // namespace ch3d_mlp

using namespace ch3d_mlp;

// One-time attribute set-up per device a process drives (cudaFuncSetAttribute
// applies to the current device only), under the library's set-up lock.
template <class F> static bool setup_on_current_device(ch3d::PerDevice& site, F&& setup) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  return ch3d::once_per_device(site, dev, setup) == cudaSuccess;
}

extern "C" {

CH3D_MLP_API size_t ch3d_mlp_workspace_bytes(int batch) {
  const size_t nb = (size_t)(batch + TILE - 1) / TILE;
  return (size_t)3 * batch * NH * 4 + (size_t)3 * batch * NH * 2 + (size_t)batch * NOUT * 4 + nb * NPARAM * 4 + nb * 4 +
         256;
}

CH3D_MLP_API int ch3d_mlp_wait_check(unsigned limit, int* status, void* stream) {
  if (!status || limit == 0) return 1;
  k_mlp_wait_check<<<1, 32, 0, (cudaStream_t)stream>>>(limit, status);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

CH3D_MLP_API int ch3d_mlp_forward(const float* X, int batch, const float* params, float* Y, int* status,
                                  void* stream) {
  if (!X || !params || !Y || !status || batch <= 0) return 1;
  static ch3d::PerDevice attr;
  if (!setup_on_current_device(attr, [] {
        cudaError_t r = cudaFuncSetAttribute(k_mlp_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_FWD);
        if (r == cudaSuccess) r = cudaFuncSetAttribute(k_mlp_fwd, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        return r;
      }))
    return 2;
  k_mlp_fwd<<<(batch + TILE - 1) / TILE, TILE, SMEM_FWD, (cudaStream_t)stream>>>(X, batch, params, Y, nullptr, nullptr,
                                                                                status);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

CH3D_MLP_API int ch3d_mlp_grad(const float* X, const float* T, int batch, const float* params, void* work,
                               float* grad, float* loss, int* status, void* stream) {
  if (!X || !T || !params || !work || !grad || !loss || !status || batch <= 0) return 1;
  static ch3d::PerDevice attr;
  if (!setup_on_current_device(attr, [] {
        cudaError_t r = cudaFuncSetAttribute(k_mlp_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_FWD);
        if (r == cudaSuccess)
          r = cudaFuncSetAttribute(k_mlp_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BWD);
        return r;
      }))
    return 2;
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = (batch + TILE - 1) / TILE;
  unsigned char* w = (unsigned char*)work;
  float* Z = (float*)w;
  w += (size_t)3 * batch * NH * 4;
  __nv_bfloat16* H = (__nv_bfloat16*)w;
  w += (size_t)3 * batch * NH * 2;
  w = (unsigned char*)(((uintptr_t)w + 255) & ~(uintptr_t)255);
  float* Y = (float*)w;
  w += (size_t)batch * NOUT * 4;
  float* part = (float*)w;
  w += (size_t)nb * NPARAM * 4;
  float* lpart = (float*)w;
  k_mlp_fwd<<<nb, TILE, SMEM_FWD, st>>>(X, batch, params, Y, Z, H, status);
  k_mlp_bwd<<<nb, TILE, SMEM_BWD, st>>>(X, T, batch, params, Y, Z, H, part, lpart, status);
  k_mlp_reduce<<<(NPARAM + 255) / 256, 256, 0, st>>>(part, lpart, nb, grad, loss);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

CH3D_MLP_API int ch3d_mlp_adam(float* params, const float* grad, float* m, float* v, float lr, float beta1,
                               float beta2, float eps, int step, void* stream) {
  if (!params || !grad || !m || !v || step < 1) return 1;
  const float bc1 = 1.0f - powf(beta1, (float)step), bc2 = 1.0f - powf(beta2, (float)step);
  k_adam<<<(NPARAM + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, grad, m, v, lr, beta1, beta2, eps, bc1, bc2);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // extern "C"
