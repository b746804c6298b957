// mlp_tc.cu -- the learned subgrid-stress closure: a 10 -> 64 -> 64 -> 64 -> 6
// MLP (GELU, BF16 operands, FP32 accumulation) on the 5th-generation tensor
// cores.  Forward (inference and training) and backward kernels issue
// tcgen05.mma from one thread of the CTA with operands in shared memory and
// the accumulator in tensor memory, read back with tcgen05.ld.  One CTA
// processes a tile of 128 points (M = 128, one TMEM lane per point).
//
// Operand layout in shared memory: the canonical K-major layout without
// swizzle: 8x8 core matrices of 16-byte rows, element (r, k) of an R-row
// tile at byte (k/8)*16R + (r/8)*128 + (r%8)*16 + (k%8)*2, i.e. leading-byte
// offset 16R between the two 8-wide K halves of one K=16 instruction and
// stride-byte offset 128 between 8-row groups.  D = A * B^T with A [M x K]
// and B [N x K] both K-major, so a linear layer y = x W^T takes B = W
// (out x in, the PyTorch weight layout) and the backward dX = dY W takes B = W^T.
//
// Every wait on an mbarrier is bounded; on expiry the kernel records an error
// code and leaves the remaining work undone.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/ch3d_mlp.h"
#include "ch3d_common.cuh"

namespace ch3d_mlp {

constexpr int TILE = 128;      // points per CTA (MMA M)
constexpr int NIN = 10, NINP = 16, NH = 64, NOUT = 6, NOUTP = 16;
constexpr unsigned WAIT_LIMIT = 1u << 24;

// parameter blob (FP32 master copy): W1 [64x10] b1 [64] W2 [64x64] b2 W3 [64x64] b3 W4 [6x64] b4 [6]
constexpr int OW1 = 0, OB1 = OW1 + NH * NIN, OW2 = OB1 + NH, OB2 = OW2 + NH * NH, OW3 = OB2 + NH,
              OB3 = OW3 + NH * NH, OW4 = OB3 + NH, OB4 = OW4 + NOUT * NH, NPARAM = OB4 + NOUT;
static_assert(NPARAM == CH3D_MLP_NPARAM, "parameter count");

// ---------------------------------------------------------------------------
// tcgen05 / mbarrier wrappers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(dst)), "r"(ncols));
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(bar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");  // visible to the tensor-core commit
}
// bounded wait for the phase with the given parity; false on expiry
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned limit = WAIT_LIMIT) {
  const uint32_t a = su32(bar);
  for (unsigned it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// D[tmem] (+)= A * B^T, BF16 x BF16 -> FP32, both operands K-major in smem
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(m0), "r"(m1), "r"(m2), "r"(m3));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
               : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// shared-memory matrix descriptor: canonical K-major, no swizzle
__device__ __forceinline__ uint64_t sdesc(const void* base, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((su32(base) & 0x3FFFF) >> 4);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor: BF16 A and B, FP32 D, K-major A and B, shape M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// byte offset of element (r, k) of a K-major tile with R rows
__device__ __forceinline__ uint32_t koff(int r, int k, int R) {
  return (uint32_t)((k >> 3) * (16 * R) + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
__device__ __forceinline__ void st_bf16(unsigned char* tile, int r, int k, int R, float v) {
  *(__nv_bfloat16*)(tile + koff(r, k, R)) = __float2bfloat16_rn(v);
}

// issue D = A[R_A=128 x K] * B[N x K]^T as K/16 instructions (one thread)
__device__ __forceinline__ void gemm_issue(uint32_t d_tmem, const unsigned char* A, const unsigned char* B, int N,
                                           int K) {
  const uint32_t idesc = idesc_bf16(TILE, N);
  for (int kk = 0; kk < K / 16; ++kk) {
    const uint64_t ad = sdesc(A + kk * 2 * 16 * TILE, 16 * TILE, 128);
    const uint64_t bd = sdesc(B + kk * 2 * 16 * N, 16 * N, 128);
    mma_bf16(d_tmem, ad, bd, idesc, kk > 0 ? 1u : 0u);
  }
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// stage a weight matrix W [rows x cols] (FP32, row-major) as a K-major B
// operand with N = rows (padded to NP with zeros) and K = cols (padded to KP):
// B = W, the forward operand
__device__ void stage_w(unsigned char* t, const float* W, int rows, int cols, int NP, int KP) {
  for (int e = threadIdx.x; e < NP * KP; e += blockDim.x) {
    const int n = e / KP, k = e % KP;
    const float v = (n < rows && k < cols) ? W[n * cols + k] : 0.f;
    st_bf16(t, n, k, NP, v);
  }
}
// B = W^T: N = cols (padded to NP), K = rows (padded to KP), the backward operand
__device__ void stage_wt(unsigned char* t, const float* W, int rows, int cols, int NP, int KP) {
  for (int e = threadIdx.x; e < NP * KP; e += blockDim.x) {
    const int n = e / KP, k = e % KP;
    const float v = (n < cols && k < rows) ? W[k * cols + n] : 0.f;
    st_bf16(t, n, k, NP, v);
  }
}

struct Smem {
  uint64_t bar;
  uint32_t tmem;
  int err;
};

// ---------------------------------------------------------------------------
// forward: X [B x 10] FP32 -> Y [B x 6] FP32.  Training mode also stores the
// pre-activations Z1..Z3 (FP32) and activations H1..H3 (BF16), [B x 64] each.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(TILE, 1) k_mlp_fwd(const float* __restrict__ X, int B,
                                                     const float* __restrict__ P, float* __restrict__ Y,
                                                     float* __restrict__ Z, __nv_bfloat16* __restrict__ H,
                                                     int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char smem[];
  Smem* S = (Smem*)smem;
  unsigned char* XA = smem + 1024;                 // 128 x 16
  unsigned char* HA = XA + TILE * NINP * 2;        // 128 x 64
  unsigned char* W1 = HA + TILE * NH * 2;          // 64 x 16
  unsigned char* W2 = W1 + NH * NINP * 2;          // 64 x 64
  unsigned char* W3 = W2 + NH * NH * 2;            // 64 x 64
  unsigned char* W4 = W3 + NH * NH * 2;            // 16 x 64
  const int tid = threadIdx.x, warp = tid >> 5;
  const long long p0 = (long long)blockIdx.x * TILE;
  const long long pt = p0 + tid;
  const bool valid = pt < B;

  if (tid == 0) { mbar_init(&S->bar, 1); S->err = 0; }
  if (warp == 0) { tmem_alloc(&S->tmem, 64); tmem_relinquish(); }
  stage_w(W1, P + OW1, NH, NIN, NH, NINP);
  stage_w(W2, P + OW2, NH, NH, NH, NH);
  stage_w(W3, P + OW3, NH, NH, NH, NH);
  stage_w(W4, P + OW4, NOUT, NH, NOUTP, NH);
  for (int k = 0; k < NINP; ++k) st_bf16(XA, tid, k, TILE, (valid && k < NIN) ? X[pt * NIN + k] : 0.f);
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tm = S->tmem;
  const uint32_t lane_addr = tm + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;
  const unsigned char* Ain = XA;
  int Kin = NINP;
  const unsigned char* Wl[4] = {W1, W2, W3, W4};
  const float* bl[4] = {P + OB1, P + OB2, P + OB3, P + OB4};
  for (int l = 0; l < 4; ++l) {
    const int N = l < 3 ? NH : NOUTP;
    if (tid == 0) {
      gemm_issue(tm, Ain, Wl[l], N, Kin);
      mma_commit(&S->bar);
    }
    // every thread takes the same branch (the warp-collective TMEM loads follow)
    const int bad = __syncthreads_or(mbar_wait(&S->bar, phase) ? 0 : 1);
    phase ^= 1;
    if (bad) { if (tid == 0) atomicExch(status, 1); break; }
    fence_after();
    float acc[64];
    for (int c = 0; c < N; c += 16) tmem_ld16(lane_addr + c, acc + c);
    fence_before();
    __syncthreads();  // every lane read before the next MMA overwrites TMEM; HA free
    if (l < 3) {
      for (int c = 0; c < NH; ++c) {
        const float z = acc[c] + bl[l][c];
        const float h = gelu(z);
        st_bf16(HA, tid, c, TILE, h);
        if (Z != nullptr && valid) {
          Z[(long long)l * B * NH + pt * NH + c] = z;
          H[(long long)l * B * NH + pt * NH + c] = __float2bfloat16_rn(h);
        }
      }
      fence_async_smem();
      fence_before();
      __syncthreads();
      fence_after();
      Ain = HA;
      Kin = NH;
    } else if (valid) {
      for (int c = 0; c < NOUT; ++c) Y[pt * NOUT + c] = acc[c] + bl[3][c];
    }
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_dealloc(tm, 64);
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

constexpr size_t SMEM_FWD = 1024 + TILE * NINP * 2 + TILE * NH * 2 + NH * NINP * 2 + 2 * NH * NH * 2 + NOUTP * NH * 2;
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
        return cudaFuncSetAttribute(k_mlp_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_FWD);
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
