// mlp_tc.cuh -- tensor-core building blocks of the learned subgrid-stress
// closure (a 10 -> 64 -> 64 -> 64 -> 6 MLP, GELU in its tanh form, BF16
// operands, FP32 accumulation): tcgen05 / mbarrier wrappers, the
// shared-memory operand layout, operand staging and the forward pass of one
// tile of 128 points.  Used by the network kernels (mlp_tc.cu) and by the LES
// step's fused closure kernel (ch3d_les.cu).
//
// Operand layout in shared memory: the canonical K-major layout without
// swizzle: 8x8 core matrices of 16-byte rows, element (r, k) of an R-row
// tile at byte (k/8)*16R + (r/8)*128 + (r%8)*16 + (k%8)*2, i.e. leading-byte
// offset 16R between the two 8-wide K halves of one K=16 instruction and
// stride-byte offset 128 between 8-row groups.  D = A * B^T with A [M x K]
// and B [N x K] both K-major, so a linear layer y = x W^T takes B = W
// (out x in, the PyTorch weight layout) and the backward dX = dY W takes B = W^T.
// Eight consecutive k of one row are 16 contiguous bytes, so a thread that
// owns a row writes it with 16-byte stores.
//
// Every wait on an mbarrier is bounded; on expiry the kernels record an
// error code and leave the remaining work undone.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/ch3d_mlp.h"

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

// 16 consecutive FP32 columns of this thread's TMEM lane; tmem_wait_ld()
// before the values are used
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// NCOLS (a multiple of 16) columns of this thread's lane into v, one wait
template <int NCOLS> __device__ __forceinline__ void tmem_ld(uint32_t taddr, float* v) {
  uint32_t r[NCOLS];
#pragma unroll
  for (int c = 0; c < NCOLS; c += 16) tmem_ld16_async(taddr + c, r + c);
  tmem_wait_ld();
#pragma unroll
  for (int q = 0; q < NCOLS; ++q) v[q] = __uint_as_float(r[q]);
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) { tmem_ld<16>(taddr, v); }

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
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 b = __floats2bfloat162_rn(lo, hi);  // lo at the lower address
  return *reinterpret_cast<const uint32_t*>(&b);
}
// elements k0..k0+7 (k0 a multiple of 8) of row r as one 16-byte store
__device__ __forceinline__ void st_bf16x8(unsigned char* tile, int r, int k0, int R, const float* v) {
  uint4 q;
  q.x = pack_bf16x2(v[0], v[1]);
  q.y = pack_bf16x2(v[2], v[3]);
  q.z = pack_bf16x2(v[4], v[5]);
  q.w = pack_bf16x2(v[6], v[7]);
  *reinterpret_cast<uint4*>(tile + koff(r, k0, R)) = q;
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

// GELU in its tanh form (Hendrycks & Gimpel 2016): 0.5 x (1 + tanh u),
// u = sqrt(2/pi) (x + 0.044715 x^3).  With r = 1 / (1 + exp(2u)),
// 1 + tanh u = 2 (1 - r), so gelu = x - x r.  exp(2u) = 2^(2u log2 e) with
// the factor log2 e folded into the cubic's coefficients, evaluated with the
// hardware's approximate base-2 exponential and reciprocal (relative errors
// near 2^-22): r to about 1e-7 (r -> 0 as the exponential overflows to
// infinity, r -> 1 as it underflows).  Derivative:
// (1 - r) + 2 x r (1 - r) u'(x), u' = sqrt(2/pi) (1 + 3 * 0.044715 x^2).
__device__ __forceinline__ float ex2_approx(float a) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(a));
  return y;
}
__device__ __forceinline__ float rcp_approx(float a) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(a));
  return y;
}
__device__ __forceinline__ float gelu_r(float x) {
  // 2u log2 e = x (2 sqrt(2/pi) log2 e + 2 sqrt(2/pi) 0.044715 log2 e x^2)
  const float t = x * fmaf(0.1029432395800235f, x * x, 2.302208198144325f);
  return rcp_approx(1.0f + ex2_approx(t));
}
__device__ __forceinline__ float gelu(float x) { return x - x * gelu_r(x); }
__device__ __forceinline__ float gelu_d(float x) {
  const float r = gelu_r(x), q = 1.0f - r;
  const float du = 0.79788456080286536f * (1.0f + 0.134145f * x * x);
  return q + 2.0f * x * r * q * du;
}

// Work item e of an operand staging: 8 elements (n, k0..k0+7) of an NP-row
// tile (NP a multiple of 8) with kq = KP/8 pieces per row.  Eight
// consecutive items take rows n..n+7 of one 8-row group (their 16-byte
// pieces fill all 32 banks), the next eight the next k piece: a warp writes
// 4 x 128 contiguous bytes (no bank conflicts) and reads 8 rows x 32 bytes
// of the FP32 source.
__device__ __forceinline__ void stage_index(int e, int kq, int& n, int& k0) {
  const int g = e >> 3;
  k0 = (g % kq) << 3;
  n = ((g / kq) << 3) + (e & 7);
}
// stage a weight matrix W [rows x cols] (FP32, row-major) as a K-major B
// operand with N = rows (padded to NP with zeros) and K = cols (padded to
// KP): B = W, the forward operand.  One 16-byte store per 8 elements.
__device__ __forceinline__ void stage_w(unsigned char* t, const float* __restrict__ W, int rows, int cols, int NP,
                                        int KP) {
  const int kq = KP >> 3;
  for (int e = threadIdx.x; e < NP * kq; e += blockDim.x) {
    int n, k0;
    stage_index(e, kq, n, k0);
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = (n < rows && k0 + q < cols) ? __ldg(W + n * cols + k0 + q) : 0.f;
    st_bf16x8(t, n, k0, NP, v);
  }
}
// B = W^T: N = cols (padded to NP), K = rows (padded to KP), the backward operand
__device__ __forceinline__ void stage_wt(unsigned char* t, const float* __restrict__ W, int rows, int cols, int NP,
                                         int KP) {
  const int kq = KP >> 3;
  for (int e = threadIdx.x; e < NP * kq; e += blockDim.x) {
    int n, k0;
    stage_index(e, kq, n, k0);
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = (n < cols && k0 + q < rows) ? __ldg(W + (k0 + q) * cols + n) : 0.f;
    st_bf16x8(t, n, k0, NP, v);
  }
}

struct Smem {
  uint64_t bar;   // tensor-core completion
  uint64_t wbar;  // arrival of the packed parameters (fwd_prologue_packed)
  uint32_t tmem;
  int err;
};

// shared memory of the forward pass: header, activation tile (its first
// 4 KB hold the X tile until the first layer's MMA has read it: the
// activations are written only after that MMA completed), the four weight
// operands and the biases; 37.8 KB, so that six CTAs fit an SM
struct FwdSmem {
  static constexpr size_t XA = 128;
  static constexpr size_t HA = XA;
  static constexpr size_t W1 = HA + TILE * NH * 2;
  static constexpr size_t W2 = W1 + NH * NINP * 2;
  static constexpr size_t W3 = W2 + NH * NH * 2;
  static constexpr size_t W4 = W3 + NH * NH * 2;
  static constexpr size_t BIAS = W4 + NOUTP * NH * 2;  // b1 b2 b3 (64 each), b4 (6, padded to 16)
  static constexpr size_t BYTES = BIAS + (3 * NH + 16) * 4;
};

// bytes of the parameter image: the four weight operands and the biases, as
// they lie in the forward pass's shared memory from FwdSmem::W1 on
constexpr size_t kPackedBytes = FwdSmem::BYTES - FwdSmem::W1;
static_assert(FwdSmem::W1 % 16 == 0 && kPackedBytes % 16 == 0, "bulk copy alignment");

// Write the parameter image of P into `img` (global or shared memory; all
// threads of the block take part): W1..W4 as BF16 K-major operands, the
// biases as FP32, at their offsets from FwdSmem::W1.
__device__ __forceinline__ void pack_params(unsigned char* img, const float* __restrict__ P) {
  stage_w(img + (FwdSmem::W1 - FwdSmem::W1), P + OW1, NH, NIN, NH, NINP);
  stage_w(img + (FwdSmem::W2 - FwdSmem::W1), P + OW2, NH, NH, NH, NH);
  stage_w(img + (FwdSmem::W3 - FwdSmem::W1), P + OW3, NH, NH, NH, NH);
  stage_w(img + (FwdSmem::W4 - FwdSmem::W1), P + OW4, NOUT, NH, NOUTP, NH);
  float* bs = (float*)(img + (FwdSmem::BIAS - FwdSmem::W1));
  for (int e = threadIdx.x; e < 3 * NH + 16; e += blockDim.x) {
    const int l = e / NH, c = e - l * NH;
    bs[e] = l < 3 ? __ldg(P + (l == 0 ? OB1 : l == 1 ? OB2 : OB3) + c) : (c < NOUT ? __ldg(P + OB4 + c) : 0.f);
  }
}

// Stage the parameters (weights as BF16 operands, biases as FP32) and the
// point's standardised inputs x[0..9] (row tid of the X tile), set up the
// mbarrier and the tensor memory (64 columns).  Ends with the barrier that
// makes all of it visible to the tensor cores and to every thread.
__device__ __forceinline__ void fwd_prologue(unsigned char* smem, const float* __restrict__ P, const float* x) {
  Smem* S = (Smem*)smem;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (tid == 0) { mbar_init(&S->bar, 1); S->err = 0; }
  if (warp == 0) { tmem_alloc(&S->tmem, 64); tmem_relinquish(); }
  pack_params(smem + FwdSmem::W1, P);
  float xp[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) xp[k] = k < NIN ? x[k] : 0.f;
  st_bf16x8(smem + FwdSmem::XA, tid, 0, TILE, xp);
  st_bf16x8(smem + FwdSmem::XA, tid, 8, TILE, xp + 8);
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
}

// The same with the parameter image `img` (kPackedBytes, 16-byte aligned,
// written by pack_params) brought in by one bulk asynchronous copy issued at
// entry: the copy runs while the caller forms the inputs; fwd_inputs then
// stages them and waits for the copy (bounded).
__device__ __forceinline__ void fwd_prologue_packed(unsigned char* smem, const unsigned char* __restrict__ img) {
  Smem* S = (Smem*)smem;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (tid == 0) {
    mbar_init(&S->bar, 1);
    mbar_init(&S->wbar, 1);
    S->err = 0;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(&S->wbar)),
                 "r"((uint32_t)kPackedBytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            su32(smem + FwdSmem::W1)),
        "l"(img), "r"((uint32_t)kPackedBytes), "r"(su32(&S->wbar))
        : "memory");
  }
  if (warp == 0) { tmem_alloc(&S->tmem, 64); tmem_relinquish(); }
}
// Stage the point's inputs x[0..9] (row tid of the X tile) and wait for the
// parameter image.  Returns false (uniformly) when the wait expired; the
// caller then skips the network, the copy having been waited for as long as
// the limit allows.
__device__ __forceinline__ bool fwd_inputs(unsigned char* smem, const float* x) {
  Smem* S = (Smem*)smem;
  const int tid = threadIdx.x;
  float xp[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) xp[k] = k < NIN ? x[k] : 0.f;
  st_bf16x8(smem + FwdSmem::XA, tid, 0, TILE, xp);
  st_bf16x8(smem + FwdSmem::XA, tid, 8, TILE, xp + 8);
  fence_async_smem();
  fence_before();
  __syncthreads();  // the barriers' initialisation, the X tile, the tensor memory
  fence_after();
  return __syncthreads_or(mbar_wait(&S->wbar, 0) ? 0 : 1) == 0;
}

// After an expired wait in fwd_inputs: wait once more (bounded) for the copy
// in flight, then release the tensor memory.
__device__ __forceinline__ void fwd_abort(unsigned char* smem) {
  Smem* S = (Smem*)smem;
  mbar_wait(&S->wbar, 0);
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) tmem_dealloc(S->tmem, 64);
}

// The four layers on the staged tile: y[0..5] = network output of this
// thread's point.  Training mode (Z != nullptr) also stores the
// pre-activations Z1..Z3 (FP32) and activations H1..H3 (BF16) of valid
// points, [B x 64] each.  Returns false (uniformly over the CTA) when a
// wait on the tensor cores expired; the tensor memory is released either way.
__device__ __forceinline__ bool fwd_layers(unsigned char* smem, float* y, float* __restrict__ Z,
                                           __nv_bfloat16* __restrict__ H, long long pt, bool valid, long long B) {
  Smem* S = (Smem*)smem;
  const int tid = threadIdx.x, warp = tid >> 5;
  unsigned char* HA = smem + FwdSmem::HA;
  const float* bs = (const float*)(smem + FwdSmem::BIAS);
  const uint32_t tm = S->tmem;
  const uint32_t lane_addr = tm + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;
  bool ok = true;
#pragma unroll 1
  for (int l = 0; l < 4; ++l) {
    if (tid == 0) {
      if (l == 0) gemm_issue(tm, smem + FwdSmem::XA, smem + FwdSmem::W1, NH, NINP);
      else gemm_issue(tm, HA, smem + (l == 1 ? FwdSmem::W2 : l == 2 ? FwdSmem::W3 : FwdSmem::W4), l < 3 ? NH : NOUTP,
                      NH);
      mma_commit(&S->bar);
    }
    // every thread takes the same branch (the warp-collective TMEM loads follow)
    ok = __syncthreads_or(mbar_wait(&S->bar, phase) ? 0 : 1) == 0;
    phase ^= 1;
    if (!ok) break;
    fence_after();
    if (l < 3) {
      // The layer's MMA has completed, so HA (its A operand) may be
      // overwritten; the next MMA, which overwrites the accumulator, is
      // issued only after the barrier below.  Sixteen columns at a time,
      // not unrolled, to keep the code within the instruction cache.
#pragma unroll 1
      for (int c0 = 0; c0 < NH; c0 += 16) {
        float acc[16], h[16];
        tmem_ld<16>(lane_addr + c0, acc);
        float bq[16];
#pragma unroll
        for (int q = 0; q < 16; q += 4) *reinterpret_cast<float4*>(bq + q) = *reinterpret_cast<const float4*>(bs + l * NH + c0 + q);
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const float z = acc[q] + bq[q];
          h[q] = gelu(z);
          if (Z != nullptr && valid) {
            Z[(long long)l * B * NH + pt * NH + c0 + q] = z;
            H[(long long)l * B * NH + pt * NH + c0 + q] = __float2bfloat16_rn(h[q]);
          }
        }
        st_bf16x8(HA, tid, c0, TILE, h);
        st_bf16x8(HA, tid, c0 + 8, TILE, h + 8);
      }
      fence_async_smem();
      fence_before();
      __syncthreads();
      fence_after();
    } else {
      float acc[16];
      tmem_ld<16>(lane_addr, acc);
#pragma unroll
      for (int c = 0; c < NOUT; ++c) y[c] = acc[c] + bs[3 * NH + c];
    }
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_dealloc(tm, 64);
  return ok;
}

}  // namespace ch3d_mlp
