// ch3d_rfft.cu -- the Poisson transforms with the register-resident FFT of
// rfft.cuh, for the line lengths that have a plan (others use the generic
// shared-memory kernels of ch3d_step.cu):
//   prsrc_xfft_r  clcPrSrcOther (src/CFD_2nd/m_TScheme.f90:213-241) fused with
//                 the forward x R2C transform (m_Poisson.f90:241-333, R2HC)
//   zfft_r        z transform of the spectrum, in place
//   xifft_r       inverse x C2R transform * normfft -> phi (m_Poisson.f90:1194-1200)
// The x kernels give each line to P <= 32 threads of one warp and loop over
// lines without block barriers; the z kernel gives a block LZ = 8 consecutive kx
// lines (coalesced 8 x 16-byte segments per kz) of P threads each.
#include "ch3d_ctx.h"
#include "ch3d_dev.cuh"
#include "rfft.cuh"

namespace ch3d {

constexpr int kXWarps = 4;  // warps per block of the x kernels
// padded exchange buffers for the 16-byte FP64 points (the 8-byte FP32 points
// conflict less without the padding)
template <class T> constexpr bool kPadX = sizeof(T) == 8;

// Plans (N, P, radices): exchange radices multiply to P, in-thread ones to N / P.
typedef RPlan<384, 32, 4, 4, 2, 12> PlanN384;
typedef RPlan<256, 32, 8, 4, 8> PlanN256;
typedef RPlan<128, 32, 4, 4, 2, 4> PlanN128;
typedef RPlan<64, 16, 4, 4, 4> PlanN64;
typedef RPlan<576, 48, 4, 4, 3, 12> PlanN576;
typedef RPlan<128, 16, 8, 2, 8> PlanZ128;

// SRC: modes 2, 3 and 4, the source (or divergence, or field) already formed in the first
// array; compiled separately so it is not held to the divergence modes' registers.
template <class T, class PL, bool SRC>
__global__ void __launch_bounds__(32 * kXWarps, SRC ? 6 : (sizeof(T) == 4 ? 6 : 4)) k_prsrc_xfft_r(Geo<T> g, Metrics<T> m, const T* __restrict__ ux,
                                                              const T* __restrict__ uy, const T* __restrict__ uz,
                                                              typename CplxOf<T>::type* __restrict__ spec,
                                                              const typename CplxOf<T>::type* __restrict__ tw,
                                                              const typename CplxOf<T>::type* __restrict__ twr,
                                                              int mode, DevScalars* __restrict__ sc, T* __restrict__ pr) {
  typedef typename CplxOf<T>::type CT;
  constexpr int M = PL::N, P = PL::P, E = PL::E, LPW = 32 / P;
  __shared__ CT sm[kXWarps * LPW][PL::padded_len()];
  __shared__ double wred[kXWarps];
  if (sc->status) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz, nxh = g.nxh;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int t = lane % P, slot = warp * LPW + lane / P;
  CT* L = sm[slot];
  const int nlines = ny * nz;
  // mode 3: the divergence of u* already formed (k_div_bsub) in the first array; mode 4:
  // any real field in the first array, transformed as it is (no scaling, no maximum)
  const T sudtal = mode == 0 || mode == 3 ? (T)(1.0 / sc->pmAlpha) : (T)1;
  const T rdx = g.rdx, rdz = g.rdz;
  double dmax = 0.0;
  // warp groups of LPW lines, grid-stride; every thread of a warp runs the same iterations
  const int ngroups = (nlines + LPW - 1) / LPW;
  for (int grp = blockIdx.x * kXWarps + warp; grp < ngroups; grp += gridDim.x * kXWarps) {
    const int line = grp * LPW + lane / P;
    const bool valid = line < nlines;
    CT z[E];
    if (valid) {
      const int j = line % ny, k = line / ny;
      const int kp = k + 1 == nz ? 0 : k + 1;
      const long long base = (long long)nx * line;
      const long long basep = (long long)nx * (j + (long long)ny * kp);
      const T sucaj = m.rdyp[j + 1];
      const bool top = j + 1 == ny;
#pragma unroll
      for (int q = 0; q < E; ++q) {
        const int n = t + P * q;
        const int i0 = 2 * n, i2 = i0 + 2 == nx ? 0 : i0 + 2;
        T r0, r1;
        if constexpr (SRC) {  // the source (or divergence) is in the first array
          typedef typename CplxOf<T>::type T2;  // (i0, i0+1) as one aligned vector load
          const T2 s01 = __ldg(reinterpret_cast<const T2*>(ux + base + i0));
          r0 = s01.x; r1 = s01.y;
        } else if (g.order == 4) {
          const C4<T> c4(g);
          r0 = div4_cell(g, c4, sucaj, ux, uy, uz, i0, j, k);
          r1 = div4_cell(g, c4, sucaj, ux, uy, uz, i0 + 1, j, k);
        } else {
          // pairs (i0, i0+1) as one aligned vector load (nx and i0 even)
          typedef typename CplxOf<T>::type T2;
          const T2 u01 = __ldg(reinterpret_cast<const T2*>(ux + base + i0));
          const T u2 = __ldg(ux + base + i2);
          const T2 v01 = __ldg(reinterpret_cast<const T2*>(uy + base + i0));
          // uy at j+1: the next row, above the top row the wall value or, periodic in y, row 0
          const T2 v01p = !top ? __ldg(reinterpret_cast<const T2*>(uy + base + nx + i0))
                          : (g.bc.hi == 0 ? __ldg(reinterpret_cast<const T2*>(uy + base - (long long)(ny - 1) * nx + i0))
                                          : mk((T)g.bc.uy_hi, (T)g.bc.uy_hi));
          const T2 w01 = __ldg(reinterpret_cast<const T2*>(uz + base + i0));
          const T2 w01p = __ldg(reinterpret_cast<const T2*>(uz + basep + i0));
          r0 = (u01.y - u01.x) * rdx + (v01p.x - v01.x) * sucaj + (w01p.x - w01.x) * rdz;
          r1 = (u2 - u01.y) * rdx + (v01p.y - v01.y) * sucaj + (w01p.y - w01.y) * rdz;
        }
        if (!SRC && mode == 0 && g.implicit == 2) {  // clcPrSrc_FIMP: pressure += -xnu/2 div (m_TScheme.f90:271)
          const T xnuhm = -(T)0.5 * g.xnu;
          pr[base + i0] = pr[base + i0] + xnuhm * r0;
          pr[base + i0 + 1] = pr[base + i0 + 1] + xnuhm * r1;
        }
        dmax = fmax(dmax, fmax(fabs((double)r0), fabs((double)r1)));
        z[q] = mk(sudtal * r0, sudtal * r1);
      }
    } else {
#pragma unroll
      for (int q = 0; q < E; ++q) z[q] = mk((T)0, (T)0);
    }
    PL::template run<kPadX<T>>(z, L, 1, t, tw, WarpSync());
    // real-to-complex split X_k = (Z_k + conj Z_{M-k})/2 - i W_nx^k (Z_k - conj Z_{M-k})/2, k = 0..M
#pragma unroll
    for (int q = 0; q < E; ++q) L[xpos<kPadX<T>>(t + P * q, 1)] = z[q];
    __syncwarp();
    if (valid) {
      const T hf = (T)0.5;
      CT* X = spec + (long long)nxh * line;
#pragma unroll
      for (int q = 0; q <= E; ++q) {
        const int kk = q < E ? t + P * q : M;
        if (q == E && t != 0) break;
        const CT a = L[xpos<kPadX<T>>(kk == M ? 0 : kk, 1)];
        const CT b = cconj(L[xpos<kPadX<T>>(kk == 0 ? 0 : M - kk, 1)]);
        const CT e = mk(hf * (a.x + b.x), hf * (a.y + b.y));
        const CT dd = csub(a, b);
        const CT o = mk(hf * dd.y, -hf * dd.x);  // (a-b)/(2i)
        X[kk] = cadd(e, cmul(__ldg(twr + kk), o));
      }
    }
    __syncwarp();
  }
  if (mode >= 3) return;  // mode 3: its maximum was taken where the divergence was formed; 4: a plain transform
  for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
  if (lane == 0) wred[warp] = dmax;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = wred[0];
    for (int w = 1; w < kXWarps; ++w) v = fmax(v, wred[w]);
    atomic_max_nonneg(&sc->divmax1, v);
  }
}

template <class T, class PL>
__global__ void __launch_bounds__(32 * kXWarps, 4) k_xifft_r(Geo<T> g, const typename CplxOf<T>::type* __restrict__ spec,
                                                         T* __restrict__ phi,
                                                         const typename CplxOf<T>::type* __restrict__ tw,
                                                         const typename CplxOf<T>::type* __restrict__ twr, T normfft,
                                                         const DevScalars* __restrict__ sc) {
  typedef typename CplxOf<T>::type CT;
  constexpr int M = PL::N, P = PL::P, E = PL::E, LPW = 32 / P;
  __shared__ CT sm[kXWarps * LPW][PL::padded_len()];
  if (sc->status) return;
  const int nx = g.nx, nxh = g.nxh;
  const int nlines = g.ny * g.nz;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int t = lane % P, slot = warp * LPW + lane / P;
  CT* L = sm[slot];
  const int ngroups = (nlines + LPW - 1) / LPW;
  for (int grp = blockIdx.x * kXWarps + warp; grp < ngroups; grp += gridDim.x * kXWarps) {
    const int line = grp * LPW + lane / P;
    const bool valid = line < nlines;
    CT z[E];
    if (valid) {
      const CT* X = spec + (long long)nxh * line;
#pragma unroll
      for (int q = 0; q < E; ++q) {
        const int kk = t + P * q;
        const CT a = X[kk];
        const CT b = cconj(X[M - kk]);
        const CT e = cadd(a, b);
        const CT o = cmul(csub(a, b), cconj(__ldg(twr + kk)));
        // Z_k = e + i o, conjugated for the forward-transform-based inverse
        z[q] = cconj(mk(e.x - o.y, e.y + o.x));
      }
    } else {
#pragma unroll
      for (int q = 0; q < E; ++q) z[q] = mk((T)0, (T)0);
    }
    PL::template run<kPadX<T>>(z, L, 1, t, tw, WarpSync());
    if (valid) {
      typedef typename CplxOf<T>::type T2;
      T2* out = reinterpret_cast<T2*>(phi + (long long)nx * line);
#pragma unroll
      for (int q = 0; q < E; ++q) out[t + P * q] = mk(z[q].x * normfft, -z[q].y * normfft);
    }
  }
}

template <class T, class PL, int LZ>
__device__ __forceinline__ void zfft_r_body(Geo<T> g, typename CplxOf<T>::type* __restrict__ spec,
                                            const typename CplxOf<T>::type* __restrict__ tw, int inverse,
                                            const DevScalars* __restrict__ sc) {
  typedef typename CplxOf<T>::type CT;
  constexpr int P = PL::P, E = PL::E;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (sc->status) return;
  CT* sm = (CT*)smem_raw;  // point p of line l at sm[p * LZ + l]
  const int ny = g.ny, nxh = g.nxh;
  const int l = threadIdx.x % LZ, t = threadIdx.x / LZ;
  const int kx = blockIdx.x * LZ + l, j = blockIdx.y;
  const bool valid = kx < nxh;
  const long long zs = (long long)nxh * ny;
  CT* col = spec + kx + (long long)nxh * j;
  CT v[E];
#pragma unroll
  for (int q = 0; q < E; ++q) {
    v[q] = valid ? col[zs * (t + P * q)] : mk((T)0, (T)0);
    if (inverse) v[q] = cconj(v[q]);
  }
  PL::template run<false>(v, sm + l, LZ, t, tw, BlockSync());
  if (valid) {
#pragma unroll
    for (int q = 0; q < E; ++q) col[zs * (t + P * q)] = inverse ? cconj(v[q]) : v[q];
  }
}
// FP64 held to two blocks per SM (80 registers); FP32 left to the compiler's own
// register choice (76 at 576 points, two blocks per SM; a minimum of one block
// raised it to 94 and cost 15%)
template <class T, class PL, int LZ>
__global__ void __launch_bounds__(LZ * PL::P, 2) k_zfft_r(Geo<T> g, typename CplxOf<T>::type* __restrict__ spec,
                                                          const typename CplxOf<T>::type* __restrict__ tw,
                                                          int inverse, const DevScalars* __restrict__ sc) {
  zfft_r_body<T, PL, LZ>(g, spec, tw, inverse, sc);
}
template <class T, class PL, int LZ>
__global__ void __launch_bounds__(LZ * PL::P) k_zfft_rf(Geo<T> g, typename CplxOf<T>::type* __restrict__ spec,
                                                        const typename CplxOf<T>::type* __restrict__ tw, int inverse,
                                                        const DevScalars* __restrict__ sc) {
  zfft_r_body<T, PL, LZ>(g, spec, tw, inverse, sc);
}

// ---------------------------------------------------------------------------
// host dispatch: returns false when the length has no plan
// ---------------------------------------------------------------------------
template <class F> static bool with_xplan(int M, F f) {
  switch (M) {
    case 384: f(PlanN384()); return true;
    case 256: f(PlanN256()); return true;
    case 128: f(PlanN128()); return true;
    case 64: f(PlanN64()); return true;
    default: return false;
  }
}
template <class F> static bool with_zplan(int nz, F f) {
  switch (nz) {
    case 576: f(PlanN576()); return true;
    case 384: f(PlanN384()); return true;
    case 256: f(PlanN256()); return true;
    case 128: f(PlanZ128()); return true;
    default: return false;
  }
}

bool xplan_exists(int m) {
  return with_xplan(m, [](auto) {});
}

static int x_grid(const ch3d_ctx* c, int lpw) {
  const long long groups = ((long long)c->ny * c->nz + lpw - 1) / lpw;
  const long long blocks = (groups + kXWarps - 1) / kXWarps;
  const long long cap = 148LL * 16;  // grid-stride beyond 16 resident blocks per SM
  return (int)(blocks < cap ? blocks : cap);
}

template <class T> static bool prsrc_r_t(ch3d_ctx* c, int mode, cudaError_t* err) {
  typedef typename CplxOf<T>::type CT;
  T** f = (T**)c->f;
  T* a = mode >= 2 ? f[10] : (mode == 1 ? f[0] : f[12]);
  T* b = mode == 1 ? f[1] : f[13];
  T* cz = mode == 1 ? f[2] : f[14];
  return with_xplan(c->nx / 2, [&](auto plan) {
    typedef decltype(plan) PL;
    if (mode >= 2)
      k_prsrc_xfft_r<T, PL, true><<<x_grid(c, 32 / PL::P), 32 * kXWarps, 0, c->stream>>>(
          make_geo<T>(c), metrics_of<T>(c), a, b, cz, (CT*)c->spec, (const CT*)c->twx, (const CT*)c->twr, mode, c->sc,
          f[3]);
    else
      k_prsrc_xfft_r<T, PL, false><<<x_grid(c, 32 / PL::P), 32 * kXWarps, 0, c->stream>>>(
          make_geo<T>(c), metrics_of<T>(c), a, b, cz, (CT*)c->spec, (const CT*)c->twx, (const CT*)c->twr, mode, c->sc,
          f[3]);
    *err = cudaGetLastError();
  });
}
bool launch_prsrc_xfft_r(ch3d_ctx* c, int mode, cudaError_t* err) {
  return c->fp32 ? prsrc_r_t<float>(c, mode, err) : prsrc_r_t<double>(c, mode, err);
}

template <class T> static bool xifft_r_t(ch3d_ctx* c, cudaError_t* err) {
  typedef typename CplxOf<T>::type CT;
  T** f = (T**)c->f;
  return with_xplan(c->nx / 2, [&](auto plan) {
    typedef decltype(plan) PL;
    k_xifft_r<T, PL><<<x_grid(c, 32 / PL::P), 32 * kXWarps, 0, c->stream>>>(
        make_geo<T>(c), (const CT*)c->spec, f[10], (const CT*)c->twx, (const CT*)c->twr, (T)c->normfft, c->sc);
    *err = cudaGetLastError();
  });
}
bool launch_xifft_r(ch3d_ctx* c, cudaError_t* err) { return c->fp32 ? xifft_r_t<float>(c, err) : xifft_r_t<double>(c, err); }

template <class T> static bool zfft_r_t(ch3d_ctx* c, int inverse, cudaError_t* err) {
  typedef typename CplxOf<T>::type CT;
  // kx lines per block: 128-byte FP64 (64-byte FP32) segments per kz.  Measured at
  // 768x384x576 FP64: 4 lines 2.79 ms per spectral group, 8 lines 2.57, 16 lines 2.91
  constexpr int LZ = 8;
  return with_zplan(c->nz, [&](auto plan) {
    typedef decltype(plan) PL;
    void (*kern)(Geo<T>, CT*, const CT*, int, const DevScalars*);
    if constexpr (sizeof(T) == 8) kern = k_zfft_r<T, PL, LZ>;
    else kern = k_zfft_rf<T, PL, LZ>;
    const size_t smem = (size_t)PL::N * LZ * sizeof(CT);
    static PerDevice attr;  // per kernel instance
    if ((*err = smem_limit_once(attr, c->device, kern, smem)) != cudaSuccess) return;
    dim3 grid((c->nxh + LZ - 1) / LZ, c->ny);
    kern<<<grid, LZ * PL::P, smem, c->stream>>>(make_geo<T>(c), (CT*)c->spec, (const CT*)c->twz, inverse, c->sc);
    *err = cudaGetLastError();
  });
}
bool launch_zfft_r(ch3d_ctx* c, int inverse, cudaError_t* err) {
  return c->fp32 ? zfft_r_t<float>(c, inverse, err) : zfft_r_t<double>(c, inverse, err);
}

}  // namespace ch3d
