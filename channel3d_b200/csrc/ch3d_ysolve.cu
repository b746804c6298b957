// ch3d_ysolve.cu -- the wall-normal tridiagonal solves of the pressure Poisson
// equation (clcPPE_z1, src/CFD_2nd/m_Poisson.f90:1126-1150: one system
// [am2Pr, ac2Pr + wx(kx) + wz(kz), ap2Pr] per (kx, kz), InverseTridiagonal,
// src/CFD_2nd/m_Tools.f90:224-251; row 1 of the (0,0) system pinned,
// :1136-1140) as a partitioned Thomas solve whose columns stay on chip.
//
// A block walks tiles of kYC consecutive kx columns of one kz plane of the
// (kx, j, kz) half spectrum.  All its threads copy a tile into shared memory
// row by row (cp.async, coalesced along kx), the next tile while the current
// one is solved (two buffers).  Warp w then solves column w: lane l owns the
// chunk of L rows [l L, l L + L).  The Thomas factors
//   rm_j = 1 / (b_j - a_j cp_{j-1}),  cp_j = c_j rm_j
// are computed in registers on the fly (FP64, the operations of the
// once-per-run factor tables of the one-column-per-thread kernel), each chunk
// starting from cp at the row before it, read from a small table of the chunk
// boundaries (computed once per run).  The two linear recurrences of the
// solve, d_j = (f_j - a_j d_{j-1}) rm_j and x_j = d_j - cp_j x_{j+1}, run
// chunk-parallel: every lane first sweeps its rows from a zero start, the
// chunk carries (the value at the chunk's edge and the product of the
// multipliers) are combined across the lanes by a warp-shuffle scan, and
// every lane then sweeps again from its true start.  d and then x overwrite
// the column in shared memory, and the tile is written back row by row.  The
// spectrum crosses HBM once in each direction: no factor tables of the
// spectrum's size and no forward values are stored in HBM.
//
// Shared-memory layout of a tile: column w, row j = l L + u at 16-byte unit
// w S + ((l (L+1) + u) ^ (w & 7)), S = 32 (L+1) (for 8-byte FP32 units the XOR
// term is doubled): the one-unit gap per chunk keeps a warp's lanes (rows L
// apart) in distinct banks, the XOR keeps the kYC columns of one row in
// distinct banks for the row-wise copies.
//
// Mixed path: the FP32 kernel skips the low modes kx < KX, |kz| <= KL, which
// a second launch with FP64 arithmetic solves (FP64 factors, FP64 forward
// values in shared memory, FP32 spectrum).
#include "ch3d_ctx.h"
#include "ch3d_dev.cuh"

namespace ch3d {

constexpr int kYC = 8;  // kx columns per tile = warps per block

template <class R> struct Pair2;
template <> struct Pair2<double> { typedef double2 type; };
template <> struct Pair2<float> { typedef float2 type; };

// Thomas factor of row j (0-based) from cp of the row below: the operations of
// the factor tables (k_ythomas_factors, ch3d_step.cu).
__device__ __forceinline__ double ythomas_rm(const Metrics<double>& m, double lam, bool pin, int j, double cpprev,
                                             double* cpj) {
  const int jc = j + 1;
  double a = m.am2Pr[jc], c = m.ap2Pr[jc], b = m.ac2Pr[jc] + lam;
  if (pin && j == 0) { a = 0.0; b = 1.0; c = 0.0; }
  const double rm = 1.0 / (j == 0 ? b : b - a * cpprev);
  *cpj = c * rm;
  return rm;
}

// cp at the row before every chunk, per (kx, |kz|) and lane chunk l of L rows:
// cpB[(kzh * 32 + l) * nxh + kx] = cp_{l L - 1} (zero for l = 0).
__global__ void __launch_bounds__(128) k_ychunk_bounds(Metrics<double> m, const double* __restrict__ wave, int nx,
                                                       int ny, int nxh, int L, double* __restrict__ cpB) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, kzh = blockIdx.y;
  if (kx >= nxh) return;
  const double lam = wave[kx] + wave[nx + kzh];
  const bool pin = (kx == 0 && kzh == 0);
  double cp = 0.0;
  for (int l = 0; l < 32; ++l) cpB[((size_t)kzh * 32 + l) * nxh + kx] = 0.0;
  for (int j = 0; j < ny; ++j) {
    double cpj;
    ythomas_rm(m, lam, pin, j, cp, &cpj);
    cp = cpj;
    if ((j + 1) % L == 0 && (j + 1) / L < 32) cpB[((size_t)kzh * 32 + (j + 1) / L) * nxh + kx] = cp;
  }
}

// MODE 0: every column (FP64 path); 1: every column but the low modes (mixed,
// FP32); 2: the low modes only (mixed, FP64 arithmetic; tiles kz = 0..KL,
// nz-KL..nz-1 of the first kYC kx).  L rows per lane.  Persistent blocks walk
// the tiles with a stride of the grid.
template <class T, class R, int MODE, int L>
__global__ void __launch_bounds__(32 * kYC) k_ychunk(Geo<T> g, Metrics<double> m, const double* __restrict__ wave,
                                                    const double* __restrict__ cpB,
                                                    typename CplxOf<T>::type* __restrict__ spec, int KL, int KX,
                                                    int ntiles, const DevScalars* __restrict__ sc) {
  typedef typename CplxOf<T>::type CT;
  typedef typename Pair2<R>::type RT;
  constexpr int S = 32 * (L + 1);  // units per column
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (sc->status) return;
  const int nxh = g.nxh, ny = g.ny, nz = g.nz;
  const int gx = (nxh + kYC - 1) / kYC;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  RT* const tiles = (RT*)smem_raw;  // two tiles of kYC * S units
  // 8-byte units (FP32 pairs): two rows of a copy step share a bank group, so the XOR moves up a bit
  constexpr int SW = sizeof(RT) == 8 ? 1 : 0;
  auto unit = [](int col, int row) {
    const int l = row / L, u = row - l * L;
    return col * S + ((l * (L + 1) + u) ^ ((col & 7) << SW));
  };
  auto tile_kx0 = [&](int t) { return MODE == 2 ? 0 : (t % gx) * kYC; };
  auto tile_kz = [&](int t) {
    const int b = MODE == 2 ? t : t / gx;
    return MODE == 2 ? (b <= KL ? b : nz - (b - KL)) : b;
  };
  auto col_active = [&](int kx, int kz) {
    const int kzh = kz <= nz - kz ? kz : nz - kz;
    const bool low = kx < KX && kzh <= KL;
    return kx < nxh && (MODE == 0 || (MODE == 1 ? !low : low));
  };
  // row-wise copy of tile t into buffer bb: consecutive threads take consecutive kx
  auto issue = [&](int t, int bb) {
    if (t < ntiles) {
      const int kx0 = tile_kx0(t), kz = tile_kz(t);
      const CT* src = spec + (size_t)nxh * ny * kz + kx0;
      RT* dst = tiles + (size_t)bb * kYC * S;
      for (int e = threadIdx.x; e < ny * kYC; e += 32 * kYC) {
        const int row = e / kYC, col = e - row * kYC;
        if (!col_active(kx0 + col, kz)) continue;
        if constexpr (sizeof(CT) == sizeof(RT)) {
          cp_async_el(dst + unit(col, row), (const RT*)(src + (size_t)nxh * row + col));
        } else {
          const CT v = src[(size_t)nxh * row + col];
          dst[unit(col, row)] = RT{(R)v.x, (R)v.y};
        }
      }
    }
    cp_async_commit();
  };
  const int j0 = lane * L;
  const int nr = max(0, min(L, ny - j0));
  issue(blockIdx.x, 0);
  int it = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
    const int bb = it & 1;
    issue(t + gridDim.x, bb ^ 1);
    cp_async_wait<1>();
    __syncthreads();  // tile t complete in buffer bb
    const int kx0 = tile_kx0(t), kz = tile_kz(t);
    const int kx = kx0 + w, kzh = kz <= nz - kz ? kz : nz - kz;
    RT* const ct = tiles + (size_t)bb * kYC * S;
    if (col_active(kx, kz)) {  // warp-uniform: warp w solves column kx
      const bool pin = (kx == 0 && kz == 0);
      R rm[L], cp[L];
      {
        const double lam = wave[kx] + wave[g.nx + kzh];
        double cpprev = __ldg(cpB + ((size_t)kzh * 32 + lane) * nxh + kx);
#pragma unroll
        for (int u = 0; u < L; ++u) {
          double r = 1.0, cpj = 0.0;
          if (u < nr) r = ythomas_rm(m, lam, pin, j0 + u, cpprev, &cpj);
          cpprev = cpj;
          rm[u] = (R)r;
          cp[u] = (R)cpj;
        }
      }
      // forward sweep from a zero start: carry (delta, pi) with d_end = delta + pi d_{start-1}
      R dx = (R)0, dy = (R)0, pi = (R)1;
#pragma unroll
      for (int u = 0; u < L; ++u)
        if (u < nr) {
          RT f = ct[unit(w, j0 + u)];
          if (pin && j0 + u == 0) f = RT{(R)0, (R)0};
          const R a = (R)__ldg(m.am2Pr + j0 + u + 1);
          dx = (f.x - a * dx) * rm[u];
          dy = (f.y - a * dy) * rm[u];
          pi = -a * rm[u] * pi;
        }
      // inclusive scan over the lanes: composing chunk a then b gives (delta_b + pi_b delta_a, pi_a pi_b)
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const R qx = __shfl_up_sync(0xffffffffu, dx, o), qy = __shfl_up_sync(0xffffffffu, dy, o);
        const R qp = __shfl_up_sync(0xffffffffu, pi, o);
        if (lane >= o) {
          dx = dx + pi * qx;
          dy = dy + pi * qy;
          pi = pi * qp;
        }
      }
      // d_{start-1} of this chunk: the inclusive value of the lane below
      R Dx = __shfl_up_sync(0xffffffffu, dx, 1), Dy = __shfl_up_sync(0xffffffffu, dy, 1);
      if (lane == 0) { Dx = (R)0; Dy = (R)0; }
#pragma unroll
      for (int u = 0; u < L; ++u)
        if (u < nr) {
          RT f = ct[unit(w, j0 + u)];
          if (pin && j0 + u == 0) f = RT{(R)0, (R)0};
          const R a = (R)__ldg(m.am2Pr + j0 + u + 1);
          Dx = (f.x - a * Dx) * rm[u];
          Dy = (f.y - a * Dy) * rm[u];
          ct[unit(w, j0 + u)] = RT{Dx, Dy};
        }
      // backward sweep from a zero end: carry (xi, rho) with x_start = xi + rho x_{end+1}
      R xx = (R)0, xy = (R)0, rho = (R)1;
#pragma unroll
      for (int u = L - 1; u >= 0; --u)
        if (u < nr) {
          const RT d = ct[unit(w, j0 + u)];
          xx = d.x - cp[u] * xx;
          xy = d.y - cp[u] * xy;
          rho = -cp[u] * rho;
        }
      // inclusive scan from the top lane down: chunk l then l+1 gives (xi_l + rho_l xi_{l+1}, rho_l rho_{l+1})
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const R qx = __shfl_down_sync(0xffffffffu, xx, o), qy = __shfl_down_sync(0xffffffffu, xy, o);
        const R qr = __shfl_down_sync(0xffffffffu, rho, o);
        if (lane + o < 32) {
          xx = xx + rho * qx;
          xy = xy + rho * qy;
          rho = rho * qr;
        }
      }
      // x_{end+1} of this chunk: the inclusive value of the lane above
      R Bx = __shfl_down_sync(0xffffffffu, xx, 1), By = __shfl_down_sync(0xffffffffu, xy, 1);
      if (lane == 31) { Bx = (R)0; By = (R)0; }
#pragma unroll
      for (int u = L - 1; u >= 0; --u)
        if (u < nr) {
          const RT d = ct[unit(w, j0 + u)];
          Bx = d.x - cp[u] * Bx;
          By = d.y - cp[u] * By;
          ct[unit(w, j0 + u)] = RT{Bx, By};
        }
    }
    __syncthreads();  // every column of the tile solved
    {
      CT* dstg = spec + (size_t)nxh * ny * kz + kx0;
      for (int e = threadIdx.x; e < ny * kYC; e += 32 * kYC) {
        const int row = e / kYC, col = e - row * kYC;
        if (!col_active(kx0 + col, kz)) continue;
        const RT v = ct[unit(col, row)];
        dstg[(size_t)nxh * row + col] = mk((T)v.x, (T)v.y);
      }
    }
    __syncthreads();  // the buffer read back before the copy of tile t + 2 gridDim.x lands in it
  }
  cp_async_wait<0>();
}

// rows per lane of the partitioned solve: ny <= 32 L, L one of the compiled chunk lengths
static int ychunk_rows(int ny) {
  const int L = (ny + 31) / 32;
  return L <= 4 ? 4 : (L <= 8 ? 8 : (L <= 12 ? 12 : (L <= 16 ? 16 : 0)));
}

// Partitioned solve for grids of 64 <= ny <= 512 rows whose low-mode band fits
// one tile; the one-column-per-thread kernel serves the others.
bool ychunk_usable(const ch3d_ctx* c) { return c->ny >= 64 && ychunk_rows(c->ny) > 0 && c->TSy <= kYC; }

size_t ychunk_bound_doubles(const ch3d_ctx* c) { return (size_t)(c->nz / 2 + 1) * 32 * c->nxh; }

cudaError_t launch_ychunk_bounds(ch3d_ctx* c) {
  k_ychunk_bounds<<<dim3((c->nxh + 127) / 128, c->nz / 2 + 1), 128, 0, c->stream>>>(
      c->m64full, c->wave, c->nx, c->ny, c->nxh, ychunk_rows(c->ny), c->yB);
  return cudaGetLastError();
}

template <class T, class R, int MODE, int L> static cudaError_t ychunk_launch(ch3d_ctx* c, int ntiles) {
  auto kern = k_ychunk<T, R, MODE, L>;
  const size_t smem = (size_t)2 * kYC * 32 * (L + 1) * sizeof(typename Pair2<R>::type);
  static PerDevice attr;  // per instance
  cudaError_t e = smem_limit_once(attr, c->device, kern, smem);
  if (e != cudaSuccess) return e;
  int bps = 0;  // persistent grid: the resident blocks of every SM
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, 32 * kYC, smem)) != cudaSuccess) return e;
  const long long cap = (long long)sm_count(c->device) * (bps > 0 ? bps : 1);
  typedef typename CplxOf<T>::type CT;
  kern<<<(unsigned)(ntiles < cap ? ntiles : cap), 32 * kYC, smem, c->stream>>>(
      make_geo<T>(c), c->m64full, c->wave, c->yB, (CT*)c->spec, c->KL, c->TSy, ntiles, c->sc);
  return cudaGetLastError();
}

template <int L> static cudaError_t ychunk_rows_launch(ch3d_ctx* c) {
  const int ntiles = ((c->nxh + kYC - 1) / kYC) * c->nz;
  if (!c->fp32) return ychunk_launch<double, double, 0, L>(c, ntiles);
  cudaError_t e = ychunk_launch<float, double, 2, L>(c, 2 * c->KL + 1);  // FP64 low modes (TSy <= kYC)
  if (e != cudaSuccess) return e;
  return ychunk_launch<float, float, 1, L>(c, ntiles);
}

cudaError_t launch_ychunk(ch3d_ctx* c) {
  switch (ychunk_rows(c->ny)) {
    case 4: return ychunk_rows_launch<4>(c);
    case 8: return ychunk_rows_launch<8>(c);
    case 12: return ychunk_rows_launch<12>(c);
    case 16: return ychunk_rows_launch<16>(c);
  }
  return cudaErrorInvalidValue;
}

}  // namespace ch3d
