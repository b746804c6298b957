// ch3d_ysolve.cu -- the wall-normal tridiagonal solves of the pressure Poisson
// equation (clcPPE_z1, src/CFD_2nd/m_Poisson.f90:1126-1150: one system
// [am2Pr, ac2Pr + wx(kx) + wz(kz), ap2Pr] per (kx, kz), InverseTridiagonal,
// src/CFD_2nd/m_Tools.f90:224-251; row 1 of the (0,0) system pinned,
// :1136-1140) as a partitioned Thomas solve whose columns stay on chip.
//
// A block owns kYC consecutive kx columns of one kz plane of the (kx, j, kz)
// half spectrum.  The columns arrive in shared memory by cp.async; each thread
// owns one chunk of kYL rows of one column.  The Thomas factors
//   rm_j = 1 / (b_j - a_j cp_{j-1}),  cp_j = c_j rm_j
// are computed in registers on the fly (FP64, the same operations as the
// once-per-run factor tables of the one-column-per-thread kernel), each chunk
// starting from cp at its first row, read from a small table of the chunk
// boundaries (computed once per run).  The two linear recurrences of the
// solve, d_j = (f_j - a_j d_{j-1}) rm_j and x_j = d_j - cp_j x_{j+1}, run
// chunk-parallel: every chunk first sweeps its rows from a zero start, the
// chunk-to-chunk carries (the value at the chunk's edge and the product of
// the multipliers) are combined across chunks by one thread per column, and
// every chunk then sweeps again from its true start.  The forward values d
// overwrite the column in shared memory; the solution is written to the
// spectrum.  The spectrum crosses HBM once in each direction: no factor
// tables of the spectrum's size and no forward values are stored in HBM.
//
// Mixed path: the FP32 kernel skips the low modes kx < KX, |kz| <= KL, which
// a second launch of the FP64 kernel solves (FP64 factors, FP64 forward values
// in shared memory, FP32 spectrum).
#include "ch3d_ctx.h"
#include "ch3d_dev.cuh"

namespace ch3d {

constexpr int kYL = 16;     // rows per chunk (per thread)
constexpr int kYC = 16;     // kx columns per tile
constexpr int kYMaxP = 32;  // chunks per column: ny <= 512

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

// cp at the last row of every chunk but the last, per (kx, |kz|):
// cpB[(kzh * P + p) * nxh + kx] = cp_{p kYL - 1}, p = 1..P-1.
__global__ void __launch_bounds__(128) k_ychunk_bounds(Metrics<double> m, const double* __restrict__ wave, int nx,
                                                       int ny, int nxh, int P, double* __restrict__ cpB) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, kzh = blockIdx.y;
  if (kx >= nxh) return;
  const double lam = wave[kx] + wave[nx + kzh];
  const bool pin = (kx == 0 && kzh == 0);
  double cp = 0.0;
  cpB[((size_t)kzh * P) * nxh + kx] = 0.0;
  for (int j = 0; j < ny; ++j) {
    double cpj;
    ythomas_rm(m, lam, pin, j, cp, &cpj);
    cp = cpj;
    if ((j + 1) % kYL == 0 && (j + 1) / kYL < P) cpB[((size_t)kzh * P + (j + 1) / kYL) * nxh + kx] = cp;
  }
}

// MODE 0: every column (FP64 path); 1: every column but the low modes (mixed,
// FP32); 2: the low modes only (mixed, FP64 arithmetic), tiles kz = 0..KL,
// nz-KL..nz-1 of the first kx tile.  Persistent blocks walk the tiles with a
// stride of the grid; the copies of a block's next tile are in flight in the
// second shared-memory buffer while the current tile is solved.
template <class T, class R, int MODE>
__global__ void __launch_bounds__(kYC * kYMaxP) k_ychunk(Geo<T> g, Metrics<double> m, const double* __restrict__ wave,
                                                        const double* __restrict__ cpB,
                                                        typename CplxOf<T>::type* __restrict__ spec, int P, int KL,
                                                        int KX, int ntiles, const DevScalars* __restrict__ sc) {
  typedef typename CplxOf<T>::type CT;
  typedef typename Pair2<R>::type RT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (sc->status) return;
  const int nxh = g.nxh, ny = g.ny, nz = g.nz;
  const int gx = (nxh + kYC - 1) / kYC;
  const int col = threadIdx.x % kYC, w = threadIdx.x / kYC;
  RT* buf0 = (RT*)smem_raw;  // two tiles [ny][kYC]
  R* s0 = (R*)(buf0 + (size_t)2 * ny * kYC);  // 5 arrays [P][kYC]: carries of the chunk sweeps
  R* s1 = s0 + P * kYC;
  R* s2 = s1 + P * kYC;
  R* s3 = s2 + P * kYC;
  R* s4 = s3 + P * kYC;
  const int j0 = w * kYL;
  const int nr = min(kYL, ny - j0);
  struct Tile { int kx, kz, kzh; bool active; };
  auto tile_of = [&](int t) {
    Tile q;
    q.kx = (MODE == 2 ? 0 : (t % gx) * kYC) + col;
    const int b = MODE == 2 ? t : t / gx;
    q.kz = MODE == 2 ? (b <= KL ? b : nz - (b - KL)) : b;
    q.kzh = q.kz <= nz - q.kz ? q.kz : nz - q.kz;
    const bool low = q.kx < KX && q.kzh <= KL;
    q.active = q.kx < nxh && (MODE == 0 || (MODE == 1 ? !low : low));
    return q;
  };
  // copies of this thread's rows of tile t into buffer bb (one commit group per tile)
  auto issue = [&](int t, int bb) {
    if (t < ntiles) {
      const Tile q = tile_of(t);
      if (q.active) {
        const CT* cg = spec + q.kx + (size_t)nxh * ny * q.kz;
        RT* ct = buf0 + (size_t)bb * ny * kYC + col;
#pragma unroll
        for (int u = 0; u < kYL; ++u)
          if (u < nr) {
            if constexpr (sizeof(CT) == sizeof(RT)) {
              cp_async_el(ct + (size_t)kYC * (j0 + u), (const RT*)(cg + (size_t)nxh * (j0 + u)));
            } else {
              const CT v = cg[(size_t)nxh * (j0 + u)];
              ct[(size_t)kYC * (j0 + u)] = RT{(R)v.x, (R)v.y};
            }
          }
      }
    }
    cp_async_commit();
  };
  issue(blockIdx.x, 0);
  int it = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
    const int bb = it & 1;
    issue(t + gridDim.x, bb ^ 1);
    const Tile q = tile_of(t);
    const bool pin = (q.kx == 0 && q.kz == 0);
    CT* cg = spec + q.kx + (size_t)nxh * ny * q.kz;  // row j at cg + nxh j
    RT* ct = buf0 + (size_t)bb * ny * kYC + col;    // row j at ct + kYC j
    // the chunk's Thomas factors, FP64 recurrence from the boundary table (overlaps the copies)
    R rm[kYL], cp[kYL];
    {
      const double lam = q.active ? wave[q.kx] + wave[g.nx + q.kzh] : 0.0;
      double cpprev = (q.active && w > 0) ? __ldg(cpB + ((size_t)q.kzh * P + w) * nxh + q.kx) : 0.0;
#pragma unroll
      for (int u = 0; u < kYL; ++u) {
        double r = 1.0, cpj = 0.0;
        if (q.active && u < nr) r = ythomas_rm(m, lam, pin, j0 + u, cpprev, &cpj);
        cpprev = cpj;
        rm[u] = (R)r;
        cp[u] = (R)cpj;
      }
    }
    cp_async_wait<1>();  // this tile's copies (the next tile's may still be in flight)
    // forward sweep from a zero start: carry (delta, pi) of d_end = delta + pi d_{start-1}
    {
      R dx = (R)0, dy = (R)0, pi = (R)1;
#pragma unroll
      for (int u = 0; u < kYL; ++u)
        if (u < nr) {
          const int j = j0 + u;
          RT f = ct[(size_t)kYC * j];
          if (pin && j == 0) f = RT{(R)0, (R)0};
          const R a = (R)m.am2Pr[j + 1];
          dx = (f.x - a * dx) * rm[u];
          dy = (f.y - a * dy) * rm[u];
          pi = -a * rm[u] * pi;
        }
      s0[w * kYC + col] = dx; s1[w * kYC + col] = dy; s2[w * kYC + col] = pi;
    }
    __syncthreads();
    if (w == 0) {  // d_{start-1} of every chunk
      R Dx = (R)0, Dy = (R)0;
      for (int p = 0; p < P; ++p) {
        s3[p * kYC + col] = Dx; s4[p * kYC + col] = Dy;
        const R px = s0[p * kYC + col], py = s1[p * kYC + col], pp = s2[p * kYC + col];
        Dx = px + pp * Dx;
        Dy = py + pp * Dy;
      }
    }
    __syncthreads();
    // forward sweep from the true start, d_j into the tile; then the backward
    // sweep from a zero end: carry (xi, rho) of x_start = xi + rho x_{end+1}
    {
      R dx = s3[w * kYC + col], dy = s4[w * kYC + col];
#pragma unroll
      for (int u = 0; u < kYL; ++u)
        if (u < nr) {
          const int j = j0 + u;
          RT f = ct[(size_t)kYC * j];
          if (pin && j == 0) f = RT{(R)0, (R)0};
          const R a = (R)m.am2Pr[j + 1];
          dx = (f.x - a * dx) * rm[u];
          dy = (f.y - a * dy) * rm[u];
          ct[(size_t)kYC * j] = RT{dx, dy};
        }
      R xx = (R)0, xy = (R)0, rho = (R)1;
#pragma unroll
      for (int u = kYL - 1; u >= 0; --u)
        if (u < nr) {
          const RT d = ct[(size_t)kYC * (j0 + u)];
          xx = d.x - cp[u] * xx;
          xy = d.y - cp[u] * xy;
          rho = -cp[u] * rho;
        }
      __syncthreads();  // every D read above before the carries overwrite the arrays
      s0[w * kYC + col] = xx; s1[w * kYC + col] = xy; s2[w * kYC + col] = rho;
    }
    __syncthreads();
    if (w == 0) {  // x_{end+1} of every chunk
      R Bx = (R)0, By = (R)0;
      for (int p = P - 1; p >= 0; --p) {
        s3[p * kYC + col] = Bx; s4[p * kYC + col] = By;
        const R px = s0[p * kYC + col], py = s1[p * kYC + col], pr = s2[p * kYC + col];
        Bx = px + pr * Bx;
        By = py + pr * By;
      }
    }
    __syncthreads();
    if (q.active) {
      R xx = s3[w * kYC + col], xy = s4[w * kYC + col];
#pragma unroll
      for (int u = kYL - 1; u >= 0; --u)
        if (u < nr) {
          const int j = j0 + u;
          const RT d = ct[(size_t)kYC * j];
          xx = d.x - cp[u] * xx;
          xy = d.y - cp[u] * xy;
          cg[(size_t)nxh * j] = mk((T)xx, (T)xy);
        }
    }
    __syncthreads();  // the carries of this tile read before the next tile's sweeps write them
  }
  cp_async_wait<0>();
}

// Partitioned solve for grids of 64 <= ny <= 512 rows whose two tiles fit in
// shared memory; the one-column-per-thread kernel serves the others.
static size_t ychunk_smem(int ny, size_t word) {
  const int P = (ny + kYL - 1) / kYL;
  return (size_t)2 * ny * kYC * 2 * word + (size_t)5 * P * kYC * word;
}

bool ychunk_usable(const ch3d_ctx* c) {
  const int P = (c->ny + kYL - 1) / kYL;
  // FP64 tiles (the mixed path's low-mode launch keeps them too)
  return c->ny >= 64 && P <= kYMaxP && ychunk_smem(c->ny, sizeof(double)) <= 220 * 1024;
}

size_t ychunk_bound_doubles(const ch3d_ctx* c) {
  const int P = (c->ny + kYL - 1) / kYL;
  return (size_t)(c->nz / 2 + 1) * P * c->nxh;
}

cudaError_t launch_ychunk_bounds(ch3d_ctx* c) {
  const int P = (c->ny + kYL - 1) / kYL;
  k_ychunk_bounds<<<dim3((c->nxh + 127) / 128, c->nz / 2 + 1), 128, 0, c->stream>>>(c->m64full, c->wave, c->nx, c->ny,
                                                                                    c->nxh, P, c->yB);
  return cudaGetLastError();
}

template <class T, class R, int MODE> static cudaError_t ychunk_launch(ch3d_ctx* c, int ntiles, int P) {
  auto kern = k_ychunk<T, R, MODE>;
  const size_t smem = ychunk_smem(c->ny, sizeof(R));
  static PerDevice attr;  // per instance
  cudaError_t e = smem_limit_once(attr, c->device, kern, 220 * 1024);
  if (e != cudaSuccess) return e;
  int bps = 0;  // persistent grid: the resident blocks of every SM
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, kYC * P, smem)) != cudaSuccess) return e;
  const long long cap = (long long)sm_count(c->device) * (bps > 0 ? bps : 1);
  const unsigned grid = (unsigned)(ntiles < cap ? ntiles : cap);
  typedef typename CplxOf<T>::type CT;
  kern<<<grid, kYC * P, smem, c->stream>>>(make_geo<T>(c), c->m64full, c->wave, c->yB, (CT*)c->spec, P, c->KL, c->TSy,
                                           ntiles, c->sc);
  return cudaGetLastError();
}

cudaError_t launch_ychunk(ch3d_ctx* c) {
  const int P = (c->ny + kYL - 1) / kYL;
  const int gx = (c->nxh + kYC - 1) / kYC;
  if (!c->fp32) return ychunk_launch<double, double, 0>(c, gx * c->nz, P);
  cudaError_t e = ychunk_launch<float, double, 2>(c, 2 * c->KL + 1, P);  // FP64 low modes
  if (e != cudaSuccess) return e;
  return ychunk_launch<float, float, 1>(c, gx * c->nz, P);
}

}  // namespace ch3d
