// ch3d_step4.cu -- sm_100a kernels specific to the 4th-order solver
// (src/CFD_4th/m_TScheme.f90): the interpolated velocities and the RHS of the
// stage entry points, and the constant-flux forcing from the mean viscous
// stress.  The step runs the RHS and y solves as the column march of
// ch3d_march.cu (4th-order branch).  The pressure Poisson pipeline, projection and
// diagnostics are the 2nd-order kernels with their 4th-order branches.
#include "ch3d_ctx.h"
#include "ch3d_dev.cuh"

namespace ch3d {

// uxhx, uyhx, uzhx, uxhz, uyhz, uzhz (src/CFD_4th/m_TScheme.f90:209-227);
// rows jc = 1..nyc.  The jc = nyp row of uyhx / uyhz is zero (:223-226) and is
// produced by the readers.
template <class T>
__global__ void __launch_bounds__(256) k_interp4(Geo<T> g, const T* __restrict__ ux, const T* __restrict__ uy,
                                                 const T* __restrict__ uz, T* __restrict__ uxhx, T* __restrict__ uyhx,
                                                 T* __restrict__ uzhx, T* __restrict__ uxhz, T* __restrict__ uyhz,
                                                 T* __restrict__ uzhz, const DevScalars* __restrict__ sc) {
  if (sc->status) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const Nbr n = make_nbr(g, i, j, k);
  const C4<T> c(g);
  uxhx[n.c] = c.in1 * at(ux, n, n.xm) + c.in2 * at(ux, n, 0) + c.in3 * at(ux, n, n.xp) + c.in4 * at(ux, n, n.xp2);
  uyhx[n.c] = c.in1 * at(uy, n, n.xm2) + c.in2 * at(uy, n, n.xm) + c.in3 * at(uy, n, 0) + c.in4 * at(uy, n, n.xp);
  uzhx[n.c] = c.in1 * at(uz, n, n.xm2) + c.in2 * at(uz, n, n.xm) + c.in3 * at(uz, n, 0) + c.in4 * at(uz, n, n.xp);
  uxhz[n.c] = c.in1 * at(ux, n, n.zm2) + c.in2 * at(ux, n, n.zm) + c.in3 * at(ux, n, 0) + c.in4 * at(ux, n, n.zp);
  uyhz[n.c] = c.in1 * at(uy, n, n.zm2) + c.in2 * at(uy, n, n.zm) + c.in3 * at(uy, n, 0) + c.in4 * at(uy, n, n.zp);
  uzhz[n.c] = c.in1 * at(uz, n, n.zm) + c.in2 * at(uz, n, 0) + c.in3 * at(uz, n, n.zp) + c.in4 * at(uz, n, n.zp2);
}

// uyhx / uyhz at j+1: zero on the jc = nyp row
template <class T> __device__ __forceinline__ T ih_jp(const T* __restrict__ a, const Nbr& n, long long o) {
  return n.jhi ? (T)0 : __ldg(a + n.c + o + n.yp);
}

struct Interp4 {
  const void* uxhx; const void* uyhx; const void* uzhx; const void* uxhz; const void* uyhz; const void* uzhz;
};

// One component of clcRhsXYZ (src/CFD_4th/m_TScheme.f90:235-343) at one cell,
// with its Hist update; uCRF = 0.
template <class T, int C>
__device__ __forceinline__ T rhs4_comp(const Geo<T>& g, const Metrics<T>& m, const Interp4& ih,
                                       const T* __restrict__ ux, const T* __restrict__ uy, const T* __restrict__ uz,
                                       const T* __restrict__ pr, T* __restrict__ h, int i, int j, int k, T pmGamma,
                                       T pmTheta, T pmAlpha, T pmBeta) {
  const Nbr n = make_nbr(g, i, j, k);
  const C4<T> c(g);
  const int jc = j + 1;
  const T two = (T)2, quarter = (T)0.25, one = (T)1;
  const T xnu = g.xnu;
  const T IY1 = m.yinterp[jc], IY2 = one - IY1;
  if (C == 0) {
    const T* uxhx = (const T*)ih.uxhx; const T* uyhx = (const T*)ih.uyhx;
    const T* uzhx = (const T*)ih.uzhx; const T* uxhz = (const T*)ih.uxhz;
    const T IY3 = m.yinterp[jc + 1], IY4 = one - IY3;
    const T sucaj = m.rdyp[jc];
    const T ux_c = at(ux, n, 0), ux_jm = at_jm(ux, g, 0, n, 0), ux_jp = at_jp(ux, g, 0, n, 0);
    const T uxhyc = IY1 * ux_jm + IY2 * ux_c;
    const T uxhyp = IY3 * ux_c + IY4 * ux_jp;
    const T a1 = at(uxhx, n, n.xm2), a2 = at(uxhx, n, n.xm), a3 = at(uxhx, n, 0), a4 = at(uxhx, n, n.xp);
    const T h11 = c.dx1 * a1 * a1 + c.dx2 * a2 * a2 + c.dx3 * a3 * a3 + c.dx4 * a4 * a4;
    const T h12 = (ih_jp(uyhx, n, 0) * uxhyp - at(uyhx, n, 0) * uxhyc) * sucaj;
    const T h13 = c.dz1 * at(uxhz, n, n.zm) * at(uzhx, n, n.zm) + c.dz2 * at(uxhz, n, 0) * at(uzhx, n, 0) +
                  c.dz3 * at(uxhz, n, n.zp) * at(uzhx, n, n.zp) + c.dz4 * at(uxhz, n, n.zp2) * at(uzhx, n, n.zp2);
    const T d11 = c.dxx1 * at(ux, n, n.xm2) + c.dxx2 * at(ux, n, n.xm) + c.dxx3 * ux_c + c.dxx4 * at(ux, n, n.xp) +
                  c.dxx5 * at(ux, n, n.xp2);
    const T d22 = m.ap2c[jc] * ux_jp + m.ac2c[jc] * ux_c + m.am2c[jc] * ux_jm;
    const T d33 = c.dzz1 * at(ux, n, n.zm2) + c.dzz2 * at(ux, n, n.zm) + c.dzz3 * ux_c + c.dzz4 * at(ux, n, n.zp) +
                  c.dzz5 * at(ux, n, n.zp2);
    const T conv = -h11 - h12 - h13 + xnu * (d11 + d33) + g.g1;
    const T gradp = c.dx1 * at(pr, n, n.xm2) + c.dx2 * at(pr, n, n.xm) + c.dx3 * at(pr, n, 0) + c.dx4 * at(pr, n, n.xp);
    const T ho = h[n.c];
    h[n.c] = conv;
    return pmGamma * conv + pmTheta * ho - pmAlpha * gradp + two * pmBeta * d22;
  } else if (C == 1) {
    const T* uyhx = (const T*)ih.uyhx; const T* uyhz = (const T*)ih.uyhz;
    const T sucac = m.rdyc[jc], qsucac = quarter * sucac;
    const T uxhym = IY1 * at_jm(ux, g, 0, n, n.xm) + IY2 * at(ux, n, n.xm);
    const T uxhyc = IY1 * at_jm(ux, g, 0, n, 0) + IY2 * at(ux, n, 0);
    const T uxhyp = IY1 * at_jm(ux, g, 0, n, n.xp) + IY2 * at(ux, n, n.xp);
    const T uxhyu = IY1 * at_jm(ux, g, 0, n, n.xp2) + IY2 * at(ux, n, n.xp2);
    const T uzhym = IY1 * at_jm(uz, g, 2, n, n.zm) + IY2 * at(uz, n, n.zm);
    const T uzhyc = IY1 * at_jm(uz, g, 2, n, 0) + IY2 * at(uz, n, 0);
    const T uzhyp = IY1 * at_jm(uz, g, 2, n, n.zp) + IY2 * at(uz, n, n.zp);
    const T uzhyu = IY1 * at_jm(uz, g, 2, n, n.zp2) + IY2 * at(uz, n, n.zp2);
    const T h21 = c.dx1 * at(uyhx, n, n.xm) * uxhym + c.dx2 * at(uyhx, n, 0) * uxhyc + c.dx3 * at(uyhx, n, n.xp) * uxhyp +
                  c.dx4 * at(uyhx, n, n.xp2) * uxhyu;
    const T uy_c = at(uy, n, 0), uy_jp = at_jp(uy, g, 1, n, 0), uy_jm = at_jm(uy, g, 1, n, 0);
    const T h22 = ((uy_jp + uy_c) * (uy_jp + uy_c) - (uy_c + uy_jm) * (uy_c + uy_jm)) * qsucac;
    const T h23 = c.dz1 * at(uyhz, n, n.zm) * uzhym + c.dz2 * at(uyhz, n, 0) * uzhyc + c.dz3 * at(uyhz, n, n.zp) * uzhyp +
                  c.dz4 * at(uyhz, n, n.zp2) * uzhyu;
    const T d11 = c.dxx1 * at(uy, n, n.xm2) + c.dxx2 * at(uy, n, n.xm) + c.dxx3 * uy_c + c.dxx4 * at(uy, n, n.xp) +
                  c.dxx5 * at(uy, n, n.xp2);
    const T d22 = m.ap2p[jc] * uy_jp + m.ac2p[jc] * uy_c + m.am2p[jc] * uy_jm;
    const T d33 = c.dzz1 * at(uy, n, n.zm2) + c.dzz2 * at(uy, n, n.zm) + c.dzz3 * uy_c + c.dzz4 * at(uy, n, n.zp) +
                  c.dzz5 * at(uy, n, n.zp2);
    const T conv = -h21 - h22 - h23 + xnu * (d11 + d33) + g.g2;
    const T gradp = (at(pr, n, 0) - at_jm(pr, g, 3, n, 0)) * sucac;
    const T ho = h[n.c];
    h[n.c] = conv;
    return pmGamma * conv + pmTheta * ho - pmAlpha * gradp + two * pmBeta * d22;
  } else {
    const T* uzhx = (const T*)ih.uzhx; const T* uxhz = (const T*)ih.uxhz;
    const T* uyhz = (const T*)ih.uyhz; const T* uzhz = (const T*)ih.uzhz;
    const T IY3 = m.yinterp[jc + 1], IY4 = one - IY3;
    const T sucaj = m.rdyp[jc];
    const T uz_c = at(uz, n, 0), uz_jm = at_jm(uz, g, 2, n, 0), uz_jp = at_jp(uz, g, 2, n, 0);
    const T uzhyc = IY1 * uz_jm + IY2 * uz_c;
    const T uzhyp = IY3 * uz_c + IY4 * uz_jp;
    const T h31 = c.dx1 * at(uzhx, n, n.xm) * at(uxhz, n, n.xm) + c.dx2 * at(uzhx, n, 0) * at(uxhz, n, 0) +
                  c.dx3 * at(uzhx, n, n.xp) * at(uxhz, n, n.xp) + c.dx4 * at(uzhx, n, n.xp2) * at(uxhz, n, n.xp2);
    const T h32 = (ih_jp(uyhz, n, 0) * uzhyp - at(uyhz, n, 0) * uzhyc) * sucaj;
    const T b1 = at(uzhz, n, n.zm2), b2 = at(uzhz, n, n.zm), b3 = at(uzhz, n, 0), b4 = at(uzhz, n, n.zp);
    const T h33 = c.dz1 * b1 * b1 + c.dz2 * b2 * b2 + c.dz3 * b3 * b3 + c.dz4 * b4 * b4;
    const T d11 = c.dxx1 * at(uz, n, n.xm2) + c.dxx2 * at(uz, n, n.xm) + c.dxx3 * uz_c + c.dxx4 * at(uz, n, n.xp) +
                  c.dxx5 * at(uz, n, n.xp2);
    const T d22 = m.ap2c[jc] * uz_jp + m.ac2c[jc] * uz_c + m.am2c[jc] * uz_jm;
    const T d33 = c.dzz1 * at(uz, n, n.zm2) + c.dzz2 * at(uz, n, n.zm) + c.dzz3 * uz_c + c.dzz4 * at(uz, n, n.zp) +
                  c.dzz5 * at(uz, n, n.zp2);
    const T conv = -h31 - h32 - h33 + xnu * (d11 + d33) + g.g3;
    const T gradp = c.dz1 * at(pr, n, n.zm2) + c.dz2 * at(pr, n, n.zm) + c.dz3 * at(pr, n, 0) + c.dz4 * at(pr, n, n.zp);
    const T ho = h[n.c];
    h[n.c] = conv;
    return pmGamma * conv + pmTheta * ho - pmAlpha * gradp + two * pmBeta * d22;
  }
}

// Stage path: clcRhsXYZ into RhsX/Y/Z (src/CFD_4th/m_TScheme.f90:189-377)
template <class T>
__global__ void __launch_bounds__(256) k_rhs4(Geo<T> g, Metrics<T> m, Interp4 ih, const T* __restrict__ ux,
                                              const T* __restrict__ uy, const T* __restrict__ uz,
                                              const T* __restrict__ pr, T* __restrict__ hx, T* __restrict__ hy,
                                              T* __restrict__ hz, T* __restrict__ rx, T* __restrict__ ry,
                                              T* __restrict__ rz, const DevScalars* __restrict__ sc) {
  if (sc->status) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= g.nx || j >= g.ny) return;
  const T pmGamma = (T)sc->pmGamma, pmTheta = (T)sc->pmTheta, pmAlpha = (T)sc->pmAlpha, pmBeta = (T)sc->pmBeta;
  const long long idx = i + (long long)g.nx * (j + (long long)g.ny * k);
  rx[idx] = rhs4_comp<T, 0>(g, m, ih, ux, uy, uz, pr, hx, i, j, k, pmGamma, pmTheta, pmAlpha, pmBeta) + (T)sc->dpmdxns;
  ry[idx] = rhs4_comp<T, 1>(g, m, ih, ux, uy, uz, pr, hy, i, j, k, pmGamma, pmTheta, pmAlpha, pmBeta);
  rz[idx] = rhs4_comp<T, 2>(g, m, ih, ux, uy, uz, pr, hz, i, j, k, pmGamma, pmTheta, pmAlpha, pmBeta);
}

// Block partial sums of (d11q1 + d33q1 + d22q1) * dyp over ux: the mean
// viscous stress of the constant-flux forcing (src/CFD_4th/m_TScheme.f90:255-262,364-377).
template <class T>
__global__ void __launch_bounds__(128) k_visc4_partial(Geo<T> g, Metrics<T> m, const T* __restrict__ ux,
                                                       double* __restrict__ part, int rows) {
  __shared__ double red[4];
  const int i = blockIdx.x * 32 + (threadIdx.x & 31), k = blockIdx.y * 4 + (threadIdx.x >> 5);
  const int j0 = blockIdx.z * rows, j1 = min(j0 + rows, g.ny);
  double s = 0.0;
  if (i < g.nx && k < g.nz) {
    const C4<T> c(g);
    Nbr n = make_nbr(g, i, j0, k);
#pragma unroll 4
    for (int j = j0; j < j1; ++j) {
      if (j > j0) nbr_next_row(n, g, j);
      const int jc = j + 1;
      const T ux_c = at(ux, n, 0);
      const T d11 = c.dxx1 * at(ux, n, n.xm2) + c.dxx2 * at(ux, n, n.xm) + c.dxx3 * ux_c + c.dxx4 * at(ux, n, n.xp) +
                    c.dxx5 * at(ux, n, n.xp2);
      const T d22 = m.ap2c[jc] * at_jp(ux, g, 0, n, 0) + m.ac2c[jc] * ux_c + m.am2c[jc] * at_jm(ux, g, 0, n, 0);
      const T d33 = c.dzz1 * at(ux, n, n.zm2) + c.dzz2 * at(ux, n, n.zm) + c.dzz3 * ux_c + c.dzz4 * at(ux, n, n.zp) +
                    c.dzz5 * at(ux, n, n.zp2);
      s += ((double)(d11 + d33) + (double)d22) * (double)m.dyp[jc];
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0)
    part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = (red[0] + red[1]) + (red[2] + red[3]);
}

// rows per k_visc4_partial block: whole columns when the x-z plane alone gives
// about eight blocks per SM, shorter chunks on small grids
static int visc4_rows(const ch3d_ctx* c) {
  const long long cols = (long long)((c->nx + 31) / 32) * ((c->nz + 3) / 4);
  const long long chunks = (148LL * 8 + cols - 1) / cols;
  const int rows = (int)((c->ny + chunks - 1) / chunks);
  return rows < 8 ? 8 : rows;
}
static dim3 visc4_grid(const ch3d_ctx* c) {
  const int rows = visc4_rows(c);
  return dim3((c->nx + 31) / 32, (c->nz + 3) / 4, (c->ny + rows - 1) / rows);
}
int visc4_npart(const ch3d_ctx* c) {
  const dim3 g = visc4_grid(c);
  return (int)(g.x * g.y * g.z);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <class T> static Interp4 interp_of(ch3d_ctx* c) {
  Interp4 ih;
  ih.uxhx = c->ih[0]; ih.uyhx = c->ih[1]; ih.uzhx = c->ih[2];
  ih.uxhz = c->ih[3]; ih.uyhz = c->ih[4]; ih.uzhz = c->ih[5];
  return ih;
}

template <class T> static cudaError_t interp4_t(ch3d_ctx* c) {
  T** f = (T**)c->f;
  T** h = (T**)c->ih;
  k_interp4<T><<<dim3((c->nx + 31) / 32, (c->ny + 7) / 8, c->nz), dim3(32, 8), 0, c->stream>>>(
      make_geo<T>(c), f[0], f[1], f[2], h[0], h[1], h[2], h[3], h[4], h[5], c->sc);
  return cudaGetLastError();
}


template <class T> static cudaError_t rhs4_t(ch3d_ctx* c) {
  cudaError_t e = interp4_t<T>(c);
  if (e != cudaSuccess) return e;
  T** f = (T**)c->f;
  k_rhs4<T><<<dim3((c->nx + 31) / 32, (c->ny + 7) / 8, c->nz), dim3(32, 8), 0, c->stream>>>(
      make_geo<T>(c), metrics_of<T>(c), interp_of<T>(c), f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9],
      c->sc);
  return cudaGetLastError();
}
cudaError_t launch_rhs4(ch3d_ctx* c) { return c->fp32 ? rhs4_t<float>(c) : rhs4_t<double>(c); }

template <class T> static cudaError_t visc4_t(ch3d_ctx* c) {
  T** f = (T**)c->f;
  k_visc4_partial<T><<<visc4_grid(c), 128, 0, c->stream>>>(make_geo<T>(c), metrics_of<T>(c), f[0], c->part,
                                                           visc4_rows(c));
  return cudaGetLastError();
}
cudaError_t launch_visc4_partials(ch3d_ctx* c) { return c->fp32 ? visc4_t<float>(c) : visc4_t<double>(c); }

// ---------------------------------------------------------------------------
// Statistics of the 4th-order solver: the moments of clcStat
// (src/CFD_4th/m_FlowCase.f90:330-640), SumStat(35,nyp) and the gradient
// moments SumGrad(98,nyp) (HighOrderGradStat, defined at :17), FP64
// accumulation in both precision modes.  One kernel per group of moments so
// that a thread's accumulators stay in registers: group 0 the 35 SumStat
// moments, groups 1..4 SumGrad(1..26), (27..50), (51..74), (75..98).
// Blocks (j, k-chunk); blockIdx.x == ny is the nyp row (:594-631).  The
// partials are summed in a fixed order by k_stats4_finalize.
// The reference's pressure array keeps zero in its planes x = nxc+2 and
// z = nzc+2 (its halo update fills one plane above, src/CFD_4th/
// m_BC_and_Halo.f90:42-45; the array starts at zero, m_Variables.f90:85), and
// dpdxx / dpdzz of the last column and plane read it there; so do these.
// ---------------------------------------------------------------------------
constexpr int kStats4Lo[5] = {0, 0, 26, 50, 74};
constexpr int kStats4N[5] = {35, 26, 24, 24, 24};

template <class T, int GRP>
__global__ void __launch_bounds__(256) k_stats4(Geo<T> g, Geo<double> gd, Metrics<double> m, const T* __restrict__ ux,
                                                const T* __restrict__ uy, const T* __restrict__ uz,
                                                const T* __restrict__ pr, double* __restrict__ part, int kch) {
  constexpr int NQ = kStats4N[GRP], LO = kStats4Lo[GRP];
  __shared__ double wred[NQ][8];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int j = blockIdx.x;  // 0..ny-1: jc = j+1; ny: the nyp row
  const int k0 = blockIdx.y * kch, k1 = min(nz, k0 + kch);
  double A[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) A[q] = 0.0;
  // 4th-order stencil constants (src/CFD_4th/m_MeshAndMetries.f90:86-91)
  const double rdx = gd.rdx, rdz = gd.rdz, rdx2 = gd.rdx2, rdz2 = gd.rdz2;
  const double dx1 = rdx / 24.0, dx2 = -rdx * 1.125, dx3 = rdx * 1.125, dx4 = -rdx / 24.0;
  const double dz1 = rdz / 24.0, dz2 = -rdz * 1.125, dz3 = rdz * 1.125, dz4 = -rdz / 24.0;
  const double dxx1 = -rdx2 / 12.0, dxx2 = 4.0 / 3.0 * rdx2, dxx3 = -2.5 * rdx2, dxx4 = 4.0 / 3.0 * rdx2,
               dxx5 = -rdx2 / 12.0;
  const double dzz1 = -rdz2 / 12.0, dzz2 = 4.0 / 3.0 * rdz2, dzz3 = -2.5 * rdz2, dzz4 = 4.0 / 3.0 * rdz2,
               dzz5 = -rdz2 / 12.0;
  const double in1 = -1.0 / 16.0, in2 = 9.0 / 16.0, in3 = 9.0 / 16.0, in4 = -1.0 / 16.0;
  const double rdxt = rdx / 12.0, rdzt = rdz / 12.0;
  auto wx = [nx](int i) { return i < 0 ? i + nx : (i >= nx ? i - nx : i); };
  auto wz = [nz](int k) { return k < 0 ? k + nz : (k >= nz ? k - nz : k); };
  const int jc = j + 1, jm = j - 1, jp = j + 1;  // 0-based rows of jc, jc-1, jc+1
  const double InterpY1 = m.yinterp[jc], InterpY2 = 1.0 - InterpY1;
  const double cac = m.rdyc[jc];
  if (j < ny) {
    const double cacU = m.rdyc[jc + 1], caj = m.rdyp[jc];
    for (int k = k0; k < k1; ++k) {
      const int ks = wz(k - 2), km = wz(k - 1), kp = wz(k + 1), ku = wz(k + 2);
      for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const int is = wx(i - 2), im = wx(i - 1), ip = wx(i + 1), iu = wx(i + 2);
        auto U = [&](int a, int b, int c) { return (double)fld(ux, g, 0, a, b, c); };
        auto V = [&](int a, int b, int c) { return (double)fld(uy, g, 1, a, b, c); };
        auto W = [&](int a, int b, int c) { return (double)fld(uz, g, 2, a, b, c); };
        auto P = [&](int a, int b, int c) { return (double)fld(pr, g, 3, a, b, c); };
        const double uxloc = U(i, j, k), uyloc = V(i, j, k), uzloc = W(i, j, k), prloc = P(i, j, k);
        const double dudy = (uxloc - U(i, jm, k)) * cac;
        const double dvdx = dx1 * V(is, j, k) + dx2 * V(im, j, k) + dx3 * uyloc + dx4 * V(ip, j, k);
        if constexpr (GRP == 0) {
          const double uxCell = in1 * U(im, j, k) + in2 * uxloc + in3 * U(ip, j, k) + in4 * U(iu, j, k);
          const double uyCell = (uyloc + V(i, jp, k)) * 0.5;
          const double uy_xc = in1 * V(is, j, k) + in2 * V(im, j, k) + in3 * uyloc + in4 * V(ip, j, k);
          const double uy_xp = in1 * V(is, jp, k) + in2 * V(im, jp, k) + in3 * V(i, jp, k) + in4 * V(ip, jp, k);
          const double uzCell = in1 * W(i, j, km) + in2 * uzloc + in3 * W(i, j, kp) + in4 * W(i, j, ku);
          const double prloc2 = InterpY1 * (in1 * P(is, jm, k) + in2 * P(im, jm, k) + in3 * P(i, jm, k) + in4 * P(ip, jm, k)) +
                                InterpY2 * (in1 * P(is, j, k) + in2 * P(im, j, k) + in3 * prloc + in4 * P(ip, j, k));
          const double dudx = dx1 * U(im, j, k) + dx2 * uxloc + dx3 * U(ip, j, k) + dx4 * U(iu, j, k);
          const double dudz = dz1 * U(i, j, ks) + dz2 * U(i, j, km) + dz3 * uxloc + dz4 * U(i, j, kp);
          const double dvdy = (V(i, jp, k) - uyloc) * caj;
          const double dvdz = dz1 * V(i, j, ks) + dz2 * V(i, j, km) + dz3 * uyloc + dz4 * V(i, j, kp);
          const double dwdx = dx1 * W(is, j, k) + dx2 * W(im, j, k) + dx3 * uzloc + dx4 * W(ip, j, k);
          const double dwdy = (uzloc - W(i, jm, k)) * cac;
          const double dwdz = dz1 * W(i, j, km) + dz2 * uzloc + dz3 * W(i, j, kp) + dz4 * W(i, j, ku);
          const double dudxx = dxx1 * U(is, j, k) + dxx2 * U(im, j, k) + dxx3 * uxloc + dxx4 * U(ip, j, k) + dxx5 * U(iu, j, k);
          const double dudyy = m.ap2c[jc] * U(i, jp, k) + m.ac2c[jc] * uxloc + m.am2c[jc] * U(i, jm, k);
          const double dudzz = dzz1 * U(i, j, ks) + dzz2 * U(i, j, km) + dzz3 * uxloc + dzz4 * U(i, j, kp) + dzz5 * U(i, j, ku);
          const double dvdxx = dxx1 * V(is, j, k) + dxx2 * V(im, j, k) + dxx3 * uyloc + dxx4 * V(ip, j, k) + dxx5 * V(iu, j, k);
          const double dvdyy = m.ap2p[jc] * V(i, jp, k) + m.ac2p[jc] * uyloc + m.am2p[jc] * V(i, jm, k);
          const double dvdzz = dzz1 * V(i, j, ks) + dzz2 * V(i, j, km) + dzz3 * uyloc + dzz4 * V(i, j, kp) + dzz5 * V(i, j, ku);
          const double dwdxx = dxx1 * W(is, j, k) + dxx2 * W(im, j, k) + dxx3 * uzloc + dxx4 * W(ip, j, k) + dxx5 * W(iu, j, k);
          const double dwdyy = m.ap2c[jc] * W(i, jp, k) + m.ac2c[jc] * uzloc + m.am2c[jc] * W(i, jm, k);
          const double dwdzz = dzz1 * W(i, j, ks) + dzz2 * W(i, j, km) + dzz3 * uzloc + dzz4 * W(i, j, kp) + dzz5 * W(i, j, ku);
          const double vor_x = dwdy - dvdz, vor_y = dudz - dwdx, vor_z = dvdx - dudy;
          const double dudxC = (-U(iu, j, k) + 8.0 * U(ip, j, k) - 8.0 * U(im, j, k) + U(is, j, k)) * rdxt;
          const double dvdxU = dx1 * V(is, jp, k) + dx2 * V(im, jp, k) + dx3 * V(i, jp, k) + dx4 * V(ip, jp, k);
          const double dudyU = (U(i, jp, k) - uxloc) * cacU;
          const double dudzC = (InterpY1 * (-U(i, jm, ku) + 8.0 * U(i, jm, kp) - 8.0 * U(i, jm, km) + U(i, jm, ks)) +
                                InterpY2 * (-U(i, j, ku) + 8.0 * U(i, j, kp) - 8.0 * U(i, j, km) + U(i, j, ks))) * rdzt;
          auto dz4c = [&](int a) { return -V(a, j, ku) + 8.0 * V(a, j, kp) - 8.0 * V(a, j, km) + V(a, j, ks); };
          const double dvdzC = (dz4c(is) * in1 + dz4c(im) * in2 + dz4c(i) * in3 + dz4c(ip) * in4) * rdzt;
          A[0] += uxloc; A[1] += uyloc; A[2] += uzloc; A[3] += prloc;
          A[4] += uxloc * uxloc; A[5] += uyloc * uyloc; A[6] += uzloc * uzloc; A[7] += prloc * prloc;
          A[8] += uxCell * uyCell; A[9] += uyCell * uzCell; A[10] += uxCell * uzCell;
          A[11] += uxCell * prloc; A[12] += uyCell * prloc; A[13] += uzCell * prloc;
          A[14] += uxCell * uxCell * uyCell; A[15] += uyloc * uyloc * uyloc; A[16] += uzCell * uzCell * uyCell;
          A[17] += uxCell * uyCell * uyCell; A[18] += uxloc * uxloc * uxloc; A[19] += uzloc * uzloc * uzloc;
          A[20] += uxloc * uxloc * uxloc * uxloc; A[21] += uyloc * uyloc * uyloc * uyloc;
          A[22] += uzloc * uzloc * uzloc * uzloc;
          A[23] += prloc * dudx; A[24] += prloc * dvdy; A[25] += prloc * dwdz;
          A[26] += prloc2 * (dudy + dvdx);
          A[27] += uxloc * (dudxx + dudyy + dudzz); A[28] += uyloc * (dvdxx + dvdyy + dvdzz);
          A[29] += uzloc * (dwdxx + dwdyy + dwdzz);
          A[30] += (dudxC * (dvdxU + dvdx) + (dudyU + dudy) * (uy_xp - uy_xc) * caj) * 0.5;
          A[31] += dudzC * dvdzC;
          A[32] += vor_x * vor_x; A[33] += vor_y * vor_y; A[34] += vor_z * vor_z;
        } else {
          // the 24 gradients of SumVec2(3..98) in their order (:496-589); each group takes six
          auto grad = [&](int t) -> double {
            switch (t) {
              case 0: return dx1 * U(im, j, k) + dx2 * uxloc + dx3 * U(ip, j, k) + dx4 * U(iu, j, k);
              case 1: return dudy;
              case 2: return dz1 * U(i, j, ks) + dz2 * U(i, j, km) + dz3 * uxloc + dz4 * U(i, j, kp);
              case 3: return dvdx;
              case 4: return (V(i, jp, k) - uyloc) * caj;
              case 5: return dz1 * V(i, j, ks) + dz2 * V(i, j, km) + dz3 * uyloc + dz4 * V(i, j, kp);
              case 6: return dx1 * W(is, j, k) + dx2 * W(im, j, k) + dx3 * uzloc + dx4 * W(ip, j, k);
              case 7: return (uzloc - W(i, jm, k)) * cac;
              case 8: return dz1 * W(i, j, km) + dz2 * uzloc + dz3 * W(i, j, kp) + dz4 * W(i, j, ku);
              case 9: return dx1 * P(is, j, k) + dx2 * P(im, j, k) + dx3 * prloc + dx4 * P(ip, j, k);
              case 10: return (prloc - P(i, jm, k)) * cac;
              case 11: return dz1 * P(i, j, ks) + dz2 * P(i, j, km) + dz3 * prloc + dz4 * P(i, j, kp);
              case 12: return dxx1 * U(is, j, k) + dxx2 * U(im, j, k) + dxx3 * uxloc + dxx4 * U(ip, j, k) + dxx5 * U(iu, j, k);
              case 13: return m.ap2c[jc] * U(i, jp, k) + m.ac2c[jc] * uxloc + m.am2c[jc] * U(i, jm, k);
              case 14: return dzz1 * U(i, j, ks) + dzz2 * U(i, j, km) + dzz3 * uxloc + dzz4 * U(i, j, kp) + dzz5 * U(i, j, ku);
              case 15: return dxx1 * V(is, j, k) + dxx2 * V(im, j, k) + dxx3 * uyloc + dxx4 * V(ip, j, k) + dxx5 * V(iu, j, k);
              case 16: return m.ap2p[jc] * V(i, jp, k) + m.ac2p[jc] * uyloc + m.am2p[jc] * V(i, jm, k);
              case 17: return dzz1 * V(i, j, ks) + dzz2 * V(i, j, km) + dzz3 * uyloc + dzz4 * V(i, j, kp) + dzz5 * V(i, j, ku);
              case 18: return dxx1 * W(is, j, k) + dxx2 * W(im, j, k) + dxx3 * uzloc + dxx4 * W(ip, j, k) + dxx5 * W(iu, j, k);
              case 19: return m.ap2c[jc] * W(i, jp, k) + m.ac2c[jc] * uzloc + m.am2c[jc] * W(i, jm, k);
              case 20: return dzz1 * W(i, j, ks) + dzz2 * W(i, j, km) + dzz3 * uzloc + dzz4 * W(i, j, kp) + dzz5 * W(i, j, ku);
              case 21: return dxx1 * P(is, j, k) + dxx2 * P(im, j, k) + dxx3 * prloc + dxx4 * P(ip, j, k) +
                              dxx5 * (i == nx - 1 ? 0.0 : P(iu, j, k));
              case 22: return m.ap2c[jc] * P(i, jp, k) + m.ac2c[jc] * prloc + m.am2c[jc] * P(i, jm, k);
              default: return dzz1 * P(i, j, ks) + dzz2 * P(i, j, km) + dzz3 * prloc + dzz4 * P(i, j, kp) +
                              dzz5 * (k == nz - 1 ? 0.0 : P(i, j, ku));
            }
          };
          constexpr int T0 = 6 * (GRP - 1), OFF = GRP == 1 ? 2 : 0;
          if constexpr (GRP == 1) {
            A[0] += prloc * prloc * prloc;
            A[1] += prloc * prloc * prloc * prloc;
          }
#pragma unroll
          for (int t = 0; t < 6; ++t) {
            const double a = grad(T0 + t);
            A[OFF + 4 * t] += a;
            A[OFF + 4 * t + 1] += a * a;
            A[OFF + 4 * t + 2] += a * a * a;
            A[OFF + 4 * t + 3] += a * a * a * a;
          }
        }
      }
    }
  } else {
    // jc = nyp: the row above the last cell (ghost values of SetBC_and_UpdateHalo)
    const int jt = ny, jb = ny - 1;  // 0-based rows of nyp and nyc
    for (int k = k0; k < k1; ++k)
      for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const int is = wx(i - 2), im = wx(i - 1), ip = wx(i + 1);
        auto P = [&](int a, int b) { return (double)fld(pr, g, 3, a, b, k); };
        const double dudy = ((double)fld(ux, g, 0, i, jt, k) - (double)fld(ux, g, 0, i, jb, k)) * cac;
        const double dwdy = ((double)fld(uz, g, 2, i, jt, k) - (double)fld(uz, g, 2, i, jb, k)) * cac;
        if constexpr (GRP == 0) {
          const double prloc2 = InterpY1 * (in1 * P(is, jb) + in2 * P(im, jb) + in3 * P(i, jb) + in4 * P(ip, jb)) +
                                InterpY2 * (in1 * P(is, jt) + in2 * P(im, jt) + in3 * P(i, jt) + in4 * P(ip, jt));
          const double vor_x = dwdy, vor_z = -dudy;
          A[26] += prloc2 * (dudy + 0.0);
          A[32] += vor_x * vor_x;
          A[34] += vor_z * vor_z;
        } else if constexpr (GRP == 1) {  // SumVec2(7..10): dudy; SumVec2(31..34) is in group 2
          A[6] += dudy; A[7] += dudy * dudy; A[8] += dudy * dudy * dudy; A[9] += dudy * dudy * dudy * dudy;
        } else if constexpr (GRP == 2) {  // SumVec2(31..34) = group-2 slots 30-26 .. 33-26
          A[4] += dwdy; A[5] += dwdy * dwdy; A[6] += dwdy * dwdy * dwdy; A[7] += dwdy * dwdy * dwdy * dwdy;
        }
      }
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double v = A[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) wred[q][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < NQ) {
    double v = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) v += wred[threadIdx.x][q];
    part[((size_t)j * gridDim.y + blockIdx.y) * NQ + threadIdx.x] = v;
  }
  (void)LO;
}

// Adds the partials of one group to its moments: dst(LO + q, jc) += sum * inxz.
__global__ void k_stats4_finalize(const double* __restrict__ part, int nch, int nq, int lo, int stride, double inxz,
                                  double* __restrict__ dst) {
  const int j = blockIdx.x, q = threadIdx.x;
  if (q < nq) {
    double v = 0.0;
    for (int c = 0; c < nch; ++c) v += part[((size_t)j * nch + c) * nq + q];
    dst[(size_t)j * stride + lo + q] += v * inxz;
  }
}

// PrGradsum += PrGradAver (src/CFD_4th/m_FlowCase.f90:634)
__global__ void k_prgrad_add(const DevScalars* __restrict__ sc, double* __restrict__ prgradsum) {
  *prgradsum += sc->PrGradAver;
}

template <class T, int GRP> static cudaError_t stats4_group(ch3d_ctx* c, int kch, int nch, double* dst, int stride) {
  T** f = (T**)c->f;
  k_stats4<T, GRP><<<dim3(c->ny + 1, nch), 256, 0, c->stream>>>(make_geo<T>(c), make_geo<double>(c), c->m64full, f[0],
                                                                f[1], f[2], f[3], c->statpart, kch);
  k_stats4_finalize<<<c->ny + 1, 64, 0, c->stream>>>(c->statpart, nch, kStats4N[GRP], kStats4Lo[GRP], stride,
                                                    1.0 / ((double)c->nx * (double)c->nz), dst);
  return cudaGetLastError();
}

template <class T> static cudaError_t stats4_t(ch3d_ctx* c) {
  const int kch = (c->nz + 7) / 8;
  const int nch = (c->nz + kch - 1) / kch;
  double* sumstat = c->stat;
  double* sumgrad = c->stat + (size_t)35 * (c->ny + 1) + 1;  // after SumStat and PrGradsum
  cudaError_t e;
  if ((e = stats4_group<T, 0>(c, kch, nch, sumstat, 35)) != cudaSuccess) return e;
  if ((e = stats4_group<T, 1>(c, kch, nch, sumgrad, 98)) != cudaSuccess) return e;
  if ((e = stats4_group<T, 2>(c, kch, nch, sumgrad, 98)) != cudaSuccess) return e;
  if ((e = stats4_group<T, 3>(c, kch, nch, sumgrad, 98)) != cudaSuccess) return e;
  if ((e = stats4_group<T, 4>(c, kch, nch, sumgrad, 98)) != cudaSuccess) return e;
  k_prgrad_add<<<1, 1, 0, c->stream>>>(c->sc, c->stat + (size_t)35 * (c->ny + 1));
  return cudaGetLastError();
}
cudaError_t launch_stats4(ch3d_ctx* c) { return c->fp32 ? stats4_t<float>(c) : stats4_t<double>(c); }

}  // namespace ch3d
