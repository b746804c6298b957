// ch3d_tg.cu -- the Taylor-Green vortex statistic of the 2nd-order solver:
// clcStat_TG (src/CFD_2nd/m_FlowType_TGVortex.f90:87-113) writes
// xnu * sum(dissp) / (nxc nyc nzc) beside SimTime, where dissp is
// CalcDissipationRate (src/CFD_2nd/m_Tools.f90:497-540): 2 S_ij S_ij per cell
// with the reference's stencils (the diagonal strains at the cell centre, the
// shear strains averaged onto it from the four surrounding edges, 1/8 each).
// Column walk per (i, k) over a chunk of rows, FP64 accumulation whatever the
// field precision, block partials summed in a fixed order.
#include "ch3d_ctx.h"
#include "ch3d_dev.cuh"

namespace ch3d {

template <class T>
__global__ void __launch_bounds__(128) k_dissipation(Geo<T> g, Metrics<double> m, const T* __restrict__ ux,
                                                     const T* __restrict__ uy, const T* __restrict__ uz,
                                                     double* __restrict__ part, int rows) {
  __shared__ double red[4];
  const int i = blockIdx.x * 32 + (threadIdx.x & 31), k = blockIdx.y * 4 + (threadIdx.x >> 5);
  const int j0 = blockIdx.z * rows, j1 = min(j0 + rows, g.ny);
  double s = 0.0;
  if (i < g.nx && k < g.nz) {
    const double rdx = g.rdx, rdz = g.rdz, e = 0.125;
    for (int j = j0; j < j1; ++j) {
      const Nbr n = make_nbr(g, i, j, k);
      const int jc = j + 1;
      const double caj = m.rdyp[jc], cac1 = m.rdyc[jc], cac2 = m.rdyc[jc + 1], cac12 = cac1 - cac2;
      auto X = [&](long long o) { return (double)at(ux, n, o); };
      auto Y = [&](long long o) { return (double)at(uy, n, o); };
      auto Z = [&](long long o) { return (double)at(uz, n, o); };
      auto Xp = [&](long long o) { return (double)at_jp(ux, g, 0, n, o); };
      auto Xm = [&](long long o) { return (double)at_jm(ux, g, 0, n, o); };
      auto Yp = [&](long long o) { return (double)at_jp(uy, g, 1, n, o); };
      auto Zp = [&](long long o) { return (double)at_jp(uz, g, 2, n, o); };
      auto Zm = [&](long long o) { return (double)at_jm(uz, g, 2, n, o); };
      const double st1 = (X(n.xp) - X(0)) * rdx;
      const double st2 = (Yp(0) - Y(0)) * caj;
      const double st3 = (Z(n.zp) - Z(0)) * rdz;
      const double st4 = e * ((Yp(n.xp) - Yp(n.xm) + Y(n.xp) - Y(n.xm)) * rdx + (Xp(n.xp) + Xp(0)) * cac2 +
                              (X(n.xp) + X(0)) * cac12 - (Xm(n.xp) + Xm(0)) * cac1);
      const double st5 = e * ((X(n.xp + n.zp) + X(n.zp) - X(n.xp + n.zm) - X(n.zm)) * rdz +
                              (Z(n.xp + n.zp) - Z(n.xm + n.zp) + Z(n.xp) - Z(n.xm)) * rdx);
      const double st6 = e * ((Yp(n.zp) + Y(n.zp) - Yp(n.zm) - Y(n.zm)) * rdz + (Zp(n.zp) + Zp(0)) * cac2 +
                              (Z(n.zp) + Z(0)) * cac12 - (Zm(n.zp) + Zm(0)) * cac1);
      s += 2.0 * (st1 * st1 + st2 * st2 + st3 * st3) + 4.0 * (st4 * st4 + st5 * st5 + st6 * st6);
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0)
    part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = (red[0] + red[1]) + (red[2] + red[3]);
}

// rows per block: whole columns when the x-z plane alone gives about eight
// blocks per SM, shorter chunks on small grids (the grid of k_diag, so the
// partials fit the step's second partial-sum buffer)
static dim3 dissipation_grid(const ch3d_ctx* c, int* rows) {
  const long long cols = (long long)((c->nx + 31) / 32) * ((c->nz + 3) / 4);
  const long long chunks = (148LL * 8 + cols - 1) / cols;
  int r = (int)((c->ny + chunks - 1) / chunks);
  if (r < 8) r = 8;
  *rows = r;
  return dim3((c->nx + 31) / 32, (c->nz + 3) / 4, (c->ny + r - 1) / r);
}

template <class T> static cudaError_t dissipation_t(ch3d_ctx* c, int* npart) {
  T** f = (T**)c->f;
  int rows = 0;
  const dim3 grid = dissipation_grid(c, &rows);
  *npart = (int)(grid.x * grid.y * grid.z);
  k_dissipation<T><<<grid, 128, 0, c->stream>>>(make_geo<T>(c), c->m64full, f[0], f[1], f[2], c->part2, rows);
  return cudaGetLastError();
}
cudaError_t launch_dissipation(ch3d_ctx* c, int* npart) {
  return c->fp32 ? dissipation_t<float>(c, npart) : dissipation_t<double>(c, npart);
}

}  // namespace ch3d
