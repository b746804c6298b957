// ch3d_interp.cu -- resampling of a channel state onto another grid, the
// reference's interpolateField tool (Tool/interpolateField/src/m_Interp.f90):
// Interp_init (:20-179) builds, per axis and staggered position, the index of
// the old cell below each new point and the linear weight; Interp_uvwp
// (:184-361) interpolates ux at (xp, yc, zc), uy at (xc, yp, zc), uz at
// (xc, yc, zp) and p at (xc, yc, zc) trilinearly from the old field with its
// ghost cells (the tool's SetBC_and_UpdateHalo_*, Tool/interpolateField/src/
// m_BC_and_Halo.f90:21-340, periodic x and z), and rescales ux to the bulk
// velocity when the flow rate is held constant (:225-236).  x and z
// coordinates are normalised by the domain length
// (Tool/interpolateField/src/m_MeshAndMetries.f90:40-59); y is the physical
// coordinate of both grids on the same height.  Both states live on the same
// GPU; the tables are built on the host and each new value is one thread.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ch3d_ctx.h"
#include "ch3d_dev.cuh"

namespace ch3d {

struct InterpAxis {
  const int* ind;       // old index below the new point (Fortran, 0..n)
  const double* rat;    // weight of that old point
};

struct OldGrid {
  int nx, ny, nz;
  int bc_lo, bc_hi;                    // BcOption(3), BcOption(4)
  double w_lo[3], w_hi[3];             // ux, uy, uz wall values at y- and y+
};

// Old value at Fortran (i, j, k), i in 0..nx+1, j in 0..ny+1, k in 0..nz+1,
// with the tool's ghost rules.  comp: 0 ux, 1 uy, 2 uz, 3 p.
template <class T>
__device__ __forceinline__ double old_at(const T* __restrict__ a, const OldGrid& o, int comp, int i, int j, int k) {
  i = i == 0 ? o.nx : (i == o.nx + 1 ? 1 : i);
  k = k == 0 ? o.nz : (k == o.nz + 1 ? 1 : k);
  auto v = [&](int jj) { return (double)__ldg(a + (i - 1) + (size_t)o.nx * ((jj - 1) + (size_t)o.ny * (k - 1))); };
  if (comp == 3) return v(j == 0 ? 1 : (j == o.ny + 1 ? o.ny : j));
  if (comp == 1) {  // uy(:,1,:) and uy(:,nyp,:) are the wall values; uy(:,0,:) is never read
    if (j == 1) return o.bc_lo == -1 ? o.w_lo[1] : 0.0;
    if (j == o.ny + 1) return o.bc_hi == -1 ? o.w_hi[1] : 0.0;
    if (j == 0) return 0.0;
    return v(j);
  }
  if (j == 0) return o.bc_lo == -1 ? o.w_lo[comp] * 2.0 - v(1) : v(1);
  if (j == o.ny + 1) return o.bc_hi == -1 ? o.w_hi[comp] * 2.0 - v(o.ny) : v(o.ny);
  return v(j);
}

template <class T>
__global__ void __launch_bounds__(128) k_interp(OldGrid o, int comp, const T* __restrict__ src, InterpAxis X,
                                                InterpAxis Y, InterpAxis Z, int nxn, int nyn, T* __restrict__ dst) {
  const int ic = blockIdx.x * blockDim.x + threadIdx.x + 1, jc = blockIdx.y + 1, kc = blockIdx.z + 1;
  if (ic > nxn) return;
  const int idz1 = Z.ind[kc], idz2 = idz1 + 1;
  const double prz1 = Z.rat[kc], prz2 = 1.0 - prz1;
  const int idy1 = Y.ind[jc], idy2 = idy1 + 1;
  const double pry1 = Y.rat[jc], pry2 = 1.0 - pry1;
  const int idx1 = X.ind[ic], idx2 = idx1 + 1;
  const double prx1 = X.rat[ic], prx2 = 1.0 - prx1;
  auto A = [&](int i, int j, int k) { return old_at(src, o, comp, i, j, k); };
  const double v = A(idx1, idy1, idz1) * prx1 * pry1 * prz1 + A(idx2, idy1, idz1) * prx2 * pry1 * prz1 +
                   A(idx1, idy2, idz1) * prx1 * pry2 * prz1 + A(idx2, idy2, idz1) * prx2 * pry2 * prz1 +
                   A(idx1, idy1, idz2) * prx1 * pry1 * prz2 + A(idx2, idy1, idz2) * prx2 * pry1 * prz2 +
                   A(idx1, idy2, idz2) * prx1 * pry2 * prz2 + A(idx2, idy2, idz2) * prx2 * pry2 * prz2;
  dst[(ic - 1) + (size_t)nxn * ((jc - 1) + (size_t)nyn * (kc - 1))] = (T)v;
}

// Flow-rate rescale (:225-236): per (j, k) row the sum of ux * dy(j) ...
template <class T>
__global__ void k_interp_rowsum(const T* __restrict__ ux, const double* __restrict__ dyn, int nx, int ny, int nz,
                                double* __restrict__ rows) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= ny * nz) return;
  const int j = r % ny;
  const T* a = ux + (size_t)nx * r;
  double s = 0.0;
  for (int i = 0; i < nx; ++i) s += (double)a[i] * dyn[j];
  rows[r] = s;
}

// ... then one block sums the rows in a fixed order and scales ux by
// ubulk / mean.
template <class T>
__global__ void __launch_bounds__(256) k_interp_rescale(T* __restrict__ ux, const double* __restrict__ rows,
                                                        long long nrow, long long n, double inv, double ubulk) {
  __shared__ double sh[256];
  __shared__ double scale;
  double s = 0.0;
  for (long long r = threadIdx.x; r < nrow; r += blockDim.x) s += rows[r];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) scale = ubulk / (sh[0] * inv);
  __syncthreads();
  for (long long q = threadIdx.x; q < n; q += blockDim.x) ux[q] = (T)(scale * (double)ux[q]);
}

namespace {

// Interp_init tables of one axis position: new points pN[1..nn] in old points
// pO[0..no+1] (uniform spacing 1/no, normalised); `centred` for cell centres.
void uniform_table(int nn, int no, const std::vector<double>& pN, const std::vector<double>& pO, bool centred,
                   std::vector<int>& ind, std::vector<double>& rat) {
  ind.assign(nn + 1, 0);
  rat.assign(nn + 1, 0.0);
  const double rd = (double)no;
  for (int i = 1; i <= nn; ++i) {
    int ic = (int)std::floor(pN[i] * rd) + 1;
    ic = std::min(ic, no);
    ic = std::max(ic, 1);
    if (centred && pN[i] < pO[ic]) ic = ic - 1;
    ind[i] = ic;
    rat[i] = (pO[ic + 1] - pN[i]) * rd;
  }
}

void norm_points(int n, std::vector<double>& xp, std::vector<double>& xc) {
  xp.assign(n + 2, 0.0);
  xc.assign(n + 2, 0.0);
  for (int j = 1; j <= n + 1; ++j) xp[j] = (double)(j - 1) / (double)n;
  xp[1] = 0.0;
  xp[n + 1] = 1.0;
  for (int j = 1; j <= n; ++j) xc[j] = 0.5 * (xp[j] + xp[j + 1]);
  xc[0] = 2.0 * xp[1] - xc[1];
  xc[n + 1] = 2.0 * xp[n + 1] - xc[n];
}

}  // namespace

template <class T> static cudaError_t interp_t(ch3d_ctx* dst, const ch3d_ctx* src) {
  const int nxo = src->nx, nyo = src->ny, nzo = src->nz, nxn = dst->nx, nyn = dst->ny, nzn = dst->nz;
  const int nypo = nyo + 1;
  std::vector<double> xpO, xcO, xpN, xcN, zpO, zcO, zpN, zcN;
  norm_points(nxo, xpO, xcO);
  norm_points(nxn, xpN, xcN);
  norm_points(nzo, zpO, zcO);
  norm_points(nzn, zpN, zcN);
  std::vector<double> ypO(nypo + 1), ycO(nypo + 1), ypN(nyn + 2), ycN(nyn + 2), dyn(nyn);
  for (int j = 1; j <= nypo; ++j) ypO[j] = src->yp[j];
  for (int j = 1; j <= nyn + 1; ++j) ypN[j] = dst->yp[j];
  for (int j = 1; j <= nyo; ++j) ycO[j] = 0.5 * (ypO[j] + ypO[j + 1]);
  ycO[0] = 2.0 * ypO[1] - ycO[1];
  ycO[nypo] = 2.0 * ypO[nypo] - ycO[nyo];
  for (int j = 1; j <= nyn; ++j) ycN[j] = 0.5 * (ypN[j] + ypN[j + 1]);
  for (int j = 1; j <= nyn; ++j) dyn[j - 1] = ypN[j + 1] - ypN[j];
  std::vector<int> ixp, ixc, izp, izc, iyp(nyn + 1, 0), iyc(nyn + 1, 0);
  std::vector<double> rxp, rxc, rzp, rzc, ryp(nyn + 1, 0.0), ryc(nyn + 1, 0.0);
  uniform_table(nxn, nxo, xpN, xpO, false, ixp, rxp);
  uniform_table(nxn, nxo, xcN, xcO, true, ixc, rxc);
  uniform_table(nzn, nzo, zpN, zpO, false, izp, rzp);
  uniform_table(nzn, nzo, zcN, zcO, true, izc, rzc);
  auto ysearch = [&](double y) {  // the tool's bisection (:148-156): largest jc with ypO(jc) <= y
    int js = 0, je = nypo + 1, jc;
    for (;;) {
      jc = (js + je) / 2;
      if (je - js == 1) break;
      if (y < ypO[jc]) je = jc; else js = jc;
    }
    return jc;
  };
  for (int j = 1; j <= nyn; ++j) {
    int jc = ysearch(ypN[j]);
    if (jc < 1 || jc > nyo) return cudaErrorInvalidValue;  // "wrong jc 1"
    iyp[j] = jc;
    ryp[j] = (ypO[jc + 1] - ypN[j]) / (ypO[jc + 1] - ypO[jc]);
    jc = ysearch(ycN[j]);
    if (jc < 1 || jc > nyo) return cudaErrorInvalidValue;  // "wrong jc 2"
    if (ycN[j] < ycO[jc]) jc = jc - 1;
    iyc[j] = jc;
    ryc[j] = (ycO[jc + 1] - ycN[j]) / (ycO[jc + 1] - ycO[jc]);
  }
  // one device buffer: 8 index tables, 8 weight tables, dy of the new grid, row sums
  const std::vector<int>* I[8] = {&ixp, &ixc, &iyp, &iyc, &izp, &izc, nullptr, nullptr};
  const std::vector<double>* R[8] = {&rxp, &rxc, &ryp, &ryc, &rzp, &rzc, nullptr, nullptr};
  size_t off[7], bytes = 0;
  for (int q = 0; q < 6; ++q) { off[q] = bytes; bytes += (I[q]->size() * sizeof(int) + 255) / 256 * 256; }
  size_t roff[6];
  for (int q = 0; q < 6; ++q) { roff[q] = bytes; bytes += (R[q]->size() * sizeof(double) + 255) / 256 * 256; }
  const size_t dyoff = bytes;
  bytes += ((size_t)nyn * sizeof(double) + 255) / 256 * 256;
  const size_t rowoff = bytes;
  bytes += (size_t)nyn * nzn * sizeof(double);
  unsigned char* buf = nullptr;
  cudaError_t e = cudaMalloc(&buf, bytes);
  if (e != cudaSuccess) return e;
  std::vector<unsigned char> h(bytes, 0);
  for (int q = 0; q < 6; ++q) std::memcpy(h.data() + off[q], I[q]->data(), I[q]->size() * sizeof(int));
  for (int q = 0; q < 6; ++q) std::memcpy(h.data() + roff[q], R[q]->data(), R[q]->size() * sizeof(double));
  std::memcpy(h.data() + dyoff, dyn.data(), dyn.size() * sizeof(double));
  cudaStream_t st = dst->stream;
  if ((e = cudaStreamSynchronize(src->stream)) == cudaSuccess &&
      (e = cudaMemcpyAsync(buf, h.data(), rowoff, cudaMemcpyHostToDevice, st)) == cudaSuccess) {
    auto ax = [&](int q) { return InterpAxis{(const int*)(buf + off[q]), (const double*)(buf + roff[q])}; };
    OldGrid o;
    o.nx = nxo; o.ny = nyo; o.nz = nzo;
    o.bc_lo = src->cfg.BcOption[2]; o.bc_hi = src->cfg.BcOption[3];
    const double* wv[3] = {src->cfg.uxBcValue, src->cfg.uyBcValue, src->cfg.uzBcValue};
    for (int q = 0; q < 3; ++q) { o.w_lo[q] = wv[q][2]; o.w_hi[q] = wv[q][3]; }
    const dim3 grid((nxn + 127) / 128, nyn, nzn);
    // ux (xp, yc, zc), uy (xc, yp, zc), uz (xc, yc, zp), p (xc, yc, zc)
    const int tx[4] = {0, 1, 1, 1}, ty[4] = {3, 2, 3, 3}, tz[4] = {5, 5, 4, 5};
    for (int comp = 0; comp < 4 && e == cudaSuccess; ++comp) {
      k_interp<T><<<grid, 128, 0, st>>>(o, comp, (const T*)src->f[comp], ax(tx[comp]), ax(ty[comp]), ax(tz[comp]), nxn,
                                        nyn, (T*)dst->f[comp]);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess && dst->cfg.IsUxConst) {
      double* rows = (double*)(buf + rowoff);
      k_interp_rowsum<T><<<(nyn * nzn + 127) / 128, 128, 0, st>>>((const T*)dst->f[0], (const double*)(buf + dyoff),
                                                                   nxn, nyn, nzn, rows);
      k_interp_rescale<T><<<1, 256, 0, st>>>((T*)dst->f[0], rows, (long long)nyn * nzn, dst->N,
                                             1.0 / (double)nxn / (double)nzn / dst->cfg.yly, dst->cfg.ubulk);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  cudaFree(buf);
  return e;
}

cudaError_t launch_interp_state(ch3d_ctx* dst, const ch3d_ctx* src) {
  return dst->fp32 ? interp_t<float>(dst, src) : interp_t<double>(dst, src);
}

}  // namespace ch3d
