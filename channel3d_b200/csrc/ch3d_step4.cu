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
__global__ void __launch_bounds__(256) k_visc4_partial(Geo<T> g, Metrics<T> m, const T* __restrict__ ux,
                                                       double* __restrict__ part) {
  __shared__ double red[256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const int tl = threadIdx.x + blockDim.x * threadIdx.y;
  double s = 0.0;
  if (i < g.nx && j < g.ny) {
    const Nbr n = make_nbr(g, i, j, k);
    const C4<T> c(g);
    const int jc = j + 1;
    const T ux_c = at(ux, n, 0);
    const T d11 = c.dxx1 * at(ux, n, n.xm2) + c.dxx2 * at(ux, n, n.xm) + c.dxx3 * ux_c + c.dxx4 * at(ux, n, n.xp) +
                  c.dxx5 * at(ux, n, n.xp2);
    const T d22 = m.ap2c[jc] * at_jp(ux, g, 0, n, 0) + m.ac2c[jc] * ux_c + m.am2c[jc] * at_jm(ux, g, 0, n, 0);
    const T d33 = c.dzz1 * at(ux, n, n.zm2) + c.dzz2 * at(ux, n, n.zm) + c.dzz3 * ux_c + c.dzz4 * at(ux, n, n.zp) +
                  c.dzz5 * at(ux, n, n.zp2);
    s = ((double)(d11 + d33) + (double)d22) * (double)m.dyp[jc];
  }
  red[tl] = s;
  __syncthreads();
  for (int w = blockDim.x * blockDim.y / 2; w > 0; w >>= 1) {
    if (tl < w) red[tl] += red[tl + w];
    __syncthreads();
  }
  if (tl == 0) part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = red[0];
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
  k_visc4_partial<T><<<dim3((c->nx + 31) / 32, (c->ny + 7) / 8, c->nz), dim3(32, 8), 0, c->stream>>>(
      make_geo<T>(c), metrics_of<T>(c), f[0], c->part);
  return cudaGetLastError();
}
cudaError_t launch_visc4_partials(ch3d_ctx* c) { return c->fp32 ? visc4_t<float>(c) : visc4_t<double>(c); }

}  // namespace ch3d
