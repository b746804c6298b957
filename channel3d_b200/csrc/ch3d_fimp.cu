// ch3d_fimp.cu -- sm_100a kernels of the fully implicit (FIMP) 2nd-order
// step: the periodic x and z Crank-Nicolson sweeps of clcU1/2/3Hat_FIMP_010
// (src/CFD_2nd/m_TSchemeFIMP_inc.f90:263-347, 636-729, 1035-1128), whose y
// sweep between walls is the PIMP Helmholtz solve (same coefficients), and
// the periodic y sweep of clcU1/2/3Hat_FIMP_000 (:187-258, 559-631, 950-1030)
// when y is periodic too.  The RHS is rhs_comp with its FIMP branch.
//
// The periodic constant-coefficient solver is InversePTriFixedCoe
// (src/CFD_2nd/m_Tools.f90:167-219): elimination of the first n-1 unknowns
// with a second right-hand side for the coupling to unknown n, then the
// closure of row n.  Its coefficient recurrences (ppj, vecn1, vecn2) are the
// same for every line and are computed once per substep.
#include "ch3d_ctx.h"
#include "ch3d_dev.cuh"

namespace ch3d {

// Factor block of one direction: ppj | vecn1 | vecn2 (n+1 each, Fortran
// index 1..n) then a, b, c, denominator.
__host__ __device__ inline int ptri_stride(int n) { return 3 * (n + 1) + 4; }

// direction d0 + blockIdx.x: 0 = x (n = nx, rdx2), 1 = z (n = nz, rdz2),
// 2 = y (n = ny, rdy2; periodic y only)
__global__ void k_ptri_factors(int d0, int nx, int ny, int nz, double rdx2, double rdy2, double rdz2,
                               double* __restrict__ pf, const DevScalars* __restrict__ sc) {
  if (sc->status || threadIdx.x != 0) return;
  const int d = d0 + blockIdx.x;
  const int n = d == 0 ? nx : (d == 1 ? nz : ny);
  const double r2 = d == 0 ? rdx2 : (d == 1 ? rdz2 : rdy2);
  double* F = pf + (d == 0 ? 0 : (d == 1 ? ptri_stride(nx) : ptri_stride(nx) + ptri_stride(nz)));
  double *ppj = F, *v1 = F + (n + 1), *v2 = F + 2 * (n + 1), *abc = F + 3 * (n + 1);
  const double pmBeta = sc->pmBeta;
  const double a = -pmBeta * r2, c = -pmBeta * r2, b = pmBeta * r2 * 2.0 + 1.0;
  v1[1] = -c / b;
  v2[1] = -a / b;
  v2[n] = 1.0;
  ppj[1] = 0.0;
  for (int j = 2; j <= n - 1; ++j) {
    ppj[j] = 1.0 / (b + a * v1[j - 1]);
    v1[j] = -c * ppj[j];
    v2[j] = -a * v2[j - 1] * ppj[j];
  }
  for (int j = n - 1; j >= 1; --j) v2[j] = v2[j] + v1[j] * v2[j + 1];
  abc[0] = a; abc[1] = b; abc[2] = c;
  abc[3] = c * v2[1] + a * v2[n - 1] + b;
}

// One periodic line f(1..n) at stride s (in place), with the factor block F
// (ppj | vecn1 | vecn2 | a b c den) in shared memory.  The two recurrences
// load YB values ahead of their dependent chain (the values do not depend on
// it), the closing pass is element-wise; the arithmetic is that of
// InversePTriFixedCoe, term for term.
template <class T, int YB>
__device__ __forceinline__ void ptri_line(const double* __restrict__ F, int n, T* f, long long s) {
  const double *ppj = F, *v1 = F + (n + 1), *v2 = F + 2 * (n + 1), *abc = F + 3 * (n + 1);
  const T a = (T)abc[0], b = (T)abc[1], c = (T)abc[2], den = (T)abc[3];
  // forward elimination, rows 1..n-1 (0-based index q = row - 1)
  T prev = f[0] / b;
  f[0] = prev;
  for (int q0 = 1; q0 < n - 1; q0 += YB) {
    T v[YB], w[YB];
#pragma unroll
    for (int u = 0; u < YB; ++u)
      if (q0 + u < n - 1) { v[u] = f[(q0 + u) * s]; w[u] = (T)ppj[q0 + u + 1]; }
#pragma unroll
    for (int u = 0; u < YB; ++u)
      if (q0 + u < n - 1) { prev = (v[u] - a * prev) * w[u]; f[(q0 + u) * s] = prev; }
  }
  // backward pass: arrmn(j) = f(j) + vecn1(j) arrmn(j+1), stored in place
  T arr = (T)0;
  for (int q0 = n - 2; q0 >= 0; q0 -= YB) {
    T v[YB], w[YB];
#pragma unroll
    for (int u = 0; u < YB; ++u)
      if (q0 - u >= 0) { v[u] = f[(q0 - u) * s]; w[u] = (T)v1[q0 - u + 1]; }
#pragma unroll
    for (int u = 0; u < YB; ++u)
      if (q0 - u >= 0) { arr = v[u] + w[u] * arr; f[(q0 - u) * s] = arr; }
  }
  const T fn = (f[(n - 1) * s] - c * f[0] - a * f[(n - 2) * s]) / den;
  f[(n - 1) * s] = fn;
  for (int q0 = 0; q0 < n - 1; q0 += YB) {
#pragma unroll
    for (int u = 0; u < YB; ++u)
      if (q0 + u < n - 1) f[(q0 + u) * s] = fn * (T)v2[q0 + u + 1] + f[(q0 + u) * s];
  }
}

// copy the factor block of one direction into shared memory
__device__ __forceinline__ void ptri_stage_factors(double* dst, const double* __restrict__ src, int n) {
  for (int t = threadIdx.x; t < ptri_stride(n); t += blockDim.x) dst[t] = src[t];
}

// x sweep: LB consecutive x lines (contiguous in memory) per block, staged
// in shared memory with a padded stride (after the factor block) by all 128
// threads; one thread per line solves.  blockIdx.y = component.
template <class T>
__global__ void __launch_bounds__(128) k_ptri_x(int nx, long long nlines, int LB, const double* __restrict__ pf,
                                               T* __restrict__ r0, T* __restrict__ r1, T* __restrict__ r2,
                                               const DevScalars* __restrict__ sc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (sc->status) return;
  double* Fs = (double*)smem_raw;
  T* S = (T*)(Fs + ptri_stride(nx));
  const int ld = nx + 1;
  T* r = blockIdx.y == 0 ? r0 : (blockIdx.y == 1 ? r1 : r2);
  const long long l0 = (long long)blockIdx.x * LB;
  const int nl = (int)min((long long)LB, nlines - l0);
  T* g = r + l0 * nx;
  // the lines by asynchronous copies, all in flight at once
  for (int l = 0; l < nl; ++l)
    for (int x = threadIdx.x; x < nx; x += blockDim.x) cp_async_el(S + l * ld + x, g + (long long)l * nx + x);
  cp_async_commit();
  ptri_stage_factors(Fs, pf, nx);
  cp_async_wait<0>();
  __syncthreads();
  for (int l = threadIdx.x; l < nl; l += blockDim.x) ptri_line<T, 8>(Fs, nx, S + l * ld, 1);
  __syncthreads();
  for (int l = 0; l < nl; ++l)
    for (int x = threadIdx.x; x < nx; x += blockDim.x) g[(long long)l * nx + x] = S[l * ld + x];
}

// z sweep: one thread per (i, j) column, in place in global memory (a warp
// covers 32 consecutive i, so every access is coalesced); 16 rows of loads in
// flight ahead of each recurrence.  blockIdx.z = component.
template <class T>
__global__ void __launch_bounds__(128) k_ptri_z(int nx, int ny, int nz, const double* __restrict__ pf,
                                                T* __restrict__ r0, T* __restrict__ r1, T* __restrict__ r2,
                                                const DevScalars* __restrict__ sc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (sc->status) return;
  double* Fs = (double*)smem_raw;
  ptri_stage_factors(Fs, pf + ptri_stride(nx), nz);
  __syncthreads();
  const int i = blockIdx.x * 32 + (threadIdx.x & 31);
  const int j = blockIdx.y * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (i >= nx || j >= ny) return;
  T* r = blockIdx.z == 0 ? r0 : (blockIdx.z == 1 ? r1 : r2);
  ptri_line<T, 16>(Fs, nz, r + i + (long long)nx * j, (long long)nx * ny);
}

// periodic y sweep (the last sweep of clcU1/2/3Hat_FIMP_000, or the one sweep
// of clcU1/2/3Hat_PIMP_0, src/CFD_2nd/m_TSchemePIMP_inc.f90:435-461, 594-621,
// 745-771): one thread per (i, k) column, in place on the right-hand side (a
// warp covers 32 consecutive i, so every access is coalesced), then
// u* = u + the solution.  The partially implicit RhsX gets the mean pressure
// gradient first (clcRhsX_PIMP adds it; the FIMP RhsX carries it already).
// blockIdx.z = component.
template <class T>
__global__ void __launch_bounds__(128) k_ptri_y(int nx, int ny, int nz, int pimp, const double* __restrict__ pf,
                                                const T* __restrict__ u0, const T* __restrict__ u1,
                                                const T* __restrict__ u2, T* __restrict__ r0, T* __restrict__ r1,
                                                T* __restrict__ r2, T* __restrict__ s0, T* __restrict__ s1,
                                                T* __restrict__ s2, const DevScalars* __restrict__ sc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (sc->status) return;
  double* Fs = (double*)smem_raw;
  ptri_stage_factors(Fs, pf + ptri_stride(nx) + ptri_stride(nz), ny);
  __syncthreads();
  const int i = blockIdx.x * 32 + (threadIdx.x & 31);
  const int k = blockIdx.y * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (i >= nx || k >= nz) return;
  const int comp = blockIdx.z;
  const T* u = comp == 0 ? u0 : (comp == 1 ? u1 : u2);
  T* r = comp == 0 ? r0 : (comp == 1 ? r1 : r2);
  T* us = comp == 0 ? s0 : (comp == 1 ? s1 : s2);
  const long long col = i + (long long)nx * ny * k;
  if (pimp && comp == 0) {
    const T add = (T)sc->dpmdxns;
    for (int j = 0; j < ny; ++j) r[col + (long long)nx * j] = r[col + (long long)nx * j] + add;
  }
  ptri_line<T, 16>(Fs, ny, r + col, (long long)nx);
  for (int j = 0; j < ny; ++j) us[col + (long long)nx * j] = u[col + (long long)nx * j] + r[col + (long long)nx * j];
}

template <class T> static cudaError_t ptri_t(ch3d_ctx* c) {
  T** f = (T**)c->f;
  k_ptri_factors<<<y_periodic(c) ? 3 : 2, 32, 0, c->stream>>>(0, c->nx, c->ny, c->nz, c->rdx2, c->rdy2, c->rdz2,
                                                              c->pfac, c->sc);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // x: one thread per line, at most 64 KB of lines per block
  int LB = (int)((64 * 1024) / ((size_t)(c->nx + 1) * sizeof(T)));
  if (LB > 128) LB = 128;
  if (LB < 1) LB = 1;
  const long long nlines = (long long)c->ny * c->nz;
  const size_t smem = (size_t)ptri_stride(c->nx) * sizeof(double) + (size_t)LB * (c->nx + 1) * sizeof(T);
  static PerDevice attr;  // per precision (template instance)
  if ((e = smem_limit_once(attr, c->device, k_ptri_x<T>, 200 * 1024)) != cudaSuccess) return e;
  k_ptri_x<T><<<dim3((unsigned)((nlines + LB - 1) / LB), 3), 128, smem, c->stream>>>(c->nx, nlines, LB, c->pfac, f[7],
                                                                                      f[8], f[9], c->sc);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const size_t smz = (size_t)ptri_stride(c->nz) * sizeof(double);
  static PerDevice attrz;  // per precision (template instance)
  if ((e = smem_limit_once(attrz, c->device, k_ptri_z<T>, 200 * 1024)) != cudaSuccess) return e;
  k_ptri_z<T><<<dim3((c->nx + 31) / 32, (c->ny + 3) / 4, 3), 128, smz, c->stream>>>(c->nx, c->ny, c->nz, c->pfac,
                                                                                   f[7], f[8], f[9], c->sc);
  return cudaGetLastError();
}
cudaError_t launch_ptri_xz(ch3d_ctx* c) { return c->fp32 ? ptri_t<float>(c) : ptri_t<double>(c); }

template <class T> static cudaError_t ptri_y_t(ch3d_ctx* c) {
  T** f = (T**)c->f;
  const int pimp = c->cfg.IsImplicit == 1;
  cudaError_t e;
  if (pimp) {  // the y factor block alone (FIMP: made by launch_ptri_xz with the x and z blocks)
    k_ptri_factors<<<1, 32, 0, c->stream>>>(2, c->nx, c->ny, c->nz, c->rdx2, c->rdy2, c->rdz2, c->pfac, c->sc);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  const size_t smy = (size_t)ptri_stride(c->ny) * sizeof(double);
  static PerDevice attr;  // per precision (template instance)
  if ((e = smem_limit_once(attr, c->device, k_ptri_y<T>, 200 * 1024)) != cudaSuccess) return e;
  k_ptri_y<T><<<dim3((c->nx + 31) / 32, (c->nz + 3) / 4, 3), 128, smy, c->stream>>>(
      c->nx, c->ny, c->nz, pimp, c->pfac, f[0], f[1], f[2], f[7], f[8], f[9], f[12], f[13], f[14], c->sc);
  return cudaGetLastError();
}
cudaError_t launch_ptri_y(ch3d_ctx* c) { return c->fp32 ? ptri_y_t<float>(c) : ptri_y_t<double>(c); }

// x, z and y factor blocks (the y block is filled only when y is periodic)
size_t ptri_factor_doubles(int nx, int ny, int nz) {
  return (size_t)ptri_stride(nx) + ptri_stride(nz) + ptri_stride(ny);
}

}  // namespace ch3d
