// ch3d_dev.cuh -- device helpers shared by the kernel files: neighbour
// addressing with periodic wrap and wall ghosts, the partitioned tridiagonal
// solve's chunk bookkeeping and interface system, and the host-side packing
// of the kernel parameters.
#pragma once
#include "ch3d_ctx.h"

namespace ch3d {

// Neighbour addressing of one cell: a base index plus signed offsets that
// already contain the periodic wrap in x and z; y neighbours past the walls
// are replaced by the ghost rules of SetBC_and_UpdateHalo
// (src/CFD_2nd/m_BC_and_Halo.f90:241-282), or by the periodic halo rows when
// y is periodic (BcOption(3:4) = 0).
struct Nbr {
  long long c;        // cell index
  int xp, xm;         // offsets to i+1, i-1
  int xp2, xm2;       // offsets to i+2, i-2
  long long zp, zm;   // offsets to k+1, k-1
  long long zp2, zm2; // offsets to k+2, k-2
  int yp;             // +nx (offset to j+1)
  bool jlo, jhi;      // j == 0, j == ny-1
};

template <class T>
__device__ __forceinline__ Nbr make_nbr(const Geo<T>& g, int i, int j, int k) {
  Nbr n;
  const long long plane = (long long)g.nx * g.ny;
  n.c = i + (long long)g.nx * j + plane * k;
  n.xp = (i + 1 == g.nx) ? 1 - g.nx : 1;
  n.xm = (i == 0) ? g.nx - 1 : -1;
  n.zp = (k + 1 == g.nz) ? -(long long)(g.nz - 1) * plane : plane;
  n.zm = (k == 0) ? (long long)(g.nz - 1) * plane : -plane;
  n.xp2 = (i + 2 >= g.nx) ? 2 - g.nx : 2;
  n.xm2 = (i < 2) ? g.nx - 2 : -2;
  n.zp2 = (k + 2 >= g.nz) ? (long long)(2 - g.nz) * plane : 2 * plane;
  n.zm2 = (k < 2) ? (long long)(g.nz - 2) * plane : -2 * plane;
  n.yp = g.nx;
  n.jlo = (j == 0);
  n.jhi = (j == g.ny - 1);
  return n;
}

// value at offset o (same j) and at j-1 / j+1 of the same offset column
template <class T> __device__ __forceinline__ T at(const T* __restrict__ a, const Nbr& n, long long o) {
  return __ldg(a + n.c + o);
}
// ux / uz (comp 0 / 2): wall ghosts 2 w - u (no-slip) or u -/+ w dyp (free-slip)
template <class T>
__device__ __forceinline__ T at_jm(const T* __restrict__ a, const Geo<T>& g, int comp, const Nbr& n, long long o) {
  if (!n.jlo) return __ldg(a + n.c + o - n.yp);
  if (g.bc.lo == 0) return __ldg(a + n.c + o + (long long)(g.ny - 1) * n.yp);  // periodic: row ny-1
  if (comp == 1) {  // uy(ic,0,kc) = 2 uy_ym - uy(ic,2,kc); zero in the 4th-order solver
    if (g.order == 4) return (T)0;
    return (T)(g.bc.uy_lo * 2.0) - __ldg(a + n.c + o + n.yp);
  }
  const T v = __ldg(a + n.c + o);
  if (comp == 3) return v;
  const double w = comp == 0 ? g.bc.ux_lo : g.bc.uz_lo;
  return g.bc.lo == -1 ? (T)(w * 2.0) - v : v - (T)(w * g.bc.dyp1);
}
template <class T>
__device__ __forceinline__ T at_jp(const T* __restrict__ a, const Geo<T>& g, int comp, const Nbr& n, long long o) {
  if (!n.jhi) return __ldg(a + n.c + o + n.yp);
  if (g.bc.hi == 0) return __ldg(a + n.c + o - (long long)(g.ny - 1) * n.yp);  // periodic: row 0
  if (comp == 1) return (T)g.bc.uy_hi;  // uy(ic,nyp,kc) = uyBcValue(yp)
  const T v = __ldg(a + n.c + o);
  if (comp == 3) return v;
  const double w = comp == 0 ? g.bc.ux_hi : g.bc.uz_hi;
  return g.bc.hi == -1 ? (T)(w * 2.0) - v : (T)(w * g.bc.dypN) + v;
}

// asynchronous 4-, 8- or 16-byte copy global -> shared (cp.async, completion by
// commit groups; 16-byte copies bypass L1)
template <class E> __device__ __forceinline__ void cp_async_el(E* smem, const E* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (sizeof(E) == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
  else if constexpr (sizeof(E) == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// 4th-order stencil constants (src/CFD_4th/m_MeshAndMetries.f90:86-91)
template <class T> struct C4 {
  T dx1, dx2, dx3, dx4, dz1, dz2, dz3, dz4;
  T dxx1, dxx2, dxx3, dxx4, dxx5, dzz1, dzz2, dzz3, dzz4, dzz5;
  T in1, in2, in3, in4;
  __device__ __forceinline__ C4(const Geo<T>& g) {
    const T rdx = g.rdx, rdz = g.rdz, rdx2 = g.rdx2, rdz2 = g.rdz2;
    dx1 = rdx / (T)24; dx2 = -rdx * (T)1.125; dx3 = rdx * (T)1.125; dx4 = -rdx / (T)24;
    dz1 = rdz / (T)24; dz2 = -rdz * (T)1.125; dz3 = rdz * (T)1.125; dz4 = -rdz / (T)24;
    dxx1 = -rdx2 / (T)12; dxx2 = (T)4 / (T)3 * rdx2; dxx3 = (T)-2.5 * rdx2; dxx4 = (T)4 / (T)3 * rdx2; dxx5 = -rdx2 / (T)12;
    dzz1 = -rdz2 / (T)12; dzz2 = (T)4 / (T)3 * rdz2; dzz3 = (T)-2.5 * rdz2; dzz4 = (T)4 / (T)3 * rdz2; dzz5 = -rdz2 / (T)12;
    in1 = (T)-1 / (T)16; in2 = (T)9 / (T)16; in3 = (T)9 / (T)16; in4 = (T)-1 / (T)16;
  }
};

// 4th-order divergence at one cell: clcPrSrc (src/CFD_4th/m_TScheme.f90:114-143)
// and CheckDivergence (src/CFD_4th/m_Tools.f90:54-81).
template <class T>
__device__ __forceinline__ T div4_at(const Geo<T>& g, const C4<T>& c, T rdyp, const T* __restrict__ ux,
                                     const T* __restrict__ uy, const T* __restrict__ uz, const Nbr& n) {
  const T dudx = c.dx1 * at(ux, n, n.xm) + c.dx2 * at(ux, n, 0) + c.dx3 * at(ux, n, n.xp) + c.dx4 * at(ux, n, n.xp2);
  const T dvdy = (at_jp(uy, g, 1, n, 0) - at(uy, n, 0)) * rdyp;
  const T dwdz = c.dz1 * at(uz, n, n.zm) + c.dz2 * at(uz, n, 0) + c.dz3 * at(uz, n, n.zp) + c.dz4 * at(uz, n, n.zp2);
  return dudx + dvdy + dwdz;
}
template <class T>
__device__ __forceinline__ T div4_cell(const Geo<T>& g, const C4<T>& c, T rdyp, const T* __restrict__ ux,
                                       const T* __restrict__ uy, const T* __restrict__ uz, int i, int j, int k) {
  return div4_at(g, c, rdyp, ux, uy, uz, make_nbr(g, i, j, k));
}
// move a neighbourhood one row up the same column (the x and z offsets do not
// depend on j)
template <class T> __device__ __forceinline__ void nbr_next_row(Nbr& n, const Geo<T>& g, int j) {
  n.c += g.nx;
  n.jlo = (j == 0);
  n.jhi = (j == g.ny - 1);
}

// ---------------------------------------------------------------------------
// Partitioned tridiagonal solve (used by clcU*Hat and the Poisson y solve).
// A system of n rows is cut into P chunks.  Each chunk is solved locally
// (Thomas) for the data and for two "spikes" (its response to the unknown
// just left of and just right of it); the 2(P-1) interface unknowns then
// satisfy a 2x2-block tridiagonal system solved by one thread.  This is the
// same decomposition as the reference's InverseTridiagonal_reduce
// (src/CFD_2nd/m_Poisson.f90:1462) applied inside one thread block.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int chunk_lo(int p, int n, int P) { return (p * n) / P; }
__device__ __forceinline__ int chunk_hi(int p, int n, int P) { return ((p + 1) * n) / P - 1; }
// the chunk p with chunk_lo(p) <= j <= chunk_hi(p): the largest p with p*n/P <= j
__device__ __forceinline__ int chunk_of(int j, int n, int P) { return ((j + 1) * P - 1) / n; }

// Coefficients of the velocity Helmholtz systems (identical for all columns).
// set 0: clcU1Hat_PIMP / clcU3Hat_PIMP (m_TSchemePIMP_inc.f90:410-416, 720-726)
// set 1: clcU2Hat_PIMP (:561-572), row 1 is the identity.
struct HelmCoef {
  const double* ap2cForCN; const double* am2cForCN;
  const double* ap2p; const double* ac2p; const double* am2p;
};

__device__ __forceinline__ void helm_abc(const HelmCoef& hc, int set, double pmBeta, int j, double& a, double& b,
                                         double& c) {
  const int jc = j + 1;
  if (set == 1) {
    if (j == 0) { a = 0.0; b = 1.0; c = 0.0; return; }
    c = -pmBeta * hc.ap2p[jc];
    b = -pmBeta * hc.ac2p[jc] + 1.0;
    a = -pmBeta * hc.am2p[jc];
  } else {
    c = -pmBeta * hc.ap2cForCN[jc];
    a = -pmBeta * hc.am2cForCN[jc];
    b = -c - a + 1.0;
  }
}

// The Helmholtz coefficient vectors inside the packed FP64 metric block
// (pack order of ch3d_api.cu).
inline HelmCoef helm_coef(const ch3d_ctx* c) {
  HelmCoef hc;
  const double* M = c->met64;
  const int L = c->ny + 3;
  hc.ap2p = M + 7 * L; hc.ac2p = M + 8 * L; hc.am2p = M + 9 * L;
  hc.ap2cForCN = M + 14 * L; hc.am2cForCN = M + 15 * L;
  return hc;
}

// Factor layout of one set: RM | AA | CP | AL | BE (ny each), then per
// interface q: M00 M01 M10 M11 l v (6 each).
__host__ __device__ inline int helm_set_stride(int ny, int P) { return 5 * ny + 6 * (P > 1 ? P - 1 : 1); }

// Interface (reduced) block-tridiagonal solve of one column, with the
// precomputed factors; F: chunk-local solutions of the column (stride fs).
template <class T, class FT>
__device__ __forceinline__ void helm_interfaces(const FT* __restrict__ IFD, const T* F, int fs, int ny, int P,
                                                T* G /* 2*(P-1) */) {
  const int Q = P - 1;
  T gu = (T)0, gw = (T)0;
  for (int q = 0; q < Q; ++q) {
    const int eq = chunk_hi(q, ny, P), sq1 = chunk_lo(q + 1, ny, P);
    const FT* R = IFD + 6 * q;
    const T ru = F[eq * fs] - (q > 0 ? (T)R[4] * gu : (T)0);
    const T rw = F[sq1 * fs];
    gu = (T)R[0] * ru + (T)R[1] * rw;
    gw = (T)R[2] * ru + (T)R[3] * rw;
    G[2 * q] = gu;
    G[2 * q + 1] = gw;
  }
  if (Q < 1) return;
  T zw = G[2 * (Q - 1) + 1];
  for (int q = Q - 2; q >= 0; --q) {
    const FT* R = IFD + 6 * q;
    const T f = (T)R[5] * zw;
    const T zu = G[2 * q] - (T)R[1] * f;
    const T zwn = G[2 * q + 1] - (T)R[3] * f;
    G[2 * q] = zu;
    G[2 * q + 1] = zwn;
    zw = zwn;
  }
}

template <class T> Geo<T> make_geo(const ch3d_ctx* c) {
  Geo<T> g;
  g.nx = c->nx; g.ny = c->ny; g.nz = c->nz; g.nxh = c->nxh; g.N = c->N;
  g.order = c->cfg.order;
  g.implicit = c->cfg.IsImplicit;
  g.les = c->cfg.LES_type > 0 ? 1 : 0;
  g.rdx = (T)c->rdx; g.rdz = (T)c->rdz; g.rdx2 = (T)c->rdx2; g.rdz2 = (T)c->rdz2;
  // periodic x and z: am1c = ap1c = rdx2, ac1c = -(am1c+ap1c) (m_MeshAndMetries.f90:243-252)
  g.ap1c = (T)c->rdx2; g.am1c = (T)c->rdx2; g.ac1c = (T)(-(c->rdx2 + c->rdx2));
  g.ap3c = (T)c->rdz2; g.am3c = (T)c->rdz2; g.ac3c = (T)(-(c->rdz2 + c->rdz2));
  g.xnu = (T)c->cfg.xnu;
  g.g1 = (T)c->cfg.gravity[0]; g.g2 = (T)c->cfg.gravity[1]; g.g3 = (T)c->cfg.gravity[2];
  g.bc.lo = c->cfg.BcOption[2]; g.bc.hi = c->cfg.BcOption[3];
  g.bc.ux_lo = c->cfg.uxBcValue[2]; g.bc.ux_hi = c->cfg.uxBcValue[3];
  g.bc.uy_lo = c->cfg.uyBcValue[2]; g.bc.uy_hi = c->cfg.uyBcValue[3];
  g.bc.uz_lo = c->cfg.uzBcValue[2]; g.bc.uz_hi = c->cfg.uzBcValue[3];
  g.bc.dyp1 = c->dyp[1]; g.bc.dypN = c->dyp[c->ny + 1];
  return g;
}

template <class T> const Metrics<T>& metrics_of(const ch3d_ctx* c);
template <> inline const Metrics<double>& metrics_of<double>(const ch3d_ctx* c) { return c->m64; }
template <> inline const Metrics<float>& metrics_of<float>(const ch3d_ctx* c) { return c->m32; }


}  // namespace ch3d
