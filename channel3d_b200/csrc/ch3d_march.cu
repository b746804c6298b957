// ch3d_march.cu -- the 2nd-order partially implicit substep's right-hand
// sides fused with its y Crank-Nicolson solves, as a column march:
// clcRhsX/Y/Z_PIMP (src/CFD_2nd/m_TSchemePIMP_inc.f90:7-75, 161-209, 277-325)
// followed by clcU1/2/3Hat_PIMP (:392-430, 542-589, 702-740), u -> u*.
//
// One thread owns one (i, k) column and all three velocity components.  A
// block of 32 x BZ columns marches j upwards through a ring of staged rows in
// shared memory (ux, uy, uz, p of the block's columns plus a one-cell halo in
// x and z, and the row's table entries; rows -1 and ny are the wall ghosts of
// SetBC_and_UpdateHalo, src/CFD_2nd/m_BC_and_Halo.f90:241-282).  At row j the
// thread evaluates the three right-hand sides from rows j-1, j, j+1 of the
// ring, updates Hist, and eliminates row j of the three tridiagonal systems
// (Thomas; the factors are the same for every column and come from a per-row
// table).  Instead of the eliminated right-hand side d_j it stores
//     g_j = u_j + d_j + cp_j u_{j+1}
// in the u* array; the back substitution x_j = d_j - cp_j x_{j+1} of
// u*_j = u_j + x_j then reads only g:  u*_j = g_j - cp_j u*_{j+1}.
// On grids with few column tiles the march runs from both walls (twisted); on
// large grids it stops at g and the divergence and projection marches of this
// file substitute u* themselves (13 values of global traffic per cell: ux uy
// uz p, Hist x3 read + written, g x3 written).  Where the march substitutes
// itself, g is read back and u* written as well (19 values).
#include "ch3d_ctx.h"
#include "ch3d_dev.cuh"

namespace ch3d {

// Row table of the march (precision T, MT_W values per row j = 0..ny-1):
// the y metrics at jc = j + 1 and the Thomas factors a, 1/m, c/m of the two
// Helmholtz sets (set 0: ux and uz, set 1: uy; m_TSchemePIMP_inc.f90:392-430,
// 542-589, 702-740).  cp of the last row is stored as 0 (it has no upper neighbour).
enum {
  MT_IY1, MT_IY3, MT_RDYP, MT_RDYC, MT_AP2C, MT_AC2C, MT_AM2C, MT_AP2P, MT_AC2P, MT_AM2P,
  MT_A0, MT_RM0, MT_CP0, MT_A1, MT_RM1, MT_CP1, MT_W
};
// Second table for the twisted march (lower half eliminated upwards, upper half
// downwards): the downward factors c, 1/m', a/m' of both sets, with
// m'_{ny-1} = b, m'_j = b_j - c_j aq_{j+1}; rows of MD_W values.
enum { MD_C0, MD_RQ0, MD_AQ0, MD_C1, MD_RQ1, MD_AQ1, MD_W = 8 };

// Layout of the march table buffer (values of precision T at the start of a
// buffer sized for FP64): the row tables of the RK substeps ns = 1..3 (ny * MT_W
// values each), their downward tables (ny * MD_W each), then per substep the
// pmBeta its factors were computed for (FP64 bit patterns; all ones = not yet
// computed).
constexpr int kMarchTables = 3;
size_t march_table_bytes(int ny) {
  return (size_t)kMarchTables * ny * (MT_W + MD_W) * sizeof(double) + kMarchTables * sizeof(unsigned long long);
}
static unsigned long long* march_beta_slots(void* mtab, int ny) {
  return (unsigned long long*)((char*)mtab + (size_t)kMarchTables * ny * (MT_W + MD_W) * sizeof(double));
}
template <class T> static T* march_down_tables(void* mtab, int ny) { return (T*)mtab + (size_t)kMarchTables * ny * MT_W; }
cudaError_t march_table_reset(ch3d_ctx* c) {
  return cudaMemsetAsync(march_beta_slots(c->mtab, c->ny), 0xff, kMarchTables * sizeof(unsigned long long),
                         c->stream);
}

// Table of substep sc->ns; skipped when it already holds the factors of this
// pmBeta (constant dt: computed once per substep of the run).
template <class T>
__global__ void k_march_table(HelmCoef hc, Metrics<T> m, int ny, T* __restrict__ tabs, T* __restrict__ dtabs,
                              unsigned long long* __restrict__ beta_slot, const DevScalars* __restrict__ sc) {
  if (sc->status) return;
  const int q = sc->ns - 1;
  const unsigned long long bits = (unsigned long long)__double_as_longlong(sc->pmBeta);
  if (beta_slot[q] == bits) return;  // uniform across the block
  T* tab = tabs + (size_t)q * ny * MT_W;
  if (threadIdx.x == 0 || threadIdx.x == 32) {  // one thread per Helmholtz set, sequential in j
    const int set = threadIdx.x == 0 ? 0 : 1;
    const double pmBeta = sc->pmBeta;
    T* col = tab + (set ? MT_A1 : MT_A0);
    double cpp = 0.0;
    for (int j = 0; j < ny; ++j) {
      double a, b, c;
      helm_abc(hc, set, pmBeta, j, a, b, c);
      const double rm = 1.0 / (j == 0 ? b : b - a * cpp);
      const double cp = c * rm;
      col[(size_t)j * MT_W + 0] = (T)a;
      col[(size_t)j * MT_W + 1] = (T)rm;
      col[(size_t)j * MT_W + 2] = j == ny - 1 ? (T)0 : (T)cp;
      cpp = cp;
    }
  }
  if (threadIdx.x == 64 || threadIdx.x == 96) {  // downward elimination, sequential from the top
    const int set = threadIdx.x == 64 ? 0 : 1;
    const double pmBeta = sc->pmBeta;
    T* col = dtabs + (size_t)q * ny * MD_W + (set ? MD_C1 : MD_C0);
    double aqn = 0.0;
    for (int j = ny - 1; j >= 0; --j) {
      double a, b, c;
      helm_abc(hc, set, pmBeta, j, a, b, c);
      const double rq = 1.0 / (j == ny - 1 ? b : b - c * aqn);
      const double aq = a * rq;
      col[(size_t)j * MD_W + 0] = (T)c;
      col[(size_t)j * MD_W + 1] = (T)rq;
      col[(size_t)j * MD_W + 2] = (T)aq;
      aqn = aq;
    }
  }
  for (int j = threadIdx.x; j < ny; j += blockDim.x) {
    const int jc = j + 1;
    T* row = tab + (size_t)j * MT_W;
    row[MT_IY1] = m.yinterp[jc]; row[MT_IY3] = m.yinterp[jc + 1];
    row[MT_RDYP] = m.rdyp[jc]; row[MT_RDYC] = m.rdyc[jc];
    row[MT_AP2C] = m.ap2c[jc]; row[MT_AC2C] = m.ac2c[jc]; row[MT_AM2C] = m.am2c[jc];
    row[MT_AP2P] = m.ap2p[jc]; row[MT_AC2P] = m.ac2p[jc]; row[MT_AM2P] = m.am2p[jc];
  }
  __syncthreads();
  if (threadIdx.x == 0) beta_slot[q] = bits;
}

// Staging geometry: x halo H rounded up to whole copy vectors of VW points, and
// points per staged row of a 32 x BZ tile.
constexpr int march_hx(int H, int VW) { return (H + VW - 1) / VW * VW; }
constexpr int march_pl(int H, int VW, int BZ) { return (32 + 2 * march_hx(H, VW)) * (BZ + 2 * H); }

// Shared memory of one thread group of the march: RS row slots of the four
// staged fields (PL points each) and of the row table (MT_W values).
template <class T> constexpr size_t march_group_smem(int RS, int PL) {
  return (size_t)4 * RS * PL * sizeof(T) + (size_t)RS * MT_W * sizeof(T);
}

// Ring of RS row slots (row r in slot (r + 1) % RS); rows j+2 .. j+D+1 are in
// flight while row j is computed.  Slot (j+D+2), written after the barrier of
// iteration j, must differ from the slots of rows j-1, j, j+1 that other
// threads still read: RS >= D + 4.
//
// O4: the 4th-order right-hand sides (clcRhsXYZ, src/CFD_4th/m_TScheme.f90:
// 189-377) with a 3-cell x/z halo; their x- and z-interpolated velocities
// (:209-227) are formed from the staged rows instead of being stored.
//
// TW (twisted, for grids with too few column tiles to fill the GPU): the block
// has two thread groups per tile; the lower marches rows 0..m-1 upwards with the
// upward elimination, the upper rows ny-1..m downwards with the downward one,
// each with its own row ring; they meet at rows m-1, m (a 2x2 solve) and
// substitute outwards.  Same right-hand sides, half the march length.
//
// BS = false: the march stops at g; k_div_bsub and k_proj_bsub substitute
// u* = g - cp u*_{j+1} themselves while they walk each column downwards, so u*
// is never stored and g is never read back here (6 arrays less traffic).
//
// VW: rows staged in copy vectors of VW elements (4: 16-byte copies of FP32
// rows, the x halo rounded up to 4 points; needs nx % 4 == 0), 1: element-wise.
template <class T, bool O4, bool TW, bool BS, int VW, int BZ, int D, int RS>
__global__ void __launch_bounds__(32 * BZ * (TW ? 2 : 1),
                                  (!BS && sizeof(T) == 4 && !O4)  // FP32 march stopping at g: 80 registers
                                      ? 6
                                      : (sizeof(T) == 4 || O4 ? (O4 ? 384 : 640) : 512) / (32 * BZ * (TW ? 2 : 1)))
    k_rhs_march(Geo<T> g, const T* __restrict__ tab, const T* __restrict__ dtab, const T* __restrict__ ux, const T* __restrict__ uy,
                const T* __restrict__ uz, const T* __restrict__ pr, T* __restrict__ hx, T* __restrict__ hy,
                T* __restrict__ hz, T* __restrict__ uxs, T* __restrict__ uys, T* __restrict__ uzs,
                const DevScalars* __restrict__ sc) {
  constexpr int H = O4 ? 3 : 1;  // x/z halo
  constexpr int HX = march_hx(H, VW);  // staged x halo
  constexpr int BX = 32, NT = BX * BZ, SX = BX + 2 * HX, PL = march_pl(H, VW, BZ);
  constexpr int NS = (PL / VW + NT - 1) / NT;  // staging vectors per thread and array
  static_assert(VW == 1 || (VW == 4 && sizeof(T) == 4), "16-byte vectors of FP32 rows only");
  typedef typename std::conditional<VW == 4, float4, T>::type VT;
  static_assert(RS >= D + 4, "ring too small for the prefetch distance");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int hf = TW ? (int)threadIdx.x / NT : 0;  // thread group: 0 lower (or the only one), 1 upper
  // per thread group: the field rows [4][RS][PL], then the table rows [RS][MT_W]
  unsigned char* const grp_smem = smem_raw + (size_t)hf * march_group_smem<T>(RS, PL);
  T (*ring)[RS][PL] = reinterpret_cast<T (*)[RS][PL]>(grp_smem);
  T (*trs)[MT_W] = reinterpret_cast<T (*)[MT_W]>(grp_smem + (size_t)4 * RS * PL * sizeof(T));
  if (sc->status) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long long plane = (long long)nx * ny;
  tab += (size_t)(sc->ns - 1) * ny * MT_W;  // this substep's tables
  dtab += (size_t)(sc->ns - 1) * ny * MD_W;
  const int tid = TW ? (int)threadIdx.x - hf * NT : (int)threadIdx.x, tx = tid & 31, tz = tid >> 5;
  const int mh = TW ? ny / 2 : ny;          // rows of the lower group (all rows without TW)
  const int nrow = TW && hf ? ny - mh : mh;  // rows this group marches
  const int dj = hf ? -1 : 1;                // march direction
  auto in_group = [&](int r) { return TW ? (hf ? r >= mh - 1 && r < ny : r >= 0 && r <= mh) : r >= 0 && r < ny; };
  auto slot = [](int r) { return (r + 1) % RS; };  // r >= -1
  // the groups march different numbers of rows (ny odd): each syncs on its own named barrier
  auto group_sync = [&]() {
    if constexpr (TW) {
      if (hf) asm volatile("bar.sync 2, %0;" ::"n"(NT) : "memory");
      else asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory");
    } else {
      __syncthreads();
    }
  };
  long long so[NS];  // staging slot offsets of the current tile
  auto issue_row = [&](int r) {  // r < ny
    const long long ro = (long long)r * nx;
    const int sl = slot(r);
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      const int s = (tid + q * NT) * VW;
      if (s < PL) {
        cp_async_el(reinterpret_cast<VT*>(&ring[0][sl][s]), reinterpret_cast<const VT*>(ux + so[q] + ro));
        cp_async_el(reinterpret_cast<VT*>(&ring[1][sl][s]), reinterpret_cast<const VT*>(uy + so[q] + ro));
        cp_async_el(reinterpret_cast<VT*>(&ring[2][sl][s]), reinterpret_cast<const VT*>(uz + so[q] + ro));
        cp_async_el(reinterpret_cast<VT*>(&ring[3][sl][s]), reinterpret_cast<const VT*>(pr + so[q] + ro));
      }
    }
    // the row's table entries (MT_W values, 16-byte copies) in the same copy group
    constexpr int TV = MT_W * (int)sizeof(T) / 16;
    if (tid < TV)
      cp_async_el(reinterpret_cast<float4*>(&trs[sl][0]) + tid, reinterpret_cast<const float4*>(tab + (size_t)r * MT_W) + tid);
  };
  // wall ghost rows from the thread's own staged slots next to them (at_jm / at_jp of ch3d_dev.cuh)
  auto ghost_row = [&](int r) {
    const int sl = slot(r);
#pragma unroll
    for (int qv = 0; qv < NS * VW; ++qv) {  // the elements of this thread's staging vectors
      const int s = (tid + (qv / VW) * NT) * VW + qv % VW;
      if (s >= PL) continue;
      if (r < 0) {
        const T u = ring[0][slot(0)][s], w = ring[2][slot(0)][s], v1 = ring[1][slot(1)][s];
        ring[0][sl][s] = g.bc.lo == -1 ? (T)(g.bc.ux_lo * 2.0) - u : u - (T)(g.bc.ux_lo * g.bc.dyp1);
        // uy(ic,0,kc) = 2 uy_ym - uy(ic,2,kc); never set (zero) in the 4th-order solver
        ring[1][sl][s] = O4 ? (T)0 : (T)(g.bc.uy_lo * 2.0) - v1;
        ring[2][sl][s] = g.bc.lo == -1 ? (T)(g.bc.uz_lo * 2.0) - w : w - (T)(g.bc.uz_lo * g.bc.dyp1);
        ring[3][sl][s] = ring[3][slot(0)][s];
      } else {
        const int sn = slot(ny - 1);
        const T u = ring[0][sn][s], w = ring[2][sn][s];
        ring[0][sl][s] = g.bc.hi == -1 ? (T)(g.bc.ux_hi * 2.0) - u : (T)(g.bc.ux_hi * g.bc.dypN) + u;
        ring[1][sl][s] = (T)g.bc.uy_hi;
        ring[2][sl][s] = g.bc.hi == -1 ? (T)(g.bc.uz_hi * 2.0) - w : (T)(g.bc.uz_hi * g.bc.dypN) + w;
        ring[3][sl][s] = ring[3][sn][s];
      }
    }
  };

  const T two = (T)2, half = (T)0.5, quarter = (T)0.25, one = (T)1;
  const T rdx = g.rdx, rdz = g.rdz, rdx2 = g.rdx2, rdz2 = g.rdz2, xnu = g.xnu;
  const T pmGamma = (T)sc->pmGamma, pmTheta = (T)sc->pmTheta, pmAlpha = (T)sc->pmAlpha, pmBeta = (T)sc->pmBeta;
  const T dpm = (T)sc->dpmdxns;
  const int c0 = (tz + H) * SX + tx + HX;
  const int ntx = (nx + BX - 1) / BX, ntiles = ntx * ((nz + BZ - 1) / BZ);

  // Persistent blocks walk tiles of 32 x BZ columns.  The back substitution of
  // a tile (HBM-bound) runs one row per forward row of the block's next tile
  // (latency-bound), so the two overlap instead of alternating in waves.
  bool pact = false;          // this thread's column of the previous tile is inside the grid
  long long pidx = 0;         // its row ny-1
  T p0 = (T)0, p1 = (T)0, p2 = (T)0;  // u* of the row above the next one to substitute
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
  const int i0 = (tile % ntx) * BX, k0 = (tile / ntx) * BZ;
  const int i = i0 + tx, k = k0 + tz;
  const bool act = i < nx && k < nz;
  // staging slots: s = tid + q NT -> halo-tile position (s % SX, s / SX), periodic in x and z
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    const int s = (tid + q * NT) * VW;  // a vector never wraps: nx and i0 - HX are multiples of VW
    int ig = (i0 - HX + s % SX) % nx, kg = (k0 - H + s / SX) % nz;
    if (ig < 0) ig += nx;
    if (kg < 0) kg += nz;
    so[q] = s < PL ? ig + plane * kg : 0;
  }
  // prologue: the first D+2 rows of the march in flight, one copy group per row
#pragma unroll
  for (int r = 0; r <= D + 1; ++r) {
    const int row = hf ? ny - 1 - r : r;
    if (in_group(row)) issue_row(row);
    cp_async_commit();
  }
  const int jstart = hf ? ny - 1 : 0;
  long long idx = act ? i + plane * k + (long long)jstart * nx : 0;
  T d0 = (T)0, d1 = (T)0, d2 = (T)0;       // eliminated right-hand sides of the previous row
  T g0 = (T)0, g1 = (T)0, g2 = (T)0;       // g of the last row (= u* of row ny-1)
  T hxo = (T)0, hyo = (T)0, hzo = (T)0;    // Hist of row j
  T hx1 = (T)0, hy1 = (T)0, hz1 = (T)0;    // Hist of row j+1
  // pmTheta = 0 (first RK3 substep): the old Hist does not enter, so it is not read
  const bool hread = act && pmTheta != (T)0;
  const long long hstep = (long long)dj * nx;
  if (hread) {
    hxo = hx[idx]; hyo = hy[idx]; hzo = hz[idx];
    if (nrow > 1) { hx1 = hx[idx + hstep]; hy1 = hy[idx + hstep]; hz1 = hz[idx + hstep]; }
  }
  T lu0 = (T)0, lu1 = (T)0, lu2 = (T)0;  // u at the group's last row (TW meeting)

  // previous tile: row rb = ny-2-j of its back substitution at forward row j, its g
  // loaded two rows ahead
  T n0 = (T)0, n1 = (T)0, n2 = (T)0, m0 = (T)0, m1 = (T)0, m2 = (T)0;
  if (pact && ny >= 2) { n0 = uxs[pidx - nx]; n1 = uys[pidx - nx]; n2 = uzs[pidx - nx]; }
  if (pact && ny >= 3) { m0 = uxs[pidx - 2 * nx]; m1 = uys[pidx - 2 * nx]; m2 = uzs[pidx - 2 * nx]; }
  for (int sj = 0; sj < nrow; ++sj) {
    const int j = jstart + dj * sj;
    const int rb = ny - 2 - j;
    const bool bsub = pact && rb >= 0;
    const long long ob = pidx - (long long)(j + 1) * nx;
    const T b0 = n0, b1 = n1, b2 = n2;
    n0 = m0; n1 = m1; n2 = m2;
    if (pact && rb >= 2) { m0 = uxs[ob - 2 * nx]; m1 = uys[ob - 2 * nx]; m2 = uzs[ob - 2 * nx]; }
    cp_async_wait<D>();  // this thread's copies of rows <= j+1 are done
    if (j + 1 == ny) ghost_row(ny);
    if (j == 0) ghost_row(-1);
    group_sync();
    if (in_group(j + dj * (D + 2))) issue_row(j + dj * (D + 2));
    cp_async_commit();
    T hxn = (T)0, hyn = (T)0, hzn = (T)0;
    if (hread && sj + 2 < nrow) { hxn = hx[idx + 2 * hstep]; hyn = hy[idx + 2 * hstep]; hzn = hz[idx + 2 * hstep]; }
    if (act) {
      T rx, ry, rz, ux_c, uy_c, uz_c, ux_jp, uy_jp, uz_jp, ux_jm, uy_jm, uz_jm;
      const T* tr = trs[slot(j)];  // row j of the table, staged with the row
      if constexpr (!O4) {
      const T* X0 = &ring[0][slot(j - 1)][c0];
      const T* X1 = &ring[0][slot(j)][c0];
      const T* X2 = &ring[0][slot(j + 1)][c0];
      const T* Y0 = &ring[1][slot(j - 1)][c0];
      const T* Y1 = &ring[1][slot(j)][c0];
      const T* Y2 = &ring[1][slot(j + 1)][c0];
      const T* Z0 = &ring[2][slot(j - 1)][c0];
      const T* Z1 = &ring[2][slot(j)][c0];
      const T* Z2 = &ring[2][slot(j + 1)][c0];
      const T* P0 = &ring[3][slot(j - 1)][c0];
      const T* P1 = &ring[3][slot(j)][c0];

      ux_c = X1[0]; const T ux_ip = X1[1], ux_im = X1[-1]; ux_jp = X2[0]; ux_jm = X0[0];
      const T ux_kp = X1[SX], ux_km = X1[-SX], ux_ip_jm = X0[1], ux_ip_km = X1[1 - SX];
      uy_c = Y1[0]; uy_jp = Y2[0]; uy_jm = Y0[0]; const T uy_ip = Y1[1], uy_im = Y1[-1];
      const T uy_im_jp = Y2[-1], uy_kp = Y1[SX], uy_km = Y1[-SX], uy_jp_km = Y2[-SX];
      uz_c = Z1[0]; uz_jp = Z2[0]; uz_jm = Z0[0]; const T uz_ip = Z1[1], uz_im = Z1[-1];
      const T uz_kp = Z1[SX], uz_km = Z1[-SX], uz_im_kp = Z1[SX - 1], uz_jm_kp = Z0[SX];
      const T p_c = P1[0], p_im = P1[-1], p_jm = P0[0], p_km = P1[-SX];

      const T IY1 = tr[MT_IY1], IY2 = one - IY1;
      const T IY3 = tr[MT_IY3], IY4 = one - IY3;
      {  // RhsX (clcRhsX_PIMP, m_TSchemePIMP_inc.f90:7-75)
        const T qdx1 = quarter * rdx, qdx3 = quarter * rdz;
        const T sucaj = half * tr[MT_RDYP];
        T h11 = ((ux_ip + ux_c) * (ux_ip + ux_c) - (ux_c + ux_im) * (ux_c + ux_im)) * qdx1;
        T h12 = ((uy_jp + uy_im_jp) * (IY3 * ux_c + IY4 * ux_jp) - (uy_c + uy_im) * (IY1 * ux_jm + IY2 * ux_c)) * sucaj;
        T h13 = ((uz_kp + uz_im_kp) * (ux_kp + ux_c) - (uz_c + uz_im) * (ux_c + ux_km)) * qdx3;
        T d11q1 = (ux_ip - two * ux_c + ux_im) * rdx2;
        T d22q1 = tr[MT_AP2C] * ux_jp + tr[MT_AC2C] * ux_c + tr[MT_AM2C] * ux_jm;
        T d33q1 = g.ap3c * ux_kp + g.ac3c * ux_c + g.am3c * ux_km;
        T dcq13 = d11q1 + d33q1;
        T gradp1 = (p_c - p_im) * rdx;
        T convEd1 = -h11 - h12 - h13 + xnu * dcq13 + g.g1;
        rx = pmGamma * convEd1 + pmTheta * hxo - pmAlpha * gradp1 + two * pmBeta * d22q1;
        hx[idx] = convEd1;
      }
      {  // RhsY (clcRhsY_PIMP, :161-209)
        const T hdx1 = half * rdx, hdx3 = half * rdz;
        const T sucac = tr[MT_RDYC], qsucac = quarter * sucac;
        T h21 = ((IY1 * ux_ip_jm + IY2 * ux_ip) * (uy_ip + uy_c) - (IY1 * ux_jm + IY2 * ux_c) * (uy_c + uy_im)) * hdx1;
        T h22 = ((uy_jp + uy_c) * (uy_jp + uy_c) - (uy_c + uy_jm) * (uy_c + uy_jm)) * qsucac;
        T h23 = ((IY1 * uz_jm_kp + IY2 * uz_kp) * (uy_kp + uy_c) - (IY1 * uz_jm + IY2 * uz_c) * (uy_c + uy_km)) * hdx3;
        T d11q2 = g.ap1c * uy_ip + g.ac1c * uy_c + g.am1c * uy_im;
        T d22q2 = tr[MT_AP2P] * uy_jp + tr[MT_AC2P] * uy_c + tr[MT_AM2P] * uy_jm;
        T d33q2 = g.ap3c * uy_kp + g.ac3c * uy_c + g.am3c * uy_km;
        T dcq13 = d11q2 + d33q2;
        T gradp2 = (p_c - p_jm) * sucac;
        T convEd2 = -h21 - h22 - h23 + xnu * dcq13 + g.g2;
        ry = pmGamma * convEd2 + pmTheta * hyo - pmAlpha * gradp2 + two * pmBeta * d22q2;
        hy[idx] = convEd2;
      }
      {  // RhsZ (clcRhsZ_PIMP, :277-325)
        const T qdx1 = quarter * rdx, qdx3 = quarter * rdz;
        const T sucaj = half * tr[MT_RDYP];
        T h31 = ((ux_ip + ux_ip_km) * (uz_ip + uz_c) - (ux_c + ux_km) * (uz_c + uz_im)) * qdx1;
        T h32 = ((uy_jp + uy_jp_km) * (IY3 * uz_c + IY4 * uz_jp) - (uy_c + uy_km) * (IY1 * uz_jm + IY2 * uz_c)) * sucaj;
        T h33 = ((uz_kp + uz_c) * (uz_kp + uz_c) - (uz_c + uz_km) * (uz_c + uz_km)) * qdx3;
        T d11q3 = g.ap1c * uz_ip + g.ac1c * uz_c + g.am1c * uz_im;
        T d22q3 = tr[MT_AP2C] * uz_jp + tr[MT_AC2C] * uz_c + tr[MT_AM2C] * uz_jm;
        T d33q3 = (uz_kp - two * uz_c + uz_km) * rdz2;
        T dcq13 = d11q3 + d33q3;
        T gradp3 = (p_c - p_km) * rdz;
        T convEd3 = -h31 - h32 - h33 + xnu * dcq13 + g.g3;
        rz = pmGamma * convEd3 + pmTheta * hzo - pmAlpha * gradp3 + two * pmBeta * d22q3;
        hz[idx] = convEd3;
      }
      } else {
        // 4th order: row r, x offset dx, z offset dz of staged array a
        auto V = [&](int a, int r, int dx, int dz) -> T { return ring[a][slot(r)][c0 + dx + dz * SX]; };
        const C4<T> q(g);
        // interpolated velocities (k_interp4 pattern): x for ux (i'-1..i'+2), uy, uz (i'-2..i'+1);
        // z for ux, uy (k'-2..k'+1), uz (k'-1..k'+2)
        auto uxhx = [&](int r, int o, int dz) {
          return q.in1 * V(0, r, o - 1, dz) + q.in2 * V(0, r, o, dz) + q.in3 * V(0, r, o + 1, dz) + q.in4 * V(0, r, o + 2, dz);
        };
        auto hxa = [&](int a, int r, int o, int dz) {
          return q.in1 * V(a, r, o - 2, dz) + q.in2 * V(a, r, o - 1, dz) + q.in3 * V(a, r, o, dz) + q.in4 * V(a, r, o + 1, dz);
        };
        auto hza = [&](int a, int r, int dx, int o) {
          return q.in1 * V(a, r, dx, o - 2) + q.in2 * V(a, r, dx, o - 1) + q.in3 * V(a, r, dx, o) + q.in4 * V(a, r, dx, o + 1);
        };
        auto uzhz = [&](int r, int o) {
          return q.in1 * V(2, r, 0, o - 1) + q.in2 * V(2, r, 0, o) + q.in3 * V(2, r, 0, o + 1) + q.in4 * V(2, r, 0, o + 2);
        };
        const bool top = j + 1 == ny;  // uyhx, uyhz vanish on the jc = nyp row (:223-226)
        const T IY1 = tr[MT_IY1], IY2 = one - IY1;
        const T IY3 = tr[MT_IY3], IY4 = one - IY3;
        const T sucaj = tr[MT_RDYP];
        ux_c = V(0, j, 0, 0); ux_jp = V(0, j + 1, 0, 0); ux_jm = V(0, j - 1, 0, 0);
        uy_c = V(1, j, 0, 0); uy_jp = V(1, j + 1, 0, 0); uy_jm = V(1, j - 1, 0, 0);
        uz_c = V(2, j, 0, 0); uz_jp = V(2, j + 1, 0, 0); uz_jm = V(2, j - 1, 0, 0);
        {  // RhsX (:235-268)
          const T uxhyc = IY1 * ux_jm + IY2 * ux_c;
          const T uxhyp = IY3 * ux_c + IY4 * ux_jp;
          const T a1 = uxhx(j, -2, 0), a2 = uxhx(j, -1, 0), a3 = uxhx(j, 0, 0), a4 = uxhx(j, 1, 0);
          const T h11 = q.dx1 * a1 * a1 + q.dx2 * a2 * a2 + q.dx3 * a3 * a3 + q.dx4 * a4 * a4;
          const T h12 = ((top ? (T)0 : hxa(1, j + 1, 0, 0)) * uxhyp - hxa(1, j, 0, 0) * uxhyc) * sucaj;
          const T h13 = q.dz1 * hza(0, j, 0, -1) * hxa(2, j, 0, -1) + q.dz2 * hza(0, j, 0, 0) * hxa(2, j, 0, 0) +
                        q.dz3 * hza(0, j, 0, 1) * hxa(2, j, 0, 1) + q.dz4 * hza(0, j, 0, 2) * hxa(2, j, 0, 2);
          const T d11 = q.dxx1 * V(0, j, -2, 0) + q.dxx2 * V(0, j, -1, 0) + q.dxx3 * ux_c + q.dxx4 * V(0, j, 1, 0) +
                        q.dxx5 * V(0, j, 2, 0);
          const T d22 = tr[MT_AP2C] * ux_jp + tr[MT_AC2C] * ux_c + tr[MT_AM2C] * ux_jm;
          const T d33 = q.dzz1 * V(0, j, 0, -2) + q.dzz2 * V(0, j, 0, -1) + q.dzz3 * ux_c + q.dzz4 * V(0, j, 0, 1) +
                        q.dzz5 * V(0, j, 0, 2);
          const T conv = -h11 - h12 - h13 + xnu * (d11 + d33) + g.g1;
          const T gradp = q.dx1 * V(3, j, -2, 0) + q.dx2 * V(3, j, -1, 0) + q.dx3 * V(3, j, 0, 0) + q.dx4 * V(3, j, 1, 0);
          rx = pmGamma * conv + pmTheta * hxo - pmAlpha * gradp + two * pmBeta * d22;
          hx[idx] = conv;
        }
        {  // RhsY (:270-305)
          const T sucac = tr[MT_RDYC], qsucac = quarter * sucac;
          const T uxhym = IY1 * V(0, j - 1, -1, 0) + IY2 * V(0, j, -1, 0);
          const T uxhyc = IY1 * V(0, j - 1, 0, 0) + IY2 * V(0, j, 0, 0);
          const T uxhyp = IY1 * V(0, j - 1, 1, 0) + IY2 * V(0, j, 1, 0);
          const T uxhyu = IY1 * V(0, j - 1, 2, 0) + IY2 * V(0, j, 2, 0);
          const T uzhym = IY1 * V(2, j - 1, 0, -1) + IY2 * V(2, j, 0, -1);
          const T uzhyc = IY1 * V(2, j - 1, 0, 0) + IY2 * V(2, j, 0, 0);
          const T uzhyp = IY1 * V(2, j - 1, 0, 1) + IY2 * V(2, j, 0, 1);
          const T uzhyu = IY1 * V(2, j - 1, 0, 2) + IY2 * V(2, j, 0, 2);
          const T h21 = q.dx1 * hxa(1, j, -1, 0) * uxhym + q.dx2 * hxa(1, j, 0, 0) * uxhyc +
                        q.dx3 * hxa(1, j, 1, 0) * uxhyp + q.dx4 * hxa(1, j, 2, 0) * uxhyu;
          const T h22 = ((uy_jp + uy_c) * (uy_jp + uy_c) - (uy_c + uy_jm) * (uy_c + uy_jm)) * qsucac;
          const T h23 = q.dz1 * hza(1, j, 0, -1) * uzhym + q.dz2 * hza(1, j, 0, 0) * uzhyc +
                        q.dz3 * hza(1, j, 0, 1) * uzhyp + q.dz4 * hza(1, j, 0, 2) * uzhyu;
          const T d11 = q.dxx1 * V(1, j, -2, 0) + q.dxx2 * V(1, j, -1, 0) + q.dxx3 * uy_c + q.dxx4 * V(1, j, 1, 0) +
                        q.dxx5 * V(1, j, 2, 0);
          const T d22 = tr[MT_AP2P] * uy_jp + tr[MT_AC2P] * uy_c + tr[MT_AM2P] * uy_jm;
          const T d33 = q.dzz1 * V(1, j, 0, -2) + q.dzz2 * V(1, j, 0, -1) + q.dzz3 * uy_c + q.dzz4 * V(1, j, 0, 1) +
                        q.dzz5 * V(1, j, 0, 2);
          const T conv = -h21 - h22 - h23 + xnu * (d11 + d33) + g.g2;
          const T gradp = (V(3, j, 0, 0) - V(3, j - 1, 0, 0)) * sucac;
          ry = pmGamma * conv + pmTheta * hyo - pmAlpha * gradp + two * pmBeta * d22;
          hy[idx] = conv;
        }
        {  // RhsZ (:307-343)
          const T uzhyc = IY1 * uz_jm + IY2 * uz_c;
          const T uzhyp = IY3 * uz_c + IY4 * uz_jp;
          const T h31 = q.dx1 * hxa(2, j, -1, 0) * hza(0, j, -1, 0) + q.dx2 * hxa(2, j, 0, 0) * hza(0, j, 0, 0) +
                        q.dx3 * hxa(2, j, 1, 0) * hza(0, j, 1, 0) + q.dx4 * hxa(2, j, 2, 0) * hza(0, j, 2, 0);
          const T h32 = ((top ? (T)0 : hza(1, j + 1, 0, 0)) * uzhyp - hza(1, j, 0, 0) * uzhyc) * sucaj;
          const T b1 = uzhz(j, -2), b2 = uzhz(j, -1), b3 = uzhz(j, 0), b4 = uzhz(j, 1);
          const T h33 = q.dz1 * b1 * b1 + q.dz2 * b2 * b2 + q.dz3 * b3 * b3 + q.dz4 * b4 * b4;
          const T d11 = q.dxx1 * V(2, j, -2, 0) + q.dxx2 * V(2, j, -1, 0) + q.dxx3 * uz_c + q.dxx4 * V(2, j, 1, 0) +
                        q.dxx5 * V(2, j, 2, 0);
          const T d22 = tr[MT_AP2C] * uz_jp + tr[MT_AC2C] * uz_c + tr[MT_AM2C] * uz_jm;
          const T d33 = q.dzz1 * V(2, j, 0, -2) + q.dzz2 * V(2, j, 0, -1) + q.dzz3 * uz_c + q.dzz4 * V(2, j, 0, 1) +
                        q.dzz5 * V(2, j, 0, 2);
          const T conv = -h31 - h32 - h33 + xnu * (d11 + d33) + g.g3;
          const T gradp = q.dz1 * V(3, j, 0, -2) + q.dz2 * V(3, j, 0, -1) + q.dz3 * V(3, j, 0, 0) + q.dz4 * V(3, j, 0, 1);
          rz = pmGamma * conv + pmTheta * hzo - pmAlpha * gradp + two * pmBeta * d22;
          hz[idx] = conv;
        }
      }
      rx += dpm;                     // mean pressure gradient (clcRhsX_PIMP :61-74)
      if (j == 0) ry = (T)0;         // duy_ym: uy_ym is constant (Update_uy_ym_CH)
      if (!TW || hf == 0) {  // upward elimination; g = u + d + cp u_{j+1}
        d0 = (rx - tr[MT_A0] * d0) * tr[MT_RM0];
        d1 = (ry - tr[MT_A1] * d1) * tr[MT_RM1];
        d2 = (rz - tr[MT_A0] * d2) * tr[MT_RM0];
        g0 = ux_c + d0 + tr[MT_CP0] * ux_jp;
        g1 = uy_c + d1 + tr[MT_CP1] * uy_jp;
        g2 = uz_c + d2 + tr[MT_CP0] * uz_jp;
      } else {               // downward elimination; g = u + e + aq u_{j-1}
        const T* td = dtab + (size_t)j * MD_W;
        d0 = (rx - __ldg(td + MD_C0) * d0) * __ldg(td + MD_RQ0);
        d1 = (ry - __ldg(td + MD_C1) * d1) * __ldg(td + MD_RQ1);
        d2 = (rz - __ldg(td + MD_C0) * d2) * __ldg(td + MD_RQ0);
        g0 = ux_c + d0 + __ldg(td + MD_AQ0) * ux_jm;
        g1 = uy_c + d1 + __ldg(td + MD_AQ1) * uy_jm;
        g2 = uz_c + d2 + __ldg(td + MD_AQ0) * uz_jm;
      }
      uxs[idx] = g0; uys[idx] = g1; uzs[idx] = g2;
      lu0 = ux_c; lu1 = uy_c; lu2 = uz_c;
    }
    if (bsub) {  // u*_rb = g_rb - cp_rb u*_{rb+1}
      const T* tb = tab + (size_t)rb * MT_W;
      const T cb0 = __ldg(tb + MT_CP0), cb1 = __ldg(tb + MT_CP1);
      p0 = b0 - cb0 * p0; p1 = b1 - cb1 * p1; p2 = b2 - cb0 * p2;
      uxs[ob] = p0; uys[ob] = p1; uzs[ob] = p2;
    }
    idx += hstep;
    hxo = hx1; hyo = hy1; hzo = hz1;
    hx1 = hxn; hy1 = hyn; hz1 = hzn;
  }
  cp_async_wait<0>();
  __syncthreads();  // the ring is refilled by the next tile's prologue (or reused below)
  if constexpr (TW) {
    // meeting of the groups at rows m-1 (lower: x = d - cp x_m) and m (upper: x = e - aq x_{m-1})
    T* xch = reinterpret_cast<T*>(smem_raw);  // [2][NT][6]
    if (act) {
      T* o = xch + ((size_t)hf * NT + tid) * 6;
      o[0] = d0; o[1] = d1; o[2] = d2; o[3] = lu0; o[4] = lu1; o[5] = lu2;
    }
    __syncthreads();
    if (!act) return;
    const T* lo = xch + (size_t)tid * 6;
    const T* up = xch + ((size_t)NT + tid) * 6;
    const T* tl = tab + (size_t)(mh - 1) * MT_W;
    const T* tu = dtab + (size_t)mh * MD_W;
    T xl[3], xu[3];
    const T cpl[3] = {__ldg(tl + MT_CP0), __ldg(tl + MT_CP1), __ldg(tl + MT_CP0)};
    const T aqu[3] = {__ldg(tu + MD_AQ0), __ldg(tu + MD_AQ1), __ldg(tu + MD_AQ0)};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      xl[q] = (lo[q] - cpl[q] * up[q]) / ((T)1 - cpl[q] * aqu[q]);
      xu[q] = up[q] - aqu[q] * xl[q];
    }
    // this group's boundary row, then outwards: u*_j = g_j - f_j u*_{j -+ 1}
    const int jb = hf ? mh : mh - 1;
    const T* uu = hf ? up : lo;
    const T* xx = hf ? xu : xl;
    long long o = i + plane * k + (long long)jb * nx;
    T c0v = uu[3] + xx[0], c1v = uu[4] + xx[1], c2v = uu[5] + xx[2];
    uxs[o] = c0v; uys[o] = c1v; uzs[o] = c2v;
    const T* ft = hf ? dtab : tab;  // substitution factors: aq (upper group) or cp (lower)
    const int fw = hf ? MD_W : MT_W, fo0 = hf ? MD_AQ0 : MT_CP0, fo1 = hf ? MD_AQ1 : MT_CP1;
    const int nout = hf ? ny - 1 - jb : jb;  // rows still to substitute
    constexpr int B = 8;
    for (int r0 = 0; r0 < nout; r0 += B) {
      T a0[B], a1[B], a2[B];
#pragma unroll
      for (int b = 0; b < B; ++b) {
        if (r0 + b < nout) {
          const long long ob = o - (long long)dj * (r0 + b + 1) * nx;
          a0[b] = uxs[ob]; a1[b] = uys[ob]; a2[b] = uzs[ob];
        }
      }
#pragma unroll
      for (int b = 0; b < B; ++b) {
        if (r0 + b < nout) {
          const int jr = jb - dj * (r0 + b + 1);
          const T* tb = ft + (size_t)jr * fw;
          const T f0 = __ldg(tb + fo0), f1 = __ldg(tb + fo1);
          c0v = a0[b] - f0 * c0v; c1v = a1[b] - f1 * c1v; c2v = a2[b] - f0 * c2v;
          const long long ob = o - (long long)dj * (r0 + b + 1) * nx;
          uxs[ob] = c0v; uys[ob] = c1v; uzs[ob] = c2v;
        }
      }
    }
    return;
  }
  pact = BS && act; pidx = idx - nx; p0 = g0; p1 = g1; p2 = g2;
  }  // tiles
  if (!pact) return;

  // back substitution of the block's last tile, rows loaded in batches of 8
  constexpr int B = 8;
  long long idx = pidx;  // row ny-1 (u* = g there)
  T g0 = p0, g1 = p1, g2 = p2;
  for (int j = ny - 2; j >= 0; j -= B) {
    T a0[B], a1[B], a2[B];
#pragma unroll
    for (int b = 0; b < B; ++b) {
      if (j - b >= 0) {
        const long long o = idx - (long long)(b + 1) * nx;
        a0[b] = uxs[o]; a1[b] = uys[o]; a2[b] = uzs[o];
      }
    }
#pragma unroll
    for (int b = 0; b < B; ++b) {
      if (j - b >= 0) {
        const T* tr = tab + (size_t)(j - b) * MT_W;
        const T cp0 = __ldg(tr + MT_CP0), cp1 = __ldg(tr + MT_CP1);
        g0 = a0[b] - cp0 * g0; g1 = a1[b] - cp1 * g1; g2 = a2[b] - cp0 * g2;
        const long long o = idx - (long long)(b + 1) * nx;
        uxs[o] = g0; uys[o] = g1; uzs[o] = g2;
      }
    }
    idx -= (long long)B * nx;
  }
}

// ---------------------------------------------------------------------------
// FluidVelUpdate (src/CFD_2nd/m_TScheme.f90:281-306) + PressureUpdate_PIMP
// (src/CFD_2nd/m_TSchemePIMP_inc.f90:852-873) as a march: a thread owns one
// (i, k) column over a chunk of MJ rows and keeps phi at j-1, j, j+1 in
// registers (Neumann ghosts of SetBC_and_UpdateHalo_pr at the walls).  The
// block's sum of ux * s1coe (the next substep's bulk constraint, clcRhsX_PIMP
// :60-74) goes to part[block].  mode 1: projection only (pmAlpha = 1, p kept).
// ---------------------------------------------------------------------------
constexpr int MJ = 32;  // rows per block of the march projection

__device__ __forceinline__ double block_sum128(double v, double* sh /* 4 */) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  return threadIdx.x == 0 ? (sh[0] + sh[1]) + (sh[2] + sh[3]) : 0.0;
}

// DIAG (last substep of a step, nx % 32 == 0, nz % 4 == 0 so that no thread
// idles): CheckDivergence, CalcVmax, the next step's CalcMaxCFL and the
// CalcUxAver partials (src/CFD_2nd/m_Tools.f90:21-104,250-270) of the new
// velocity, fused in.  The i+1, j+1 and k+1 neighbours of the new velocity
// are recomputed from u* and phi with the same expressions their own threads
// use, so they equal the stored values bit for bit.
template <class T, bool DIAG>
__global__ void __launch_bounds__(128) k_proj_march(Geo<T> g, Metrics<T> m, const T* uxs, const T* uys,
                                                    const T* uzs, T* ux, T* uy, T* uz, T* __restrict__ pr,
                                                    const T* __restrict__ phi, double* __restrict__ part,
                                                    double* __restrict__ part2, int mode, DevScalars* __restrict__ sc) {
  __shared__ double red[7][4];
  if (sc->status) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long long plane = (long long)nx * ny;
  const int i = blockIdx.x * 32 + (threadIdx.x & 31), k = blockIdx.y * 4 + (threadIdx.x >> 5);
  const int j0 = blockIdx.z * MJ, j1 = min(j0 + MJ, ny);
  double s = 0.0, s2 = 0.0, dv = 0.0, v0 = 0.0, v1 = 0.0, v2 = 0.0, cf = 0.0;
  if (i < nx && k < nz) {
    const long long col = i + plane * k;
    const long long dxm = i == 0 ? nx - 1 : -1;                           // offset to i-1
    const long long dzm = k == 0 ? (long long)(nz - 1) * plane : -plane;  // offset to k-1
    const long long dxp = i + 1 == nx ? 1 - nx : 1;                       // offset to i+1
    const long long dzp = k + 1 == nz ? -(long long)(nz - 1) * plane : plane;  // offset to k+1
    const T pmAlpha = mode == 0 ? (T)sc->pmAlpha : (T)1;
    const T pmBeta = (T)sc->pmBeta;
    const T rdxEta2 = g.rdx * pmAlpha, rdzEta2 = g.rdz * pmAlpha;
    const double rdx = g.rdx, rdz = g.rdz;
    T pm = __ldg(phi + col + (long long)(j0 > 0 ? j0 - 1 : 0) * nx);
    T pc = __ldg(phi + col + (long long)j0 * nx);
    // rows in batches of PB: all loads of a batch before its stores (u* and u may
    // be the same arrays, mode 1, so the compiler cannot reorder them itself)
    constexpr int PB = DIAG ? 2 : 4;
    for (int jb = j0; jb < j1; jb += PB) {
      T vpp[PB], vpx[PB], vpz[PB], vu[PB], vv[PB], vw[PB], vp[PB], mr[PB], mp[PB], mc[PB], mm[PB], ms[PB];
      T qux[PB], qpx[PB], quz[PB], qpz[PB], quy[PB], qr[PB], qrp[PB], qdy[PB];  // DIAG neighbours, metrics
#pragma unroll
      for (int b = 0; b < PB; ++b) {
        const int j = jb + b < j1 ? jb + b : j1 - 1;
        const long long idx = col + (long long)j * nx;
        const int jn = j + 1 < ny ? j + 1 : ny - 1;
        vpp[b] = __ldg(phi + col + (long long)jn * nx);
        vpx[b] = __ldg(phi + idx + dxm);
        vpz[b] = __ldg(phi + idx + dzm);
        vu[b] = uxs[idx]; vv[b] = uys[idx]; vw[b] = uzs[idx];
        vp[b] = mode == 0 ? pr[idx] : (T)0;
        mr[b] = m.rdyc[j + 1]; mp[b] = m.ap2Pr[j + 1]; mc[b] = m.ac2Pr[j + 1]; mm[b] = m.am2Pr[j + 1];
        ms[b] = m.s1coe[j + 1];
        if (DIAG) {
          qux[b] = uxs[idx + dxp]; qpx[b] = __ldg(phi + idx + dxp);
          quz[b] = uzs[idx + dzp]; qpz[b] = __ldg(phi + idx + dzp);
          quy[b] = uys[col + (long long)jn * nx];
          qr[b] = m.rdyc[jn + 1]; qrp[b] = m.rdyp[j + 1]; qdy[b] = m.dyp[j + 1];
        }
      }
#pragma unroll
      for (int b = 0; b < PB; ++b) {
        const int j = jb + b;
        if (j >= j1) break;
        const long long idx = col + (long long)j * nx;
        const T pp = vpp[b];
        const T sucacEta2 = mr[b] * pmAlpha;
        const T uxn = vu[b] - (pc - vpx[b]) * rdxEta2;
        const T uyn = vv[b] - (pc - pm) * sucacEta2;
        const T uzn = vw[b] - (pc - vpz[b]) * rdzEta2;
        ux[idx] = uxn; uy[idx] = uyn; uz[idx] = uzn;
        if (mode == 0) {
          const T pmBetap = -pmBeta * mp[b];
          const T pmBetac = -pmBeta * mc[b] + (T)1;
          const T pmBetam = -pmBeta * mm[b];
          pr[idx] = vp[b] + pmBetap * pp + pmBetac * pc + pmBetam * pm;
        }
        s += (double)uxn * (double)ms[b];
        if (DIAG) {
          // the new velocity at i+1, k+1 and j+1, as the threads that own them compute it
          const T uxp = qux[b] - (qpx[b] - pc) * rdxEta2;
          const T uzp = quz[b] - (qpz[b] - pc) * rdzEta2;
          const T uyp = j + 1 < ny ? quy[b] - (pp - pc) * (qr[b] * pmAlpha) : (T)g.bc.uy_hi;
          const double a = uxn, bb = uyn, c = uzn, aip = uxp, bjp = uyp, ckp = uzp, rdyp = qrp[b];
          double d = fabs((aip - a) * rdx + (bjp - bb) * rdyp + (ckp - c) * rdz);
          if (!(d == d)) d = INFINITY;  // NaN folded into +inf: a NaN field trips the limits
          dv = fmax(dv, d);
          v0 = fmax(v0, a == a ? fabs(a) : INFINITY);
          v1 = fmax(v1, bb == bb ? fabs(bb) : INFINITY);
          v2 = fmax(v2, c == c ? fabs(c) : INFINITY);
          cf = fmax(cf, fabs(a + aip) * rdx + fabs(bb + bjp) * rdyp + fabs(c + ckp) * rdz);
          s2 += a * (double)qdy[b];
        }
        pm = pc; pc = pp;
      }
    }
  }
  if constexpr (!DIAG) {
    const double bs = block_sum128(s, red[0]);
    if (threadIdx.x == 0) part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = bs;
  } else {
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    dv = fmax(dv, __shfl_xor_sync(0xffffffffu, dv, o));
    v0 = fmax(v0, __shfl_xor_sync(0xffffffffu, v0, o));
    v1 = fmax(v1, __shfl_xor_sync(0xffffffffu, v1, o));
    v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, o));
    cf = fmax(cf, __shfl_xor_sync(0xffffffffu, cf, o));
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][w] = s; red[1][w] = s2; red[2][w] = cf; red[3][w] = dv; red[4][w] = v0; red[5][w] = v1; red[6][w] = v2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double r[7];
    for (int q = 0; q < 2; ++q) r[q] = (red[q][0] + red[q][1]) + (red[q][2] + red[q][3]);
    for (int q = 2; q < 7; ++q) r[q] = fmax(fmax(red[q][0], red[q][1]), fmax(red[q][2], red[q][3]));
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    part[bid] = r[0];
    part2[bid] = r[1];
    atomic_max_nonneg(&sc->uddx, r[2] * 0.5);
    atomic_max_nonneg(&sc->divmax2, r[3]);
    atomic_max_nonneg(&sc->vmax[0], r[4]);
    atomic_max_nonneg(&sc->vmax[1], r[5]);
    atomic_max_nonneg(&sc->vmax[2], r[6]);
  }
  }
}

// the same partial sums of ux * s1coe for a freshly uploaded field
template <class T>
__global__ void __launch_bounds__(128) k_bulk_march(Geo<T> g, Metrics<T> m, const T* __restrict__ ux,
                                                    double* __restrict__ part) {
  __shared__ double red[4];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = blockIdx.x * 32 + (threadIdx.x & 31), k = blockIdx.y * 4 + (threadIdx.x >> 5);
  const int j0 = blockIdx.z * MJ, j1 = min(j0 + MJ, ny);
  double s = 0.0;
  if (i < nx && k < nz) {
    const long long col = i + (long long)nx * ny * k;
    for (int j = j0; j < j1; ++j) s += (double)ux[col + (long long)j * nx] * (double)m.s1coe[j + 1];
  }
  const double bs = block_sum128(s, red);
  if (threadIdx.x == 0) part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = bs;
}

// ---------------------------------------------------------------------------
// Marches that substitute the march's g themselves (BS = false above): one
// thread per (i, k) column, 32 x 4 columns per block, walking j downwards with
// u*_j = g_j - cp_j u*_{j+1} (cp of the substep's row table; u*_{ny-1} = g_{ny-1}
// since cp_{ny-1} = 0) for its own column and, where a stencil needs them, for
// the columns at i+1 (ux) and k+1 (uz), with the same expressions as the
// threads that own them.  All loads of a batch of PB rows are issued before its
// recurrence steps.
// ---------------------------------------------------------------------------

// clcPrSrcOther (src/CFD_2nd/m_TScheme.f90:213-241): div(u*) per cell into dv
// (scaled by 1/pmAlpha and transformed by the x kernel, mode 3), its maximum
// |div| into divmax1 (CheckDivergence before the projection).  PB rows of loads
// in flight: 8 (168 registers, three blocks per SM) where the grid runs many
// waves anyway, 4 (100 registers) where the column blocks fit in one wave at five.
template <class T, int PB>
__global__ void __launch_bounds__(128) k_div_bsub(Geo<T> g, Metrics<T> m, const T* __restrict__ tab,
                                                  const T* __restrict__ gx, const T* __restrict__ gy,
                                                  const T* __restrict__ gz, T* __restrict__ dv,
                                                  DevScalars* __restrict__ sc) {
  __shared__ double red[4];
  if (sc->status) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long long plane = (long long)nx * ny;
  tab += (size_t)(sc->ns - 1) * ny * MT_W;
  const int i = blockIdx.x * 32 + (threadIdx.x & 31), k = blockIdx.y * 4 + (threadIdx.x >> 5);
  double dmax = 0.0;
  if (i < nx && k < nz) {
    const long long col = i + plane * k;
    const long long dxp = i + 1 == nx ? 1 - nx : 1;                            // offset to i+1
    const long long dzp = k + 1 == nz ? -(long long)(nz - 1) * plane : plane;  // offset to k+1
    const T rdx = g.rdx, rdz = g.rdz;
    T ax = (T)0, axp = (T)0, ay = (T)0, az = (T)0, azp = (T)0;  // u* of row j+1
    T ayn = (T)g.bc.uy_hi;  // uy at j+1: the wall value above the top row
    // rows ny-1-b, ny-1-b-PB, ... pass through register slot b; a slot is refilled
    // with the row PB below as soon as it is consumed
    T vx[PB], vxp[PB], vy[PB], vz[PB], vzp[PB], c0[PB], c1[PB], sy[PB];
    auto load = [&](int b, int j) {
      const long long idx = col + (long long)j * nx;
      vx[b] = gx[idx]; vxp[b] = gx[idx + dxp]; vy[b] = gy[idx];
      vz[b] = gz[idx]; vzp[b] = gz[idx + dzp];
      c0[b] = __ldg(tab + (size_t)j * MT_W + MT_CP0);
      c1[b] = __ldg(tab + (size_t)j * MT_W + MT_CP1);
      sy[b] = m.rdyp[j + 1];
    };
#pragma unroll
    for (int b = 0; b < PB; ++b) load(b, ny - 1 - b >= 0 ? ny - 1 - b : 0);
    for (int jb = ny - 1; jb >= 0; jb -= PB) {
#pragma unroll
      for (int b = 0; b < PB; ++b) {
        const int j = jb - b;
        if (j < 0) break;
        ax = vx[b] - c0[b] * ax;
        axp = vxp[b] - c0[b] * axp;
        ay = vy[b] - c1[b] * ay;
        az = vz[b] - c0[b] * az;
        azp = vzp[b] - c0[b] * azp;
        const T r = (axp - ax) * rdx + (ayn - ay) * sy[b] + (azp - az) * rdz;
        if (j >= PB) load(b, j - PB);
        dv[col + (long long)j * nx] = r;
        dmax = fmax(dmax, fabs((double)r));
        ayn = ay;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dmax;
  __syncthreads();
  if (threadIdx.x == 0) atomic_max_nonneg(&sc->divmax1, fmax(fmax(red[0], red[1]), fmax(red[2], red[3])));
}

// FluidVelUpdate + PressureUpdate_PIMP (m_TScheme.f90:281-306, m_TSchemePIMP_inc.f90:
// 852-873) from g, as k_proj_march in mode 0; DIAG: the step diagnostics of the
// last substep (CheckDivergence, CalcVmax, CalcMaxCFL, CalcUxAver).  Partial sums
// go to the slots of the chunked projection grid (npz row chunks), the unused
// chunk slots of each block set to zero.
template <class T, bool DIAG>
__global__ void __launch_bounds__(128) k_proj_bsub(Geo<T> g, Metrics<T> m, const T* __restrict__ tab,
                                                   const T* __restrict__ gx, const T* __restrict__ gy,
                                                   const T* __restrict__ gz, T* __restrict__ ux, T* __restrict__ uy,
                                                   T* __restrict__ uz, T* __restrict__ pr, const T* __restrict__ phi,
                                                   double* __restrict__ part, double* __restrict__ part2, int npz,
                                                   DevScalars* __restrict__ sc) {
  __shared__ double red[7][4];
  if (sc->status) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long long plane = (long long)nx * ny;
  tab += (size_t)(sc->ns - 1) * ny * MT_W;
  const int i = blockIdx.x * 32 + (threadIdx.x & 31), k = blockIdx.y * 4 + (threadIdx.x >> 5);
  double s = 0.0, s2 = 0.0, dvm = 0.0, v0 = 0.0, v1 = 0.0, v2 = 0.0, cf = 0.0;
  if (i < nx && k < nz) {
    const long long col = i + plane * k;
    const long long dxm = i == 0 ? nx - 1 : -1;                                // offset to i-1
    const long long dzm = k == 0 ? (long long)(nz - 1) * plane : -plane;       // offset to k-1
    const long long dxp = i + 1 == nx ? 1 - nx : 1;                            // offset to i+1
    const long long dzp = k + 1 == nz ? -(long long)(nz - 1) * plane : plane;  // offset to k+1
    const T pmAlpha = (T)sc->pmAlpha, pmBeta = (T)sc->pmBeta;
    const T rdxEta2 = g.rdx * pmAlpha, rdzEta2 = g.rdz * pmAlpha;
    const double rdx = g.rdx, rdz = g.rdz;
    T ax = (T)0, ay = (T)0, az = (T)0, axp = (T)0, azp = (T)0;  // u* of row j+1
    T pc = __ldg(phi + col + (long long)(ny - 1) * nx);         // phi(j)
    T pp = pc;                                                   // phi(j+1), clamped at the top row
    T uyp = (T)g.bc.uy_hi;                                       // new uy at j+1 (DIAG)
    // rows pass through PB register slots, each refilled with the row PB below once consumed
    constexpr int PB = DIAG ? 2 : 4;
    T vx[PB], vy[PB], vz[PB], vp[PB], vpm[PB], vpx[PB], vpz[PB], c0[PB], c1[PB];
    T mr[PB], mp[PB], mc[PB], mm[PB], ms[PB];
    T qx[PB], qz[PB], qpx[PB], qpz[PB], qrp[PB], qdy[PB];  // DIAG neighbours, metrics
    auto load = [&](int b, int j) {
      const long long idx = col + (long long)j * nx;
      const int jm = j > 0 ? j - 1 : 0;
      vx[b] = gx[idx]; vy[b] = gy[idx]; vz[b] = gz[idx]; vp[b] = pr[idx];
      vpm[b] = __ldg(phi + col + (long long)jm * nx);
      vpx[b] = __ldg(phi + idx + dxm);
      vpz[b] = __ldg(phi + idx + dzm);
      c0[b] = __ldg(tab + (size_t)j * MT_W + MT_CP0);
      c1[b] = __ldg(tab + (size_t)j * MT_W + MT_CP1);
      mr[b] = m.rdyc[j + 1]; mp[b] = m.ap2Pr[j + 1]; mc[b] = m.ac2Pr[j + 1]; mm[b] = m.am2Pr[j + 1];
      ms[b] = m.s1coe[j + 1];
      if (DIAG) {
        qx[b] = gx[idx + dxp]; qpx[b] = __ldg(phi + idx + dxp);
        qz[b] = gz[idx + dzp]; qpz[b] = __ldg(phi + idx + dzp);
        qrp[b] = m.rdyp[j + 1]; qdy[b] = m.dyp[j + 1];
      }
    };
#pragma unroll
    for (int b = 0; b < PB; ++b) load(b, ny - 1 - b >= 0 ? ny - 1 - b : 0);
    for (int jb = ny - 1; jb >= 0; jb -= PB) {
#pragma unroll
      for (int b = 0; b < PB; ++b) {
        const int j = jb - b;
        if (j < 0) break;
        const long long idx = col + (long long)j * nx;
        ax = vx[b] - c0[b] * ax;
        ay = vy[b] - c1[b] * ay;
        az = vz[b] - c0[b] * az;
        const T pm = vpm[b];
        const T sucacEta2 = mr[b] * pmAlpha;
        const T uxn = ax - (pc - vpx[b]) * rdxEta2;
        const T uyn = ay - (pc - pm) * sucacEta2;
        const T uzn = az - (pc - vpz[b]) * rdzEta2;
        ux[idx] = uxn; uy[idx] = uyn; uz[idx] = uzn;
        const T pmBetap = -pmBeta * mp[b];
        const T pmBetac = -pmBeta * mc[b] + (T)1;
        const T pmBetam = -pmBeta * mm[b];
        pr[idx] = vp[b] + pmBetap * pp + pmBetac * pc + pmBetam * pm;
        s += (double)uxn * (double)ms[b];
        if (DIAG) {
          // the new velocity at i+1, k+1 and j+1, as the threads that own them compute it
          axp = qx[b] - c0[b] * axp;
          azp = qz[b] - c0[b] * azp;
          const T uxp = axp - (qpx[b] - pc) * rdxEta2;
          const T uzp = azp - (qpz[b] - pc) * rdzEta2;
          const double a = uxn, bb = uyn, c = uzn, aip = uxp, bjp = uyp, ckp = uzp, rdyp = qrp[b];
          double d = fabs((aip - a) * rdx + (bjp - bb) * rdyp + (ckp - c) * rdz);
          if (!(d == d)) d = INFINITY;  // NaN folded into +inf: a NaN field trips the limits
          dvm = fmax(dvm, d);
          v0 = fmax(v0, a == a ? fabs(a) : INFINITY);
          v1 = fmax(v1, bb == bb ? fabs(bb) : INFINITY);
          v2 = fmax(v2, c == c ? fabs(c) : INFINITY);
          cf = fmax(cf, fabs(a + aip) * rdx + fabs(bb + bjp) * rdyp + fabs(c + ckp) * rdz);
          s2 += a * (double)qdy[b];
          uyp = uyn;
        }
        pp = pc; pc = pm;
        if (j >= PB) load(b, j - PB);
      }
    }
  }
  const int bid = blockIdx.x + gridDim.x * blockIdx.y, nb = gridDim.x * gridDim.y;
  for (int z = 1 + threadIdx.x; z < npz; z += blockDim.x) {  // the chunk slots this grid leaves empty
    part[bid + (long long)nb * z] = 0.0;
    if (DIAG) part2[bid + (long long)nb * z] = 0.0;
  }
  if constexpr (!DIAG) {
    const double bs = block_sum128(s, red[0]);
    if (threadIdx.x == 0) part[bid] = bs;
  } else {
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
      dvm = fmax(dvm, __shfl_xor_sync(0xffffffffu, dvm, o));
      v0 = fmax(v0, __shfl_xor_sync(0xffffffffu, v0, o));
      v1 = fmax(v1, __shfl_xor_sync(0xffffffffu, v1, o));
      v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, o));
      cf = fmax(cf, __shfl_xor_sync(0xffffffffu, cf, o));
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
      red[0][w] = s; red[1][w] = s2; red[2][w] = cf; red[3][w] = dvm; red[4][w] = v0; red[5][w] = v1; red[6][w] = v2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double r[7];
      for (int q = 0; q < 2; ++q) r[q] = (red[q][0] + red[q][1]) + (red[q][2] + red[q][3]);
      for (int q = 2; q < 7; ++q) r[q] = fmax(fmax(red[q][0], red[q][1]), fmax(red[q][2], red[q][3]));
      part[bid] = r[0];
      part2[bid] = r[1];
      atomic_max_nonneg(&sc->uddx, r[2] * 0.5);
      atomic_max_nonneg(&sc->divmax2, r[3]);
      atomic_max_nonneg(&sc->vmax[0], r[4]);
      atomic_max_nonneg(&sc->vmax[1], r[5]);
      atomic_max_nonneg(&sc->vmax[2], r[6]);
    }
  }
}

static dim3 march_proj_grid(const ch3d_ctx* c) { return dim3((c->nx + 31) / 32, (c->nz + 3) / 4, (c->ny + MJ - 1) / MJ); }
int march_npart(const ch3d_ctx* c) {
  const dim3 g = march_proj_grid(c);
  return (int)(g.x * g.y * g.z);
}

bool march_diag_fusable(const ch3d_ctx* c) { return c->march && c->nx % 32 == 0 && c->nz % 4 == 0; }

template <class T> static cudaError_t proj_march_t(ch3d_ctx* c, int mode, bool diag) {
  T** f = (T**)c->f;
  T* in[3] = {mode == 1 ? f[0] : f[12], mode == 1 ? f[1] : f[13], mode == 1 ? f[2] : f[14]};
  if (diag)
    k_proj_march<T, true><<<march_proj_grid(c), 128, 0, c->stream>>>(make_geo<T>(c), metrics_of<T>(c), in[0], in[1],
                                                                      in[2], f[0], f[1], f[2], f[3], f[10], c->part,
                                                                      c->part2, mode, c->sc);
  else
    k_proj_march<T, false><<<march_proj_grid(c), 128, 0, c->stream>>>(make_geo<T>(c), metrics_of<T>(c), in[0], in[1],
                                                                       in[2], f[0], f[1], f[2], f[3], f[10], c->part,
                                                                       c->part2, mode, c->sc);
  return cudaGetLastError();
}
cudaError_t launch_proj_march(ch3d_ctx* c, int mode, bool diag) {
  return c->fp32 ? proj_march_t<float>(c, mode, diag) : proj_march_t<double>(c, mode, diag);
}
template <class T> static cudaError_t bulk_march_t(ch3d_ctx* c) {
  T** f = (T**)c->f;
  k_bulk_march<T><<<march_proj_grid(c), 128, 0, c->stream>>>(make_geo<T>(c), metrics_of<T>(c), f[0], c->part);
  return cudaGetLastError();
}
cudaError_t launch_bulk_march(ch3d_ctx* c) { return c->fp32 ? bulk_march_t<float>(c) : bulk_march_t<double>(c); }

template <class T> static cudaError_t div_bsub_t(ch3d_ctx* c) {
  T** f = (T**)c->f;
  const dim3 grid((c->nx + 31) / 32, (c->nz + 3) / 4);
  const int nsm = sm_count(c->device);
  // 256x192x256 (512 blocks): 74 us with 4 rows, 93 with 8; 768x384x576 (3456 blocks):
  // 0.84 ms with 8 rows against 0.88 with 4
  if ((long long)grid.x * grid.y > 6LL * nsm)
    k_div_bsub<T, 8><<<grid, 128, 0, c->stream>>>(make_geo<T>(c), metrics_of<T>(c), (const T*)c->mtab, f[12], f[13],
                                                   f[14], f[10], c->sc);
  else
    k_div_bsub<T, 4><<<grid, 128, 0, c->stream>>>(make_geo<T>(c), metrics_of<T>(c), (const T*)c->mtab, f[12], f[13],
                                                   f[14], f[10], c->sc);
  return cudaGetLastError();
}
cudaError_t launch_div_bsub(ch3d_ctx* c) { return c->fp32 ? div_bsub_t<float>(c) : div_bsub_t<double>(c); }

template <class T> static cudaError_t proj_bsub_t(ch3d_ctx* c, bool diag) {
  T** f = (T**)c->f;
  const dim3 grid((c->nx + 31) / 32, (c->nz + 3) / 4);
  const int npz = (int)march_proj_grid(c).z;
  if (diag)
    k_proj_bsub<T, true><<<grid, 128, 0, c->stream>>>(make_geo<T>(c), metrics_of<T>(c), (const T*)c->mtab, f[12],
                                                      f[13], f[14], f[0], f[1], f[2], f[3], f[10], c->part, c->part2,
                                                      npz, c->sc);
  else
    k_proj_bsub<T, false><<<grid, 128, 0, c->stream>>>(make_geo<T>(c), metrics_of<T>(c), (const T*)c->mtab, f[12],
                                                       f[13], f[14], f[0], f[1], f[2], f[3], f[10], c->part, c->part2,
                                                       npz, c->sc);
  return cudaGetLastError();
}
cudaError_t launch_proj_bsub(ch3d_ctx* c, bool diag) {
  return c->fp32 ? proj_bsub_t<float>(c, diag) : proj_bsub_t<double>(c, diag);
}

// The march runs twisted when all column tiles fit on the GPU at once as
// two-group blocks.
template <class T, bool O4> struct MarchShape {
  static constexpr int BZ = 4, D = sizeof(T) == 8 ? 2 : 4, RS = D + 4;
  // resident blocks per SM of the 2nd-order kernel (FP32: 6 when it stops at g, 5 otherwise)
  static constexpr int bps(bool stops_at_g) { return sizeof(T) == 8 ? 4 : (stops_at_g ? 6 : 5); }
  static constexpr int H = O4 ? 3 : 1, PL = march_pl(H, 1, BZ);
  static constexpr size_t smem = march_group_smem<T>(RS, PL);
  // FP32 march that stops at g, staged in 16-byte vectors
  static constexpr size_t smem_v4 = march_group_smem<T>(RS, march_pl(H, 4, BZ));
};
template <class T, bool O4> static bool march_twisted_t(const ch3d_ctx* c) {
  typedef MarchShape<T, O4> S;
  static PerDevice site;                  // per instance: the twisted kernel's limit and occupancy
  static int occ_dev[kMaxDevices] = {};   // twisted blocks per SM, written once per device under the set-up lock
  auto kern_tw = k_rhs_march<T, O4, true, true, 1, S::BZ, S::D, S::RS>;
  const cudaError_t e = once_per_device(site, c->device, [&] {
    cudaError_t r = cudaFuncSetAttribute(kern_tw, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(2 * S::smem));
    if (r != cudaSuccess) return r;
    int occ = 0;
    if ((r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern_tw, 64 * S::BZ, 2 * S::smem)) != cudaSuccess)
      return r;
    occ_dev[c->device] = occ;
    return cudaSuccess;
  });
  if (e != cudaSuccess) return false;  // the one-directional march has no such requirement
  const long long ntiles = (long long)((c->nx + 31) / 32) * ((c->nz + S::BZ - 1) / S::BZ);
  return c->ny >= 2 && ntiles <= (long long)sm_count(c->device) * occ_dev[c->device];
}
bool march_twisted(const ch3d_ctx* c) {
  if (c->cfg.order == 4) return c->fp32 ? march_twisted_t<float, true>(c) : march_twisted_t<double, true>(c);
  return c->fp32 ? march_twisted_t<float, false>(c) : march_twisted_t<double, false>(c);
}

template <class T, bool O4> static cudaError_t rhs_march_t(ch3d_ctx* c) {
  typedef MarchShape<T, O4> S;
  constexpr int BZ = S::BZ, D = S::D, RS = S::RS;
  const size_t smem = S::smem;
  T** f = (T**)c->f;
  k_march_table<T><<<1, 128, 0, c->stream>>>(helm_coef(c), metrics_of<T>(c), c->ny, (T*)c->mtab,
                                             march_down_tables<T>(c->mtab, c->ny),
                                             march_beta_slots(c->mtab, c->ny), c->sc);
  auto kern = k_rhs_march<T, O4, false, true, 1, BZ, D, RS>;
  auto kern_tw = k_rhs_march<T, O4, true, true, 1, BZ, D, RS>;
  const bool tw = march_twisted_t<T, O4>(c);  // also sets the twisted kernel's shared-memory limit
  static PerDevice site;  // per instance: the one-directional kernels' limits
  cudaError_t e = once_per_device(site, c->device, [&] {
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t r = cudaFuncSetAttribute(kern, a, (int)smem);
    if constexpr (!O4) {
      if (r == cudaSuccess) r = cudaFuncSetAttribute(k_rhs_march<T, O4, false, false, 1, BZ, D, RS>, a, (int)smem);
      if constexpr (sizeof(T) == 4)
        if (r == cudaSuccess)
          r = cudaFuncSetAttribute(k_rhs_march<T, O4, false, false, 4, BZ, D, RS>, a, (int)S::smem_v4);
    }
    return r;
  });
  if (e != cudaSuccess) return e;
  const int nsm = sm_count(c->device);
  const long long ntiles = (long long)((c->nx + 31) / 32) * ((c->nz + BZ - 1) / BZ);
  auto args = [&](auto k, unsigned grid, int threads, size_t sm) {
    k<<<grid, threads, sm, c->stream>>>(make_geo<T>(c), (const T*)c->mtab, march_down_tables<T>(c->mtab, c->ny), f[0],
                                        f[1], f[2], f[3], f[4], f[5], f[6], f[12], f[13], f[14], c->sc);
  };
  if (tw) {
    // few column tiles: all fit at once as two-group (twisted) blocks, half the march length
    args(kern_tw, (unsigned)ntiles, 64 * BZ, 2 * smem);
  } else {
    // 2nd order: persistent blocks (back substitution, if any, overlapped with the next
    // tile's march); 4th order: one tile per block
    const long long cap = !O4 ? (long long)nsm * S::bps(c->gsub) : ntiles;
    const unsigned grid = (unsigned)(ntiles < cap ? ntiles : cap);
    bool done = false;
    if constexpr (!O4) {
      if (c->gsub) {  // stops at g: the divergence and projection marches substitute
        bool v4 = false;
        if constexpr (sizeof(T) == 4) {
          if (c->nx % 4 == 0) {  // FP32 rows in 16-byte vectors
            args(k_rhs_march<T, O4, false, false, 4, BZ, D, RS>, grid, 32 * BZ, S::smem_v4);
            v4 = true;
          }
        }
        if (!v4) args(k_rhs_march<T, O4, false, false, 1, BZ, D, RS>, grid, 32 * BZ, smem);
        done = true;
      }
    }
    if (!done) args(kern, grid, 32 * BZ, smem);
  }
  return cudaGetLastError();
}
cudaError_t launch_rhs_march(ch3d_ctx* c) {
  if (c->cfg.order == 4) return c->fp32 ? rhs_march_t<float, true>(c) : rhs_march_t<double, true>(c);
  return c->fp32 ? rhs_march_t<float, false>(c) : rhs_march_t<double, false>(c);
}

}  // namespace ch3d
