// ch3d_spectra.cu -- spectra of the 4th-order statistics: clcStat's
// clcSpectra1D branch (src/CFD_4th/m_FlowCase.f90:642-880) and its 2-D
// spectra (clcSpectra2D, :881-935):
// per row jc and per direction 18 spectra: the energy spectra of ux, of uy
// at the faces transform_uy picks (:2303-2332), of uz and of p; the cospectra
// of the cell-centred ux and uy (UV) and of ux and the cell-centred uy (UV2);
// and for ux, uy, uz, p the linear coherence spectra R1, I1, R2 (clcLTS_x/z,
// :1271-1632: the cross spectrum with the same quantity at row jForLCS(1) or
// jForLCS(2), mirrored into the upper half of the channel).
//
// Each quantity is formed in phi's array and transformed along x (the
// real-to-complex transform of the Poisson solve): X(kx, j, z).  The x spectra
// are sums over z of X_A conj(X_B) (the reference's sums over its R2HC
// coefficients).  The z transform of X then gives the 2-D spectrum
// Y(kx, j, kz), and the z spectra, sums over x of the z-line spectra in the
// reference, follow from Parseval's theorem along x:
//   sum_x Z_A(x, kz) conj Z_B(x, kz) = (1/nx) sum over all kx of Y_A conj Y_B,
// where the half spectrum supplies kx > nx/2 as Y(nx - kx, kz) =
// conj Y(kx, nz - kz).  The 2-D spectra are the same products of Y (k_spec2d).
// Accumulation in FP64.
#include "ch3d_ctx.h"
#include "ch3d_dev.cuh"

namespace ch3d {

// the quantity `which` into out: 0 ux (+ uCRF = 0), 1 transform_uy(uy), 2 uz,
// 3 p, 4 cell-centred ux (4-point interpolation in x), 5 cell-centred uy
template <class T>
__global__ void __launch_bounds__(256) k_spec_field(Geo<T> g, const T* __restrict__ ux, const T* __restrict__ uy,
                                                    const T* __restrict__ uz, const T* __restrict__ pr, int which,
                                                    T* __restrict__ out) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= g.N) return;
  const int nx = g.nx, ny = g.ny;
  const int i = (int)(q % nx), j = (int)((q / nx) % ny), k = (int)(q / ((long long)nx * ny));
  T v;
  switch (which) {
    case 0: v = ux[q]; break;
    case 1: v = fld(uy, g, 1, i, j < ny / 2 ? j + 1 : j, k); break;  // uy(jc+1) in the lower half, uy(jc) above
    case 2: v = uz[q]; break;
    case 3: v = pr[q]; break;
    case 4: {
      const int im = i == 0 ? nx - 1 : i - 1, ip = i + 1 == nx ? 0 : i + 1, iu = ip + 1 == nx ? 0 : ip + 1;
      const long long row = q - i;
      v = (T)(-1.0 / 16.0) * ux[row + im] + (T)(9.0 / 16.0) * ux[q] + (T)(9.0 / 16.0) * ux[row + ip] +
          (T)(-1.0 / 16.0) * ux[row + iu];
      break;
    }
    default: v = (T)0.5 * (uy[q] + fld(uy, g, 1, i, j + 1, k)); break;
  }
  out[q] = v;
}

// x spectra: out[j * nxh + kx] += norm * w * sum_z part(A(kx, j, z) conj B(kx, jb, z)),
// part 0 the real, 1 the imaginary part; jb = j, or the coherence reference row of
// j for jref >= 0 (jref below the centre, ny-1-jref above); w = 2 for 0 < kx <
// nx/2 when doubled, else 1; the imaginary part is zero at kx = 0 and nx/2.
template <class CT>
__global__ void k_specx(const CT* __restrict__ A, const CT* __restrict__ B, int nx, int ny, int nz, int jref, int part,
                        int doubled, double norm, double* __restrict__ out) {
  const int nxh = nx / 2 + 1;
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (kx >= nxh) return;
  const int jb = jref < 0 ? j : (j < ny / 2 ? jref : ny - 1 - jref);
  const bool edge = kx == 0 || kx == nx / 2;
  double s = 0.0;
  if (!(part == 1 && edge)) {
    for (int z = 0; z < nz; ++z) {
      const CT a = A[kx + (size_t)nxh * (j + (size_t)ny * z)], b = B[kx + (size_t)nxh * (jb + (size_t)ny * z)];
      s += part == 0 ? (double)a.x * b.x + (double)a.y * b.y : (double)a.y * b.x - (double)a.x * b.y;
    }
  }
  out[(size_t)j * nxh + kx] += s * norm * (doubled && !edge ? 2.0 : 1.0);
}

// z spectra from the 2-D spectra Y_A, Y_B (kx, j, kz): one block per (kz, j),
// kz = 0..nz/2; out[j * nzh1 + kz] += norm * w / nx * part(sum over all kx).
template <class CT>
__global__ void __launch_bounds__(128) k_specz(const CT* __restrict__ A, const CT* __restrict__ B, int nx, int ny,
                                               int nz, int jref, int part, int doubled, double norm,
                                               double* __restrict__ out) {
  __shared__ double sh[4];
  const int nxh = nx / 2 + 1, nzh1 = nz / 2 + 1;
  const int kz = blockIdx.x, j = blockIdx.y;
  const int jb = jref < 0 ? j : (j < ny / 2 ? jref : ny - 1 - jref);
  const int kzm = kz == 0 ? 0 : nz - kz;
  const bool edge = kz == 0 || 2 * kz == nz;
  double s = 0.0;
  if (!(part == 1 && edge)) {
    for (int kx = threadIdx.x; kx < nxh; kx += blockDim.x) {
      const CT a = A[kx + (size_t)nxh * (j + (size_t)ny * kz)], b = B[kx + (size_t)nxh * (jb + (size_t)ny * kz)];
      double re = (double)a.x * b.x + (double)a.y * b.y, im = (double)a.y * b.x - (double)a.x * b.y;
      if (kx != 0 && 2 * kx != nx) {  // kx and nx - kx: the conjugate of the (kx, -kz) term
        const CT c = A[kx + (size_t)nxh * (j + (size_t)ny * kzm)], d = B[kx + (size_t)nxh * (jb + (size_t)ny * kzm)];
        re += (double)c.x * d.x + (double)c.y * d.y;
        im -= (double)c.y * d.x - (double)c.x * d.y;
      }
      s += part == 0 ? re : im;
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    const double t = sh[0] + sh[1] + sh[2] + sh[3];
    out[(size_t)j * nzh1 + kz] += t / (double)nx * norm * (doubled && !edge ? 2.0 : 1.0);
  }
}

// 2-D spectra (clcSpecAndLCSR2DFrom1D / clcCosSpectra2D, :1896-2298): the
// reference transforms the real and imaginary parts of the x spectrum along z
// separately (R2HC) and sums Re(R_A conj R_B) + Re(I_A conj I_B), which is
// Re(T(kx, kz) + T(kx, -kz)) / 2 of T = Y_A conj Y_B for 0 < kz < nz/2 and
// Re T(kx, kz) at kz = 0, nz/2.  Rows folded about the centre:
// out(kx, jc, kz) += norm (F(jc) + sgn F(ny-1-jc)), jc < ny/2, the layout
// EnergySpec2D(nxc/2+1, nyc/2, nzc/2+1).  jref >= 0: B is row jref (below the
// centre) or ny-1-jref (above) of the same spectrum.
template <class CT>
__global__ void k_spec2d(const CT* __restrict__ A, const CT* __restrict__ B, int nx, int ny, int nz, int jref, int sgn,
                         double norm, double* __restrict__ out) {
  const int nxh = nx / 2 + 1, nyh = ny / 2;
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, kz = blockIdx.y, jc = blockIdx.z;
  if (kx >= nxh) return;
  const int kzm = kz == 0 ? 0 : nz - kz;
  const bool edge = kz == 0 || 2 * kz == nz;
  auto F = [&](int j) {
    const int jb = jref < 0 ? j : (j < nyh ? jref : ny - 1 - jref);
    const CT a = A[kx + (size_t)nxh * (j + (size_t)ny * kz)], b = B[kx + (size_t)nxh * (jb + (size_t)ny * kz)];
    double re = (double)a.x * b.x + (double)a.y * b.y;
    if (edge) return re;
    const CT c = A[kx + (size_t)nxh * (j + (size_t)ny * kzm)], d = B[kx + (size_t)nxh * (jb + (size_t)ny * kzm)];
    return 0.5 * (re + (double)c.x * d.x + (double)c.y * d.y);
  };
  out[kx + (size_t)nxh * (jc + (size_t)nyh * kz)] += norm * (F(jc) + (double)sgn * F(ny - 1 - jc));
}

template <class T> static cudaError_t spectra_t(ch3d_ctx* c, int jf1, int jf2) {
  typedef typename CplxOf<T>::type CT;
  T** f = (T**)c->f;
  const int nx = c->nx, ny = c->ny, nz = c->nz, nxh = c->nxh, nzh1 = nz / 2 + 1;
  const double normX = 1.0 / ((double)nx * (double)nx * (double)nz), normZ = 1.0 / ((double)nx * (double)nz * (double)nz);
  double* SX = c->specacc;                          // [m][j][kx]
  double* SZ = c->specacc + (size_t)18 * ny * nxh;  // [m][j][kz]
  double* S2 = SZ + (size_t)18 * ny * nzh1;          // [m][kz][jc][kx], jc < ny/2
  const double norm2 = 0.5 / ((double)nx * (double)nz * (double)nx * (double)nz);
  const size_t sbytes = (size_t)c->NS * sizeof(CT);
  cudaError_t e;
  auto field = [&](int which) {
    k_spec_field<T><<<(unsigned)((c->N + 255) / 256), 256, 0, c->stream>>>(make_geo<T>(c), f[0], f[1], f[2], f[3], which,
                                                                          f[10]);
    cudaError_t r = cudaGetLastError();
    return r != cudaSuccess ? r : launch_prsrc_xfft(c, 4);  // X(kx, j, z) of phi's array into the spectrum
  };
  auto zfwd = [&](void* buf) {  // Y(kx, j, kz) of the spectrum in buf, in place
    void* keep = c->spec;
    c->spec = buf;
    cudaError_t r = launch_zfft_forward(c);
    c->spec = keep;
    return r;
  };
  auto sx = [&](const void* A, const void* B, int m, int jref, int part, int dbl) {
    k_specx<CT><<<dim3((nxh + 127) / 128, ny), 128, 0, c->stream>>>((const CT*)A, (const CT*)B, nx, ny, nz, jref, part,
                                                                    dbl, normX, SX + (size_t)m * ny * nxh);
    return cudaGetLastError();
  };
  auto sz = [&](const void* A, const void* B, int m, int jref, int part, int dbl) {
    k_specz<CT><<<dim3(nzh1, ny), 128, 0, c->stream>>>((const CT*)A, (const CT*)B, nx, ny, nz, jref, part, dbl, normZ,
                                                      SZ + (size_t)m * ny * nzh1);
    return cudaGetLastError();
  };
  auto s2 = [&](const void* A, const void* B, int m, int jref, int sgn) {
    k_spec2d<CT><<<dim3((nxh + 127) / 128, nzh1, ny / 2), 128, 0, c->stream>>>(
        (const CT*)A, (const CT*)B, nx, ny, nz, jref, sgn, norm2, S2 + (size_t)m * nxh * (ny / 2) * nzh1);
    return cudaGetLastError();
  };
  // energy spectrum m and the coherence spectra (n, n+1, n+2) of the spectrum in c->spec, in both directions
  auto energy_lcs = [&](int m, int n, bool x) {
    cudaError_t r;
    auto S = [&](const void* A, const void* B, int mm, int jref, int part, int dbl) {
      return x ? sx(A, B, mm, jref, part, dbl) : sz(A, B, mm, jref, part, dbl);
    };
    if ((r = S(c->spec, c->spec, m, -1, 0, 1)) != cudaSuccess) return r;
    if ((r = S(c->spec, c->spec, n, jf1, 0, 0)) != cudaSuccess) return r;
    if ((r = S(c->spec, c->spec, n + 1, jf1, 1, 0)) != cudaSuccess) return r;
    return S(c->spec, c->spec, n + 2, jf2, 0, 0);
  };
#define CK(x) if ((e = (x)) != cudaSuccess) return e
  // cell-centred uy, kept in the second buffer; UV from the cell-centred ux (x);
  // UU, its coherence spectra and UV2 from ux (x, then z); UV (z)
  CK(field(5));
  CK(cudaMemcpyAsync(c->spec2, c->spec, sbytes, cudaMemcpyDeviceToDevice, c->stream));
  CK(field(4));
  CK(sx(c->spec, c->spec2, 4, -1, 0, 1));
  CK(field(0));
  CK(energy_lcs(0, 6, true));
  CK(sx(c->spec, c->spec2, 5, -1, 0, 1));
  CK(zfwd(c->spec));
  CK(zfwd(c->spec2));
  CK(energy_lcs(0, 6, false));
  CK(s2(c->spec, c->spec, 0, -1, 1));
  CK(s2(c->spec, c->spec, 5, jf1, 1));
  CK(sz(c->spec, c->spec2, 5, -1, 0, 1));
  CK(field(4));
  CK(zfwd(c->spec));
  CK(sz(c->spec, c->spec2, 4, -1, 0, 1));
  CK(s2(c->spec, c->spec2, 4, -1, -1));  // UV: antisymmetric about the centre
  // VV, WW, PP
  const int which[3] = {1, 2, 3};
  for (int q = 0; q < 3; ++q) {
    CK(field(which[q]));
    CK(energy_lcs(1 + q, 9 + 3 * q, true));
    CK(zfwd(c->spec));
    CK(energy_lcs(1 + q, 9 + 3 * q, false));
    CK(s2(c->spec, c->spec, 1 + q, -1, 1));
    CK(s2(c->spec, c->spec, 6 + q, jf1, 1));
  }
#undef CK
  return cudaSuccess;
}

cudaError_t launch_spectra(ch3d_ctx* c, int jfor1, int jfor2) {
  // 0-based reference rows; the step's arrays f[10] (phi) and the spectrum are free between steps
  return c->fp32 ? spectra_t<float>(c, jfor1 - 1, jfor2 - 1) : spectra_t<double>(c, jfor1 - 1, jfor2 - 1);
}

}  // namespace ch3d
