// fft.cuh -- batched mixed-radix (2/3/4) Stockham FFT in shared memory.
//
// Replaces the FFTW r2r transforms of the Poisson solver
// (src/CFD_2nd/m_Poisson.f90:241-333, kinds R2HC/HC2R).  A block transforms
// several lines at once; each pass reads one shared buffer and writes the
// other (Stockham auto-sort), so the result is in natural order.  Element
// (line l, position n) of a buffer lives at l*ls + n*es.  Twiddles come from a
// table W_N^q = exp(-2 pi i q / N), q = 0..N-1, built on the host in long
// double.  Inverse transforms use conj(FFT(conj(x))) and are unnormalised like
// FFTW's HC2R.
#pragma once
#include "ch3d_common.cuh"

namespace ch3d {

#define CH3D_MAX_PASSES 16


// Exact integer division by a runtime constant d: q = (n * m) >> 40 with
// m = floor(2^40 / d) + 1, exact whenever n * d < 2^40 (here n < 2^24 and
// d < 2^16).
__host__ __device__ inline unsigned long long fdiv_magic(unsigned d) { return ((1ull << 40) / d) + 1ull; }
__device__ __forceinline__ int fdiv(int n, unsigned long long m) {
  return (int)(((unsigned long long)(unsigned)n * m) >> 40);
}

struct FFTPlanDev {
  int n;                          // complex length
  int npass;
  int radix[CH3D_MAX_PASSES];
  unsigned long long mNB[CH3D_MAX_PASSES];  // division by n / radix[p]
  unsigned long long mNs[CH3D_MAX_PASSES];  // division by radix[0] * ... * radix[p-1]
};

template <class CT, int R> struct Bfly;

template <class CT> struct Bfly<CT, 2> {
  static __device__ __forceinline__ void run(CT* v) {
    CT a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

// forward radix-4: multiply by -i where W4 appears
template <class CT> struct Bfly<CT, 4> {
  static __device__ __forceinline__ void run(CT* v) {
    CT t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    CT t2 = cadd(v[1], v[3]), t3 = csub(v[1], v[3]);
    CT mit3 = mk(t3.y, -t3.x);  // -i * t3
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, mit3);
    v[3] = csub(t1, mit3);
  }
};

// forward radix-3 with W3 = exp(-2 pi i / 3) = -1/2 - i sqrt(3)/2
template <class CT> struct Bfly<CT, 3> {
  static __device__ __forceinline__ void run(CT* v) {
    typedef decltype(v[0].x) RT;
    const RT s3 = (RT)0.86602540378443864676372317075293618;
    CT t1 = cadd(v[1], v[2]);
    CT t2 = csub(v[1], v[2]);
    CT m = mk(v[0].x - (RT)0.5 * t1.x, v[0].y - (RT)0.5 * t1.y);
    CT jt = mk(s3 * t2.y, -s3 * t2.x);  // -i*sqrt(3)/2 * t2
    v[0] = cadd(v[0], t1);
    v[1] = cadd(m, jt);
    v[2] = csub(m, jt);
  }
};

// One Stockham pass of radix R over `nlines` lines of length N, from
// buffer src to buffer dst.  LFAST selects the thread mapping: line index
// fastest (lines interleaved in memory) or butterfly index fastest (lines
// contiguous).
template <class CT, int R, bool LFAST>
__device__ __forceinline__ void fft_pass(const CT* __restrict__ src, CT* __restrict__ dst, int N, int Ns, int nlines,
                                         int ls, int es, const CT* __restrict__ tw, unsigned long long mNB,
                                         unsigned long long mNs, unsigned long long mL) {
  const int NB = N / R;
  const int total = nlines * NB;
  const int step = N / (Ns * R);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    int l, b;
    if (LFAST) { b = fdiv(t, mL); l = t - b * nlines; }
    else { l = fdiv(t, mNB); b = t - l * NB; }
    const int kk = b - fdiv(b, mNs) * Ns;
    CT v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[l * ls + (b + r * NB) * es];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], __ldg(tw + r * kk * step));
    }
    Bfly<CT, R>::run(v);
    const int idxD = (b - kk) * R + kk;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[l * ls + (idxD + r * Ns) * es] = v[r];
  }
}

// Full forward FFT of the lines in buffer a (b is scratch of the same size).
// Returns the buffer holding the result.  The caller synchronises before the
// call; the function ends with a __syncthreads().
template <class CT, bool LFAST>
__device__ CT* fft_lines(CT* a, CT* b, const FFTPlanDev& pl, int nlines, int ls, int es, const CT* __restrict__ tw) {
  int Ns = 1;
  const unsigned long long mL = fdiv_magic((unsigned)nlines);
  for (int p = 0; p < pl.npass; ++p) {
    const int R = pl.radix[p];
    if (R == 4) fft_pass<CT, 4, LFAST>(a, b, pl.n, Ns, nlines, ls, es, tw, pl.mNB[p], pl.mNs[p], mL);
    else if (R == 2) fft_pass<CT, 2, LFAST>(a, b, pl.n, Ns, nlines, ls, es, tw, pl.mNB[p], pl.mNs[p], mL);
    else fft_pass<CT, 3, LFAST>(a, b, pl.n, Ns, nlines, ls, es, tw, pl.mNB[p], pl.mNs[p], mL);
    __syncthreads();
    CT* t = a; a = b; b = t;
    Ns *= R;
  }
  return a;
}

}  // namespace ch3d
