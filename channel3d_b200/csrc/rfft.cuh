// rfft.cuh -- register-resident Stockham FFT for the Poisson transforms.
//
// A line of N complex points is owned by P threads; thread t holds the E =
// N / P points t + P m (m = 0..E-1) in registers.  In a Stockham pass of
// radix R (R | E) with stride NS, butterfly b = t + P q (q = 0..E/R-1) reads
// the points b + r N/R = t + P (q + r E/R): always the thread's own points.
// Its outputs go to (b - kk) R + kk + r NS (kk = b mod NS); while NS is not a
// multiple of P they belong to other threads and are exchanged through
// shared memory, once NS is a multiple of P they stay in the thread.  A plan
// therefore starts with radices whose product is P (one exchange after each)
// and ends with in-thread radices whose product is E.  The first pass reads
// the line straight from global memory and the result is left in the same
// t + P m order, so loads and stores are coalesced across the threads of a
// line.  Twiddles come from the W_N table of the generic transform (fft.cuh).
#pragma once
#include "fft.cuh"

namespace ch3d {

// multiply by the constant (c, s) = cos - i sin pattern of a twiddle
template <class CT, class RT> __device__ __forceinline__ CT cmulk(CT a, RT c, RT s) {
  return mk(a.x * c - a.y * s, a.x * s + a.y * c);
}

// forward radix-8: two radix-4 transforms of the even and odd points, W8 = exp(-i pi/4)
template <class CT> struct Bfly<CT, 8> {
  static __device__ __forceinline__ void run(CT* v) {
    typedef decltype(v[0].x) RT;
    const RT h = (RT)0.70710678118654752440084436210484903928;  // sqrt(1/2)
    CT e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    Bfly<CT, 4>::run(e);
    Bfly<CT, 4>::run(o);
    const CT o1 = mk(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));   // W8^1 o1
    const CT o2 = mk(o[2].y, -o[2].x);                                // W8^2 o2 = -i o2
    const CT o3 = mk(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));  // W8^3 o3
    v[0] = cadd(e[0], o[0]); v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);   v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);   v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);   v[7] = csub(e[3], o3);
  }
};

// forward radix-12 as 4 x 3: n = 3 n1 + n2, k = k1 + 4 k2; radix-4 over n1,
// twiddle W12^(n2 k1), radix-3 over n2
template <class CT> struct Bfly<CT, 12> {
  static __device__ __forceinline__ void run(CT* v) {
    typedef decltype(v[0].x) RT;
    const RT s3 = (RT)0.86602540378443864676372317075293618;  // sqrt(3)/2
    const RT hf = (RT)0.5;
    CT y[3][4];
#pragma unroll
    for (int n2 = 0; n2 < 3; ++n2) {
#pragma unroll
      for (int n1 = 0; n1 < 4; ++n1) y[n2][n1] = v[3 * n1 + n2];
      Bfly<CT, 4>::run(y[n2]);
    }
    // W12^1 = (s3, -1/2), W12^2 = (1/2, -s3), W12^3 = -i, W12^4 = (-1/2, -s3), W12^6 = -1
    y[1][1] = cmulk(y[1][1], s3, -hf);
    y[1][2] = cmulk(y[1][2], hf, -s3);
    y[1][3] = mk(y[1][3].y, -y[1][3].x);
    y[2][1] = cmulk(y[2][1], hf, -s3);
    y[2][2] = cmulk(y[2][2], -hf, -s3);
    y[2][3] = mk(-y[2][3].x, -y[2][3].y);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      CT w[3] = {y[0][k1], y[1][k1], y[2][k1]};
      Bfly<CT, 3>::run(w);
#pragma unroll
      for (int k2 = 0; k2 < 3; ++k2) v[k1 + 4 * k2] = w[k2];
    }
  }
};

struct WarpSync {
  __device__ __forceinline__ void operator()() const { __syncwarp(); }
};
struct BlockSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

// Position of point p in a line's exchange buffer: p * ss, or with PAD one
// 16-byte gap after every 8 points (p + p / 8), which spreads the stride-R
// writes of the first pass over all shared-memory banks.
template <bool PAD> __device__ __forceinline__ int xpos(int p, int ss) { return PAD ? p + (p >> 3) : p * ss; }

// One pass (radix R, stride NS) over the thread's E points; sm: the line's
// exchange buffer (point p at xpos<PAD>(p, ss)).
template <class CT, int N, int P, int E, int NS, int R, bool PAD, class Sync>
__device__ __forceinline__ void rs_pass(CT (&v)[E], CT* sm, int ss, int t, const CT* __restrict__ tw, Sync sync) {
  static_assert(E % R == 0, "radix must divide the points per thread");
  constexpr int Q = E / R;
  constexpr int STEP = N / (NS * R);
  constexpr bool EXCH = NS % P != 0;
  CT o[E];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int b = t + P * q;
    const int kk = b % NS;
    CT x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = v[q + r * Q];
    if (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) x[r] = cmul(x[r], __ldg(tw + r * kk * STEP));
    }
    Bfly<CT, R>::run(x);
    if (EXCH) {
      const int base = (b - kk) * R + kk;
#pragma unroll
      for (int r = 0; r < R; ++r) sm[xpos<PAD>(base + r * NS, ss)] = x[r];
    } else {
      constexpr int s = EXCH ? 1 : NS / P;
#pragma unroll
      for (int r = 0; r < R; ++r) o[(q - q % s) * R + q % s + r * s] = x[r];
    }
  }
  if (EXCH) {
    sync();
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = sm[xpos<PAD>(t + P * m, ss)];
    sync();
  } else {
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = o[m];
  }
}

template <class CT, int N, int P, int E, bool PAD, int NS, int... Rs> struct RRun;
template <class CT, int N, int P, int E, bool PAD, int NS> struct RRun<CT, N, P, E, PAD, NS> {
  template <class Sync> __device__ __forceinline__ static void run(CT (&)[E], CT*, int, int, const CT*, Sync) {
    static_assert(NS == N, "plan radices must multiply to N");
  }
};
template <class CT, int N, int P, int E, bool PAD, int NS, int R, int... Rs> struct RRun<CT, N, P, E, PAD, NS, R, Rs...> {
  template <class Sync>
  __device__ __forceinline__ static void run(CT (&v)[E], CT* sm, int ss, int t, const CT* __restrict__ tw, Sync sync) {
    rs_pass<CT, N, P, E, NS, R, PAD>(v, sm, ss, t, tw, sync);
    RRun<CT, N, P, E, PAD, NS * R, Rs...>::run(v, sm, ss, t, tw, sync);
  }
};

// A plan: N points, P threads per line, radices in pass order.  run<PAD>:
// PAD for a line-contiguous buffer of padded_len() points (ss unused),
// otherwise point p at sm[p * ss].
template <int N_, int P_, int... Rs> struct RPlan {
  static constexpr int N = N_, P = P_, E = N_ / P_;
  static constexpr int padded_len() { return N_ + N_ / 8; }
  template <bool PAD, class CT, class Sync>
  __device__ __forceinline__ static void run(CT (&v)[E], CT* sm, int ss, int t, const CT* __restrict__ tw, Sync sync) {
    RRun<CT, N, P, E, PAD, 1, Rs...>::run(v, sm, ss, t, tw, sync);
  }
};

}  // namespace ch3d
