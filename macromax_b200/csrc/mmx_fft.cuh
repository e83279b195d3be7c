// Shared-memory mixed-radix Stockham FFT over a tile of pencils.
//
// A tile holds C components x n samples x P pencils in shared memory, laid out [c][j][pencil] with a row pitch
// sP = P + 1 (odd, so that both the pencil-fastest and the sample-fastest access patterns are free of bank
// conflicts for 8- and 16-byte words).  One radix-r stage (self-sorting formulation):
//
//   T = n / r butterflies per pencil, L = product of the radices of the previous stages,
//   butterfly i:  k = i mod L,   inputs  x[i + q T]           (q = 0 .. r-1)
//                 u_q = x[i + q T] * w^(q k),   w = exp(-+2 pi i / (L r))
//                 u = DFT_r(u)
//                 outputs y[(i - k) r + k + q L] = u_q
//
// which needs no bit-reversal and leaves the result in natural order.  Each thread keeps its butterflies of a
// stage in registers (at most EPT complex values), so the stage runs in place: load + compute, barrier, store,
// barrier.  The launch must provide at least ceil(butterflies / (EPT / r)) threads for every stage.
#pragma once
#include "mmx_complex.cuh"

#define MMX_EPT 8
#define MMX_MAX_STAGES 12

struct FFTAxis {
  int n;                      // transform length
  int nst;                    // number of stages
  int radix[MMX_MAX_STAGES];  // radices, product == n
  const void* tw;             // twiddle table cpx<R>[n]: exp(-2 pi i t / n)
};

template <class R, int RAD, int DIR>
__device__ __noinline__ void fft_stage(cpx<R>* __restrict__ sm, int C, int n, int P, int sP, int L,
                                          const cpx<R>* __restrict__ tw) {
  constexpr int MAXB = (MMX_EPT / RAD) > 0 ? (MMX_EPT / RAD) : 1;
  const int T = n / RAD;
  const int nb = C * P * T;
  const int tstride = n / (L * RAD);
  const int nthr = blockDim.x;
  const int tid = threadIdx.x;
  cpx<R> u[MAXB][RAD];
  int dst[MAXB];
#pragma unroll
  for (int k = 0; k < MAXB; ++k) {
    const int b = tid + k * nthr;
    dst[k] = -1;
    if (b < nb) {
      const int pl = b % P;
      const int rest = b / P;
      const int i = rest % T;
      const int c = rest / T;
      const int kk = i % L;
      const int base = (c * n) * sP + pl;
#pragma unroll
      for (int q = 0; q < RAD; ++q) u[k][q] = sm[base + (i + q * T) * sP];
      if (L > 1) {
#pragma unroll
        for (int q = 1; q < RAD; ++q) {
          cpx<R> w = tw[q * kk * tstride];
          if (DIR > 0) w = conjc(w);
          u[k][q] = u[k][q] * w;
        }
      }
      bfly<R, RAD, DIR>(u[k], tw, n);
      dst[k] = base + ((i - kk) * RAD + kk) * sP;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < MAXB; ++k) {
    if (dst[k] >= 0) {
#pragma unroll
      for (int q = 0; q < RAD; ++q) sm[dst[k] + q * L * sP] = u[k][q];
    }
  }
  __syncthreads();
}

template <class R, int DIR>
__device__ __forceinline__ void fft_tile(cpx<R>* sm, int C, int P, int sP, const FFTAxis& ax) {
  const cpx<R>* tw = (const cpx<R>*)ax.tw;
  const int n = ax.n;
  int L = 1;
  for (int s = 0; s < ax.nst; ++s) {
    const int r = ax.radix[s];
    switch (r) {
#ifndef MMX_NO_R2
      case 2: fft_stage<R, 2, DIR>(sm, C, n, P, sP, L, tw); break;
#endif
#ifndef MMX_NO_R3
      case 3: fft_stage<R, 3, DIR>(sm, C, n, P, sP, L, tw); break;
#endif
#ifndef MMX_NO_R4
      case 4: fft_stage<R, 4, DIR>(sm, C, n, P, sP, L, tw); break;
#endif
#ifndef MMX_NO_R5
      case 5: fft_stage<R, 5, DIR>(sm, C, n, P, sP, L, tw); break;
#endif
#ifndef MMX_NO_R7
      case 7: fft_stage<R, 7, DIR>(sm, C, n, P, sP, L, tw); break;
#endif
#ifndef MMX_NO_R8
      case 8: fft_stage<R, 8, DIR>(sm, C, n, P, sP, L, tw); break;
#endif
#ifndef MMX_NO_R11
      case 11: fft_stage<R, 11, DIR>(sm, C, n, P, sP, L, tw); break;
#endif
#ifndef MMX_NO_R13
      case 13: fft_stage<R, 13, DIR>(sm, C, n, P, sP, L, tw); break;
#endif
#ifndef MMX_NO_R16
      case 16: fft_stage<R, 16, DIR>(sm, C, n, P, sP, L, tw); break;
#endif
      default: break;  // rejected at plan creation
    }
    L *= r;
  }
}

// threads needed by fft_tile for C*P pencils of the given radix plan (host side)
static inline int fft_tile_threads(int C, int P, const FFTAxis& ax) {
  int need = 1;
  for (int s = 0; s < ax.nst; ++s) {
    int r = ax.radix[s];
    int maxb = MMX_EPT / r;
    if (maxb < 1) maxb = 1;
    int nb = C * P * (ax.n / r);
    int t = (nb + maxb - 1) / maxb;
    if (t > need) need = t;
  }
  return need;
}
