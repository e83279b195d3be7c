// Register-staged FFT-only passes for mmx_fftn (BackEnd.ft / ift, backend/__init__.py:234-257), complex64, axis
// lengths 64, 128, 256 and 512, built from the stages of the iteration's own passes (mmx_reg.cuh): the first radix
// stage reads its butterfly inputs from global memory into registers and the last one writes its outputs straight
// back, so a pass exchanges data through shared memory only between stages (the runtime-radix k_fft_pass stages
// every element through shared memory and recomputes its pencil addresses per element).
//   k_fftr_strided: a strided axis, tiles of 16 consecutive pencils (inner a multiple of 16), 128-byte rows.
//   k_fftr_contig:  the contiguous axis, tiles of PC whole rows; `scale` multiplies the input (the inverse
//                   transform's 1 / N, applied once, in this pass).
// Either may run in place (in == out): every thread has read its tile's inputs before the tile's first store.
#pragma once
#include "mmx_reg.cuh"

template <int DIR, int N>
__global__ void __launch_bounds__(RegThreads<1, N>::value) k_fftr_strided(const float2* __restrict__ in,
                                                                           float2* __restrict__ out, int64_t inner,
                                                                           const float2* __restrict__ twg) {
  constexpr int P = kRegP, THREADS = RegThreads<1, N>::value;
  extern __shared__ __align__(16) unsigned char mmx_smem_raw[];
  float2* sm = reinterpret_cast<float2*>(mmx_smem_raw);
  float2* smtw = sm + N * P;
  for (int t = threadIdx.x; t < N; t += THREADS) smtw[t] = twg[t];
  __syncthreads();
  const int64_t p0 = (int64_t)blockIdx.x * P;
  const int64_t o = p0 / inner;
  const int64_t off = o * (int64_t)N * inner + (p0 - o * inner);
  rfft<DIR, N, 1, true, true>(sm, smtw, in + off, out + off, inner, 0, typename RegPlan<N>::type{});
}

template <int DIR, int N, int PC>
__global__ void __launch_bounds__(RegC<1, N, PC>::THREADS) k_fftr_contig(const float2* __restrict__ in,
                                                                          float2* __restrict__ out,
                                                                          const float2* __restrict__ twg,
                                                                          float scale) {
  using G = RegC<1, N, PC>;
  using PA = RegPlanArgs<typename RegPlan<N>::type>;
  constexpr int TPP = G::TPP, THREADS = G::THREADS;
  extern __shared__ __align__(16) unsigned char mmx_smem_raw[];
  float2* sm = reinterpret_cast<float2*>(mmx_smem_raw);
  float2* smtw = sm + PC * G::PITCH;
  for (int t = threadIdx.x; t < N; t += THREADS) smtw[t] = twg[t];
  __syncthreads();
  const int tid = threadIdx.x;
  const int ii = tid % TPP;
  const int row = tid / TPP;
  const int64_t rowbase = ((int64_t)blockIdx.x * PC + row) * N;
  const float2* __restrict__ src = in + rowbase;
  float2* __restrict__ dst = out + rowbase;
  {  // first stage (span 1, no twiddles) from global memory, one butterfly at a time
    constexpr int RAD = PA::R_first;
    constexpr int T = N / RAD;
    constexpr int NBT = T / TPP;
#pragma unroll 1
    for (int m = 0; m < NBT; ++m) {
      const int i = ii + m * TPP;
      float2 u[RAD];
#pragma unroll
      for (int q = 0; q < RAD; ++q) u[q] = src[i + q * T] * scale;
      bfly<float, RAD, DIR>(u, smtw, N);
#pragma unroll
      for (int q = 0; q < RAD; ++q) sm[G::idx(0, row, i * RAD + q)] = u[q];
    }
  }
  __syncthreads();
  PA::template mid<DIR, N, 1, PC>(sm, smtw);
  constexpr int RL = PA::R_last;
  constexpr int TL = N / RL;
  constexpr int NBL = TL / TPP;
#pragma unroll 1
  for (int m = 0; m < NBL; ++m) {  // last stage to global memory
    const int i = ii + m * TPP;
    float2 v[RL];
#pragma unroll
    for (int q = 0; q < RL; ++q) v[q] = sm[G::idx(0, row, i + q * TL)];
#pragma unroll
    for (int q = 1; q < RL; ++q) {
      float2 w = smtw[q * i];
      if (DIR > 0) w = conjc(w);
      v[q] = v[q] * w;
    }
    bfly<float, RL, DIR>(v, smtw, N);
#pragma unroll
    for (int q = 0; q < RL; ++q) dst[i + q * TL] = v[q];
  }
}
